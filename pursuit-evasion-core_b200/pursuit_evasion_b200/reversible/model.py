"""Reversible-car physical model: the configuration objects of the game.

Mirrors the configuration contract of pursuit-evasion-core
src/pursuit_evasion/reversible/model.py:13-79 (VehicleLimits,
ReversibleConfig, JSON round trip) so that configuration files such as
configs/reversible_free_a3.json load unchanged.  Any object with the same
attributes (including the reference's own ReversibleConfig) is accepted by
the solvers of this package.

Relative state: [x, y, thetaE - thetaP, vP, vE].  Each command:
[acceleration (m/s^2), curvature (1/m)].
"""

from __future__ import annotations

from dataclasses import asdict, dataclass, field
import math


def _finite(*values):
    return all(math.isfinite(float(v)) for v in values)


@dataclass(frozen=True)
class VehicleLimits:
    speed_min: float
    speed_max: float
    acceleration: float
    max_curvature: float

    def __post_init__(self):
        if not _finite(
            self.speed_min, self.speed_max, self.acceleration, self.max_curvature
        ) or not self.speed_min < 0 < self.speed_max:
            raise ValueError("Signed finite speed bounds must straddle zero.")
        if self.acceleration <= 0 or self.max_curvature <= 0:
            raise ValueError("Acceleration and curvature bounds must be positive.")

    @property
    def max_abs_speed(self):
        return max(abs(self.speed_min), self.speed_max)

    def to_dict(self):
        return asdict(self)


@dataclass(frozen=True)
class ReversibleConfig:
    name: str = "reversible_cars"
    pursuer: VehicleLimits = field(
        default_factory=lambda: VehicleLimits(-1.0, 2.0, 2.0, 1.0)
    )
    evader: VehicleLimits = field(
        default_factory=lambda: VehicleLimits(-0.5, 1.0, 1.0, 2.0)
    )
    capture_radius: float = 0.3
    control_dt: float = 0.05
    arena_half_width: float = 3.0
    boundary_rule: str = "first_fault_loses"
    point_vehicles: bool = True
    capture_rule: str = "center_distance"

    def __post_init__(self):
        values = (self.capture_radius, self.control_dt, self.arena_half_width)
        if not _finite(*values) or min(values) <= 0:
            raise ValueError(
                "Radius, control interval and square extent must be positive."
            )
        if self.boundary_rule not in (
            "first_fault_loses",
            "collision_constrained",
        ) or not isinstance(self.point_vehicles, bool):
            raise ValueError(
                "Use a declared boundary rule and an explicit point/footprint flag."
            )
        if self.capture_rule not in ("center_distance", "rectangle_contact"):
            raise ValueError("Unknown capture rule")
        if self.point_vehicles and (
            self.capture_rule != "center_distance"
            or self.boundary_rule != "first_fault_loses"
        ):
            raise ValueError("Finite-body game rules require point_vehicles=False")

    def to_dict(self):
        return asdict(self)

    @classmethod
    def from_dict(cls, value):
        data = dict(value)
        for role in ("pursuer", "evader"):
            if role in data and not isinstance(data[role], VehicleLimits):
                data[role] = VehicleLimits(**data[role])
        return cls(**data)


def config_dict(config):
    """JSON-ready dictionary of any ReversibleConfig-like object."""
    if hasattr(config, "to_dict"):
        return config.to_dict()
    return asdict(config)
