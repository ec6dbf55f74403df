"""Point-vehicle game configuration of the legacy 6D square game
(src/pursuit_evasion/model.py:16-74): fixed speeds, bounded turn rates, a
square arena whose wall is a fault for whichever car reaches it first."""

from __future__ import annotations

from dataclasses import asdict, dataclass
import json
from pathlib import Path

import numpy as np


@dataclass(frozen=True)
class Vehicle:
    speed: float
    max_turn_rate: float

    def __post_init__(self):
        if (not np.isfinite([self.speed, self.max_turn_rate]).all() or self.speed <= 0
                or self.max_turn_rate <= 0):
            raise ValueError("Fixed speed and turn bound must be finite and positive.")

    @property
    def minimum_turn_radius(self) -> float:
        return self.speed / self.max_turn_rate


@dataclass(frozen=True)
class GameConfig:
    name: str = "square6d"
    arena_half_width: float = 3.0
    capture_radius: float = 0.3
    control_dt: float = 0.05
    pursuer: Vehicle = Vehicle(1.0, 1.0)
    evader: Vehicle = Vehicle(0.3, 2.0)
    boundary_rule: str = "first_fault_loses"
    point_vehicles: bool = True

    def __post_init__(self):
        scalars = [self.arena_half_width, self.capture_radius, self.control_dt]
        if not np.isfinite(scalars).all() or min(scalars) <= 0:
            raise ValueError("Map size, capture radius and command interval must be finite "
                             "and positive.")
        if self.boundary_rule != "first_fault_loses" or not self.point_vehicles:
            raise ValueError("This version implements point vehicles and first_fault_loses "
                             "only.")

    def to_dict(self) -> dict:
        return asdict(self)

    @classmethod
    def from_dict(cls, data: dict) -> "GameConfig":
        d = dict(data)
        for name in ("pursuer", "evader"):
            if name in d:
                d[name] = Vehicle(**d[name])
        return cls(**d)

    @classmethod
    def load(cls, path) -> "GameConfig":
        return cls.from_dict(json.loads(Path(path).read_text()))


def wrap_angle(angle):
    return (np.asarray(angle) + np.pi) % (2 * np.pi) - np.pi
