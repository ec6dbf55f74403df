"""Grid of the 6D square game, [xP, yP, thetaP, xE, yE, thetaE]
(src/pursuit_evasion/dp/grid.py:9-100)."""

from __future__ import annotations

from dataclasses import asdict, dataclass

import numpy as np

from ..model import GameConfig


@dataclass(frozen=True)
class GridSpec:
    positions: int = 17
    headings: int = 16
    extent: float = 3.5

    def __post_init__(self):
        counts = (self.positions, self.headings)
        if (any(not isinstance(n, (int, np.integer)) or isinstance(n, bool) for n in counts)
                or self.positions < 5 or self.headings < 4):
            raise ValueError("Grid counts must be integers with at least five position "
                             "samples and four periodic headings.")
        if not np.isfinite(self.extent) or self.extent <= 0:
            raise ValueError("Grid extent must be finite and positive.")

    @property
    def shape(self):
        n, h = self.positions, self.headings
        return (n, n, h, n, n, h)

    @property
    def states(self):
        return self.positions ** 4 * self.headings ** 2

    @property
    def axes(self):
        x = np.linspace(-self.extent, self.extent, self.positions)
        theta = -np.pi + np.arange(self.headings) * 2 * np.pi / self.headings
        return (x, x, theta, x, x, theta)

    @property
    def spacings(self):
        d = 2 * self.extent / (self.positions - 1)
        h = 2 * np.pi / self.headings
        return (d, d, h, d, d, h)

    def to_dict(self):
        return dict(**asdict(self), shape=list(self.shape), states=self.states,
                    spacings=list(self.spacings), periodic_axes=[2, 5],
                    state_order=["xP", "yP", "thetaP", "xE", "yE", "thetaE"])


def target_and_avoid(grid: GridSpec, config: GameConfig, dtype=np.float32):
    """Target: capture or evader boundary fault; avoid: pursuer boundary
    fault (signed, zero-sublevel convention, with a 1e-6 margin that makes a
    pursuer exactly on the wall lose)."""
    if grid.extent <= config.arena_half_width:
        raise ValueError("The numerical domain must extend outside the physical square.")
    x = np.asarray(grid.axes[0], dtype=dtype)
    xp, yp = x[:, None, None, None, None, None], x[None, :, None, None, None, None]
    xe, ye = x[None, None, None, :, None, None], x[None, None, None, None, :, None]
    capture = np.sqrt((xp - xe) ** 2 + (yp - ye) ** 2) - config.capture_radius
    e_fault = config.arena_half_width - np.maximum(abs(xe), abs(ye))
    target = np.broadcast_to(np.minimum(capture, e_fault), grid.shape).copy()
    avoid = np.broadcast_to(np.maximum(abs(xp), abs(yp)) - config.arena_half_width + 1e-6,
                            grid.shape).copy()
    return target.astype(dtype, copy=False), avoid.astype(dtype, copy=False)


def output_times(horizon, output_dt):
    if not np.isfinite([horizon, output_dt]).all() or horizon <= 0 or output_dt <= 0:
        raise ValueError("Horizon and output spacing must be finite and positive.")
    times = np.minimum(np.arange(int(np.ceil(horizon / output_dt)) + 1) * output_dt, horizon)
    return np.unique(times)


def global_rate_bound(grid: GridSpec, config: GameConfig):
    dx, _, dh, *_ = grid.spacings
    return (2 * (config.pursuer.speed + config.evader.speed) / dx
            + (config.pursuer.max_turn_rate + config.evader.max_turn_rate) / dh)
