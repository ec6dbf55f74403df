"""Grid of the legacy 6D square game, state order [xP, yP, thetaP, xE, yE,
thetaE].

The interface is the reference's (dp/grid.py:9-100): the GridSpec fields
and their defaults, its validation errors, the `shape` / `states` / `axes`
/ `spacings` properties and the metadata keys of `to_dict`, which the table
folders carry; and `output_times`.  The surfaces and the time-step bound
that the reference's Python backends build here are computed by this
package's C ABI (pe_square_init, pe_square_dt_limit), so they are not
repeated in Python.
"""

from __future__ import annotations

from dataclasses import dataclass
import math

import numpy as np

_STATE_ORDER = ("xP", "yP", "thetaP", "xE", "yE", "thetaE")
_PERIODIC = (2, 5)


def _is_count(n):
    return isinstance(n, (int, np.integer)) and not isinstance(n, bool)


@dataclass(frozen=True)
class GridSpec:
    """`positions` nodes per position axis on [-extent, extent] and
    `headings` periodic heading nodes from -pi, for each car."""

    positions: int = 17
    headings: int = 16
    extent: float = 3.5

    def __post_init__(self):
        if not (_is_count(self.positions) and _is_count(self.headings)
                and self.positions >= 5 and self.headings >= 4):
            raise ValueError("Grid counts must be integers with at least five position "
                             "samples and four periodic headings.")
        if not (math.isfinite(self.extent) and self.extent > 0):
            raise ValueError("Grid extent must be finite and positive.")

    # per-car axes: position, position, heading
    def _position_axis(self):
        return np.linspace(-self.extent, self.extent, self.positions)

    def _heading_axis(self):
        # node k at k * 2 pi / headings - pi, rounded as the tables' writer does
        return np.arange(self.headings) * 2 * np.pi / self.headings - np.pi

    @property
    def shape(self):
        car = (self.positions, self.positions, self.headings)
        return car + car

    @property
    def states(self):
        return int(np.prod(self.shape))

    @property
    def axes(self):
        x, theta = self._position_axis(), self._heading_axis()
        return (x, x, theta) * 2

    @property
    def spacings(self):
        car = (2 * self.extent / (self.positions - 1),) * 2 + (2 * np.pi / self.headings,)
        return car * 2

    def to_dict(self):
        return {
            "positions": self.positions,
            "headings": self.headings,
            "extent": self.extent,
            "shape": list(self.shape),
            "states": self.states,
            "spacings": list(self.spacings),
            "periodic_axes": list(_PERIODIC),
            "state_order": list(_STATE_ORDER),
        }


def output_times(horizon, output_dt):
    """Frame times 0, dt, 2 dt, ... up to and including `horizon` (the last
    interval may be shorter)."""
    if not (np.isfinite(horizon) and np.isfinite(output_dt) and horizon > 0
            and output_dt > 0):
        raise ValueError("Horizon and output spacing must be finite and positive.")
    frames = int(np.ceil(horizon / output_dt))
    times = [min(k * output_dt, horizon) for k in range(frames + 1)]
    return np.array(sorted(set(times)))
