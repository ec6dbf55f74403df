"""Footprints, the circular arena record and the oriented-rectangle contact
value (src/pursuit_evasion/local_game/geometry.py:15-70,
reversible/footprint_map.py:11-30), as used by the compact contact game.

`CircleArena.clearance` is the signed separation of a car's rectangle from
the walls and circles (geometry.py:131-152), used on the host when queries
are sampled; grid construction asks the GPU engine of local_game/engine.py.
Loading BARN occupancy maps (geometry.py:76-129) stays with the caller."""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


@dataclass(frozen=True)
class Footprint:
    """A car's rectangle: length along its heading, width across it."""
    length: float
    width: float

    def __post_init__(self):
        if (not np.isfinite([self.length, self.width]).all()
                or min(self.length, self.width) <= 0):
            raise ValueError("Footprint dimensions must be positive and finite")

    def to_dict(self):
        return dict(length=self.length, width=self.width)


def rectangle_separation(p, e, p_body=Footprint(0.8, 0.5), e_body=Footprint(0.4, 0.25)):
    """Positive iff the oriented rectangles are separated; <= 0 means contact
    (the largest gap along the four body axes, in double precision)."""
    p, e = np.asarray(p, np.float64), np.asarray(e, np.float64)
    d = e[..., :2] - p[..., :2]
    rel = e[..., 2] - p[..., 2]
    ca, sa = np.abs(np.cos(rel)), np.abs(np.sin(rel))
    gaps = []
    for pose, own, other in ((p, p_body, e_body), (e, e_body, p_body)):
        c, s = np.cos(pose[..., 2]), np.sin(pose[..., 2])
        along = d[..., 0] * c + d[..., 1] * s
        across = d[..., 1] * c - d[..., 0] * s
        gaps.append(np.abs(along) - own.length / 2 - (other.length * ca + other.width * sa) / 2)
        gaps.append(np.abs(across) - own.width / 2 - (other.length * sa + other.width * ca) / 2)
    return np.maximum.reduce(gaps)


@dataclass
class CircleArena:
    """Square arena of half width `half_width` with circular obstacles
    [x, y, r]; the footprints of both cars."""
    circles: np.ndarray
    half_width: float
    pursuer: Footprint = Footprint(0.8, 0.5)
    evader: Footprint = Footprint(0.4, 0.25)
    source: dict | None = field(default=None)

    def __post_init__(self):
        self.circles = np.asarray(self.circles, np.float64).reshape(-1, 3)
        if not np.isfinite(self.circles).all() or np.any(self.circles[:, 2] <= 0):
            raise ValueError("Finite circles[x,y,r] with positive radii required")
        if not np.isfinite(self.half_width) or self.half_width <= 0:
            raise ValueError("Positive bounded arena size required")

    def to_dict(self):
        return dict(circles=self.circles.tolist(), half_width=self.half_width,
                    pursuer=self.pursuer.to_dict(), evader=self.evader.to_dict(),
                    source=self.source, capture_rule="oriented_rectangle_contact",
                    pose_reference="rectangle_center")

    @classmethod
    def from_dict(cls, d):
        return cls(d["circles"], d["half_width"], Footprint(**d["pursuer"]),
                   Footprint(**d["evader"]), d.get("source"))

    def clearance(self, poses, role="pursuer"):
        """Signed separation of `role`'s rectangle at poses [..., >= 3]
        (x, y, heading) from the arena walls and every circle; <= 0 means
        contact."""
        s = np.asarray(poses, float)
        body = getattr(self, role)
        c, q = np.cos(s[..., 2]), np.sin(s[..., 2])
        half_x = (body.length * np.abs(c) + body.width * np.abs(q)) / 2
        half_y = (body.length * np.abs(q) + body.width * np.abs(c)) / 2
        out = np.minimum(self.half_width - np.abs(s[..., 0]) - half_x,
                         self.half_width - np.abs(s[..., 1]) - half_y)
        for cx, cy, r in self.circles:
            dx, dy = cx - s[..., 0], cy - s[..., 1]
            along = np.abs(dx * c + dy * q) - body.length / 2
            across = np.abs(dy * c - dx * q) - body.width / 2
            inside = np.minimum(np.maximum(along, across), 0)
            out = np.minimum(out, np.hypot(np.maximum(along, 0), np.maximum(across, 0))
                             + inside - r)
        return out

    def capture_value(self, state):
        s = np.asarray(state)
        return rectangle_separation(s[..., :4], s[..., 4:], self.pursuer, self.evader)
