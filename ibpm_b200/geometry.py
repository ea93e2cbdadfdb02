"""Body geometry for the IBPM time step: the reference's `.geom` DSL and
rigid-body motions, expressed as the plain arrays the C-ABI takes.

Follows the reference's parser (src/Geometry.cc:143-205, src/RigidBody.cc:248-529)
for the commands the time step uses: ``body``/``end``, ``circle``, ``circle_n``,
``line``, ``line_n``, ``line_aoa``, ``point``, ``raw``, ``center`` and
``motion fixed | pitchplunge``.  Point generation follows
src/RigidBody.cc:92-170.  Other motion types are rejected with a clear error.
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field
from typing import List, Tuple

import numpy as np

MOTION_NONE = 0
MOTION_FIXED = 1
MOTION_PITCHPLUNGE = 2


@dataclass
class RigidBody:
    name: str = ""
    points: List[Tuple[float, float]] = field(default_factory=list)
    center: Tuple[float, float] = (0.0, 0.0)
    motion: int = MOTION_NONE
    params: Tuple[float, ...] = (0.0,) * 6

    @property
    def stationary(self) -> bool:
        return self.motion != MOTION_PITCHPLUNGE

    def add_circle_n(self, xc, yc, r, n):  # src/RigidBody.cc:105-118
        twopi = 8.0 * math.atan(1.0)
        dth = twopi / n
        for i in range(n):
            self.points.append((xc + r * math.cos(i * dth), yc + r * math.sin(i * dth)))

    def add_circle(self, xc, yc, r, dx):  # src/RigidBody.cc:92-103
        twopi = 8.0 * math.atan(1.0)
        n = int(math.floor(twopi / (dx / r) + 1 + 0.5))
        self.add_circle_n(xc, yc, r, n)

    def add_line_n(self, x1, y1, x2, y2, n):  # src/RigidBody.cc:133-146
        dX = (x2 - x1) / (n - 1)
        dY = (y2 - y1) / (n - 1)
        for i in range(n):
            self.points.append((x1 + i * dX, y1 + i * dY))

    def add_line(self, x1, y1, x2, y2, dx):  # src/RigidBody.cc:120-131
        length = math.sqrt((x2 - x1) ** 2 + (y2 - y1) ** 2)
        self.add_line_n(x1, y1, x2, y2, int(math.floor(length / dx + 1 + 0.5)))

    def add_line_aoa(self, l, xC, yC, aoa, n):  # src/RigidBody.cc:148-170
        pi = 3.141592653589793238462643383279502884197169399375
        a = aoa / 180 * pi
        ca, sa = math.cos(a), math.sin(a)
        d = l / (n - 1)
        for i in range(n):
            x0r, y0r = i * d - xC, 0.0 - yC
            self.points.append((x0r * ca - y0r * sa + xC, x0r * sa + y0r * ca + yC))


@dataclass
class Geometry:
    bodies: List[RigidBody] = field(default_factory=list)

    @property
    def num_points(self) -> int:
        return sum(len(b.points) for b in self.bodies)

    @property
    def stationary(self) -> bool:
        return all(b.stationary for b in self.bodies)

    def ref_points(self) -> np.ndarray:
        return np.array([p for b in self.bodies for p in b.points], dtype=np.float64).reshape(-1, 2)

    def points_velocities(self, t: float):
        """Geometry::moveBodies + getPoints/getVelocities at time t
        (src/Geometry.cc:79-121, src/RigidBody.cc:586-609)."""
        pos, vel = [], []
        for b in self.bodies:
            P = np.array(b.points, dtype=np.float64).reshape(-1, 2)
            if b.motion == MOTION_NONE:
                pos.append(P)
                vel.append(np.zeros_like(P))
                continue
            if b.motion == MOTION_FIXED:
                x, y, th = b.params[:3]
                xd = yd = thd = 0.0
            else:
                twopi = 8.0 * math.atan(1.0)
                ap, fp, php, ay, fy, phy = b.params
                wp, wy = fp * twopi, fy * twopi
                x, xd = 0.0, 0.0
                y = ay * math.sin(wy * t + phy)
                yd = ay * wy * math.cos(wy * t + phy)
                th = ap * math.sin(wp * t + php)
                thd = ap * wp * math.cos(wp * t + php)
            a = P[:, 0] - b.center[0]
            bb = P[:, 1] - b.center[1]
            c, s = math.cos(th), math.sin(th)
            pos.append(np.stack([x + a * c - bb * s + b.center[0], y + a * s + bb * c + b.center[1]], 1))
            vel.append(np.stack([-a * s * thd - bb * c * thd + xd, a * c * thd - bb * s * thd + yd], 1))
        return np.concatenate(pos), np.concatenate(vel)


class GeometryError(ValueError):
    pass


def parse(text: str, basedir: str = ".") -> Geometry:
    """Parse the `.geom` DSL (src/Geometry.cc:143-205, src/RigidBody.cc:248-529)."""
    geo = Geometry()
    lines = iter(text.splitlines())
    for raw in lines:
        tok = raw.split()
        if not tok or tok[0].startswith("#"):
            continue
        cmd = tok[0].lower()
        if cmd == "end":
            break
        if cmd != "body":
            raise GeometryError(f"could not parse line: {raw!r}")
        body = RigidBody(name=" ".join(tok[1:]))
        for braw in lines:
            bt = braw.split()
            if not bt or bt[0].startswith("#"):
                continue
            c = bt[0].lower()
            a = bt[1:]
            try:
                if c == "end":
                    break
                elif c == "center":
                    body.center = (float(a[0]), float(a[1]))
                elif c == "circle":
                    body.add_circle(*map(float, a[:4]))
                elif c == "circle_n":
                    body.add_circle_n(float(a[0]), float(a[1]), float(a[2]), int(a[3]))
                elif c == "line":
                    body.add_line(*map(float, a[:5]))
                elif c == "line_n":
                    body.add_line_n(float(a[0]), float(a[1]), float(a[2]), float(a[3]), int(a[4]))
                elif c == "line_aoa":
                    body.add_line_aoa(float(a[0]), float(a[1]), float(a[2]), float(a[3]), int(a[4]))
                elif c == "point":
                    body.points.append((float(a[0]), float(a[1])))
                elif c == "raw":
                    path = a[0] if os.path.isabs(a[0]) else os.path.join(basedir, a[0])
                    with open(path) as fh:
                        vals = fh.read().split()
                    n = int(vals[0])
                    for k in range(n):
                        body.points.append((float(vals[1 + 2 * k]), float(vals[2 + 2 * k])))
                elif c == "name":
                    body.name = " ".join(a)
                elif c == "motion":
                    kind = a[0].lower()
                    if kind == "fixed":
                        body.motion = MOTION_FIXED
                        body.params = tuple(float(v) for v in a[1:4]) + (0.0, 0.0, 0.0)
                    elif kind == "pitchplunge":
                        body.motion = MOTION_PITCHPLUNGE
                        body.params = tuple(float(v) for v in a[1:7])
                        if len(body.params) != 6:
                            raise GeometryError("pitchplunge takes 6 numbers (src/RigidBody.cc:373-384)")
                    else:
                        raise GeometryError(f"motion type {kind!r} is not supported by the GPU time step")
                else:
                    raise GeometryError(f"could not parse line: {braw!r}")
            except (IndexError, ValueError) as e:
                if isinstance(e, GeometryError):
                    raise
                raise GeometryError(f"bad arguments in line: {braw!r}") from e
        geo.bodies.append(body)
    return geo


def load(path: str) -> Geometry:
    with open(path) as fh:
        return parse(fh.read(), os.path.dirname(os.path.abspath(path)))
