"""Body geometry for the IBPM time step: the reference's `.geom` DSL and
rigid-body motions, expressed as the plain arrays the C-ABI takes.

Follows the reference's parser (src/Geometry.cc:143-205, src/RigidBody.cc:248-529)
for the commands the time step uses: ``body``/``end``, ``circle``, ``circle_n``,
``line``, ``line_n``, ``line_aoa``, ``point``, ``raw``, ``center``, ``name`` and
every ``motion`` type of src/RigidBody.cc:349-493 (fixed, fixedvel,
pitchplunge, sigmoidalstep, lagstep1, lagstep2, eldredge, eldredgecombined2,
eldredge1, eldredge2, motionfile, motionfileperiodic).  Point generation
follows src/RigidBody.cc:92-170; a motion file is read as src/MotionFile.h:47-69
reads it (a row count, then rows of t x y theta xdot ydot thetadot).  The
kinematics themselves are evaluated on the device.
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field
from typing import List, Optional, Tuple

import numpy as np

MOTION_NONE = 0
MOTION_FIXED = 1
MOTION_PITCHPLUNGE = 2
MOTION_FIXEDVEL = 3
MOTION_SIGMOIDALSTEP = 4
MOTION_LAGSTEP1 = 5
MOTION_LAGSTEP2 = 6
MOTION_ELDREDGE = 7
MOTION_ELDREDGECOMBINED2 = 8
MOTION_ELDREDGE1 = 9
MOTION_ELDREDGE2 = 10
MOTION_FILE = 11
MOTION_FILE_PERIODIC = 12

# `motion` keyword -> (code, count of numbers after it) (src/RigidBody.cc:349-493)
MOTIONS = {
    "fixed": (MOTION_FIXED, 3),
    "fixedvel": (MOTION_FIXEDVEL, 3),
    "pitchplunge": (MOTION_PITCHPLUNGE, 6),
    "sigmoidalstep": (MOTION_SIGMOIDALSTEP, 3),
    "lagstep1": (MOTION_LAGSTEP1, 4),
    "lagstep2": (MOTION_LAGSTEP2, 4),
    "eldredge": (MOTION_ELDREDGE, 6),
    "eldredgecombined2": (MOTION_ELDREDGECOMBINED2, 12),
    "eldredge1": (MOTION_ELDREDGE1, 6),
    "eldredge2": (MOTION_ELDREDGE2, 6),
    "motionfile": (MOTION_FILE, 0),
    "motionfileperiodic": (MOTION_FILE_PERIODIC, 1),
}
MOTION_NAMES = {code: name for name, (code, _) in MOTIONS.items()}
MOTION_NAMES[MOTION_NONE] = "none"


@dataclass
class RigidBody:
    name: str = ""
    points: List[Tuple[float, float]] = field(default_factory=list)
    center: Tuple[float, float] = (0.0, 0.0)
    motion: int = MOTION_NONE
    params: Tuple[float, ...] = ()
    table: Optional[np.ndarray] = None    # motion file rows (t, x, y, theta, xdot, ydot, thetadot)

    @property
    def stationary(self) -> bool:
        # Motion::isStationary is true only for FixedPosition (src/Motion.h:28, src/FixedPosition.h:39)
        return self.motion in (MOTION_NONE, MOTION_FIXED)

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
                    if kind not in MOTIONS:
                        raise GeometryError(f"unknown motion type {kind!r}")
                    code, npar = MOTIONS[kind]
                    body.motion = code
                    if code in (MOTION_FILE, MOTION_FILE_PERIODIC):
                        path = a[1] if os.path.isabs(a[1]) else os.path.join(basedir, a[1])
                        body.table = read_motion_file(path)
                        body.params = tuple(float(v) for v in a[2:2 + npar])
                    else:
                        body.params = tuple(float(v) for v in a[1:1 + npar])
                    if len(body.params) != npar:
                        raise GeometryError(f"motion {kind} takes {npar} numbers")
                else:
                    raise GeometryError(f"could not parse line: {braw!r}")
            except (IndexError, ValueError) as e:
                if isinstance(e, GeometryError):
                    raise
                raise GeometryError(f"bad arguments in line: {braw!r}") from e
        geo.bodies.append(body)
    return geo


def read_motion_file(path: str) -> np.ndarray:
    """Rows (t, x, y, theta, xdot, ydot, thetadot) of a motion file: a row
    count, then that many rows (src/MotionFile.h:47-69); t non-decreasing."""
    with open(path) as fh:
        vals = fh.read().split()
    try:
        n = int(vals[0])
        rows = np.array([float(v) for v in vals[1:1 + 7 * n]], dtype=np.float64)
    except (IndexError, ValueError) as e:
        raise GeometryError(f"motion file {path} formatted incorrectly") from e
    if n < 0 or rows.size != 7 * n:
        raise GeometryError(f"motion file {path} formatted incorrectly")
    rows = rows.reshape(n, 7)
    if n > 1 and np.any(np.diff(rows[:, 0]) < 0):
        raise GeometryError(f"motion file {path}: time must increase monotonically")
    return rows


def load(path: str) -> Geometry:
    with open(path) as fh:
        return parse(fh.read(), os.path.dirname(os.path.abspath(path)))
