"""The named IBPM workloads (grid, bodies, flow parameters) as data.

Each entry mirrors one workload description: the fixed cylinder at 200x200
(one domain), the multi-domain shedding cylinder at 400x200 with five nested
domains, the pitching-and-plunging flat plate at 500x250 with three domains,
the ensemble of ellipses, and the two plunging cylinders at 1024x1024.
Geometry is emitted in the reference's `.geom` DSL so that the CPU oracle
(the reference library) and this package read identical bodies.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Optional

import numpy as np


@dataclass
class Workload:
    name: str
    nx: int
    ny: int
    ngrid: int
    length: float
    xoffset: float
    yoffset: float
    geom: str
    Re: float
    dt: float
    nsteps: int
    scheme: str = "rk3"
    tol: float = 1e-7
    noise_amp: float = 0.0          # seeded N(0, amp^2) level-0 vorticity in the wake
    noise_seed: int = 0
    noise_box: tuple = (0.6, 1e9, -1.0, 1.0)   # x0, x1, y0, y1 of the seeded region
    extra: dict = field(default_factory=dict)

    @property
    def dx(self) -> float:
        return self.length / self.nx

    def initial_vorticity(self) -> Optional[np.ndarray]:
        """Seeded noise IC on level 0 (other levels zero), reference Scalar layout."""
        if self.noise_amp == 0.0:
            return None
        rng = np.random.default_rng(self.noise_seed)
        w = np.zeros((self.ngrid, self.nx - 1, self.ny - 1))
        x = self.xoffset + self.dx * np.arange(1, self.nx)
        y = self.yoffset + self.dx * np.arange(1, self.ny)
        X, Y = np.meshgrid(x, y, indexing="ij")
        x0, x1, y0, y1 = self.noise_box
        m = (X > x0) & (X < x1) & (Y > y0) & (Y < y1)
        w[0][m] = self.noise_amp * rng.standard_normal(int(m.sum()))
        return w


def cylinder_geom(n: int, r: float = 0.5, xc: float = 0.0, yc: float = 0.0) -> str:
    return f"body Cylinder\n  circle_n {xc!r} {yc!r} {r!r} {n}\nend\n"


def plate_geom(chord=1.0, npts=51, mean_aoa_deg=20.0, pitch_amp_deg=10.0, freq=0.25, plunge=0.25) -> str:
    """Flat plate of `chord` centred at the origin, pitching about its quarter chord.
    Positive angle of attack is a clockwise rotation (leading edge up), so the
    reference points carry the mean angle as a rotation by -mean_aoa and the
    PitchPlunge amplitude (counter-clockwise theta, radians) is -pitch_amp."""
    xq = -0.25 * chord
    a = -math.radians(mean_aoa_deg)
    pts = []
    for i in range(npts):
        x0 = -0.5 * chord + i * chord / (npts - 1)
        dxr = x0 - xq
        pts.append((xq + dxr * math.cos(a), dxr * math.sin(a)))
    lines = ["body Plate"] + [f"  point {x!r} {y!r}" for (x, y) in pts]
    lines.append(f"  center {xq!r} 0.0")
    lines.append(f"  motion pitchplunge {-math.radians(pitch_amp_deg)!r} {freq!r} 0 {plunge!r} {freq!r} 0")
    lines.append("end")
    return "\n".join(lines) + "\n"


def two_cylinders_geom(seed=5, n=201, amp=0.2, freq=0.2) -> str:
    rng = np.random.default_rng(seed)
    e1, e2 = (float(e) for e in rng.uniform(-0.1, 0.1, size=2))
    out = []
    for (yc, sgn) in ((0.75 + e1, 1.0), (-0.75 + e2, -1.0)):
        out.append(f"body Cylinder\n  circle_n 0 {yc!r} 0.5 {n}\n  center 0 {yc!r}\n"
                   f"  motion pitchplunge 0 0 0 {sgn * amp!r} {freq!r} 0\nend")
    return "\n".join(out) + "\n"


def c1_fixed_cylinder() -> Workload:
    return Workload("cylinder_200x200_ngrid1", 200, 200, 1, 4.0, -2.0, -2.0, cylinder_geom(157),
                    Re=100.0, dt=0.01, nsteps=250)


def c2_shedding_cylinder() -> Workload:
    return Workload("cylinder_400x200_ngrid5_shedding", 400, 200, 5, 8.0, -2.0, -2.0, cylinder_geom(157),
                    Re=200.0, dt=0.005, nsteps=4000, noise_amp=1e-3, noise_seed=2024)


def c3_pitching_plate() -> Workload:
    return Workload("plate_500x250_ngrid3_pitchplunge", 500, 250, 3, 10.0, -5.0, -2.5, plate_geom(),
                    Re=300.0, dt=0.004, nsteps=5000, tol=1e-10)


def c5_two_cylinders() -> Workload:
    return Workload("two_cylinders_1024x1024_ngrid5", 1024, 1024, 5, 16.0, -8.0, -8.0, two_cylinders_geom(),
                    Re=500.0, dt=0.005, nsteps=10000, tol=1e-10)


def ensemble_members(count=64, seed=11):
    """Ensemble of independent ellipse runs with seeded n, ngrid, b, orientation, Re."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        n = int(rng.choice([128, 192, 256, 384, 512]))
        ngrid = int(rng.integers(1, 4))
        b = float(rng.uniform(0.1, 0.5))
        th = float(rng.uniform(0, math.pi))
        Re = float(rng.uniform(50, 300))
        dx = 4.0 / n
        # ellipse with semi-axes a = 0.5, b; points equally spaced in arc length, spacing ~ dx
        t = np.linspace(0.0, 2 * math.pi, 20001)
        ex, ey = 0.5 * np.cos(t), b * np.sin(t)
        arc = np.concatenate([[0.0], np.cumsum(np.hypot(np.diff(ex), np.diff(ey)))])
        npts = max(8, int(round(arc[-1] / dx)))
        ts = np.interp(np.arange(npts) * arc[-1] / npts, arc, t)
        ex, ey = 0.5 * np.cos(ts), b * np.sin(ts)
        px = ex * math.cos(th) - ey * math.sin(th)
        py = ex * math.sin(th) + ey * math.cos(th)
        geom = "body Ellipse\n" + "".join(f"  point {float(x)!r} {float(y)!r}\n" for x, y in zip(px, py)) + "end\n"
        out.append(Workload(f"ellipse_{k}", n, n, ngrid, 4.0, -2.0, -2.0, geom, Re=Re, dt=0.5 * dx,
                            nsteps=1000))
    return out


ALL = {
    "c1": c1_fixed_cylinder,
    "c2": c2_shedding_cylinder,
    "c3": c3_pitching_plate,
    "c5": c5_two_cylinders,
}
