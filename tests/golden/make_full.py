"""Generate the benchmark-size fixtures (full_*.npz) from the reference itself.

Runs the reference IBPM library (oracle/_ref/ref_driver_parity: the reference
sources built by oracle/Makefile, -O2 without fast-math, with the project's
FFTW shim) on the named workloads at their full grid sizes, for a truncated
number of steps, and stores the per-step forces and the final state:

* full_c1        200x200 fixed cylinder, Re 100, dt 0.01, RK3: all 250 steps;
                 final omega, q, f, and psi = L^-1(-omega) from the reference's
                 own Poisson solver (oracle/refops.py)
* full_c2        400x200 x5-domain shedding cylinder with the seeded wake noise,
                 Re 200, dt 0.005: the first 20 steps; final omega and f
* full_c3        500x250 x3-domain pitching/plunging plate, plain CG at tol 1e-10:
                 the first 3 steps; final omega and f
* full_c4_<k>    two ensemble members (the first two with n <= 256): 10 steps each;
                 final omega and f
* full_c5        1024x1024 x5-domain pair of plunging cylinders, plain CG at tol
                 1e-10: the first 2 steps; f, the per-level L2 norms of omega and
                 omega on every 8th node in i and j of every level (the full field
                 is 42 MB)

The initial vorticity of the seeded cases is not stored: the tests regenerate it
from the workload's seed (ibpm_b200.configs).

Usage (from the repository root, with the reference built):
    make -C oracle all && python tests/golden/make_full.py [c1 c2 c3 c4 c5]
C5 takes several minutes of CPU per step.
"""
import os
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from ibpm_b200 import configs, geometry  # noqa: E402
from oracle import ibpm_oracle as O  # noqa: E402

DRIVER = os.path.join(ROOT, "oracle", "_ref", "ref_driver_parity")
HERE = os.path.dirname(os.path.abspath(__file__))
C5_SAMPLE = 8


def reference_run(wl, nsteps):
    """The reference's forces per step and its final state after `nsteps` steps."""
    with tempfile.TemporaryDirectory() as td:
        gpath = os.path.join(td, "body.geom")
        with open(gpath, "w") as fh:
            fh.write(wl.geom)
        args = [DRIVER, "-nx", str(wl.nx), "-ny", str(wl.ny), "-ngrid", str(wl.ngrid), "-length", repr(wl.length),
                "-xoffset", repr(wl.xoffset), "-yoffset", repr(wl.yoffset), "-geom", gpath, "-Re", repr(wl.Re),
                "-dt", repr(wl.dt), "-scheme", wl.scheme, "-nsteps", str(nsteps), "-tol", repr(wl.tol),
                "-out", os.path.join(td, "run")]
        w0 = wl.initial_vorticity()
        if w0 is not None:
            g = O.Grid(wl.nx, wl.ny, wl.ngrid, wl.length, wl.xoffset, wl.yoffset)
            st = O.State(g, geometry.parse(wl.geom).num_points, omega=w0)
            ic = os.path.join(td, "ic.bin")
            O.save_restart(ic, st, g)
            args += ["-ic", ic]
        subprocess.run(args, check=True, stdout=subprocess.DEVNULL, cwd=td)
        forces = np.loadtxt(os.path.join(td, "run.forces")).reshape(-1, 6)
        fin = O.load_restart(os.path.join(td, "run_final.bin"))
    return forces, fin


def save(name, wl, nsteps, forces, fin, **arrays):
    np.savez_compressed(os.path.join(HERE, name + ".npz"), workload=wl.name, nsteps=nsteps, forces=forces,
                        f=fin["f"], timestep=fin["timestep"], time=fin["time"], **arrays)
    print(name, "written:", nsteps, "steps, final force", forces[-1, 2:4])


def make_c1():
    from oracle import refops
    wl = configs.c1_fixed_cylinder()
    forces, fin = reference_run(wl, 250)
    g = O.Grid(wl.nx, wl.ny, wl.ngrid, wl.length, wl.xoffset, wl.yoffset)
    psi = refops.elliptic(g, "poisson", 0.0, -fin["omega"])
    save("full_c1", wl, 250, forces, fin, omega=fin["omega"], q=fin["q"], psi=psi)


def make_c2():
    wl = configs.c2_shedding_cylinder()
    forces, fin = reference_run(wl, 20)
    save("full_c2", wl, 20, forces, fin, omega=fin["omega"])


def make_c3():
    wl = configs.c3_pitching_plate()
    forces, fin = reference_run(wl, 3)
    save("full_c3", wl, 3, forces, fin, omega=fin["omega"])


def c4_members():
    """The two ensemble members the fixtures cover: the first two with n <= 256."""
    return [(k, w) for k, w in enumerate(configs.ensemble_members()) if w.nx <= 256][:2]


def make_c4():
    for k, wl in c4_members():
        forces, fin = reference_run(wl, 10)
        save(f"full_c4_{k}", wl, 10, forces, fin, member=k, omega=fin["omega"])


def make_c5():
    wl = configs.c5_two_cylinders()
    forces, fin = reference_run(wl, 2)
    w = fin["omega"]
    save("full_c5", wl, 2, forces, fin, omega_sample=w[:, ::C5_SAMPLE, ::C5_SAMPLE].copy(), sample=C5_SAMPLE,
         omega_level_norms=np.linalg.norm(w.reshape(w.shape[0], -1), axis=1))


if __name__ == "__main__":
    which = sys.argv[1:] or ["c1", "c2", "c3", "c4", "c5"]
    for c in which:
        globals()["make_" + c]()
