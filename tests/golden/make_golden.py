"""Generate the golden fixtures in this directory from the reference itself.

Runs the reference IBPM library (oracle/_ref/ref_driver_parity, built from the
reference sources by oracle/Makefile with the project's FFTW shim) on small
seeded cases and stores per-step forces and the final state as .npz.

Usage (from the repository root, with the reference sources present):
    make -C oracle all && python tests/golden/make_golden.py
"""
import os
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from ibpm_b200 import configs  # noqa: E402
from oracle import ibpm_oracle as O  # noqa: E402

DRIVER = os.path.join(ROOT, "oracle", "_ref", "ref_driver_parity")
HERE = os.path.dirname(os.path.abspath(__file__))

CASES = [
    # name, nx, ny, ngrid, length, xoff, yoff, geom, Re, dt, nsteps, scheme, tol, noise(amp, seed)
    ("cyl_l1_rk3", 48, 48, 1, 4.0, -2.0, -2.0, configs.cylinder_geom(36), 100.0, 0.02, 8, "rk3", 1e-7, None),
    ("cyl_l3_noise_rk3", 64, 32, 3, 4.0, -1.5, -1.0, configs.cylinder_geom(32, r=0.4), 200.0, 0.01, 8, "rk3",
     1e-7, (1e-3, 7)),
    ("cyl_l2_euler", 32, 32, 2, 3.0, -1.5, -1.5, configs.cylinder_geom(24, r=0.4), 150.0, 0.02, 6, "euler",
     1e-7, (1e-2, 3)),
    ("cyl_l2_ab2", 32, 32, 2, 3.0, -1.5, -1.5, configs.cylinder_geom(24, r=0.4), 150.0, 0.02, 6, "ab2",
     1e-7, (1e-2, 3)),
    ("plate_l2_pitchplunge_cg", 64, 32, 2, 4.0, -2.0, -1.0,
     configs.plate_geom(chord=1.0, npts=17, freq=0.5), 300.0, 0.01, 6, "rk3", 1e-10, None),
    ("cyl_l1_rk3b", 40, 40, 1, 4.0, -2.0, -2.0, configs.cylinder_geom(30), 80.0, 0.02, 5, "rk3b", 1e-7, None),
    # ny = 2 (mod 4) with several domains, as in the 500x250 plate workload (release-build nesting)
    ("cyl_l3_ny2mod4", 48, 26, 3, 4.8, -2.0, -1.3, configs.cylinder_geom(18, r=0.3), 120.0, 0.02, 5, "rk3",
     1e-7, (1e-3, 5)),
    ("plate_l3_ny2mod4_cg", 60, 30, 3, 6.0, -3.0, -1.5,
     configs.plate_geom(chord=1.0, npts=11, freq=0.5), 300.0, 0.01, 4, "rk3", 1e-10, None),
]


# cases whose final state the reference also writes as Tecplot files of every level (-tecplot)
TECPLOT_CASES = {"cyl_l3_noise_rk3"}


def run(case, files=None, ubf=False):
    """files: {name: text} written beside the geometry file; the driver runs
    there, so a `motion motionfile NAME` line finds NAME as the reference does.
    ubf: the body's motion is carried by the base flow (the CLI's -ubf)."""
    name, nx, ny, ngrid, length, xoff, yoff, geom, Re, dt, nsteps, scheme, tol, noise = case
    files = files or {}
    with tempfile.TemporaryDirectory() as td:
        gpath = os.path.join(td, "body.geom")
        with open(gpath, "w") as fh:
            fh.write(geom)
        for fname, text in files.items():
            with open(os.path.join(td, fname), "w") as fh:
                fh.write(text)
        args = [DRIVER, "-nx", str(nx), "-ny", str(ny), "-ngrid", str(ngrid), "-length", repr(length),
                "-xoffset", repr(xoff), "-yoffset", repr(yoff), "-geom", gpath, "-Re", repr(Re),
                "-dt", repr(dt), "-scheme", scheme, "-nsteps", str(nsteps), "-tol", repr(tol),
                "-out", os.path.join(td, "run")] + (["-ubf", "1"] if ubf else [])
        if name in TECPLOT_CASES:
            args += ["-tecplot", os.path.join(td, "tec")]
        w0 = None
        if noise is not None:
            wl = configs.Workload(name, nx, ny, ngrid, length, xoff, yoff, geom, Re, dt, nsteps,
                                  noise_amp=noise[0], noise_seed=noise[1], noise_box=(0.0, 1e9, -0.8, 0.8))
            w0 = wl.initial_vorticity()
            g = O.Grid(nx, ny, ngrid, length, xoff, yoff)
            from ibpm_b200 import geometry
            npts = geometry.parse(geom).num_points
            st = O.State(g, npts, omega=w0)
            ic = os.path.join(td, "ic.bin")
            O.save_restart(ic, st, g)
            args += ["-ic", ic]
        subprocess.run(args, check=True, stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL, cwd=td)
        forces = np.loadtxt(os.path.join(td, "run.forces")).reshape(-1, 6)
        fin = O.load_restart(os.path.join(td, "run_final.bin"))
        tecs = []
        if name in TECPLOT_CASES:
            for lev in range(ngrid):
                with open(os.path.join(td, "tec%05d_g%01d.plt" % (nsteps, lev))) as fh:
                    tecs.append(fh.read())
    extra = {"ubf": 1} if ubf else {}
    if name in TECPLOT_CASES:
        extra["tecplot_texts"] = np.array(tecs)
    if files:
        extra.update(file_names=np.array(list(files.keys())), file_texts=np.array(list(files.values())))
    np.savez_compressed(
        os.path.join(HERE, name + ".npz"),
        nx=nx, ny=ny, ngrid=ngrid, length=length, xoffset=xoff, yoffset=yoff, geom=geom, Re=Re, dt=dt,
        nsteps=nsteps, scheme=scheme, tol=tol,
        omega0=(w0 if w0 is not None else np.zeros((ngrid, nx - 1, ny - 1))),
        forces=forces, omega=fin["omega"], q=fin["q"], f=fin["f"], timestep=fin["timestep"], time=fin["time"],
        **extra)
    print(name, "written", forces[-1, 2:4])


# Every other `motion` type of the reference's geometry files (src/RigidBody.cc:349-493) on the
# pitching-plate case above, its parameters chosen so that the 6 steps (t in [0, 0.06]) cross the
# motions' branches and ramps.
def _motion_table(t, seed):
    rng = np.random.default_rng(seed)
    rows = np.column_stack([t] + [np.cumsum(rng.uniform(-0.02, 0.02, len(t))) for _ in range(3)] +
                           [rng.uniform(-1.0, 1.0, len(t)) for _ in range(3)])
    return "%d\n" % len(t) + "".join(" ".join(repr(float(v)) for v in r) + "\n" for r in rows)


MOTION_FILE = _motion_table(np.array([0.0, 0.008, 0.02, 0.033, 0.041, 0.05, 0.07]), 1)
MOTION_FILE_PERIODIC = _motion_table(np.array([0.0, 0.007, 0.015, 0.022, 0.03]), 2)
MOTION_CASES = [
    # name, motion line, files
    ("fixedvel", "fixedvel 0.4 -0.25 0.8", None),
    ("sigmoidalstep", "sigmoidalstep 15 0.08 0.005", None),
    ("lagstep1", "lagstep1 5 0.03 0.01 0.005", None),
    ("lagstep2", "lagstep2 5 0.03 0.008 0.004", None),
    ("eldredge", "eldredge 10 120 0.005 0.02 0.035 0.05", None),
    ("eldredge1", "eldredge1 0.05 120 0.005 0.02 0.035 0.05", None),
    ("eldredge2", "eldredge2 0.5 120 0.005 0.02 0.035 0.05", None),
    ("eldredgecombined2", "eldredgecombined2 0.5 120 0.005 0.02 0.035 0.05 8 100 0.0 0.015 0.03 0.045", None),
    ("motionfile", "motionfile plate.motion", {"plate.motion": MOTION_FILE}),
    ("motionfileperiodic", "motionfileperiodic plate.motion 0.03", {"plate.motion": MOTION_FILE_PERIODIC}),
]


def run_motion(case, ubf=False):
    kind, line, files = case
    geom = configs.plate_geom(chord=1.0, npts=17, freq=0.5)
    geom = "\n".join(("  motion " + line) if ln.strip().startswith("motion") else ln for ln in geom.splitlines()) + "\n"
    name = ("ubf_" if ubf else "motion_") + kind
    run((name, 64, 32, 2, 4.0, -2.0, -1.0, geom, 300.0, 0.01, 6, "rk3", 1e-10, None), files, ubf)


# The unsteady base flow (the CLI's -ubf): the same plate, its motion carried by the base flow, so the
# force solve is the fixed-body Cholesky one; stateful and rotating motions among them.
UBF_CASES = [
    ("pitchplunge", "pitchplunge -0.3 0.5 0 0.25 0.5 0", None),
    ("fixedvel", "fixedvel 0.4 -0.25 0.8", None),
    ("eldredge2", "eldredge2 0.5 120 0.005 0.02 0.035 0.05", None),
    ("eldredgecombined2", "eldredgecombined2 0.5 120 0.005 0.02 0.035 0.05 8 100 0.0 0.015 0.03 0.045", None),
    ("motionfile", "motionfile plate.motion", {"plate.motion": MOTION_FILE}),
]


# Motions under the other schemes (AB2 keeps the previous sub-step's nonlinear term, Euler has one
# sub-step), and two bodies with different motions in one geometry (a history-dependent plunge and a
# fixed cylinder).
def _plate_with(line):
    geom = configs.plate_geom(chord=1.0, npts=17, freq=0.5)
    return "\n".join(("  motion " + line) if ln.strip().startswith("motion") else ln for ln in geom.splitlines()) + "\n"


def _two_bodies():
    plate = _plate_with("eldredge2 0.5 120 0.005 0.02 0.035 0.05")
    cyl = configs.cylinder_geom(16, r=0.15).replace("0.0 0.0", "1.2 0.3", 1)
    return plate + cyl


MIXED_CASES = [
    # name, geometry, scheme, ubf
    ("motion_sigmoidalstep_ab2", _plate_with("sigmoidalstep 15 0.08 0.005"), "ab2", False),
    ("motion_lagstep2_euler", _plate_with("lagstep2 5 0.03 0.008 0.004"), "euler", False),
    ("ubf_pitchplunge_rk3b", _plate_with("pitchplunge -0.3 0.5 0 0.25 0.5 0"), "rk3b", True),
    ("motion_two_bodies_rk3", None, "rk3", False),
]


def run_mixed(case):
    name, geom, scheme, ubf = case
    if geom is None:
        geom = _two_bodies()
    run((name, 64, 32, 2, 4.0, -2.0, -1.0, geom, 300.0, 0.01, 6, scheme, 1e-10, None), None, ubf)


# The other N(x) variants of the reference (src/IBSolver.cc:211-311) on one small two-domain case.
# The base states of the linear models are states of a short nonlinear run written by the reference.
VARIANT_GRID = dict(nx=32, ny=32, ngrid=2, length=3.0, xoff=-1.5, yoff=-1.5)
VARIANT_GEOM = configs.cylinder_geom(24, r=0.4)
VARIANTS = [
    # name, model, Re, dt, nsteps, scheme, extra
    ("var_linear_l2_rk3", "linear", 150.0, 0.02, 6, "rk3", {}),
    ("var_linearperiodic_l2_rk3", "linearperiodic", 150.0, 0.02, 6, "rk3", {"period": 2}),
    ("var_adjoint_l2_rk3", "adjoint", 150.0, 0.02, 6, "rk3", {}),
    ("var_sfd_l2_rk3", "sfd", 150.0, 0.02, 6, "rk3", {"chi": 0.5, "Delta": 2.0}),
    ("var_sfd_l2_ab2", "sfd", 150.0, 0.02, 6, "ab2", {"chi": 0.5, "Delta": 2.0}),
]


def run_variant(case):
    name, model, Re, dt, nsteps, scheme, extra = case
    G = VARIANT_GRID
    nx, ny, ngrid = G["nx"], G["ny"], G["ngrid"]
    from ibpm_b200 import geometry
    npts = geometry.parse(VARIANT_GEOM).num_points
    g = O.Grid(nx, ny, ngrid, G["length"], G["xoff"], G["yoff"])
    with tempfile.TemporaryDirectory() as td:
        gpath = os.path.join(td, "body.geom")
        with open(gpath, "w") as fh:
            fh.write(VARIANT_GEOM)
        common = [DRIVER, "-nx", str(nx), "-ny", str(ny), "-ngrid", str(ngrid), "-length", repr(G["length"]),
                  "-xoffset", repr(G["xoff"]), "-yoffset", repr(G["yoff"]), "-geom", gpath, "-Re", repr(Re),
                  "-dt", repr(dt), "-scheme", scheme]
        wl = configs.Workload(name, nx, ny, ngrid, G["length"], G["xoff"], G["yoff"], VARIANT_GEOM, Re, dt, nsteps,
                              noise_amp=1e-2, noise_seed=11, noise_box=(0.0, 1e9, -0.8, 0.8))
        w0 = wl.initial_vorticity()
        ic = os.path.join(td, "ic.bin")
        O.save_restart(ic, O.State(g, npts, omega=w0), g)
        # base states: a nonlinear run from the same noise, steps 3 and 4
        subprocess.run(common + ["-nsteps", "4", "-ic", ic, "-out", os.path.join(td, "base"), "-dump_every", "1"],
                       check=True, stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        bases = [O.load_restart(os.path.join(td, "base_%05d.bin" % k)) for k in (3, 4)]
        args = common + ["-nsteps", str(nsteps), "-model", model, "-out", os.path.join(td, "run")]
        rec = {"model": model}
        if model in ("linear", "linearperiodic", "adjoint"):
            # the perturbation starts as the noise alone (no base flow in a linear model)
            period = extra.get("period", 1)
            for k in range(period):
                O.save_restart(os.path.join(td, "pb_%d.bin" % k),
                               O.State(g, npts, omega=bases[k]["omega"], q=bases[k]["q"]), g)
            if model in ("linear", "adjoint"):
                args += ["-baseflow", os.path.join(td, "pb_0.bin")]
            else:
                args += ["-pbase", os.path.join(td, "pb"), "-period", str(period)]
            rec["period"] = period
            rec["base_omega"] = np.stack([bases[k]["omega"] for k in range(period)])
            rec["base_q"] = np.stack([bases[k]["q"] for k in range(period)])
        else:
            args += ["-chi", repr(extra["chi"]), "-Delta", repr(extra["Delta"])]
            rec["chi"], rec["Delta"] = extra["chi"], extra["Delta"]
        args += ["-ic", ic]
        subprocess.run(args, check=True, stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        forces = np.loadtxt(os.path.join(td, "run.forces")).reshape(-1, 6)
        fin = O.load_restart(os.path.join(td, "run_final.bin"))
    np.savez_compressed(
        os.path.join(HERE, name + ".npz"),
        nx=nx, ny=ny, ngrid=ngrid, length=G["length"], xoffset=G["xoff"], yoffset=G["yoff"], geom=VARIANT_GEOM,
        Re=Re, dt=dt, nsteps=nsteps, scheme=scheme, tol=1e-7, omega0=w0,
        forces=forces, omega=fin["omega"], q=fin["q"], f=fin["f"], timestep=fin["timestep"], time=fin["time"], **rec)
    print(name, "written", forces[-1, 2:4])


if __name__ == "__main__":
    only = set(sys.argv[1:])
    for c in CASES:
        if not only or c[0] in only:
            run(c)
    for c in MOTION_CASES:
        if not only or "motion_" + c[0] in only:
            run_motion(c)
    for c in UBF_CASES:
        if not only or "ubf_" + c[0] in only:
            run_motion(c, ubf=True)
    for c in MIXED_CASES:
        if not only or c[0] in only:
            run_mixed(c)
    for c in VARIANTS:
        if not only or c[0] in only:
            run_variant(c)
