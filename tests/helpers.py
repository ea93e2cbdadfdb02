"""Shared test helpers: golden fixtures, oracle construction, tolerances."""
import glob
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN_DIR = os.path.join(ROOT, "tests", "golden")

# FP64 parity bar against the reference (relative L2 / relative max for forces)
FP64_TOL = 1e-10


def golden_names():
    """Fixtures of the nonlinear solver (NonlinearIBSolver)."""
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN_DIR, "*.npz"))
                  if not os.path.basename(p).startswith(("var_", "full_")))


def variant_names():
    """Fixtures of the other N(x) forms: linearized, linearized-periodic, SFD."""
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN_DIR, "var_*.npz")))


def load_golden(name):
    z = np.load(os.path.join(GOLDEN_DIR, name + ".npz"), allow_pickle=False)
    return {k: (z[k].item() if z[k].ndim == 0 else z[k]) for k in z.files}


def golden_geometry(d):
    """The fixture's geometry, with the files its `motion` lines name (motion
    files) written beside it first, as the reference reads them."""
    import tempfile
    from ibpm_b200 import geometry
    if "file_names" not in d:
        return geometry.parse(str(d["geom"]))
    with tempfile.TemporaryDirectory() as td:
        for name, text in zip(np.atleast_1d(d["file_names"]), np.atleast_1d(d["file_texts"])):
            with open(os.path.join(td, str(name)), "w") as fh:
                fh.write(str(text))
        return geometry.parse(str(d["geom"]), td)


def oracle_from_golden(d):
    from oracle import ibpm_oracle as O
    from ibpm_b200 import geometry
    g = O.Grid(int(d["nx"]), int(d["ny"]), int(d["ngrid"]), float(d["length"]), float(d["xoffset"]),
               float(d["yoffset"]))
    geo = golden_geometry(d)
    bodies = []
    for b in geo.bodies:
        motion = geometry.MOTION_NAMES[b.motion]
        bodies.append(O.Body(np.array(b.points, dtype=float), tuple(b.center), motion, tuple(b.params), b.table))
    model = O.Model(g, bodies, float(d["Re"]))
    if int(d.get("ubf", 0)):
        model.moving_frame()
    solver = O.IBSolver(model, float(d["dt"]), str(d["scheme"]), float(d["tol"]))
    x = O.State(g, model.npts, omega=np.array(d["omega0"], dtype=float))
    return g, model, solver, x


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def oracle_from_variant(d):
    """Oracle solver and initial state for a fixture of tests/golden/var_*.npz."""
    from oracle import ibpm_oracle as O
    from ibpm_b200 import geometry
    g = O.Grid(int(d["nx"]), int(d["ny"]), int(d["ngrid"]), float(d["length"]), float(d["xoffset"]),
               float(d["yoffset"]))
    geo = geometry.parse(str(d["geom"]))
    bodies = [O.Body(np.array(b.points, dtype=float)) for b in geo.bodies]
    model_name = str(d["model"])
    linear = model_name in ("linear", "linearperiodic", "adjoint")
    # the linear models run without the uniform base flow, as the reference CLI builds them
    model = O.Model(g, bodies, float(d["Re"]), u_mag=0.0 if linear else 1.0)
    base = sfd = None
    if linear:
        base = [(np.array(d["base_omega"][k]), np.array(d["base_q"][k])) for k in range(int(d["period"]))]
    else:
        sfd = (float(d["chi"]), float(d["Delta"]), g.scalar())
    adj = model_name == "adjoint"
    solver = O.IBSolver(model, float(d["dt"]), str(d["scheme"]), float(d["tol"]), base=base, sfd=sfd, adjoint=adj)
    x = O.State(g, model.npts, omega=np.array(d["omega0"], dtype=float))
    return g, model, solver, x
