"""The reference's own `ibpm` CLI (src/ibpm.cc, unmodified) linked with the
drop-in classes (ibpm_b200/dropin/ibpm_gpu.cc -> libibpm_b200.so) against the
same CLI linked with the reference's solver objects (oracle/_ref/ibpm, built
by oracle/Makefile).  Both write the CLI's .force file (%.5e) and restart
files (full precision); the drop-in's must agree.

Bars: forces to the printed precision; the final state to 1e-10 (relative L2)
for fixed bodies; for a moving body both CLIs run CG at the CLI's fixed
tolerance 1e-7 (absolute, on |r|), so their states agree to that tolerance:
1e-6 relative.
"""
import os
import subprocess

import numpy as np
import pytest

from helpers import ROOT, rel_l2

pytestmark = pytest.mark.gpu

DROPIN = os.path.join(ROOT, "ibpm_b200", "dropin", "_build", "ibpm_gpu")
REFCLI = os.path.join(ROOT, "oracle", "_ref", "ibpm")


def _run(exe, td, geom, args, ic=None):
    os.makedirs(td, exist_ok=True)
    gpath = os.path.join(td, "body.geom")
    with open(gpath, "w") as fh:
        fh.write(geom)
    cmd = [exe, "-geom", gpath, "-outdir", td + "/", "-name", "run", "-tecplot", "0", "-energy", "0",
           "-force", "1"] + [str(a) for a in args]
    if ic:
        cmd += ["-ic", ic]
    p = subprocess.run(cmd, cwd=td, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stdout[-2000:] + p.stderr[-2000:]
    return np.loadtxt(os.path.join(td, "run.force")).reshape(-1, 4), p


CASES = {
    # name: (geometry, CLI arguments, seeded initial vorticity (amp, seed) or None)
    "cylinder_48x48_rk3": ("cylinder", ["-nx", 48, "-ny", 48, "-ngrid", 1, "-length", 4.0, "-xoffset", -2.0,
                                        "-yoffset", -2.0, "-Re", 100.0, "-dt", 0.02, "-nsteps", 8, "-scheme",
                                        "rk3", "-restart", 8], None),
    "cylinder_64x32x3_noise_ab2": ("cylinder", ["-nx", 64, "-ny", 32, "-ngrid", 3, "-length", 4.0, "-xoffset",
                                                -1.5, "-yoffset", -1.0, "-Re", 200.0, "-dt", 0.01, "-nsteps", 6,
                                                "-scheme", "ab2", "-restart", 6], (1e-3, 7)),
    "plate_64x32x2_pitchplunge_rk3": ("plate", ["-nx", 64, "-ny", 32, "-ngrid", 2, "-length", 4.0, "-xoffset",
                                                -2.0, "-yoffset", -1.0, "-Re", 300.0, "-dt", 0.01, "-nsteps", 6,
                                                "-scheme", "rk3", "-restart", 6], None),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_dropin_cli_matches_reference_cli(name, tmp_path):
    if not (os.path.exists(DROPIN) and os.path.exists(REFCLI)):
        pytest.skip("drop-in CLI or reference CLI not built (make -C ibpm_b200/dropin; make -C oracle)")
    from ibpm_b200 import configs, geometry
    from oracle import ibpm_oracle as O
    kind, args, noise = CASES[name]
    geom = configs.cylinder_geom(32, r=0.4) if kind == "cylinder" else configs.plate_geom(npts=17, freq=0.5)
    a = dict(zip(args[0::2], args[1::2]))
    nx, ny, L = a["-nx"], a["-ny"], a["-ngrid"]
    ic = None
    if noise is not None:
        wl = configs.Workload(name, nx, ny, L, a["-length"], a["-xoffset"], a["-yoffset"], geom, a["-Re"], a["-dt"],
                              a["-nsteps"], noise_amp=noise[0], noise_seed=noise[1],
                              noise_box=(0.0, 1e9, -0.8, 0.8))
        g = O.Grid(nx, ny, L, a["-length"], a["-xoffset"], a["-yoffset"])
        ic = str(tmp_path / "ic.bin")
        O.save_restart(ic, O.State(g, geometry.parse(geom).num_points, omega=wl.initial_vorticity()), g)
    f_gpu, p = _run(DROPIN, str(tmp_path / "gpu"), geom, args, ic)
    f_ref, _ = _run(REFCLI, str(tmp_path / "ref"), geom, args, ic)
    assert "(GPU)" in p.stderr  # the drop-in's solver ran
    n = a["-nsteps"]
    assert f_gpu.shape == f_ref.shape == (n + 1, 4)  # the initial line and one per step
    # forces to the %.5e the CLI prints (half a unit in the 6th digit, relative to the largest)
    scale = np.abs(f_ref[:, 2:]).max()
    assert np.abs(f_gpu[:, 2:] - f_ref[:, 2:]).max() <= 1e-5 * scale
    assert np.array_equal(f_gpu[:, 0], f_ref[:, 0])
    # the restart files of the last step, at full precision
    sg = O.load_restart(str(tmp_path / "gpu" / ("run%05d.bin" % n)))
    sr = O.load_restart(str(tmp_path / "ref" / ("run%05d.bin" % n)))
    tol = 1e-6 if kind == "plate" else 1e-10
    assert rel_l2(sg["omega"], sr["omega"]) < tol
    assert rel_l2(sg["q"], sr["q"]) < tol
    assert rel_l2(sg["f"], sr["f"]) < 10 * tol
    assert sg["timestep"] == sr["timestep"] == n
