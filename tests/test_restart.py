"""Restart files (State::save / State::load, src/State.cc:65-223).

CPU: the oracle's reader parses a restart file the reference itself wrote.
GPU: a restart file written from the device holds exactly the device state in
the reference's layout; loading one continues a run exactly; an asynchronous
snapshot holds the state of the step it was taken at while later steps run.
"""
import os
import subprocess

import numpy as np
import pytest

from helpers import FP64_TOL, load_golden, rel_l2
from oracle import ibpm_oracle as O

CASE = "cyl_l3_noise_rk3"


def _case(name=CASE):
    import ibpm_b200 as ib
    d = load_golden(name)
    grid = ib.Grid(int(d["nx"]), int(d["ny"]), int(d["ngrid"]), float(d["length"]), float(d["xoffset"]),
                   float(d["yoffset"]))
    geo = ib.geometry.parse(str(d["geom"]))
    return ib, d, grid, geo


def _solver(ib, d, grid, geo):
    s = ib.NonlinearIBSolver(grid, ib.NavierStokesModel(grid, geo, float(d["Re"])), float(d["dt"]),
                             str(d["scheme"]), float(d["tol"]))
    s.init()
    return s


def test_oracle_reads_a_restart_file_the_reference_wrote(tmp_path):
    from oracle import ref_runner
    drv = os.path.join(os.path.dirname(ref_runner.DRIVER), "ref_driver_parity")
    if not os.path.exists(drv):
        pytest.skip("oracle/_ref not built (needs the reference sources)")
    d = load_golden(CASE)
    gpath = tmp_path / "body.geom"
    gpath.write_text(str(d["geom"]))
    out = str(tmp_path / "run")
    subprocess.run([drv, "-nx", str(d["nx"]), "-ny", str(d["ny"]), "-ngrid", str(d["ngrid"]),
                    "-length", repr(float(d["length"])), "-xoffset", repr(float(d["xoffset"])),
                    "-yoffset", repr(float(d["yoffset"])), "-geom", str(gpath), "-Re", repr(float(d["Re"])),
                    "-dt", repr(float(d["dt"])), "-scheme", str(d["scheme"]), "-nsteps", "2", "-out", out],
                   check=True, capture_output=True, timeout=600)
    r = O.load_restart(out + "_final.bin")
    nx, ny, L = int(d["nx"]), int(d["ny"]), int(d["ngrid"])
    assert (r["nx"], r["ny"], r["ngrid"], r["timestep"]) == (nx, ny, L, 2)
    assert r["time"] == pytest.approx(2 * float(d["dt"]))
    size = 40 + 8 * L * (2 * nx * ny + nx + ny) + 8 * L * (nx - 1) * (ny - 1) + 16 * r["npts"] + 12
    assert os.path.getsize(out + "_final.bin") == size
    assert np.isfinite(r["omega"]).all() and np.abs(r["f"]).max() > 0


@pytest.mark.gpu
def test_gpu_restart_file_holds_the_device_state(tmp_path):
    ib, d, grid, geo = _case()
    s = _solver(ib, d, grid, geo)
    x = ib.State(grid, geo.num_points, omega=np.array(d["omega0"], dtype=float))
    s.set_state(x, with_q=False)
    n = int(d["nsteps"])
    s.advance_resident(n)
    path = str(tmp_path / "gpu.bin")
    assert s.save_restart(path)
    r = O.load_restart(path)
    s.get_state(x)
    assert (r["nx"], r["ny"], r["ngrid"], r["npts"]) == (grid.nx, grid.ny, grid.ngrid, geo.num_points)
    assert (r["dx"], r["x0"], r["y0"]) == (grid.dx, grid.xoffset, grid.yoffset)
    assert r["timestep"] == x.timestep == n and r["time"] == x.time
    assert np.array_equal(r["omega"].ravel(), np.asarray(x.omega).ravel())
    assert np.array_equal(r["q"].ravel(), np.asarray(x.q).ravel())
    assert np.array_equal(r["f"], np.asarray(x.f))
    assert rel_l2(r["omega"], d["omega"]) < FP64_TOL
    s.close()


@pytest.mark.gpu
def test_gpu_load_restart_continues_the_run(tmp_path):
    ib, d, grid, geo = _case()
    n = int(d["nsteps"])
    a = _solver(ib, d, grid, geo)
    a.set_state(ib.State(grid, geo.num_points, omega=np.array(d["omega0"], dtype=float)), with_q=False)
    a.advance_resident(2)
    path = str(tmp_path / "mid.bin")
    assert a.save_restart(path)
    a.advance_resident(n - 2)
    fa = a.force_history(n - 2)
    b = _solver(ib, d, grid, geo)
    assert b.load_restart(path)
    b.advance_resident(n - 2)
    # the atomic smear makes the FP64 step reproducible to ~1 ulp, not bit for bit, from run to run
    assert rel_l2(b.force_history(n - 2), fa) < 1e-12
    xa, xb = ib.State(grid, geo.num_points), ib.State(grid, geo.num_points)
    a.get_state(xa)
    b.get_state(xb)
    assert rel_l2(xb.omega, xa.omega) < 1e-12 and xa.timestep == xb.timestep == n
    assert rel_l2(xb.omega, d["omega"]) < FP64_TOL
    # a file of another grid is refused, not resized
    other = ib.Grid(grid.nx + 2, grid.ny, grid.ngrid, grid.length, grid.xoffset, grid.yoffset)
    c = ib.NonlinearIBSolver(other, ib.NavierStokesModel(other, geo, float(d["Re"])), float(d["dt"]),
                             str(d["scheme"]))
    with pytest.raises(ib.IbgError):
        c.load_restart(path)
    assert c.load_restart(str(tmp_path / "missing.bin")) is False
    for s in (a, b, c):
        s.close()


@pytest.mark.gpu
def test_gpu_snapshot_keeps_the_step_it_was_taken_at(tmp_path):
    ib, d, grid, geo = _case()
    a = _solver(ib, d, grid, geo)
    b = _solver(ib, d, grid, geo)
    for s in (a, b):
        s.set_state(ib.State(grid, geo.num_points, omega=np.array(d["omega0"], dtype=float)), with_q=False)
    a.advance_resident(2)
    a.snapshot()
    a.advance_resident(3)           # runs while the snapshot travels to the host
    a.snapshot()                    # a second snapshot waits for the first's copy, then replaces it
    a.advance_resident(1)
    path = str(tmp_path / "snap.bin")
    assert a.snapshot_save(path)
    b.advance_resident(5)
    r = O.load_restart(path)
    xb = ib.State(grid, geo.num_points)
    b.get_state(xb)
    assert r["timestep"] == 5
    assert rel_l2(r["omega"].ravel(), np.asarray(xb.omega).ravel()) < 1e-12
    assert rel_l2(r["f"], xb.f) < 1e-12
    a.close()
    b.close()
