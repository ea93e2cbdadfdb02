"""Tecplot output of the state (the reference's OutputTecplot with every level).

CPU: the writer, fed the oracle's FluxToVelocity of a fixture's final state,
reproduces the files the reference wrote for that state token for token,
wherever the reference's values are defined (it leaves the coarse-level
interior overlap of u and v uninitialised).

GPU: ``ibg_flux_to_velocity`` of the device state against the oracle, and
the files written from it against the reference's to their 5 printed digits.
"""
import numpy as np
import pytest

from helpers import load_golden

CASE = "cyl_l3_noise_rk3"


def _grid_and_velocities(d):
    from oracle import ibpm_oracle as O
    g = O.Grid(int(d["nx"]), int(d["ny"]), int(d["ngrid"]), float(d["length"]), float(d["xoffset"]),
               float(d["yoffset"]))
    q = np.asarray(d["q"])
    u = O.flux_to_xvel(g, q)   # Scalar layout, NaN where the reference leaves u undefined
    v = O.flux_to_yvel(g, q)
    return g, u, v


def _rows(text):
    lines = text.splitlines()
    return lines[:6], [ln.split() for ln in lines[6:]]


def _defined(u, v, lev):
    """per written row (j outer, i inner): whether the reference's u and v are defined there"""
    return (np.isfinite(u[lev]) & np.isfinite(v[lev])).T.reshape(-1)


def test_writer_reproduces_reference_files(tmp_path):
    from ibpm_b200 import tecplot
    d = load_golden(CASE)
    g, u, v = _grid_and_velocities(d)
    n = int(d["nsteps"])
    for lev, ref in enumerate(d["tecplot_texts"]):
        fn = str(tmp_path / ("tec%05d_g%01d.plt" % (n, lev)))
        assert tecplot.write(fn, "Test run, step%05d" % n, g, np.nan_to_num(u), np.nan_to_num(v), d["omega"], lev)
        head, rows = _rows(open(fn).read())
        rhead, rrows = _rows(str(ref))
        assert head == rhead
        assert len(rows) == len(rrows) == (g.nx - 1) * (g.ny - 1)
        ok = _defined(u, v, lev)
        assert ok.sum() == len(rows) if lev == 0 else 0 < ok.sum() < len(rows)
        for k in np.flatnonzero(ok):
            assert rows[k] == rrows[k], (lev, k)
        # x, y and the vorticity are defined everywhere
        for k in np.flatnonzero(~ok):
            assert [rows[k][c] for c in (0, 1, 4)] == [rrows[k][c] for c in (0, 1, 4)], (lev, k)


@pytest.mark.gpu
def test_device_velocities_and_files_match_reference(tmp_path):
    import ibpm_b200 as ib
    from ibpm_b200 import tecplot
    d = load_golden(CASE)
    _, u_o, v_o = _grid_and_velocities(d)
    grid = ib.Grid(int(d["nx"]), int(d["ny"]), int(d["ngrid"]), float(d["length"]), float(d["xoffset"]),
                   float(d["yoffset"]))
    geo = ib.geometry.parse(str(d["geom"]))
    s = ib.NonlinearIBSolver(grid, ib.NavierStokesModel(grid, geo, float(d["Re"])), float(d["dt"]))
    n = int(d["nsteps"])
    x = ib.State(grid, geo.num_points, omega=np.array(d["omega"], dtype=float))
    x.q[...] = np.asarray(d["q"]).reshape(x.q.shape)
    x.timestep = n
    s.set_state(x)
    u, v = s.flux_to_velocity()
    ok = np.isfinite(u_o) & np.isfinite(v_o)
    scale = np.max(np.abs(u_o[ok]))
    assert np.max(np.abs(u[ok] - u_o[ok])) < 1e-13 * scale
    assert np.max(np.abs(v[ok] - v_o[ok])) < 1e-13 * scale
    assert not np.any(u[~ok]) and not np.any(v[~ok])
    out = tecplot.OutputTecplot(str(tmp_path / "tec%05d_g%01d.plt"), "Test run, step%05d", all_grids=True)
    assert out.do_output(s, x)
    for lev, ref in enumerate(d["tecplot_texts"]):
        head, rows = _rows(open(str(tmp_path / ("tec%05d_g%01d.plt" % (n, lev)))).read())
        rhead, rrows = _rows(str(ref))
        assert head == rhead
        a = np.array(rows, dtype=float)
        b = np.array(rrows, dtype=float)
        keep = _defined(u_o, v_o, lev)
        assert np.allclose(a[keep], b[keep], rtol=2e-5, atol=1e-5 * scale)
    s.close()
