"""Tecplot output of the IBPM state (the reference's OutputTecplot).

The node velocities come from the device (``ibg_flux_to_velocity``,
FluxToVelocity of the device state); this module only formats the ASCII
file the way src/ScalarToTecplot.cc:36-78 writes it: x, y, u, v and the
vorticity at every interior node of one level, j outer and i inner, each
value as ``%.5e``.  ``OutputTecplot`` mirrors src/OutputTecplot.cc:24-69
(file name and title patterns formatted with the timestep, and with the
level when every grid is written).
"""
from __future__ import annotations

import numpy as np


def write(filename: str, title: str, grid, u: np.ndarray, v: np.ndarray, omega: np.ndarray, lev: int = 0) -> bool:
    """ScalarToTecplot({u, v, omega}, {"u", "v", "Vorticity"}, filename, title, lev)
    (src/ScalarToTecplot.cc:80-121); u, v, omega in the Scalar layout (ngrid, nx-1, ny-1)."""
    nx, ny = grid.nx, grid.ny
    if not 0 <= lev < grid.ngrid:
        raise ValueError("level out of range")
    dx = grid.length / nx * (1 << lev)
    # Grid::getXEdge / getYEdge with zero shift (src/Grid.cc:104-139)
    x0 = grid.xoffset + 0.5 * (0.0 - 1) * ((1 << lev) - 1) * (nx * (grid.length / nx))
    y0 = grid.yoffset + 0.5 * (0.0 - 1) * ((1 << lev) - 1) * (ny * (grid.length / nx))
    xs = x0 + np.arange(1, nx) * dx
    ys = y0 + np.arange(1, ny) * dx
    cols = [np.broadcast_to(xs[:, None], (nx - 1, ny - 1)), np.broadcast_to(ys[None, :], (nx - 1, ny - 1)),
            np.asarray(u)[lev], np.asarray(v)[lev], np.asarray(omega)[lev]]
    # rows in the reference's order: j outer, i inner
    data = np.stack([c.T.reshape(-1) for c in cols], axis=1)
    try:
        with open(filename, "w") as fh:
            fh.write('TITLE = "%s"\n' % title)
            fh.write('VARIABLES = "x" "y" "u" "v" "Vorticity" \n')
            fh.write('ZONE T="Rectangular zone"\n')
            fh.write("I=%d, J=%d, K=1, ZONETYPE=Ordered\n" % (nx - 1, ny - 1))
            fh.write("DATAPACKING=POINT\n")
            fh.write("DT=(SINGLE SINGLE SINGLE SINGLE SINGLE )\n")
            fh.writelines("".join("%.5e " % val for val in row) + "\n" for row in data)
    except OSError:
        return False
    return True


class OutputTecplot:
    """OutputTecplot(filename, title, all_grids) (src/OutputTecplot.cc:24-69): ``filename`` and
    ``title`` are printf patterns of the timestep (and, with all_grids, of the level)."""

    def __init__(self, filename: str, title: str, all_grids: bool = False):
        self.filename, self.title, self.all_grids = filename, title, all_grids

    def do_output(self, solver, x) -> bool:
        """Write the state x; its velocities are computed on the device from the solver's state."""
        u, v = solver.flux_to_velocity()
        title = self.title % x.timestep if "%" in self.title else self.title
        if not self.all_grids:
            return write(self.filename % x.timestep, title, solver.grid, u, v, x.omega, 0)
        ok = True
        for lev in range(solver.grid.ngrid):
            ok = write(self.filename % (x.timestep, lev), title, solver.grid, u, v, x.omega, lev) and ok
        return ok
