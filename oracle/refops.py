"""ctypes access to the reference's own operators (oracle/_ref/libibpm_refops.so).

TEST INFRASTRUCTURE ONLY: used by tests/ to pin the numpy restatement in
oracle/ibpm_oracle.py against the reference library built by oracle/Makefile.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_ref", "libibpm_refops.so")
_lib = None

_P = ctypes.POINTER(ctypes.c_double)


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        _lib = ctypes.CDLL(LIB_PATH)
    return _lib


def _d(a):
    return np.ascontiguousarray(a, dtype=np.float64).ctypes.data_as(_P)


def _gi(g):
    arr = (ctypes.c_int * 3)(g.nx, g.ny, g.ngrid)
    d = (ctypes.c_double * 3)(g.length, g.xoffset, g.yoffset)
    return arr, d


def _call(name, g, *arrays_in, outs):
    gi, gd = _gi(g)
    keep = [np.ascontiguousarray(a, dtype=np.float64) for a in arrays_in]
    outs = [np.zeros(s) for s in outs]
    getattr(lib(), name)(gi, gd, *[k.ctypes.data_as(_P) for k in keep], *[o.ctypes.data_as(_P) for o in outs])
    return outs[0] if len(outs) == 1 else outs


def coarsify(g, s):
    a = np.ascontiguousarray(s, dtype=np.float64).copy()
    gi, gd = _gi(g)
    lib().refops_coarsify(gi, gd, a.ctypes.data_as(_P))
    return a


def getbc_ring(g, s, lev):
    gi, gd = _gi(g)
    a = np.ascontiguousarray(s, dtype=np.float64)
    out = np.zeros(2 * (g.nx + g.ny))
    lib().refops_getbc(gi, gd, a.ctypes.data_as(_P), ctypes.c_int(lev), out.ctypes.data_as(_P))
    return out


def curl_flux(g, q):
    return _call("refops_curl_flux", g, q, outs=[g.scalar().shape])


def curl_scalar(g, s):
    return _call("refops_curl_scalar", g, s, outs=[g.flux().shape])


def laplacian(g, s):
    return _call("refops_laplacian", g, s, outs=[g.scalar().shape])


def flux_to_velocity(g, q):
    return _call("refops_flux_to_velocity", g, q, outs=[g.scalar().shape, g.scalar().shape])


def velocity_to_flux(g, u, v):
    return _call("refops_velocity_to_flux", g, u, v, outs=[g.flux().shape])


def cross_product(g, q, w):
    return _call("refops_cross_product", g, q, w, outs=[g.flux().shape])


def nonlinear(g, q, w):
    return _call("refops_nonlinear", g, q, w, outs=[g.scalar().shape])


def elliptic(g, kind, alpha, f):
    gi, gd = _gi(g)
    a = np.ascontiguousarray(f, dtype=np.float64)
    out = np.zeros(g.scalar().shape)
    lib().refops_elliptic(gi, gd, ctypes.c_int(0 if kind == "poisson" else 1), ctypes.c_double(alpha),
                          a.ctypes.data_as(_P), out.ctypes.data_as(_P))
    return out


def elliptic2d(nx, ny, dx, kind, alpha, f, ring=None):
    a = np.ascontiguousarray(f, dtype=np.float64)
    out = np.zeros((nx - 1, ny - 1))
    r = None if ring is None else np.ascontiguousarray(ring, dtype=np.float64)
    lib().refops_elliptic2d(ctypes.c_int(nx), ctypes.c_int(ny), ctypes.c_double(dx),
                            ctypes.c_int(0 if kind == "poisson" else 1), ctypes.c_double(alpha),
                            a.ctypes.data_as(_P), None if r is None else r.ctypes.data_as(_P),
                            out.ctypes.data_as(_P))
    return out


def dst2d(x):
    a = np.ascontiguousarray(x, dtype=np.float64)
    out = np.zeros_like(a)
    lib().refops_dst2d(ctypes.c_int(a.shape[0]), ctypes.c_int(a.shape[1]), a.ctypes.data_as(_P),
                       out.ctypes.data_as(_P))
    return out


def reg_toflux(g, xy, f):
    gi, gd = _gi(g)
    xy = np.ascontiguousarray(xy, dtype=np.float64)
    fa = np.ascontiguousarray(f, dtype=np.float64)
    out = np.zeros(g.flux().shape)
    lib().refops_reg_toflux(gi, gd, ctypes.c_int(xy.shape[0]), xy.ctypes.data_as(_P), fa.ctypes.data_as(_P),
                            out.ctypes.data_as(_P))
    return out


def reg_toboundary(g, xy, q):
    gi, gd = _gi(g)
    xy = np.ascontiguousarray(xy, dtype=np.float64)
    qa = np.ascontiguousarray(q, dtype=np.float64)
    out = np.zeros(2 * xy.shape[0])
    lib().refops_reg_toboundary(gi, gd, ctypes.c_int(xy.shape[0]), xy.ctypes.data_as(_P), qa.ctypes.data_as(_P),
                                out.ctypes.data_as(_P))
    return out


def projection(g, xy, Re, beta, a, b, f0, use_cg=False, tol=1e-7):
    gi, gd = _gi(g)
    xy = np.ascontiguousarray(xy, dtype=np.float64)
    aa = np.ascontiguousarray(a, dtype=np.float64)
    bb = np.ascontiguousarray(b, dtype=np.float64)
    f = np.ascontiguousarray(f0, dtype=np.float64).copy()
    w = np.zeros(g.scalar().shape)
    lib().refops_projection(gi, gd, ctypes.c_int(xy.shape[0]), xy.ctypes.data_as(_P), ctypes.c_double(Re),
                            ctypes.c_double(beta), ctypes.c_int(1 if use_cg else 0), ctypes.c_double(tol),
                            aa.ctypes.data_as(_P), bb.ctypes.data_as(_P), w.ctypes.data_as(_P),
                            f.ctypes.data_as(_P))
    return w, f


def apply_m(g, xy, Re, beta, f):
    gi, gd = _gi(g)
    xy = np.ascontiguousarray(xy, dtype=np.float64)
    fa = np.ascontiguousarray(f, dtype=np.float64)
    out = np.zeros(2 * xy.shape[0])
    lib().refops_apply_m(gi, gd, ctypes.c_int(xy.shape[0]), xy.ctypes.data_as(_P), ctypes.c_double(Re),
                         ctypes.c_double(beta), fa.ctypes.data_as(_P), out.ctypes.data_as(_P))
    return out


def inner_product(g, kind, a, b):
    """kind 0 InnerProduct(Scalar), 1 FineGridInnerProduct(Scalar), 2 InnerProduct(Flux), 3 FineGrid(Flux)."""
    gi, gd = _gi(g)
    out = np.zeros(1)
    lib().refops_inner_product(gi, gd, ctypes.c_int(kind), _d(a), _d(b), out.ctypes.data_as(_P))
    return float(out[0])
