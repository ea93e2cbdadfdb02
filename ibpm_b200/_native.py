"""ctypes binding of libibpm_b200.so (the C ABI in include/ibpm_b200.h).

The library is built in-tree (``python -m ibpm_b200.build``).  Loading fails
loudly when it is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libibpm_b200.so")

c_double_p = ctypes.POINTER(ctypes.c_double)


class ibg_grid(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("ngrid", ctypes.c_int),
                ("length", ctypes.c_double), ("xoffset", ctypes.c_double), ("yoffset", ctypes.c_double)]


class ibg_body(ctypes.Structure):
    _fields_ = [("npoints", ctypes.c_int), ("xy", c_double_p), ("xcenter", ctypes.c_double),
                ("ycenter", ctypes.c_double), ("motion", ctypes.c_int), ("params", ctypes.c_double * 12),
                ("table_rows", ctypes.c_int), ("table", c_double_p)]


class ibg_params(ctypes.Structure):
    _fields_ = [("Re", ctypes.c_double), ("dt", ctypes.c_double), ("scheme", ctypes.c_int),
                ("cg_tol", ctypes.c_double), ("cg_max_iter", ctypes.c_int), ("u_mag", ctypes.c_double),
                ("alpha", ctypes.c_double), ("precision", ctypes.c_int), ("device", ctypes.c_int),
                ("cg_precond", ctypes.c_int), ("pc_refresh", ctypes.c_int), ("cg_graph", ctypes.c_int),
                ("pc_fallback_iter", ctypes.c_int)]


SCHEMES = {"euler": 0, "ab2": 1, "rk3": 2, "rk3b": 3}
PRECISIONS = {"fp64": 0, "fp32_refined": 1, "fp32": 2}
PRECONDS = {"none": 0, "cholesky": 1, "learned": 2}

# every entry point declared in include/ibpm_b200.h: name -> (restype, argtypes)
_VP = ctypes.c_void_p
_I = ctypes.c_int
_D = ctypes.c_double
SIGNATURES = {
    "ibg_create": (_I, [ctypes.POINTER(ibg_grid), _I, ctypes.POINTER(ibg_body), ctypes.POINTER(ibg_params), _VP,
                        ctypes.POINTER(_VP)]),
    "ibg_destroy": (_I, [_VP]),
    "ibg_last_error": (ctypes.c_char_p, [_VP]),
    "ibg_init": (_I, [_VP]),
    "ibg_save": (_I, [_VP, ctypes.c_char_p]),
    "ibg_load": (_I, [_VP, ctypes.c_char_p]),
    "ibg_set_state": (_I, [_VP, _VP, _VP, _VP, _I, _D]),
    "ibg_get_state": (_I, [_VP, _VP, _VP, _VP, ctypes.POINTER(_I), ctypes.POINTER(_D)]),
    "ibg_get_boundary_force": (_I, [_VP, _VP, ctypes.POINTER(_I), ctypes.POINTER(_D)]),
    "ibg_update_operators": (_I, [_VP, _D]),
    "ibg_get_boundary": (_I, [_VP, _VP, _VP]),
    "ibg_flux_to_velocity": (_I, [_VP, _VP, _VP]),
    "ibg_set_moving_frame": (_I, [_VP]),
    "ibg_refresh_state": (_I, [_VP]),
    "ibg_advance": (_I, [_VP, _I]),
    "ibg_get_net_force": (_I, [_VP, ctypes.POINTER(_D), ctypes.POINTER(_D)]),
    "ibg_get_force_history": (_I, [_VP, _I, _VP]),
    "ibg_sizes": (_I, [_VP, ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_longlong),
                       ctypes.POINTER(_I)]),
    "ibg_cg_stats": (_I, [_VP, ctypes.POINTER(_I), ctypes.POINTER(_I), ctypes.POINTER(_I)]),
    "ibg_cg_totals": (_I, [_VP, ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_longlong)]),
    "ibg_stream": (_VP, [_VP]),
    "ibg_last_launch_count": (ctypes.c_longlong, [_VP]),
    "ibg_run_kernel": (ctypes.c_longlong, [_VP, _I, _I]),
    "ibg_lpc_set_tensor_cores": (_I, [_VP, _I]),
    "ibg_lpc_status": (_I, [_VP]),
    "ibg_set_dst_gemm": (_I, [_VP, _I]),
    "ibg_dst_form_log": (_I, [_VP, _I]),
    "ibg_dst_gemm_status": (_I, [_VP]),
    "ibg_solve_fp32": (_I, [_VP, _I, _VP, _VP]),
    "ibg_graph_kernel_nodes": (ctypes.c_longlong, [_VP]),
    "ibg_graph_launch_claim": (ctypes.c_longlong, [_VP]),
    "ibg_ensemble_kernel_nodes": (ctypes.c_longlong, [_VP]),
    "ibg_set_sweep_form": (_I, [_VP, _I]),
    "ibg_sweep_form_log": (_I, [_VP, _I]),
    "ibg_pass_form_log": (_I, [_VP, _I]),
    "ibg_set_pass_form": (_I, [_VP, _I]),
    "ibg_autotune_log": (_I, [_VP, _I]),
    "ibg_set_linearized": (_I, [_VP, _I, _VP, _VP]),
    "ibg_set_sfd": (_I, [_VP, _D, _D, _VP]),
    "ibg_set_adjoint": (_I, [_VP, _VP, _VP]),
    "ibg_inner_product": (_I, [_VP, _I, _VP, _VP, _VP]),
    "ibg_energy": (_I, [_VP, _VP]),
    "ibg_get_sfd_state": (_I, [_VP, _VP]),
    "ibg_ensemble_set_shapes": (_I, [_VP, _I, _I, _I]),
    "ibg_save_restart": (_I, [_VP, ctypes.c_char_p]),
    "ibg_load_restart": (_I, [_VP, ctypes.c_char_p]),
    "ibg_snapshot": (_I, [_VP]),
    "ibg_snapshot_save": (_I, [_VP, ctypes.c_char_p]),
    "ibg_lpc_num_params": (ctypes.c_size_t, []),
    "ibg_lpc_generate": (_I, [_VP, _I, _D, _D, _VP, _VP]),
    "ibg_lpc_train": (_I, [_VP, _I, _VP, _VP, _I, _I, ctypes.c_float, ctypes.c_uint, _VP]),
    "ibg_lpc_loss_grad": (_I, [_VP, _I, _VP, _VP, _VP, _VP, _VP]),
    "ibg_lpc_get_params": (_I, [_VP, _VP, ctypes.c_size_t]),
    "ibg_lpc_set_params": (_I, [_VP, _VP, ctypes.c_size_t]),
    "ibg_lpc_apply": (_I, [_VP, _I, _VP, _VP, _VP]),
    "ibg_substep_beta": (_I, [_VP, _I, _VP]),
    "ibg_poisson_solve": (_I, [_VP, _VP, _VP]),
    "ibg_helmholtz_solve": (_I, [_VP, _D, _VP, _VP]),
    "ibg_nonlinear": (_I, [_VP, _VP, _VP, _VP]),
    "ibg_laplacian": (_I, [_VP, _VP, _VP]),
    "ibg_model_B": (_I, [_VP, _VP, _VP]),
    "ibg_model_C": (_I, [_VP, _VP, _VP]),
    "ibg_reg_to_boundary": (_I, [_VP, _VP, _VP]),
    "ibg_reg_to_flux": (_I, [_VP, _VP, _VP]),
    "ibg_elliptic_create": (_I, [ctypes.POINTER(ibg_grid), _I, ctypes.c_double, _VP, _VP]),
    "ibg_elliptic_solve": (_I, [_VP, _VP, _VP]),
    "ibg_elliptic_destroy": (_I, [_VP]),
    "ibg_elliptic_last_error": (ctypes.c_char_p, [_VP]),
    "ibg_set_external_kinematics": (_I, [_VP]),
    "ibg_set_step_kinematics": (_I, [_VP, _I, _VP, _VP]),
    "ibg_projection_solve": (_I, [_VP, _I, _VP, _VP, _VP, _VP]),
    "ibg_poisson_solve_static": (_I, [ctypes.POINTER(ibg_grid), _VP, _VP, _VP]),
    "ibg_ensemble_create": (_I, [_I, ctypes.POINTER(_VP), ctypes.POINTER(_VP)]),
    "ibg_ensemble_advance": (_I, [_VP, _I]),
    "ibg_ensemble_destroy": (_I, [_VP]),
    "ibg_ensemble_stream": (_VP, [_VP]),
    "ibg_ensemble_launches_per_step": (ctypes.c_longlong, [_VP]),
    "ibg_ensemble_advance_host": (_I, [_VP, _I, _VP, _VP, _VP]),
    "ibg_ensemble_autotune": (_I, [_VP, _I, _VP, _I]),
    "ibg_ensemble_host_launches_per_step": (ctypes.c_longlong, [_VP]),
    "ibg_ensemble_last_error": (ctypes.c_char_p, [_VP]),
    "ibg_static_last_error": (ctypes.c_char_p, []),
}

_lib = None


def lib():
    """Load the library (raises OSError if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise OSError(f"{LIB_PATH} is missing: build it with `python -m ibpm_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


class IbgError(RuntimeError):
    pass


def check(status: int, ctx=None) -> int:
    if status < 0:
        msg = lib().ibg_last_error(ctx)
        raise IbgError(f"ibg status {status}: {msg.decode() if msg else ''}")
    return status
