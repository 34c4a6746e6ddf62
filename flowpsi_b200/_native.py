"""ctypes binding of ``libfpsi.so`` (the C ABI declared in ``include/fpsi.h``).

The structures below mirror the C declarations field by field.  Loading fails
loudly when the shared object is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "libfpsi.so"

FPSI_OK = 0
ERRORS = {
    -1: "FPSI_E_INVALID", -2: "FPSI_E_CUDA", -3: "FPSI_E_NOMEM", -4: "FPSI_E_UNSUPPORTED",
    -5: "FPSI_E_SINGULAR", -6: "FPSI_E_NAN", -7: "FPSI_E_TIMEOUT", -8: "FPSI_E_STATE",
}

FLUX = {"hllc": 0, "roe": 1, "hlle": 2, "kec": 3, "ssf": 4}
LIMITER = {"venkatakrishnan": 0, "barth": 1, "none": 2, "zero": 3}
SOLVER = {"sgs": 0, "lsgs": 1, "fsgs": 2}
PRECISION = {"fp64": 0, "ref": 1, "mixed": 2}
BC = {"farfield": 1, "supersonicInflow": 2, "supersonicOutflow": 3, "extrapolate": 4,
      "reflecting": 5, "viscousWall": 6, "outflow": 7, "outflowMean": 8,
      "isentropicInflow": 9, "fixedMass": 10, "fixedMassOutflow": 11, "inflow": 12}


class Params(C.Structure):
    _fields_ = [
        ("gamma", C.c_double), ("Rtilde", C.c_double), ("Pambient", C.c_double),
        ("Minf", C.c_double), ("flux", C.c_int32), ("limiter", C.c_int32),
        ("Kl", C.c_double), ("urelax", C.c_double), ("dtmax", C.c_double),
        ("cflmax", C.c_double), ("solver", C.c_int32), ("gauss_seidel_iter", C.c_int32),
        ("lsgs_relaxation", C.c_double), ("lsgs_abs_tol", C.c_double),
        ("lsgs_rel_tol", C.c_double), ("lsgs_max_iter", C.c_int32),
        ("precision", C.c_int32), ("viscous", C.c_int32), ("turbulence", C.c_int32),
        ("Prt", C.c_double), ("mu_a1", C.c_double), ("mu_a2", C.c_double),
        ("mu_a3", C.c_double), ("k_a1", C.c_double), ("k_a2", C.c_double),
        ("k_a3", C.c_double), ("time_accurate", C.c_int32), ("newton_iters", C.c_int32),
        ("lds_comp_factor", C.c_double), ("lds_dissipation_limit", C.c_double),
        ("lds_ducros_factor", C.c_double), ("lds_use_upwind", C.c_double),
        ("lds_nonsym_coeff", C.c_double), ("lds_nonsym_factor", C.c_double),
        ("lds_miles_filter", C.c_double), ("ssf_coeff", C.c_double),
        ("step_graphs", C.c_int32), ("reserved2", C.c_int32),
    ]


class BCSpec(C.Structure):
    _fields_ = [("kind", C.c_int32), ("reserved", C.c_int32), ("T", C.c_double),
                ("pg", C.c_double), ("u", C.c_double * 3), ("nu_t", C.c_double),
                ("mass_flux", C.c_double), ("mdot", C.c_double), ("mass_relax", C.c_double)]


class Mesh(C.Structure):
    _fields_ = [
        ("nnodes", C.c_int64), ("ncells", C.c_int64), ("nfaces", C.c_int64),
        ("xyz", C.POINTER(C.c_double)), ("face_off", C.POINTER(C.c_int64)),
        ("face_nodes", C.POINTER(C.c_int32)), ("cl", C.POINTER(C.c_int32)),
        ("cr", C.POINTER(C.c_int32)), ("pshift", C.POINTER(C.c_double)),
        ("nbc", C.c_int32), ("reserved", C.c_int32), ("bcs", C.POINTER(BCSpec)),
    ]


class MeshSpec(C.Structure):
    _fields_ = [
        ("kind", C.c_int32), ("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32),
        ("Lx", C.c_double), ("Ly", C.c_double), ("Lz", C.c_double), ("jitter", C.c_double),
        ("dy0", C.c_double), ("growth", C.c_double), ("seed", C.c_uint64),
        ("bc_side", C.c_int32 * 6), ("nbc", C.c_int32), ("reserved", C.c_int32),
        ("bcs", BCSpec * 8),
    ]


class Resid(C.Structure):
    _fields_ = [
        ("rtrms", C.c_double), ("etrms", C.c_double), ("mtrms", C.c_double),
        ("rtmax", C.c_double), ("etmax", C.c_double), ("mtmax", C.c_double),
        ("ccmaxr_center", C.c_double * 3), ("ccmaxe_center", C.c_double * 3),
        ("bcErrorCode", C.c_uint64),
    ]

    def as_dict(self) -> dict:
        d = {k: getattr(self, k) for k in ("rtrms", "etrms", "mtrms", "rtmax", "etmax", "mtmax")}
        d["bcErrorCode"] = int(self.bcErrorCode)
        return d


class LsInfo(C.Structure):
    _fields_ = [("iterations", C.c_int32), ("status", C.c_int32), ("resid0", C.c_double),
                ("resid", C.c_double)]


class StepInfo(C.Structure):
    _fields_ = [("resid", Resid), ("ls", LsInfo), ("min_alpha", C.c_double),
                ("dtau_min", C.c_double), ("dtau_max", C.c_double),
                ("resid_after", Resid), ("start_used", C.c_int32), ("rejected", C.c_int32)]


START = {"jacobi": 0, "zero": 1, "learned": 2}


class StepOpts(C.Structure):
    _fields_ = [("start", C.c_int32), ("reject", C.c_int32), ("lin_rtol", C.c_double),
                ("max_sweeps", C.c_int32), ("check_every", C.c_int32)]


_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)
_vp = C.c_void_p
_ctx = C.c_void_p

_SIGS = {
    "fpsi_default_params": (None, [C.POINTER(Params)]),
    "fpsi_strerror": (C.c_char_p, [C.c_int]),
    "fpsi_last_error": (C.c_char_p, []),
    "fpsi_device_available": (C.c_int, []),
    "fpsi_mesh_generate": (C.c_int, [C.POINTER(MeshSpec), C.POINTER(C.POINTER(Mesh))]),
    "fpsi_mesh_free": (None, [C.POINTER(Mesh)]),
    "fpsi_create": (C.c_int, [C.POINTER(_ctx), C.POINTER(Mesh), C.POINTER(Params)]),
    "fpsi_destroy": (C.c_int, [_ctx]),
    "fpsi_set_params": (C.c_int, [_ctx, C.POINTER(Params)]),
    "fpsi_info": (C.c_int, [_ctx, C.POINTER(C.c_int64), C.POINTER(C.c_int64), _ip,
                            C.POINTER(C.c_int64)]),
    "fpsi_get_geometry": (C.c_int, [_ctx, _dp, _dp, _dp, _dp, _dp]),
    "fpsi_get_colours": (C.c_int, [_ctx, _ip]),
    "fpsi_set_lines": (C.c_int, [_ctx, C.c_int64, C.POINTER(C.c_int64), _ip]),
    "fpsi_get_lines": (C.c_int, [_ctx, _ip, _ip, _ip, C.POINTER(C.c_int64)]),
    "fpsi_set_state": (C.c_int, [_ctx, _dp, _dp, _dp]),
    "fpsi_set_eddy_viscosity": (C.c_int, [_ctx, _dp]),
    "fpsi_set_nutilde": (C.c_int, [_ctx, _dp]),
    "fpsi_get_nutilde": (C.c_int, [_ctx, _dp]),
    "fpsi_get_eddy_viscosity": (C.c_int, [_ctx, _dp]),
    "fpsi_get_wall_distance": (C.c_int, [_ctx, _dp]),
    "fpsi_sa_residual": (C.c_int, [_ctx, _dp]),
    "fpsi_sa_get_system": (C.c_int, [_ctx, _dp, _dp, _dp]),
    "fpsi_sa_solve": (C.c_int, [_ctx, _dp]),
    "fpsi_sa_update": (C.c_int, [_ctx]),
    "fpsi_get_state": (C.c_int, [_ctx, _dp, _dp, _dp]),
    "fpsi_residual": (C.c_int, [_ctx, _dp, C.POINTER(Resid)]),
    "fpsi_get_reconstruction": (C.c_int, [_ctx, _dp, _dp]),
    "fpsi_get_dtau": (C.c_int, [_ctx, _dp]),
    "fpsi_assemble": (C.c_int, [_ctx]),
    "fpsi_get_blocks": (C.c_int, [_ctx, _vp, _vp, _vp, _vp]),
    "fpsi_linear_solve": (C.c_int, [_ctx, _dp, _dp, C.POINTER(LsInfo)]),
    "fpsi_linear_residual": (C.c_int, [_ctx, _dp, _dp]),
    "fpsi_set_iterate": (C.c_int, [_ctx, _dp]),
    "fpsi_get_iterate": (C.c_int, [_ctx, _dp]),
    "fpsi_linear_sweeps": (C.c_int, [_ctx, C.c_int32]),
    "fpsi_gnn_create": (C.c_int, [C.POINTER(C.c_void_p), C.c_uint64]),
    "fpsi_gnn_destroy": (C.c_int, [C.c_void_p]),
    "fpsi_gnn_num_params": (C.c_int64, [C.c_void_p]),
    "fpsi_gnn_get_params": (C.c_int, [C.c_void_p, C.POINTER(C.c_float)]),
    "fpsi_gnn_set_params": (C.c_int, [C.c_void_p, C.POINTER(C.c_float)]),
    "fpsi_gnn_add_snapshot": (C.c_int, [C.c_void_p, _ctx, _dp]),
    "fpsi_gnn_add_snapshot_region": (C.c_int, [C.c_void_p, _ctx, _dp, _dp, _dp, C.c_int32]),
    "fpsi_gnn_clear_snapshots": (C.c_int, [C.c_void_p]),
    "fpsi_gnn_num_snapshots": (C.c_int, [C.c_void_p]),
    "fpsi_gnn_snapshot_cells": (C.c_int64, [C.c_void_p, C.c_int32]),
    "fpsi_gnn_get_snapshot": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_float),
                                        C.POINTER(C.c_float), C.POINTER(C.c_float),
                                        C.POINTER(C.c_float)]),
    "fpsi_gnn_loss_grad": (C.c_int, [C.c_void_p, C.c_int32, C.c_int64, C.c_uint64, _dp,
                                     C.POINTER(C.c_float)]),
    "fpsi_gnn_train": (C.c_int, [C.c_void_p, C.c_int32, C.c_int64, C.c_uint64, C.c_double, _dp]),
    "fpsi_gnn_predict": (C.c_int, [C.c_void_p, _ctx, _dp]),
    "fpsi_update": (C.c_int, [_ctx, _dp]),
    "fpsi_newton_step": (C.c_int, [_ctx, C.POINTER(StepInfo)]),
    "fpsi_newton_step_ex": (C.c_int, [_ctx, C.c_void_p, C.POINTER(StepOpts), C.POINTER(StepInfo)]),
    "fpsi_run": (C.c_int, [_ctx, C.c_int32, C.POINTER(Resid)]),
    "fpsi_time_step": (C.c_int, [_ctx, C.POINTER(Resid)]),
    "fpsi_run_timed": (C.c_int, [_ctx, C.c_int32, C.POINTER(Resid), _dp]),
    "fpsi_kernel_times": (C.c_int, [_ctx, C.c_int32, C.c_int32, C.c_char_p, _dp,
                                    C.POINTER(C.c_int64), _ip]),
    "fpsi_keep_blocks": (C.c_int, [_ctx, C.c_int32]),
    "fpsi_face_flux": (C.c_int, [C.c_int32, C.c_int64, _dp, _dp, _dp, _dp, C.c_double,
                                 C.c_double, C.c_double, C.c_double, C.c_double, _dp]),
    "fpsi_face_jacobian": (C.c_int, [C.c_int64, _dp, _dp, _dp, _dp, C.c_double, C.c_double,
                                     C.c_double, C.c_double, C.c_double, C.c_int32, C.c_int32,
                                     _vp]),
}

_lib = None


def lib() -> C.CDLL:
    """Load libfpsi.so (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with `python -m flowpsi_b200._build` "
                "(the CUDA path has no fallback)")
        L = C.CDLL(str(LIB_PATH))
        for name, (res, args) in _SIGS.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


class FpsiError(RuntimeError):
    def __init__(self, code: int, where: str):
        detail = lib().fpsi_last_error().decode(errors="replace")
        super().__init__(f"{where}: {ERRORS.get(code, code)} ({detail})")
        self.code = code


def check(code: int, where: str) -> None:
    if code != FPSI_OK:
        raise FpsiError(code, where)


def dptr(a: np.ndarray | None):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_dp)


def iptr(a: np.ndarray):
    assert a.dtype == np.int32 and a.flags.c_contiguous
    return a.ctypes.data_as(_ip)


def vptr(a: np.ndarray | None):
    if a is None:
        return None
    assert a.flags.c_contiguous
    return C.c_void_p(a.ctypes.data)
