"""ctypes binding of libkcfd.so (the C ABI declared in include/kcfd.h).

The library is loaded on first use. There is no CPU fallback: if the library is
missing or no CUDA device is present, every device entry point raises.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG_DIR, "libkcfd.so")

OK, MAXITER, BREAKDOWN, BAD_INPUT, CUDA_ERROR, TIMEOUT = 0, 1, 2, 3, 4, 5
STATUS_NAMES = {0: "OK", 1: "MAXITER", 2: "BREAKDOWN", 3: "BAD_INPUT", 4: "CUDA_ERROR", 5: "TIMEOUT"}
PREC = {"none": 0, "jacobi": 1, "ilu0": 2, "amg": 3}
STOP_SCIPY, STOP_GPU = 0, 1
MODE_FP64, MODE_MIXED = 0, 1
METHOD_BICGSTAB, METHOD_CG = 0, 1

i32, i64, f64, vp = C.c_int32, C.c_int64, C.c_double, C.c_void_p
P_i32, P_i64, P_f64 = C.POINTER(C.c_int32), C.POINTER(C.c_int64), C.POINTER(C.c_double)


class KcfdError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"kcfd {STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


class MeshExport(C.Structure):
    _fields_ = [(n, vp) for n in ("owner", "neighbour", "face_nodes", "cell_faces", "area", "normal", "fcenter",
                                  "ccenter", "volume", "face_patch", "indptr", "indices", "slot_on", "slot_no",
                                  "diag_slot", "face_color", "cell_color", "level_natural")]


class FaceLayout(C.Structure):
    """kcfd_face_layout_t: output arrays of kcfd_mesh_device_layout."""
    _fields_ = [(n, vp) for n in ("order", "color_ptr", "owner", "neigh", "area", "normal", "fcenter", "gc", "dlen",
                                  "dorth", "slot_on", "slot_no", "cf_ptr", "cf_face")]


class Csr(C.Structure):
    _fields_ = [("n", i32), ("nnz", i32), ("indptr", vp), ("indices", vp), ("vals64", vp), ("vals32", vp)]


class SolverOpts(C.Structure):
    _fields_ = [("precond", i32), ("stop", i32), ("mode", i32), ("nrhs", i32), ("maxiter", i32), ("team", i32),
                ("lanes", i32), ("block", i32), ("rtol", f64), ("atol", f64), ("inner_rtol", f64),
                ("max_refine", i32), ("inner_maxiter", i32), ("fill_level", i32), ("amg_max_levels", i32),
                ("amg_coarse_max", i32), ("method", i32)]


class AmgOpts(C.Structure):
    _fields_ = [("mode", i32), ("coarse_max", i32), ("max_levels", i32), ("power_iters", i32)]


AMG_ITEMS = {"aggregates": 0, "indptr": 1, "indices": 2, "values": 3, "p_indptr": 4, "p_indices": 5,
             "p_values": 6, "omega": 7, "coarse_inverse": 8}


class TfParams(C.Structure):
    """kcfd_tf_params_t: two-fluid properties and model constants."""
    _fields_ = [(n, f64) for n in ("rho_l", "rho_g", "mu_l", "mu_g", "cp_l", "cp_g", "k_l", "k_g", "d_b")] + \
        [("g", f64 * 3)] + [(n, f64) for n in ("h_i_coeff", "a_i_coeff", "T_sat", "h_fg", "r_phase_change", "dt")]


# name -> (restype, argtypes)
SIGNATURES = {
    "kcfd_version": (i32, []),
    "kcfd_last_error": (i32, [C.c_char_p, i32]),
    "kcfd_device_info": (i32, [P_i32, P_i32, P_i32]),
    "kcfd_mesh_build": (i32, [i32, i64, vp, i64, vp, vp, vp, vp, vp, vp, i64, vp, vp, vp, C.POINTER(vp)]),
    "kcfd_mesh_info": (i32, [vp, P_i64]),
    "kcfd_mesh_export": (i32, [vp, C.POINTER(MeshExport)]),
    "kcfd_mesh_free": (None, [vp]),
    "kcfd_mesh_device_layout": (i32, [i32, i64, i64, i64, i32, i32, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp,
                                      C.POINTER(FaceLayout)]),
    "kcfd_cast_f64_f32": (i32, [i64, vp, vp, vp]),
    "kcfd_spmv_f64": (i32, [C.POINTER(Csr), vp, vp, i32, vp]),
    "kcfd_spmv_f32": (i32, [C.POINTER(Csr), vp, vp, i32, vp]),
    "kcfd_solver_create": (i32, [C.POINTER(Csr), C.POINTER(SolverOpts), vp, C.POINTER(vp)]),
    "kcfd_solver_destroy": (None, [vp]),
    "kcfd_solver_setup": (i32, [vp, C.POINTER(Csr), vp]),
    "kcfd_solver_solve": (i32, [vp, C.POINTER(Csr), vp, vp, vp, vp, vp, vp]),
    "kcfd_solver_error": (i32, [vp, P_i32, vp]),
    "kcfd_solver_info": (i32, [vp, P_i32]),
    "kcfd_solver_apply_precond": (i32, [vp, C.POINTER(Csr), vp, vp, vp]),
    "kcfd_solver_amg": (i32, [vp, C.POINTER(vp)]),
    "kcfd_amg_create": (i32, [C.POINTER(Csr), C.POINTER(AmgOpts), C.POINTER(vp)]),
    "kcfd_amg_setup": (i32, [vp, C.POINTER(Csr), vp]),
    "kcfd_amg_apply": (i32, [vp, vp, vp, vp]),
    "kcfd_amg_info": (i32, [vp, P_i32, P_i64, P_i64]),
    "kcfd_amg_export": (i32, [vp, i32, i32, vp]),
    "kcfd_amg_destroy": (None, [vp]),
    "kcfd_lsq_gradient": (i32, [vp, vp, vp, vp, vp]),
    "kcfd_tf_drag": (i32, [vp, vp, vp, vp, vp, vp, vp]),
    "kcfd_tf_interfacial": (i32, [vp, vp, vp, vp, vp, vp, vp]),
    "kcfd_tf_phase_change": (i32, [vp, vp, vp, vp, vp, vp, vp, vp]),
    "kcfd_tf_gamma": (i32, [vp, vp, i32, vp, f64, vp, vp, vp, vp, vp]),
    "kcfd_tf_face_flux": (i32, [vp, i32, vp, vp, f64, vp, vp]),
    "kcfd_tf_mass_flux": (i32, [vp, f64, vp, vp, vp, vp]),
    "kcfd_tf_zero_gradient": (i32, [vp, vp, vp, i32, vp, vp]),
    "kcfd_tf_momentum_sources": (i32, [vp, vp, i32, i32, f64, vp, vp, vp, vp, vp, vp, vp, vp, vp]),
    "kcfd_tf_boundary": (i32, [vp, vp, vp, vp, i32, vp, vp, vp, vp, vp, vp]),
    "kcfd_tf_relax": (i32, [vp, f64, vp, i32, i32, vp, vp, vp, vp]),
    "kcfd_tf_update_ap": (i32, [vp, vp, vp, i32, vp]),
    "kcfd_tf_pressure_assemble": (i32, [vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp]),
    "kcfd_tf_correct": (i32, [vp, f64, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp]),
    "kcfd_tf_alpha_source": (i32, [vp, f64, vp, vp, vp]),
    "kcfd_tf_energy_sources": (i32, [vp, vp, f64, f64, vp, vp, vp, vp, vp, f64, vp, vp, vp, vp, vp, vp, vp]),
    "kcfd_tf_guard": (i32, [i64, vp, vp, i32, f64, f64, vp, vp]),
    "kcfd_tf_alpha_finish": (i32, [i32, vp, vp, vp, vp, vp]),
    "kcfd_tf_copy": (i32, [i32, i32, vp, i32, i32, vp, i32, i32, vp]),
    "kcfd_mass_flux": (i32, [vp, vp, vp, f64, vp, vp]),
    "kcfd_momentum_assemble": (i32, [vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp]),
    "kcfd_pressure_assemble": (i32, [vp, vp, f64, vp, vp, vp, vp, vp, vp, vp]),
    "kcfd_gg_gradient": (i32, [vp, i32, vp, vp, vp, vp, vp]),
    "kcfd_simple_correct": (i32, [vp, f64, vp, vp, vp, vp, vp, vp, vp, vp]),
    "kcfd_residual_norms": (i32, [C.POINTER(Csr), vp, vp, i32, vp, vp, vp]),
    "kcfd_simple_residual": (i32, [i32, vp, vp, vp, vp, vp, i32, vp]),
    "kcfd_op_diffusion": (i32, [vp, vp, vp, vp, vp]),
    "kcfd_op_convection_upwind": (i32, [vp, vp, vp, vp, vp]),
    "kcfd_op_boundary": (i32, [vp, vp, vp, vp, vp, vp, vp, vp, vp, vp]),
    "kcfd_op_cells": (i32, [vp, i32, f64, f64, vp, vp, vp, vp, vp, vp]),
    "kcfd_muscl_correction": (i32, [vp, i32, vp, vp, vp, vp, vp]),
    "kcfd_batch_create": (i32, [i32, vp, vp, vp, vp, vp, C.POINTER(vp)]),
    "kcfd_batch_plan": (i32, [i32, vp, vp, i32, vp]),
    "kcfd_batch_destroy": (None, [vp]),
    "kcfd_batch_info": (i32, [vp, P_i64]),
    "kcfd_batch_tiers": (i32, [vp, P_i32]),
    "kcfd_selftest_barrier": (i32, [i32, i32, i64, vp, vp, vp]),
    "kcfd_graph_capture_begin": (i32, [vp]),
    "kcfd_graph_capture_end": (i32, [vp, C.POINTER(vp)]),
    "kcfd_graph_launch": (i32, [vp, vp]),
    "kcfd_graph_destroy": (None, [vp]),
    "kcfd_batch_solve": (i32, [vp, vp, vp, vp, vp, vp, vp, vp]),
    "kcfd_vec_norms2": (i32, [i32, i32, vp, vp, vp, vp]),
    "kcfd_record_norm": (i32, [vp, vp, vp, i32, vp]),
    "kcfd_noalloc_max_rows": (i32, []),
    "kcfd_bicgstab_noalloc": (i32, [C.POINTER(Csr), vp, vp, i32, i32, f64, f64, i32, vp, vp, vp, vp]),
}

REDUCE_SCRATCH = 8192
LIMITERS = {None: -1, "none": -1, "minmod": 0, "superbee": 1, "van_albada": 2, "van_leer": 3}


class MomParams(C.Structure):
    _fields_ = [("rho", f64), ("mu", f64), ("alpha_u", f64), ("dt", f64), ("limiter", i32), ("nonorth", i32)]

_lib = None
_lock = threading.Lock()


def lib():
    """Load libkcfd.so (building it first if the sources are newer)."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            from . import build
            build.build()
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def last_error():
    buf = C.create_string_buffer(2048)
    lib().kcfd_last_error(buf, 2048)
    return buf.value.decode(errors="replace")


def check(status, what=""):
    if status != OK:
        raise KcfdError(status, f"{what}: {last_error()}" if what else last_error())
    return status


def ptr(t):
    """Device or host address of a torch tensor / numpy array (None -> NULL)."""
    if t is None:
        return None
    if hasattr(t, "data_ptr"):
        return t.data_ptr()
    return t.ctypes.data


def require_cuda():
    import torch
    if not torch.cuda.is_available():
        raise KcfdError(CUDA_ERROR, "no CUDA device: the kcfd device path has no CPU fallback")
    return torch


def stream_handle(stream=None):
    import torch
    s = stream if stream is not None else torch.cuda.current_stream()
    return s.cuda_stream


_deferred = []
_deferred_lock = threading.Lock()


def release(fn_name, handle):
    """Destroy a native handle (kcfd_*_destroy by name). A destroy frees device memory,
    which would invalidate a stream capture in progress on this thread (a handle
    dropped by the garbage collector while a CUDA graph is being captured), so inside
    a capture the handle is queued and destroyed at the next release outside one."""
    capturing = False
    try:
        import torch
        capturing = torch.cuda.is_available() and torch.cuda.is_current_stream_capturing()
    except Exception:
        capturing = False
    with _deferred_lock:
        if capturing:
            _deferred.append((fn_name, handle))
            return
        pending = list(_deferred)
        _deferred.clear()
    for name, h in pending + [(fn_name, handle)]:
        try:
            getattr(lib(), name)(h)
        except Exception:
            pass

