"""ctypes binding of libmsgb.so (the C ABI declared in include/msgb.h).

The library is loaded from this package directory.  There is no fallback: if
the shared library is missing or fails to load, every compute entry point
raises ``RuntimeError``.  Status codes other than ``MSGB_OK`` are raised as
``RuntimeError`` carrying ``msgb_last_error()``.
"""

from __future__ import annotations

import ctypes
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmsgb.so")

c_i32 = ctypes.c_int32
c_i64 = ctypes.c_int64
c_dbl = ctypes.c_double
c_vp = ctypes.c_void_p
c_sz = ctypes.c_size_t

STATUS = {0: "OK", 1: "ARG", 2: "WORKSPACE", 3: "CUDA", 4: "UNSUPPORTED", 5: "NONFINITE", 6: "TIMEOUT"}


class Problem(ctypes.Structure):
    _fields_ = [("ndim", c_i32), ("periodic", c_i32 * 3), ("L", c_dbl * 3), ("c", c_dbl),
                ("nt", c_i64), ("ts", c_vp), ("ns", c_i64), ("sensors", c_vp)]


class BeamSet(ctypes.Structure):
    _fields_ = [("n", c_i64), ("x0", c_vp), ("p0", c_vp), ("alpha", c_vp), ("a0", c_vp),
                ("omega", c_vp), ("modes", c_i32)]


class SensorTiling(ctypes.Structure):
    _fields_ = [("n_tiles", c_i64), ("order", c_vp), ("tile_offsets", c_vp)]


class SumOpts(ctypes.Structure):
    _fields_ = [("cutoff", c_dbl), ("eval_count", c_vp), ("tiling", c_vp)]


class MswptDesc(ctypes.Structure):
    _fields_ = [("ndim", c_i32), ("N", c_i32 * 3), ("aspect", c_i32 * 3), ("redundancy", c_i32),
                ("num_levels", c_i32), ("total_boxes", c_i32), ("box_length", c_vp),
                ("box_level", c_vp), ("centres", c_vp),
                ("box_shape", c_vp), ("coeffs_cumsum", c_vp), ("boxes_cumsum", c_vp),
                ("gfilt", c_vp), ("gfilt_offset", c_vp), ("sum_gsquare", c_vp),
                ("lattice_counts", c_vp), ("lattice_first", c_vp), ("lattice_step", c_vp),
                ("lattice_offset", c_vp), ("lattice_box", c_vp)]


class Medium(ctypes.Structure):
    _fields_ = [("kind", c_i32), ("boundary", c_i32), ("n", c_i32 * 3), ("spacing", c_dbl * 3),
                ("origin", c_dbl * 3), ("coeffs", c_vp), ("c", c_dbl), ("lam", c_dbl), ("coeffs32", c_vp),
                ("c_ref", c_dbl)]


class OdeOpts(ctypes.Structure):
    _fields_ = [("method", c_i32), ("substeps", c_i32), ("rtol", c_dbl), ("atol", c_dbl), ("dt0", c_dbl),
                ("max_steps", c_i64), ("only_flagged", c_i32), ("dense_output", c_i32), ("step_count", c_vp),
                ("medium_fp32", c_i32)]


class SurrogateIO(ctypes.Structure):
    _fields_ = [("nb", c_i64), ("b_first", c_i64), ("nq_t", c_i64), ("t_index", c_vp), ("ld", c_i32)]


class SurrogateAccept(ctypes.Structure):
    _fields_ = [("residual_tol", c_dbl), ("phase_tol", c_dbl), ("pos_err", c_dbl)]


class Trajectories(ctypes.Structure):
    _fields_ = [("nb", c_i64), ("b_first", c_i64), ("rec64", c_vp), ("rec32", c_vp), ("cull", c_vp),
                ("status", c_vp), ("slot", c_vp), ("pool", c_vp), ("pool_cull", c_vp), ("pool_blocks", c_i64),
                ("pool_next", c_vp), ("live_boxes", c_vp), ("n_boxes", c_i64), ("live_cutoff", c_dbl)]


class Gemm(ctypes.Structure):
    _fields_ = [("A", c_vp), ("sAm", c_i64), ("sAk", c_i64), ("B", c_vp), ("sBn", c_i64), ("sBk", c_i64),
                ("M", c_i32), ("N", c_i32), ("K", c_i32), ("bias", c_vp), ("act", c_i32), ("C32", c_vp),
                ("ldc32", c_i64), ("C16", c_vp), ("ldc16", c_i64), ("error_flag", c_vp)]


class BeamOut(ctypes.Structure):
    _fields_ = [("x0", c_vp), ("p0", c_vp), ("alpha", c_vp), ("a0", c_vp), ("omega", c_vp),
                ("a0_unit", c_vp)]


class TrGeometry(ctypes.Structure):
    _fields_ = [("normal_axis", c_i32), ("normal_value", c_dbl), ("inward", c_dbl)]


class TrBeams(ctypes.Structure):
    _fields_ = [("n", c_i64), ("x", c_vp), ("p", c_vp), ("M", c_vp), ("a", c_vp), ("omega", c_vp),
                ("mode", c_vp), ("t0", c_vp)]


# name -> (restype, argtypes)
SIGNATURES = {
    "msgb_last_error": (ctypes.c_char_p, []),
    "msgb_version": (ctypes.c_char_p, []),
    "msgb_sum_fwd_f64": (ctypes.c_int, [c_vp, c_vp, c_vp, c_vp]),
    "msgb_adj_gather_f64": (ctypes.c_int, [c_vp, c_vp, c_vp, c_vp, c_vp]),
    "msgb_sum_f32_workspace_size": (c_sz, [c_vp, c_i64]),
    "msgb_sum_fwd_f32": (ctypes.c_int, [c_vp, c_vp, c_vp, c_vp, c_sz, c_vp, c_vp]),
    "msgb_adj_gather_f32": (ctypes.c_int, [c_vp, c_vp, c_vp, c_vp, c_sz, c_vp, c_vp, c_vp]),
    "msgb_sum_fwd_f32_static": (ctypes.c_int, [c_vp, c_vp, c_vp, c_vp, c_vp]),
    "msgb_rk4_trajectories": (ctypes.c_int, [c_vp, c_vp, c_vp, ctypes.c_int, c_vp, c_vp]),
    "msgb_ode_trajectories": (ctypes.c_int, [c_vp, c_vp, c_vp, c_vp, c_vp, c_vp]),
    "msgb_threshold_workspace_size": (c_sz, [c_i64]),
    "msgb_coefficients_dpdt": (ctypes.c_int, [c_vp, c_vp, c_vp, c_vp, c_vp, ctypes.c_int, ctypes.c_int, c_vp, c_vp,
                                              c_vp]),
    "msgb_threshold": (ctypes.c_int, [ctypes.c_int, c_dbl, c_vp, c_vp, c_i64, c_vp, c_vp, c_vp, c_vp, c_vp, c_sz,
                                      c_vp]),
    "msgb_surrogate_features": (ctypes.c_int, [c_vp, c_vp, c_vp, c_vp, c_vp, c_vp]),
    "msgb_surrogate_targets": (ctypes.c_int, [c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp]),
    "msgb_surrogate_records": (ctypes.c_int, [c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp]),
    "msgb_sum_fwd_f64_traj": (ctypes.c_int, [c_vp, c_vp, c_vp, c_vp, c_vp]),
    "msgb_adj_gather_f64_traj": (ctypes.c_int, [c_vp, c_vp, c_vp, c_vp, c_vp, c_vp]),
    "msgb_sum_f32_traj_workspace_size": (c_sz, [c_vp, c_i64]),
    "msgb_sum_fwd_f32_traj": (ctypes.c_int, [c_vp, c_vp, c_vp, c_vp, ctypes.c_int, ctypes.c_int, c_vp, c_sz,
                                              c_vp, c_vp]),
    "msgb_adj_gather_f32_traj": (ctypes.c_int, [c_vp, c_vp, c_vp, c_vp, c_vp, c_sz, c_vp, c_vp, c_vp]),
    "msgb_gemm_bf16": (ctypes.c_int, [c_vp, c_vp]),
    "msgb_silu_backward": (ctypes.c_int, [c_vp, c_vp, c_i64, c_vp, c_vp, c_vp]),
    "msgb_colsum": (ctypes.c_int, [c_vp, ctypes.c_int, ctypes.c_int, c_i64, c_vp, c_vp]),
    "msgb_adam": (ctypes.c_int, [c_vp, c_vp, c_vp, c_vp, c_i64, c_dbl, c_dbl, c_dbl, c_dbl, c_i64, c_vp, c_vp]),
    "msgb_to_bf16": (ctypes.c_int, [c_vp, c_i64, c_vp, c_vp]),
    "msgb_mswpt_create": (ctypes.c_int, [c_vp, c_vp]),
    "msgb_mswpt_destroy": (ctypes.c_int, [c_vp]),
    "msgb_mswpt_total_coeffs": (c_i64, [c_vp]),
    "msgb_mswpt_workspace_size": (c_sz, [c_vp]),
    "msgb_mswpt_forward": (ctypes.c_int, [c_vp, c_vp, ctypes.c_int, ctypes.c_int, c_dbl,
                                           ctypes.c_int, c_vp, c_vp, c_vp, c_sz, c_vp]),
    "msgb_mswpt_synthesis": (ctypes.c_int, [c_vp, c_vp, ctypes.c_int, ctypes.c_int, c_vp, c_vp,
                                             c_sz, c_vp]),
    "msgb_topn_workspace_size": (c_sz, [c_i64, c_i64]),
    "msgb_topn": (ctypes.c_int, [c_vp, c_vp, c_i64, c_i64, c_vp, c_vp, c_vp, c_sz, c_vp]),
    "msgb_beam_init": (ctypes.c_int, [c_vp, c_vp, c_vp, c_vp, c_i64, c_vp, c_vp]),
    "msgb_tr_init": (ctypes.c_int, [c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_i64, ctypes.c_int, c_dbl, c_vp, c_vp]),
    "msgb_adjoint_source_workspace_size": (c_sz, [c_i64, c_i64]),
    "msgb_adjoint_source": (ctypes.c_int, [c_vp, c_vp, ctypes.c_int, c_i64, c_i64, c_dbl, c_vp, c_vp, c_vp, c_sz,
                                           c_vp]),
    "msgb_medium_speed": (ctypes.c_int, [c_i32, c_vp, c_vp, c_i64, c_vp, c_vp]),
    "msgb_tr_final_states": (ctypes.c_int, [c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp]),
    "msgb_scatter_coeff_grad": (ctypes.c_int, [c_vp, c_vp, c_i64, c_dbl, c_vp, ctypes.c_int,
                                                c_vp, c_vp]),
    "msgb_sum_f32_tile_count": (c_i64, [c_vp, c_vp]),
    "msgb_sum_f32_tile_boxes": (ctypes.c_int, [c_vp, c_vp, c_vp, c_sz, c_vp, c_vp]),
    "msgb_peak_probe_ops": (c_dbl, [ctypes.c_int, c_i64, ctypes.c_int, ctypes.c_int]),
    "msgb_peak_probe": (ctypes.c_int, [ctypes.c_int, c_i64, ctypes.c_int, ctypes.c_int, c_vp, c_vp]),
}

_lock = threading.Lock()
_lib = None


def lib():
    """Load libmsgb.so once; raises RuntimeError when it is absent."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise RuntimeError(
                    f"libmsgb.so not found at {LIB_PATH}; build it with "
                    "`python -m beamax_b200.build` (the CUDA path has no fallback)")
            L = ctypes.CDLL(LIB_PATH)
            for name, (res, args) in SIGNATURES.items():
                fn = getattr(L, name, None)
                if fn is None:
                    continue  # reported by missing_symbols(); calls raise AttributeError
                fn.restype = res
                fn.argtypes = args
            _lib = L
    return _lib


def missing_symbols():
    """Entry points of include/msgb.h that the loaded library does not export."""
    L = lib()
    return [n for n in SIGNATURES if getattr(L, n, None) is None]


def last_error() -> str:
    return lib().msgb_last_error().decode(errors="replace")


def check(status: int, what: str) -> None:
    if status != 0:
        raise RuntimeError(f"{what} failed ({STATUS.get(status, status)}): {last_error()}")


def ref(obj) -> int:
    return ctypes.addressof(obj)
