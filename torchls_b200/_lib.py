"""ctypes binding of ``libtorchls_b200.so`` (declared in ``include/torchls_b200.h``).

The library is loaded from the package directory. There is no fallback: if
it is missing, every CUDA entry point raises ``ImportError`` with the build
command. Status codes map to ``ValueError`` (invalid argument),
``torch.linalg.LinAlgError`` (non-positive-definite block) and
``RuntimeError`` (CUDA or unsupported shape).
"""

from __future__ import annotations

import ctypes as C
import os

import torch

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libtorchls_b200.so")

TLS_OK, TLS_ERR_INVALID, TLS_ERR_CUDA, TLS_ERR_UNSUPPORTED, TLS_ERR_NOT_PD = range(5)
F32, F64 = 0, 1
LOSS_NONE, LOSS_HUBER, LOSS_GENERIC = 0, 1, 2
RES_PACKED, RES_REPROJECTION, RES_SE3_BETWEEN, RES_SIM3_BETWEEN = 0, 1, 2, 3
KIND = {"euclidean": 0, "so3": 1, "se3": 2, "sim3": 3, "se2": 4}
MAX_SLOTS, MAX_GROUPS, MAX_FACTOR_GROUPS = 8, 8, 16
PCG_ACTIVE, PCG_CONVERGED, PCG_NONFINITE, PCG_NONPOSITIVE, PCG_MAX_ITERATIONS = range(5)
PCG_PARTIALS = 65536 + 3 * 1024

vp = C.c_void_p
i32, i64, f64 = C.c_int32, C.c_int64, C.c_double


class VarGroup(C.Structure):
    _fields_ = [("offset", i64), ("count", i32), ("dim", i32)]


class FactorGroup(C.Structure):
    _fields_ = [
        ("count", i64), ("rdim", i32), ("nslots", i32), ("total_dim", i32), ("jac_dtype", i32),
        ("slot_group", i32 * MAX_SLOTS), ("slot_dim", i32 * MAX_SLOTS), ("slot_col", i32 * MAX_SLOTS),
        ("slot_gram", i32 * MAX_SLOTS), ("index", vp * MAX_SLOTS), ("jac", vp), ("jac_stride", i64),
    ]


class Segments(C.Structure):
    _fields_ = [("count", i32), ("width", i32), ("lanes", i32), ("pad_", i32), ("ptr", vp), ("src", vp)]


class LinearizeArgs(C.Structure):
    _fields_ = [
        ("fg", FactorGroup), ("residual_kind", i32), ("loss_kind", i32), ("loss_delta", f64),
        ("has_loss", i32), ("want_jacobian", i32), ("packed_residual", vp), ("packed_blocks", vp * MAX_SLOTS),
        ("arg_data", vp * 4), ("arg_stride", i64 * 4), ("arg_slot", i32 * 4), ("weights", vp),
        ("rho1", vp), ("rho2", vp), ("residual", vp), ("raw_residual", vp), ("squared_norm", vp),
        ("objective", vp), ("grad_contrib", vp), ("gram_contrib", vp), ("elim_mask", i32), ("elim_dim", i32),
        ("slot_cross", i32 * MAX_SLOTS), ("cross_width", i32), ("pad2_", i32), ("cross_contrib", vp),
    ]


class NormalTiles(C.Structure):
    _fields_ = [
        ("ncta", i32), ("ntiles", i32), ("stage_doubles", i32), ("acc_doubles", i32), ("ntargets", i32),
        ("gather_lanes", i32), ("xbuf_doubles", i32), ("nheavy", i32), ("tile_factors", i32 * MAX_FACTOR_GROUPS),
        ("tile_base", i32 * MAX_FACTOR_GROUPS), ("cta_base", i32 * (MAX_FACTOR_GROUPS + 1)),
        ("pos", vp * MAX_FACTOR_GROUPS), ("cta_tile", vp), ("tile_run", vp), ("run_col", vp), ("run_meta", vp),
        ("run_dest", vp), ("run_xoff", vp), ("cta_flush", vp), ("flush_col", vp),
        ("flush_meta", vp), ("flush_dest", vp), ("target_col", vp), ("target_dim", vp), ("target_ptr", vp),
        ("target_src", vp), ("partials", vp),
    ]


class NormalArgs(C.Structure):
    _fields_ = [
        ("nfactor_groups", i32), ("nvar_groups", i32), ("vec_dtype", i32), ("pad_", i32),
        ("fg", FactorGroup * MAX_FACTOR_GROUPS), ("contrib_offset", i64 * MAX_FACTOR_GROUPS),
        ("vg", VarGroup * MAX_GROUPS), ("seg", Segments * MAX_GROUPS), ("scale", vp), ("contrib", vp),
        ("damping", f64), ("tiles", C.POINTER(NormalTiles)),
    ]


class BlockGroup(C.Structure):
    _fields_ = [
        ("count", i32), ("dim", i32), ("nmembers", i32), ("pad_", i32), ("member_offset", i64 * 4),
        ("member_dim", i32 * 4), ("blocks", vp), ("factor", vp), ("scale", vp),
    ]


class PcgControl(C.Structure):
    _fields_ = [
        ("rhs_norm", f64), ("threshold", f64), ("residual_norm", f64), ("rz", f64), ("curvature", f64),
        ("alpha", f64), ("beta", f64), ("rz_new", f64), ("rr", f64), ("true_rr", f64), ("drift_rr", f64),
        ("rz_true", f64), ("iterations", i32), ("status", i32), ("restarts", i32), ("checks", i32),
        ("mode", i32), ("stop_at", i32), ("max_iterations", i32), ("check_interval", i32),
        ("periodic", i32), ("pad_", i32 * 3), ("drift_tolerance", f64), ("ticket", C.c_uint32 * 4),
    ]


class SchurArgs(C.Structure):
    _fields_ = [
        ("nedges", i32), ("nchunks", i32), ("dr", i32), ("de", i32), ("nretained", i32), ("nelim", i32),
        ("wdtype", i32), ("vec_dtype", i32), ("cap", i32), ("meta_ints", i32), ("nruns", i32), ("pad_", i32),
        ("retained_offset", i64), ("elim_offset", i64), ("meta", vp), ("slab_r", vp), ("slab_e", vp),
        ("elim_ptr", vp), ("elim_slab", vp), ("rrun_ptr", vp), ("crun_start", vp), ("crun_len", vp),
        ("cross", vp), ("elim_diag", vp), ("ret_diag", vp), ("scale", vp), ("inv_l", vp), ("w", vp),
        ("run_partial", vp), ("ybuf", vp), ("damping", f64), ("bad", vp), ("err", vp), ("wait_cycles", i64),
        ("cross_contrib", vp), ("cross_ptr", vp), ("cross_src", vp),
    ]


class PcgArgs(C.Structure):
    _fields_ = [
        ("n", i64), ("vec_dtype", i32), ("op_kind", i32), ("normal", C.POINTER(NormalArgs)),
        ("schur", C.POINTER(SchurArgs)), ("pre", C.POINTER(BlockGroup)), ("npre", i32), ("pad_", i32),
        ("rhs", vp), ("x", vp), ("r", vp), ("z", vp), ("p", vp), ("ap", vp), ("ztrue", vp), ("psave", vp),
        ("partials", vp), ("control", vp), ("schur_general", vp), ("graph_key", C.c_uint64),
    ]


class FixedSystem(C.Structure):
    _fields_ = [
        ("m", i64), ("n", i64), ("nnz", i64), ("ntargets", i64), ("row_ptr", vp), ("row", vp), ("col", vp),
        ("val", vp), ("col_ptr", vp), ("col_entry", vp), ("target", vp), ("target_ptr", vp), ("pair_left", vp),
        ("pair_right", vp),
    ]


class SchurGeneralArgs(C.Structure):
    _fields_ = [
        ("de", i32), ("nelim", i32), ("nretained", i32), ("wdtype", i32), ("nedges", i64), ("reduced_dim", i64),
        ("full_dim", i64), ("elim_offset", i64), ("var_dim", vp), ("var_row", vp), ("var_full", vp),
        ("var_diag", vp), ("var_ptr", vp), ("edge_var", vp), ("edge_elim", vp), ("edge_w", vp), ("elim_ptr", vp),
        ("elim_edge", vp), ("cross", vp), ("elim_diag", vp), ("ret_diag", vp), ("scale", vp), ("inv_l", vp),
        ("w", vp), ("tbuf", vp), ("ybuf", vp), ("normal", C.POINTER(NormalArgs)), ("xfull", vp), ("yfull", vp),
        ("damping", f64), ("bad", vp), ("max_dim", i32), ("pad2_", i32), ("retained", vp),
    ]


class RetainedMatrix(C.Structure):
    _fields_ = [("row_ptr", vp), ("block_col", vp), ("block_off", vp), ("values", vp)]


# termination codes of tls_batched_lm_update's reason array
BATCH_MAX_ITERATIONS, BATCH_GRADIENT_TOLERANCE, BATCH_COST_TOLERANCE, BATCH_TRIALS_EXHAUSTED = 0, 1, 2, 3


class BatchedSystems(C.Structure):
    _fields_ = [
        ("nproblems", i32), ("nretained", i32), ("dr", i32), ("sdtype", i32), ("ret_ptr", vp), ("ret_problem", vp),
        ("s_off", vp), ("S", vp), ("diag", vp),
    ]


class BatchedPcgArgs(C.Structure):
    _fields_ = [
        ("rhs", vp), ("x", vp), ("iterations", vp), ("status", vp), ("order", vp), ("task_first", vp),
        ("task_size", vp), ("task_groups", vp), ("queue", vp), ("err", vp), ("rtol", f64), ("atol", f64),
        ("ntasks", i32), ("max_iterations", i32), ("smem_bytes", i32), ("pad_", i32),
    ]


class BatchedLm(C.Structure):
    _fields_ = [
        ("nproblems", i32), ("pad_", i32), ("lambda_factor", f64), ("lambda_min", f64), ("lambda_max", f64),
        ("step_quality_min", f64), ("cost_tolerance", f64), ("actual", vp), ("predicted", vp), ("new_cost", vp),
        ("cost", vp), ("lam", vp), ("tried", vp), ("ok", vp), ("active", vp), ("pending", vp), ("accepted", vp),
        ("rejected", vp), ("reason", vp),
    ]


_SIGNATURES = {
    "tls_linearize": [C.POINTER(LinearizeArgs), vp],
    "tls_segment_reduce": [C.POINTER(Segments), vp, i32, i32, i32, vp, i32, vp],
    "tls_normal_matvec": [C.POINTER(NormalArgs), vp, vp, vp],
    "tls_permute_columns": [vp, vp, i32, i64, i64, i64, vp, vp],
    "tls_jacobian_matvec": [C.POINTER(NormalArgs), vp, vp, vp],
    "tls_squared_matvec_norm": [C.POINTER(NormalArgs), vp, vp, vp, vp],
    "tls_squared_matvec_norm_static": [C.POINTER(NormalArgs), vp, vp, vp],
    "tls_jacobian_rmatvec": [C.POINTER(NormalArgs), vp, vp, vp],
    "tls_block_cholesky": [C.POINTER(BlockGroup), i32, f64, vp, vp],
    "tls_block_solve": [C.POINTER(BlockGroup), i32, vp, vp, i32, vp],
    "tls_pcg_start": [C.POINTER(PcgArgs), f64, f64, i32, i32, i32, f64, vp],
    "tls_pcg_run": [C.POINTER(PcgArgs), i32, vp],
    "tls_pcg_state_bytes": [],
    "tls_schur_damp": [C.POINTER(SchurArgs), vp],
    "tls_schur_matvec": [C.POINTER(SchurArgs), vp, vp, vp],
    "tls_schur_reduced_rhs": [C.POINTER(SchurArgs), vp, vp, vp],
    "tls_schur_backsubstitute": [C.POINTER(SchurArgs), vp, vp, vp],
    "tls_schur_preconditioner_blocks": [C.POINTER(SchurArgs), vp, vp],
    "tls_schur_general_damp": [C.POINTER(SchurGeneralArgs), vp],
    "tls_schur_general_matvec": [C.POINTER(SchurGeneralArgs), vp, vp, vp],
    "tls_schur_general_reduced_rhs": [C.POINTER(SchurGeneralArgs), vp, vp, vp],
    "tls_schur_general_backsubstitute": [C.POINTER(SchurGeneralArgs), vp, vp, vp],
    "tls_schur_general_preconditioner_blocks": [C.POINTER(SchurGeneralArgs), vp, vp],
    "tls_schur_general_pair_blocks": [C.POINTER(SchurGeneralArgs), i32, vp, vp, vp, i32, i32, vp, vp],
    "tls_schur_dense_matrix": [C.POINTER(SchurArgs), i64, vp, vp, vp, vp, vp, vp, vp],
    "tls_dense_cholesky": [i64, vp, i64, vp, vp],
    "tls_fixed_matvec": [C.POINTER(FixedSystem), vp, i64, vp, vp],
    "tls_fixed_rmatvec": [C.POINTER(FixedSystem), vp, i64, vp, vp],
    "tls_fixed_normal": [C.POINTER(FixedSystem), vp, f64, vp, vp],
    "tls_admm_step": [i64, vp, vp, vp, vp, vp, vp, f64, vp, vp, vp],
    "tls_dense_cholesky_solve": [i64, vp, i64, i64, vp, i64, vp],
    "tls_batched_schur_dense": [C.POINTER(SchurArgs), C.POINTER(BatchedSystems), i64, vp, vp, vp, vp, vp, vp],
    "tls_batched_pcg": [C.POINTER(BatchedSystems), C.POINTER(BatchedPcgArgs), vp],
    "tls_batched_share_bytes": [i32, i32, i32, i32],
    "tls_factor_terms": [i64, i32, vp, vp, i32, f64, vp, vp, vp, vp],
    "tls_factor_sqnorm": [i64, i32, vp, vp, vp],
    "tls_batched_lm_update": [C.POINTER(BatchedLm), vp],
    "tls_retract": [i32, i32, i32, vp, vp, vp, vp, vp, vp, vp],
    "tls_reduce": [vp, i32, i64, i32, vp, vp, vp],
    "tls_trial_terms": [i64, i32, vp, vp, i32, f64, vp, vp, vp, i32, vp, vp, vp],
    "tls_launch_count": [],
    "tls_last_error": [],
    "tls_version": [],
    "tls_device_init": [i32],
}

_lib = None


def lib():
    """Load the shared library (once); raise ImportError when it is absent."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"torchls_b200 CUDA library not built ({LIB_PATH}); run `python -m torchls_b200.build`"
            )
        handle = C.CDLL(LIB_PATH)
        for name, argtypes in _SIGNATURES.items():
            fn = getattr(handle, name)
            fn.argtypes = argtypes
            fn.restype = {"tls_last_error": C.c_char_p, "tls_launch_count": C.c_int64,
                          "tls_batched_share_bytes": C.c_int64}.get(name, C.c_int)
        _lib = handle
    return _lib


def check(status: int, what: str = "") -> None:
    if status == TLS_OK:
        return
    msg = lib().tls_last_error().decode(errors="replace")
    text = f"{what}: {msg}" if what else msg
    if status == TLS_ERR_INVALID:
        raise ValueError(text)
    if status == TLS_ERR_NOT_PD:
        raise torch.linalg.LinAlgError(text)
    raise RuntimeError(text)


def call(name: str, *args) -> None:
    check(getattr(lib(), name)(*args), name)


def ptr(t: torch.Tensor | None):
    return None if t is None else t.data_ptr()


def stream_handle(device=None):
    return torch.cuda.current_stream(device).cuda_stream


def dtype_code(dtype: torch.dtype) -> int:
    if dtype == torch.float64:
        return F64
    if dtype == torch.float32:
        return F32
    raise ValueError(f"unsupported dtype {dtype}")


def require_cuda(t: torch.Tensor, what: str = "CUDA backend") -> None:
    if t.device.type != "cuda":
        raise ValueError(f"{what} requires CUDA tensors; got device {t.device}")


def launch_count() -> int:
    """Kernels launched by the library so far in this process."""
    return int(lib().tls_launch_count())
