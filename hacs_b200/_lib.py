"""ctypes binding of libhme.so (the C ABI declared in include/hme.h).

The library is built in-tree by ``hacs_b200.build()`` (nvcc, sm_100a).  There
is no fallback: if libhme.so is missing or cannot be loaded, every entry point
raises, so no result can silently come from anywhere but the CUDA library.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libhme.so")

HME_OK = 0
HME_EINVAL = -1
HME_ECUDA = -2
HME_ENOMEM = -3
HME_ETIMEOUT = -4
HME_EUNSUPPORTED = -5
HME_ENOTINSPAN = -6

HME_SET, HME_ADD, HME_SUB = 0, 1, 2

u32p = C.POINTER(C.c_uint32)
vp = C.c_void_p
sz = C.c_size_t
u32 = C.c_uint32

# name -> (restype, argtypes); mirrors include/hme.h
PROTOTYPES = {
    "hme_ctx_create": (C.c_int, [C.c_int, C.POINTER(vp)]),
    "hme_ctx_destroy": (C.c_int, [vp]),
    "hme_ctx_set_stream": (C.c_int, [vp, vp]),
    "hme_ctx_own_stream": (vp, [vp]),
    "hme_ctx_sync": (C.c_int, [vp]),
    "hme_ctx_set_workspace_retain": (C.c_int, [vp, C.c_int]),
    "hme_ctx_launches": (C.c_uint64, [vp]),
    "hme_ctx_set_timing": (C.c_int, [vp, C.c_int]),
    "hme_ctx_kernel_time": (C.c_int, [vp, C.c_char_p, C.POINTER(C.c_double), C.POINTER(C.c_uint64)]),
    "hme_ctx_timing_reset": (C.c_int, [vp]),
    "hme_last_error": (C.c_char_p, []),
    "hme_version": (C.c_char_p, []),
    "hme_fnv1a_u32": (C.c_uint64, [u32p, u32, u32, sz]),
    "hme_rref_u32": (C.c_int, [vp, u32, u32, u32, u32p, sz, u32p, u32p]),
    "hme_rref_u32_dev": (C.c_int, [vp, u32, u32, u32, vp, sz, u32p, u32p]),
    "hme_rank_profile_u32": (C.c_int, [vp, u32, u32, u32, u32p, sz, u32p, u32p]),
    "hme_det_u32": (C.c_int, [vp, u32, u32, u32p, sz, u32p]),
    "hme_rref_det_u32": (C.c_int, [vp, u32, u32, u32p, sz, u32p, u32p, u32p]),
    "hme_kernel_basis_u32": (C.c_int, [vp, u32, u32, u32, u32p, sz, u32p, sz, u32p]),
    "hme_inverse_u32": (C.c_int, [vp, u32, u32, u32p, sz, u32p, sz, C.POINTER(C.c_int)]),
    "hme_solve_u32": (C.c_int, [vp, u32, u32, u32, u32, u32p, sz, u32p, sz, u32p, sz]),
    "hme_ctx_set_elim_options": (C.c_int, [vp, C.c_int, C.c_int, C.c_int, C.c_int]),
    "hme_ctx_set_panel_kernel": (C.c_int, [vp, C.c_int]),
    "hme_ctx_set_elim_lookahead": (C.c_int, [vp, C.c_int]),
    "hme_ctx_elim_panel_stats": (C.c_int, [vp, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
    "hme_howell_u32": (C.c_int, [vp, u32, u32, u32, u32, u32p, sz, u32p, sz, u32p, u32p, u32p]),
    "hme_smith_u32": (C.c_int, [vp, u32, u32, u32, u32, u32p, sz, u32p, u32p]),
    "hme_gemm_u32": (C.c_int, [vp, u32, u32, u32, u32, u32p, sz, u32p, sz, u32p, sz, C.c_int]),
    "hme_gemm_u32_dev": (C.c_int, [vp, u32, u32, u32, u32, vp, sz, vp, sz, vp, sz, C.c_int]),
    "hme_gemm_u32_dev_noalloc": (C.c_int, [u32, u32, u32, u32, vp, sz, vp, sz, vp, sz, C.c_int, vp]),
    "hme_gemm_nt_u32_dev": (C.c_int, [vp, u32, u32, u32, u32, vp, sz, vp, sz, vp, sz, C.c_int]),
    "hme_schur_update_u32_dev": (C.c_int, [vp, u32, u32, u32, u32, vp, sz, vp, sz, vp, sz]),
    "hme_gemv_u32_dev": (C.c_int, [vp, u32, u32, u32, vp, sz, sz, vp, sz, vp, sz, C.c_int]),
    "hme_axpy_u32_dev": (C.c_int, [vp, u32, u32, u32, u32, vp, sz, sz, vp, sz, sz, C.c_int]),
    "hme_scal_u32_dev": (C.c_int, [vp, u32, u32, u32, u32, vp, sz, sz]),
    "hme_copy_u32_dev": (C.c_int, [vp, u32, u32, vp, sz, sz, vp, sz, sz]),
    "hme_transpose_u32_dev": (C.c_int, [vp, u32, u32, vp, sz, sz, vp, sz, sz]),
    "hme_fill_u32_dev": (C.c_int, [vp, u32, u32, vp, sz, sz, u32]),
    "hme_axpy_identity_u32_dev": (C.c_int, [vp, u32, u32, u32, u32, vp, sz, sz, C.c_int]),
    "hme_gather_u32_dev": (C.c_int, [vp, u32, u32, u32, vp, u32, u32, sz, sz, u32, vp, vp, u32, u32, vp, sz, sz,
                                     C.c_int]),
    "hme_canonicalise_u32_dev": (C.c_int, [vp, u32, u32, u32, vp, sz, sz]),
    "hme_canonicalise_acc64_u32_dev": (C.c_int, [vp, u32, u32, u32, vp, sz, sz, vp, sz, sz]),
    "hme_trsm_unit_u32_dev": (C.c_int, [vp, u32, C.c_int, u32, u32, vp, sz, vp, sz]),
    "hme_gemm_u64": (C.c_int, [vp, C.c_uint64, u32, u32, u32, vp, sz, vp, sz, vp, sz, C.c_int]),
    "hme_gemm_u64_dev": (C.c_int, [vp, C.c_uint64, u32, u32, u32, vp, sz, vp, sz, vp, sz, C.c_int]),
}



class HmeJob(C.Structure):
    """struct hme_job (include/hme.h)."""
    _fields_ = [("p", u32), ("m", u32), ("n", u32), ("k", u32), ("A", vp), ("lda", sz), ("B", vp), ("ldb", sz),
                ("C", vp), ("ldc", sz)]


class HmeGenSpec(C.Structure):
    """struct hme_gen_spec (include/hme.h)."""
    _fields_ = [("dst", vp), ("ld", sz), ("rows", u32), ("cols", u32), ("p", u32), ("family", C.c_int),
                ("seed", C.c_uint64)]


PROTOTYPES.update({
    "hme_batch_gemm_u32_dev": (C.c_int, [vp, u32, C.POINTER(HmeJob)]),
    "hme_batch_rank_u32_dev": (C.c_int, [vp, u32, C.POINTER(HmeJob), u32p]),
    "hme_batch_gemm_rank_u32_dev": (C.c_int, [vp, u32, C.POINTER(HmeJob), u32p]),
    "hme_gen_jobs_u32_dev": (C.c_int, [vp, u32, C.POINTER(HmeGenSpec)]),
    "hme_gemm_variant_count": (C.c_int, []),
    "hme_gemm_u32_dev_variant": (C.c_int, [vp, C.c_int, u32, u32, u32, u32, vp, sz, vp, sz, vp, sz, C.c_int]),
    "hme_ctx_set_gemm_variant": (C.c_int, [vp, C.c_int]),
    "hme_ctx_set_sched_policy": (C.c_int, [vp, C.c_int]),
    "hme_autotune_gemm": (C.c_int, [vp, u32, u32, u32, u32, C.c_int, C.POINTER(C.c_float)]),
    "hme_mlp_param_count": (C.c_int, []),
    "hme_mlp_create": (C.c_int, [vp, C.c_uint64, C.POINTER(vp)]),
    "hme_mlp_destroy": (C.c_int, [vp]),
    "hme_mlp_get_params": (C.c_int, [vp, C.POINTER(C.c_float)]),
    "hme_mlp_set_params": (C.c_int, [vp, C.POINTER(C.c_float)]),
    "hme_mlp_loss_grad": (C.c_int, [vp, u32, C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(C.c_float),
                                    C.POINTER(C.c_float)]),
    "hme_mlp_train": (C.c_int, [vp, u32, C.POINTER(C.c_float), C.POINTER(C.c_float), u32, u32, C.c_float,
                                C.c_uint64, C.POINTER(C.c_float)]),
    "hme_mlp_predict_bf16": (C.c_int, [vp, u32, C.POINTER(C.c_float), C.POINTER(C.c_float)]),
    "hme_sched_plan": (C.c_int, [vp, vp, u32, u32p, C.POINTER(C.c_float), C.POINTER(C.c_float),
                                 C.POINTER(C.c_int)]),
    "hme_sched_plan_rank": (C.c_int, [vp, vp, u32, u32p, C.POINTER(C.c_float), C.POINTER(C.c_float),
                                      C.POINTER(C.c_int)]),
    "hme_sched_plan_set": (C.c_int, [vp, C.c_int, u32, u32p, C.POINTER(C.c_int)]),
    "hme_batch_gemm_u32_dev_plan": (C.c_int, [vp, u32, C.POINTER(HmeJob), C.POINTER(C.c_int)]),
    "hme_batch_gemm_rank_u32_dev_plan": (C.c_int, [vp, u32, C.POINTER(HmeJob), C.POINTER(C.c_int), u32p]),
    "hme_autotune_batch": (C.c_int, [vp, u32, u32, u32, u32, u32, C.c_int, C.POINTER(C.c_float)]),
    "hme_autotune_batch_rank": (C.c_int, [vp, u32, u32, u32, u32, C.c_float, u32, C.c_int, C.POINTER(C.c_float)]),
    "hme_batch_rank_u32_dev_sched": (C.c_int, [vp, u32, C.POINTER(HmeJob), C.POINTER(C.c_int), u32p]),
    "hme_batch_gemm_rank_u32_dev_sched": (C.c_int, [vp, u32, C.POINTER(HmeJob), C.POINTER(C.c_int),
                                                    C.POINTER(C.c_int), u32p]),
})


class HmeR2kStep(C.Structure):
    """struct hme_r2k_step_args (include/hme.h)."""
    _fields_ = [("m", u32), ("r", u32), ("np", u32), ("pc0", u32), ("pc1", u32), ("panel", vp), ("ldp", sz),
                ("swaps", u32p), ("nswaps", u32), ("L", vp), ("ldl", sz), ("u0", u32), ("la0", u32), ("la1", u32),
                ("w", u32)]


u64 = C.c_uint64
PROTOTYPES.update({
    "hme_axpy_u64_dev": (C.c_int, [vp, u64, u64, u32, u32, vp, sz, sz, vp, sz, sz, C.c_int]),
    "hme_scal_u64_dev": (C.c_int, [vp, u64, u64, u32, u32, vp, sz, sz]),
    "hme_copy_u64_dev": (C.c_int, [vp, u32, u32, vp, sz, sz, vp, sz, sz]),
    "hme_transpose_u64_dev": (C.c_int, [vp, u32, u32, vp, sz, sz, vp, sz, sz]),
    "hme_fill_u64_dev": (C.c_int, [vp, u32, u32, vp, sz, sz, u64]),
    "hme_axpy_identity_u64_dev": (C.c_int, [vp, u64, u64, u32, u32, vp, sz, sz, C.c_int]),
    "hme_gather_u64_dev": (C.c_int, [vp, u64, u64, u64, vp, u32, u32, sz, sz, u32, vp, vp, u32, u32, vp, sz, sz,
                                     C.c_int]),
    "hme_canonicalise_u64_dev": (C.c_int, [vp, u64, u32, u32, vp, sz, sz]),
})

PROTOTYPES.update({
    "hme_r2k_plan": (u32, [C.c_int, u32, u32, u32, u32, C.c_uint64]),
    "hme_r2k_session_bytes": (sz, [u32, u32, u32, u32]),
    "hme_r2k_open": (C.c_int, [C.c_int, u32, u32, u32, u32, C.POINTER(vp)]),
    "hme_r2k_put": (C.c_int, [vp, vp, sz, u32, u32, u32, u32]),
    "hme_r2k_get": (C.c_int, [vp, vp, sz, u32, u32, u32, u32]),
    "hme_r2k_step": (C.c_int, [vp, C.POINTER(HmeR2kStep)]),
    "hme_r2k_fetch": (C.c_int, [vp, vp, sz]),
    "hme_r2k_close": (C.c_int, [vp]),
})

_lib = None
_lock = threading.Lock()


class HmeError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"hme error {code}: {msg}")
        self.code = code


def lib():
    global _lib
    if _lib is None:
        with _lock:
            if _lib is None:
                if not os.path.exists(LIB_PATH):
                    raise ImportError(f"libhme.so not built at {LIB_PATH}; run hacs_b200.build()")
                L = C.CDLL(LIB_PATH)
                for name, (res, args) in PROTOTYPES.items():
                    f = getattr(L, name)
                    f.restype = res
                    f.argtypes = args
                _lib = L
    return _lib


def check(rc: int) -> None:
    if rc != HME_OK:
        raise HmeError(rc, lib().hme_last_error().decode(errors="replace"))
