"""hacs_b200 -- host-side Python mirror of the B200-native exact modular matrix engine.

The engine itself is libhme.so (CUDA C++ for sm_100a, C ABI in include/hme.h).
This module mirrors the reference engine's operator names and argument meaning
(drjanosch42/hacs 0.2.1, ``engine::kernels`` / ``engine::elim`` /
``engine::ring2k`` / ``engine::ring3k``) over numpy host arrays, and offers
device-pointer variants over torch CUDA tensors:

  ``Engine.gemm(p, A, B, C=None, op=SET)``   engine::kernels::gemm<uint32_t> (Kernels.h:178-185)
  ``Engine.rref(p, A)``                      engine::elim::rref (DenseElim.h:153-158)
  ``Engine.column_rank_profile(p, A)``       engine::elim::column_rank_profile (DenseElim.h:160-169)
  ``Engine.det(p, A)``                       determinant mod p (no reference entry point)
  ``Engine.kernel_basis(p, A)``              engine::elim::kernel_basis of rref(A) (DenseElim.h:171-179)
  ``Engine.inverse(p, A)``                   engine::elim::inverse (DenseElim.h:186-189)
  ``Engine.solve_multi_rhs(p, B, Y)``        engine::elim::solve_multi_rhs (DenseElim.h:191-197)
  ``Engine.howell(ell, k, A)``               elim::howell / ring2k::howell / ring3k::howell (ENGINE_API.md Sec. 13.5)
  ``Engine.smith(ell, k, A)``                ring2k::smith / ring3k::smith valuations (Ring2k.h:702, Ring3k.h:100)
  ``Engine.gemm_u64(p, A, B, C=None, op)``   engine::kernels::gemm<uint64_t> (any modulus below 2^64)
  ``Engine.gemv_dev / axpy_dev / scal_dev / copy_dev / transpose_dev / fill_dev / axpy_identity_dev /
  gather_dev / canonicalise_dev / canonicalise_acc64_dev / trsm_unit_dev / gemm_nt_dev /
  schur_update_dev``                         engine::cuda level-1/2 ops (CudaKernels.h:120-247)

Every call goes to libhme; there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from . import _lib
from ._lib import HME_ADD as ADD, HME_SET as SET, HME_SUB as SUB, HmeError, check

__all__ = ["Engine", "SET", "ADD", "SUB", "HmeError", "build", "limbs_for"]

HERE = os.path.dirname(os.path.abspath(__file__))


def build(verbose: bool = False) -> str:
    """Compile libhme.so in-tree with nvcc for sm_100a; returns its path."""
    out = None if verbose else subprocess.DEVNULL
    subprocess.check_call(["make", "-j8", "-C", os.path.join(HERE, "csrc")], stdout=out)
    return _lib.LIB_PATH


def limbs_for(p: int) -> int:
    """Unsigned 8-bit limbs per residue of Z/p: 1, 2, 3 or 4."""
    return 1 if p <= 256 else 2 if p <= 65536 else 3 if p <= (1 << 24) else 4


def _u32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.uint32)


def _p32(a: np.ndarray):
    return a.ctypes.data_as(_lib.u32p)


def _dev_ptr(t) -> int:
    import torch

    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise TypeError("device entry points take CUDA torch tensors")
    if t.element_size() != 4:
        raise TypeError("device tensors must hold 32-bit words (torch.int32 or torch.uint32)")
    if t.dim() != 2 or t.stride(1) != 1:
        raise ValueError("device tensors must be 2-D with unit column stride")
    return t.data_ptr()


def _view(t, elem: int = 4):
    """(pointer, rows, cols, row stride, column stride) of a 1-D (a column) or
    2-D CUDA tensor view with any strides, strides in elements."""
    import torch

    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise TypeError("device entry points take CUDA torch tensors")
    if t.element_size() != elem:
        raise TypeError(f"device view must hold {8 * elem}-bit words")
    if t.dim() == 1:
        return t.data_ptr(), t.shape[0], 1, t.stride(0), 1
    if t.dim() != 2:
        raise ValueError("device views are 1-D or 2-D")
    return t.data_ptr(), t.shape[0], t.shape[1], t.stride(0), t.stride(1)


def _index_ptr(idx, count: int):
    """Device pointer of a contiguous 32-bit index list of `count` entries, or None."""
    if idx is None:
        return None
    if idx.numel() != count or not idx.is_contiguous() or idx.element_size() != 4 or not idx.is_cuda:
        raise ValueError("index lists are contiguous 32-bit CUDA tensors, one entry per output row / column")
    return idx.data_ptr()


class Engine:
    """One libhme context: a device, a stream and the device workspace."""

    def __init__(self, device: int = 0):
        self._lib = _lib.lib()
        h = C.c_void_p()
        check(self._lib.hme_ctx_create(device, C.byref(h)))
        self._h = h
        self.device = device

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.hme_ctx_destroy(self._h)
            self._h = None

    def __del__(self):  # pragma: no cover - interpreter teardown order
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ---- context ------------------------------------------------------------
    def set_stream(self, stream_ptr: int | None) -> None:
        """Run on a cudaStream_t handle (0 / None = the CUDA legacy default stream)."""
        check(self._lib.hme_ctx_set_stream(self._h, C.c_void_p(stream_ptr or 0)))

    def use_own_stream(self) -> None:
        check(self._lib.hme_ctx_set_stream(self._h, self._lib.hme_ctx_own_stream(self._h)))

    def use_torch_stream(self) -> None:
        """Run on torch's current CUDA stream (so torch and libhme order their work)."""
        import torch

        self.set_stream(torch.cuda.current_stream(self.device).cuda_stream)

    def sync(self) -> None:
        check(self._lib.hme_ctx_sync(self._h))

    @property
    def launches(self) -> int:
        return int(self._lib.hme_ctx_launches(self._h))

    def set_timing(self, on: bool) -> None:
        check(self._lib.hme_ctx_set_timing(self._h, 1 if on else 0))

    def kernel_time(self, name: str | None = None) -> tuple[float, int]:
        """(total ms, launches) of one kernel name since the last timing reset."""
        ms, cnt = C.c_double(), C.c_uint64()
        check(self._lib.hme_ctx_kernel_time(self._h, name.encode() if name else None, C.byref(ms), C.byref(cnt)))
        return ms.value, cnt.value

    def timing_reset(self) -> None:
        check(self._lib.hme_ctx_timing_reset(self._h))

    # ---- GEMM -------------------------------------------------------------------
    def gemm(self, p: int, A, B, C=None, op: int = SET, out: np.ndarray | None = None) -> np.ndarray:
        """C op= A*B mod p on host arrays (engine::kernels::gemm<uint32_t>).

        Returns a new array unless `out` (a C-contiguous uint32 m x n array,
        e.g. a pinned buffer) is given; for Add / Sub `out` starts as C."""
        A, B = _u32(A), _u32(B)
        m, k = A.shape
        k2, n = B.shape
        if k != k2:
            raise ValueError("gemm: inner dimensions differ")
        if out is None:
            out = np.zeros((m, n), np.uint32) if C is None else _u32(C).copy()
        else:
            if out.dtype != np.uint32 or out.shape != (m, n) or not out.flags.c_contiguous:
                raise ValueError("gemm: out must be a C-contiguous uint32 m x n array")
            if C is not None and op != SET:
                out[...] = C
        check(self._lib.hme_gemm_u32(self._h, p, m, n, k, _p32(A), k, _p32(B), n, _p32(out), n, op))
        return out

    def gemm_dev(self, p: int, A, B, C, op: int = SET) -> None:
        """C op= A*B mod p on CUDA tensors, asynchronous on the engine's stream."""
        m, k = A.shape
        n = B.shape[1]
        if B.shape[0] != k or tuple(C.shape) != (m, n):
            raise ValueError("gemm_dev: shape mismatch")
        check(self._lib.hme_gemm_u32_dev(self._h, p, m, n, k, _dev_ptr(A), A.stride(0), _dev_ptr(B), B.stride(0),
                                         _dev_ptr(C), C.stride(0), op))

    # ---- GEMM over u64 residues (engine::kernels::gemm<uint64_t>, Kernels.h:178-185) ----
    def gemm_u64(self, p: int, A, B, C=None, op: int = SET) -> np.ndarray:
        """C op= A*B mod p on host uint64 arrays, any modulus 2 <= p < 2^64 (canonical inputs)."""
        A = np.ascontiguousarray(A, dtype=np.uint64)
        B = np.ascontiguousarray(B, dtype=np.uint64)
        m, k = A.shape
        k2, n = B.shape
        if k != k2:
            raise ValueError("gemm_u64: inner dimensions differ")
        out = np.zeros((m, n), np.uint64) if C is None else np.array(C, dtype=np.uint64, copy=True)
        check(self._lib.hme_gemm_u64(self._h, p, m, n, k, A.ctypes.data, max(k, 1), B.ctypes.data, max(n, 1),
                                     out.ctypes.data, max(n, 1), op))
        return out

    def gemm_u64_dev(self, p: int, A, B, C, op: int = SET) -> None:
        """C op= A*B mod p on CUDA int64 / uint64 tensors (row-major), asynchronous on the engine's stream."""
        for t in (A, B, C):
            if t.element_size() != 8 or t.dim() != 2 or t.stride(1) != 1 or not t.is_cuda:
                raise ValueError("gemm_u64_dev: 2-D CUDA 64-bit tensors with unit column stride")
        m, k = A.shape
        n = B.shape[1]
        if B.shape[0] != k or tuple(C.shape) != (m, n):
            raise ValueError("gemm_u64_dev: shape mismatch")
        check(self._lib.hme_gemm_u64_dev(self._h, p, m, n, k, A.data_ptr(), A.stride(0), B.data_ptr(), B.stride(0),
                                         C.data_ptr(), C.stride(0), op))

    # ---- device level-1 / level-2 operations (engine::cuda::*, src/Cuda/CudaKernels.h:120-247) ----
    def gemm_nt_dev(self, p: int, A, B, C, op: int = SET) -> None:
        """C op= A*B^T mod p with B given n x k (row-major)."""
        m, k = A.shape
        n = B.shape[0]
        if B.shape[1] != k or tuple(C.shape) != (m, n):
            raise ValueError("gemm_nt_dev: shape mismatch")
        check(self._lib.hme_gemm_nt_u32_dev(self._h, p, m, n, k, _dev_ptr(A), A.stride(0), _dev_ptr(B), B.stride(0),
                                            _dev_ptr(C), C.stride(0), op))

    def schur_update_dev(self, p: int, L, U, C) -> None:
        """C -= L*U mod p."""
        m, k = L.shape
        n = U.shape[1]
        if U.shape[0] != k or tuple(C.shape) != (m, n):
            raise ValueError("schur_update_dev: shape mismatch")
        check(self._lib.hme_schur_update_u32_dev(self._h, p, m, n, k, _dev_ptr(L), L.stride(0), _dev_ptr(U),
                                                 U.stride(0), _dev_ptr(C), C.stride(0)))

    def gemv_dev(self, p: int, A, x, y, op: int = SET) -> None:
        """y op= A*x mod p; A any strides, x (k,) / (k, 1) and y (m,) / (m, 1) views."""
        a, xv, yv = _view(A), _view(x), _view(y)
        m, k = a[1], a[2]
        if xv[1] != k or yv[1] != m or xv[2] != 1 or yv[2] != 1:
            raise ValueError("gemv_dev: shape mismatch")
        check(self._lib.hme_gemv_u32_dev(self._h, p, m, k, a[0], a[3], a[4], xv[0], xv[3], yv[0], yv[3], op))

    def axpy_dev(self, p: int, alpha: int, x, y, subtract: bool = False) -> None:
        """y = y +/- alpha*x mod p (equal-shape views, any strides)."""
        xv, yv = _view(x), _view(y)
        if xv[1:3] != yv[1:3]:
            raise ValueError("axpy_dev: shape mismatch")
        check(self._lib.hme_axpy_u32_dev(self._h, p, alpha, xv[1], xv[2], xv[0], xv[3], xv[4], yv[0], yv[3], yv[4],
                                         1 if subtract else 0))

    def scal_dev(self, p: int, alpha: int, x) -> None:
        """x = alpha*x mod p."""
        v = _view(x)
        check(self._lib.hme_scal_u32_dev(self._h, p, alpha, v[1], v[2], v[0], v[3], v[4]))

    def copy_dev(self, src, dst) -> None:
        s, d = _view(src), _view(dst)
        if s[1:3] != d[1:3]:
            raise ValueError("copy_dev: shape mismatch")
        check(self._lib.hme_copy_u32_dev(self._h, s[1], s[2], s[0], s[3], s[4], d[0], d[3], d[4]))

    def transpose_dev(self, src, dst) -> None:
        """dst(i, j) = src(j, i)."""
        s, d = _view(src), _view(dst)
        if (s[1], s[2]) != (d[2], d[1]):
            raise ValueError("transpose_dev: shape mismatch")
        check(self._lib.hme_transpose_u32_dev(self._h, d[1], d[2], s[0], s[3], s[4], d[0], d[3], d[4]))

    def fill_dev(self, x, value: int) -> None:
        v = _view(x)
        check(self._lib.hme_fill_u32_dev(self._h, v[1], v[2], v[0], v[3], v[4], value))

    def axpy_identity_dev(self, p: int, alpha: int, y, subtract: bool = False) -> None:
        """y(i, i) +/-= alpha for every diagonal cell of the window."""
        v = _view(y)
        check(self._lib.hme_axpy_identity_u32_dev(self._h, p, alpha, v[1], v[2], v[0], v[3], v[4],
                                                  1 if subtract else 0))

    def gather_dev(self, p: int, alpha: int, beta: int, a, row_off: int, cols, c, accumulate: bool = False,
                   rows=None) -> None:
        """c(i, t) [+]= alpha [row_off + r(i) == col(t)] + beta a(r(i), col(t)); r(i) = rows[i] or i,
        col(t) = cols[t] or t; `a` may be None (identity source)."""
        cv = _view(c)
        av = _view(a) if a is not None else (0, 0, 0, 0, 0)
        check(self._lib.hme_gather_u32_dev(self._h, p, alpha, beta, av[0] or None, av[1], av[2], av[3], av[4],
                                           row_off, _index_ptr(cols, cv[2]), _index_ptr(rows, cv[1]), cv[1], cv[2],
                                           cv[0], cv[3], cv[4], 1 if accumulate else 0))

    def canonicalise_dev(self, p: int, v) -> None:
        """v = v >= p ? v - p : v in place (entries below 2p)."""
        x = _view(v)
        check(self._lib.hme_canonicalise_u32_dev(self._h, p, x[1], x[2], x[0], x[3], x[4]))

    def canonicalise_acc64_dev(self, p: int, acc, dst) -> None:
        """dst = acc mod p for an int64 / uint64 accumulator view."""
        a, d = _view(acc, 8), _view(dst)
        if a[1:3] != d[1:3]:
            raise ValueError("canonicalise_acc64_dev: shape mismatch")
        check(self._lib.hme_canonicalise_acc64_u32_dev(self._h, p, a[1], a[2], a[0], a[3], a[4], d[0], d[3], d[4]))

    def trsm_unit_dev(self, p: int, T, B, lower: bool) -> None:
        """B <- T^-1 B mod p in place; T m x m unit lower / upper triangular (strict triangle read)."""
        m = T.shape[0]
        if T.shape[1] != m or B.shape[0] != m:
            raise ValueError("trsm_unit_dev: shape mismatch")
        check(self._lib.hme_trsm_unit_u32_dev(self._h, p, 1 if lower else 0, m, B.shape[1], _dev_ptr(T),
                                              T.stride(0), _dev_ptr(B), B.stride(0)))

    # ---- elimination over F_p ------------------------------------------------------
    def set_elim_options(self, panel: int = 0, rows_per_cta: int = 0, panel_ctas: int = 0, back_block: int = 0):
        check(self._lib.hme_ctx_set_elim_options(self._h, panel, rows_per_cta, panel_ctas, back_block))

    def set_elim_lookahead(self, on: bool) -> None:
        """Factor the next LU panel on a second stream during the current trailing update (tuning only)."""
        check(self._lib.hme_ctx_set_elim_lookahead(self._h, 1 if on else 0))

    def set_panel_kernel(self, mode: int) -> None:
        """LU panel kernel: 0 automatic (over a field the top-block path first, then a searching
        kernel), 1 cooperative grid kernel, 2 thread-block cluster kernel, 3 cluster kernel with
        1024 threads per CTA."""
        check(self._lib.hme_ctx_set_panel_kernel(self._h, mode))

    def elim_panel_stats(self) -> tuple[int, int]:
        """(panels settled by the top-block path, panels factored by a searching kernel) so far."""
        b, s = C.c_uint64(0), C.c_uint64(0)
        check(self._lib.hme_ctx_elim_panel_stats(self._h, C.byref(b), C.byref(s)))
        return b.value, s.value

    def rref(self, p: int, A):
        """(RREF(A), pivot columns): the reference's elim::rref result."""
        R = _u32(A).copy()
        m, n = R.shape
        piv = np.zeros(max(1, min(m, n)), np.uint32)
        rank = C.c_uint32()
        check(self._lib.hme_rref_u32(self._h, p, m, n, _p32(R), n, _p32(piv), C.byref(rank)))
        return R, piv[: rank.value].copy()

    def column_rank_profile(self, p: int, A) -> np.ndarray:
        A = _u32(A)
        m, n = A.shape
        piv = np.zeros(max(1, min(m, n)), np.uint32)
        rank = C.c_uint32()
        check(self._lib.hme_rank_profile_u32(self._h, p, m, n, _p32(A), n, _p32(piv), C.byref(rank)))
        return piv[: rank.value].copy()

    def rank(self, p: int, A) -> int:
        return len(self.column_rank_profile(p, A))

    def det(self, p: int, A) -> int:
        A = _u32(A)
        n = A.shape[0]
        if A.shape != (n, n):
            raise ValueError("det: square matrix required")
        d = C.c_uint32()
        check(self._lib.hme_det_u32(self._h, p, n, _p32(A), n, C.byref(d)))
        return d.value

    def rref_det(self, p: int, A):
        """(RREF, pivots, det) of a square matrix from one factorisation."""
        R = _u32(A).copy()
        n = R.shape[0]
        piv = np.zeros(max(1, n), np.uint32)
        rank, d = C.c_uint32(), C.c_uint32()
        check(self._lib.hme_rref_det_u32(self._h, p, n, _p32(R), n, _p32(piv), C.byref(rank), C.byref(d)))
        return R, piv[: rank.value].copy(), d.value

    def kernel_basis(self, p: int, A) -> np.ndarray:
        A = _u32(A)
        m, n = A.shape
        K = np.zeros((max(1, n), n), np.uint32)
        f = C.c_uint32()
        check(self._lib.hme_kernel_basis_u32(self._h, p, m, n, _p32(A), n, _p32(K), n, C.byref(f)))
        return K[: f.value].copy()

    def inverse(self, p: int, A):
        A = _u32(A)
        n = A.shape[0]
        X = np.zeros((n, n), np.uint32)
        ok = C.c_int()
        check(self._lib.hme_inverse_u32(self._h, p, n, _p32(A), n, _p32(X), n, C.byref(ok)))
        return X if ok.value else None

    def solve_multi_rhs(self, p: int, B, Y):
        """X with B X = Y (nb x ny), or None when some column of Y is outside span(B)."""
        B, Y = _u32(B), _u32(Y)
        m, nb = B.shape
        ny = Y.shape[1]
        X = np.zeros((max(1, nb), max(1, ny)), np.uint32)
        rc = self._lib.hme_solve_u32(self._h, p, m, nb, ny, _p32(B), nb, _p32(Y), ny, _p32(X), max(1, ny))
        if rc == _lib.HME_ENOTINSPAN:
            return None
        check(rc)
        return X[:nb, :ny].copy()

    def rref_dev(self, p: int, A):
        """In-place RREF of a CUDA tensor (m x n, int32/uint32 words); returns the pivots."""
        m, n = A.shape
        piv = np.zeros(max(1, min(m, n)), np.uint32)
        rank = C.c_uint32()
        check(self._lib.hme_rref_u32_dev(self._h, p, m, n, _dev_ptr(A), A.stride(0), _p32(piv), C.byref(rank)))
        return piv[: rank.value].copy()

    # ---- Z/ell^k --------------------------------------------------------------------------
    def howell(self, ell: int, k: int, A):
        """(H, pivots, pivot_v): the Howell form of rowspan(A) over Z/ell^k."""
        A = _u32(A)
        m, n = A.shape
        H = np.zeros((max(1, n), max(1, n)), np.uint32)
        piv = np.zeros(max(1, n), np.uint32)
        pv = np.zeros(max(1, n), np.uint32)
        h = C.c_uint32()
        check(self._lib.hme_howell_u32(self._h, ell, k, m, n, _p32(A), max(1, n), _p32(H), max(1, n), _p32(piv),
                                       _p32(pv), C.byref(h)))
        return H[: h.value, :n].copy(), piv[: h.value].copy(), pv[: h.value].copy()

    def smith(self, ell: int, k: int, A) -> np.ndarray:
        """Smith valuations sigma (ascending, each < k) of A over Z/ell^k."""
        A = _u32(A)
        m, n = A.shape
        s = np.zeros(max(1, min(m, n)), np.uint32)
        cnt = C.c_uint32()
        check(self._lib.hme_smith_u32(self._h, ell, k, m, n, _p32(A), max(1, n), _p32(s), C.byref(cnt)))
        return s[: cnt.value].copy()

    def invariant_factors(self, ell: int, k: int, A) -> np.ndarray:
        """elim::invariant_factors: the exponents k - sigma, descending."""
        return np.sort(k - self.smith(ell, k, A).astype(np.int64))[::-1].astype(np.uint32)

    # ---- batched job stream -----------------------------------------------------------------
    @staticmethod
    def _jobs(jobs):
        arr = (_lib.HmeJob * max(1, len(jobs)))()
        for t, j in enumerate(jobs):
            A, B, Cm, p = j["A"], j["B"], j["C"], j["p"]
            m, n = Cm.shape
            k = A.shape[1] if A is not None else 0
            arr[t] = _lib.HmeJob(p, m, n, k, A.data_ptr() if A is not None else None, A.stride(0) if A is not None else 0,
                                 B.data_ptr() if B is not None else None, B.stride(0) if B is not None else 0,
                                 Cm.data_ptr(), Cm.stride(0))
        return arr

    def batch_gemm_dev(self, jobs) -> None:
        """Every C_j = A_j B_j mod p_j (jobs: dicts with CUDA tensors A, B, C and p)."""
        arr = self._jobs(jobs)
        check(self._lib.hme_batch_gemm_u32_dev(self._h, len(jobs), arr))

    @staticmethod
    def _variants(v, n):
        if v is None:
            return None
        a = np.ascontiguousarray(np.broadcast_to(np.asarray(v, dtype=np.int32), (n,)))
        return a

    def batch_rank_dev(self, jobs, rank_variants=None) -> np.ndarray:
        """rank of each C_j over F_{p_j} (destroys C_j).  rank_variants: per-job
        schedules of the rank rounds (0..3, -1 the batch rule; a scalar applies to
        every job; None: the context's scheduler)."""
        arr = self._jobs(jobs)
        ranks = np.zeros(max(1, len(jobs)), np.uint32)
        rv = self._variants(rank_variants, len(jobs))
        if rv is None:
            check(self._lib.hme_batch_rank_u32_dev(self._h, len(jobs), arr, _p32(ranks)))
        else:
            check(self._lib.hme_batch_rank_u32_dev_sched(self._h, len(jobs), arr,
                                                         rv.ctypes.data_as(C.POINTER(C.c_int)), _p32(ranks)))
        return ranks[: len(jobs)].copy()

    def batch_gemm_rank_dev(self, jobs, gemm_variants=None, rank_variants=None) -> np.ndarray:
        """C_j = A_j B_j mod p_j, then rank(C_j): the GEMM phase under per-job GEMM
        schedules, the rank phase under per-job rank schedules (None: the
        context's scheduler for that phase)."""
        arr = self._jobs(jobs)
        ranks = np.zeros(max(1, len(jobs)), np.uint32)
        if gemm_variants is None and rank_variants is None:
            check(self._lib.hme_batch_gemm_rank_u32_dev(self._h, len(jobs), arr, _p32(ranks)))
        else:
            gv = self._variants(gemm_variants, len(jobs))
            rv = self._variants(rank_variants, len(jobs))
            ip = C.POINTER(C.c_int)
            check(self._lib.hme_batch_gemm_rank_u32_dev_sched(
                self._h, len(jobs), arr, gv.ctypes.data_as(ip) if gv is not None else None,
                rv.ctypes.data_as(ip) if rv is not None else None, _p32(ranks)))
        return ranks[: len(jobs)].copy()

    def gen_jobs_dev(self, specs) -> None:
        """Fill CUDA tensors with the seeded job-stream matrices: specs are
        (tensor, p, family, seed) tuples."""
        arr = (_lib.HmeGenSpec * max(1, len(specs)))()
        for t, (T, p, fam, seed) in enumerate(specs):
            arr[t] = _lib.HmeGenSpec(T.data_ptr(), T.stride(0), T.shape[0], T.shape[1], p, fam, int(seed))
        check(self._lib.hme_gen_jobs_u32_dev(self._h, len(specs), arr))
