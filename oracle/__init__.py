"""ORACLE / TEST INFRASTRUCTURE ONLY.

numpy wrappers over the two CPU checkers of the exact modular matrix engine:

* ``liboracle.so`` -- the plain-C restatement of the reference's algorithms
  (oracle.c; each function cites the reference file:line it follows);
* ``_ref/libhacsref.so`` -- the reference's own CPU engine (drjanosch42/hacs
  0.2.1, src/ModArithmetic), compiled from its sources by oracle/Makefile,
  reached through the shim ref_shim.cpp.  Present only where the reference
  sources were available at build time; ``ref_available()`` says whether.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's cpu_baseline leg may
import this package.  The product library never calls into it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_ORC = None
_REF = None
# Where the reference's sources lie (only the build of oracle/_ref reads them).
REFERENCE = os.environ.get("HACS_REFERENCE", "/root/reference")

u32p = C.POINTER(C.c_uint32)


def build(with_ref: bool | None = None) -> None:
    """Compile liboracle.so, and the reference library when its sources exist."""
    subprocess.check_call(["make", "-s", "-C", HERE], stdout=subprocess.DEVNULL)
    if with_ref is None:
        with_ref = os.path.isdir(os.path.join(REFERENCE, "src", "ModArithmetic"))
    if with_ref:
        subprocess.check_call(["make", "-s", "-j8", "-C", HERE, "ref", f"REF={REFERENCE}"], stdout=subprocess.DEVNULL)


def _p(a: np.ndarray):
    return a.ctypes.data_as(u32p)


def lib():
    global _ORC
    if _ORC is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build(with_ref=False)
        L = C.CDLL(path)
        L.orc_splitmix64.restype = C.c_uint64
        L.orc_seed_for.restype = C.c_uint64
        L.orc_seed_for.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint64]
        L.orc_random_entries.argtypes = [u32p, C.c_uint64, C.c_uint32, C.c_uint64]
        L.orc_fnv_matrix.restype = C.c_uint64
        L.orc_fnv_matrix.argtypes = [u32p, C.c_uint32, C.c_uint32, C.c_uint32]
        L.orc_gemm_u32.argtypes = [C.c_uint32] * 4 + [u32p, C.c_uint32, u32p, C.c_uint32, u32p, C.c_uint32, C.c_int]
        u64p_ = C.POINTER(C.c_uint64)
        L.orc_gemm_u64.argtypes = [C.c_uint64] + [C.c_uint32] * 3 + [u64p_, C.c_uint32, u64p_, C.c_uint32, u64p_,
                                                                       C.c_uint32, C.c_int]
        L.orc_rref_u32.restype = C.c_int64
        L.orc_rref_u32.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32, u32p, C.c_uint32, u32p]
        L.orc_det_u32.restype = C.c_int64
        L.orc_det_u32.argtypes = [C.c_uint32, C.c_uint32, u32p, C.c_uint32]
        L.orc_kernel_basis_u32.argtypes = [C.c_uint32, C.c_uint32, u32p, C.c_uint32, u32p, C.c_uint32, u32p]
        L.orc_inverse_u32.argtypes = [C.c_uint32, C.c_uint32, u32p, u32p]
        L.orc_solve_u32.argtypes = [C.c_uint32] * 4 + [u32p, u32p, u32p]
        L.orc_howell_u32.restype = C.c_int64
        L.orc_howell_u32.argtypes = [C.c_uint32] * 4 + [u32p, C.c_uint32, u32p, u32p, u32p]
        L.orc_smith_u32.restype = C.c_int64
        L.orc_smith_u32.argtypes = [C.c_uint32] * 4 + [u32p, C.c_uint32, u32p]
        L.orc_inv_mod.restype = C.c_uint32
        L.orc_inv_mod.argtypes = [C.c_uint32, C.c_uint32]
        _ORC = L
    return _ORC


def ref_path() -> str:
    return os.path.join(HERE, "_ref", "libhacsref.so")


def ref_available() -> bool:
    return os.path.exists(ref_path())


def ref():
    """The reference's compiled CPU engine (raises if it was not built)."""
    global _REF
    if _REF is None:
        L = C.CDLL(ref_path())
        L.ref_last_error.restype = C.c_char_p
        L.ref_gemm_u32.argtypes = [C.c_uint32] * 4 + [u32p, C.c_uint32, u32p, C.c_uint32, u32p, C.c_uint32,
                                                      C.c_int, C.c_int]
        L.ref_rref_u32.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32, u32p, C.c_uint32, u32p, u32p]
        L.ref_rank_profile_u32.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32, u32p, C.c_uint32, u32p, u32p]
        L.ref_kernel_basis_u32.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32, u32p, C.c_uint32, u32p,
                                           C.c_uint32, u32p]
        L.ref_inverse_u32.argtypes = [C.c_uint32, C.c_uint32, u32p, u32p, C.POINTER(C.c_int)]
        L.ref_elim_howell_u32.argtypes = [C.c_uint32] * 4 + [u32p] * 4 + [u32p]
        L.ref_howell_2k_u32.argtypes = [C.c_uint32] * 3 + [u32p] * 5 + [C.c_int]
        L.ref_smith_2k_u32.argtypes = [C.c_uint32] * 3 + [u32p, u32p, u32p, C.c_int]
        L.ref_smith_3k_u32.argtypes = [C.c_uint32] * 3 + [u32p, u32p, u32p, C.c_int]
        L.ref_howell_3k_u32.argtypes = [C.c_uint32] * 3 + [u32p] * 5 + [C.c_int]
        u32 = C.c_uint32
        u64p = C.POINTER(C.c_uint64)
        L.ref_gemm_nt_u32.argtypes = [u32] * 4 + [u32p, u32, u32p, u32, u32p, u32, C.c_int]
        L.ref_gemv_u32.argtypes = [u32] * 3 + [u32p, u32, u32p, u32p, C.c_int]
        L.ref_axpy_scal_u32.argtypes = [u32] * 4 + [u32p, u32, u32p, u32, C.c_int]
        L.ref_trmm_unit_u32.argtypes = [u32, C.c_int, u32, u32, u32p, u32, u32p, u32, u32p, u32]
        L.ref_transpose_u32.argtypes = [u32, u32, u32p, u32, u32p, u32]
        L.ref_canonicalise_u32.argtypes = [u32] * 3 + [u32p, u32]
        L.ref_canonicalise_acc64_u32.argtypes = [u32] * 3 + [u64p, u32, u32p, u32]
        L.ref_gemm_u64.argtypes = [C.c_uint64, u32, u32, u32, u64p, u32, u64p, u32, u64p, u32, C.c_int]
        if hasattr(L, "ref_tape_gemm_u32"):
            L.ref_tape_gemm_u32.argtypes = [u32] * 4 + [u32p, u32p, u32p, C.c_int, C.c_int,
                                                        C.POINTER(C.c_double)]
            L.ref_rref_par_u32.argtypes = [u32, u32, u32, u32p, u32, u32p, u32p, C.c_int]
        _REF = L
    return _REF


def _chk(rc: int, which: str = "oracle") -> None:
    if rc < 0:
        msg = ref().ref_last_error().decode() if which == "ref" else "contract violation"
        raise RuntimeError(f"{which} call failed ({rc}): {msg}")


def _u32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.uint32)


# ---- generators -------------------------------------------------------------
def seed_for(r: int, c: int, ell: int, salt: int) -> int:
    return int(lib().orc_seed_for(r, c, ell, salt))


def random_entries(count: int, ell: int, seed: int) -> np.ndarray:
    out = np.empty(count, dtype=np.uint32)
    lib().orc_random_entries(_p(out), count, ell, seed)
    return out


def engine_matrix(rows: int, cols: int, ell: int, salt: int) -> np.ndarray:
    """EngineMatrixImpl(rows, cols, ell, salt): PerformanceSmokeValidation.cpp:329-337."""
    return random_entries(rows * cols, ell, seed_for(rows, cols, ell, salt)).reshape(rows, cols)


def fnv_matrix(M: np.ndarray) -> int:
    M = _u32(M)
    return int(lib().orc_fnv_matrix(_p(M), M.shape[0], M.shape[1], M.shape[1]))


# ---- restatement ---------------------------------------------------------------
def gemm(p: int, A, B, C=None, op: int = 0) -> np.ndarray:
    A, B = _u32(A), _u32(B)
    m, k = A.shape
    n = B.shape[1]
    Cm = np.zeros((m, n), np.uint32) if C is None else _u32(C).copy()
    _chk(lib().orc_gemm_u32(p, m, n, k, _p(A), k, _p(B), n, _p(Cm), n, op))
    return Cm


def rref(p: int, A):
    R = _u32(A).copy()
    m, n = R.shape
    piv = np.zeros(max(1, min(m, n)), np.uint32)
    r = lib().orc_rref_u32(p, m, n, _p(R), n, _p(piv))
    _chk(r)
    return R, piv[:r].copy()


def det(p: int, A) -> int:
    A = _u32(A)
    r = lib().orc_det_u32(p, A.shape[0], _p(A), A.shape[1])
    _chk(r)
    return int(r)


def kernel_basis(p: int, R, pivots) -> np.ndarray:
    R = _u32(R)
    pv = _u32(pivots)
    n = R.shape[1]
    K = np.zeros((n - len(pv), n), np.uint32)
    lib().orc_kernel_basis_u32(p, n, _p(R), n, _p(pv), len(pv), _p(K))
    return K


def inverse(p: int, A):
    A = _u32(A)
    n = A.shape[0]
    X = np.zeros((n, n), np.uint32)
    ok = lib().orc_inverse_u32(p, n, _p(A), _p(X))
    return X if ok == 1 else None


def solve(p: int, B, Y):
    B, Y = _u32(B), _u32(Y)
    m, nb = B.shape
    ny = Y.shape[1]
    X = np.zeros((nb, ny), np.uint32)
    rc = lib().orc_solve_u32(p, m, nb, ny, _p(B), _p(Y), _p(X))
    if rc == -3:
        return None
    _chk(rc)
    return X


def howell(ell: int, k: int, A):
    A = _u32(A)
    m, n = A.shape
    H = np.zeros((max(1, n), n), np.uint32)
    piv = np.zeros(max(1, n), np.uint32)
    pv = np.zeros(max(1, n), np.uint32)
    h = lib().orc_howell_u32(ell, k, m, n, _p(A), n, _p(H), _p(piv), _p(pv))
    _chk(h)
    return H[:h].copy(), piv[:h].copy(), pv[:h].copy()


def smith(ell: int, k: int, A) -> np.ndarray:
    A = _u32(A)
    m, n = A.shape
    s = np.zeros(max(1, min(m, n)), np.uint32)
    c = lib().orc_smith_u32(ell, k, m, n, _p(A), n, _p(s))
    _chk(c)
    return s[:c].copy()


# ---- the reference's own engine ----------------------------------------------------
def ref_gemm(p: int, A, B, C=None, op: int = 0, threads: int = 1) -> np.ndarray:
    A, B = _u32(A), _u32(B)
    m, k = A.shape
    n = B.shape[1]
    Cm = np.zeros((m, n), np.uint32) if C is None else _u32(C).copy()
    _chk(ref().ref_gemm_u32(p, m, n, k, _p(A), k, _p(B), n, _p(Cm), n, op, threads), "ref")
    return Cm


def ref_rref(p: int, A):
    R = _u32(A).copy()
    m, n = R.shape
    piv = np.zeros(max(1, min(m, n)), np.uint32)
    rank = C.c_uint32(0)
    _chk(ref().ref_rref_u32(p, m, n, _p(R), n, _p(piv), C.byref(rank)), "ref")
    return R, piv[: rank.value].copy()


def ref_tape_gemm(p: int, A, B, threads: int = 1, reps: int = 1):
    """C = A*B mod p through the reference's tape (Recorder::gemm, compile, Executor::run on a
    pool of `threads` workers, run `reps` times); returns (C, mean seconds per run)."""
    A, B = _u32(A), _u32(B)
    m, k = A.shape
    n = B.shape[1]
    Cm = np.zeros((m, n), np.uint32)
    secs = C.c_double(0.0)
    _chk(ref().ref_tape_gemm_u32(p, m, n, k, _p(A), _p(B), _p(Cm), threads, reps, C.byref(secs)), "ref")
    return Cm, secs.value


def ref_rref_par(p: int, A, threads: int = 1):
    """elim::rref under the tape's host elimination hook on a pool of `threads` workers."""
    R = _u32(A).copy()
    m, n = R.shape
    piv = np.zeros(max(1, min(m, n)), np.uint32)
    rank = C.c_uint32(0)
    _chk(ref().ref_rref_par_u32(p, m, n, _p(R), n, _p(piv), C.byref(rank), threads), "ref")
    return R, piv[: rank.value].copy()


def ref_job(spec):
    """One job of the batched stream on the reference CPU engine, one thread:
    spec = (j, side, family, p, seed_a, seed_b); A, B from gen.job_matrix,
    C = kernels::gemm(A, B), rank = |elim::column_rank_profile(C)|.  Returns
    (j, rank, FNV-1a-64 of C).  A module-level function so that process pools
    (started with spawn) can run it."""
    from hacs_b200 import gen

    j, s, fam, p, sa, sb = spec
    A = gen.job_matrix(s, s, p, fam, sa)
    B = gen.job_matrix(s, s, p, fam, sb)
    Cm = ref_gemm(p, A, B)
    return j, len(ref_rank_profile(p, Cm)), fnv_matrix(Cm)


def ref_rank_profile(p: int, A):
    R = _u32(A).copy()
    m, n = R.shape
    piv = np.zeros(max(1, min(m, n)), np.uint32)
    rank = C.c_uint32(0)
    _chk(ref().ref_rank_profile_u32(p, m, n, _p(R), n, _p(piv), C.byref(rank)), "ref")
    return piv[: rank.value].copy()


def ref_kernel_basis(p: int, R, pivots) -> np.ndarray:
    R = _u32(R)
    pv = _u32(pivots)
    n = R.shape[1]
    K = np.zeros((max(1, n - len(pv)), n), np.uint32)
    _chk(ref().ref_kernel_basis_u32(p, R.shape[0], n, _p(R), n, _p(pv), len(pv), _p(K)), "ref")
    return K[: n - len(pv)]


def ref_inverse(p: int, A):
    A = _u32(A)
    n = A.shape[0]
    X = np.zeros((n, n), np.uint32)
    ok = C.c_int(0)
    _chk(ref().ref_inverse_u32(p, n, _p(A), _p(X), C.byref(ok)), "ref")
    return X if ok.value else None


def _howell_out(n):
    return (np.zeros((max(1, n), n), np.uint32), np.zeros(max(1, n), np.uint32), np.zeros(max(1, n), np.uint32))


def ref_elim_howell(ell: int, k: int, A):
    A = _u32(A)
    m, n = A.shape
    H, piv, pv = _howell_out(n)
    h = C.c_uint32(0)
    _chk(ref().ref_elim_howell_u32(ell, k, m, n, _p(A), _p(H), _p(piv), _p(pv), C.byref(h)), "ref")
    return H[: h.value].copy(), piv[: h.value].copy(), pv[: h.value].copy()


def ref_howell_2k(k: int, A, threads: int = 1):
    A = _u32(A)
    m, n = A.shape
    H, piv, pv = _howell_out(n)
    h = C.c_uint32(0)
    _chk(ref().ref_howell_2k_u32(k, m, n, _p(A), _p(H), _p(piv), _p(pv), C.byref(h), threads), "ref")
    return H[: h.value].copy(), piv[: h.value].copy(), pv[: h.value].copy()


def ref_howell_3k(k: int, A, threads: int = 1):
    A = _u32(A)
    m, n = A.shape
    H, piv, pv = _howell_out(n)
    h = C.c_uint32(0)
    _chk(ref().ref_howell_3k_u32(k, m, n, _p(A), _p(H), _p(piv), _p(pv), C.byref(h), threads), "ref")
    return H[: h.value].copy(), piv[: h.value].copy(), pv[: h.value].copy()


def ref_smith_2k(k: int, A, threads: int = 1) -> np.ndarray:
    A = _u32(A)
    m, n = A.shape
    s = np.zeros(max(1, min(m, n)), np.uint32)
    c = C.c_uint32(0)
    _chk(ref().ref_smith_2k_u32(k, m, n, _p(A), _p(s), C.byref(c), threads), "ref")
    return s[: c.value].copy()


def ref_smith_3k(k: int, A, threads: int = 1) -> np.ndarray:
    A = _u32(A)
    m, n = A.shape
    s = np.zeros(max(1, min(m, n)), np.uint32)
    c = C.c_uint32(0)
    _chk(ref().ref_smith_3k_u32(k, m, n, _p(A), _p(s), C.byref(c), threads), "ref")
    return s[: c.value].copy()


# ---- the reference's level-1 / level-2 CPU kernels (Kernels.h:188-259) -------------
def ref_gemm_nt(p: int, A, B, C, op: int) -> np.ndarray:
    A, B = _u32(A), _u32(B)
    m, k = A.shape
    n = B.shape[0]
    Cm = _u32(C).copy()
    _chk(ref().ref_gemm_nt_u32(p, m, n, k, _p(A), max(k, 1), _p(B), max(k, 1), _p(Cm), n, op), "ref")
    return Cm


def ref_gemv(p: int, A, x, y, op: int) -> np.ndarray:
    A, x = _u32(A), _u32(np.reshape(x, -1))
    m, k = A.shape
    yv = _u32(np.reshape(y, -1)).copy()
    _chk(ref().ref_gemv_u32(p, m, k, _p(A), k, _p(x), _p(yv), op), "ref")
    return yv


def ref_axpy(p: int, alpha: int, x, y, subtract: bool) -> np.ndarray:
    x = _u32(x).copy()
    yv = _u32(y).copy()
    r, c = x.shape
    _chk(ref().ref_axpy_scal_u32(p, alpha, r, c, _p(x), c, _p(yv), c, 1 if subtract else 0), "ref")
    return yv


def ref_scal(p: int, alpha: int, x) -> np.ndarray:
    xv = _u32(x).copy()
    r, c = xv.shape
    _chk(ref().ref_axpy_scal_u32(p, alpha, r, c, _p(xv), c, None, c, 0), "ref")
    return xv


def ref_trmm_unit(p: int, T, B, lower: bool) -> np.ndarray:
    T, B = _u32(T), _u32(B)
    m, n = B.shape
    Cm = np.zeros((m, n), np.uint32)
    _chk(ref().ref_trmm_unit_u32(p, 1 if lower else 0, m, n, _p(T), m, _p(B), n, _p(Cm), n), "ref")
    return Cm


def ref_transpose(A) -> np.ndarray:
    A = _u32(A)
    r, c = A.shape
    T = np.zeros((c, r), np.uint32)
    _chk(ref().ref_transpose_u32(r, c, _p(A), c, _p(T), r), "ref")
    return T


def ref_canonicalise(p: int, v) -> np.ndarray:
    v = _u32(v).copy()
    r, c = v.shape
    _chk(ref().ref_canonicalise_u32(p, r, c, _p(v), c), "ref")
    return v


def ref_canonicalise_acc64(p: int, acc) -> np.ndarray:
    acc = np.ascontiguousarray(acc, dtype=np.uint64)
    r, c = acc.shape
    d = np.zeros((r, c), np.uint32)
    _chk(ref().ref_canonicalise_acc64_u32(p, r, c, acc.ctypes.data_as(C.POINTER(C.c_uint64)), c, _p(d), c), "ref")
    return d


# ---- u64 residues ------------------------------------------------------------------
def _u64a(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.uint64)


def _p64(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_uint64))


def gemm_u64(p: int, A, B, C_=None, op: int = 0) -> np.ndarray:
    """C op= A*B mod p over u64 residues (restatement, oracle.c orc_gemm_u64)."""
    A, B = _u64a(A), _u64a(B)
    m, k = A.shape
    n = B.shape[1]
    Cm = np.zeros((m, n), np.uint64) if C_ is None else _u64a(C_).copy()
    _chk(lib().orc_gemm_u64(p, m, n, k, _p64(A), max(k, 1), _p64(B), max(n, 1), _p64(Cm), max(n, 1), op))
    return Cm


def ref_gemm_u64(p: int, A, B, C_=None, op: int = 0) -> np.ndarray:
    """The reference's kernels::gemm<uint64_t> (oracle/_ref)."""
    A, B = _u64a(A), _u64a(B)
    m, k = A.shape
    n = B.shape[1]
    Cm = np.zeros((m, n), np.uint64) if C_ is None else _u64a(C_).copy()
    _chk(ref().ref_gemm_u64(p, m, n, k, _p64(A), max(k, 1), _p64(B), max(n, 1), _p64(Cm), max(n, 1), op), "ref")
    return Cm
