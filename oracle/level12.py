"""ORACLE / TEST INFRASTRUCTURE ONLY.

numpy restatements of the reference's device level-1 / level-2 operations
(engine::cuda::*, declared in src/Cuda/CudaKernels.h:120-247, bodies in
src/Cuda/cuda_kernels.cu:952-1130), for the parity tests of the device entry
points.  Integer arithmetic only: every product of two residues below
p < 2^32 fits uint64 and is reduced before it is summed; the dot products go
through the C oracle's GEMM (oracle.gemm).  Only tests/ import this module.
"""
from __future__ import annotations

import numpy as np

from . import gemm

SET, ADD, SUB = 0, 1, 2


def _u64(a) -> np.ndarray:
    return np.asarray(a, dtype=np.uint64)


def _apply(p: int, old, v, op: int) -> np.ndarray:
    old, v = _u64(old), _u64(v)
    if op == SET:
        out = v
    elif op == ADD:
        out = (old + v) % p
    else:
        out = (old + p - v) % p
    return out.astype(np.uint32)


def gemv(p: int, A, x, y, op: int) -> np.ndarray:
    """y op= A x (CudaKernels.h:189-192, cuda_kernels.cu:952-984)."""
    v = gemm(p, np.ascontiguousarray(A, np.uint32), np.ascontiguousarray(np.reshape(x, (-1, 1)), np.uint32))
    return _apply(p, np.reshape(y, (-1,)), v[:, 0], op)


def axpy(p: int, alpha: int, x, y, subtract: bool) -> np.ndarray:
    """y +/- alpha x (cuda_kernels.cu:986-998)."""
    ax = (_u64(x) * alpha) % p
    return _apply(p, y, ax, SUB if subtract else ADD)


def scal(p: int, alpha: int, x) -> np.ndarray:
    """alpha x (cuda_kernels.cu:1000-1008)."""
    return ((_u64(x) * alpha) % p).astype(np.uint32)


def axpy_identity(p: int, alpha: int, y, subtract: bool) -> np.ndarray:
    """y(i, i) +/- alpha for i < min(rows, cols) (cuda_kernels.cu:1062-1069)."""
    out = np.array(y, dtype=np.uint32, copy=True)
    n = min(out.shape)
    d = np.arange(n)
    out[d, d] = _apply(p, out[d, d], np.full(n, alpha, np.uint64), SUB if subtract else ADD)
    return out


def gather(p: int, alpha: int, beta: int, a, row_off: int, cols, c, accumulate: bool, rows=None) -> np.ndarray:
    """c(i, t) [+]= alpha [row_off + r(i) == col(t)] + beta a(r(i), col(t)),
    r(i) = rows[i] or i, col(t) = cols[t] or t (CudaKernels.h:221-231,
    cuda_kernels.cu:1071-1088)."""
    c = np.asarray(c, dtype=np.uint32)
    nr, nc = c.shape
    r = np.arange(nr, dtype=np.uint64) if rows is None else _u64(rows)
    col = np.arange(nc, dtype=np.uint64) if cols is None else _u64(cols)
    v = np.zeros((nr, nc), np.uint64)
    if a is not None and beta != 0:
        v = (_u64(np.asarray(a)[np.ix_(r.astype(np.int64), col.astype(np.int64))]) * beta) % p
    if alpha != 0:
        hit = (np.uint64(row_off) + r)[:, None] == col[None, :]
        v = np.where(hit, (v + alpha) % p, v)
    return _apply(p, c, v, ADD if accumulate else SET)


def canonicalise(p: int, v) -> np.ndarray:
    """v >= p ? v - p : v (cuda_kernels.cu:1010-1017)."""
    v = _u64(v)
    return np.where(v >= p, v - p, v).astype(np.uint32)


def canonicalise_acc64(p: int, acc) -> np.ndarray:
    """acc mod p for 64-bit accumulators (cuda_kernels.cu:1019-1027)."""
    return (_u64(acc) % p).astype(np.uint32)


def trsm_unit(p: int, T, B, lower: bool) -> np.ndarray:
    """T^-1 B with T unit lower / upper triangular, only the strict triangle
    read (CudaKernels.h:240-247, cuda_kernels.cu:1090-1130): row-by-row
    substitution, X(i) = B(i) - sum over the solved rows s of T(i, s) X(s)."""
    T = np.asarray(T, dtype=np.uint32)
    X = np.array(B, dtype=np.uint32, copy=True)
    m = T.shape[0]
    for i in range(m) if lower else range(m - 1, -1, -1):
        if lower and i > 0:
            s = gemm(p, np.ascontiguousarray(T[i : i + 1, :i]), np.ascontiguousarray(X[:i]))[0]
        elif not lower and i < m - 1:
            s = gemm(p, np.ascontiguousarray(T[i : i + 1, i + 1 :]), np.ascontiguousarray(X[i + 1 :]))[0]
        else:
            continue
        X[i] = _apply(p, X[i], s, SUB)
    return X


def gemm_nt(p: int, A, B, C, op: int) -> np.ndarray:
    """C op= A B^T with B given n x k (CudaKernels.h:126-129)."""
    return gemm(p, np.ascontiguousarray(A, np.uint32), np.ascontiguousarray(np.asarray(B, np.uint32).T),
                np.asarray(C, np.uint32), op)


# ---- the u64 element type (any modulus below 2^64): exact Python integers ----------------------
def _obj(a) -> np.ndarray:
    return np.asarray(a, dtype=np.uint64).astype(object)


def axpy64(p: int, alpha: int, x, y, subtract: bool) -> np.ndarray:
    """y +/- alpha x mod p over u64 residues (kernels::axpy<uint64_t>, the uint64_t twin of the above)."""
    v = (_obj(y) - alpha * _obj(x)) % p if subtract else (_obj(y) + alpha * _obj(x)) % p
    return v.astype(np.uint64)


def scal64(p: int, alpha: int, x) -> np.ndarray:
    return ((alpha * _obj(x)) % p).astype(np.uint64)


def axpy_identity64(p: int, alpha: int, y, subtract: bool) -> np.ndarray:
    out = _obj(y)
    n = min(out.shape)
    for i in range(n):
        out[i, i] = (out[i, i] - alpha) % p if subtract else (out[i, i] + alpha) % p
    return out.astype(np.uint64)


def gather64(p: int, alpha: int, beta: int, a, row_off: int, cols, c, accumulate: bool, rows=None) -> np.ndarray:
    c = _obj(c)
    nr, nc = c.shape
    r = list(range(nr)) if rows is None else [int(x) for x in rows]
    col = list(range(nc)) if cols is None else [int(x) for x in cols]
    A = None if a is None else _obj(a)
    out = np.empty((nr, nc), dtype=object)
    for i in range(nr):
        for t in range(nc):
            v = alpha if row_off + r[i] == col[t] else 0
            if A is not None:
                v = (v + beta * A[r[i], col[t]]) % p
            out[i, t] = (c[i, t] + v) % p if accumulate else v
    return out.astype(np.uint64)


def canonicalise64(p: int, v) -> np.ndarray:
    v = _obj(v)
    return np.where(v >= p, v - p, v).astype(np.uint64)
