"""Seeded input generators of the reference's benchmarks, vectorised.

splitmix64 / SeedFor / RandomEntries / EngineMatrixImpl follow
src/ModArithmetic/PerformanceSmokeValidation.cpp:64-88 and :329-337 of the
reference; the FNV-1a-64 matrix checksum follows :104-120 and
src/ModArithmetic/Fnv.h.  Element i of a splitmix64 stream seeded with s is
mix(s + (i + 1) * gamma), so a whole matrix is one vectorised expression.
"""
from __future__ import annotations

import numpy as np

GAMMA = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)
MASK64 = (1 << 64) - 1


def seed_for(r: int, c: int, ell: int, salt: int) -> int:
    s = 0xC0FFEE123456789 ^ salt
    s = (s * 0x100000001B3 + r) & MASK64
    s = (s * 0x100000001B3 + c) & MASK64
    s = (s * 0x100000001B3 + ell) & MASK64
    return s


def splitmix_stream(seed: int, count: int, start: int = 0) -> np.ndarray:
    """Outputs start .. start+count-1 of splitmix64 seeded with `seed`."""
    with np.errstate(over="ignore"):
        i = np.arange(start + 1, start + count + 1, dtype=np.uint64)
        z = np.uint64(seed) + i * GAMMA
        z = (z ^ (z >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
        return z ^ (z >> np.uint64(31))


def random_entries(count: int, ell: int, seed: int) -> np.ndarray:
    out = np.empty(count, dtype=np.uint32)
    step = 1 << 24
    for s0 in range(0, count, step):
        n = min(step, count - s0)
        out[s0:s0 + n] = (splitmix_stream(seed, n, s0) % np.uint64(ell)).astype(np.uint32)
    return out


def engine_matrix(rows: int, cols: int, ell: int, salt: int) -> np.ndarray:
    """EngineMatrixImpl(rows, cols, ell, salt)."""
    return random_entries(rows * cols, ell, seed_for(rows, cols, ell, salt)).reshape(rows, cols)


def ranked_factors(rows: int, cols: int, rank: int, ell: int):
    """The two factors of RankedMatrix(rows, cols, rank, ell) (salts 0x21 / 0x22,
    PerformanceSmokeValidation.cpp:144-160); the matrix is their product mod ell."""
    L = random_entries(rows * rank, ell, seed_for(rows, rank, ell, 0x21)).reshape(rows, rank)
    R = random_entries(rank * cols, ell, seed_for(rank, cols, ell, 0x22)).reshape(rank, cols)
    return L, R


def fnv_matrix(M: np.ndarray) -> int:
    """FNV-1a-64 over (rows, cols, entries), each fed as a 64-bit word, low byte
    first: the reference micro-bench checksum (computed by libhme on the host)."""
    from . import _lib
    import ctypes as C
    M = np.ascontiguousarray(M, dtype=np.uint32)
    return int(_lib.lib().hme_fnv1a_u32(M.ctypes.data_as(C.POINTER(C.c_uint32)), M.shape[0], M.shape[1], M.shape[1]))


def planted_udv(n: int, ell: int, k: int, salt: int = 0x33, ops: int = 64):
    """Config-3 input: M = U * D * V mod ell^k, n x n.

    U and V are each the product of `ops` seeded elementary row operations
    row_i += c * row_j (i != j, c uniform in [-5, 5]) applied to the identity,
    so both are unimodular; D = diag(ell^e_i) with e_i ~ Geometric(1/2) on
    {0, 1, ...} truncated at k (e_i = k gives a zero diagonal entry).  Returns
    (M, e) with M uint32 canonical in [0, ell^k).  The Smith valuations of M
    over Z/ell^k are exactly sorted({e_i : e_i < k}).  All arithmetic is mod
    ell^k, which is the exact integer product reduced mod ell^k.
    """
    q = ell ** k
    st = seed_for(n, n, q, salt)
    stream = splitmix_stream(st, 3 * 2 * ops + n)
    pos = 0

    def nxt():
        nonlocal pos
        v = int(stream[pos])
        pos += 1
        return v

    e = []
    for _ in range(n):
        w = nxt()
        tz = (w & -w).bit_length() - 1 if w else 64
        e.append(min(tz, k))
    mats = []
    for _ in range(2):
        T = np.eye(n, dtype=np.int64)
        for _ in range(ops):
            i = nxt() % n
            j = nxt() % (n - 1)
            if j >= i:
                j += 1
            c = int(nxt() % 11) - 5
            T[i] = (T[i] + c * T[j]) % q
        mats.append(T)
    U, V = mats
    d = np.array([pow(ell, x, q) if x < k else 0 for x in e], dtype=np.int64)
    UD = (U * d[None, :]) % q
    # exact product mod q in int64: entries < q <= 2^31, so chunk K to keep sums < 2^63
    M = np.zeros((n, n), dtype=np.int64)
    step = max(1, (1 << 62) // (q * q))
    for k0 in range(0, n, step):
        M = (M + UD[:, k0:k0 + step] @ V[k0:k0 + step]) % q
    return M.astype(np.uint32), np.array(e, dtype=np.uint32)


P_JOBS = (65521, 2147483629)


def _mix(z):
    with np.errstate(over="ignore"):
        z = (z ^ (z >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
        return z ^ (z >> np.uint64(31))


def job_stream(n_jobs: int, salt: int = 0x44):
    """The batched job stream (config 4): per job j, side s = round(16 * 64^u)
    with u uniform in [0, 1) (sides log-uniform in [16, 1024]), family j % 2
    (0 banded sparse boundary-like, 1 dense Hecke-like), modulus p from a
    seeded coin over {65521, 2^31 - 19}, and the splitmix64 seeds of A and B.
    Returns numpy arrays (s, family, p, seed_a, seed_b)."""
    j = np.arange(n_jobs, dtype=np.uint64)
    with np.errstate(over="ignore"):
        base = (np.uint64(0xC0FFEE123456789 ^ salt) * np.uint64(0x100000001B3) + j)
        base = base * np.uint64(0x100000001B3) * np.uint64(0x100000001B3)
        z0 = _mix(base + np.uint64(1) * GAMMA)
        z1 = _mix(base + np.uint64(2) * GAMMA)
    u = (z0 >> np.uint64(11)).astype(np.float64) * (1.0 / (1 << 53))
    s = np.clip(np.rint(16.0 * np.power(64.0, u)), 16, 1024).astype(np.int64)
    fam = (j % np.uint64(2)).astype(np.int64)
    p = np.where((z1 & np.uint64(1)) == 0, P_JOBS[0], P_JOBS[1]).astype(np.int64)
    seed_a = np.array([seed_for(int(i), 0, int(q), 0x45) for i, q in zip(range(n_jobs), p)], dtype=np.uint64)
    seed_b = np.array([seed_for(int(i), 1, int(q), 0x45) for i, q in zip(range(n_jobs), p)], dtype=np.uint64)
    return s, fam, p, seed_a, seed_b


def job_matrix(rows: int, cols: int, p: int, family: int, seed: int) -> np.ndarray:
    """Host twin of the device generator (hme_gen_jobs_u32_dev): element (r, c)
    is output r*cols + c of splitmix64(seed); family 1 dense uniform mod p,
    family 0 banded (|r - c| <= 8) with 5 % density and values in [-3, 3]."""
    z = splitmix_stream(int(seed), rows * cols)
    if family == 1:
        return (z % np.uint64(p)).astype(np.uint32).reshape(rows, cols)
    r = np.arange(rows)[:, None]
    c = np.arange(cols)[None, :]
    band = (np.abs(r - c) <= 8).reshape(-1)
    hit = band & ((z % np.uint64(100)) < np.uint64(5))
    w = ((z >> np.uint64(32)) % np.uint64(7)).astype(np.int64) - 3
    v = np.where(w < 0, p + w, w)
    out = np.where(hit, v, 0).astype(np.uint32)
    return out.reshape(rows, cols)
