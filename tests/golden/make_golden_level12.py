"""Generate tests/golden/level12.json from the reference's own CPU engine.

Run in a container where the reference sources are present and
oracle/_ref/libhacsref.so has been built (``make -C oracle ref``):

    python tests/golden/make_golden_level12.py

The values come from the reference library's level-1 / level-2 kernels
(drjanosch42/hacs 0.2.1, src/ModArithmetic/Kernels.h:188-259: gemv, gemm_nt,
axpy, scal, transpose, canonicalise, trmm) on inputs from the reference's
seeded EngineMatrix generator, and from its u64 GEMM (kernels::gemm
<uint64_t>) on seeded numpy inputs (`gemm_u64`), stored as FNV-1a-64 checksums (the reference
micro bench's checksum).  The `micro_gemv` and `micro_transpose` entries are
the workloads of the reference's `--bench micro gemv|transpose` (EngineMatrix
salts 3 / 4 and 5, src/Cuda/CudaBench.cpp:91-135).  The reference's CPU engine
has no triangular solve; the `trsm` entries hold the solution X of the
oracle's restatement, accepted only after the reference's trmm gives T X = B.
"""
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle as O  # noqa: E402
from hacs_b200 import gen  # noqa: E402
from oracle import level12 as L12  # noqa: E402


def fnv(M):
    return "0x%016x" % O.fnv_matrix(np.ascontiguousarray(M, dtype=np.uint32))


def acc64(rows, cols, p, salt_hi, salt_lo):
    """64-bit accumulators from two EngineMatrix draws: hi * 2^32 + lo."""
    hi = gen.engine_matrix(rows, cols, p, salt_hi).astype(np.uint64)
    lo = gen.engine_matrix(rows, cols, 4294967291, salt_lo).astype(np.uint64)
    return (hi << np.uint64(32)) | lo


def main():
    assert O.ref_available(), "build oracle/_ref first (make -C oracle ref)"
    out = {"source": "drjanosch42/hacs 0.2.1 CPU engine via oracle/_ref/libhacsref.so"}

    out["micro_gemv"] = []
    out["micro_transpose"] = []
    for n, p in [(1024, 65521), (1000, 2147483629), (512, 4294967291), (300, 13)]:
        A = gen.engine_matrix(n, n, p, 0x03)
        x = gen.engine_matrix(n, 1, p, 0x04)
        y = O.ref_gemv(p, A, x, np.zeros(n, np.uint32), 0)
        out["micro_gemv"].append({"n": n, "p": p, "salts": [3, 4], "fnv": fnv(y.reshape(n, 1))})
        T = O.ref_transpose(gen.engine_matrix(n, n, p, 0x05))
        out["micro_transpose"].append({"n": n, "p": p, "salt": 5, "fnv": fnv(T)})

    out["gemm_nt"] = []
    for m, n, k, p, op in [(300, 200, 129, 65521, 0), (257, 513, 64, 2147483629, 1), (128, 96, 1000, 4294967291, 2)]:
        A = gen.engine_matrix(m, k, p, 0x06)
        B = gen.engine_matrix(n, k, p, 0x07)
        C = gen.engine_matrix(m, n, p, 0x08)
        out["gemm_nt"].append({"m": m, "n": n, "k": k, "p": p, "op": op, "salts": [6, 7, 8],
                               "fnv": fnv(O.ref_gemm_nt(p, A, B, C, op))})

    out["axpy_scal"] = []
    for r, c, p, alpha in [(100, 300, 65521, 12345), (64, 1028, 4294967291, 4000000000)]:
        x = gen.engine_matrix(r, c, p, 0x09)
        y = gen.engine_matrix(r, c, p, 0x0A)
        out["axpy_scal"].append({"rows": r, "cols": c, "p": p, "alpha": alpha, "salts": [9, 10],
                                 "axpy_fnv": fnv(O.ref_axpy(p, alpha, x, y, False)),
                                 "axpy_sub_fnv": fnv(O.ref_axpy(p, alpha, x, y, True)),
                                 "scal_fnv": fnv(O.ref_scal(p, alpha, x))})

    out["canonicalise"] = []
    for r, c, p in [(70, 130, 2147483629), (33, 1024, 65521)]:
        lazy = gen.engine_matrix(r, c, 2 * p, 0x0B)
        acc = acc64(r, c, 4294967291, 0x0C, 0x0D)
        out["canonicalise"].append({"rows": r, "cols": c, "p": p, "lazy_salt": 11, "acc_salts": [12, 13],
                                    "lazy_fnv": fnv(O.ref_canonicalise(p, lazy)),
                                    "acc64_fnv": fnv(O.ref_canonicalise_acc64(p, acc))})

    out["trsm"] = []
    for m, n, p in [(300, 70, 2147483629), (257, 129, 65521), (128, 256, 4294967291)]:
        T = gen.engine_matrix(m, m, p, 0x0E)
        B = gen.engine_matrix(m, n, p, 0x0F)
        for lower in (True, False):
            X = L12.trsm_unit(p, T, B, lower)
            assert np.array_equal(O.ref_trmm_unit(p, T, X, lower), B), "reference trmm disagrees"
            out["trsm"].append({"m": m, "n": n, "p": p, "lower": lower, "salts": [14, 15], "fnv": fnv(X)})

    # u64 residues: the reference's kernels::gemm<uint64_t> on seeded numpy inputs; the checksum is the FNV
    # of the result viewed as u32 words (rows x 2 cols, low word first)
    out["gemm_u64"] = []
    for m, n, k, p, op, seed in [(64, 48, 200, 2305843009213693951, 0, 1), (100, 70, 513, 18446744073709551557, 1, 2),
                                 (33, 129, 1000, 134217757, 2, 3), (40, 40, 64, 1099511627776, 0, 4),
                                 (57, 31, 300, 9223372036854775837, 2, 5), (20, 20, 20, 2, 1, 6)]:
        rng = np.random.default_rng(seed)
        A = rng.integers(0, p, (m, k), dtype=np.uint64)
        B = rng.integers(0, p, (k, n), dtype=np.uint64)
        C = rng.integers(0, p, (m, n), dtype=np.uint64)
        R = O.ref_gemm_u64(p, A, B, C, op)
        out["gemm_u64"].append({"m": m, "n": n, "k": k, "p": p, "op": op, "seed": seed,
                                "fnv": fnv(R.view(np.uint32).reshape(m, 2 * n))})

    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "level12.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", path)


if __name__ == "__main__":
    main()
