"""Generate tests/golden/golden.json from the reference's own CPU engine.

Run in a container where the reference sources are present and
oracle/_ref/libhacsref.so has been built (``make -C oracle ref``):

    python tests/golden/make_golden.py

Every value here comes from the reference library (drjanosch42/hacs 0.2.1,
src/ModArithmetic: kernels::gemm, elim::rref, elim::howell, ring2k::howell /
smith, ring3k::howell / smith), on inputs from the reference's own seeded
generators (splitmix64 EngineMatrix / RankedMatrix factors) or the planted
U*D*V construction; the fixtures pin the oracle restatement and the GPU path
without needing the reference at test time.  Matrices are stored as FNV-1a-64
checksums (the reference micro bench's checksum), small ones in full.
"""
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle as O  # noqa: E402
from hacs_b200 import gen  # noqa: E402


def fnv(M):
    return "0x%016x" % O.fnv_matrix(np.ascontiguousarray(M, dtype=np.uint32))


def main():
    assert O.ref_available(), "build oracle/_ref first (make -C oracle ref)"
    out = {"source": "drjanosch42/hacs 0.2.1 CPU engine via oracle/_ref/libhacsref.so"}

    g = []
    for (n, k, p) in [(64, 64, 65521), (257, 130, 2147483629), (1024, 1024, 65521), (512, 300, 4294967291),
                      (300, 200, 13), (200, 1000, 16777213)]:
        A = gen.engine_matrix(n, k, p, 0x01)
        B = gen.engine_matrix(k, n, p, 0x02)
        C = O.ref_gemm(p, A, B, threads=8)
        g.append({"p": p, "n": n, "k": k, "salts": [1, 2], "fnv": fnv(C)})
    out["gemm"] = g

    r = []
    for (m, n, rank, p) in [(64, 64, 40, 2147483629), (200, 150, 100, 65521), (257, 300, 257, 2147483629),
                            (300, 257, 200, 65521), (512, 512, 480, 2147483629)]:
        L, R = gen.ranked_factors(m, n, rank, p)
        A = O.ref_gemm(p, L, R, threads=8)
        Rr, piv = O.ref_rref(p, A)
        r.append({"p": p, "m": m, "n": n, "rank_target": rank, "input_fnv": fnv(A), "rank": int(len(piv)),
                  "pivots": [int(x) for x in piv], "rref_fnv": fnv(Rr)})
    out["rref"] = r

    h = []
    for (ell, k, n, salt) in [(2, 16, 48, 0x33), (2, 16, 96, 0x34), (3, 10, 48, 0x33), (3, 10, 96, 0x34),
                              (2, 2, 40, 0x35)]:
        M, e = gen.planted_udv(n, ell, k, salt)
        if ell == 2:
            H, piv, pv = O.ref_howell_2k(k, M)
            sig = O.ref_smith_2k(k, M)
        else:
            H, piv, pv = O.ref_howell_3k(k, M)
            sig = O.ref_smith_3k(k, M)
        H2, piv2, pv2 = O.ref_elim_howell(ell, k, M)
        assert np.array_equal(H, H2) and np.array_equal(piv, piv2) and np.array_equal(pv, pv2)
        h.append({"ell": ell, "k": k, "n": n, "salt": salt, "input_fnv": fnv(M), "h": int(len(piv)),
                  "howell_fnv": fnv(H), "pivots": [int(x) for x in piv], "pivot_v": [int(x) for x in pv],
                  "sigma": [int(x) for x in sig], "planted_e": [int(x) for x in e]})
    out["ring"] = h

    # full-size configurations: config 2 (RankedMatrix 4096 x 4096, rank 3900, p = 2^31 - 19) and
    # config 3 (planted U*D*V 2048 x 2048, Howell over Z/2^16 and Smith over Z/3^10)
    if os.environ.get("GOLDEN_FULL", "1") == "1":
        p = 2147483629
        L, R = gen.ranked_factors(4096, 4096, 3900, p)
        A = O.ref_gemm(p, L, R, threads=8)
        Rr, piv = O.ref_rref(p, A)
        out["config2"] = {"p": p, "m": 4096, "n": 4096, "rank_target": 3900, "input_fnv": fnv(A),
                          "rank": int(len(piv)), "pivots_fnv": fnv(piv.reshape(1, -1)), "rref_fnv": fnv(Rr),
                          "det": 0}
        c3 = {}
        for (ell, k) in [(2, 16), (3, 10)]:
            M, e = gen.planted_udv(2048, ell, k, 0x33)
            if ell == 2:
                H, hp, hv = O.ref_howell_2k(k, M, threads=8)
                sig = O.ref_smith_2k(k, M, threads=8)
            else:
                H, hp, hv = O.ref_howell_3k(k, M, threads=8)
                sig = O.ref_smith_3k(k, M, threads=8)
            c3[f"{ell}^{k}"] = {"ell": ell, "k": k, "n": 2048, "salt": 0x33, "input_fnv": fnv(M),
                                "h": int(len(hp)), "howell_fnv": fnv(H), "pivots_fnv": fnv(hp.reshape(1, -1)),
                                "pivot_v_fnv": fnv(hv.reshape(1, -1)), "sigma": [int(x) for x in sig],
                                "planted_e_fnv": fnv(e.reshape(1, -1))}
        out["config3"] = c3

    # known answers (ENGINE_API.md Sec. 13.5 and HeckeReductionValidation's Z/4 arms)
    H, piv, pv = O.ref_elim_howell(2, 2, np.array([[2, 1]], np.uint32))
    H2, piv2, pv2 = O.ref_elim_howell(2, 2, np.array([[2], [1]], np.uint32))
    out["known"] = {
        "howell_z4_row_2_1": {"H": H.tolist(), "pivots": piv.tolist(), "pivot_v": pv.tolist()},
        "howell_z4_col_2_1": {"H": H2.tolist(), "pivots": piv2.tolist(), "pivot_v": pv2.tolist()},
        "smith_z4_col_2_1": O.ref_smith_2k(2, np.array([[2], [1]], np.uint32)).tolist(),
    }
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", path)


if __name__ == "__main__":
    main()
