"""Generate tests/golden/jobs10000.json: the reference's own result for every job
of the 10,000-job stream (sides log-uniform in [16, 1024], half banded sparse,
half dense, p in {65521, 2^31 - 19}; hacs_b200.gen.job_stream /
gen.job_matrix).

Run in a container where the reference sources are present and
oracle/_ref/libhacsref.so has been built (``make -C oracle ref``):

    python tests/golden/make_golden_jobs.py [--jobs 10000] [--workers N]

Per job j it computes, with the reference's CPU engine (drjanosch42/hacs 0.2.1,
src/ModArithmetic), C_j = A_j B_j mod p_j by engine::kernels::gemm<uint32_t>
(Kernels.h:178-185) and the rank of C_j by engine::elim::column_rank_profile
(DenseElim.h:160-169), and stores the rank and the FNV-1a-64 checksum of C_j
(the reference micro bench's checksum).  The jobs are independent, so they are
spread over worker processes (started with spawn), one reference call per job
on each.
"""
import argparse
import json
import multiprocessing as mp
import os
import sys
import time

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--jobs", type=int, default=10000)
    ap.add_argument("--workers", type=int, default=os.cpu_count() or 1)
    ap.add_argument("--out", default=os.path.join(ROOT, "tests", "golden", "jobs10000.json"))
    a = ap.parse_args()

    import oracle as O
    from hacs_b200 import gen

    assert O.ref_available(), "build oracle/_ref first (make -C oracle ref)"
    s, fam, p, sa, sb = gen.job_stream(a.jobs)
    # largest jobs first so the pool's tail is short
    order = sorted(range(a.jobs), key=lambda j: -int(s[j]))
    tasks = [(j, int(s[j]), int(fam[j]), int(p[j]), int(sa[j]), int(sb[j])) for j in order]
    ranks = [0] * a.jobs
    fnvs = [0] * a.jobs
    t0 = time.time()
    with mp.get_context("spawn").Pool(a.workers) as pool:
        for done, (j, r, f) in enumerate(pool.imap_unordered(O.ref_job, tasks, chunksize=4), 1):
            ranks[j] = r
            fnvs[j] = f
            if done % 1000 == 0:
                print(f"{done}/{a.jobs} jobs, {time.time() - t0:.0f} s", flush=True)
    out = {
        "source": "drjanosch42/hacs 0.2.1 CPU engine via oracle/_ref/libhacsref.so: kernels::gemm<uint32_t> "
                  "and elim::column_rank_profile per job",
        "stream": "hacs_b200.gen.job_stream(n_jobs) (salt 0x44), matrices gen.job_matrix (seeds salt 0x45)",
        "n_jobs": a.jobs,
        "rank": ranks,
        "c_fnv": ["%016x" % f for f in fnvs],
    }
    with open(a.out, "w") as f:
        json.dump(out, f, separators=(",", ":"))
        f.write("\n")
    print(f"wrote {a.out}: {a.jobs} jobs in {time.time() - t0:.0f} s")


if __name__ == "__main__":
    main()
