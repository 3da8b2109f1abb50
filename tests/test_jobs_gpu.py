"""The batched job stream (through the C ABI): device generator parity with the
host generator, grouped GEMMs and batched ranks bit-exact against the oracle
on uneven jobs, both families, both moduli."""
import numpy as np
import pytest

import oracle as O
from hacs_b200 import gen

pytestmark = pytest.mark.gpu


def _dev(M):
    import torch

    return torch.from_numpy(np.ascontiguousarray(M).view(np.int32)).cuda()


def test_device_generator_matches_host(engine):
    import torch

    s, fam, p, sa, sb = gen.job_stream(40)
    specs, host = [], []
    for j in range(40):
        n = int(min(s[j], 200))
        T = torch.zeros((n, n + 3), dtype=torch.int32, device="cuda")
        specs.append((T[:, :n], int(p[j]), int(fam[j]), int(sa[j])))
        host.append(gen.job_matrix(n, n, int(p[j]), int(fam[j]), int(sa[j])))
    engine.gen_jobs_dev(specs)
    for (T, *_), H in zip(specs, host):
        assert np.array_equal(T.cpu().numpy().view(np.uint32), H)


def test_batch_gemm_and_rank_match_oracle(engine):
    import torch

    rng = np.random.default_rng(3)
    jobs, want_c, want_r = [], [], []
    shapes = [(1, 1, 1), (16, 16, 16), (37, 20, 53), (128, 128, 128), (200, 150, 90), (300, 300, 300),
              (64, 500, 40), (513, 257, 129), (90, 90, 5)]
    for t, (m, k, n) in enumerate(shapes * 2):
        p = (65521, 2147483629)[t % 2]
        fam = (t // 2) % 2
        A = gen.job_matrix(m, k, p, fam, 1000 + t)
        B = gen.job_matrix(k, n, p, fam, 2000 + t)
        C = O.gemm(p, A, B)
        want_c.append(C)
        want_r.append(len(O.rref(p, C)[1]))
        jobs.append({"p": p, "A": _dev(A), "B": _dev(B), "C": torch.zeros((m, n), dtype=torch.int32, device="cuda")})
    engine.use_own_stream()
    engine.batch_gemm_dev(jobs)
    for j, C in zip(jobs, want_c):
        assert np.array_equal(j["C"].cpu().numpy().view(np.uint32), C)
    ranks = engine.batch_rank_dev(jobs)
    assert list(ranks) == want_r


def test_batch_gemm_rank_config4_sample(engine):
    """The first 64 jobs of the config-4 stream (sides capped at 384 to keep the
    oracle fast), generated on the device, GEMM + rank in one call."""
    import torch

    s, fam, p, sa, sb = gen.job_stream(64)
    jobs, want = [], []
    for j in range(64):
        n = int(min(s[j], 384))
        A = torch.zeros((n, n), dtype=torch.int32, device="cuda")
        B = torch.zeros((n, n), dtype=torch.int32, device="cuda")
        jobs.append({"p": int(p[j]), "A": A, "B": B, "C": torch.zeros((n, n), dtype=torch.int32, device="cuda")})
        Ah = gen.job_matrix(n, n, int(p[j]), int(fam[j]), int(sa[j]))
        Bh = gen.job_matrix(n, n, int(p[j]), int(fam[j]), int(sb[j]))
        want.append(len(O.rref(int(p[j]), O.gemm(int(p[j]), Ah, Bh))[1]))
    engine.gen_jobs_dev([(jb["A"], jb["p"], int(fam[j]), int(sa[j])) for j, jb in enumerate(jobs)] +
                        [(jb["B"], jb["p"], int(fam[j]), int(sb[j])) for j, jb in enumerate(jobs)])
    ranks = engine.batch_gemm_rank_dev(jobs)
    assert list(ranks) == want


@pytest.mark.parametrize("p", [251, 65521, 16777213, 2147483629, 4294967291])
def test_batch_gemm_short_k_matches_oracle(engine, p):
    """A batch whose every K is at most 32 runs with 32-byte k-blocks (no zero
    padding to the 128-byte row): ragged M and N, K from 1 to 32, tiles that
    share the stacked plane tensors, all limb counts."""
    import torch

    rng = np.random.default_rng(p % 991)
    shapes = [(1, 1, 1), (5, 32, 7), (130, 17, 65), (128, 32, 128), (257, 31, 300), (64, 9, 500), (300, 24, 33)]
    jobs, want = [], []
    for (m, k, n) in shapes:
        A = rng.integers(0, p, (m, k), dtype=np.uint64).astype(np.uint32)
        B = rng.integers(0, p, (k, n), dtype=np.uint64).astype(np.uint32)
        want.append(O.gemm(p, A, B))
        jobs.append({"p": p, "A": _dev(A), "B": _dev(B), "C": torch.zeros((m, n), dtype=torch.int32, device="cuda")})
    torch.cuda.synchronize()
    engine.batch_gemm_dev(jobs)
    engine.sync()
    for j, C in zip(jobs, want):
        assert np.array_equal(j["C"].cpu().numpy().view(np.uint32), C), (p, j["C"].shape)


def test_batch_rank_wide_panels_and_tall_jobs(engine):
    """Rank rounds with panels up to 128 columns (a job of side <= 128 finishes
    in one panel, larger ones take several rounds with widths set by their
    active rows), rank-deficient jobs, and jobs taller than one panel CTA
    holds (more than 1024 rows: the single-matrix elimination)."""
    import torch

    rng = np.random.default_rng(11)
    jobs, want = [], []
    for t, (m, n, r) in enumerate([(100, 120, 90), (128, 128, 128), (129, 200, 60), (390, 390, 390),
                                   (700, 500, 300), (1024, 1024, 1000), (1100, 300, 250), (2000, 64, 64)]):
        p = (65521, 2147483629)[t % 2]
        L = rng.integers(0, p, (m, r), dtype=np.uint64).astype(np.uint32)
        R = rng.integers(0, p, (r, n), dtype=np.uint64).astype(np.uint32)
        A = O.gemm(p, L, R)
        want.append(len(O.rref(p, A)[1]))
        jobs.append({"p": p, "A": None, "B": None, "C": _dev(A)})
    torch.cuda.synchronize()
    ranks = engine.batch_rank_dev(jobs)
    assert list(ranks) == want


def test_config4_full_stream_matches_reference(engine):
    """All 10,000 jobs of the config-4 stream at full size (sides up to 1024),
    generated on the device: every job's C checksum and every rank against the
    reference CPU engine's own results (tests/golden/jobs10000.json, made by
    tests/golden/make_golden_jobs.py from kernels::gemm and
    elim::column_rank_profile).  The GEMMs and the ranks are checked apart
    (the rank destroys C), then once more through the one-call GEMM + rank."""
    from hacs_b200 import stream

    gold = stream.golden_jobs()
    assert gold is not None, "tests/golden/jobs10000.json is missing"
    want_rank, want_fnv = gold
    st = stream.DeviceStream(len(want_rank))
    engine.use_own_stream()
    engine.gen_jobs_dev(st.specs)
    engine.batch_gemm_dev(st.jobs)
    engine.sync()
    got_fnv = st.job_checksums()
    bad = [j for j in range(st.n_jobs) if got_fnv[j] != want_fnv[j]]
    assert not bad, f"{len(bad)} jobs' C differ from the reference, first {bad[:5]}"
    ranks = engine.batch_rank_dev(st.jobs)
    bad = np.nonzero(ranks != want_rank)[0]
    assert bad.size == 0, f"{bad.size} ranks differ from the reference, first {bad[:5].tolist()}"
    engine.gen_jobs_dev(st.specs)
    ranks = engine.batch_gemm_rank_dev(st.jobs)
    assert np.array_equal(ranks, want_rank)
    # every rank-round schedule at full size: job j on schedule j mod 4
    engine.gen_jobs_dev(st.specs)
    ranks = engine.batch_gemm_rank_dev(st.jobs, rank_variants=np.arange(st.n_jobs) % 4)
    bad = np.nonzero(ranks != want_rank)[0]
    assert bad.size == 0, f"{bad.size} ranks differ under the mixed rank schedules, first {bad[:5].tolist()}"


def test_batch_mixed_with_jobs_taller_than_one_panel_cta(engine):
    """Stream jobs mixed with jobs of more than 1024 rows (those take the
    single-matrix elimination inside the batched call): GEMM + rank of every
    job against the oracle."""
    import torch

    s, fam, p, sa, sb = gen.job_stream(12)
    sides = [int(min(x, 300)) for x in s[:10]] + [1100, 1150]
    jobs, want = [], []
    for j, n in enumerate(sides):
        pj = int(p[j % len(p)])
        f = int(fam[j % len(fam)])
        Ah = gen.job_matrix(n, n, pj, f, int(sa[j]))
        Bh = gen.job_matrix(n, n, pj, f, int(sb[j]))
        want.append(len(O.rref(pj, O.gemm(pj, Ah, Bh))[1]))
        jobs.append({"p": pj, "A": _dev(Ah), "B": _dev(Bh), "C": torch.zeros((n, n), dtype=torch.int32, device="cuda")})
    torch.cuda.synchronize()
    ranks = engine.batch_gemm_rank_dev(jobs)
    assert list(ranks) == want


def test_batch_plan_variants_match_oracle(engine):
    """Every job of a batch on an explicit GEMM schedule (tensor-core wide /
    half-width tiles, CUDA-core 32 / 64 tiles, or the batch rule), mixed in one
    call over two moduli: C and the ranks bit-exact against the oracle, and the
    same for every schedule (a schedule changes only the launch a job runs in)."""
    import ctypes as C_

    import torch

    from hacs_b200 import _lib

    shapes = [(16, 16, 16), (37, 20, 53), (128, 128, 128), (200, 150, 90), (300, 300, 300), (64, 500, 40),
              (513, 257, 129), (90, 90, 5), (1, 1, 1), (700, 33, 640)]
    jobs, want_c, want_r, hjobs = [], [], [], []
    for t, (m, k, n) in enumerate(shapes * 2):
        p = (65521, 2147483629)[t % 2]
        fam = (t // 3) % 2
        A = gen.job_matrix(m, k, p, fam, 3000 + t)
        B = gen.job_matrix(k, n, p, fam, 4000 + t)
        Cw = O.gemm(p, A, B)
        want_c.append(Cw)
        want_r.append(len(O.rref(p, Cw)[1]))
        jobs.append({"p": p, "A": _dev(A), "B": _dev(B), "C": torch.zeros((m, n), dtype=torch.int32, device="cuda")})
    arr = engine._jobs(jobs)
    L = _lib.lib()
    for rot in range(5):
        var = np.array([((t + rot) % 5) - 1 for t in range(len(jobs))], dtype=np.int32)
        for j in jobs:
            j["C"].zero_()
        torch.cuda.synchronize()
        rc = L.hme_batch_gemm_u32_dev_plan(engine._h, len(jobs), arr, var.ctypes.data_as(C_.POINTER(C_.c_int)))
        assert rc == 0, L.hme_last_error().decode()
        for j, Cw in zip(jobs, want_c):
            assert np.array_equal(j["C"].cpu().numpy().view(np.uint32), Cw), (rot, j["C"].shape)
    ranks = np.zeros(len(jobs), np.uint32)
    var = np.array([(t % 5) - 1 for t in range(len(jobs))], dtype=np.int32)
    rc = L.hme_batch_gemm_rank_u32_dev_plan(engine._h, len(jobs), arr, var.ctypes.data_as(C_.POINTER(C_.c_int)),
                                            ranks.ctypes.data_as(C_.POINTER(C_.c_uint32)))
    assert rc == 0, L.hme_last_error().decode()
    assert list(ranks) == want_r
    bad = np.full(len(jobs), 7, np.int32)
    assert L.hme_batch_gemm_u32_dev_plan(engine._h, len(jobs), arr, bad.ctypes.data_as(C_.POINTER(C_.c_int))) == \
        _lib.HME_EINVAL


def test_batch_autotuner_times_every_variant(engine):
    import ctypes as C_

    from hacs_b200 import _lib

    ms = np.zeros(4, np.float32)
    for (p, m, n, k, count) in [(65521, 32, 32, 32, 64), (2147483629, 256, 256, 256, 4)]:
        rc = _lib.lib().hme_autotune_batch(engine._h, p, m, n, k, count, 3, ms.ctypes.data_as(C_.POINTER(C_.c_float)))
        assert rc == 0, _lib.lib().hme_last_error().decode()
        assert np.all(ms > 0) and np.all(np.isfinite(ms))


def _planted(rng, m, n, r, p):
    L = rng.integers(0, p, (m, r), dtype=np.uint64).astype(np.uint32)
    R = rng.integers(0, p, (r, n), dtype=np.uint64).astype(np.uint32)
    return O.gemm(p, L, R)


def test_batch_rank_schedules_match_oracle(engine):
    """Every rank-round schedule (trailing update on the grouped tensor-core limb
    GEMM or on CUDA cores; a last panel of up to 128 columns or 32-column rounds
    to the end; and -1 the batch rule), mixed
    in one call over five moduli (one to four limbs, p above 2^31 included), under
    five rotations of the schedules over the jobs.  The jobs have planted ranks
    below their sides (a wrong trailing update raises the rank), wide, tall and
    ragged shapes, trailing blocks both smaller and larger than one 64 x 64
    CUDA-core tile; every rank equals the oracle's."""
    import torch

    rng = np.random.default_rng(17)
    cases = [(100, 300, 40), (64, 700, 64), (200, 150, 150), (129, 200, 60), (390, 390, 200), (700, 500, 300),
             (33, 1000, 20), (500, 64, 30), (16, 16, 16), (1, 50, 1), (50, 1, 1), (1024, 700, 650), (77, 77, 77)]
    moduli = [251, 65521, 16777213, 2147483629, 4294967291]
    mats, want = [], []
    for t, (m, n, r) in enumerate(cases * 2):
        p = moduli[t % len(moduli)]
        A = _planted(rng, m, n, r, p)
        mats.append((p, A))
        want.append(len(O.rref(p, A)[1]))
    for rot in range(5):
        jobs = [{"p": p, "A": None, "B": None, "C": _dev(A)} for p, A in mats]
        var = np.array([((t + rot) % 5) - 1 for t in range(len(jobs))], dtype=np.int32)
        torch.cuda.synchronize()
        ranks = engine.batch_rank_dev(jobs, rank_variants=var)
        assert list(ranks) == want, f"rotation {rot}"


def test_batch_gemm_rank_sched_config4_sample(engine):
    """The first 64 config-4 jobs (sides capped at 384) through
    hme_batch_gemm_rank_u32_dev_sched with both phases' schedules mixed: every
    GEMM schedule against every rank schedule; ranks equal the oracle's."""
    import torch

    s, fam, p, sa, sb = gen.job_stream(64)
    jobs, want = [], []
    for j in range(64):
        n = int(min(s[j], 384))
        jobs.append({"p": int(p[j]), "A": torch.zeros((n, n), dtype=torch.int32, device="cuda"),
                     "B": torch.zeros((n, n), dtype=torch.int32, device="cuda"),
                     "C": torch.zeros((n, n), dtype=torch.int32, device="cuda")})
        Ah = gen.job_matrix(n, n, int(p[j]), int(fam[j]), int(sa[j]))
        Bh = gen.job_matrix(n, n, int(p[j]), int(fam[j]), int(sb[j]))
        want.append(len(O.rref(int(p[j]), O.gemm(int(p[j]), Ah, Bh))[1]))
    engine.gen_jobs_dev([(jb["A"], jb["p"], int(fam[j]), int(sa[j])) for j, jb in enumerate(jobs)] +
                        [(jb["B"], jb["p"], int(fam[j]), int(sb[j])) for j, jb in enumerate(jobs)])
    gv = np.array([(j % 5) - 1 for j in range(64)], np.int32)
    rv = np.array([((j // 5) % 5) - 1 for j in range(64)], np.int32)
    ranks = engine.batch_gemm_rank_dev(jobs, gemm_variants=gv, rank_variants=rv)
    assert list(ranks) == want


def test_rank_autotuner_times_every_schedule(engine):
    import ctypes as C_

    from hacs_b200 import _lib, sched

    for (p, m, n, k, dens, count) in [(65521, 48, 48, 48, 1.0, 16), (2147483629, 300, 300, 280, 1.0, 2),
                                      (65521, 200, 200, 200, 0.05, 2)]:
        ms = sched.autotune_batch_rank(engine, p, m, n, k, dens, count=count, reps=2)
        assert ms.shape == (sched.N_RANK_VARIANTS,)
        assert np.all(ms > 0) and np.all(np.isfinite(ms))
    L = _lib.lib()
    ms = np.zeros(4, np.float32)
    fp = ms.ctypes.data_as(C_.POINTER(C_.c_float))
    # rows beyond one panel CTA, and a composite modulus, are refused before anything runs
    assert L.hme_autotune_batch_rank(engine._h, 65521, 1100, 64, 64, 1.0, 1, 1, fp) == _lib.HME_EINVAL
    assert L.hme_autotune_batch_rank(engine._h, 65536, 64, 64, 64, 1.0, 1, 1, fp) == _lib.HME_EINVAL
    jobs = [{"p": 65521, "A": None, "B": None, "C": _dev(np.zeros((8, 8), np.uint32))}]
    with pytest.raises(_lib.HmeError):
        engine.batch_rank_dev(jobs, rank_variants=[4])
