"""The batched job stream on the device: buffers, job tables and checksums.

A job is C = A*B mod p followed by rank(C) over F_p (hme_batch_gemm_rank_u32_dev).
``device_stream(n)`` lays the first n jobs of ``gen.job_stream`` out in three
device arenas (A, B, C; job j's n_j x n_j matrices back to back), returns the
job dicts the Engine's batch methods take and the generator specs of
``Engine.gen_jobs_dev``; ``job_checksums`` reads C back and gives each job's
FNV-1a-64 (the reference micro bench's checksum, computed by libhme on the
host), the form in which tests/golden/jobs10000.json holds the reference's
results.
"""
from __future__ import annotations

import json
import os

import numpy as np

from . import gen

GOLDEN_JOBS = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "tests", "golden",
                           "jobs10000.json")


class DeviceStream:
    """Jobs [first, first + n_jobs) of the stream, or the jobs `indices` of its
    first n_jobs (one rank's share of a sharded stream)."""

    def __init__(self, n_jobs: int, salt: int = 0x44, first: int = 0, indices=None):
        import torch

        s, fam, p, sa, sb = gen.job_stream(first + n_jobs, salt)
        sel = np.arange(first, first + n_jobs) if indices is None else np.asarray(indices, dtype=np.int64)
        self.s, self.fam, self.p = s[sel], fam[sel], p[sel]
        self.seed_a, self.seed_b = sa[sel], sb[sel]
        self.indices = sel
        self.n_jobs = len(sel)
        n_jobs = self.n_jobs
        sq = self.s * self.s
        self.offsets = np.concatenate([[0], np.cumsum(sq)]).astype(np.int64)
        tot = int(self.offsets[-1])
        self.bufA = torch.empty(max(1, tot), dtype=torch.int32, device="cuda")
        self.bufB = torch.empty_like(self.bufA)
        self.bufC = torch.empty_like(self.bufA)
        self.jobs, self.specs = [], []
        for j in range(n_jobs):
            n, off = int(self.s[j]), int(self.offsets[j])
            A, B, Cm = (b[off:off + n * n].view(n, n) for b in (self.bufA, self.bufB, self.bufC))
            pj = int(self.p[j])
            self.jobs.append({"p": pj, "A": A, "B": B, "C": Cm})
            self.specs.append((A, pj, int(self.fam[j]), int(self.seed_a[j])))
            self.specs.append((B, pj, int(self.fam[j]), int(self.seed_b[j])))

    def work_modmac(self) -> float:
        """GEMM work sum_j s_j^3 (multiply-adds mod p)."""
        return float((self.s.astype(np.float64) ** 3).sum())

    def job_checksums(self) -> list[int]:
        """FNV-1a-64 of every job's C (reads the C arena back to the host)."""
        Ch = self.bufC.cpu().numpy().view(np.uint32)
        out = []
        for j in range(self.n_jobs):
            n, off = int(self.s[j]), int(self.offsets[j])
            out.append(gen.fnv_matrix(Ch[off:off + n * n].reshape(n, n)))
        return out


def golden_jobs(path: str = GOLDEN_JOBS):
    """(ranks, C checksums) of the reference's own CPU engine on the stream's jobs, or None."""
    if not os.path.exists(path):
        return None
    d = json.load(open(path))
    return np.array(d["rank"], dtype=np.int64), [int(h, 16) for h in d["c_fnv"]]


# ---- the config-5 mixed stream -------------------------------------------------------------------
P_CONFIG2 = 2147483629
CONFIG1_FNV = 0x572E8347446366C6  # C of --bench micro gemm 1024 1024 65521 (EngineMatrix salts 0x01 / 0x02)


class MixedStream:
    """The learned scheduler's serving stream: n_jobs GEMM + rank jobs drawn from
    the configurations, in a seeded order, served in chunks of `chunk` jobs.

    Kinds (a job is C = A B mod p, then rank(C) over F_p):
      0  config 4: job j of gen.job_stream (sides log-uniform 16..1024, banded
         sparse or dense, p in {65521, 2^31 - 19}); the first 10,000 of them are
         exactly config 4's stream (tests/golden/jobs10000.json holds the
         reference's ranks);
      1  config 2: the RankedMatrix construction at p = 2^31 - 19 on a smaller
         side: A = F1 (s x r), B = F2 (r x s), s log-uniform 64..1024,
         r = s - s // 20, so rank(C) = r (with probability 1 - r/p);
      2  config 1: A, B the 1024 x 1024 EngineMatrix operands (salts 0x01 /
         0x02) at p = 65521, whose product has the reference's micro-bench FNV
         and rank 1024.
    Mix: 10,000 config-4 jobs (the golden ones), then of the rest 70 % config
    4, 25 % config 2, 5 % config 1."""

    def __init__(self, n_jobs: int = 50000, chunk: int = 5000, seed: int = 2027):
        n_gold = min(10000, n_jobs)
        rest = n_jobs - n_gold
        n1 = rest * 5 // 100
        n2 = rest * 25 // 100
        n4 = n_gold + rest - n1 - n2
        s4, f4, p4, sa4, sb4 = gen.job_stream(n4)
        rng = np.random.default_rng(seed)
        u = rng.random(n2)
        s2 = np.clip(np.rint(64.0 * np.power(16.0, u)), 64, 1024).astype(np.int64)
        kind = np.concatenate([np.zeros(n4, np.int64), np.ones(n2, np.int64), np.full(n1, 2, np.int64)])
        idx = np.concatenate([np.arange(n4), np.arange(n2), np.arange(n1)])
        order = rng.permutation(n_jobs)
        self.kind, self.idx = kind[order], idx[order]
        self.n_jobs, self.chunk = n_jobs, chunk
        # per job: p, m, n, k, (family, seed) for A and B
        self.p = np.zeros(n_jobs, np.int64)
        self.m = np.zeros(n_jobs, np.int64)
        self.k = np.zeros(n_jobs, np.int64)
        self.fam = np.ones(n_jobs, np.int64)
        self.sa = np.zeros(n_jobs, np.uint64)
        self.sb = np.zeros(n_jobs, np.uint64)
        for t in range(n_jobs):
            kd, i = int(self.kind[t]), int(self.idx[t])
            if kd == 0:
                self.p[t], self.m[t], self.k[t], self.fam[t] = p4[i], s4[i], s4[i], f4[i]
                self.sa[t], self.sb[t] = sa4[i], sb4[i]
            elif kd == 1:
                s = int(s2[i])
                self.p[t], self.m[t], self.k[t] = P_CONFIG2, s, s - s // 20
                self.sa[t] = gen.seed_for(i, 2, P_CONFIG2, 0x56)
                self.sb[t] = gen.seed_for(i, 3, P_CONFIG2, 0x56)
            else:
                self.p[t], self.m[t], self.k[t] = 65521, 1024, 1024
                self.sa[t] = gen.seed_for(1024, 1024, 65521, 0x01)
                self.sb[t] = gen.seed_for(1024, 1024, 65521, 0x02)
        self.gold_rank = None
        g = golden_jobs()
        if g is not None:
            self.gold_rank = g[0]
        self._bufs = None

    def shapes(self) -> np.ndarray:
        """Rows (p, m, n, k) of every job's product, in stream order."""
        return np.column_stack([self.p, self.m, self.m, self.k]).astype(np.uint32)

    def density(self) -> np.ndarray:
        return np.where(self.fam == 0, 0.05, 1.0)

    def chunks(self):
        for c0 in range(0, self.n_jobs, self.chunk):
            yield c0, min(self.n_jobs, c0 + self.chunk)

    def device_chunk(self, c0: int, c1: int):
        """Device buffers, job dicts and generator specs of jobs [c0, c1) (arenas reused across chunks)."""
        import torch

        ea = self.m[c0:c1] * self.k[c0:c1]
        ec = self.m[c0:c1] * self.m[c0:c1]
        oa = np.concatenate([[0], np.cumsum(2 * ea)]).astype(np.int64)
        oc = np.concatenate([[0], np.cumsum(ec)]).astype(np.int64)
        need_ab, need_c = int(oa[-1]), int(oc[-1])
        if self._bufs is None or self._bufs[0].numel() < need_ab or self._bufs[1].numel() < need_c:
            self._bufs = None
            torch.cuda.empty_cache()
            self._bufs = (torch.empty(max(1, need_ab), dtype=torch.int32, device="cuda"),
                          torch.empty(max(1, need_c), dtype=torch.int32, device="cuda"))
        AB, Cb = self._bufs
        jobs, specs = [], []
        for t in range(c0, c1):
            u = t - c0
            m, k, p = int(self.m[t]), int(self.k[t]), int(self.p[t])
            A = AB[oa[u]:oa[u] + m * k].view(m, k)
            B = AB[oa[u] + m * k:oa[u] + 2 * m * k].view(k, m)
            Cm = Cb[oc[u]:oc[u] + m * m].view(m, m)
            jobs.append({"p": p, "A": A, "B": B, "C": Cm})
            specs.append((A, p, int(self.fam[t]), int(self.sa[t])))
            specs.append((B, p, int(self.fam[t]), int(self.sb[t])))
        return jobs, specs

    def check_ranks(self, ranks: np.ndarray) -> dict:
        """Size-independent checks of a served stream's ranks: config-4 jobs
        against the reference's golden ranks, config-2 jobs rank = r, config-1
        jobs rank 1024."""
        out = {}
        r = np.asarray(ranks, np.int64)
        k4 = self.kind == 0
        if self.gold_rank is not None:
            g = k4 & (self.idx < len(self.gold_rank))
            out["config4_jobs_vs_reference"] = int(g.sum())
            out["config4_ranks_equal_reference"] = bool(np.array_equal(r[g], self.gold_rank[self.idx[g]]))
        k2 = self.kind == 1
        out["config2_jobs"] = int(k2.sum())
        out["config2_rank_equals_inner_dim"] = int((r[k2] == self.k[k2]).sum())
        k1 = self.kind == 2
        out["config1_jobs"] = int(k1.sum())
        out["config1_rank_1024"] = int((r[k1] == 1024).sum())
        return out
