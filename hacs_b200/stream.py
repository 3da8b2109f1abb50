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
    def __init__(self, n_jobs: int, salt: int = 0x44, first: int = 0):
        import torch

        s, fam, p, sa, sb = gen.job_stream(first + n_jobs, salt)
        self.s, self.fam, self.p = s[first:], fam[first:], p[first:]
        self.seed_a, self.seed_b = sa[first:], sb[first:]
        self.n_jobs = n_jobs
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
