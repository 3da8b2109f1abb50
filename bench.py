#!/usr/bin/env python
"""Headline benchmark of the B200-native exact modular matrix engine.

Workload (one "step"): the mod-p GEMM C = A*B mod p of the reference's
micro bench, `--bench micro gemm 1024 1024 65521`: A, B 1024 x 1024 uint32
from the reference's seeded splitmix64 generator (EngineMatrix salts
0x01 / 0x02), p = 65521, on the INT8-limb tcgen05 GEMM.  Metric: Tops/s with
ops = 2*m*n*k (one modular multiply-add = 2 ops).  Inputs (4 MiB each) fit L2,
so L2 is flushed (a 256 MiB write) before every timed step.

The JSON line also carries: the dominant kernel's roofline (INT8 tensor ops
L^2 * 2mnk per launch over its CUDA-event time, against the measured peak),
the reference CPU engine timed on this host (cpu_baseline), the end-to-end
rate through the public host-pointer API (pinned host buffers, H2D + D2H
inside the timed region), SM clocks sampled during the timed region, and the
8192^3 GEMM at p = 65521 (2 limbs) and p = 2^31 - 19 (4 limbs) next to the
reference's own CUDA-core GEMM (the plain method) on the same buffers, and
the u64-residue GEMM 2048^3 at p = 2^61 - 1 beside the reference's u64 plain
method.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl hme|reference]

Under torchrun (N > 1) every rank runs its own replica of the step (GEMMs
shard by independent output tiles / jobs; no collective is needed): value =
all ranks' ops / max-over-ranks time, scaling "weak".
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

P_HEAD = 65521
N_HEAD = 1024
METRIC = "mod-p GEMM Tops/s (C = A*B mod p, bit-exact)"
UNIT = "Tops/s"
L2_FLUSH_BYTES = 256 << 20
PEAK_FALLBACK_BF16_TFLOPS = 1590.0
DATA_HEAD = "synthetic (reference splitmix64 EngineMatrix, salts 0x01/0x02)"


def head_config(n: int, p: int, ws: int, checksum_ok: bool) -> dict:
    """The headline workload's config (the same dict on both arms)."""
    from hacs_b200 import limbs_for

    return {"workload": f"GEMM {n}^3 p={p} (config 1: --bench micro gemm {n} {n} {p})", "m": n, "n": n,
            "k": n, "p": p, "limbs": limbs_for(p), "parallelism": f"replicas x{ws}",
            "l2": "flushed before every step", "checksum_ok": checksum_ok}


def _json(o):
    """json default for numpy scalars and arrays."""
    if hasattr(o, "item") and getattr(o, "ndim", 0) == 0:
        return o.item()
    if hasattr(o, "tolist"):
        return o.tolist()
    return str(o)


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return d, "measured"
    return {"bf16_tflops": PEAK_FALLBACK_BF16_TFLOPS, "hbm_gbs": 6650.0}, "fallback"


def profile_traffic(name: str):
    """dram bytes per launch recorded in the committed ncu summary, or None."""
    path = os.path.join(ROOT, "profiles", name)
    if not os.path.exists(path):
        return None
    for line in open(path):
        if line.startswith("dram_bytes_per_launch:"):
            return float(line.split(":", 1)[1].split()[0])
    return None


class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        time.sleep(0.15)
        return self

    def __exit__(self, *exc):
        self.rows = []
        if self.proc is None:
            return
        time.sleep(0.15)
        self.proc.terminate()
        out, _ = self.proc.communicate(timeout=10)
        for line in out.splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) >= 9:
                self.rows.append(f)

    def summary(self):
        if not getattr(self, "rows", None):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


class GpuLocalCpus:
    """Bind the process to the CPUs of the GPU's own NUMA node (NVML's CPU
    affinity of the device, read only) for the duration of a block, so that
    pinned host buffers allocated inside it sit next to the GPU's PCIe root;
    the previous affinity is restored on exit.  A no-op where NVML or the
    affinity call is not available.  `note` says what was applied."""

    def __init__(self, device: int):
        self.device = device
        self.saved = None
        self.note = "default affinity"

    def __enter__(self):
        try:
            import pynvml
            import torch

            pr = torch.cuda.get_device_properties(self.device)
            bus = "%08X:%02X:%02X.0" % (pr.pci_domain_id, pr.pci_bus_id, pr.pci_device_id)
            pynvml.nvmlInit()
            try:
                h = pynvml.nvmlDeviceGetHandleByPciBusId(bus)
                words = pynvml.nvmlDeviceGetCpuAffinity(h, 64)
            finally:
                pynvml.nvmlShutdown()
            local = {64 * i + b for i, w in enumerate(words) for b in range(64) if (int(w) >> b) & 1}
            allowed = os.sched_getaffinity(0)
            use = local & allowed
            if use and use != allowed:
                self.saved = allowed
                os.sched_setaffinity(0, use)
                self.note = f"GPU-local CPUs ({len(use)} of {len(allowed)}) while allocating and timing"
        except Exception:
            self.saved = None
        return self

    def __exit__(self, *exc):
        if self.saved is not None:
            os.sched_setaffinity(0, self.saved)


def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    return ws, rank, local


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(x: float, ws: int) -> float:
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def host_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def cpu_info() -> dict:
    """Model name and the SIMD flags the reference's kernels dispatch on, from /proc/cpuinfo."""
    model, flags = "unknown", set()
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name") and model == "unknown":
                model = line.split(":", 1)[1].strip()
            elif line.startswith("flags") and not flags:
                flags = set(line.split(":", 1)[1].split())
    except OSError:
        pass
    isa = [f for f in ("avx2", "avx512f", "avx512dq", "avx512bw", "avx512vl", "avx512_vnni", "avx512ifma")
           if f in flags]
    return {"cpu_model": model, "isa": isa, "host_threads": host_threads()}


def cpu_gemm_rate(p: int, n: int, budget_s: float = 10.0, min_reps: int = 3):
    """The reference's CPU engine (oracle/_ref) on the headline GEMM through its
    own multi-thread path: one Recorder::gemm node compiled and run by the
    tape Executor on a ThreadPool of all host threads (Recorder.h:147,
    Executor.h:79); falls back to the oracle's C port (one thread) when the
    reference library is not built."""
    import oracle as O
    from hacs_b200 import gen

    A = gen.engine_matrix(n, n, p, 0x01)
    B = gen.engine_matrix(n, n, p, 0x02)
    if O.ref_available():
        thr = host_threads()
        C0, _ = O.ref_tape_gemm(p, A, B, threads=thr, reps=1)  # warm: pool start, program compile
        t0 = time.perf_counter()
        reps, secs = 0, 0.0
        while reps < min_reps or time.perf_counter() - t0 < budget_s:
            _, s1 = O.ref_tape_gemm(p, A, B, threads=thr, reps=2)
            secs += 2 * s1
            reps += 2
        ok = O.fnv_matrix(C0) == 0x572E8347446366C6
        return {"value": 2.0 * n ** 3 * reps / secs / 1e12, "unit": UNIT, "cores": thr, "kind": "reference",
                "sample": f"{reps} x GEMM {n}^3 p={p} (EngineMatrix salts 1/2) through tape::Recorder::gemm + "
                          f"Executor::run on a {thr}-worker pool, {secs:.1f} s of runs",
                "checksum_ok": bool(ok), **cpu_info()}
    else:
        thr = 1
        kind = "port"
        sample_n = 256
        A, B = A[:sample_n, :sample_n].copy(), B[:sample_n, :sample_n].copy()
        fn = lambda: O.gemm(p, A, B)  # noqa: E731
    fn()  # warm
    reps, t0 = 0, time.perf_counter()
    while reps < min_reps or time.perf_counter() - t0 < budget_s:
        fn()
        reps += 1
    dt = time.perf_counter() - t0
    ops = 2.0 * sample_n ** 3 * reps
    return {"value": ops / dt / 1e12, "unit": UNIT, "cores": thr, "kind": kind,
            "sample": f"{reps} x GEMM {sample_n}^3 p={p} (EngineMatrix salts 1/2), {dt:.1f} s"}


def run_reference(args):
    ws, rank, _ = int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")), 0
    if rank != 0:
        return 0
    import oracle as O
    from hacs_b200 import gen

    p, n = P_HEAD, N_HEAD
    A = gen.engine_matrix(n, n, p, 0x01)
    B = gen.engine_matrix(n, n, p, 0x02)
    if O.ref_available():
        # the reference's own multi-thread GEMM path: a tape program of one Recorder::gemm node run by
        # the Executor on a pool of all host threads; one program run per step
        thr, kind = host_threads(), "reference"
        how = "tape::Recorder::gemm + Executor::run"
        for _ in range(args.warmup):
            O.ref_tape_gemm(p, A, B, threads=thr, reps=1)
        C_, s1 = O.ref_tape_gemm(p, A, B, threads=thr, reps=args.steps)
        dt = s1 * args.steps
    else:
        thr, kind, how = 1, "port", "oracle C port"
        for _ in range(args.warmup):
            O.gemm(p, A, B)
        t0 = time.perf_counter()
        for _ in range(args.steps):
            C_ = O.gemm(p, A, B)
        dt = time.perf_counter() - t0
    ok = O.fnv_matrix(C_) == 0x572E8347446366C6
    val = 2.0 * n ** 3 * args.steps / dt / 1e12
    line = {
        "impl": "reference", "metric": METRIC, "value": val, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32", "data": DATA_HEAD,
        "config": head_config(n, p, ws, bool(ok)),
        "cpu_baseline": {"value": val, "unit": UNIT, "cores": thr, "kind": kind,
                         "sample": f"{args.steps} x GEMM {n}^3 p={p} on {thr} host threads ({how})", **cpu_info()},
        "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line, default=_json), flush=True)
    return 0


def load_plain():
    path = os.path.join(ROOT, "baseline", "_ref", "libplain.so")
    if not os.path.exists(path):
        return None
    L = C.CDLL(path)
    L.plain_gemm_u32_dev.restype = C.c_int
    L.plain_gemm_u32_dev.argtypes = [C.c_uint32] * 4 + [C.c_void_p, C.c_size_t, C.c_void_p, C.c_size_t,
                                                        C.c_void_p, C.c_size_t, C.c_int, C.c_void_p]
    if hasattr(L, "plain_gemm_u64_dev"):
        L.plain_gemm_u64_dev.restype = C.c_int
        L.plain_gemm_u64_dev.argtypes = [C.c_uint64] + [C.c_uint32] * 3 + [C.c_void_p, C.c_size_t, C.c_void_p,
                                                                          C.c_size_t, C.c_void_p, C.c_size_t,
                                                                          C.c_int, C.c_void_p]
    L.plain_last_error.restype = C.c_char_p
    return L


def time_device(fn, steps, warmup, flush=None):
    """Sum of per-step CUDA-event times (ms) on torch's current stream."""
    import torch

    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    total = 0.0
    for _ in range(steps):
        if flush is not None:
            flush()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        fn()
        b.record()
        b.synchronize()
        total += a.elapsed_time(b)
    return total


def big_gemm(eng, plain, p, n, steps=5, warmup=3):
    """8192^3-class GEMM: inputs resident (256 MiB each, larger than L2)."""
    import torch

    from hacs_b200 import limbs_for

    g = torch.Generator(device="cuda").manual_seed(p)
    A = torch.randint(0, p, (n, n), dtype=torch.int64, device="cuda", generator=g).to(torch.int32)
    B = torch.randint(0, p, (n, n), dtype=torch.int64, device="cuda", generator=g).to(torch.int32)
    Cm = torch.empty((n, n), dtype=torch.int32, device="cuda")
    eng.set_timing(True)
    eng.timing_reset()
    ms = time_device(lambda: eng.gemm_dev(p, A, B, Cm), steps, warmup)
    kms, kl = eng.kernel_time("limb_gemm")
    eng.set_timing(False)
    L = limbs_for(p)
    out = {"p": p, "n": n, "limbs": L, "tops": 2.0 * n ** 3 * steps / ms / 1e9, "ms": ms / steps,
           "kernel_ms": kms / max(1, kl), "int8_tops_kernel": L * L * 2.0 * n ** 3 / (kms / max(1, kl)) / 1e9}
    if plain is not None:
        Cp = torch.empty_like(Cm)
        st = torch.cuda.current_stream().cuda_stream

        def run_plain():
            rc = plain.plain_gemm_u32_dev(p, n, n, n, A.data_ptr(), n, B.data_ptr(), n, Cp.data_ptr(), n, 0, st)
            if rc != 0:
                raise RuntimeError(plain.plain_last_error().decode())

        pms = time_device(run_plain, 2, 1)
        out["plain_gpu_tops"] = 2.0 * n ** 3 * 2 / pms / 1e9
        out["plain_gpu_ms"] = pms / 2
        out["speedup_vs_plain"] = out["tops"] / out["plain_gpu_tops"]
        out["bit_exact_vs_plain"] = bool(torch.equal(Cm, Cp))
    return out


def _golden():
    path = os.path.join(ROOT, "tests", "golden", "golden.json")
    return json.load(open(path)) if os.path.exists(path) else {}


def int8_peak_tops():
    pk, src = peaks()
    return 2.0 * float(pk["bf16_tflops"]), f"2 x {src} bf16 dense TFLOP/s (INT8 dense rate = 2 x bf16 on B200)"


def hbm_peak_gbs():
    pk, src = peaks()
    return float(pk["hbm_gbs"]), f"{src} copy bandwidth"


def kernel_breakdown(eng, names):
    """{name: [total ms, launches]} of the library's per-kernel CUDA-event timer."""
    out = {}
    for nm in names:
        ms, c = eng.kernel_time(nm)
        if c:
            out[nm] = [round(ms, 4), int(c)]
    return out


def extra_rref(eng, reps=3):
    """Config 2: RREF + rank + det of RankedMatrix(4096, 4096, 3900, 2^31 - 19), device-resident;
    beside it the reference's elim::rref under the tape's host elimination hook on all host threads."""
    import torch

    import oracle as O
    from hacs_b200 import gen

    g = _golden().get("config2", {})
    p, n, r = 2147483629, 4096, 3900
    L, R = gen.ranked_factors(n, n, r, p)
    A0 = torch.empty((n, n), dtype=torch.int32, device="cuda")
    eng.gemm_dev(p, torch.from_numpy(L.view(np.int32)).cuda(), torch.from_numpy(R.view(np.int32)).cuda(), A0)
    eng.sync()
    A = torch.empty_like(A0)
    times = []
    for _ in range(reps + 1):
        A.copy_(A0)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        piv = eng.rref_dev(p, A)
        times.append(time.perf_counter() - t0)
    t = min(times[1:])
    ok = gen.fnv_matrix(A.cpu().numpy().view(np.uint32)) == int(g.get("rref_fnv", "0x0"), 16)
    # per-kernel device times of one more RREF (CUDA events around each launch)
    A.copy_(A0)
    eng.set_timing(True)
    eng.timing_reset()
    b0, s0 = eng.elim_panel_stats()
    eng.rref_dev(p, A)
    eng.sync()
    b1, s1 = eng.elim_panel_stats()
    kern = kernel_breakdown(eng, ["panel_block", "panel_w", "panel_factor", "limb_split", "limb_gemm", "trsm", "row_permute",
                                  "tri_inv", "gather_cols", "assemble_rref", "gather", "copy"])
    eng.set_timing(False)
    lu = n * n * r - (n + n) * r * r / 2 + r ** 3 / 3
    back = r * r * (n - r) / 2
    work = lu + back
    peak, psrc = int8_peak_tops()
    hbm, hsrc = hbm_peak_gbs()
    # tensor part: every modMAC of the LU and the back substitution is L^2 = 16 int8 limb products (2 ops each)
    achieved = 16 * 2 * work / t / 1e12
    gemm_ms = kern.get("limb_gemm", [0, 0])[0]
    panel_ms = kern.get("panel_factor", [0, 0])[0] + kern.get("panel_block", [0, 0])[0]
    panel_bytes = 8.0 * n * 64 * (n // 64)  # read + write of the active rows of every 64-column panel (upper bound m)
    out = {"workload": "RREF/rank/det 4096^2 rank 3900 p=2^31-19 (config 2)", "ms": t * 1e3, "rank": int(len(piv)),
           "modmac_per_s": work / t, "checksum_ok_vs_reference": bool(ok), "kernels_ms": kern,
           "panels": {"settled_by_top_block": b1 - b0, "searched": s1 - s0},
           "roofline": {"bound": "tensor (trailing updates) / latency (panels)", "achieved_int8_tops": achieved,
                        "peak": peak, "unit": "TOPS", "frac": achieved / peak, "peak_source": psrc,
                        "algorithmic": f"LU {lu:.3e} + back substitution {back:.3e} modMAC, 32 int8 ops each",
                        "limb_gemm_int8_tops": (32 * work / (gemm_ms / 1e3) / 1e12) if gemm_ms else None,
                        "panel_share": panel_ms / max(1e-9, sum(v[0] for v in kern.values())),
                        "panel_gbs": (panel_bytes / (panel_ms / 1e3) / 1e9) if panel_ms else None,
                        "panel_hbm_frac": (panel_bytes / (panel_ms / 1e3) / 1e9 / hbm) if panel_ms else None,
                        "hbm_peak_source": hsrc}}
    if O.ref_available():
        thr = host_threads()
        Ah = A0.cpu().numpy().view(np.uint32).copy()
        t0 = time.perf_counter()
        Rr, pr = O.ref_rref_par(p, Ah, threads=thr)
        tc = time.perf_counter() - t0
        out["cpu_baseline"] = {"value_ms": tc * 1e3, "modmac_per_s": work / tc, "cores": thr, "kind": "reference",
                               "sample": "the full config: elim::rref under tape::ScopedHostElimHook on a "
                                         f"{thr}-worker consumer pool, one run",
                               "checksum_ok": bool(O.fnv_matrix(Rr) == int(g.get("rref_fnv", "0x0"), 16)),
                               **cpu_info()}
        out["speedup_vs_cpu"] = tc / t
    return out


def extra_ring(eng, reps=3):
    """Config 3: Howell over Z/2^16 and Smith over Z/3^10 of planted 2048^2 U*D*V; beside each
    the reference's ring2k::howell / ring3k::smith under smithpar::ScopedEnable on all host threads."""
    import oracle as O
    from hacs_b200 import gen

    g = _golden().get("config3", {})
    out = {}
    peak, psrc = int8_peak_tops()
    for (ell, k, kind) in [(2, 16, "howell"), (3, 10, "smith"), (2, 16, "smith"), (3, 10, "howell")]:
        M, e = gen.planted_udv(2048, ell, k, 0x33)
        fn = (lambda: eng.howell(ell, k, M)) if kind == "howell" else (lambda: eng.smith(ell, k, M))
        fn()
        ts = []
        for _ in range(reps):
            t0 = time.perf_counter()
            res = fn()
            ts.append(time.perf_counter() - t0)
        c = g.get(f"{ell}^{k}", {})
        if kind == "howell":
            ok = gen.fnv_matrix(res[0]) == int(c.get("howell_fnv", "0x0"), 16)
        else:
            ok = list(res) == c.get("sigma")
        t = min(ts)
        n = 2048
        work = n ** 3 / 3.0
        # limb products per multiply-add mod ell^k: 4 for 2^16 (two limbs) and for 3^10 (two limbs)
        achieved = 4 * 2 * work / t / 1e12
        rec = {"ms": t * 1e3, "bit_exact_vs_reference": bool(ok), "api": "host pointers (H2D + D2H inside)",
               "roofline": {"bound": "tensor (trailing updates) / latency (panels, Howell pass)",
                            "achieved_int8_tops": achieved, "peak": peak, "unit": "TOPS", "frac": achieved / peak,
                            "peak_source": psrc, "algorithmic": "n^3/3 multiply-adds mod ell^k, 4 limb products each"}}
        if O.ref_available() and (ell, kind) in ((2, "howell"), (3, "smith")):
            thr = host_threads()
            t0 = time.perf_counter()
            if kind == "howell":
                H, _, _ = O.ref_howell_2k(k, M, threads=thr)
                cok = gen.fnv_matrix(H) == int(c.get("howell_fnv", "0x0"), 16)
                what = "ring2k::howell<Traits<uint32_t>>"
            else:
                sg = O.ref_smith_3k(k, M, threads=thr)
                cok = list(sg) == c.get("sigma")
                what = "ring3k::smith"
            tc = time.perf_counter() - t0
            rec["cpu_baseline"] = {"value_ms": tc * 1e3, "cores": thr, "kind": "reference",
                                   "sample": f"the full config: {what} under smithpar::ScopedEnable, one run",
                                   "checksum_ok": bool(cok), **cpu_info()}
            rec["speedup_vs_cpu"] = tc / t
        out[f"{kind}_2048_{ell}^{k}"] = rec
    return out


def cpu_job_rate(stream_s, fam, p, sa, sb, idx, threads):
    """The reference CPU engine on the jobs `idx` of the stream (kernels::gemm + column_rank_profile per
    job, one job per worker process, spawn pool of `threads`); returns (jobs/s, seconds, results)."""
    import multiprocessing as mp

    import oracle as O

    tasks = [(int(j), int(stream_s[j]), int(fam[j]), int(p[j]), int(sa[j]), int(sb[j])) for j in idx]
    tasks.sort(key=lambda t: -t[1])
    with mp.get_context("spawn").Pool(threads) as pool:
        pool.map(O.ref_job, tasks[-threads:])  # warm the workers (library load)
        t0 = time.perf_counter()
        res = pool.map(O.ref_job, tasks, chunksize=1)
        dt = time.perf_counter() - t0
    return len(tasks) / dt, dt, {j: (r, f) for j, r, f in res}


def extra_jobstream(eng, plain, n_jobs=10000, sample=500):
    """Config 4: the 10,000-job stream (GEMM + rank per job, sides 16..1024), batched, checked job by job
    against the reference CPU engine's results (tests/golden/jobs10000.json); beside it one-launch-per-job
    plain dispatch and the reference CPU engine, both on a strided sample of `sample` jobs."""
    import ctypes as C_

    import torch

    import hacs_b200
    import oracle as O
    from hacs_b200 import stream

    st = stream.DeviceStream(n_jobs)
    arr = eng._jobs(st.jobs)

    def batched(nj, a):
        ranks = np.zeros(nj, np.uint32)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        hacs_b200.check(eng._lib.hme_batch_gemm_rank_u32_dev(eng._h, nj, a, ranks.ctypes.data_as(C_.POINTER(C_.c_uint32))))
        return time.perf_counter() - t0, ranks

    eng.gen_jobs_dev(st.specs)
    batched(n_jobs, arr)  # warm: workspace growth, module load
    eng.gen_jobs_dev(st.specs)
    t_all, ranks = batched(n_jobs, arr)
    work = st.work_modmac()
    out = {"workload": f"{n_jobs} jobs GEMM + rank mod p in {{65521, 2^31-19}}, sides log-uniform 16..1024 (config 4)",
           "jobs_per_s": n_jobs / t_all, "s": t_all, "modmac_gemm": work}
    # parity: every rank and every C checksum against the reference's own results
    gold = stream.golden_jobs()
    eng.gen_jobs_dev(st.specs)
    hacs_b200.check(eng._lib.hme_batch_gemm_u32_dev(eng._h, n_jobs, arr))
    eng.sync()
    fnvs = st.job_checksums()
    if gold is not None and len(gold[0]) == n_jobs:
        out["ranks_equal_vs_reference"] = bool(np.array_equal(ranks.astype(np.int64), gold[0]))
        out["c_fnv_equal_vs_reference"] = bool(fnvs == gold[1])
        out["parity_source"] = "tests/golden/jobs10000.json (reference kernels::gemm + elim::column_rank_profile)"
    # roofline: GEMM + rank at the limb GEMM's INT8 rate; a rank of an s x s job is ~ s^3/3 multiply-adds
    limbs2 = np.where(st.p == 65521, 4, 16).astype(np.float64)
    s3 = st.s.astype(np.float64) ** 3
    int8_ops = float((limbs2 * 2 * (s3 + s3 / 3)).sum())
    peak, psrc = int8_peak_tops()
    out["roofline"] = {"bound": "tensor (GEMMs, trailing updates) / latency (panels)",
                       "achieved_int8_tops": int8_ops / t_all / 1e12, "peak": peak, "unit": "TOPS",
                       "frac": int8_ops / t_all / 1e12 / peak, "peak_source": psrc,
                       "algorithmic": "sum_j L_j^2 * 2 * (s_j^3 + s_j^3 / 3) int8 ops (GEMM + rank)"}
    # strided sample: every (n_jobs / sample)-th job
    idx = np.arange(0, n_jobs, max(1, n_jobs // sample))[:sample]
    sub_jobs = [st.jobs[j] for j in idx]
    sub_specs = [st.specs[2 * j + t] for j in idx for t in (0, 1)]
    eng.gen_jobs_dev(sub_specs)
    t_b, r_b = batched(len(idx), eng._jobs(sub_jobs))
    out["sample_jobs"] = int(len(idx))
    out["sample"] = f"every {max(1, n_jobs // sample)}th job of the stream"
    out["sample_batched_jobs_per_s"] = len(idx) / t_b
    if plain is not None:
        # (a) one plain CUDA-core GEMM launch per job (the reference's cuda::gemm) + this library's
        #     single-job device rank, synchronised per job
        eng.gen_jobs_dev(sub_specs)
        eng.use_torch_stream()
        cst = torch.cuda.current_stream().cuda_stream
        r2 = np.zeros(len(idx), np.uint32)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for t, jb in enumerate(sub_jobs):
            n = jb["C"].shape[0]
            if plain.plain_gemm_u32_dev(jb["p"], n, n, n, jb["A"].data_ptr(), n, jb["B"].data_ptr(), n,
                                        jb["C"].data_ptr(), n, 0, cst) != 0:
                raise RuntimeError(plain.plain_last_error().decode())
            rr = np.zeros(1, np.uint32)
            hacs_b200.check(eng._lib.hme_batch_rank_u32_dev(eng._h, 1, eng._jobs([jb]),
                                                            rr.ctypes.data_as(C_.POINTER(C_.c_uint32))))
            r2[t] = rr[0]
        t_p = time.perf_counter() - t0
        out["sample_plain_dispatch_jobs_per_s"] = len(idx) / t_p
        out["speedup_vs_plain_dispatch"] = t_p / t_b
        # (b) the reference's own path for p > 127: one plain GEMM launch per job, C back to the host,
        #     elim::column_rank_profile on the host (the reference has no device rank at these p)
        if O.ref_available():
            eng.gen_jobs_dev(sub_specs)
            r3 = np.zeros(len(idx), np.uint32)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            for t, jb in enumerate(sub_jobs):
                n = jb["C"].shape[0]
                if plain.plain_gemm_u32_dev(jb["p"], n, n, n, jb["A"].data_ptr(), n, jb["B"].data_ptr(), n,
                                            jb["C"].data_ptr(), n, 0, cst) != 0:
                    raise RuntimeError(plain.plain_last_error().decode())
                Ch = jb["C"].cpu().numpy().view(np.uint32)
                r3[t] = len(O.ref_rank_profile(jb["p"], Ch))
            t_r = time.perf_counter() - t0
            out["sample_reference_path_jobs_per_s"] = len(idx) / t_r
            out["speedup_vs_reference_path"] = t_r / t_b
            out["reference_path"] = "cuda::gemm per job (plain, sm_100a) + C to host + elim::column_rank_profile"
        eng.use_own_stream()
        out["sample_ranks_equal_plain"] = bool((r2 == r_b).all())
    if O.ref_available():
        thr = host_threads()
        rate, tc, res = cpu_job_rate(st.s, st.fam, st.p, st.seed_a, st.seed_b, idx, thr)
        out["cpu_baseline"] = {"value_jobs_per_s": rate, "cores": thr, "kind": "reference",
                               "sample": f"{len(idx)} jobs (every {max(1, n_jobs // sample)}th), kernels::gemm + "
                                         f"elim::column_rank_profile per job on a {thr}-process pool, {tc:.1f} s",
                               "ranks_equal": bool(all(res[int(j)][0] == int(r_b[t]) for t, j in enumerate(idx))),
                               **cpu_info()}
        out["speedup_vs_cpu"] = (n_jobs / t_all) / rate
    return out


def serve_stream(eng, ms, plan, rank_plan=None, warm: bool = False):
    """Serve the mixed stream in its chunks with per-job GEMM schedules `plan` and
    rank schedules `rank_plan` (hme_batch_gemm_rank_u32_dev_sched; None: the rank
    rounds' batch rule); returns (seconds inside the calls, ranks)."""
    import ctypes as C_

    import torch

    import hacs_b200

    ranks = np.zeros(ms.n_jobs, np.uint32)
    total = 0.0
    for c0, c1 in ms.chunks():
        jobs, specs = ms.device_chunk(c0, c1)
        eng.gen_jobs_dev(specs)
        arr = eng._jobs(jobs)
        var = np.ascontiguousarray(plan[c0:c1], dtype=np.int32)
        rvar = np.ascontiguousarray(np.full(c1 - c0, -1) if rank_plan is None else rank_plan[c0:c1], dtype=np.int32)
        out = np.zeros(c1 - c0, np.uint32)
        ip = C_.POINTER(C_.c_int)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        hacs_b200.check(eng._lib.hme_batch_gemm_rank_u32_dev_sched(eng._h, c1 - c0, arr, var.ctypes.data_as(ip),
                                                                   rvar.ctypes.data_as(ip),
                                                                   out.ctypes.data_as(C_.POINTER(C_.c_uint32))))
        total += time.perf_counter() - t0
        ranks[c0:c1] = out
        if warm:
            break
    return total, ranks


def extra_scheduler(eng, n_stream=50000):
    """Config 5: the 50,000-job mixed stream (stream.MixedStream: config-4 jobs, config-2 rank-deficient
    products, config-1 products) served end to end through the batched GEMM + rank call under four plans,
    each a per-job GEMM schedule and a per-job rank-round schedule (trailing-update variant, widest last
    panel): the learned planners' (two MLPs trained on this engine's batch autotuner timings of the GEMM
    phase and of the rank rounds, one BF16 inference launch each for the whole stream), the same networks
    with the exhaustive autotuner as their fallback in the shape classes where a network is not
    confident, the batch rules (the method without the networks) and the exhaustive batch autotuners'
    best per shape class.  Ranks are checked across plans and against the reference / the construction."""
    from hacs_b200 import sched, stream

    if not os.path.exists(sched.BATCH_WEIGHTS):
        return {"unavailable": "no trained batch-planner weights in the package"}
    have_rank = os.path.exists(sched.RANK_WEIGHTS)
    ms = stream.MixedStream(n_stream)
    shapes, dens = ms.shapes(), ms.density()
    mlp = sched.MLP(eng)
    mlp.load(sched.BATCH_WEIGHTS)
    mlp.plan(shapes[:64], dens[:64])  # warm
    t0 = time.perf_counter()
    learned = mlp.plan(shapes, dens)
    t_plan = time.perf_counter() - t0
    t0 = time.perf_counter()
    learned_fb, fb_classes = sched.plan_with_fallback(mlp, eng, shapes, dens)
    t_fb = time.perf_counter() - t0
    mlp.close()
    rule_rank = np.full(ms.n_jobs, sched.BATCH_RULE, np.int32)
    learned_rank = learned_fb_rank = rule_rank
    t_plan_rank = t_fb_rank = 0.0
    fb_classes_rank = 0
    if have_rank:
        mlp_r = sched.MLP(eng)
        mlp_r.load(sched.RANK_WEIGHTS)
        mlp_r.plan_rank(shapes[:64], dens[:64])  # warm
        t0 = time.perf_counter()
        learned_rank = mlp_r.plan_rank(shapes, dens)
        t_plan_rank = time.perf_counter() - t0
        t0 = time.perf_counter()
        learned_fb_rank, fb_classes_rank = sched.plan_with_fallback(mlp_r, eng, shapes, dens, rank=True)
        t_fb_rank = time.perf_counter() - t0
        mlp_r.close()
    # the exhaustive autotuners: every variant timed inside a batch, once per shape class of the stream
    t0 = time.perf_counter()
    first = {}
    for t in range(ms.n_jobs):
        first.setdefault(sched.shape_class(*shapes[t]), t)
    T = {key: sched.autotune_batch(eng, *shapes[t]) for key, t in first.items()}
    TR = ({key: sched.autotune_batch_rank(eng, *shapes[t], dens[t]) for key, t in first.items()}
          if have_rank else {})
    t_tune = time.perf_counter() - t0
    keys = [sched.shape_class(*row) for row in shapes]
    best = np.array([int(np.argmin(T[k])) for k in keys], np.int32)
    best_rank = np.array([int(np.argmin(TR[k])) for k in keys], np.int32) if have_rank else rule_rank
    rule = np.full(ms.n_jobs, sched.BATCH_RULE, np.int32)
    serve_stream(eng, ms, rule, warm=True)  # workspace growth, module load
    res = {}
    for name, plan, rplan in (("heuristic", rule, rule_rank), ("learned", learned, learned_rank),
                              ("learned_with_fallback", learned_fb, learned_fb_rank),
                              ("autotuner_best", best, best_rank)):
        ts, rk = [], None
        for _ in range(2):
            t, r = serve_stream(eng, ms, plan, rplan)
            ts.append(t)
            if rk is not None:
                assert np.array_equal(rk, r)
            rk = r
        res[name] = (min(ts), rk)
    t_h, r_h = res["heuristic"]
    t_l, r_l = res["learned"]
    t_n, r_n = res["learned_with_fallback"]
    t_b, r_b = res["autotuner_best"]
    per_job = np.array([T[k] for k in keys])  # per-job batch times of every variant, by class
    rows = np.arange(ms.n_jobs)
    out = {"workload": f"{ms.n_jobs}-job mixed stream (config-4 jobs incl. all 10,000 of config 4, config-2 "
                       "rank-deficient products at 2^31-19, config-1 1024^3 products), GEMM + rank per job, "
                       f"served in chunks of {ms.chunk} (config 5)",
           "jobs_per_s_served": {"learned": ms.n_jobs / t_l, "heuristic": ms.n_jobs / t_h,
                                 "learned_with_fallback": ms.n_jobs / t_n, "autotuner_best": ms.n_jobs / t_b},
           "served_s": {"learned": t_l, "heuristic": t_h, "learned_with_fallback": t_n, "autotuner_best": t_b},
           "regret_served_learned": (t_l - t_b) / t_b, "regret_served_heuristic": (t_h - t_b) / t_b,
           "regret_served_learned_with_fallback": (t_n - t_b) / t_b,
           "learned_vs_heuristic": t_h / t_l,
           "fallback": {"margin": 0.03, "gemm_classes": fb_classes, "rank_classes": fb_classes_rank,
                        "gemm_s": t_fb, "rank_s": t_fb_rank,
                        "rule": "a class falls back to the exhaustive autotuner when the network's best predicted "
                                "time is within 3 % of its second best (sched.plan_with_fallback)"},
           "regret_per_job_model_learned": float(np.mean((per_job[rows, learned] - per_job.min(1)) / per_job.min(1))),
           "plan_ms": t_plan * 1e3, "plan_rank_ms": t_plan_rank * 1e3, "autotune_s": t_tune,
           "shape_classes": len(first),
           "variant_share_learned": np.bincount(learned, minlength=sched.N_VARIANTS).tolist(),
           "variant_share_best": np.bincount(best, minlength=sched.N_VARIANTS).tolist(),
           "rank_variants": list(sched.RANK_VARIANT_NAMES),
           "rank_variant_share_learned": np.bincount(np.maximum(learned_rank, 0),
                                                     minlength=sched.N_RANK_VARIANTS).tolist(),
           "rank_variant_share_best": np.bincount(np.maximum(best_rank, 0), minlength=sched.N_RANK_VARIANTS).tolist(),
           "ranks_equal_across_plans": bool(np.array_equal(r_h, r_l) and np.array_equal(r_h, r_b)
                                            and np.array_equal(r_h, r_n)),
           "rank_checks": ms.check_ranks(r_l),
           "planner": "MLP 5-64-64-64-4 (hand-written FP32 training / BF16 inference kernels) trained on "
                      "hme_autotune_batch timings (python -m hacs_b200.sched_train --batch); the rank rounds' "
                      "planner: the same network trained on hme_autotune_batch_rank timings "
                      "(python -m hacs_b200.sched_train --rank)" + ("" if have_rank else " -- not trained: rule")}
    if have_rank:
        per_job_r = np.array([TR[k] for k in keys])
        out["regret_per_job_model_learned_rank"] = float(np.mean(
            (per_job_r[rows, learned_rank] - per_job_r.min(1)) / per_job_r.min(1)))
        rr = sched.rank_rule(shapes[:, 1])
        out["regret_per_job_model_rule_rank"] = float(np.mean((per_job_r[rows, rr] - per_job_r.min(1)) /
                                                              per_job_r.min(1)))
    return out


def gemm64_rate(n, p, steps=3, warmup=2):
    """n^3 GEMM over u64 residues: hme (residue system over the limb GEMM) vs the plain method."""
    import torch

    import hacs_b200

    torch.cuda.set_stream(torch.cuda.Stream())
    eng = hacs_b200.Engine(0)
    eng.use_torch_stream()
    rng = np.random.default_rng(11)
    A = torch.from_numpy(rng.integers(0, p, (n, n), dtype=np.uint64).view(np.int64)).cuda()
    B = torch.from_numpy(rng.integers(0, p, (n, n), dtype=np.uint64).view(np.int64)).cuda()
    Cm = torch.empty((n, n), dtype=torch.int64, device="cuda")
    ms = time_device(lambda: eng.gemm_u64_dev(p, A, B, Cm), steps, warmup) / steps
    eng.sync()
    out = {"p": p, "n": n, "ms": ms, "tops": 2.0 * n ** 3 / ms / 1e9}
    # per-kernel CUDA-event times of one more call (library timer on the launching stream)
    eng.set_timing(True)
    eng.timing_reset()
    eng.gemm_u64_dev(p, A, B, Cm)
    eng.sync()
    out["kernels_ms"] = {k: round(eng.kernel_time(k)[0], 4) for k in
                         ("rns_split", "rns_crt", "narrow", "widen", "limb_split", "limb_gemm", "simt_gemm")
                         if eng.kernel_time(k)[1]}
    eng.set_timing(False)
    plain = load_plain()
    if plain is not None and hasattr(plain, "plain_gemm_u64_dev"):
        Cp = torch.empty_like(Cm)
        st = torch.cuda.current_stream().cuda_stream

        def run_plain():
            rc = plain.plain_gemm_u64_dev(p, n, n, n, A.data_ptr(), n, B.data_ptr(), n, Cp.data_ptr(), n, 0, st)
            if rc != 0:
                raise RuntimeError(plain.plain_last_error().decode())

        pms = time_device(run_plain, 1, 1)
        out.update({"plain_gpu_ms": pms, "plain_gpu_tops": 2.0 * n ** 3 / pms / 1e9, "speedup_vs_plain": pms / ms,
                    "bit_exact_vs_plain": bool(torch.equal(Cm, Cp))})
    eng.close()
    return out


def run_case(args):
    """One kernel configuration for an ncu capture (prints a short JSON, not a bench line)."""
    import torch

    import hacs_b200

    parts = args.case.split(":")
    kind = parts[0]
    if kind == "rref":
        # rref:<n>:<rank>:<p>: the config-2 family (RankedMatrix factors, device-resident elimination)
        from hacs_b200 import gen

        n, r, p = int(parts[1]), int(parts[2]), int(parts[3])
        eng = hacs_b200.Engine(0)
        if len(parts) > 4:  # rref:<n>:<rank>:<p>:<panel>:<rows per CTA>[:<lookahead 0|1>] (tuning only)
            eng.set_elim_options(panel=int(parts[4]), rows_per_cta=int(parts[5]) if len(parts) > 5 else 0)
        if len(parts) > 6:
            eng.set_elim_lookahead(parts[6] != "0")
        L, R = gen.ranked_factors(n, n, r, p)
        A = eng.gemm(p, L, R)
        t0 = time.perf_counter()
        for _ in range(max(1, args.warmup + args.steps)):
            Rr, piv, d = eng.rref_det(p, A)
        dt = (time.perf_counter() - t0) / max(1, args.warmup + args.steps)
        print(json.dumps(default=_json, obj={"case": args.case, "rank": int(len(piv)), "det": int(d), "s_per_rref": dt,
                          "rref_fnv": hex(gen.fnv_matrix(Rr))}), flush=True)
        eng.close()
        return 0
    if kind in ("howell", "smith"):
        # howell:<n>:<ell>:<k> / smith:<n>:<ell>:<k>: planted U*D*V (the config-3 family), host pointers
        from hacs_b200 import gen

        n, ell, k = int(parts[1]), int(parts[2]), int(parts[3])
        eng = hacs_b200.Engine(0)
        M, _ = gen.planted_udv(n, ell, k, 0x33)
        fn = (lambda: eng.howell(ell, k, M)) if kind == "howell" else (lambda: eng.smith(ell, k, M))
        t0 = time.perf_counter()
        for _ in range(max(1, args.warmup + args.steps)):
            out = fn()
        dt = (time.perf_counter() - t0) / max(1, args.warmup + args.steps)
        size = int(out[0].shape[0]) if kind == "howell" else int(len(out))
        print(json.dumps(default=_json, obj={"case": args.case, "s_per_call": dt, "rows_or_invariants": size}),
              flush=True)
        eng.close()
        return 0
    if kind == "jobs":
        # jobs:<count>[:<rank schedule>]: the first <count> jobs of the config-4 stream, batched GEMM + rank
        # (every job's rank rounds on the given schedule, 0..3; default: the batch rule)
        import ctypes as C_

        from hacs_b200 import gen, stream

        nj = int(parts[1])
        rv = int(parts[2]) if len(parts) > 2 else -1
        eng = hacs_b200.Engine(0)
        s, fam, pj, sa, sb = gen.job_stream(10000)
        s, fam, pj, sa, sb = s[:nj], fam[:nj], pj[:nj], sa[:nj], sb[:nj]
        tot = int((s * s).sum())
        bufs = [torch.empty(tot, dtype=torch.int32, device="cuda") for _ in range(3)]
        jobs, specs, off = [], [], 0
        for j in range(nj):
            n = int(s[j])
            A, B, Cm = (b[off:off + n * n].view(n, n) for b in bufs)
            off += n * n
            jobs.append({"p": int(pj[j]), "A": A, "B": B, "C": Cm})
            specs += [(A, int(pj[j]), int(fam[j]), int(sa[j])), (B, int(pj[j]), int(fam[j]), int(sb[j]))]
        arr = eng._jobs(jobs)
        ranks = np.zeros(nj, np.uint32)
        rvar = np.full(nj, rv, np.int32)
        ip = C_.POINTER(C_.c_int)

        def stream_once():
            hacs_b200.check(eng._lib.hme_batch_gemm_rank_u32_dev_sched(eng._h, nj, arr, None, rvar.ctypes.data_as(ip),
                                                                       ranks.ctypes.data_as(C_.POINTER(C_.c_uint32))))

        for _ in range(max(0, args.warmup)):
            eng.gen_jobs_dev(specs)
            stream_once()
        dt = 0.0
        for _ in range(max(1, args.steps)):
            eng.gen_jobs_dev(specs)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            stream_once()
            dt += time.perf_counter() - t0
        dt /= max(1, args.steps)
        out = {"case": args.case, "s_per_stream": dt, "jobs_per_s": nj / dt, "rank_sum": int(ranks.sum())}
        gold = stream.golden_jobs() if nj <= 10000 else None
        if gold is not None:
            out["ranks_equal_reference"] = bool(np.array_equal(ranks.astype(np.int64), gold[0][:nj]))
        # per-kernel device times of one more stream (library timer: rounds launched directly, no graph)
        eng.set_timing(True)
        eng.timing_reset()
        eng.gen_jobs_dev(specs)
        stream_once()
        eng.sync()
        names = ("grouped_gemm", "grouped_split", "batch_panel", "batch_simt_update", "batch_trsm",
                 "batch_permute", "batch_gather", "rank_post", "rank_plan", "limb_gemm", "simt_gemm")
        out["kernels_ms"] = {k: round(eng.kernel_time(k)[0], 3) for k in names if eng.kernel_time(k)[1]}
        eng.set_timing(False)
        print(json.dumps(default=_json, obj=out), flush=True)
        eng.close()
        return 0
    if kind == "mlp":
        # mlp:<rows>: scheduler MLP training epochs (FP32 forward + backward, Adam) and a BF16 plan
        from hacs_b200 import sched

        rows = int(parts[1])
        eng = hacs_b200.Engine(0)
        rng = np.random.default_rng(5)
        X = rng.standard_normal((rows, 5)).astype(np.float32)
        Y = rng.standard_normal((rows, sched.N_VARIANTS)).astype(np.float32)
        mlp = sched.MLP(eng)
        loss = mlp.train_normalised(X, Y, epochs=max(1, args.steps), batch=256)
        shapes, dens = sched.sample_shapes(rows, seed=3)
        plan = mlp.plan(shapes, dens)
        print(json.dumps(default=_json, obj={"case": args.case, "loss": float(loss),
                          "plan_share": np.bincount(plan, minlength=sched.N_VARIANTS).tolist()}), flush=True)
        mlp.close()
        eng.close()
        return 0
    if kind == "sched5":
        # sched5[:<jobs>]: the config-5 mixed stream served under the learned, batch-rule and autotuned plans
        # (both phases' schedules), the same figures as the bench line's extras.scheduler_config5
        torch.cuda.set_stream(torch.cuda.Stream())
        eng = hacs_b200.Engine(0)
        eng.use_torch_stream()
        out = extra_scheduler(eng, int(parts[1]) if len(parts) > 1 else 50000)
        print(json.dumps(default=_json, obj={"case": args.case, **out}), flush=True)
        eng.close()
        return 0
    if kind == "gemm64":
        # gemm64:<n>:<p>: n^3 GEMM over u64 residues mod p (any p < 2^64) through hme_gemm_u64_dev, next to the
        # reference's own u64 CUDA-core GEMM (the plain method) on the same device buffers
        n, p = int(parts[1]), int(parts[2])
        out = gemm64_rate(n, p, max(1, args.steps), args.warmup)
        print(json.dumps(default=_json, obj={"case": args.case, **out}), flush=True)
        return 0
    if kind == "level12":
        # level12:<m>:<n>:<p>: the device level-1 / level-2 operations on m x n operands (larger than L2 at
        # 8192 x 8192), each timed alone with CUDA events; GB/s of algorithmic bytes
        m, n, p = int(parts[1]), int(parts[2]), int(parts[3])
        torch.cuda.set_stream(torch.cuda.Stream())
        eng = hacs_b200.Engine(0)
        eng.use_torch_stream()
        g = torch.Generator(device="cuda").manual_seed(2)

        def rnd(*shape):
            return torch.randint(0, p, shape, dtype=torch.int64, device="cuda", generator=g).to(torch.int32)

        X, Y, Z = rnd(m, n), rnd(m, n), torch.empty((n, m), dtype=torch.int32, device="cuda")
        x, y = rnd(n), rnd(m)
        rows = torch.randperm(m, device="cuda", generator=g)[: m // 2].to(torch.int32)
        W = torch.empty((m // 2, n), dtype=torch.int32, device="cuda")
        acc = torch.randint(0, 2**62, (m, n), dtype=torch.int64, device="cuda", generator=g)
        nrhs = 256
        T, Bt = rnd(m, m), rnd(m, nrhs)
        steps, warm = max(1, args.steps), args.warmup
        ops = {  # name -> (call, algorithmic bytes per call)
            "gemv": (lambda: eng.gemv_dev(p, X, x, y), 4 * (m * n + n + 2 * m)),
            "axpy": (lambda: eng.axpy_dev(p, 7 % p, X, Y), 12 * m * n),
            "scal": (lambda: eng.scal_dev(p, 3 % p, Y), 8 * m * n),
            "copy": (lambda: eng.copy_dev(X, Y), 8 * m * n),
            "transpose": (lambda: eng.transpose_dev(X, Z), 8 * m * n),
            "fill": (lambda: eng.fill_dev(Y, 1), 4 * m * n),
            "gather_rows": (lambda: eng.gather_dev(p, 1, 5 % p, X, 0, None, W, False, rows), 8 * (m // 2) * n),
            "canonicalise_acc64": (lambda: eng.canonicalise_acc64_dev(p, acc, Y), 12 * m * n),
            "trsm_unit_lower": (lambda: eng.trsm_unit_dev(p, T, Bt, True), 4 * (m * m // 2 + 2 * m * nrhs)),
        }
        out = {"case": args.case}
        for name, (fn, nbytes) in ops.items():
            ms = time_device(fn, steps, warm) / steps
            out[name] = {"ms": round(ms, 4), "gbs": round(nbytes / ms / 1e6, 1)}
        eng.sync()
        print(json.dumps(default=_json, obj=out), flush=True)
        eng.close()
        return 0
    # gemm:<n>:<p> (scheduler's variant) or gemm:<n>:<p>:<variant> (0 wide, 1 narrow, 2 simt32, 3 simt64)
    n, p = int(parts[1]), int(parts[2])
    assert kind == "gemm"
    torch.cuda.set_stream(torch.cuda.Stream())
    eng = hacs_b200.Engine(0)
    eng.use_torch_stream()
    if len(parts) > 3:
        hacs_b200.check(eng._lib.hme_ctx_set_gemm_variant(eng._h, int(parts[3])))
    g = torch.Generator(device="cuda").manual_seed(1)
    A = torch.randint(0, p, (n, n), dtype=torch.int64, device="cuda", generator=g).to(torch.int32)
    B = torch.randint(0, p, (n, n), dtype=torch.int64, device="cuda", generator=g).to(torch.int32)
    Cm = torch.empty((n, n), dtype=torch.int32, device="cuda")
    ms = time_device(lambda: eng.gemm_dev(p, A, B, Cm), max(1, args.steps), args.warmup)
    eng.sync()
    print(json.dumps(default=_json, obj={"case": args.case, "ms_per_gemm": ms / max(1, args.steps),
                      "tops": 2.0 * n ** 3 * max(1, args.steps) / ms / 1e9}), flush=True)
    eng.close()
    return 0


def multi_gpu_extras(eng, ws, rank, local):
    """The paths that shard across N GPUs (one process per GPU), timed on the device as the max over ranks:
    one 8192^3 GEMM split by rows of C (A's row block and B on every rank, C all-gathered over NCCL; no
    reduction), and the 10,000-job stream split by predicted cost (each rank one batched call on its share;
    ranks gathered on the host).  Every rank takes the same collective steps in the same order."""
    import ctypes as C_

    import torch
    import torch.distributed as dist

    import hacs_b200
    from hacs_b200 import shard, stream

    out = {}
    for p in (65521, 2147483629):
        n = 8192
        g = torch.Generator(device="cuda").manual_seed(p)
        A = torch.randint(0, p, (n, n), dtype=torch.int64, device="cuda", generator=g).to(torch.int32)
        B = torch.randint(0, p, (n, n), dtype=torch.int64, device="cuda", generator=g).to(torch.int32)
        blocks = shard.row_blocks(n, ws)
        r0, r1 = blocks[rank]
        Cb = torch.empty((r1 - r0, n), dtype=torch.int32, device="cuda")

        def block_gemm(pp, Ab, Bb):
            eng.gemm_dev(pp, Ab, Bb, Cb)
            return Cb

        for _ in range(2):  # warm: workspace, modules, NCCL channels
            shard.gemm_row_split(block_gemm, p, A, B, rank, ws)
        torch.cuda.synchronize()
        dist.barrier()
        e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        e0.record()
        eng.gemm_dev(p, A[r0:r1], B, Cb)
        e1.record()
        C = shard.gemm_row_split(lambda pp, Ab, Bb: Cb, p, A, B, rank, ws)  # the gather of the computed blocks
        e2.record()
        torch.cuda.synchronize()
        t_gemm = max_over_ranks(e0.elapsed_time(e1), ws)
        t_all = max_over_ranks(e0.elapsed_time(e2), ws)
        ok = None
        if rank == 0:
            Cf = torch.empty_like(C)
            eng.gemm_dev(p, A, B, Cf)
            torch.cuda.synchronize()
            ok = bool(torch.equal(Cf, C))
        out[f"gemm_{n}_rowsplit_p{p}"] = {
            "ranks": ws, "rows_per_rank": [b1 - b0 for b0, b1 in blocks], "ms_gemm_max": t_gemm,
            "ms_with_allgather_max": t_all, "tops_gemm": 2.0 * n ** 3 / t_gemm / 1e9,
            "tops_with_allgather": 2.0 * n ** 3 / t_all / 1e9, "bit_exact_vs_one_gpu": ok}
        del A, B, Cb, C
        torch.cuda.empty_cache()
    # the job stream, sharded by predicted cost
    from hacs_b200 import gen

    s = gen.job_stream(10000)[0]
    shards = shard.shard_jobs(shard.job_cost(s, s, s), ws)
    st = stream.DeviceStream(10000, indices=shards[rank])
    arr = eng._jobs(st.jobs)
    ranks = np.zeros(max(1, st.n_jobs), np.uint32)

    def call():
        hacs_b200.check(eng._lib.hme_batch_gemm_rank_u32_dev(eng._h, st.n_jobs, arr,
                                                             ranks.ctypes.data_as(C_.POINTER(C_.c_uint32))))

    eng.gen_jobs_dev(st.specs)
    call()  # warm
    eng.gen_jobs_dev(st.specs)
    torch.cuda.synchronize()
    dist.barrier()
    t0 = time.perf_counter()
    call()
    t_rank = time.perf_counter() - t0
    t_max = max_over_ranks(t_rank, ws)
    parts = [None] * ws if rank == 0 else None
    dist.gather_object(ranks[: st.n_jobs].tolist(), parts, dst=0)
    rec = {"ranks": ws, "jobs_per_rank": [len(x) for x in shards], "s_max": t_max, "jobs_per_s": 10000 / t_max}
    if rank == 0:
        allr = np.full(10000, -1, np.int64)
        for r in range(ws):
            allr[shards[r]] = parts[r]
        gold = stream.golden_jobs()
        rec["ranks_equal_vs_reference"] = bool(gold is not None and np.array_equal(allr, gold[0]))
    out["jobstream_config4_sharded"] = rec
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="hme", choices=["hme", "reference"])
    ap.add_argument("--no-extras", action="store_true", help="skip the 8192^3 and plain-method lines")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline")
    ap.add_argument("--case", default=None,
                    help="profiling case instead of the bench line: gemm:<n>:<p>[:<variant>] runs W + K GEMMs "
                         "of n^3 mod p; rref:<n>:<rank>:<p> runs W + K device RREFs of a rank-deficient n x n "
                         "matrix; howell:<n>:<ell>:<k> / smith:<n>:<ell>:<k> runs W + K forms of a planted "
                         "U*D*V; jobs:<count> runs W + K batched GEMM + rank streams of the first <count> jobs; "
                         "mlp:<rows> trains the scheduler MLP for K epochs and plans <rows> shapes; level12:<m>:<n>:<p> "
                         "times the device level-1 / level-2 operations on m x n operands; gemm64:<n>:<p> runs the "
                         "u64-residue GEMM beside the plain method; sched5[:<jobs>] serves the config-5 mixed stream under "
                         "the learned, batch-rule and autotuned plans")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.case:
        return run_case(args)
    args.warmup = max(3, args.warmup)

    ws, rank, local = dist_setup()
    import torch

    import hacs_b200
    from hacs_b200 import gen, limbs_for

    torch.cuda.set_device(local)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)  # torch's events and the library's kernels share one stream
    eng = hacs_b200.Engine(local)
    eng.use_torch_stream()

    p, n = P_HEAD, N_HEAD
    A_h = gen.engine_matrix(n, n, p, 0x01)
    B_h = gen.engine_matrix(n, n, p, 0x02)
    A = torch.from_numpy(A_h.view(np.int32)).cuda()
    B = torch.from_numpy(B_h.view(np.int32)).cuda()
    Cm = torch.empty((n, n), dtype=torch.int32, device="cuda")
    flush_buf = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.int32, device="cuda")

    def flush():
        flush_buf.fill_(1)

    # ---- device-resident timed region ----
    eng.gemm_dev(p, A, B, Cm)
    torch.cuda.synchronize()
    ok = gen.fnv_matrix(Cm.cpu().numpy().view(np.uint32)) == 0x572E8347446366C6
    for _ in range(args.warmup):
        flush()
        eng.gemm_dev(p, A, B, Cm)
    l0 = eng.launches
    barrier(ws)
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        total_ms = time_device(lambda: eng.gemm_dev(p, A, B, Cm), args.steps, 0, flush=flush)
        torch.cuda.synchronize()
    barrier(ws)
    launches = eng.launches - l0
    # per-kernel CUDA events (on the launching stream) in a second pass of the same
    # K steps: events between the launches would stop the GEMM's programmatic
    # dependent launch from overlapping the split in the timed pass above
    eng.set_timing(True)
    eng.timing_reset()
    time_device(lambda: eng.gemm_dev(p, A, B, Cm), args.steps, 0, flush=flush)
    kms, kl = eng.kernel_time("limb_gemm")
    sp, _ = eng.kernel_time("limb_split")
    eng.set_timing(False)
    t_max = max_over_ranks(total_ms, ws)
    ops = 2.0 * n ** 3
    value = ops * args.steps * ws / (t_max / 1e3) / 1e12

    # ---- end to end through the host-pointer API (pinned buffers on the GPU's NUMA node) ----
    with GpuLocalCpus(local) as numa:
        A_pin = torch.from_numpy(A_h.view(np.int32)).pin_memory().numpy().view(np.uint32)
        B_pin = torch.from_numpy(B_h.view(np.int32)).pin_memory().numpy().view(np.uint32)
        C_pin = torch.empty((n, n), dtype=torch.int32).pin_memory().numpy().view(np.uint32)
        for _ in range(3):
            eng.gemm(p, A_pin, B_pin, out=C_pin)
        barrier(ws)
        e2e_s = 0.0
        for _ in range(args.steps):
            flush()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            eng.gemm(p, A_pin, B_pin, out=C_pin)  # synchronous: H2D copies, split, GEMM, D2H copy
            e2e_s += time.perf_counter() - t0
    barrier(ws)
    e2e_s = max_over_ranks(e2e_s, ws)
    e2e_ok = gen.fnv_matrix(C_pin) == 0x572E8347446366C6

    pk, pk_src = peaks()
    int8_peak = 2.0 * float(pk["bf16_tflops"])
    L = limbs_for(p)
    k_avg_ms = kms / max(1, kl)
    achieved = L * L * ops / (k_avg_ms / 1e3) / 1e12
    roof = {"kernel": "limb_gemm", "bound": "tensor", "achieved": achieved, "peak": int8_peak, "unit": "TOPS",
            "frac": achieved / int8_peak, "traffic": profile_traffic("limb_gemm_1024_p65521.md"),
            "peak_source": f"2 x {pk_src} bf16 dense TFLOP/s (INT8 dense rate = 2 x bf16 on B200)",
            "algorithmic_ops_per_launch": L * L * ops, "kernel_ms": k_avg_ms,
            "limb_split_ms": sp / max(1, args.steps),
            "kernel_timing": "CUDA events around each launch, second pass of the same K steps"}

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": t_max / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "u32 residues (u8 limbs x u8 -> s32 tensor-core accumulation)",
        "data": DATA_HEAD,
        "config": head_config(n, p, ws, bool(ok)),
        "e2e": {"value": ops * args.steps * ws / e2e_s / 1e12, "unit": UNIT, "h2d_bytes_per_step": 8 * n * n,
                "d2h_bytes_per_step": 4 * n * n, "api": "hme_gemm_u32 (host pointers, pinned)", "host_numa": numa.note,
                "checksum_ok": bool(e2e_ok)},
        "gpu_launches": launches,
        "roofline": roof,
    }
    if rank == 0 and not args.no_cpu:
        line["cpu_baseline"] = cpu_gemm_rate(p, n)
    line["clocks"] = clk.summary()
    if not args.no_extras and ws > 1:
        line["extras"] = multi_gpu_extras(eng, ws, rank, local)
    elif not args.no_extras:
        plain = load_plain()
        ext = {}
        for pp in (65521, 2147483629):
            ext[f"gemm_8192_p{pp}"] = big_gemm(eng, plain, pp, 8192)
        eng.use_own_stream()
        ext["rref_config2"] = extra_rref(eng)
        ext.update(extra_ring(eng))
        ext["jobstream_config4"] = extra_jobstream(eng, plain)
        ext["scheduler_config5"] = extra_scheduler(eng)
        ext["gemm_u64_2048_p2^61-1"] = gemm64_rate(2048, 2**61 - 1)
        line["extras"] = ext
    if rank == 0:
        print(json.dumps(line, default=_json), flush=True)
    eng.close()
    if ws > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
