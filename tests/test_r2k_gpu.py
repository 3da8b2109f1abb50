"""The Z/2^W device LU session (hme_r2k_*, the device side of the reference's
ring2k::device::Ops table) through the C ABI, step by step, against the
oracle's numpy restatement of a step (oracle/ring2k_ops.py): window
writes, ordered swaps, the unit-lower solve, the wraparound trailing update
(Z/2^32 on the INT8-limb tensor-core GEMM, Z/2^64 on CUDA cores), the
lookahead block, put / get / fetch, and the argument checks.  Bit-exact."""
import ctypes as C

import numpy as np
import pytest

from hacs_b200 import _lib
from oracle import ring2k_ops

pytestmark = pytest.mark.gpu


def _open(elem, m, cw, panel):
    s = C.c_void_p()
    rc = _lib.lib().hme_r2k_open(0, elem, m, cw, panel, C.byref(s))
    assert rc == 0, _lib.lib().hme_last_error().decode()
    return s


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p)


def _step(s, a, dtype):
    L = _lib.lib()
    swaps = np.ascontiguousarray(np.array(a.get("swaps", []), dtype=np.uint32).reshape(-1))
    st = _lib.HmeR2kStep()
    st.m, st.r, st.np, st.pc0, st.pc1 = a["m"], a["r"], a["np"], a["pc0"], a["pc1"]
    panel = a.get("panel")
    if panel is not None:
        panel = np.ascontiguousarray(panel, dtype=dtype)
        st.panel, st.ldp = _ptr(panel), panel.shape[1]
    st.swaps = swaps.ctypes.data_as(_lib.u32p) if swaps.size else None
    st.nswaps = swaps.size // 2
    Lm = a.get("L")
    if Lm is not None:
        Lm = np.ascontiguousarray(Lm, dtype=dtype)
        st.L, st.ldl = _ptr(Lm), Lm.shape[1]
    st.u0, st.la0, st.la1, st.w = a["u0"], a.get("la0", 0), a.get("la1", 0), a.get("w", 0)
    rc = L.hme_r2k_step(s, C.byref(st))
    return rc


@pytest.mark.parametrize("elem,m,cw,panel", [(4, 300, 520, 64), (4, 777, 1030, 128), (8, 260, 300, 32),
                                             (4, 129, 97, 48)])
def test_session_steps_match_oracle(elem, m, cw, panel):
    dt = np.uint32 if elem == 4 else np.uint64
    rng = np.random.default_rng(m + cw)
    info = np.iinfo(dt)
    W0 = rng.integers(0, info.max, (m, cw), dtype=dt, endpoint=True)
    Wref = W0.copy()
    L = _lib.lib()
    s = _open(elem, m, cw, panel)
    try:
        assert L.hme_r2k_put(s, _ptr(W0), cw, 0, m, 0, cw) == 0
        r = 0
        c = 0
        have_la = None
        while c < cw and r < m:
            c1 = min(c + panel, cw)
            pw = c1 - c
            rows = m - r
            np_ = int(min(pw, rows, rng.integers(0, pw + 1)))
            panel_blk = rng.integers(0, info.max, (rows, pw), dtype=dt, endpoint=True)
            swaps = [(int(r + rng.integers(0, rows)), int(r + rng.integers(0, rows))) for _ in range(np_)]
            Lm = rng.integers(0, info.max, (rows, max(np_, 1)), dtype=dt, endpoint=True)
            nc1 = min(c1 + panel, cw)
            nxt = c1 < cw and r + np_ < m
            a = {"m": m, "r": r, "np": np_, "pc0": c, "pc1": c1, "panel": panel_blk, "swaps": swaps, "L": Lm,
                 "u0": c1 if (np_ > 0 and c1 < cw) else cw, "la0": c1 if nxt else 0, "la1": nc1 if nxt else 0}
            if have_la is not None:
                got = np.zeros_like(have_la)
                assert L.hme_r2k_fetch(s, _ptr(got), got.shape[1]) == 0
                assert np.array_equal(got, have_la), "lookahead block differs"
            assert _step(s, a, dt) == 0, L.hme_last_error().decode()
            la = ring2k_ops.step(Wref, a)
            have_la = la
            r += np_
            c = c1
        got = np.zeros_like(W0)
        assert L.hme_r2k_get(s, _ptr(got), cw, 0, m, 0, cw) == 0
        assert np.array_equal(got, Wref)
        # a block get with a padded host leading dimension
        blk = np.zeros((m // 2, cw // 3 + 5), dtype=dt)
        assert L.hme_r2k_get(s, _ptr(blk), blk.shape[1], 3, m // 2, 7, cw // 3) == 0
        assert np.array_equal(blk[:, : cw // 3], Wref[3:3 + m // 2, 7:7 + cw // 3])
    finally:
        assert L.hme_r2k_close(s) == 0


def test_session_rejects_bad_steps():
    L = _lib.lib()
    s = _open(4, 64, 64, 16)
    try:
        a = {"m": 65, "r": 0, "np": 0, "pc0": 0, "pc1": 16, "u0": 64}
        assert _step(s, a, np.uint32) == _lib.HME_EINVAL  # m differs from the session's
        a = {"m": 64, "r": 60, "np": 8, "pc0": 0, "pc1": 16, "u0": 64}
        assert _step(s, a, np.uint32) == _lib.HME_EINVAL  # pivot rows past the matrix
        a = {"m": 64, "r": 0, "np": 0, "pc0": 0, "pc1": 40, "u0": 64}
        assert _step(s, a, np.uint32) == _lib.HME_EINVAL  # panel wider than the session's
        a = {"m": 64, "r": 0, "np": 1, "pc0": 0, "pc1": 16, "swaps": [(0, 64)], "u0": 64}
        assert _step(s, a, np.uint32) == _lib.HME_EINVAL  # swap row outside the matrix
        blk = np.zeros((8, 8), np.uint32)
        assert L.hme_r2k_get(s, _ptr(blk), 8, 60, 8, 0, 8) == _lib.HME_EINVAL
        assert L.hme_r2k_fetch(s, _ptr(blk), 8) == _lib.HME_EINVAL  # no lookahead asked
    finally:
        assert L.hme_r2k_close(s) == 0


def test_plan_windows():
    L = _lib.lib()
    assert L.hme_r2k_plan(0, 4, 2048, 2048, 128, 0) == 2048  # resident
    base = L.hme_r2k_session_bytes(4, 4096, 0, 128)
    cap = base + 8 * (L.hme_r2k_session_bytes(4, 4096, 1024, 128) - base)  # room for 8192 window columns
    cw = L.hme_r2k_plan(0, 4, 4096, 100000, 128, cap)
    assert cw == 8192
    assert L.hme_r2k_plan(0, 3, 64, 64, 16, 0) == 0  # elem must be 4 or 8
    assert L.hme_r2k_plan(0, 4, 4096, 100000, 128, 1 << 20) == 0  # too little memory: decline
