"""ORACLE / TEST INFRASTRUCTURE ONLY.

numpy restatement of one step of the Z/2^W device LU's operations table
(engine::ring2k::device::Ops::step with StepArgs, reference
src/ModArithmetic/Binary/Ring2kDevice.h:49-62; what a step must do to the
device window is fixed by its host driver, Ring2kDeviceLU.h:116-300, and by
the host LU it replays, ring2k::echelon_blocked, Ring2k.h:539-695):

  * the factored panel (rows r .. m-1, columns [pc0, pc1)) overwrites the window;
  * the swap pairs, in order, exchange rows on every other column of [0, w);
  * the unit-lower solve on the pivot rows, columns [u0, w): row r+t -=
    sum_{t2 < t} L[t][t2] row r+t2 (Ring2k.h:673-677);
  * C -= L21 U12 on rows r+np .. m-1, columns [u0, w) (Ring2k.h:679-680);
  * the lookahead block: rows r+np .. m-1 of columns [la0, la1) after that.

All arithmetic is native wraparound in W bits (numpy's unsigned integer ops
wrap silently), as the reference's Tr::axpy / Tr::gemm_sub.
"""
from __future__ import annotations

import numpy as np


def step(W: np.ndarray, a: dict) -> np.ndarray | None:
    """Apply one step to the window W (m x cw, uint32 or uint64) in place;
    returns the lookahead block (or None when la0 == la1)."""
    dt = W.dtype.type
    m = W.shape[0]
    w = a.get("w", 0) or W.shape[1]
    r, np_, pc0, pc1 = a["r"], a["np"], a["pc0"], a["pc1"]
    if a.get("panel") is not None and pc1 > pc0:
        W[r:m, pc0:pc1] = a["panel"]
    cols = np.r_[0:pc0, pc1:w]
    for x, y in a.get("swaps", []):
        tmp = W[x, cols].copy()
        W[x, cols] = W[y, cols]
        W[y, cols] = tmp
    u0 = a["u0"]
    if np_ > 0 and u0 < w:
        L = a["L"]  # rows r .. m-1 (row 0 = matrix row r), columns 0 .. np-1
        with np.errstate(over="ignore"):
            for t in range(1, np_):
                acc = W[r + t, u0:w].copy()
                for t2 in range(t):
                    acc = acc - dt(L[t, t2]) * W[r + t2, u0:w]
                W[r + t, u0:w] = acc
            if r + np_ < m:
                L21 = L[np_:m - r, :np_].astype(W.dtype)
                U12 = W[r:r + np_, u0:w]
                prod = np.zeros((m - r - np_, w - u0), dtype=W.dtype)
                for t in range(np_):
                    prod = prod + L21[:, t:t + 1] * U12[t:t + 1, :]
                W[r + np_:m, u0:w] = W[r + np_:m, u0:w] - prod
    la0, la1 = a.get("la0", 0), a.get("la1", 0)
    if la1 > la0:
        return W[r + np_:m, la0:la1].copy()
    return None
