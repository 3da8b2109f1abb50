"""The algebra of the batched rank rounds, checked on the CPU against classical
elimination and the oracle (no GPU).

Each round of the batched rank (one CTA per job) factors a panel of the job's
active rows fraction-free: at the step of pivot t (value w_t) every other
active row becomes (w_t row - x pivot_row) rho, rho = 2^-32 mod p for odd
p < 2^31 (one Montgomery reduction per element) or 1, so no column needs an
inverse; the multiplier positions keep the scaled x.  Once per panel the
classical values come back: a multiplier is divided by its pivot w_t, every
other entry by the product of (w_u rho) over the steps u that updated it.
Then the pivot rows move to the top of the active rows by swaps (at most 2k
rows move), U12 = L11^-1 A12, and A22 -= L21 U12 on the trailing columns.

Here those steps are restated in exact integer arithmetic: the panel after the
fix-up must equal classical elimination with the same pivot rule (topmost
active row with a non-zero in the current column, pivot rows in place,
multipliers in the pivot columns), the swap lists must put pivot t at row
r0 + t and move every other row to a free position, and the rank after all
rounds must equal the oracle's under every schedule the device offers: the
panel width of the rounds and the widest last panel.
"""
import numpy as np
import pytest

import oracle as O


def _inv(x, p):
    return pow(int(x) % p, p - 2, p)


def _classical_panel(P, p):
    """Classical elimination of the panel P (rows x w lists of ints): returns the
    packed panel, the pivot rows and the pivot columns."""
    rows, w = len(P), len(P[0]) if P else 0
    S = [[v % p for v in r] for r in P]
    active = [True] * rows
    prow, pcol = [], []
    for it in range(w):
        piv = next((r for r in range(rows) if active[r] and S[r][it] % p), None)
        if piv is None:
            continue
        iw = _inv(S[piv][it], p)
        for r in range(rows):
            if r == piv or not active[r]:
                continue
            m = S[r][it] * iw % p
            S[r][it] = m
            for j in range(it + 1, w):
                S[r][j] = (S[r][j] - m * S[piv][j]) % p
        active[piv] = False
        prow.append(piv)
        pcol.append(it)
    return S, prow, pcol


def _fraction_free_panel(P, p):
    """The device panel: fraction-free updates with the scale rho, then the
    one-pass fix-up (multipliers times w_t^-1, every other entry times the
    inverse of the scale in force when its row left the active set or its
    column was passed)."""
    rows, w = len(P), len(P[0]) if P else 0
    mont = (p & 1) == 1 and p < (1 << 31)
    rho = _inv(1 << 32, p) if mont else 1
    S = [[v % p for v in r] for r in P]
    step = [0] * rows  # 0 active, t + 1 once the row is pivot t
    colstep = [0] * w
    wts, prow, pcol = [], [], []
    k = 0
    for it in range(w):
        piv = next((r for r in range(rows) if step[r] == 0 and S[r][it] % p), None)
        if piv is None:
            colstep[it] = -1 - k
            continue
        wt = S[piv][it]
        wts.append(wt)
        colstep[it] = k
        prow.append(piv)
        pcol.append(it)
        step[piv] = k + 1
        for r in range(rows):
            if r == piv or step[r]:
                continue
            xn = (p - S[r][it]) % p
            for j in range(it + 1, w):
                S[r][j] = (wt * S[r][j] + xn * S[piv][j]) * rho % p
        k += 1
    inv_w = [_inv(x, p) for x in wts]
    rinv = (1 << 32) % p if mont else 1 % p
    sinv = [1 % p]  # exclusive prefix products of f_t = w_t^-1 rho^-1
    for t in range(k):
        sinv.append(sinv[-1] * inv_w[t] * rinv % p)
    for r in range(rows):
        tau = step[r] - 1 if step[r] else k
        sc = sinv[tau]
        for j in range(w):
            t = colstep[j]
            f = (inv_w[t] if t < tau else sc) if t >= 0 else sinv[min(tau, -1 - t)]
            S[r][j] = S[r][j] * f % p
    return S, prow, pcol


@pytest.mark.parametrize("p", [65521, 2147483629, 251, 4294967291, 3])
def test_fraction_free_panel_equals_classical(p):
    rng = np.random.default_rng(p % 1009)
    for trial in range(12):
        rows, w = int(rng.integers(1, 24)), int(rng.integers(1, 10))
        r = int(rng.integers(1, min(rows, w) + 1))
        # planted rank r, and a zero column or a run of zero leading entries now and then
        P = (rng.integers(0, p, (rows, r), dtype=np.uint64).astype(object) @
             rng.integers(0, p, (r, w), dtype=np.uint64).astype(object)) % p
        if trial % 3 == 0:
            P[:, int(rng.integers(0, w))] = 0
        if trial % 4 == 1:
            P[: rows // 2, 0] = 0
        P = [[int(v) for v in row] for row in P]
        got, gr, gc = _fraction_free_panel(P, p)
        want, wr, wc = _classical_panel(P, p)
        assert (gr, gc) == (wr, wc)
        assert got == want, (p, trial)


def _swap_moves(pivot_rows, r0, k):
    """The device's row moves (rank_post_kernel): (sources, destinations) so
    that position r0 + t receives pivot row t; every moved row goes to a free
    position, at most 2k rows move."""
    pos, cont = [], []

    def find(x):
        for i, v in enumerate(pos):
            if v == x:
                return i
        pos.append(x)
        cont.append(x)
        return len(pos) - 1

    for t in range(k):
        a = find(t)
        orig = pivot_rows[t] - r0
        b = next((i for i, v in enumerate(cont) if v == orig), -1)
        if b < 0:
            b = find(orig)
        if a != b:
            cont[a], cont[b] = cont[b], cont[a]
    moves = [(r0 + c, r0 + q) for q, c in zip(pos, cont) if c != q]
    assert len(moves) <= 2 * k
    return moves


def test_swap_moves_place_pivots_and_permute():
    rng = np.random.default_rng(5)
    for _ in range(300):
        rows = int(rng.integers(1, 40))
        k = int(rng.integers(0, min(rows, 12) + 1))
        r0 = int(rng.integers(0, 5))
        pivots = [r0 + int(x) for x in rng.permutation(rows)[:k]]
        moves = _swap_moves(pivots, r0, k)
        old = list(range(r0, r0 + rows))
        new = list(old)
        for src, dst in moves:  # all rows read (into the scratch) before any is written
            new[dst - r0] = old[src - r0]
        assert sorted(new) == old  # a permutation of the active rows
        assert new[:k] == pivots  # pivot t at row r0 + t


def _batched_rank(A, p, bw, last_max):
    """The rounds of one job: panels of bw columns (the last one up to last_max
    when the remaining columns fit it), fraction-free panel, swaps, U12 solve,
    trailing update; returns the rank."""
    A = [[int(v) % p for v in row] for row in A]
    m, n = len(A), len(A[0])
    r0 = c0 = 0
    while r0 < m and c0 < n:
        left = n - c0
        w = left if left <= last_max else min(bw, left)
        c1 = c0 + w
        panel = [row[c0:c1] for row in A[r0:]]
        S, prow, pcol = _fraction_free_panel(panel, p)
        for i in range(m - r0):
            A[r0 + i][c0:c1] = S[i]
        k = len(prow)
        below, ntrail = m - r0 - k, n - c1
        if k and ntrail and below:
            moves = _swap_moves([r0 + x for x in prow], r0, k)
            tmp = [list(A[src][c0:]) for src, _ in moves]
            for (_, dst), row in zip(moves, tmp):
                A[dst][c0:] = row
            pc = [c0 + x for x in pcol]
            # U12 = L11^-1 A12, L11 unit lower from the pivot rows' multipliers
            for t in range(k):
                for s in range(t):
                    l = A[r0 + t][pc[s]]
                    if l:
                        for j in range(c1, n):
                            A[r0 + t][j] = (A[r0 + t][j] - l * A[r0 + s][j]) % p
            # A22 -= L21 U12
            for i in range(r0 + k, m):
                for t in range(k):
                    l = A[i][pc[t]]
                    if l:
                        for j in range(c1, n):
                            A[i][j] = (A[i][j] - l * A[r0 + t][j]) % p
        r0 += k
        c0 = c1
    return r0


@pytest.mark.parametrize("bw,last_max", [(4, 16), (4, 4), (8, 8), (3, 40)])
def test_rank_rounds_under_every_schedule_equal_oracle(bw, last_max):
    rng = np.random.default_rng(bw * 100 + last_max)
    for p in (65521, 2147483629, 251):
        for _ in range(6):
            m, n = int(rng.integers(1, 30)), int(rng.integers(1, 30))
            r = int(rng.integers(0, min(m, n) + 1))
            L = rng.integers(0, p, (m, max(r, 1)), dtype=np.uint64).astype(np.uint32)
            R = rng.integers(0, p, (max(r, 1), n), dtype=np.uint64).astype(np.uint32)
            A = O.gemm(p, L, R) if r else np.zeros((m, n), np.uint32)
            want = len(O.rref(p, A)[1])
            assert _batched_rank(A, p, bw, last_max) == want, (p, m, n, r)


def _barrett(x, p):
    """reduce_u64: x - floor(x * floor(2^64 / p) / 2^64) * p, one correction."""
    m = (1 << 64) // p
    r = x - ((x * m) >> 64) * p
    assert 0 <= r < 2 * p
    return r - p if r >= p else r


@pytest.mark.parametrize("p", [251, 65521, 16777213, 759250125, 759250133, 2147483629, 4294967291])
def test_cuda_core_update_sums(p):
    """The CUDA-core update's exact dot products of k <= 32 products: a 64-bit
    sum when 32 (p - 1)^2 fits 64 bits, else a 96-bit sum (a0, a1, a2 words)
    reduced as ((a2 2^32 + a1) mod p) 2^32 + a0 mod p; both equal the exact
    sum mod p, worst case (p - 1)^2 included."""
    rng = np.random.default_rng(p % 997)
    narrow = (p - 1) * (p - 1) <= ((1 << 64) - 1) // 32
    assert narrow == (p <= 759250125)
    for trial in range(200):
        k = int(rng.integers(1, 33))
        if trial < 2:
            x = [p - 1] * k
            y = [p - 1] * k
        else:
            x = [int(v) for v in rng.integers(0, p, k, dtype=np.uint64)]
            y = [int(v) for v in rng.integers(0, p, k, dtype=np.uint64)]
        exact = sum(a * b for a, b in zip(x, y))
        if narrow:
            acc = 0
            for a, b in zip(x, y):
                acc = (acc + a * b) & ((1 << 64) - 1)
            assert acc == exact  # no wraparound
            d = _barrett(acc, p)
        else:
            a0 = a1 = a2 = 0
            for a, b in zip(x, y):  # mad.lo.cc / madc.hi.cc / addc
                prod = a * b
                s0 = a0 + (prod & 0xFFFFFFFF)
                a0, c0 = s0 & 0xFFFFFFFF, s0 >> 32
                s1 = a1 + (prod >> 32) + c0
                a1, c1 = s1 & 0xFFFFFFFF, s1 >> 32
                a2 = (a2 + c1) & 0xFFFFFFFF
            assert (a2 << 64) | (a1 << 32) | a0 == exact
            h = _barrett((a2 << 32) | a1, p)
            d = _barrett((h << 32) | a0, p)
        assert d == exact % p
