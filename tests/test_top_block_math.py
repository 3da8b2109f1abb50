"""The algebra of the elimination's top-block path, checked on the CPU against
the oracle (no GPU).

When the top w x w block B of a panel factors as B = L U with non-zero
diagonal entries, the device replaces the panel step (pivot search, row moves,
U12 = L^-1 A12, A22 -= L21 U12) by one product
    [A12; A22] += [L^-1 - I; -A21 B^-1] A12,
and keeps the packed L\\U in the block.  Here that step is done in exact
integer arithmetic mod p: the top rows must become U12 = L^-1 A12, the rows
below the Schur complement, the panel columns below the block the multipliers'
span (they are dropped), and the RREF of the stepped matrix [U U12; 0 S] must
equal the oracle's RREF of the input (row operations keep the row space).  And
the reference's pivot rule (topmost non-zero in the leftmost column of the
Schur complement) picks rows 0 .. w-1 exactly when those diagonals are non-zero.
"""
import numpy as np

import oracle as O


def _inv(x, p):
    return pow(int(x), p - 2, p)


def _lu_no_pivot(B, p):
    """Doolittle LU of B mod p without row exchanges; None on a zero pivot."""
    w = B.shape[0]
    U = [[int(v) for v in row] for row in B]
    L = [[int(i == j) for j in range(w)] for i in range(w)]
    for t in range(w):
        if U[t][t] % p == 0:
            return None
        it = _inv(U[t][t], p)
        for r in range(t + 1, w):
            f = U[r][t] * it % p
            L[r][t] = f
            for j in range(t, w):
                U[r][j] = (U[r][j] - f * U[t][j]) % p
    return np.array(L, dtype=object), np.array(U, dtype=object)


def _tri_inv_lower_unit(L, p):
    w = L.shape[0]
    X = np.zeros((w, w), dtype=object)
    for c in range(w):
        for r in range(w):
            s = 1 if r == c else 0
            for t in range(r):
                s -= L[r][t] * X[t][c]
            X[r][c] = s % p
    return X


def _inv_matrix(M, p):
    """M^-1 mod p by Gauss-Jordan (M invertible)."""
    w = M.shape[0]
    A = [[int(M[i][j]) % p for j in range(w)] + [int(i == j) for j in range(w)] for i in range(w)]
    for c in range(w):
        r = next(i for i in range(c, w) if A[i][c] % p)
        A[c], A[r] = A[r], A[c]
        ic = _inv(A[c][c], p)
        A[c] = [v * ic % p for v in A[c]]
        for i in range(w):
            if i != c and A[i][c]:
                f = A[i][c]
                A[i] = [(a - f * b) % p for a, b in zip(A[i], A[c])]
    return np.array([row[w:] for row in A], dtype=object)


def _mm(X, Y, p):
    return np.array((X.astype(object) @ Y.astype(object)) % p, dtype=object)


def _top_rows_pivot_by_reference_rule(A, w, p):
    """Row indices the reference's rule picks for the first w columns (topmost
    non-zero of the Schur complement, column by column), by plain elimination."""
    M = [[int(v) for v in row] for row in A]
    active = list(range(len(M)))
    rows = []
    for c in range(w):
        piv = next((r for r in active if M[r][c] % p), None)
        if piv is None:
            continue
        rows.append(piv)
        active.remove(piv)
        ip = _inv(M[piv][c], p)
        for r in active:
            f = M[r][c] * ip % p
            M[r] = [(a - f * b) % p for a, b in zip(M[r], M[piv])]
    return rows


def test_fused_update_keeps_the_row_space():
    p = 65521
    rng = np.random.default_rng(2024)
    for (m, n, w) in [(20, 16, 8), (33, 40, 8), (12, 30, 12)]:
        A = rng.integers(0, p, (m, n), dtype=np.uint64).astype(np.uint32)
        lu = _lu_no_pivot(A[:w, :w], p)
        assert lu is not None
        L, U = lu
        assert _top_rows_pivot_by_reference_rule(A, w, p) == list(range(w))
        A12 = A[:w, w:].astype(object)
        A21 = A[w:, :w].astype(object)
        A22 = A[w:, w:].astype(object)
        Linv = _tri_inv_lower_unit(L, p)
        Binv = _inv_matrix(A[:w, :w].astype(object), p)
        W_top = (Linv - np.eye(w, dtype=object)) % p
        W_bot = (-_mm(A21, Binv, p)) % p
        top = (A12 + _mm(W_top, A12, p)) % p
        bot = (A22 + _mm(W_bot, A12, p)) % p
        # the top rows are U12 = L^-1 A12, the rows below the Schur complement A22 - L21 U12
        U12 = _mm(Linv, A12, p)
        assert np.array_equal(top, U12)
        L21 = _mm(A21, _inv_matrix(U, p), p)
        assert np.array_equal(bot, (A22 - _mm(L21, U12, p)) % p)
        # the stepped matrix [U U12; 0 S] has the input's RREF
        stepped = np.zeros((m, n), dtype=np.uint32)
        stepped[:w, :w] = U.astype(np.uint64).astype(np.uint32)
        stepped[:w, w:] = top.astype(np.uint64).astype(np.uint32)
        stepped[w:, w:] = bot.astype(np.uint64).astype(np.uint32)
        R1, p1 = O.rref(p, A)
        R2, p2 = O.rref(p, stepped)
        assert np.array_equal(R1, R2) and np.array_equal(p1, p2)


def test_zero_diagonal_means_another_pivot_row():
    """A zero on the block's diagonal after the first t steps: the reference's rule
    then picks a row outside 0 .. w-1 (or none), which is why the device falls back
    to the search exactly then."""
    p = 65521
    rng = np.random.default_rng(7)
    A = rng.integers(0, p, (24, 20), dtype=np.uint64).astype(np.uint32)
    A[3] = A[1]  # row 3 equals row 1: step 3 meets a zero pivot in the top block
    assert _lu_no_pivot(A[:8, :8], p) is None
    rows = _top_rows_pivot_by_reference_rule(A, 8, p)
    assert rows != list(range(8)) and 3 not in rows
