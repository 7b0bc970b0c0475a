"""The order of operations of gj_invert_gmem (walker_eval.cuh), restated in
Python: Gauss-Jordan inversion with implicit pivot rows (the pivot rule of
izamax/dcabs1, reptation.f:9079, 9219) applied in blocks of pivot steps (a
panel of columns first, then the scaled pivot rows, then every other row
once per block) performs on every element exactly the operations of the
step-by-step inversion, in the same order, so the two give bit-identical
matrices and pivot sequences. Host-only: complex numbers as (re, im) pairs
with the device's formulas for products and updates."""
import numpy as np
import pytest


def _cmul(a, b):
    return (a[0] * b[0] - a[1] * b[1], a[0] * b[1] + a[1] * b[0])


def _sub(v, f, a):  # v -= f * a, as the device forms it
    return (v[0] - (f[0] * a[0] - f[1] * a[1]), v[1] - (f[0] * a[1] + f[1] * a[0]))


def _pivot(col, used, n, k):
    best, bi = -1.0, n
    for r in range(n):
        if not used[r]:
            a = abs(col[r][0]) + abs(col[r][1])
            if a > best:
                best, bi = a, r
    return bi if bi < n else k


def _inv(piv):
    d = piv[0] * piv[0] + piv[1] * piv[1]
    rd = 1.0 / d
    return (piv[0] * rd, -piv[1] * rd)


def step_by_step(W, n):
    W = [row[:] for row in W]
    used, perm = [0] * n, []
    for k in range(n):
        p = _pivot([W[r][k] for r in range(n)], used, n, k)
        inv = _inv(W[p][k])
        f = [W[r][k] for r in range(n)]
        used[p] = 1
        perm.append(p)
        W[p] = [inv if c == k else _cmul(W[p][c], inv) for c in range(n)]
        for r in range(n):
            if r == p:
                continue
            for c in range(n):
                if c == k:
                    t = _cmul(f[r], inv)
                    W[r][c] = (-t[0], -t[1])
                else:
                    W[r][c] = _sub(W[r][c], f[r], W[p][c])
    return W, perm


def blocked(W, n, B):
    W = [row[:] for row in W]
    used, perm = [0] * n, []
    for k0 in range(0, n, B):
        nb = min(B, n - k0)
        P = [[W[r][k0 + j] for j in range(nb)] for r in range(n)]  # panel
        F, pj, invj = [], [], []
        for j in range(nb):
            p = _pivot([P[r][j] for r in range(n)], used, n, k0 + j)
            inv = _inv(P[p][j])
            pj.append(p)
            invj.append(inv)
            F.append([P[r][j] for r in range(n)])  # multipliers of step j
            used[p] = 1
            perm.append(p)
            P[p] = [inv if jj == j else _cmul(P[p][jj], inv) for jj in range(nb)]
            for r in range(n):
                if r == p:
                    continue
                for jj in range(nb):
                    if jj == j:
                        t = _cmul(F[j][r], inv)
                        P[r][jj] = (-t[0], -t[1])
                    else:
                        P[r][jj] = _sub(P[r][jj], F[j][r], P[p][jj])
        for r in range(n):
            for j in range(nb):
                W[r][k0 + j] = P[r][j]
        outside = [c for c in range(n) if not k0 <= c < k0 + nb]
        Q = [dict() for _ in range(nb)]  # scaled pivot rows outside the panel
        for c in outside:
            for j in range(nb):
                x = W[pj[j]][c]
                for jj in range(j):
                    x = _sub(x, F[jj][pj[j]], Q[jj][c])
                Q[j][c] = _cmul(x, invj[j])
        for r in range(n):
            role = pj.index(r) if r in pj else -1
            for c in outside:
                v = Q[role][c] if role >= 0 else W[r][c]
                for j in range(role + 1, nb):
                    v = _sub(v, F[j][r], Q[j][c])
                W[r][c] = v
    return W, perm


@pytest.mark.parametrize("B", [4, 8])
@pytest.mark.parametrize("n", [1, 3, 8, 9, 17, 23])
def test_blocked_inversion_is_bit_identical(n, B):
    rng = np.random.default_rng(7 * n + B)
    A = rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))
    W = [[(float(A[r, c].real), float(A[r, c].imag)) for c in range(n)] for r in range(n)]
    a, pa = step_by_step(W, n)
    b, pb = blocked(W, n, B)
    assert pa == pb
    assert all(a[r][c] == b[r][c] for r in range(n) for c in range(n))
    # and it is the inverse: A^-1(k, pi(c)) = W(pi(k), c)
    inv = np.empty((n, n), complex)
    for k in range(n):
        for c in range(n):
            inv[k, pa[c]] = complex(*a[pa[k]][c])
    assert np.allclose(inv @ A, np.eye(n), atol=1e-9)


def test_ties_and_a_zero_column_follow_the_pivot_rule():
    # equal |re|+|im| in a column: the lowest unused row is the pivot
    n = 4
    W = [[(1.0, 0.0) if r == c or (c == 0) else (0.0, 0.0) for c in range(n)] for r in range(n)]
    a, pa = step_by_step(W, n)
    b, pb = blocked(W, n, 4)
    assert pa == pb and pa[0] == 0
    assert all(a[r][c] == b[r][c] for r in range(n) for c in range(n))
