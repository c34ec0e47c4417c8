"""Host-side model of the band eigensolver of the shift-invert path (csrc/band_eig.cu).

Two things the device kernel relies on are checked here on the CPU:
* the task sequence of the bulge chase (sweep j, task s: reflector from column j or from the
  bulge's first column, O_s <- H O_s, D_s <- H D_s H, O_{s+1} <- O_{s+1} H, only these blocks
  touched) reduces a symmetric band matrix to tridiagonal form with the same eigenvalues, and
  the reflectors applied last-first back-transform the tridiagonal eigenvectors;
* the hand-off rule between sweeps: sweep j+1 may run task s' once sweep j has written the beta
  of its task s'+2 (the last task of a sweep is handed off only when complete), and a CTA loads
  task s+1's blocks while its task s runs, once sweep j-1 has handed off task s+4. Every pair of
  tasks (and loads) that the rule lets run at the same time touches disjoint matrix elements.
"""
import numpy as np
import pytest


def _house(x):
    a = x[0]
    sig = float(np.dot(x[1:], x[1:]))
    v = np.zeros_like(x)
    v[0] = 1.0
    if sig == 0.0:
        return v, 0.0, a
    beta = -np.copysign(np.sqrt(a * a + sig), a)
    v[1:] = x[1:] / (a - beta)
    return v, (beta - a) / beta, beta


def _ntask(n, b, j):
    return (n - 2 - j) // b + 1


def _chase(M, b):
    """Bulge chasing of the lower triangle of M (band of half-width b), task by task."""
    n = M.shape[0]
    A = np.tril(M).copy()
    refl = []
    for j in range(n - 2):
        O = None
        for s in range(_ntask(n, b, j)):
            r0 = j + 1 + s * b
            L = min(b, n - r0)
            x = A[r0:r0 + L, j].copy() if s == 0 else O[:, 0].copy()
            v, tau, beta = _house(x)
            refl.append((j, s, v, tau))
            if s == 0:
                A[r0:r0 + L, j] = 0.0
                A[r0, j] = beta
            else:
                O[:, 0] = 0.0
                O[0, 0] = beta
                if tau != 0.0:
                    O[:, 1:] -= tau * np.outer(v, v @ O[:, 1:])
                A[r0:r0 + L, r0 - b:r0] = O
            D = np.tril(A[r0:r0 + L, r0:r0 + L])
            D = D + D.T - np.diag(np.diag(D))
            if tau != 0.0:
                y = D @ v
                w = tau * y - 0.5 * tau * tau * (v @ y) * v
                D -= np.outer(v, w) + np.outer(w, v)
            A[r0:r0 + L, r0:r0 + L] = np.tril(D)
            r1 = r0 + b
            if r1 < n:
                O = A[r1:r1 + min(b, n - r1), r0:r0 + b].copy()
                if tau != 0.0:
                    O -= tau * np.outer(O @ v, v)
    return A, refl


@pytest.mark.parametrize("n,b", [(40, 4), (67, 8), (130, 32), (33, 32), (90, 7)])
def test_bulge_chase_reduces_band_to_tridiagonal(n, b):
    rng = np.random.default_rng(n * 100 + b)
    M = rng.standard_normal((n, n))
    M = M + M.T
    M[np.abs(np.subtract.outer(np.arange(n), np.arange(n))) > b] = 0.0
    A, refl = _chase(M, b)
    assert np.abs(np.tril(A, -2)).max() == 0.0
    d, e = np.diag(A), np.diag(A, -1)
    T = np.diag(d) + np.diag(e, -1) + np.diag(e, 1)
    lam, Z = np.linalg.eigh(T)
    assert np.abs(lam - np.linalg.eigvalsh(M)).max() < 1e-12 * max(1.0, np.abs(lam).max())
    X = Z.copy()
    for j, s, v, tau in reversed(refl):
        r0 = j + 1 + s * b
        X[r0:r0 + len(v)] -= tau * np.outer(v, v @ X[r0:r0 + len(v)])
    assert np.abs(M @ X - X * lam).max() < 1e-12 * max(1.0, np.abs(lam).max())


def _rows(n, b, j, s):
    r0 = j + 1 + s * b
    return range(r0, min(r0 + b, n)) if r0 < n else range(0)


def _touched(n, b, j, s):
    """Lower-triangle elements task (j, s) reads or writes (O_s, D_s and the O_{s+1} it keeps)."""
    E = set()
    Rs, Rp = _rows(n, b, j, s), _rows(n, b, j, s + 1)
    if s == 0:
        E.update((r, j) for r in Rs)
    else:
        E.update((r, c) for r in Rs for c in _rows(n, b, j, s - 1))
    E.update((r, c) for r in Rs for c in Rs if r >= c)
    E.update((r, c) for r in Rp for c in Rs)
    return E


def _beta(j, s, b):
    return (j + 1, j) if s == 0 else (j + 1 + s * b, j + 1 + (s - 1) * b)


def _loads(n, b, j, s):
    """Blocks a CTA loads for task s: D_s, the raw O_{s+1} and, for task 0, column j."""
    P = {(r, c) for r in _rows(n, b, j, s) for c in _rows(n, b, j, s) if r >= c}
    P |= {(r, c) for r in _rows(n, b, j, s + 1) for c in _rows(n, b, j, s)}
    if s == 0:
        P |= {(r, j) for r in _rows(n, b, j, 0)}
    return P


@pytest.mark.parametrize("n,b", [(60, 4), (70, 8), (100, 32), (45, 3), (90, 6)])
def test_handoff_rule_keeps_concurrent_tasks_disjoint(n, b):
    T = {(j, s): _touched(n, b, j, s) for j in range(n - 2) for s in range(_ntask(n, b, j))}
    bad = []
    for j in range(n - 2):
        last = _ntask(n, b, j) - 1
        for d in (1, 2, 3):
            if j + d >= n - 2:
                break
            for s2 in range(_ntask(n, b, j + d)):
                # while sweep j+d runs task s2, sweep j has handed off at least task s2 + 2 d
                # (its beta written, the tasks before it complete); a last task is handed off
                # complete
                p = s2 + 2 * d
                if p >= last:
                    continue
                for s in range(p, last + 1):
                    E = T[(j, s)] - {_beta(j, s, b)} if s == p else T[(j, s)]
                    if E & T[(j + d, s2)]:
                        bad.append(((j, s), (j + d, s2)))
    assert not bad, bad[:5]


@pytest.mark.parametrize("n,b", [(60, 4), (70, 8), (100, 32), (45, 3)])
def test_prefetch_rule_keeps_loads_disjoint(n, b):
    T = {(j, s): _touched(n, b, j, s) for j in range(n - 2) for s in range(_ntask(n, b, j))}
    bad = []
    for j in range(1, n - 2):
        ntp = _ntask(n, b, j - 1)
        for s in range(_ntask(n, b, j)):
            P = _loads(n, b, j, s)
            # while the CTA still runs its own task s-1
            if s > 0 and P & T[(j, s - 1)]:
                bad.append(("own", j, s))
            need = min(s + 3, ntp)  # predecessor tasks handed off before the loads
            if need < ntp:
                q = need - 1
                if P & (T[(j - 1, q)] - {_beta(j - 1, q, b)}):
                    bad.append(("pred-rest", j, s))
                for q2 in range(need, ntp):
                    if P & T[(j - 1, q2)]:
                        bad.append(("pred", j, s, q2))
            if j + 1 < n - 2:  # the successor runs tasks <= s - 2 at most
                for s2 in range(0, min(s - 1, _ntask(n, b, j + 1))):
                    if P & T[(j + 1, s2)]:
                        bad.append(("succ", j, s, s2))
    assert not bad, bad[:5]
