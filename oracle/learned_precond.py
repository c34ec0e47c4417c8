"""CPU restatement (numpy) of the Davidson preconditioner of dvr3d_b200: the channel blocks of
the contracted Hamiltonian and the learned per-mode correction (network forward and
backward). Test infrastructure only: it checks the device kernels (learned_precond.cu);
nothing in the product imports it.

The reference (ExoMol/dvr3d) has no iterative solver and no learned component; this file
restates the model the product defines (learned_precond.cuh):

    channel c   = the c-th contracted function of every angle block that has more than c
    H_c         = H3[ix_c, ix_c] = Q_c diag(lam_c) Q_c^T
    t[ix_c]     = Q_c diag( g_cq / safe(lam_cq - theta) ) Q_c^T r[ix_c]
    g           = 1 + f(phi),  phi = ((lam - theta)/s, f1, f2, f3)
    f           = w3 . tanh(W2 tanh(W1 phi + b1) + b2) + b3

Parameter layout: W1[16][4] @0, b1[16] @64, W2[16][16] @80, b2[16] @336, w3[16] @352, b3 @368.
"""
from __future__ import annotations

import numpy as np

NFEAT, NHID = 4, 16
NPARAM = NHID * NFEAT + NHID + NHID * NHID + NHID + NHID + 1


def unpack(w):
    w = np.asarray(w, dtype=np.float64)
    o = 0
    W1 = w[o:o + NHID * NFEAT].reshape(NHID, NFEAT); o += NHID * NFEAT
    b1 = w[o:o + NHID]; o += NHID
    W2 = w[o:o + NHID * NHID].reshape(NHID, NHID); o += NHID * NHID
    b2 = w[o:o + NHID]; o += NHID
    w3 = w[o:o + NHID]; o += NHID
    return W1, b1, W2, b2, w3, w[o]


def safe(d):
    eps = 1.0e-4
    d = np.asarray(d, dtype=np.float64)
    return np.where(np.abs(d) < eps, np.where(d < 0.0, -eps, eps), d)


def features(lam, f1, f2, f3, scale, theta):
    """(ncol, nmode, 4) features of every (mode, Ritz value) item."""
    lam = np.asarray(lam)
    th = np.asarray(theta)[:, None]
    b = lambda a: np.broadcast_to(np.asarray(a)[None, :], (th.shape[0], lam.size))
    return np.stack([(lam[None, :] - th) / scale, b(f1), b(f2), b(f3)], axis=-1)


def forward(w, phi):
    W1, b1, W2, b2, w3, b3 = unpack(w)
    z1 = np.tanh(phi @ W1.T + b1)
    z2 = np.tanh(z1 @ W2.T + b2)
    return z2 @ w3 + b3, z1, z2


def eval_network(w, lam, f1, f2, f3, scale, theta, delta):
    """g (nmode x ncol) = 1 + f, and grad = sum over items delta * dg/dw (backpropagation)."""
    W1, b1, W2, b2, w3, b3 = unpack(w)
    phi = features(lam, f1, f2, f3, scale, theta)       # (J, M, 4)
    f, z1, z2 = forward(w, phi)
    dl = np.asarray(delta).T                             # (J, M)
    d2 = dl[..., None] * w3 * (1.0 - z2 ** 2)
    d1 = (d2 @ W2) * (1.0 - z1 ** 2)
    grad = np.concatenate([np.einsum("jma,jmc->ac", d1, phi).ravel(), d1.sum((0, 1)),
                           np.einsum("jma,jmb->ab", d2, z1).ravel(), d2.sum((0, 1)),
                           np.einsum("jm,jma->a", dl, z2), [dl.sum()]])
    return (1.0 + f).T, grad


def channels(iv2):
    """Member lists of the channels for per-block counts iv2 (blocks in solve order)."""
    col0 = np.concatenate([[0], np.cumsum(iv2)[:-1]])
    kmax = int(max(iv2))
    return [np.array([col0[b] + c for b in range(len(iv2)) if iv2[b] > c]) for c in range(kmax)]


def channel_apply(H, chans, theta, R, g=None):
    """Corrections of the residuals R (N x ncol) for Ritz values theta; g: optional list of
    per-channel (n_c x ncol) factors (None: exact channel inverse)."""
    T = np.zeros_like(R)
    for c, ix in enumerate(chans):
        lam, Q = np.linalg.eigh(H[np.ix_(ix, ix)])
        Z = (Q.T @ R[ix]) / safe(lam[:, None] - np.asarray(theta)[None, :])
        if g is not None:
            Z = Z * g[c]
        T[ix] = Q @ Z
    return T
