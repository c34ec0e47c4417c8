"""Davidson preconditioner and its learned correction: the CPU oracle of the network (pinned
by finite differences), the device forward/backward kernels against it, the training
gradient against finite differences of the training loss on the device, and what the trained
correction gains over the exact channel-block preconditioner on surfaces it was not trained on."""
from __future__ import annotations

import numpy as np
import pytest

import dvr3d_b200
from dvr3d_b200 import AUTOCM, configs, parse_deck
from oracle import learned_precond as lpo


def _network_case(seed=3, nmode=300, ncol=7):
    rng = np.random.default_rng(seed)
    lam = rng.uniform(0.0, 1.5, nmode)
    f1 = rng.uniform(-2, 2, nmode)
    f2 = rng.uniform(0, 1, nmode)
    f3 = rng.uniform(0, 1, nmode)
    theta = rng.uniform(0.0, 0.2, ncol)
    delta = rng.standard_normal((nmode, ncol))
    w = rng.standard_normal(lpo.NPARAM) * 0.4
    return w, lam, f1, f2, f3, 0.3, theta, delta


def test_oracle_network_gradient_matches_finite_differences():
    w, *args = _network_case(nmode=30, ncol=3)
    delta = args[-1]
    _, g = lpo.eval_network(w, *args)
    obj = lambda v: float(np.sum(delta * lpo.eval_network(v, *args)[0]))
    rng = np.random.default_rng(0)
    for p in list(rng.choice(lpo.NPARAM, 40, replace=False)) + [lpo.NPARAM - 1]:
        d = np.zeros_like(w)
        d[p] = 1e-6
        fd = (obj(w + d) - obj(w - d)) / 2e-6
        assert abs(fd - g[p]) <= 1e-6 * max(1.0, abs(g[p])), (p, fd, g[p])


def test_untrained_output_layer_gives_the_exact_channel_inverse():
    w, *args = _network_case()
    w[-(lpo.NHID + 1):] = 0.0
    g, _ = lpo.eval_network(w, *args)
    np.testing.assert_array_equal(g, 1.0)


def test_channel_preconditioner_solves_the_channel_blocks():
    rng = np.random.default_rng(5)
    iv2 = [5, 7, 6, 3, 7]
    n = sum(iv2)
    X = rng.standard_normal((n, n))
    H = X @ X.T / n + np.diag(rng.uniform(1, 2, n))
    chans = lpo.channels(iv2)
    assert sorted(np.concatenate(chans)) == list(range(n))
    theta = np.array([0.1, 0.3])
    R = rng.standard_normal((n, 2))
    T = lpo.channel_apply(H, chans, theta, R)
    for ix in chans:
        for j in range(2):
            np.testing.assert_allclose((H[np.ix_(ix, ix)] - theta[j] * np.eye(len(ix))) @ T[ix, j], R[ix, j],
                                       rtol=0, atol=1e-11)


@pytest.mark.gpu
def test_device_network_matches_oracle(ctx):
    w, *args = _network_case()
    g_ref, grad_ref = lpo.eval_network(w, *args)
    g, grad = ctx.lp_eval(w, *args)
    np.testing.assert_allclose(g, g_ref, rtol=0, atol=1e-13)
    np.testing.assert_allclose(grad, grad_ref, rtol=1e-10, atol=1e-12 * np.abs(grad_ref).max())


@pytest.mark.gpu
def test_weights_round_trip_and_validation(ctx):
    w = _network_case()[0]
    ctx.lp_set_weights(w)
    np.testing.assert_array_equal(ctx.lp_get_weights(), w)
    with pytest.raises(dvr3d_b200.DVR3DError):
        ctx.lp_set_weights(w[:10])


def _solve(ctx, wl, lp):
    ctx.set_pes(wl.pes)
    return ctx.solve(parse_deck(wl.deck), 0, precision=dvr3d_b200.DVR3D_PREC_MIXED_DAVIDSON, learned_precond=lp,
                     want_resid=True)


def _surface(seed, levels=20):
    return configs.jacobi_h3p_like(14, 14, 24, 45000.0, 40000.0, levels, seed=seed, title=f"lp {seed}")


@pytest.mark.gpu
def test_training_gradient_matches_finite_differences(ctx):
    t = _solve(ctx, _surface(11), 2)
    assert t.extra["path"] == dvr3d_b200.DVR3D_PATH_DAVIDSON and t.extra["lp_pairs"] > 0
    w = ctx.lp_get_weights()
    loss, g = ctx.lp_train_loss(w)
    assert abs(loss - t.extra["lp_loss_last"]) <= 1e-12
    rng = np.random.default_rng(1)
    for p in rng.choice(dvr3d_b200.DVR3D_LP_NPARAM, 12, replace=False):
        h = 1e-5
        d = np.zeros_like(w)
        d[p] = h
        fd = (ctx.lp_train_loss(w + d, False)[0] - ctx.lp_train_loss(w - d, False)[0]) / (2 * h)
        assert abs(fd - g[p]) <= 1e-6 * max(1e-3, abs(g[p])), (p, fd, g[p])


@pytest.mark.gpu
def test_trained_correction_gains_on_unseen_surfaces(ctx):
    """Train on one seeded surface (pairs recorded by the solver itself), then solve two
    other surfaces with the exact channel preconditioner and with the trained correction:
    the same levels (within 1e-3 cm-1 of the dense FP64 solve), fewer H3 products."""
    t = _solve(ctx, _surface(11), 2)
    assert t.extra["lp_loss_last"] < t.extra["lp_loss_first"]
    base = learned = 0
    for seed in (12, 13):
        wl = _surface(seed)
        plain = _solve(ctx, wl, 0)
        lrn = _solve(ctx, wl, 1)
        ctx.set_pes(wl.pes)
        dense = ctx.solve(parse_deck(wl.deck), 0)
        for r in (plain, lrn):
            assert r.extra["path"] == dvr3d_b200.DVR3D_PATH_DAVIDSON
            assert np.abs(r.eval - dense.eval).max() * AUTOCM <= 1e-3
            assert r.max_resid < 1e-5
        print(f"surface {seed}: exact channel blocks {plain.iterations} iterations / {plain.extra['matvecs']} "
              f"H3 products; learned {lrn.iterations} / {lrn.extra['matvecs']}")
        base += plain.extra["matvecs"]
        learned += lrn.extra["matvecs"]
    print(f"training loss {t.extra['lp_loss_first']:.4f} -> {t.extra['lp_loss_last']:.4f}; "
          f"H3 products {base} -> {learned}")
    assert learned < base


@pytest.mark.gpu
def test_learned_without_training_is_an_error():
    fresh = dvr3d_b200.Context(0)
    try:
        with pytest.raises(dvr3d_b200.DVR3DError):
            _solve(fresh, configs.jacobi_h3p_like(10, 12, 16, 45000.0, 40000.0, 10, title="no lp"), 1)
    finally:
        fresh.close()
