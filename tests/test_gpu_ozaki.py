"""FP64 GEMM from int8 Ozaki slices on the tensor cores (dvr3d_b200_ozaki_gemm), against numpy
FP64 and against the DMMA GEMM on the same operands; and the shift-invert solve whose
Cholesky-inverse runs its large products that way, against the oracle's fixture.

Error bound of the 8-slice product (per output entry): the slice remainders and the dropped
slice pairs weigh below 2^-50 max|op(a)(i,:)| max|op(b)(:,j)| per term, so the test allows
K 2^-49 amax_i bmax_j (plus FP64 rounding of the reference)."""
from __future__ import annotations

import os

import numpy as np
import pytest

import dvr3d_b200
from dvr3d_b200 import AUTOCM, configs, parse_deck

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    with dvr3d_b200.Context(0) as c:
        yield c


def _op(x, t):
    return x.T if t else x


def _bound(a_op, b_op, nslice=8):
    k = a_op.shape[1]
    amax = np.abs(a_op).max(axis=1)
    bmax = np.abs(b_op).max(axis=0)
    unit = 2.0 ** (-7 * nslice + 7)  # 2^-49 at 8 slices
    return k * unit * np.outer(amax, bmax) + k * 2.0 ** -52 * (np.abs(a_op) @ np.abs(b_op))


def test_integer_products_are_exact(ctx):
    rng = np.random.default_rng(11)
    a = rng.integers(-1000, 1001, size=(300, 520)).astype(np.float64)
    b = rng.integers(-1000, 1001, size=(520, 190)).astype(np.float64)
    got = ctx.ozaki_gemm(a, b)
    exact = (a.astype(np.int64) @ b.astype(np.int64)).astype(np.float64)
    assert np.array_equal(got, exact)


@pytest.mark.parametrize("m,n,k", [(700, 700, 700), (50, 333, 100), (1024, 256, 1), (257, 129, 4100)])
def test_general_product_within_bound(ctx, m, n, k):
    rng = np.random.default_rng(m + n + k)
    # rows and columns over many orders of magnitude exercise the per-row / per-column scales
    a = rng.standard_normal((m, k)) * np.exp(rng.uniform(-18, 18, size=(m, 1)))
    b = rng.standard_normal((k, n)) * np.exp(rng.uniform(-18, 18, size=(1, n)))
    got = ctx.ozaki_gemm(a, b)
    ref = a @ b
    assert np.all(np.abs(got - ref) <= _bound(a, b))
    dmma = ctx.ozaki_gemm(a, b, nslice=0)
    assert np.all(np.abs(dmma - ref) <= _bound(a, b))


@pytest.mark.parametrize("ta,tb,tri,tri_b", [(False, True, 0, 2), (False, False, 1, 0), (False, False, 0, 1),
                                             (True, False, 2, 0), (True, True, 0, 0)])
def test_transposed_and_triangular_operands(ctx, ta, tb, tri, tri_b):
    rng = np.random.default_rng(7 + 3 * tri + tri_b)
    m, n, k = 640, 448, 640 if (tri or tri_b) else 500
    if tri:
        k = m
    if tri_b:
        k = n
    a_op = rng.standard_normal((m, k))
    b_op = rng.standard_normal((k, n))
    if tri == 1:
        a_op = np.tril(a_op)
    elif tri == 2:
        a_op = np.triu(a_op)
    if tri_b == 1:
        b_op = np.tril(b_op)
    elif tri_b == 2:
        b_op = np.triu(b_op)
    a = np.asfortranarray(_op(a_op, ta))
    b = np.asfortranarray(_op(b_op, tb))
    c0 = rng.standard_normal((m, n))
    got = ctx.ozaki_gemm(a, b, ta=ta, tb=tb, tri=tri, tri_b=tri_b, alpha=-0.75, beta=0.5, c=c0)
    ref = -0.75 * (a_op @ b_op) + 0.5 * c0
    assert np.all(np.abs(got - ref) <= 0.75 * _bound(a_op, b_op) + 1e-15 * np.abs(c0))
    dmma = ctx.ozaki_gemm(a, b, ta=ta, tb=tb, tri=tri, tri_b=tri_b, alpha=-0.75, beta=0.5, c=c0, nslice=0)
    assert np.all(np.abs(got - dmma) <= 1.5 * _bound(a_op, b_op) + 1e-15 * np.abs(c0))


@pytest.mark.parametrize("ta,tri", [(False, 1), (True, 2)])
def test_thin_triangular_products_in_k_chunks(ctx, ta, tri):
    # the Krylov step's shapes: inv(L) Q_k and inv(L)^T Y with 32 columns (128 x 32 tiles, K
    # split into chunks summed in order by a second kernel)
    rng = np.random.default_rng(21 + tri)
    n = 3000
    low = np.tril(rng.standard_normal((n, n))) + n * np.eye(n)
    a_op = low.T if ta else low
    q = rng.standard_normal((n, 32))
    got = ctx.ozaki_gemm(low, q, ta=ta, tri=tri)
    ref = a_op @ q
    assert np.all(np.abs(got - ref) <= _bound(a_op, q))
    dmma = ctx.ozaki_gemm(low, q, ta=ta, tri=tri, nslice=0)
    assert np.all(np.abs(got - dmma) <= 2 * _bound(a_op, q))


def test_lower_output_update(ctx):
    # A22 <- A22 - L21 L21^T on the lower triangle only (the Cholesky's SYRK step); the upper
    # triangle of c must come back untouched
    rng = np.random.default_rng(5)
    n, k = 600, 384
    l21 = rng.standard_normal((n, k))
    c0 = rng.standard_normal((n, n))
    got = ctx.ozaki_gemm(l21, l21, tb=True, lower_out=True, alpha=-1.0, beta=1.0, c=c0)
    ref = c0 - l21 @ l21.T
    lo = np.tril(np.ones((n, n), dtype=bool))
    assert np.all(np.abs(got - ref)[lo] <= _bound(l21, l21.T)[lo] + 1e-15 * np.abs(c0)[lo])
    assert np.array_equal(got[~lo], c0[~lo])


@pytest.mark.parametrize("nslice", [4, 6])
def test_fewer_slices_within_their_bound(ctx, nslice):
    rng = np.random.default_rng(nslice)
    a = rng.standard_normal((300, 800))
    b = rng.standard_normal((800, 200))
    got = ctx.ozaki_gemm(a, b, nslice=nslice)
    assert np.all(np.abs(got - a @ b) <= _bound(a, b, nslice))


def test_non_finite_entries_propagate(ctx):
    rng = np.random.default_rng(3)
    a = rng.standard_normal((200, 300))
    b = rng.standard_normal((300, 100))
    a[17, 5] = np.nan
    got = ctx.ozaki_gemm(a, b)
    assert np.all(np.isnan(got[17]))
    assert np.all(np.isfinite(np.delete(got, 17, axis=0)))


def test_rejects_k_beyond_exact_accumulation(ctx):
    a = np.zeros((2, 16386))
    b = np.zeros((16386, 2))
    with pytest.raises(dvr3d_b200.DVR3DError):
        ctx.ozaki_gemm(a, b)


def _cfg2_levels(ctx, ozaki: str, krylov: str = "0"):
    w = configs.config2()
    deck = parse_deck(w.deck)
    ctx.set_pes(w.pes)
    keys = {"DVR3D_OZAKI": ozaki, "DVR3D_OZAKI_KRYLOV": krylov}
    old = {k: os.environ.get(k) for k in keys}
    os.environ.update(keys)
    try:
        return ctx.solve(deck, 0, precision=dvr3d_b200.DVR3D_PREC_MIXED_DAVIDSON, nlevels=300)
    finally:
        for k, v in old.items():
            if v is None:
                del os.environ[k]
            else:
                os.environ[k] = v


def test_shift_invert_with_int8_factorisation_matches_oracle(ctx):
    fx = np.load(os.path.join(os.path.dirname(__file__), "golden", "config2_oracle.npz"))
    oz = _cfg2_levels(ctx, "1")
    plain = _cfg2_levels(ctx, "0")
    assert oz.fallback == 0 and len(oz.eval) == 300
    lv = fx["levels"][:300]
    assert np.abs(oz.eval - lv).max() * AUTOCM <= 1e-6
    assert np.abs(oz.eval - plain.eval).max() * AUTOCM <= 1e-6
    # the opt-in int8 Krylov products (inv(L) sliced once, 32-column blocks in K chunks)
    kr = _cfg2_levels(ctx, "1", krylov="1")
    assert kr.fallback == 0 and len(kr.eval) == 300
    assert np.abs(kr.eval - lv).max() * AUTOCM <= 1e-6
