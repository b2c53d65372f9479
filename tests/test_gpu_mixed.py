"""Mixed-precision Laplace path (FP32 near field and M2L, FP64 expansions)
against the FP64 direct sum (error below eps) and against the oracle."""
import numpy as np
import pytest

import fmm2d_b200 as fmm
from conftest import rel_l2

pytestmark = pytest.mark.gpu


def _gauss16(rng, n):
    c = rng.uniform(0, 1, (2, 16))
    sig = 10 ** rng.uniform(-4, -1, 16)
    k = rng.integers(0, 16, n)
    return c[:, k] + sig[k] * rng.normal(size=(2, n))


@pytest.mark.parametrize("eps", [1e-3, 1e-6])
def test_mixed_lfmm_vs_direct(gpu, oracle, eps):
    rng = np.random.default_rng(21)
    n = 40000
    src = _gauss16(rng, n)
    q = rng.normal(size=n) + 1j * rng.normal(size=n)
    d = rng.normal(size=n) + 0j
    ph = rng.uniform(0, 2 * np.pi, n)
    v = np.stack([np.cos(ph), np.sin(ph)])
    out = fmm.lfmm2d(eps=eps, sources=src, charges=q, dipstr=d, dipvec=v, pg=2,
                     precision="mixed")
    assert out.ier == 0
    idx = rng.choice(n, 300, replace=False)
    ex = oracle.l2ddir(src, src[:, idx], charges=q, dipstr=d, dipvec=v, ifpgh=2)
    err = np.sqrt((np.linalg.norm(out.pot[idx] - ex["pottarg"][0]) ** 2 +
                   np.linalg.norm(out.grad[:, idx] - ex["gradtarg"][0]) ** 2) /
                  (np.linalg.norm(ex["pottarg"][0]) ** 2 + np.linalg.norm(ex["gradtarg"][0]) ** 2))
    assert err < eps


@pytest.mark.parametrize("pg", [1, 2, 3])
def test_mixed_st_vs_oracle(gpu, oracle, pg):
    rng = np.random.default_rng(30 + pg)
    n, nt, nd = 6000, 2500, 2
    src = rng.uniform(0, 1, (2, n))
    trg = rng.uniform(0, 1, (2, nt))
    q = rng.normal(size=(nd, n)) + 1j * rng.normal(size=(nd, n))
    d = rng.normal(size=(nd, n)) + 1j * rng.normal(size=(nd, n))
    v = rng.uniform(-1, 1, (nd, 2, n))
    out = fmm.lfmm2d(eps=1e-6, sources=src, charges=q, dipstr=d, dipvec=v, targets=trg, pg=pg,
                     pgt=pg, nd=nd, precision="mixed")
    ref = oracle.lfmm2d(1e-6, src, charges=q, dipstr=d, dipvec=v, targets=trg, ifpgh=pg,
                        ifpghtarg=pg, nd=nd)
    for k in ["pot", "grad", "hess"][:pg]:
        assert rel_l2(getattr(out, k), ref[k]) < 1e-6, k
        assert rel_l2(getattr(out, k + "targ"), ref[k + "targ"]) < 1e-6, k + "targ"


def test_mixed_cfmm_nd3_and_auto(gpu, oracle):
    rng = np.random.default_rng(8)
    n = 8000
    src = _gauss16(rng, n)
    q = rng.normal(size=(3, n)) + 0j
    out = fmm.cfmm2d(eps=1e-6, sources=src, charges=q, pg=2, nd=3)  # auto -> mixed
    ref = oracle.cfmm2d(1e-6, src, charges=q, ifpgh=2, nd=3)
    assert rel_l2(out.pot.real, ref["pot"].real) < 1e-6
    assert rel_l2(out.grad, ref["grad"]) < 1e-6


def test_mixed_graded_curve_nearly_coincident_sources(gpu):
    """Sources on a curve with density graded over 1e3 (separations down to
    ~1e-11): the mixed path stays within eps for the potential and the
    gradient (pair differences are formed in FP64)."""
    from fmm2d_b200.costmodel import make_problem
    src, q = make_problem("curve", 400000, 11)
    d = np.sort(np.hypot(*np.diff(src[:, np.argsort(np.arctan2(src[1] - 0.5, src[0] - 0.5))],
                                  axis=1)))
    assert d[0] < 1e-10
    out = fmm.rfmm2d(eps=1e-6, sources=src, charges=q, pg=2, precision="mixed")
    rng = np.random.default_rng(0)
    idx = np.sort(rng.choice(400000, 300, replace=False))
    ex = fmm.r2ddir(sources=src, targets=src[:, idx], charges=q, pgt=2)
    assert rel_l2(out.pot[idx], ex.pottarg) < 1e-6
    assert rel_l2(out.grad[:, idx], ex.gradtarg) < 1e-6


def test_mixed_close_pairs_duplicates_and_targets(gpu, oracle):
    """Uniform sources with 300 partners 1e-10 away (far below the near-field
    pass's 2^-20 box-size threshold), 50 exact duplicates, and targets 1e-10
    from sources: at exactly those points the mixed potential and gradient
    (dominated by the close partner) match the FP64 direct sum to 1e-6, and
    duplicates are left out as the reference leaves out pairs at r = 0."""
    rng = np.random.default_rng(77)
    base = rng.uniform(0, 1, (2, 20000))
    ang = rng.uniform(0, 2 * np.pi, 300)
    close = base[:, :300] + 1e-10 * np.stack([np.cos(ang), np.sin(ang)])
    dup = base[:, 300:350].copy()
    src = np.concatenate([base, close, dup], axis=1)
    n = src.shape[1]
    q = rng.normal(size=n) + 1j * rng.normal(size=n)
    d = rng.normal(size=n) + 1j * rng.normal(size=n)
    v = rng.uniform(-1, 1, (2, n))
    trg = base[:, 400:600] + 1e-10 * rng.normal(size=(2, 200))
    out = fmm.lfmm2d(eps=1e-6, sources=src, charges=q, dipstr=d, dipvec=v, targets=trg, pg=2,
                     pgt=2, precision="mixed")
    assert out.ier == 0
    idx = np.concatenate([np.arange(300), np.arange(300, 350), 20000 + np.arange(300),
                          20300 + np.arange(50)])
    ex = oracle.l2ddir(src, src[:, idx], charges=q, dipstr=d, dipvec=v, ifpgh=2)
    # the direct sum at a source includes the source itself only at r = 0,
    # which the kernel leaves out, as it does for the exact duplicates
    assert rel_l2(out.pot[idx], ex["pottarg"][0]) < 1e-6
    assert rel_l2(out.grad[:, idx], ex["gradtarg"][0]) < 1e-6
    ext = oracle.l2ddir(src, trg, charges=q, dipstr=d, dipvec=v, ifpgh=2)
    assert rel_l2(out.pottarg, ext["pottarg"][0]) < 1e-6
    assert rel_l2(out.gradtarg, ext["gradtarg"][0]) < 1e-6


def test_near_field_tile_shapes_agree(gpu, oracle):
    """Every near-field tile shape, on every leaf-size class, gives the same
    result as shape 0 to FP32 round-off and stays within eps of the oracle;
    unknown classes or shapes are refused."""
    from fmm2d_b200 import _lib, autotune
    L = _lib.lib()
    saved = [L.b2fmm_get_p2p_shape(c) for c in range(autotune.NCLASSES)]
    assert L.b2fmm_set_p2p_shape(3, 0) == 100 and L.b2fmm_set_p2p_shape(0, 3) == 100
    assert L.b2fmm_get_p2p_shape(-1) == -1
    rng = np.random.default_rng(12)
    n = 30000
    src = _gauss16(rng, n)
    q = rng.normal(size=n) + 1j * rng.normal(size=n)
    d = rng.normal(size=n) + 1j * rng.normal(size=n)
    v = rng.uniform(-1, 1, (2, n))
    ref = oracle.lfmm2d(1e-6, src, charges=q, dipstr=d, dipvec=v, ifpgh=2)
    try:
        for c, nd in enumerate(autotune.CLASS_NDIV):
            outs = []
            for s in range(len(autotune.SHAPES)):
                assert L.b2fmm_set_p2p_shape(c, s) == 0 and L.b2fmm_get_p2p_shape(c) == s
                o = fmm.lfmm2d(eps=1e-6, sources=src, charges=q, dipstr=d, dipvec=v, pg=2,
                               precision="mixed", ndiv=nd)
                assert o.ier == 0
                outs.append(o)
            for o in outs:
                assert rel_l2(o.pot, outs[0].pot) < 1e-7 and rel_l2(o.grad, outs[0].grad) < 1e-7
            assert rel_l2(outs[0].grad, ref["grad"]) < 1e-6
    finally:
        for c, s in enumerate(saved):
            L.b2fmm_set_p2p_shape(c, s)


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
@pytest.mark.parametrize("nd", [4, 8, 11])
def test_many_densities_vs_oracle(gpu, oracle, precision, nd):
    """nd = 4 and 8 density vectors (one chunk of the widest near-field and
    far-field kernels) and nd = 11 (chunks of 8, 2 and 1), with hessians:
    equal to the oracle within eps (mixed) or round-off (FP64)."""
    rng = np.random.default_rng(40 + nd)
    n, nt = 9000, 3000
    src = _gauss16(rng, n)
    trg = rng.uniform(src.min(), src.max(), (2, nt))
    q = rng.normal(size=(nd, n)) + 1j * rng.normal(size=(nd, n))
    d = rng.normal(size=(nd, n)) + 1j * rng.normal(size=(nd, n))
    out = fmm.cfmm2d(eps=1e-6, sources=src, charges=q, dipstr=d, targets=trg, pg=3, pgt=3,
                     nd=nd, precision=precision)
    ref = oracle.cfmm2d(1e-6, src, charges=q, dipstr=d, targets=trg, ifpgh=3, ifpghtarg=3,
                        nd=nd)
    tol = 1e-6 if precision == "mixed" else 1e-11
    for k in ("pot", "grad", "hess"):
        assert rel_l2(getattr(out, k), ref[k]) < tol, k
    for k in ("pottarg", "gradtarg", "hesstarg"):
        assert rel_l2(getattr(out, k), ref[k]) < tol, k
