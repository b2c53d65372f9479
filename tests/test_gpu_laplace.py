"""GPU Laplace/Cauchy FMM against the oracle (same tree, FP64: agreement to
round-off) and against direct sums (within eps), through the python front end
and so through the C ABI."""
import numpy as np
import pytest

import fmm2d_b200 as fmm
from conftest import rel_l2

pytestmark = pytest.mark.gpu
TOL_FP64 = 1e-11  # GPU FP64 vs oracle on the identical tree


def _inputs(seed, n, nt, nd=1):
    rng = np.random.default_rng(seed)
    src = rng.uniform(0, 1, (2, n))
    trg = rng.uniform(0, 1, (2, nt))
    shape = (n,) if nd == 1 else (nd, n)
    q = rng.normal(size=shape) + 1j * rng.normal(size=shape)
    d = rng.normal(size=shape) + 1j * rng.normal(size=shape)
    v = rng.uniform(-1, 1, (2, n) if nd == 1 else (nd, 2, n))
    return src, trg, q, d, v


@pytest.mark.parametrize("kind", ["c", "d", "cd"])
@pytest.mark.parametrize("pg", [1, 2, 3])
@pytest.mark.parametrize("nd", [1, 2])
def test_lfmm_st_vs_oracle(gpu, oracle, kind, pg, nd):
    src, trg, q, d, v = _inputs(10 + pg, 4000, 1500, nd)
    qq = q if "c" in kind else None
    dd = d if "d" in kind else None
    vv = v if "d" in kind else None
    eps = 1e-6
    out = fmm.lfmm2d(eps=eps, sources=src, charges=qq, dipstr=dd, dipvec=vv, targets=trg, pg=pg,
                     pgt=pg, nd=nd, precision="fp64")
    assert out.ier == 0
    ref = oracle.lfmm2d(eps, src, charges=qq, dipstr=dd, dipvec=vv, targets=trg, ifpgh=pg,
                        ifpghtarg=pg, nd=nd)
    sq = (lambda a: a[0] if nd == 1 else a)
    for k in ["pot", "grad", "hess"][:pg]:
        assert rel_l2(getattr(out, k), sq(ref[k])) < TOL_FP64, k
        assert rel_l2(getattr(out, k + "targ"), sq(ref[k + "targ"])) < TOL_FP64, k + "targ"


@pytest.mark.parametrize("pg", [1, 2, 3])
def test_cfmm_vs_oracle(gpu, oracle, pg):
    src, trg, q, d, _ = _inputs(3, 5000, 0, nd=3)
    out = fmm.cfmm2d(eps=1e-9, sources=src, charges=q, dipstr=d, pg=pg, nd=3, precision="fp64")
    ref = oracle.cfmm2d(1e-9, src, charges=q, dipstr=d, ifpgh=pg, nd=3)
    for k in ["pot", "grad", "hess"][:pg]:
        assert rel_l2(getattr(out, k), ref[k]) < TOL_FP64, k


def test_rfmm_targets_only(gpu, oracle):
    rng = np.random.default_rng(5)
    src = rng.uniform(0, 1, (2, 6000))
    trg = rng.uniform(-0.2, 1.2, (2, 3000))
    q = rng.normal(size=6000)
    out = fmm.rfmm2d(eps=1e-6, sources=src, charges=q, targets=trg, pgt=2, precision="fp64")
    assert out.pot is None and out.gradtarg.shape == (2, 3000)
    ref = oracle.rfmm2d(1e-6, src, charges=q, targets=trg, ifpghtarg=2)
    assert rel_l2(out.pottarg, ref["pottarg"][0]) < TOL_FP64
    assert rel_l2(out.gradtarg, ref["gradtarg"][0]) < TOL_FP64
    ex = oracle.r2ddir(src, trg[:, :100], charges=q, ifpgh=2)
    assert rel_l2(out.pottarg[:100], ex["pottarg"][0]) < 1e-6
    assert rel_l2(out.gradtarg[:, :100], ex["gradtarg"][0]) < 1e-6


@pytest.mark.parametrize("eps", [1e-3, 1e-6, 1e-9, 1e-12])
def test_lfmm_clustered_vs_direct(gpu, oracle, eps):
    """16-Gaussian cloud (deep adaptive tree) against the FP64 direct sum."""
    rng = np.random.default_rng(2)
    n = 30000
    c = rng.uniform(0, 1, (2, 16))
    sig = 10 ** rng.uniform(-4, -1, 16)
    k = rng.integers(0, 16, n)
    src = c[:, k] + sig[k] * rng.normal(size=(2, n))
    q = rng.normal(size=n) + 1j * rng.normal(size=n)
    d = rng.normal(size=n) + 0j
    ph = rng.uniform(0, 2 * np.pi, n)
    v = np.stack([np.cos(ph), np.sin(ph)])
    out = fmm.lfmm2d(eps=eps, sources=src, charges=q, dipstr=d, dipvec=v, pg=2, precision="fp64")
    idx = rng.choice(n, 200, replace=False)
    ex = oracle.l2ddir(src, src[:, idx], charges=q, dipstr=d, dipvec=v, ifpgh=2)
    err = np.sqrt((np.linalg.norm(out.pot[idx] - ex["pottarg"][0]) ** 2 +
                   np.linalg.norm(out.grad[:, idx] - ex["gradtarg"][0]) ** 2) /
                  (np.linalg.norm(ex["pottarg"][0]) ** 2 + np.linalg.norm(ex["gradtarg"][0]) ** 2))
    assert err < eps


def test_torch_device_inputs(gpu, oracle):
    import torch
    src, trg, q, d, v = _inputs(9, 3000, 700)
    ts = torch.as_tensor(src, device=gpu)
    out = fmm.lfmm2d(eps=1e-6, sources=ts, charges=torch.as_tensor(q, device=gpu),
                     targets=torch.as_tensor(trg, device=gpu), pg=2, pgt=2, precision="fp64")
    assert out.pot.is_cuda and out.grad.shape == (2, 3000)
    ref = oracle.lfmm2d(1e-6, src, charges=q, targets=trg, ifpgh=2, ifpghtarg=2)
    assert rel_l2(out.pot.cpu().numpy(), ref["pot"][0]) < TOL_FP64
    assert rel_l2(out.gradtarg.cpu().numpy(), ref["gradtarg"][0]) < TOL_FP64


def test_small_and_degenerate(gpu, oracle):
    # one source, coincident points, all points identical
    for src in (np.array([[0.3], [0.4]]), np.zeros((2, 40)) + 0.5,
                np.concatenate([np.zeros((2, 10)), np.ones((2, 10))], 1)):
        n = src.shape[1]
        q = np.arange(1, n + 1) + 0.5j
        out = fmm.lfmm2d(eps=1e-6, sources=src, charges=q, pg=2, precision="fp64")
        ref = oracle.lfmm2d(1e-6, src, charges=q, ifpgh=2)
        np.testing.assert_allclose(out.pot, ref["pot"][0], rtol=1e-12, atol=1e-12)
        np.testing.assert_allclose(out.grad, ref["grad"][0], rtol=1e-12, atol=1e-12)


def test_direct_sums_vs_oracle(gpu, oracle):
    import os
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "laplace_direct.npz"))
    o = fmm.l2ddir(sources=g["src"], targets=g["trg"], charges=g["q"], dipstr=g["d"],
                   dipvec=g["v"], pgt=3)
    assert rel_l2(o.pottarg, g["lpot"]) < 1e-13
    assert rel_l2(o.gradtarg, g["lgrad"]) < 1e-13
    assert rel_l2(o.hesstarg, g["lhess"]) < 1e-13
    o = fmm.c2ddir(sources=g["src"], targets=g["trg"], charges=g["q"], dipstr=g["d"], pgt=3)
    assert rel_l2(o.pottarg, g["cpot"]) < 1e-13
    assert rel_l2(o.gradtarg, g["cgrad"]) < 1e-13
    assert rel_l2(o.hesstarg, g["chess"]) < 1e-13
    o = fmm.r2ddir(sources=g["src"], targets=g["trg"], charges=g["qr"], dipstr=g["dr"],
                   dipvec=g["v"], pgt=3)
    assert rel_l2(o.pottarg, g["rpot"]) < 1e-13
    assert rel_l2(o.hesstarg, g["rhess"]) < 1e-13
