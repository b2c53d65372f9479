"""GPU Helmholtz FMM against the oracle (same tree, FP64: agreement to
round-off of the special functions), against direct sums (within eps) and
the golden fixtures, through the python front end and the C ABI."""
import ctypes as C
import os

import numpy as np
import pytest

import fmm2d_b200 as fmm
from conftest import rel_l2
from fmm2d_b200.fmm2d import _helm_run

pytestmark = pytest.mark.gpu
TOL = 1e-10  # GPU vs oracle on the identical tree (Hankel/Bessel round-off)
GOLD = os.path.join(os.path.dirname(__file__), "golden", "helm_golden.npz")


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
@pytest.mark.parametrize("zk", [10.0, 3 + 0.5j])
def test_hfmm_st_vs_oracle(gpu, oracle, kind, pg, zk):
    src, trg, q, d, v = _inputs(20 + pg, 4000, 1500)
    qq = q if "c" in kind else None
    dd = d if "d" in kind else None
    vv = v if "d" in kind else None
    eps = 1e-9
    res = _helm_run(eps, zk, src, qq, dd, vv, trg, pg, pg, 1)
    assert res["ier"] == 0
    ref = oracle.hfmm2d(eps, zk, src, charges=qq, dipstr=dd, dipvec=vv, targets=trg, ifpgh=pg,
                        ifpghtarg=pg)
    for k in ["pot", "grad", "hess"][:pg]:
        assert rel_l2(res[k], ref[k][0]) < TOL, k
        assert rel_l2(res[k + "targ"], ref[k + "targ"][0]) < TOL, k + "targ"


@pytest.mark.parametrize("pg", [1, 2])
def test_hfmm_front_end_vs_direct(gpu, pg):
    """python/test/test_hfmm.py pattern: n=2000, nt=1880, zk=1.1, eps=1e-5,
    first 10 points against h2ddir."""
    src, trg, q, d, v = _inputs(5, 2000, 1880)
    eps, zk, nt = 1e-5, 1.1, 10
    out = fmm.hfmm2d(eps=eps, zk=zk, sources=src, charges=q, dipstr=d, dipvec=v, targets=trg,
                     pg=pg, pgt=pg)
    assert out.ier == 0
    exs = fmm.h2ddir(zk=zk, sources=src, targets=src[:, :nt], charges=q, dipstr=d, dipvec=v,
                     pgt=pg)
    ext = fmm.h2ddir(zk=zk, sources=src, targets=trg[:, :nt], charges=q, dipstr=d, dipvec=v,
                     pgt=pg)
    exs.pot, exs.grad = exs.pottarg, exs.gradtarg
    assert fmm.comperr(ntest=nt, out=out, outex=exs, pg=pg) < eps
    assert fmm.comperr(ntest=nt, out=out, outex=ext, pgt=pg) < eps


@pytest.mark.parametrize("eps", [1e-3, 1e-6, 1e-9, 1e-12])
def test_hfmm_clustered_vs_direct(gpu, eps):
    rng = np.random.default_rng(8)
    n = 20000
    c = rng.uniform(0, 1, (2, 8))
    sig = 10 ** rng.uniform(-3, -1, 8)
    k = rng.integers(0, 8, n)
    src = c[:, k] + sig[k] * rng.normal(size=(2, n))
    q = rng.normal(size=n) + 1j * rng.normal(size=n)
    zk = 20.0
    out = fmm.hfmm2d(eps=eps, zk=zk, sources=src, charges=q, pg=2)
    assert out.ier == 0
    ex = fmm.h2ddir(zk=zk, sources=src, targets=src[:, :200], charges=q, pgt=2)
    assert rel_l2(out.pot[:200], ex.pottarg) < 10 * eps
    assert rel_l2(out.grad[:, :200], ex.gradtarg) < 10 * eps


def test_hfmm_nd3_targets_only_vs_oracle(gpu, oracle):
    src, trg, q, d, v = _inputs(9, 5000, 3000, nd=3)
    zk = 5 + 0.2j
    out = fmm.hfmm2d(eps=1e-6, zk=zk, sources=src, charges=q, dipstr=d, dipvec=v, targets=trg,
                     pgt=2, nd=3)
    assert out.pot is None and out.gradtarg.shape == (3, 2, 3000)
    ref = oracle.hfmm2d(1e-6, zk, src, charges=q, dipstr=d, dipvec=v, targets=trg, ifpghtarg=2,
                        nd=3)
    assert rel_l2(out.pottarg, ref["pottarg"]) < TOL
    assert rel_l2(out.gradtarg, ref["gradtarg"]) < TOL


def test_hfmm_torch_inputs(gpu, oracle):
    import torch
    src, trg, q, d, v = _inputs(11, 3000, 0)
    ts = torch.as_tensor(src, device=gpu)
    tq = torch.as_tensor(q, device=gpu)
    out = fmm.hfmm2d(eps=1e-9, zk=7.0, sources=ts, charges=tq, pg=2)
    assert out.pot.is_cuda
    ref = oracle.hfmm2d(1e-9, 7.0, src, charges=q, ifpgh=2)
    assert rel_l2(out.pot.cpu().numpy(), ref["pot"][0]) < TOL
    assert rel_l2(out.grad.cpu().numpy(), ref["grad"][0]) < TOL


def test_hfmm_high_frequency_runs(gpu, ref):
    """zk = 500 (boxes above 16 wavelengths): the wideband translations run
    (no ier 20) and agree with the reference's own wideband path."""
    src, _, q, _, _ = _inputs(12, 4000, 0)
    out = fmm.hfmm2d(eps=1e-6, zk=500.0, sources=src, charges=q, pg=1)
    assert out.ier == 0
    r = ref.hfmm2d(1e-6, 500.0, src, charges=q, ifpgh=1)
    assert rel_l2(out.pot, r["pot"][0]) < 1e-10


def test_hfmm_high_order_curve(gpu, oracle):
    """Sources on a closed curve with zk = 40 (expansion orders up to ~35)."""
    t = np.linspace(0, 2 * np.pi, 6000, endpoint=False)
    r = 0.4 + 0.05 * np.cos(5 * t)
    src = np.stack([0.5 + r * np.cos(t), 0.5 + r * np.sin(t)])
    rng = np.random.default_rng(13)
    q = rng.normal(size=6000) + 1j * rng.normal(size=6000)
    trg = rng.uniform(0, 1, (2, 2000))
    res = _helm_run(1e-9, 40.0, src, q, None, None, trg, 1, 2, 1)
    assert res["ier"] == 0
    ref = oracle.hfmm2d(1e-9, 40.0, src, charges=q, targets=trg, ifpgh=1, ifpghtarg=2)
    assert rel_l2(res["pot"], ref["pot"][0]) < TOL
    assert rel_l2(res["pottarg"], ref["pottarg"][0]) < TOL
    assert rel_l2(res["gradtarg"], ref["gradtarg"][0]) < TOL


@pytest.mark.parametrize("case", ["k10", "kc"])
def test_h2ddir_device_vs_golden(gpu, case):
    """Device direct sums with Hessians through the C ABI."""
    import torch
    g = np.load(GOLD)
    zk = complex(g["zk"][0 if case == "k10" else 1])
    ref = g["dir_" + case]
    dev = lambda a, dt: torch.as_tensor(np.ascontiguousarray(a), dtype=dt, device=gpu)
    s = dev(g["src"].T, torch.float64)
    t = dev(g["trg"].T, torch.float64)
    q = dev(g["q"], torch.complex128)
    d = dev(g["d"], torch.complex128)
    v = dev(g["v"].T, torch.float64)
    nt = t.shape[0]
    pot = torch.zeros(nt, dtype=torch.complex128, device=gpu)
    grad = torch.zeros((nt, 2), dtype=torch.complex128, device=gpu)
    hess = torch.zeros((nt, 3), dtype=torch.complex128, device=gpu)
    ier = C.c_int(-1)
    P = lambda x: C.c_void_p(x.data_ptr())
    fmm._lib.lib().b2fmm_h2ddir_dev(1, zk.real, zk.imag, s.shape[0], P(s), P(q), P(d), P(v), nt,
                                    P(t), 3, P(pot), P(grad), P(hess), 1e-16,
                                    C.c_void_p(torch.cuda.current_stream().cuda_stream),
                                    C.byref(ier))
    assert ier.value == 0
    assert rel_l2(pot.cpu().numpy(), ref[0]) < 1e-12
    assert rel_l2(grad.cpu().numpy().T, ref[1:3]) < 1e-12
    assert rel_l2(hess.cpu().numpy().T, ref[3:6]) < 1e-11


def test_h2ddir_vs_oracle(gpu, oracle):
    src, trg, q, d, v = _inputs(14, 3000, 500, nd=2)
    zk = 12 + 0.3j
    for pgt in (1, 2):
        out = fmm.h2ddir(zk=zk, sources=src, targets=trg, charges=q, dipstr=d, dipvec=v, pgt=pgt,
                         nd=2)
        ref = oracle.h2ddir(zk, src, trg, charges=q, dipstr=d, dipvec=v, ifpgh=pgt, nd=2)
        assert rel_l2(out.pottarg, ref["pottarg"]) < 1e-12
        if pgt == 2:
            assert rel_l2(out.gradtarg, ref["gradtarg"]) < 1e-12


def test_hfmm_degenerate(gpu):
    src = np.full((2, 50), 0.3)
    q = np.ones(50, complex)
    out = fmm.hfmm2d(eps=1e-6, zk=2.0, sources=src, charges=q, pg=2)
    assert out.ier == 0
    assert np.all(out.pot == 0) and np.all(out.grad == 0)
