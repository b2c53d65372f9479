"""Biharmonic (bhfmm2d) and Stokes (stfmm2d) on the GPU against the reference.

The GPU evaluates both through one FP64 Cauchy FMM over 4 nd densities
(fmm2d_b200/csrc/biharmonic.cu); the reference has its own biharmonic
expansions (src/biharmonic/bhrouts2d.f).  So:
  * the all-pairs sums (bh2ddir, st2ddir) equal the reference's direct
    kernels (bh2d_directcdg, st2ddirectstokstrsg) to round-off;
  * the FMMs are within the requested eps of those direct sums (the
    reference test's criterion, test/biharmonic/test_bhfmm2d.f: relative l2
    error over sample points below eps) and within eps of the reference's
    own FMM output;
  * the Fortran entry points bhfmm2d_ / stfmm2d_ of libfmm2d.so do the same.
"""
import ctypes as C
import os

import numpy as np
import pytest

import fmm2d_b200 as fmm
from conftest import rel_l2
from test_ref_pin import hk_inputs

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def _I(v):
    return C.byref(C.c_int(v))


def _cx(rng, *shape):
    return rng.normal(size=shape) + 1j * rng.normal(size=shape)


def ref_bh_direct(r, src, charges, dip, trg, nd):
    """bh2d_directcdg of the reference (charges (nd,2,ns), dip (nd,3,ns))."""
    ns, nt = src.shape[1], trg.shape[1]
    vel = np.zeros((nt, nd), complex)
    grad = np.zeros((nt, 3, nd), complex)
    ch = np.ascontiguousarray(np.transpose(charges.reshape(nd, 2, ns), (2, 1, 0)))
    dp = np.ascontiguousarray(np.transpose(dip.reshape(nd, 3, ns), (2, 1, 0)))
    r.bh2d_directcdg_(_I(nd), _p(np.ascontiguousarray(src.T)), _I(ns), _p(ch), _p(dp),
                      _p(np.ascontiguousarray(trg.T)), _I(nt), _p(vel), _p(grad),
                      C.byref(C.c_double(1e-14)))
    return vel.T, np.transpose(grad, (2, 1, 0))


def ref_bhfmm(lib, eps, src, charges, dip, trg, nd, ifc=1, ifd=1, pg=2):
    ns, nt = src.shape[1], trg.shape[1]
    ch = np.ascontiguousarray(np.transpose(charges.reshape(nd, 2, ns), (2, 1, 0)))
    dp = np.ascontiguousarray(np.transpose(dip.reshape(nd, 3, ns), (2, 1, 0)))
    pot = np.zeros((ns, nd), complex)
    grad = np.zeros((ns, 3, nd), complex)
    hess = np.zeros((ns, 3, nd), complex)
    pt = np.zeros((nt, nd), complex)
    gt = np.zeros((nt, 3, nd), complex)
    ht = np.zeros((nt, 3, nd), complex)
    ier = C.c_int(-1)
    lib.bhfmm2d_(_I(nd), C.byref(C.c_double(eps)), _I(ns), _p(np.ascontiguousarray(src.T)),
                 _I(ifc), _p(ch), _I(ifd), _p(dp), _I(0), _I(pg), _p(pot), _p(grad), _p(hess),
                 _I(nt), _p(np.ascontiguousarray(trg.T)), _I(pg), _p(pt), _p(gt), _p(ht),
                 C.byref(ier))
    t = lambda a: np.transpose(a, tuple(reversed(range(a.ndim))))
    return ier.value, t(pot), t(grad), t(pt), t(gt)


def test_bh_direct_equals_reference_kernel(gpu, ref):
    r = ref.lib()
    rng = np.random.default_rng(1)
    nd, ns, nt = 2, 700, 500
    src, trg = rng.uniform(0, 1, (2, ns)), rng.uniform(0, 1, (2, nt))
    ch, dp = _cx(rng, nd, 2, ns), _cx(rng, nd, 3, ns)
    out = fmm.bh2ddir(sources=src, targets=trg, charges=ch, dipoles=dp, pgt=2, nd=nd)
    v, g = ref_bh_direct(r, src, ch, dp, trg, nd)
    # the terms in w/conj(w) come from r conj(A) - conj(B), two sums of size
    # |r| sum |q/w| that cancel to sum |q|: round-off grows by about |r|/|w|
    assert rel_l2(out.pottarg, v) < 1e-12
    assert rel_l2(out.gradtarg, g) < 1e-12


def test_reference_test_case(gpu, ref):
    """test/biharmonic/test_bhfmm2d.f: 9998 sources, 9999 targets (hkrand),
    dipoles only, eps 0.5e-6, pg = pgt = 2; relative l2 error of the first
    20 sources and targets against the direct sum below eps."""
    r = ref.lib()
    src, trg, _, _, _ = hk_inputs(ref, 9998, 9999)
    rng = np.random.default_rng(2)
    dp = _cx(rng, 3, src.shape[1])
    eps = 0.5e-6
    out = fmm.bhfmm2d(eps=eps, sources=src, dipoles=dp, targets=trg, pg=2, pgt=2)
    assert out.ier == 0
    zero = np.zeros((1, 2, src.shape[1]), complex)
    vs, gs = ref_bh_direct(r, src, zero, dp, src[:, :20], 1)
    vt, gt = ref_bh_direct(r, src, zero, dp, trg[:, :20], 1)
    # the sources' own terms are skipped by the direct sum's threshold
    assert rel_l2(out.pot[:20], vs[0]) < eps
    assert rel_l2(out.grad[:, :20], gs[0]) < eps
    assert rel_l2(out.pottarg[:20], vt[0]) < eps
    assert rel_l2(out.gradtarg[:, :20], gt[0]) < eps


@pytest.mark.parametrize("eps", [1e-6, 1e-9])
@pytest.mark.parametrize("nd", [1, 2])
def test_bhfmm_vs_direct_and_reference(gpu, ref, eps, nd):
    r = ref.lib()
    rng = np.random.default_rng(3 + nd)
    ns, nt = 20000, 5000
    # a clustered cloud: deep trees, lists 3 and 4 in use
    ctr = rng.uniform(0.2, 0.8, (2, 5))
    src = ctr[:, rng.integers(0, 5, ns)] + 0.03 * rng.normal(size=(2, ns))
    trg = rng.uniform(0, 1, (2, nt))
    ch, dp = _cx(rng, nd, 2, ns), _cx(rng, nd, 3, ns)
    args = dict(charges=ch if nd > 1 else ch[0], dipoles=dp if nd > 1 else dp[0])
    out = fmm.bhfmm2d(eps=eps, sources=src, targets=trg, pg=2, pgt=2, nd=nd, **args)
    assert out.ier == 0
    pot = out.pot.reshape(nd, ns)
    grad = out.grad.reshape(nd, 3, ns)
    pt = out.pottarg.reshape(nd, nt)
    gt = out.gradtarg.reshape(nd, 3, nt)
    k = 400
    vs, gs = ref_bh_direct(r, src, ch, dp, src[:, :k], nd)
    vt, gtx = ref_bh_direct(r, src, ch, dp, trg[:, :k], nd)
    for a, b in ((pot[:, :k], vs), (grad[:, :, :k], gs), (pt[:, :k], vt), (gt[:, :, :k], gtx)):
        assert rel_l2(a, b) < eps
    ier, rp, rg, rpt, rgt = ref_bhfmm(r, eps, src, ch, dp, trg, nd)
    assert ier == 0
    for a, b in ((pot, rp), (grad, rg), (pt, rpt), (gt, rgt)):
        assert rel_l2(a, b) < 2 * eps


def test_bhfmm_fortran_entry(gpu, ref):
    r = ref.lib()
    f77 = C.CDLL(os.path.join(ROOT, "fmm2d_b200", "libfmm2d.so"))
    rng = np.random.default_rng(7)
    ns, nt, nd = 6000, 2000, 1
    src, trg = rng.uniform(0, 1, (2, ns)), rng.uniform(0, 1, (2, nt))
    ch, dp = _cx(rng, nd, 2, ns), _cx(rng, nd, 3, ns)
    ier, p1, g1, pt1, gt1 = ref_bhfmm(f77, 1e-9, src, ch, dp, trg, nd)
    ier2, p2, g2, pt2, gt2 = ref_bhfmm(r, 1e-9, src, ch, dp, trg, nd)
    assert ier == 0 and ier2 == 0
    for a, b in ((p1, p2), (g1, g2), (pt1, pt2), (gt1, gt2)):
        assert rel_l2(a, b) < 2e-9


def ref_stokes(lib, eps, src, sto, sl, sv, trg, nd, lev=3, direct=False):
    ns, nt = src.shape[1], trg.shape[1]
    T = lambda a: np.ascontiguousarray(np.transpose(a.reshape(nd, 2, ns), (2, 1, 0)))
    S, Tg = np.ascontiguousarray(src.T), np.ascontiguousarray(trg.T)
    pot, pre, grad = np.zeros((ns, 2, nd)), np.zeros((ns, nd)), np.zeros((ns, 2, 2, nd))
    pt, prt, gt = np.zeros((nt, 2, nd)), np.zeros((nt, nd)), np.zeros((nt, 2, 2, nd))
    ier = C.c_int(0)
    if direct:
        lib.st2ddirectstokstrsg_(_I(nd), _p(S), _I(1), _p(T(sto)), _I(1), _p(T(sl)), _p(T(sv)),
                                 _I(ns), _p(Tg), _I(nt), _p(pt), _p(prt), _p(gt),
                                 C.byref(C.c_double(1e-16)))
    else:
        lib.stfmm2d_(_I(nd), C.byref(C.c_double(eps)), _I(ns), _p(S), _I(1), _p(T(sto)), _I(1),
                     _p(T(sl)), _p(T(sv)), _I(lev), _p(pot), _p(pre), _p(grad), _I(nt), _p(Tg),
                     _I(lev), _p(pt), _p(prt), _p(gt), C.byref(ier))
    t = lambda a: np.transpose(a, tuple(reversed(range(a.ndim))))
    return ier.value, t(pot), t(pre), t(grad), t(pt), t(prt), t(gt)


@pytest.mark.parametrize("eps", [1e-6, 1e-10])
def test_stfmm_vs_reference(gpu, ref, eps):
    r = ref.lib()
    rng = np.random.default_rng(8)
    ns, nt, nd = 15000, 4000, 2
    src, trg = rng.uniform(0, 1, (2, ns)), rng.uniform(0, 1, (2, nt))
    sto, sl, sv = (rng.normal(size=(nd, 2, ns)) for _ in range(3))
    out = fmm.stfmm2d(eps=eps, sources=src, stoklet=sto, strslet=sl, strsvec=sv, targets=trg,
                      ifppreg=3, ifppregtarg=3, nd=nd)
    assert out.ier == 0
    ier, pot, pre, grad, pt, prt, gt = ref_stokes(r, eps, src, sto, sl, sv, trg, nd)
    assert ier == 0
    for k, b in (("pot", pot), ("pre", pre), ("grad", grad), ("pottarg", pt), ("pretarg", prt),
                 ("gradtarg", gt)):
        assert rel_l2(getattr(out, k), b) < 5 * eps, k
    # targets against the reference's direct Stokes kernel
    _, _, _, _, dpt, dprt, dgt = ref_stokes(r, eps, src, sto, sl, sv, trg[:, :300], nd,
                                            direct=True)
    assert rel_l2(out.pottarg[:, :, :300], dpt) < 5 * eps
    assert rel_l2(out.pretarg[:, :300], dprt) < 5 * eps
    assert rel_l2(out.gradtarg[..., :300], dgt) < 5 * eps


def test_st2ddir_equals_reference_kernel(gpu, ref):
    r = ref.lib()
    rng = np.random.default_rng(9)
    ns, nt, nd = 800, 300, 1
    src, trg = rng.uniform(0, 1, (2, ns)), rng.uniform(0, 1, (2, nt))
    sto, sl, sv = (rng.normal(size=(nd, 2, ns)) for _ in range(3))
    out = fmm.st2ddir(eps=1e-16, sources=src, stoklet=sto[0], strslet=sl[0], strsvec=sv[0],
                      targets=trg, ifppregtarg=3)
    _, _, _, _, pt, prt, gt = ref_stokes(r, 0, src, sto, sl, sv, trg, nd, direct=True)
    assert rel_l2(out.pottarg, pt) < 1e-12
    assert rel_l2(out.pretarg, prt) < 1e-12
    assert rel_l2(out.gradtarg, gt) < 1e-12


def test_stfmm_fortran_entry(gpu, ref):
    r = ref.lib()
    f77 = C.CDLL(os.path.join(ROOT, "fmm2d_b200", "libfmm2d.so"))
    rng = np.random.default_rng(10)
    ns, nt, nd = 5000, 1000, 1
    src, trg = rng.uniform(0, 1, (2, ns)), rng.uniform(0, 1, (2, nt))
    sto, sl, sv = (rng.normal(size=(nd, 2, ns)) for _ in range(3))
    a = ref_stokes(f77, 1e-9, src, sto, sl, sv, trg, nd)
    b = ref_stokes(r, 1e-9, src, sto, sl, sv, trg, nd)
    assert a[0] == 0 and b[0] == 0
    for x, y in zip(a[1:], b[1:]):
        assert rel_l2(x, y) < 1e-8
