"""Helmholtz on the CPU: the oracle restatement pinned against the mpmath
golden fixtures and the reference's own test cases; the host build of the
special functions the CUDA kernels use (same source) against the fixtures;
front-end argument handling that needs no GPU."""
import ctypes as C
import os

import numpy as np
import pytest

import fmm2d_b200 as fmm
from conftest import rel_l2
from fmm2d_b200 import _lib

GOLD = os.path.join(os.path.dirname(__file__), "golden", "helm_golden.npz")


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLD)


def _lib_special(kind, n, z, rs):
    out = np.zeros(4 if kind == 0 else 2 * (n + 1))
    _lib.lib().b2fmm_helm_special(kind, n, complex(z).real, complex(z).imag, rs,
                                  out.ctypes.data_as(C.c_void_p))
    return out[0::2] + 1j * out[1::2]


def _htol(z):
    # power-series regions lose accuracy like exp(2 Im z) off the real axis
    return 1e-13 if complex(z).imag == 0 else 1e-12


def test_oracle_hankel_matches_golden(oracle, gold):
    for z, (e0, e1) in zip(gold["hankel_z"], gold["hankel"]):
        h0, h1 = oracle.hankel01(z)
        assert abs(h0 - e0) / abs(e0) < _htol(z), z
        assert abs(h1 - e1) / abs(e1) < _htol(z), z


def test_device_hankel_source_matches_golden(gold):
    """hank01 of the CUDA kernels, compiled for the host."""
    for z, (e0, e1) in zip(gold["hankel_z"], gold["hankel"]):
        h0, h1 = _lib_special(0, 0, z, 1.0)
        assert abs(h0 - e0) / abs(e0) < _htol(z), z
        assert abs(h1 - e1) / abs(e1) < _htol(z), z


@pytest.mark.parametrize("which", ["oracle", "device"])
def test_scaled_sequences_match_golden(oracle, gold, which):
    for z, rs, n, ej, eh in zip(gold["seq_z"], gold["seq_rs"], gold["seq_n"], gold["seq_j"],
                                gold["seq_h"]):
        n = int(n)
        if which == "oracle":
            j = oracle.jbessel2d(n, z, rs)
            h = oracle.h2dall(n, z, rs)
        else:
            j = _lib_special(1, n, z, rs)
            h = _lib_special(2, n, z, rs)
        m = np.abs(ej[: n + 1]) > 1e-250
        assert np.max(np.abs(j[: n + 1][m] - ej[: n + 1][m]) / np.abs(ej[: n + 1][m])) < 1e-12
        assert np.max(np.abs(h[: n + 1] - eh[: n + 1]) / np.abs(eh[: n + 1])) < 1e-12


def test_h2dterms_device_source_matches_oracle(oracle):
    ier = C.c_int(0)
    for zk in (1.1, 10.0, 40.0, 3 + 0.5j):
        for eps in (1e-3, 1e-6, 0.51e-8, 1e-9, 1e-12):
            for l in range(8):
                bs = 1.0 / 2**l
                p = _lib.lib().b2fmm_h2dterms(bs, complex(zk).real, complex(zk).imag, eps,
                                              C.byref(ier))
                assert ier.value == 0
                assert p == oracle.h2dterms(bs, zk, eps), (zk, eps, l)


@pytest.mark.parametrize("case", ["k10", "kc"])
def test_oracle_direct_matches_golden(oracle, gold, case):
    zk = gold["zk"][0 if case == "k10" else 1]
    g = gold["dir_" + case]
    o = oracle.h2ddir(zk, gold["src"], gold["trg"], charges=gold["q"], dipstr=gold["d"],
                      dipvec=gold["v"], ifpgh=3)
    assert rel_l2(o["pottarg"][0], g[0]) < 1e-12
    assert rel_l2(o["gradtarg"][0], g[1:3]) < 1e-12
    assert rel_l2(o["hesstarg"][0], g[3:6]) < 1e-11


def _ref_python_inputs():
    """python/test/test_hfmm.py:17-31: n=2000 sources, 1880 targets,
    zk = 1.1, eps = 1e-5 (seeded here)."""
    rng = np.random.default_rng(7)
    n, nt = 2000, 1880
    src = rng.uniform(0, 1, (2, n))
    trg = rng.uniform(0, 1, (2, nt))
    q = rng.uniform(0, 1, n) + 1j * rng.uniform(0, 1, n)
    d = rng.uniform(0, 1, n) + 1j * rng.uniform(0, 1, n)
    v = rng.uniform(0, 1, (2, n))
    return src, trg, q, d, v


@pytest.mark.parametrize("kind", ["c", "d", "cd"])
@pytest.mark.parametrize("pg", [1, 2])
def test_oracle_hfmm_reference_python_cases(oracle, kind, pg):
    src, trg, q, d, v = _ref_python_inputs()
    zk, eps, ntest = 1.1, 1e-5, 10
    qq = q if "c" in kind else None
    dd = d if "d" in kind else None
    vv = v if "d" in kind else None
    o = oracle.hfmm2d(eps, zk, src, charges=qq, dipstr=dd, dipvec=vv, targets=trg, ifpgh=pg,
                      ifpghtarg=pg)
    assert o["ier"] == 0
    exs = oracle.h2ddir(zk, src, src[:, :ntest], charges=qq, dipstr=dd, dipvec=vv, ifpgh=pg)
    ext = oracle.h2ddir(zk, src, trg[:, :ntest], charges=qq, dipstr=dd, dipvec=vv, ifpgh=pg)
    assert rel_l2(o["pot"][0, :ntest], exs["pottarg"][0]) < eps
    assert rel_l2(o["pottarg"][0, :ntest], ext["pottarg"][0]) < eps
    if pg == 2:
        assert rel_l2(o["grad"][0, :, :ntest], exs["gradtarg"][0]) < eps
        assert rel_l2(o["gradtarg"][0, :, :ntest], ext["gradtarg"][0]) < eps


@pytest.mark.parametrize("pg", [1, 2, 3])
def test_oracle_hfmm_fortran_reference_case(oracle, pg):
    """test/helmholtz/test_hfmm2d.f:19-69: 1000 sources, 1001 targets from
    hkrand, zk = 10, eps = 0.51e-8, first 20 points against the direct sum
    with thresh 2^-51."""
    n, nt = 1000, 1001
    vals = oracle.hkrand(8 * n, seed=0).reshape(n, 8)
    src = vals[:, 0:2].T.copy()
    q = vals[:, 2] + 1j * vals[:, 3]
    d = vals[:, 4] + 1j * vals[:, 5]
    v = vals[:, 6:8].T.copy()
    trg = oracle.hkrand(2 * nt).reshape(nt, 2).T.copy()
    zk, eps = 10.0, 0.51e-8
    o = oracle.hfmm2d(eps, zk, src, charges=q, dipstr=d, dipvec=v, targets=trg, ifpgh=pg,
                      ifpghtarg=pg)
    assert o["ier"] == 0
    exs = oracle.h2ddir(zk, src, src[:, :20], charges=q, dipstr=d, dipvec=v, ifpgh=pg,
                        thresh=2.0**-51)
    ext = oracle.h2ddir(zk, src, trg[:, :20], charges=q, dipstr=d, dipvec=v, ifpgh=pg,
                        thresh=2.0**-51)
    for k in ["pot", "grad", "hess"][:pg]:
        sl = (slice(None), slice(0, 20)) if k == "pot" else (slice(None), slice(None), slice(0, 20))
        assert rel_l2(o[k][0][sl[1:]], exs[k + "targ"][0]) < eps, k
        assert rel_l2(o[k + "targ"][0][sl[1:]], ext[k + "targ"][0]) < eps, k


def test_oracle_hfmm_complex_zk_nd(oracle):
    rng = np.random.default_rng(3)
    n, nd = 3000, 2
    src = rng.uniform(0, 1, (2, n))
    q = rng.normal(size=(nd, n)) + 1j * rng.normal(size=(nd, n))
    zk, eps = 10 + 1j, 1e-9
    o = oracle.hfmm2d(eps, zk, src, charges=q, ifpgh=2, nd=nd)
    ex = oracle.h2ddir(zk, src, src[:, :30], charges=q, ifpgh=2, nd=nd)
    assert rel_l2(o["pot"][:, :30], ex["pottarg"]) < 1e-8
    assert rel_l2(o["grad"][:, :, :30], ex["gradtarg"]) < 1e-8


def test_oracle_high_frequency_returns_20(oracle):
    rng = np.random.default_rng(4)
    src = rng.uniform(0, 1, (2, 4000))
    q = rng.normal(size=4000) + 0j
    o = oracle.hfmm2d(1e-6, 500.0, src, charges=q, ifpgh=1)
    assert o["ier"] == 20


def test_hfmm_front_end_checks():
    src = np.zeros((2, 5))
    with pytest.raises(AssertionError, match="same pg must be equal to pgt"):
        fmm.hfmm2d(eps=1e-6, zk=1.0, sources=src, charges=np.ones(5, complex),
                   targets=np.zeros((2, 3)), pg=1, pgt=2)
    with pytest.raises(AssertionError, match="The first dimension of sources must be 2"):
        fmm.hfmm2d(eps=1e-6, zk=1.0, sources=np.zeros((3, 5)), charges=np.ones(5), pg=1)
    out = fmm.hfmm2d(eps=1e-6, zk=1.0, sources=src, charges=np.ones(5, complex))
    assert out.pot is None and out.ier == 0
