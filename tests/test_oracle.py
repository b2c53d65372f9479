"""Pins of the CPU oracle (no GPU): golden direct sums, the reference's own
FMM-vs-direct test cases, the reference test RNG and tree invariants."""
import os

import numpy as np
import pytest

from conftest import rel_l2

GOLD = os.path.join(os.path.dirname(__file__), "golden", "laplace_direct.npz")


def test_direct_sums_match_golden(oracle):
    g = np.load(GOLD)
    src, trg = g["src"], g["trg"]
    c = oracle.c2ddir(src, trg, charges=g["q"], dipstr=g["d"], ifpgh=3)
    assert rel_l2(c["pottarg"][0], g["cpot"]) < 1e-13
    assert rel_l2(c["gradtarg"][0], g["cgrad"]) < 1e-13
    assert rel_l2(c["hesstarg"][0], g["chess"]) < 1e-13
    l = oracle.l2ddir(src, trg, charges=g["q"], dipstr=g["d"], dipvec=g["v"], ifpgh=3)
    assert rel_l2(l["pottarg"][0], g["lpot"]) < 1e-13
    assert rel_l2(l["gradtarg"][0], g["lgrad"]) < 1e-13
    assert rel_l2(l["hesstarg"][0], g["lhess"]) < 1e-13
    r = oracle.r2ddir(src, trg, charges=g["qr"], dipstr=g["dr"], dipvec=g["v"], ifpgh=3)
    assert rel_l2(r["pottarg"][0], g["rpot"]) < 1e-13
    assert rel_l2(r["gradtarg"][0], g["rgrad"]) < 1e-13
    assert rel_l2(r["hesstarg"][0], g["rhess"]) < 1e-13


def test_fmm_matches_golden(oracle):
    g = np.load(GOLD)
    src, trg = g["src"], g["trg"]
    o = oracle.lfmm2d(1e-12, src, charges=g["q"], dipstr=g["d"], dipvec=g["v"], targets=trg,
                      ifpghtarg=3, ndiv=2)
    assert rel_l2(o["pottarg"][0], g["lpot"]) < 1e-11
    assert rel_l2(o["gradtarg"][0], g["lgrad"]) < 1e-11
    assert rel_l2(o["hesstarg"][0], g["lhess"]) < 1e-10


def _ref_inputs(seed, n=2000, nt=1880):
    rng = np.random.default_rng(seed)
    src = rng.uniform(0, 1, (2, n))
    trg = rng.uniform(0, 1, (2, nt))
    q = rng.uniform(0, 1, n) + 1j * rng.uniform(0, 1, n)
    d = rng.uniform(0, 1, n) + 1j * rng.uniform(0, 1, n)
    v = rng.uniform(0, 1, (2, n))
    return src, trg, q, d, v


@pytest.mark.parametrize("kind", ["c", "d", "cd"])
@pytest.mark.parametrize("pg", [1, 2, 3])
def test_lfmm_reference_python_cases(oracle, kind, pg):
    """python/test/test_lfmm.py:18-27 parameters: n=2000, nt=1880, eps=1e-5."""
    src, trg, q, d, v = _ref_inputs(7)
    eps, ntest = 1e-5, 10
    qq = q if "c" in kind else None
    dd = d if "d" in kind else None
    vv = v if "d" in kind else None
    o = oracle.lfmm2d(eps, src, charges=qq, dipstr=dd, dipvec=vv, targets=trg, ifpgh=pg,
                      ifpghtarg=pg)
    for pts, key in ((src, ""), (trg, "targ")):
        ex = oracle.l2ddir(src, pts[:, :ntest], charges=qq, dipstr=dd, dipvec=vv, ifpgh=pg,
                           thresh=1e-14)
        num = den = 0.0
        for k in ["pot", "grad", "hess"][:pg]:
            a = o[k + key][0][..., :ntest]
            b = ex[k + "targ"][0]
            num += np.linalg.norm((a - b).ravel()) ** 2
            den += np.linalg.norm(b.ravel()) ** 2
        assert np.sqrt(num / den) < eps


def test_cfmm_reference_python_case(oracle):
    """python/test/test_cfmm.py: real charges, Re(pot) compared (cauchy=1)."""
    rng = np.random.default_rng(3)
    n, ntest, eps = 2000, 100, 1e-5
    src = rng.uniform(0, 1, (2, n))
    q = rng.uniform(0, 1, n) + 0j
    d = rng.uniform(0, 1, n) + 1j * rng.uniform(0, 1, n)
    o = oracle.cfmm2d(eps, src, charges=q, dipstr=d, ifpgh=3)
    ex = oracle.c2ddir(src, src[:, :ntest], charges=q, dipstr=d, ifpgh=3, thresh=1e-14)
    num = np.linalg.norm(o["pot"][0, :ntest].real - ex["pottarg"][0].real) ** 2
    den = np.linalg.norm(ex["pottarg"][0].real) ** 2
    for k in ("grad", "hess"):
        num += np.linalg.norm(o[k][0, :ntest] - ex[k + "targ"][0]) ** 2
        den += np.linalg.norm(ex[k + "targ"][0]) ** 2
    assert np.sqrt(num / den) < eps


def test_rfmm_nd2(oracle):
    rng = np.random.default_rng(4)
    n, nd, eps = 3000, 2, 1e-6
    src = rng.uniform(0, 1, (2, n))
    q = rng.normal(size=(nd, n))
    o = oracle.rfmm2d(eps, src, charges=q, ifpgh=2, nd=nd)
    ex = oracle.r2ddir(src, src[:, :50], charges=q, ifpgh=2, nd=nd, thresh=1e-14)
    assert rel_l2(o["pot"][:, :50], ex["pottarg"]) < eps
    assert rel_l2(o["grad"][:, :, :50], ex["gradtarg"]) < eps


def test_hkrand_restates_dlaran(oracle):
    # first draw from seed (0,0,0,1): limbs (494, 322, 2508, 2549) / 4096
    r = 1.0 / 4096
    first = r * (494 + r * (322 + r * (2508 + r * 2549)))
    x = oracle.hkrand(3, seed=0)
    assert x[0] == first
    assert np.all((x > 0) & (x < 1))


def test_lfmm_fortran_reference_case(oracle):
    """test/laplace/test_lfmm2d.f:30-101: 10000 sources/targets from hkrand,
    eps=0.5e-6, first 20 points against the direct sum (thresh 1e-14)."""
    n = 10000
    oracle.hkrand(0, seed=0)
    # the Fortran loop draws x, y, Re q, Im q, Re d, Im d, v1, v2 per source
    vals = oracle.hkrand(8 * n, seed=0).reshape(n, 8)
    src = vals[:, 0:2].T.copy()
    q = vals[:, 2] + 1j * vals[:, 3]
    d = vals[:, 4] + 1j * vals[:, 5]
    v = vals[:, 6:8].T.copy()
    trg = oracle.hkrand(2 * n).reshape(n, 2).T.copy()
    eps = 0.5e-6
    o = oracle.lfmm2d(eps, src, charges=q, dipstr=d, dipvec=v, targets=trg, ifpgh=2, ifpghtarg=2)
    exs = oracle.l2ddir(src, src[:, :20], charges=q, dipstr=d, dipvec=v, ifpgh=2, thresh=1e-14)
    ext = oracle.l2ddir(src, trg[:, :20], charges=q, dipstr=d, dipvec=v, ifpgh=2, thresh=1e-14)
    assert rel_l2(o["pot"][0, :20], exs["pottarg"][0]) < eps
    assert rel_l2(o["grad"][0, :, :20], exs["gradtarg"][0]) < eps
    assert rel_l2(o["pottarg"][0, :20], ext["pottarg"][0]) < eps
    assert rel_l2(o["gradtarg"][0, :, :20], ext["gradtarg"][0]) < eps


def _leaf_levels_adjacent_ok(t):
    """Level restriction: touching leaves differ by at most one level."""
    leaves = np.nonzero(t["nchild"] == 0)[0]
    for b in leaves:
        for j in t["list1"][b][: t["nlist1"][b]]:
            if abs(int(t["ilevel"][b]) - int(t["ilevel"][j])) > 1:
                return False
    return True


@pytest.mark.parametrize("dist", ["uniform", "cluster", "curve"])
def test_tree_invariants(oracle, dist):
    rng = np.random.default_rng(11)
    n = 5000
    if dist == "uniform":
        src = rng.uniform(0, 1, (2, n))
    elif dist == "cluster":
        src = np.concatenate([rng.normal(0.3, 1e-3, (2, n // 2)), rng.uniform(0, 1, (2, n // 2))], 1)
    else:
        th = rng.uniform(0, 2 * np.pi, n)
        r = 0.3 * (1 + 0.2 * np.cos(5 * th))
        src = np.stack([0.5 + r * np.cos(th), 0.5 + r * np.sin(th)])
    t = oracle.tree(src, None, 0, 15)
    nb = t["nboxes"]
    assert t["laddr"][0].tolist() == [0, 0]
    assert t["laddr"][-1][1] == nb - 1
    # every source in exactly one leaf; children partition the parent
    leaves = t["nchild"] == 0
    counts = t["isrcse"][:, 1] - t["isrcse"][:, 0]
    assert counts[leaves].sum() == n
    assert sorted(t["isrc"].tolist()) == list(range(n))
    for b in np.nonzero(~leaves)[0]:
        ch = t["ichild"][b]
        assert counts[ch].sum() == counts[b]
        assert t["isrcse"][ch[0], 0] == t["isrcse"][b, 0]
    assert _leaf_levels_adjacent_ok(t)
    # lists within their fixed widths and symmetric list 1 between leaves
    assert t["nlist1"].max() <= 13 and t["nlist2"].max() <= 27
    assert t["nlist3"].max() <= 20 and t["nlist4"].max() <= 5
    for b in np.nonzero(leaves)[0][:200]:
        for j in t["list1"][b][: t["nlist1"][b]]:
            assert b in t["list1"][j][: t["nlist1"][j]]
