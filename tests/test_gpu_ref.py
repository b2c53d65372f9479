"""The CUDA path against the reference itself.

``ref`` runs the reference's own Fortran (translated to C, oracle/ref.py).
The device tree must equal the reference's tree array for array, at the
headline size too (4M points of the 16-Gaussian mixture, 20 levels); FP64
FMM results must equal the reference's to round-off (same tree, same
expansion orders; 1e-11 relative l2 for Laplace, 1e-10 for Helmholtz), on
the reference's own test inputs, on deep clustered trees (lists 3 and 4
exercised) and through the reference-named host entry points of the C ABI.
The mixed-precision path must stay within the requested eps of the
reference's output.
"""
import ctypes as C

import numpy as np
import pytest
import torch

import fmm2d_b200 as fmm
from conftest import rel_l2
from gpu_util import device_tree
from test_ref_pin import gauss16, graded_curve, hk_inputs

pytestmark = pytest.mark.gpu
TOL_LAP = 1e-11
TOL_HELM = 1e-10


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def test_tree_headline_4m_vs_reference(gpu, ref):
    """The C2 workload's tree: 4,000,000 points of the 16-Gaussian mixture
    (sigma log-uniform in [1e-4, 1e-1], seed 1), ndiv 15."""
    import bench
    src = bench.make_inputs(4_000_000, seed=1)[0]
    a = ref.tree(src, None, 0, 15)
    b = device_tree(src, None, 0, 15)
    assert (a["nlevels"], a["nboxes"]) == (b["nlevels"], b["nboxes"])
    assert a["nlevels"] >= 19
    for k in ["laddr", "ilevel", "iparent", "nchild", "ichild", "ncoll", "coll", "isrcse",
              "nlist1", "list1", "nlist2", "list2", "nlist3", "list3", "nlist4", "list4"]:
        assert np.array_equal(a[k], b[k]), k
    assert np.array_equal(a["centers"].view(np.int64), b["centers"].view(np.int64))
    assert np.array_equal(a["boxsize"], b["boxsize"])
    # points within each leaf: the same sets (the order inside a leaf may differ)
    se = a["isrcse"]
    key_a = np.empty(src.shape[1], np.int64)
    key_b = np.empty(src.shape[1], np.int64)
    leaves = np.nonzero(a["nchild"] == 0)[0]
    for lb in leaves:
        s, e = se[lb]
        key_a[a["isrc"][s:e]] = lb
        key_b[b["isrc"][s:e]] = lb
    assert np.array_equal(key_a, key_b)


@pytest.mark.parametrize("kind", ["c", "d", "cd"])
@pytest.mark.parametrize("pg", [1, 2, 3])
def test_lfmm_fp64_reference_inputs(gpu, ref, kind, pg):
    """test/laplace/test_lfmm2d.f:30-101: 10000 hkrand sources and targets,
    eps 0.5e-6, every output compared with the reference's."""
    src, trg, q, d, v = hk_inputs(ref, 10000, 10000)
    kw = dict(charges=q if "c" in kind else None, dipstr=d if "d" in kind else None,
              dipvec=v if "d" in kind else None, targets=trg)
    out = fmm.lfmm2d(eps=0.5e-6, sources=src, pg=pg, pgt=pg, precision="fp64", **kw)
    r = ref.lfmm2d(0.5e-6, src, ifpgh=pg, ifpghtarg=pg, **kw)
    assert out.ier == 0 and r["ier"] == 0
    for k in ["pot", "grad", "hess"][:pg]:
        assert rel_l2(getattr(out, k), r[k][0]) < TOL_LAP, k
        assert rel_l2(getattr(out, k + "targ"), r[k + "targ"][0]) < TOL_LAP, k + "targ"


@pytest.mark.parametrize("eps", [1e-3, 1e-6, 1e-9])
def test_lfmm_fp64_clustered_vs_reference(gpu, ref, eps):
    """250,000 points of the 16-Gaussian mixture (deep tree: lists 3 and 4,
    i.e. M2P and P2L, carry real work), charges + dipoles, pg 2."""
    rng = np.random.default_rng(21)
    n = 250_000
    src = gauss16(n, 22)
    q = rng.normal(size=n) + 1j * rng.normal(size=n)
    d = rng.normal(size=n) + 0j
    ph = rng.uniform(0, 2 * np.pi, n)
    v = np.stack([np.cos(ph), np.sin(ph)])
    out = fmm.lfmm2d(eps=eps, sources=src, charges=q, dipstr=d, dipvec=v, pg=2,
                     precision="fp64")
    r = ref.lfmm2d(eps, src, charges=q, dipstr=d, dipvec=v, ifpgh=2)
    assert rel_l2(out.pot, r["pot"][0]) < TOL_LAP
    assert rel_l2(out.grad, r["grad"][0]) < TOL_LAP
    t = ref.tree(src, None, 0, ref.lndiv2d(eps, n, 0, 1, 1, 2, 0)[0])
    assert t["nlist3"].sum() > 0 and t["nlist4"].sum() > 0


@pytest.mark.parametrize("kind", ["c", "d", "cd"])
@pytest.mark.parametrize("pg", [1, 2, 3])
def test_rfmm_sources_vs_reference(gpu, ref, kind, pg):
    """rfmm2d at the sources (src/laplace/rfmm2d.f:27-215), pg 1-3."""
    rng = np.random.default_rng(30 + pg)
    n = 20000
    src = gauss16(n, 31)
    q = rng.normal(size=n)
    d = rng.normal(size=n)
    v = rng.normal(size=(2, n))
    kw = dict(charges=q if "c" in kind else None, dipstr=d if "d" in kind else None,
              dipvec=v if "d" in kind else None)
    out = fmm.rfmm2d(eps=1e-6, sources=src, pg=pg, precision="fp64", **kw)
    r = ref.rfmm2d(1e-6, src, ifpgh=pg, **kw)
    for k in ["pot", "grad", "hess"][:pg]:
        assert rfmm_ok(getattr(out, k), r[k][0]), k


def rfmm_ok(a, b):
    return rel_l2(a, b) < TOL_LAP


def test_rfmm_uniform_100k_pg2_vs_reference(gpu, ref):
    """The plain-rfmm2d workload: 100,000 uniform sources, real N(0,1)
    charges, eps 1e-6, pg 2, no targets."""
    rng = np.random.default_rng(0)
    src = rng.uniform(0, 1, (2, 100_000))
    q = rng.normal(size=100_000)
    out = fmm.rfmm2d(eps=1e-6, sources=src, charges=q, pg=2, precision="fp64")
    r = ref.rfmm2d(1e-6, src, charges=q, ifpgh=2)
    assert rel_l2(out.pot, r["pot"][0]) < TOL_LAP
    assert rel_l2(out.grad, r["grad"][0]) < TOL_LAP


def test_host_entry_points_vs_reference(gpu, ref):
    """b2fmm_lfmm2d / b2fmm_rfmm2d / b2fmm_cfmm2d_ndiv / b2fmm_hfmm2d with host
    pointers, argument for argument as the reference's lfmm2d_ / rfmm2d_ /
    cfmm2d_ndiv_ / hfmm2d_ (iper included)."""
    from fmm2d_b200 import _lib
    L = _lib.lib()
    rng = np.random.default_rng(40)
    n, nt, nd = 6000, 2500, 2
    src = gauss16(n, 41)
    trg = rng.uniform(0, 1, (2, nt))
    S, T = np.ascontiguousarray(src.T), np.ascontiguousarray(trg.T)
    qc = rng.normal(size=(nd, n)) + 1j * rng.normal(size=(nd, n))
    dc = rng.normal(size=(nd, n)) + 1j * rng.normal(size=(nd, n))
    v = rng.normal(size=(nd, 2, n))
    Q, D = np.ascontiguousarray(qc.T), np.ascontiguousarray(dc.T)
    V = np.ascontiguousarray(v.transpose(2, 1, 0))
    ier = C.c_int(-1)

    def outs(dt, k, m):
        return [np.zeros((m,) + ((kk, nd) if kk > 1 else (nd,)), dt) for kk in k]

    # lfmm2d: pot (nd,n), grad (nd,2,n), hess (nd,3,n)
    ps, gs, hs = outs(np.complex128, (1, 2, 3), n)
    pt, gt, ht = outs(np.complex128, (1, 2, 3), nt)
    L.b2fmm_lfmm2d(nd, 1e-9, n, _p(S), 1, _p(Q), 1, _p(D), _p(V), 0, 3, _p(ps), _p(gs), _p(hs),
                   nt, _p(T), 3, _p(pt), _p(gt), _p(ht), C.byref(ier))
    assert ier.value == 0
    r = ref.lfmm2d(1e-9, src, charges=qc, dipstr=dc, dipvec=v, targets=trg, ifpgh=3,
                   ifpghtarg=3, nd=nd)
    for a, k in ((ps, "pot"), (pt, "pottarg")):
        assert rel_l2(a.T, r[k]) < TOL_LAP, k
    for a, k in ((gs, "grad"), (hs, "hess"), (gt, "gradtarg"), (ht, "hesstarg")):
        assert rel_l2(a.transpose(2, 1, 0), r[k]) < TOL_LAP, k
    # rfmm2d: real densities
    qr, dr = np.ascontiguousarray(qc.real.T), np.ascontiguousarray(dc.real.T)
    ps, gs, hs = outs(np.float64, (1, 2, 3), n)
    L.b2fmm_rfmm2d(nd, 1e-9, n, _p(S), 1, _p(qr), 1, _p(dr), _p(V), 0, 2, _p(ps), _p(gs), _p(hs),
                   0, None, 0, None, None, None, C.byref(ier))
    assert ier.value == 0
    r = ref.rfmm2d(1e-9, src, charges=qc.real, dipstr=dc.real, dipvec=v, ifpgh=2, nd=nd)
    assert rel_l2(ps.T, r["pot"]) < TOL_LAP
    assert rel_l2(gs.transpose(2, 1, 0), r["grad"]) < TOL_LAP
    # cfmm2d_ndiv: caller's leaf size, phase times out
    pc = [np.zeros((m, nd), np.complex128) for m in (n, n, n, nt, nt, nt)]
    ti = np.zeros(8)
    L.b2fmm_cfmm2d_ndiv(nd, 1e-6, n, _p(S), 1, _p(Q), 1, _p(D), 0, 2, _p(pc[0]), _p(pc[1]),
                        _p(pc[2]), nt, _p(T), 2, _p(pc[3]), _p(pc[4]), _p(pc[5]), 30, 0, 1,
                        _p(ti), C.byref(ier))
    assert ier.value == 0
    r = ref.cfmm2d(1e-6, src, charges=qc, dipstr=dc, targets=trg, ifpgh=2, ifpghtarg=2, nd=nd,
                   ndiv=30)
    for a, k in ((pc[0], "pot"), (pc[1], "grad"), (pc[3], "pottarg"), (pc[4], "gradtarg")):
        assert rel_l2(a.T, r[k]) < 1e-6, k  # auto precision at eps 1e-6 is the mixed path
    assert ti.sum() > 0
    # hfmm2d
    ps, gs, hs = outs(np.complex128, (1, 2, 3), n)
    pt, gt, ht = outs(np.complex128, (1, 2, 3), nt)
    L.b2fmm_hfmm2d(nd, 1e-9, 20.0, 0.0, n, _p(S), 1, _p(Q), 1, _p(D), _p(V), 0, 2, _p(ps),
                   _p(gs), _p(hs), nt, _p(T), 2, _p(pt), _p(gt), _p(ht), C.byref(ier))
    assert ier.value == 0
    r = ref.hfmm2d(1e-9, 20.0, src, charges=qc, dipstr=dc, dipvec=v, targets=trg, ifpgh=2,
                   ifpghtarg=2, nd=nd)
    for a, k in ((ps, "pot"), (pt, "pottarg")):
        assert rel_l2(a.T, r[k]) < TOL_HELM, k
    for a, k in ((gs, "grad"), (gt, "gradtarg")):
        assert rel_l2(a.transpose(2, 1, 0), r[k]) < TOL_HELM, k


@pytest.mark.parametrize("zk", [10.0, 3 + 0.5j, 500.0])
@pytest.mark.parametrize("pg", [1, 2, 3])
def test_hfmm_reference_inputs(gpu, ref, zk, pg):
    """test/helmholtz/test_hfmm2d.f:19-51 inputs (1000 sources, 1001 targets),
    eps 0.51e-8, through the reference-named host entry b2fmm_hfmm2d (the
    python front end, like fmm2dpy's, stops at pg 2).  zk = 500 is
    test/helmholtz/test_hfmm2d_hf.f: boxes of 40 and 20 wavelengths at levels
    1 and 2 take the wideband (signature) translations."""
    from fmm2d_b200 import _lib
    src, trg, q, d, v = hk_inputs(ref, 1000, 1001)
    n, nt = src.shape[1], trg.shape[1]
    S, T = np.ascontiguousarray(src.T), np.ascontiguousarray(trg.T)
    V = np.ascontiguousarray(v.T)
    o = [np.zeros((m,) + sh, np.complex128) for m, sh in
         ((n, ()), (n, (2,)), (n, (3,)), (nt, ()), (nt, (2,)), (nt, (3,)))]
    ier = C.c_int(-1)
    zk = complex(zk)
    _lib.lib().b2fmm_hfmm2d(1, 0.51e-8, zk.real, zk.imag, n, _p(S), 1, _p(q), 1, _p(d), _p(V),
                            0, pg, *[_p(a) for a in o[:3]], nt, _p(T), pg,
                            *[_p(a) for a in o[3:]], C.byref(ier))
    assert ier.value == 0
    r = ref.hfmm2d(0.51e-8, zk, src, charges=q, dipstr=d, dipvec=v, targets=trg, ifpgh=pg,
                   ifpghtarg=pg)
    for i, k in enumerate(["pot", "grad", "hess"][:pg]):
        assert rel_l2(o[i].T, r[k][0]) < TOL_HELM, k
        assert rel_l2(o[3 + i].T, r[k + "targ"][0]) < TOL_HELM, k + "targ"
    if pg <= 2:
        out = fmm.hfmm2d(eps=0.51e-8, zk=zk, sources=src, charges=q, dipstr=d, dipvec=v,
                         targets=trg, pg=pg, pgt=pg)
        assert out.ier == 0
        assert rel_l2(out.pottarg, r["pottarg"][0]) < TOL_HELM


def test_hfmm_curve_targets_vs_reference(gpu, ref):
    """The Helmholtz workload's shape at a reduced size: zk 40, sources on the
    curve r = 0.3 (1 + 0.2 cos 5t), uniform targets, eps 1e-9, pgt 2."""
    rng = np.random.default_rng(50)
    ns, nt = 60000, 30000
    th = rng.uniform(0, 2 * np.pi, ns)
    r0 = 0.3 * (1 + 0.2 * np.cos(5 * th))
    src = np.stack([0.5 + r0 * np.cos(th), 0.5 + r0 * np.sin(th)])
    trg = rng.uniform(0, 1, (2, nt))
    q = rng.normal(size=ns) + 1j * rng.normal(size=ns)
    d = rng.normal(size=ns) + 1j * rng.normal(size=ns)
    ph = rng.uniform(0, 2 * np.pi, ns)
    v = np.stack([np.cos(ph), np.sin(ph)])
    out = fmm.hfmm2d(eps=1e-9, zk=40.0, sources=src, charges=q, dipstr=d, dipvec=v, targets=trg,
                     pgt=2)
    r = ref.hfmm2d(1e-9, 40.0, src, charges=q, dipstr=d, dipvec=v, targets=trg, ifpghtarg=2)
    assert rel_l2(out.pottarg, r["pottarg"][0]) < TOL_HELM
    assert rel_l2(out.gradtarg, r["gradtarg"][0]) < TOL_HELM


@pytest.mark.parametrize("eps", [1e-3, 1e-6])
def test_mixed_within_eps_of_reference(gpu, ref, eps):
    """The mixed-precision path (FP32 near field, tensor-core M2L) on a
    clustered cloud: within eps of the reference's FP64 output."""
    rng = np.random.default_rng(60)
    n = 300_000
    src = gauss16(n, 61)
    q = rng.normal(size=n) + 1j * rng.normal(size=n)
    d = rng.normal(size=n) + 0j
    ph = rng.uniform(0, 2 * np.pi, n)
    v = np.stack([np.cos(ph), np.sin(ph)])
    dev = torch.device("cuda:0")
    T = lambda a: torch.as_tensor(a, device=dev)
    out = fmm.lfmm2d(eps=eps, sources=T(src), charges=T(q), dipstr=T(d), dipvec=T(v), pg=2,
                     precision="mixed")
    r = ref.lfmm2d(eps, src, charges=q, dipstr=d, dipvec=v, ifpgh=2)
    num = (np.linalg.norm(out.pot.cpu().numpy() - r["pot"][0]) ** 2
           + np.linalg.norm((out.grad.cpu().numpy() - r["grad"][0]).ravel()) ** 2)
    den = np.linalg.norm(r["pot"][0]) ** 2 + np.linalg.norm(r["grad"][0].ravel()) ** 2
    assert np.sqrt(num / den) < eps


@pytest.mark.parametrize("precision", ["fp64", "auto"])
def test_batch_graph_vs_reference(gpu, ref, precision):
    """Ten uneven cfmm2d problems (nd 1, 2, 4) evaluated by one captured graph
    launch, each against the reference's cfmm2d (FP64 plans to round-off,
    mixed-precision plans within eps)."""
    from fmm2d_b200.plan import BatchGraph, Plan
    rng = np.random.default_rng(70)
    probs = []
    for i in range(10):
        n = int(10 ** rng.uniform(np.log10(2000), np.log10(50000)))
        nd = [1, 2, 4][i % 3]
        src = rng.uniform(0, 1, (2, n)) if i % 2 else gauss16(n, 71 + i)
        q = rng.normal(size=(nd, n)) + 1j * rng.normal(size=(nd, n))
        probs.append((src, q))
    dev = lambda a: torch.as_tensor(np.ascontiguousarray(a), device="cuda")
    plans = [Plan("cfmm2d", eps=1e-6, sources=dev(s.T), charges=True, pg=1, nd=q.shape[0],
                  precision=precision) for s, q in probs]
    g = BatchGraph(plans, charges=[dev(q.T) for _, q in probs], nbranch=4)
    g.launch()
    torch.cuda.synchronize()
    assert g.status() == 0
    tol = TOL_LAP if precision == "fp64" else 1e-6
    for (src, q), o in zip(probs, g.outs):
        r = ref.cfmm2d(1e-6, src, charges=q, ifpgh=1, nd=q.shape[0])
        assert rel_l2(o["pot"].cpu().numpy().T, r["pot"]) < tol
    g.close()
    for p in plans:
        p.close()


@pytest.mark.parametrize("case", ["uniform", "curve"])
def test_hfmm_wideband_vs_reference(gpu, ref, case):
    """Larger wideband problems: wideband and tabulated levels in one tree,
    nd = 2, sources and targets, pg = pgt = 2."""
    rng = np.random.default_rng(60)
    if case == "uniform":
        ns, nt, zk = 40000, 10000, 600.0
        src = rng.uniform(0, 1, (2, ns))
    else:
        ns, nt, zk = 60000, 10000, 150.0 + 2.0j
        th = rng.uniform(0, 2 * np.pi, ns)
        r0 = 0.3 * (1 + 0.2 * np.cos(5 * th))
        src = np.stack([0.5 + r0 * np.cos(th), 0.5 + r0 * np.sin(th)])
    trg = rng.uniform(0, 1, (2, nt))
    nd = 2
    q = rng.normal(size=(nd, ns)) + 1j * rng.normal(size=(nd, ns))
    d = rng.normal(size=(nd, ns)) + 1j * rng.normal(size=(nd, ns))
    ph = rng.uniform(0, 2 * np.pi, (nd, ns))
    v = np.stack([np.cos(ph), np.sin(ph)], axis=1)
    out = fmm.hfmm2d(eps=1e-9, zk=zk, sources=src, charges=q, dipstr=d, dipvec=v, targets=trg,
                     pg=2, pgt=2, nd=nd)
    assert out.ier == 0
    r = ref.hfmm2d(1e-9, zk, src, charges=q, dipstr=d, dipvec=v, targets=trg, ifpgh=2,
                   ifpghtarg=2, nd=nd)
    for k in ("pot", "grad", "pottarg", "gradtarg"):
        assert rel_l2(getattr(out, k), r[k]) < TOL_HELM, k
