"""Learned cost model on the GPU: the hand-written forward / backward / Adam
kernels against the CPU oracle (oracle/mlp_oracle.py), the point
histogram against numpy, and what the trained network gains over the
lndiv2d table on held-out problems (both error-checked against the FP64
direct sum)."""
import ctypes as C

import numpy as np
import pytest

from fmm2d_b200 import _lib
from fmm2d_b200 import costmodel as cm
from oracle import mlp_oracle as M

pytestmark = pytest.mark.gpu
NIN, H1, H2 = cm.NIN, cm.H1, cm.H2


def _dev(a, dtype=None):
    import torch
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype, device="cuda")


def _stream():
    import torch
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def _data(seed, B):
    rng = np.random.default_rng(seed)
    X = rng.uniform(-1, 1, (B, NIN)).astype(np.float32)
    T = (np.sin(2 * X[:, 0]) + X[:, 1] * X[:, 2] - 0.5 * X[:, 8] ** 2).astype(np.float32)
    return X, T


def test_forward_matches_oracle(gpu):
    import torch
    X, _ = _data(1, 300)
    p = cm.CostModel.init(3).params
    y = torch.empty(300, dtype=torch.float32, device="cuda")
    tx, tp = _dev(X), _dev(p)  # keep the device copies alive during the call
    ier = C.c_int(-1)
    _lib.lib().b2fmm_mlp_forward(C.c_void_p(tx.data_ptr()), 300, NIN, H1, H2,
                                 C.c_void_p(tp.data_ptr()), C.c_void_p(y.data_ptr()),
                                 _stream(), C.byref(ier))
    assert ier.value == 0
    ref, _, _ = M.forward(X.astype(np.float64), p, NIN, H1, H2)
    assert np.max(np.abs(y.cpu().numpy() - ref)) < 1e-5 * max(1.0, np.max(np.abs(ref)))


@pytest.mark.parametrize("B", [1, 37, 1000])
def test_gradient_matches_oracle(gpu, B):
    import torch
    X, T = _data(2 + B, B)
    p = cm.CostModel.init(5).params
    n = p.size
    g = torch.empty(n, dtype=torch.float32, device="cuda")
    loss = torch.empty(1, dtype=torch.float32, device="cuda")
    tx, tt, tp = _dev(X), _dev(T), _dev(p)
    ier = C.c_int(-1)
    _lib.lib().b2fmm_mlp_gradient(C.c_void_p(tx.data_ptr()), C.c_void_p(tt.data_ptr()),
                                  B, NIN, H1, H2, C.c_void_p(tp.data_ptr()),
                                  C.c_void_p(g.data_ptr()), C.c_void_p(loss.data_ptr()),
                                  _stream(), C.byref(ier))
    assert ier.value == 0
    ref = M.gradient(X.astype(np.float64), T.astype(np.float64), p, NIN, H1, H2)
    gg = g.cpu().numpy()
    assert np.linalg.norm(gg - ref) < 1e-4 * np.linalg.norm(ref)
    assert abs(loss.item() - M.loss(X.astype(np.float64), T, p, NIN, H1, H2)) < 1e-5


def test_training_kernels_follow_oracle_adam_and_reduce_loss(gpu):
    import torch
    X, T = _data(7, 512)
    p0 = cm.CostModel.init(9).params
    tp = _dev(p0)
    steps = 400
    hist = np.zeros(steps, dtype=np.float32)
    tx, tt = _dev(X), _dev(T)
    ier = C.c_int(-1)
    _lib.lib().b2fmm_mlp_train(C.c_void_p(tx.data_ptr()), C.c_void_p(tt.data_ptr()),
                               512, NIN, H1, H2, C.c_void_p(tp.data_ptr()), steps, C.c_float(3e-3),
                               hist.ctypes.data_as(C.c_void_p), _stream(), C.byref(ier))
    assert ier.value == 0
    assert hist[-1] < 0.1 * hist[0]
    # the same Adam steps on the CPU oracle
    p, m, v = p0.astype(np.float64), np.zeros(p0.size), np.zeros(p0.size)
    for t in range(1, steps + 1):
        p, m, v = M.adam_step(p, M.gradient(X, T, p, NIN, H1, H2), m, v, t, 3e-3)
    lc = M.loss(X, T, p, NIN, H1, H2)
    lg = M.loss(X, T, tp.cpu().numpy(), NIN, H1, H2)
    assert abs(lg - lc) < 0.05 * lc + 1e-4


def test_point_histogram_matches_numpy(gpu):
    import torch
    rng = np.random.default_rng(4)
    src = rng.normal(0.3, 0.05, (20000, 2))
    trg = rng.uniform(0, 1, (5000, 2))
    h = torch.zeros(128 * 128, dtype=torch.int32, device="cuda")
    ts, tt = _dev(src), _dev(trg)
    ier = C.c_int(-1)
    _lib.lib().b2fmm_point_stats(C.c_void_p(ts.data_ptr()), C.c_int64(20000),
                                 C.c_void_p(tt.data_ptr()), C.c_int64(5000),
                                 C.c_void_p(h.data_ptr()), _stream(), C.byref(ier))
    assert ier.value == 0
    pts = np.concatenate([src, trg])
    lo, hi = pts.min(0), pts.max(0)
    w = max(hi - lo)
    c = 0.5 * (lo + hi)
    ij = np.clip(np.floor((pts - (c - 0.5 * w)) * (128.0 / w)).astype(int), 0, 127)
    ref = np.zeros((128, 128), dtype=np.int64)
    np.add.at(ref, (ij[:, 1], ij[:, 0]), 1)
    assert np.array_equal(h.cpu().numpy().reshape(128, 128), ref)


def test_trained_model_beats_table_on_held_out_problems(gpu):
    """The committed network, trained on FMM timings, on 6 held-out
    problems: its ndiv keeps every error below eps and the total time is
    not above the lndiv2d table's (it is lower on this GPU)."""
    model = cm.CostModel.load()
    assert model is not None, "costmodel_weights.json missing"
    res = cm.evaluate(model, cm.sweep_problems(6, seed0=9000, nmin=2e5, nmax=2e6))
    assert res["max_err_over_eps_mlp"] < 1.0 and res["max_err_over_eps_table"] < 1.0
    assert res["total_ms_mlp"] <= 1.05 * res["total_ms_table"]


def test_front_end_auto_ndiv(gpu):
    """ndiv='auto' through the fmm2dpy-style front end gives the same
    result as the table's leaf size, within eps."""
    import fmm2d_b200 as fmm
    from conftest import rel_l2
    src, q = cm.make_problem("mixture", 200000, 3)
    a = fmm.rfmm2d(eps=1e-6, sources=src, charges=q, pg=2, ndiv="auto")
    b = fmm.rfmm2d(eps=1e-6, sources=src, charges=q, pg=2)
    assert a.ier == 0
    assert rel_l2(a.pot, b.pot) < 1e-6 and rel_l2(a.grad, b.grad) < 1e-6


@pytest.mark.parametrize("balance", [-0.5, 0.5])
def test_level_balance_changes_the_tree_not_the_accuracy(gpu, balance):
    """A nonzero level balance builds a different tree (the leaf capacity
    varies by level) and the FMM stays within eps of the FP64 direct sum,
    for the mixed and the FP64 path."""
    import torch
    import fmm2d_b200 as fmm
    from conftest import rel_l2
    src, q = cm.make_problem("mixture", 120000, 5)
    L = _lib.lib()
    boxes = {}
    for b in (0.0, balance):
        L.b2fmm_set_stats(1)
        out = fmm.rfmm2d(eps=1e-6, sources=src, charges=q, pg=2, level_balance=b)
        L.b2fmm_set_stats(0)
        boxes[b] = _lib.get_stats()["nboxes"]
        assert out.ier == 0
        idx = np.sort(np.random.default_rng(1).choice(src.shape[1], 300, replace=False))
        ex = fmm.r2ddir(sources=src, targets=src[:, idx], charges=q, pgt=2)
        assert rel_l2(out.pot[idx], ex.pottarg) < 1e-6
        assert rel_l2(out.grad[:, idx], ex.gradtarg) < 1e-6
        o64 = fmm.rfmm2d(eps=1e-6, sources=src, charges=q, pg=2, level_balance=b,
                         precision="fp64")
        assert rel_l2(o64.pot[idx], ex.pottarg) < 1e-6
    assert boxes[balance] != boxes[0.0]
