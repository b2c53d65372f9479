"""Tensor-core (tcgen05) M2L: the tile path against an FP64 GEMM, and the
mixed-precision FMM with the tensor-core M2L against the CUDA-core M2L, the
FP64 FMM and the direct sum."""
import ctypes as C

import numpy as np
import pytest

import fmm2d_b200 as fmm
from conftest import rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture
def tc_on():
    L = fmm._lib.lib()
    L.b2fmm_set_m2l_tensor_cores(1)
    yield L
    L.b2fmm_set_m2l_tensor_cores(1)


@pytest.mark.parametrize("k", [8, 16, 24, 32])
@pytest.mark.parametrize("n", [16, 32])
def test_tc_gemm_probe_split_tf32(gpu, k, n):
    """D = A B^T through the shared-memory layout, split-TF32 tcgen05.mma and
    tcgen05.ld of the M2L kernel: FP32-level accuracy."""
    import torch
    rng = np.random.default_rng(k * 100 + n)
    a = rng.normal(size=(128, k)).astype(np.float32)
    b = rng.normal(size=(n, k)).astype(np.float32)
    ta = torch.as_tensor(a, device=gpu)
    tb = torch.as_tensor(b, device=gpu)
    td = torch.full((128, n), np.nan, dtype=torch.float32, device=gpu)
    ier = C.c_int(-1)
    fmm._lib.lib().b2fmm_tc_gemm_probe(C.c_void_p(ta.data_ptr()), C.c_void_p(tb.data_ptr()), k, n,
                                       C.c_void_p(td.data_ptr()),
                                       C.c_void_p(torch.cuda.current_stream().cuda_stream),
                                       C.byref(ier))
    assert ier.value == 0
    d = td.cpu().numpy().astype(np.float64)
    ref = a.astype(np.float64) @ b.astype(np.float64).T
    scale = np.abs(a).astype(np.float64) @ np.abs(b).astype(np.float64).T
    assert np.all(np.isfinite(d))
    assert np.max(np.abs(d - ref) / scale) < 2e-6


def _cloud(seed, n):
    rng = np.random.default_rng(seed)
    c = rng.uniform(0, 1, (2, 8))
    sig = 10 ** rng.uniform(-3, -1, 8)
    k = rng.integers(0, 8, n)
    src = c[:, k] + sig[k] * rng.normal(size=(2, n))
    q = rng.normal(size=n) + 1j * rng.normal(size=n)
    d = rng.normal(size=n) + 1j * rng.normal(size=n)
    v = rng.uniform(-1, 1, (2, n))
    return src, q, d, v


@pytest.mark.parametrize("eps", [1e-3, 1e-6])
@pytest.mark.parametrize("nd", [1, 3])
def test_mixed_tc_matches_cuda_core_m2l(gpu, tc_on, eps, nd):
    src, q, d, v = _cloud(3, 40000)
    if nd > 1:
        rng = np.random.default_rng(4)
        q = rng.normal(size=(nd, 40000)) + 1j * rng.normal(size=(nd, 40000))
        d = v = None
    kw = dict(eps=eps, sources=src, charges=q, dipstr=d, dipvec=v, pg=2, nd=nd,
              precision="mixed")
    out_tc = fmm.lfmm2d(**kw)
    tc_on.b2fmm_set_m2l_tensor_cores(0)
    out_cc = fmm.lfmm2d(**kw)
    tc_on.b2fmm_set_m2l_tensor_cores(1)
    out_64 = fmm.lfmm2d(**{**kw, "precision": "fp64"})
    assert out_tc.ier == 0 and out_cc.ier == 0
    # both mixed engines agree with the FP64 FMM far below eps
    assert rel_l2(out_tc.pot, out_64.pot) < 1e-6
    assert rel_l2(out_tc.grad, out_64.grad) < 1e-6
    assert rel_l2(out_tc.pot, out_cc.pot) < 1e-6


def test_mixed_tc_vs_direct_4_densities(gpu, tc_on):
    """nd = 2 complex -> 4 Cauchy densities per chunk (ND = 4 tiles)."""
    src, q, d, v = _cloud(5, 60000)
    rng = np.random.default_rng(6)
    q2 = rng.normal(size=(2, 60000)) + 1j * rng.normal(size=(2, 60000))
    out = fmm.lfmm2d(eps=1e-6, sources=src, charges=q2, pg=2, nd=2, precision="mixed")
    ex = fmm.l2ddir(sources=src, targets=src[:, :500], charges=q2, pgt=2, nd=2)
    assert rel_l2(out.pot[:, :500], ex.pottarg) < 1e-6
    assert rel_l2(out.grad[:, :, :500], ex.gradtarg) < 1e-6


@pytest.mark.parametrize("eps", [0.1, 0.01, 1e-3, 1e-4, 1e-6, 3e-7])
@pytest.mark.parametrize("kind", ["cfmm_nd1", "lfmm_nd4"])
def test_tc_every_expansion_length(gpu, tc_on, eps, kind):
    """All operator sizes of the tensor-core kernel (P = 4, 7, 10, 13, 19 ->
    KH = 4, 8, 12, 16, 20 coefficients per row) with 1 and 8 densities per
    row group; P = 21 (eps 3e-7) runs the CUDA-core M2L.
    The tensor-core result equals the CUDA-core FP32 M2L and the FP64 FMM to
    FP32 accuracy."""
    src, q, d, v = _cloud(11, 30000)
    if kind == "cfmm_nd1":
        f = fmm.cfmm2d
        kw = dict(eps=eps, sources=src, charges=q, dipstr=d, pg=2)
    else:
        rng = np.random.default_rng(12)
        q4 = rng.normal(size=(4, 30000)) + 1j * rng.normal(size=(4, 30000))
        f = fmm.lfmm2d
        kw = dict(eps=eps, sources=src, charges=q4, pg=2, nd=4)
    out_tc = f(**kw, precision="mixed")
    tc_on.b2fmm_set_m2l_tensor_cores(0)
    out_cc = f(**kw, precision="mixed")
    tc_on.b2fmm_set_m2l_tensor_cores(1)
    out_64 = f(**kw, precision="fp64")
    assert out_tc.ier == 0 and out_cc.ier == 0 and out_64.ier == 0
    assert rel_l2(out_tc.pot, out_cc.pot) < 1e-6
    assert rel_l2(out_tc.grad, out_cc.grad) < 1e-6
    assert rel_l2(out_tc.pot, out_64.pot) < 1e-6


def test_tc_super_tiles(gpu, tc_on):
    """1.2M points: the targets are interleaved into super-tiles of several
    targets per row group (T > 1), each row walks its targets' list-2
    entries back to back and flushes a target's locals after its last
    entry.  The result equals the FP64 FMM to FP32 accuracy, and the steps
    issued stay within 2 % of the translations x densities / 128 rows.
    Accuracy against the CUDA-core FP32 M2L: the tensor cores truncate each
    MMA's FP32 sum, and an accumulator kept across the offsets of a tile
    made the error ~5x that of the FP32 M2L; per-step products summed with
    round-to-nearest keep it within 2x."""
    n = 1_200_000
    src, q, d, v = _cloud(21, n)
    kw = dict(eps=1e-6, sources=src, charges=q, dipstr=d, dipvec=v, pg=2)
    L = tc_on
    L.b2fmm_set_stats(1)
    out_tc = fmm.lfmm2d(**kw, precision="mixed")
    L.b2fmm_set_stats(0)
    st = fmm._lib.get_stats()
    L.b2fmm_set_m2l_tensor_cores(0)
    out_cc = fmm.lfmm2d(**kw, precision="mixed")
    L.b2fmm_set_m2l_tensor_cores(1)
    out_64 = fmm.lfmm2d(**kw, precision="fp64")
    assert out_tc.ier == 0 and out_cc.ier == 0 and out_64.ier == 0
    assert rel_l2(out_tc.pot, out_64.pot) < 1e-6
    assert rel_l2(out_tc.grad, out_64.grad) < 1e-6
    for k in ("pot", "grad"):
        e_tc = rel_l2(getattr(out_tc, k), getattr(out_64, k))
        e_cc = rel_l2(getattr(out_cc, k), getattr(out_64, k))
        assert e_tc < 2.0 * e_cc + 1e-9, (k, e_tc, e_cc)
    rows = st["m2l_pairs"] * 2  # lfmm2d: 2 Cauchy densities per target
    assert st["m2l_tc_steps"] >= rows / 128
    assert st["m2l_tc_steps"] <= 1.02 * rows / 128 + 4 * 148
