"""The allocation-free direct sum (b2fmm_lap_direct_noalloc_dev) against the
allocating one (b2fmm_lap_direct_dev), through the C ABI.

The entry point exists for callers that cannot allocate device memory while
they call us (a device already reserved by another framework's allocator,
latency-critical loops, fixed memory plans); its scratch lives in a static
device array.  Two calls in a row must both match, and a size beyond the
static array must be rejected without touching the outputs.  Collected last
so that a stop-at-first-failure run has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
TOL = 1e-13  # same tolerance as the other direct-sum tests


def _inputs(dev, kind, ns, nt, nd, seed):
    import torch
    rng = np.random.default_rng(seed)
    dt = torch.float64 if kind == 2 else torch.complex128
    mk = (lambda *s: rng.normal(size=s)) if kind == 2 else (
        lambda *s: rng.normal(size=s) + 1j * rng.normal(size=s))
    T = lambda a, t=torch.float64: torch.as_tensor(np.ascontiguousarray(a), device=dev).to(t)
    src = T(rng.uniform(0, 1, (ns, 2)))
    trg = T(rng.uniform(0, 1, (nt, 2)))
    q = T(mk(ns, nd), dt)
    d = T(mk(ns, nd), dt)
    v = T(rng.uniform(-1, 1, (ns, 2, nd)))
    return src, trg, q, d, v


def _outputs(dev, kind, nt, nd):
    import torch
    dt = torch.float64 if kind == 2 else torch.complex128
    gk, hk = (1, 1) if kind == 0 else (2, 3)
    return (torch.full((nt, nd), 7.0, dtype=dt, device=dev),
            torch.full((nt, gk, nd), 7.0, dtype=dt, device=dev),
            torch.full((nt, hk, nd), 7.0, dtype=dt, device=dev))


def _call(fn, kind, nd, src, q, d, v, trg, outs, stream):
    p = lambda t: C.c_void_p(t.data_ptr())
    ier = C.c_int(-1)
    fn(kind, nd, C.c_int64(src.shape[0]), p(src), p(q), p(d), p(v) if kind else None,
       C.c_int64(trg.shape[0]), p(trg), 3, p(outs[0]), p(outs[1]), p(outs[2]),
       C.c_double(1e-16), C.c_void_p(stream), C.byref(ier))
    return ier.value


def _rel(a, b):
    return float((a - b).abs().max() / b.abs().max())


@pytest.mark.parametrize("kind", [0, 1, 2])
def test_noalloc_matches_allocating_twice(gpu, kind):
    import torch
    from fmm2d_b200 import _lib
    L = _lib.lib()
    stream = torch.cuda.current_stream(gpu).cuda_stream
    nd = 2
    src, trg, q, d, v = _inputs(gpu, kind, 5000, 3000, nd, seed=kind)
    ref = _outputs(gpu, kind, 3000, nd)
    assert _call(L.b2fmm_lap_direct_dev, kind, nd, src, q, d, v, trg, ref, stream) == 0
    for _ in range(2):
        got = _outputs(gpu, kind, 3000, nd)
        assert _call(L.b2fmm_lap_direct_noalloc_dev, kind, nd, src, q, d, v, trg, got,
                     stream) == 0
        torch.cuda.synchronize()
        for a, b in zip(got, ref):
            assert _rel(a, b) < TOL


def test_noalloc_rejects_oversize(gpu):
    import torch
    from fmm2d_b200 import _lib
    L = _lib.lib()
    stream = torch.cuda.current_stream(gpu).cuda_stream
    nt = 262144 // 6 + 1  # one target more than the static scratch holds (kind 1)
    src, trg, q, d, v = _inputs(gpu, 1, 100, nt, 1, seed=9)
    outs = _outputs(gpu, 1, nt, 1)
    assert _call(L.b2fmm_lap_direct_noalloc_dev, 1, 1, src, q, d, v, trg, outs, stream) == 103
    torch.cuda.synchronize()
    assert bool((outs[0] == 7.0).all())


@pytest.mark.parametrize("kind,limit", [(0, 262144 // 3), (1, 262144 // 6)])
def test_noalloc_at_the_limit_and_one_beyond(gpu, kind, limit):
    """Exactly as many targets as the static scratch holds (one slice of
    partial sums) matches the allocating entry point; one more is refused."""
    import torch
    from fmm2d_b200 import _lib
    L = _lib.lib()
    stream = torch.cuda.current_stream(gpu).cuda_stream
    src, trg, q, d, v = _inputs(gpu, kind, 300, limit + 1, 1, seed=20 + kind)
    ref = _outputs(gpu, kind, limit, 1)
    got = _outputs(gpu, kind, limit, 1)
    assert _call(L.b2fmm_lap_direct_dev, kind, 1, src, q, d, v, trg[:limit], ref, stream) == 0
    assert _call(L.b2fmm_lap_direct_noalloc_dev, kind, 1, src, q, d, v, trg[:limit], got,
                 stream) == 0
    torch.cuda.synchronize()
    for a, b in zip(got, ref):
        assert _rel(a, b) < TOL
    over = _outputs(gpu, kind, limit + 1, 1)
    assert _call(L.b2fmm_lap_direct_noalloc_dev, kind, 1, src, q, d, v, trg, over, stream) == 103
    torch.cuda.synchronize()
    assert bool((over[0] == 7.0).all())
