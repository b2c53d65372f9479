"""Calls that do not wait for their tree on the host.

By default a Laplace/Cauchy call takes its box ranges from the tree's device
level table and checks the tree once, at the end.  A tree that needs more
boxes than the capacity guess, or more than 32 levels, makes the call run
again with the tree read back.  With options.async_call = 1 the
device-pointer entry points return once the call is queued, and
b2fmm_async_status reports device-side failures.  These tests require every
one of these paths to give the results of the read-back path, bit for bit.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from conftest import rel_l2
from fmm2d_b200 import _lib
from test_ref_pin import gauss16, graded_curve

pytestmark = pytest.mark.gpu


def _dev(a):
    return torch.as_tensor(np.ascontiguousarray(a), device="cuda")


def _p(t):
    return C.c_void_p(t.data_ptr())


class Call:
    """lfmm2d on device pointers (charges + dipoles, pg 2)."""

    def __init__(self, src, seed=0):
        rng = np.random.default_rng(seed)
        n = src.shape[1]
        self.n = n
        self.s = _dev(src.T)
        self.q = _dev((rng.normal(size=n) + 1j * rng.normal(size=n)).reshape(n, 1))
        self.d = _dev((rng.normal(size=n) + 0j).reshape(n, 1))
        ph = rng.uniform(0, 2 * np.pi, n)
        self.v = _dev(np.stack([np.cos(ph), np.sin(ph)], 1).reshape(n, 2, 1))
        self.src, self.qh, self.dh = src, self.q.cpu().numpy()[:, 0], self.d.cpu().numpy()[:, 0]
        self.vh = self.v.cpu().numpy()[:, :, 0].T

    def run(self, eps, precision="mixed", async_call=0):
        L = _lib.lib()
        pot = torch.empty((self.n, 1), dtype=torch.complex128, device="cuda")
        grad = torch.empty((self.n, 2, 1), dtype=torch.complex128, device="cuda")
        o = _lib.Options()
        o.ndiv, o.idivflag, o.ifnear, o.precision = 0, 0, 1, _lib.PREC[precision]
        o.async_call = async_call
        ier = C.c_int(-1)
        st = torch.cuda.current_stream().cuda_stream
        L.b2fmm_lfmm2d_dev(1, C.c_double(eps), C.c_int64(self.n), _p(self.s), 1, _p(self.q), 1,
                           _p(self.d), _p(self.v), 2, _p(pot), _p(grad), None, C.c_int64(0), None,
                           0, None, None, None, C.byref(o), None, C.c_void_p(st), C.byref(ier))
        return ier.value, pot, grad


def _status():
    ier = C.c_int(-1)
    _lib.lib().b2fmm_async_status(C.c_void_p(torch.cuda.current_stream().cuda_stream),
                                  C.byref(ier))
    return ier.value


@pytest.fixture
def read_back():
    """Runs the body with every call reading its tree back, then restores."""
    L = _lib.lib()
    L.b2fmm_set_device_ranges(0)
    yield
    L.b2fmm_set_device_ranges(1)


def _reference(call, eps, precision):
    L = _lib.lib()
    L.b2fmm_set_device_ranges(0)
    try:
        ier, pot, grad = call.run(eps, precision)
    finally:
        L.b2fmm_set_device_ranges(1)
    assert ier == 0
    return pot.cpu().numpy(), grad.cpu().numpy()


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_device_ranges_equal_read_back(gpu, precision):
    """A clustered tree deeper than the first-call level guess: the
    cooperative tail kernel takes the deep levels."""
    n = 150_000 + (1 if precision == "fp64" else 0)  # a size no earlier call had
    call = Call(gauss16(n, 90), 1)
    ier, pot0, grad0 = call.run(1e-6, precision)  # depth guessed from n: too shallow
    assert ier == 0
    rp, rg = _reference(call, 1e-6, precision)
    assert np.array_equal(pot0.cpu().numpy(), rp)
    assert np.array_equal(grad0.cpu().numpy(), rg)
    ier, pot, grad = call.run(1e-6, precision)  # depth remembered
    assert ier == 0
    assert np.array_equal(pot.cpu().numpy(), rp)
    assert np.array_equal(grad.cpu().numpy(), rg)


def test_async_calls_queue_and_match(gpu):
    call = Call(gauss16(200_000, 91), 2)
    rp, rg = _reference(call, 1e-6, "mixed")
    assert _status() == 0
    outs = []
    for _ in range(4):
        ier, pot, grad = call.run(1e-6, "mixed", async_call=1)
        assert ier == 0
        outs.append((pot, grad))
    assert _status() == 0
    for pot, grad in outs:
        assert np.array_equal(pot.cpu().numpy(), rp)
        assert np.array_equal(grad.cpu().numpy(), rg)


def test_capacity_shortfall_async_reports_and_blocking_retries(gpu):
    """A uniform cloud teaches the library a small tree for n points (22K
    boxes); a graded curve of the same n needs 95K.  Asynchronous: the
    status reports 104 (repeat synchronously).  Blocking: the call is
    redone with the tree read back, transparently."""
    n = 120_000
    uni = Call(np.random.default_rng(92).uniform(0, 1, (2, n)), 3)
    ier, _, _ = uni.run(1e-6)
    assert ier == 0
    clu = Call(graded_curve(n, 3), 4)
    rp, rg = _reference(clu, 1e-6, "mixed")
    ier, _, _ = uni.run(1e-6)  # the uniform shape is the remembered one again
    assert ier == 0
    ier, _, _ = clu.run(1e-6, async_call=1)
    assert ier == 0
    assert _status() == 104
    assert _status() == 0  # cleared by the query
    ier, _, _ = uni.run(1e-6)
    assert ier == 0
    ier, pot, grad = clu.run(1e-6)  # blocking: retried with the read-back tree
    assert ier == 0
    assert np.array_equal(pot.cpu().numpy(), rp)
    assert np.array_equal(grad.cpu().numpy(), rg)


def test_deep_duplicate_tree(gpu, oracle):
    """Coincident points refine to the 51-level cap: more than the 32 levels
    of the first sort, so the call is redone with the full keys."""
    base = np.random.default_rng(94).uniform(0, 1, (2, 40))
    src = np.repeat(base, 30, axis=1)  # clusters of 30 > ndiv 20 coincident points
    call = Call(src, 5)
    ier, pot, grad = call.run(1e-9, "fp64")
    assert ier == 0
    o = oracle.lfmm2d(1e-9, src, charges=call.qh, dipstr=call.dh, dipvec=call.vh, ifpgh=2)
    assert rel_l2(pot.cpu().numpy()[:, 0], o["pot"][0]) < 1e-11
    assert rel_l2(grad.cpu().numpy()[:, :, 0].T, o["grad"][0]) < 1e-11


def test_queued_host_calls_on_two_streams(gpu):
    """b2fmm_lfmm2d_host_async / cfmm2d / rfmm2d with pinned host arrays:
    four calls queued on two streams in turn give, bit for bit, the blocking
    host call's results, and b2fmm_async_status reports no failure."""
    L = _lib.lib()
    n = 60000
    call = Call(gauss16(n, 7), 3)
    pin = lambda a: torch.as_tensor(np.ascontiguousarray(a)).pin_memory()
    hs, hq, hd, hv = (pin(x.cpu()) for x in (call.s, call.q, call.d, call.v))
    o = _lib.Options()
    o.ndiv, o.idivflag, o.ifnear, o.precision = 0, 0, 1, _lib.PREC["mixed"]
    ier = C.c_int(-1)
    bpot = torch.empty((n, 1), dtype=torch.complex128).pin_memory()
    bgrad = torch.empty((n, 2, 1), dtype=torch.complex128).pin_memory()
    L.b2fmm_lfmm2d_ex(1, C.c_double(1e-6), C.c_int64(n), _p(hs), 1, _p(hq), 1, _p(hd), _p(hv),
                      2, _p(bpot), _p(bgrad), None, C.c_int64(0), None, 0, None, None, None,
                      C.byref(o), None, C.byref(ier))
    assert ier.value == 0
    streams = [torch.cuda.Stream(), torch.cuda.Stream()]
    outs = [(torch.empty_like(bpot).pin_memory(), torch.empty_like(bgrad).pin_memory())
            for _ in range(4)]
    for k, (po, gr) in enumerate(outs):
        L.b2fmm_lfmm2d_host_async(1, C.c_double(1e-6), C.c_int64(n), _p(hs), 1, _p(hq), 1,
                                  _p(hd), _p(hv), 2, _p(po), _p(gr), None, C.c_int64(0), None,
                                  0, None, None, None, C.byref(o),
                                  C.c_void_p(streams[k % 2].cuda_stream), C.byref(ier))
        assert ier.value == 0
    for s in streams:
        L.b2fmm_async_status(C.c_void_p(s.cuda_stream), C.byref(ier))
        assert ier.value == 0
    for po, gr in outs:
        assert torch.equal(po, bpot) and torch.equal(gr, bgrad)
    # the Cauchy and real entry points, against their blocking calls
    hqr = pin(call.q.real.contiguous().cpu())
    for fn_async, fn_ex, args in (
            (L.b2fmm_cfmm2d_host_async, L.b2fmm_cfmm2d_ex, [_p(hq), 0, None]),
            (L.b2fmm_rfmm2d_host_async, L.b2fmm_rfmm2d_ex, [_p(hqr), 0, None, None])):
        real = fn_ex is L.b2fmm_rfmm2d_ex
        dt = torch.float64 if real else torch.complex128
        p1 = torch.empty((n, 1), dtype=dt).pin_memory()
        p2 = torch.empty((n, 1), dtype=dt).pin_memory()
        fn_ex(1, C.c_double(1e-6), C.c_int64(n), _p(hs), 1, *args, 1, _p(p1), None, None,
              C.c_int64(0), None, 0, None, None, None, C.byref(o), None, C.byref(ier))
        assert ier.value == 0
        fn_async(1, C.c_double(1e-6), C.c_int64(n), _p(hs), 1, *args, 1, _p(p2), None, None,
                 C.c_int64(0), None, 0, None, None, None, C.byref(o),
                 C.c_void_p(streams[0].cuda_stream), C.byref(ier))
        assert ier.value == 0
        L.b2fmm_async_status(C.c_void_p(streams[0].cuda_stream), C.byref(ier))
        assert ier.value == 0 and torch.equal(p1, p2)
