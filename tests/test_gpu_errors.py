"""Error paths, with every failure made on the host side.

ier codes (as in the reference: 0 ok, 4 allocation failure; added here: 100
invalid argument, 102 a bounded device wait gave up).  Bad arguments and
non-finite coordinates are refused; an allocation failure injected by a test
hook returns 4 whichever allocation of the call it hits; a grid-barrier
wait limit shortened by a test hook makes the tree build give up and the
call return 102.  After each failure the next call must succeed with the
right result: the device context stays usable.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from fmm2d_b200 import _lib
from test_gpu_async import Call
from test_ref_pin import gauss16

pytestmark = pytest.mark.gpu


def _lfmm(n, src, q, d, v, pot, grad, eps=1e-6, nd=1, pg=2, dipvec=True, async_call=0):
    L = _lib.lib()
    o = _lib.Options()
    o.ndiv, o.idivflag, o.ifnear, o.precision = 0, 0, 1, 0
    o.async_call = async_call
    p = lambda t: C.c_void_p(t.data_ptr()) if t is not None else None
    ier = C.c_int(-1)
    L.b2fmm_lfmm2d_dev(nd, C.c_double(eps), C.c_int64(n), p(src), 1, p(q), 1, p(d),
                       p(v) if dipvec else None, pg, p(pot), p(grad), None, C.c_int64(0), None,
                       0, None, None, None, C.byref(o), None,
                       C.c_void_p(torch.cuda.current_stream().cuda_stream), C.byref(ier))
    return ier.value


@pytest.fixture
def call():
    return Call(gauss16(30_000, 80), 8)


def _good(call, ref=None):
    ier, pot, grad = call.run(1e-6)
    assert ier == 0
    if ref is not None:
        assert np.array_equal(pot.cpu().numpy(), ref[0])
        assert np.array_equal(grad.cpu().numpy(), ref[1])
    return pot.cpu().numpy(), grad.cpu().numpy()


def test_bad_arguments_return_100(gpu, call):
    ref = _good(call)
    n = call.n
    pot = torch.empty((n, 1), dtype=torch.complex128, device="cuda")
    grad = torch.empty((n, 2, 1), dtype=torch.complex128, device="cuda")
    args = (call.s, call.q, call.d, call.v, pot, grad)
    assert _lfmm(n, *args, nd=0) == 100          # no density vector
    assert _lfmm(-5, *args) == 100               # negative point count
    assert _lfmm(n, *args, pg=4) == 100          # no such output level
    assert _lfmm(n, *args, dipvec=False) == 100  # dipoles without directions
    _good(call, ref)


@pytest.mark.parametrize("bad", [np.nan, np.inf, -np.inf])
@pytest.mark.parametrize("mode", [1, 0])
def test_non_finite_coordinates_return_100(gpu, call, bad, mode):
    L = _lib.lib()
    ref = _good(call)
    src = call.s.clone()
    src[1234, 1] = bad
    n = call.n
    pot = torch.empty((n, 1), dtype=torch.complex128, device="cuda")
    grad = torch.empty((n, 2, 1), dtype=torch.complex128, device="cuda")
    L.b2fmm_set_device_ranges(mode)
    try:
        assert _lfmm(n, src, call.q, call.d, call.v, pot, grad) == 100
        assert _lfmm(n, src, call.q, call.d, call.v, pot, grad, eps=1e-9) == 100  # FP64 path
    finally:
        L.b2fmm_set_device_ranges(1)
    # asynchronous: reported by the status query
    assert _lfmm(n, src, call.q, call.d, call.v, pot, grad, async_call=1) == 0
    ier = C.c_int(-1)
    L.b2fmm_async_status(C.c_void_p(torch.cuda.current_stream().cuda_stream), C.byref(ier))
    assert ier.value == 100
    _good(call, ref)


@pytest.mark.parametrize("after", [0, 1, 5, 20, 40])
def test_injected_allocation_failure_returns_4(gpu, call, after):
    L = _lib.lib()
    ref = _good(call)
    L.b2fmm_test_fail_alloc(after)
    try:
        ier, _, _ = call.run(1e-6)
    finally:
        L.b2fmm_test_fail_alloc(-1)
    assert ier == 4
    torch.cuda.synchronize()
    _good(call, ref)


@pytest.mark.parametrize("mode", [1, 0])
def test_barrier_wait_limit_returns_102(gpu, call, mode):
    L = _lib.lib()
    ref = _good(call)
    L.b2fmm_set_device_ranges(mode)
    L.b2fmm_test_barrier_limit(C.c_longlong(1))
    try:
        ier, _, _ = call.run(1e-6)
    finally:
        L.b2fmm_test_barrier_limit(C.c_longlong(0))
        L.b2fmm_set_device_ranges(1)
    assert ier == 102
    torch.cuda.synchronize()
    _good(call, ref)
