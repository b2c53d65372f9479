"""fmm2dpy-compatible front end (python/fmm2dpy/fmm2d.py of the reference).

Same keyword-only signatures, argument meaning, output shapes, assertion
messages and dispatch as ``fmm2dpy.hfmm2d / lfmm2d / rfmm2d / cfmm2d`` and
the direct sums ``h2ddir / l2ddir / r2ddir / c2ddir``, plus ``comperr`` and
``Output``.  Arrays
may be numpy arrays (host; results come back as numpy) or CUDA torch tensors
(device; zero host copies, results are CUDA tensors).  Every evaluation runs
in ``libfmm2d_b200.so`` on the GPU; there is no CPU fallback.

Optional keyword extensions (not in the reference, defaults reproduce it):
``precision`` ('auto' = mixed when eps >= 1e-6, 'fp64', 'mixed'), ``ndiv``
(leaf capacity override, or 'auto' for the learned cost model of
fmm2d_b200/costmodel.py, which then also picks the level balance),
``level_balance`` (Laplace: the leaf capacity at level l is
ndiv 2^(b (lp - l)), lp the level whose boxes hold ndiv points of a uniform
cloud; 0, the default, keeps ndiv at every level) and ``timeinfo`` (a
length-8 float64 numpy array that receives the per-step device times).
"""
import ctypes as C

import numpy as np
import numpy.linalg as la

from . import _lib

FE_CAUCHY, FE_LAPLACE, FE_REAL = 0, 1, 2


class Output():
    pot = None
    grad = None
    hess = None
    pottarg = None
    gradtarg = None
    hesstarg = None
    pre = None
    pretarg = None
    ier = 0


def _is_torch(x):
    return x is not None and type(x).__module__.split(".")[0] == "torch"


def _ptr(a):
    if a is None:
        return None
    if _is_torch(a):
        return C.c_void_p(a.data_ptr())
    return a.ctypes.data_as(C.c_void_p)


def _ns_of(sources):
    return sources.shape[1] if len(sources.shape) == 2 else 1


class _NP:
    """numpy arrays: host entry points."""

    @staticmethod
    def prep(a, shape, perm, dtype):
        a = np.asarray(a).reshape(shape)
        return np.ascontiguousarray(np.transpose(a, perm), dtype=dtype)

    @staticmethod
    def empty(shape, dtype):
        return np.zeros(shape, dtype=dtype)

    @staticmethod
    def T(a, perm):
        return np.transpose(a, perm)


class _TH:
    """CUDA torch tensors: device entry points on the current stream."""

    @staticmethod
    def prep(a, shape, perm, dtype):
        import torch
        td = {np.float64: torch.float64, np.complex128: torch.complex128}[dtype]
        return a.reshape(shape).permute(*perm).contiguous().to(td)

    @staticmethod
    def empty(shape, dtype, device=None):
        import torch
        td = {np.float64: torch.float64, np.complex128: torch.complex128}[dtype]
        return torch.zeros(shape, dtype=td, device=device)

    @staticmethod
    def T(a, perm):
        return a.permute(*perm)


def _options(precision, ndiv, level_balance=0.0):
    o = _lib.Options()
    o.ndiv = int(ndiv) if ndiv else 0
    o.idivflag = 0
    o.ifnear = 1
    o.precision = _lib.PREC[precision]
    o.level_balance = float(level_balance or 0.0)
    return o


def _lap_run(fe, eps, sources, charges, dipstr, dipvec, targets, ifpgh, ifpghtarg, nd,
             precision="auto", ndiv=None, timeinfo=None, level_balance=0.0):
    """One Cauchy-engine FMM call; returns user-shaped outputs and ier."""
    torch_mode = _is_torch(sources)
    B = _TH if torch_mode else _NP
    ns = _ns_of(sources)
    dt = np.float64 if fe == FE_REAL else np.complex128
    s = B.prep(sources, (2, ns), (1, 0), np.float64)
    q = None if charges is None else B.prep(charges, (nd, ns), (1, 0), dt)
    d = None if dipstr is None else B.prep(dipstr, (nd, ns), (1, 0), dt)
    v = None
    if dipstr is not None and fe != FE_CAUCHY:
        v = B.prep(dipvec, (nd, 2, ns), (2, 1, 0), np.float64)
    nt = 0
    t = None
    if targets is not None and ifpghtarg > 0:
        nt = _ns_of(targets)
        t = B.prep(targets, (2, nt), (1, 0), np.float64)
    kw = dict(device=sources.device) if torch_mode else {}
    gshape = (lambda n: (n, nd)) if fe == FE_CAUCHY else (lambda n: (n, 2, nd))
    hshape = (lambda n: (n, nd)) if fe == FE_CAUCHY else (lambda n: (n, 3, nd))
    pot = B.empty((ns, nd), dt, **kw) if ifpgh >= 1 else None
    grad = B.empty(gshape(ns), dt, **kw) if ifpgh >= 2 else None
    hess = B.empty(hshape(ns), dt, **kw) if ifpgh >= 3 else None
    pott = B.empty((nt, nd), dt, **kw) if ifpghtarg >= 1 and nt else None
    gradt = B.empty(gshape(nt), dt, **kw) if ifpghtarg >= 2 and nt else None
    hesst = B.empty(hshape(nt), dt, **kw) if ifpghtarg >= 3 and nt else None
    if ndiv == "auto":
        # leaf size and level balance from the learned cost model (lndiv2d
        # table, balance 0, without weights)
        import torch
        from . import costmodel
        dsrc = s if torch_mode else torch.as_tensor(s, device="cuda")
        dtrg = None if t is None else (t if torch_mode else torch.as_tensor(t, device="cuda"))
        ndiv, level_balance = costmodel.auto_tree(dsrc, dtrg, eps)
    opts = _options(precision, ndiv, level_balance)
    ti = np.zeros(8) if timeinfo is None else timeinfo
    ier = C.c_int(0)
    L = _lib.lib()
    head = [C.c_int(nd), C.c_double(eps), C.c_int64(ns), _ptr(s), C.c_int(q is not None), _ptr(q),
            C.c_int(d is not None), _ptr(d)]
    if fe != FE_CAUCHY:
        head.append(_ptr(v))
    tail = [C.c_int(ifpgh), _ptr(pot), _ptr(grad), _ptr(hess), C.c_int64(nt), _ptr(t),
            C.c_int(ifpghtarg), _ptr(pott), _ptr(gradt), _ptr(hesst), C.byref(opts),
            ti.ctypes.data_as(C.c_void_p)]
    name = {FE_CAUCHY: "cfmm2d", FE_LAPLACE: "lfmm2d", FE_REAL: "rfmm2d"}[fe]
    if torch_mode:
        import torch
        stream = torch.cuda.current_stream(sources.device).cuda_stream
        getattr(L, f"b2fmm_{name}_dev")(*head, *tail, C.c_void_p(stream), C.byref(ier))
    else:
        getattr(L, f"b2fmm_{name}_ex")(*head, *tail, C.byref(ier))

    def user(a, kind):
        if a is None:
            return None
        if kind == "p" or fe == FE_CAUCHY:
            return a[:, 0] if nd == 1 else B.T(a, (1, 0))
        return B.T(a[:, :, 0], (1, 0)) if nd == 1 else B.T(a, (2, 1, 0))

    return dict(pot=user(pot, "p"), grad=user(grad, "g"), hess=user(hess, "h"),
                pottarg=user(pott, "p"), gradtarg=user(gradt, "g"), hesstarg=user(hesst, "h"),
                ier=ier.value)


def _check_common(sources, charges, dipstr, dipvec, targets, nd, need_dipvec=True):
    """Shape assertions of the reference front end (fmm2d.py:515-546)."""
    assert sources.shape[0] == 2, "The first dimension of sources must be 2"
    ns = _ns_of(sources)
    ifcharge = ifdipole = 0
    if charges is not None:
        if nd == 1:
            assert charges.shape[0] == ns, "Charges must be same length as second dimension of sources"
        if nd > 1:
            assert charges.shape[0] == nd and charges.shape[1] == ns, "Charges must be of shape [nd,ns] where nd is number of densities, and ns is number of sources"
        ifcharge = 1
    if (need_dipvec and (dipvec is not None or dipstr is not None)) or (not need_dipvec and dipstr is not None):
        if nd == 1 and ns > 1:
            assert dipstr.shape[0] == ns, "Dipole strengths must be same length as second dimension of sources"
            if need_dipvec:
                assert dipvec.shape[0] == 2 and dipvec.shape[1] == ns, "dipole vectors must be of shape [2,number of sources]"
        if nd == 1 and ns == 1:
            assert dipstr.shape[0] == ns, "Dipole strengths must be same length as second dimension of sources"
            if need_dipvec:
                assert dipvec.shape[0] == 2, "dipole vectors must be of shape [2,number of sources]"
        if nd > 1:
            if need_dipvec:
                assert dipvec.shape[0] == nd and dipvec.shape[1] == 2 and dipvec.shape[2] == ns, "Dipole vectors must be of shape [nd,2,ns] where nd is number of densities, and ns is number of sources"
            assert dipstr.shape[0] == nd and dipstr.shape[1] == ns, "Dipole strengths must be of shape [nd,ns] where nd is number of densities, and ns is number of sources"
        ifdipole = 1
    if targets is not None:
        assert targets.shape[0] == 2, "The first dimension of targets must be 2"
    return ns, ifcharge, ifdipole


def _dispatch(fe, out, eps, sources, charges, dipstr, dipvec, targets, pg, pgt, nd, ifcharge,
              ifdipole, pmax, st_msg, ext):
    """Source / target / source+target dispatch of the reference front end
    (fmm2d.py:548-713): the source branch runs whenever pg is set; with
    targets it is superseded by the source+target call keyed on pgt."""
    if not (ifcharge or ifdipole):
        return out
    valid = tuple(range(1, pmax + 1))
    q = charges if ifcharge else None
    d = dipstr if ifdipole else None
    v = dipvec if ifdipole else None
    res = None
    if pg in valid and targets is not None:
        assert pg == pgt, st_msg
        res = _lap_run(fe, eps, sources, q, d, v, targets, pgt, pgt, nd, **ext)
    elif pg in valid:
        res = _lap_run(fe, eps, sources, q, d, v, None, pg, 0, nd, **ext)
    elif targets is not None and pgt in valid:
        res = _lap_run(fe, eps, sources, q, d, v, targets, 0, pgt, nd, **ext)
    if res is not None:
        for k in ("pot", "grad", "hess", "pottarg", "gradtarg", "hesstarg"):
            if res[k] is not None:
                setattr(out, k, res[k])
        out.ier = res["ier"]
    return out


_ST_MSG = "if output is requested at both sources and targets, then the same pg must be equal to pgt"


def lfmm2d(*, eps, sources, charges=None, dipstr=None, dipvec=None, targets=None, pg=0, pgt=0,
           nd=1, **ext):
    """Complex Laplace FMM (python/fmm2dpy/fmm2d.py:459-713).

    u(x) = sum_j c_j log|x - x_j| - d_j v_j.(x - x_j)/|x - x_j|^2 (the
    kernel the Fortran evaluates), with gradients (2 components) and
    Hessians (xx, xy, yy).  Self interactions are omitted.
    """
    out = Output()
    ns, ifcharge, ifdipole = _check_common(sources, charges, dipstr, dipvec, targets, nd)
    if pg == 0 and pgt == 0:
        print("Nothing to compute, set either pg or pgt to non-zero")
        return out
    return _dispatch(FE_LAPLACE, out, eps, sources, charges, dipstr, dipvec, targets, pg, pgt, nd,
                     ifcharge, ifdipole, 3, _ST_MSG, ext)


def rfmm2d(*, eps, sources, charges=None, dipstr=None, dipvec=None, targets=None, pg=0, pgt=0,
           nd=1, **ext):
    """Real Laplace FMM (python/fmm2dpy/fmm2d.py:201-457)."""
    out = Output()
    ns, ifcharge, ifdipole = _check_common(sources, charges, dipstr, dipvec, targets, nd)
    if pg == 0 and pgt == 0:
        print("Nothing to compute, set either pg or pgt to non-zero")
        return out
    return _dispatch(FE_REAL, out, eps, sources, charges, dipstr, dipvec, targets, pg, pgt, nd,
                     ifcharge, ifdipole, 3, _ST_MSG, ext)


def cfmm2d(*, eps, sources, charges=None, dipstr=None, targets=None, pg=0, pgt=0, nd=1, **ext):
    """Cauchy FMM (python/fmm2dpy/fmm2d.py:715-964): pot, d/dz, d2/dz2."""
    out = Output()
    ns, ifcharge, ifdipole = _check_common(sources, charges, dipstr, None, targets, nd,
                                           need_dipvec=False)
    if pg == 0 and pgt == 0:
        print("Nothing to compute, set either pg or pgt to non-zero")
        return out
    return _dispatch(FE_CAUCHY, out, eps, sources, charges, dipstr, None, targets, pg, pgt, nd,
                     ifcharge, ifdipole, 3, _ST_MSG, ext)


# ---------------------------------------------------------------------------
# direct sums (python/fmm2dpy/fmm2d.py:1370-1740), evaluated on the GPU
# ---------------------------------------------------------------------------
def _to_dev(a, dtype):
    import torch
    if a is None:
        return None
    if _is_torch(a):
        return a.to(device="cuda", dtype=dtype)
    return torch.as_tensor(np.asarray(a)).to(device="cuda", dtype=dtype)


def _direct_run(kind, sources, targets, charges, dipstr, dipvec, pgt, nd, thresh):
    import torch
    torch_mode = _is_torch(sources)
    ns = _ns_of(sources)
    nt = _ns_of(targets)
    cd = torch.float64 if kind == 2 else torch.complex128
    s = _to_dev(sources, torch.float64).reshape(2, ns).T.contiguous()
    t = _to_dev(targets, torch.float64).reshape(2, nt).T.contiguous()
    q = None if charges is None else _to_dev(charges, cd).reshape(nd, ns).T.contiguous()
    d = None if dipstr is None else _to_dev(dipstr, cd).reshape(nd, ns).T.contiguous()
    v = None
    if dipstr is not None and kind != 0:
        v = _to_dev(dipvec, torch.float64).reshape(nd, 2, ns).permute(2, 1, 0).contiguous()
    gk = 1 if kind == 0 else 2
    hk = 1 if kind == 0 else 3
    pot = torch.zeros((nt, nd), dtype=cd, device="cuda")
    grad = torch.zeros((nt, gk, nd), dtype=cd, device="cuda") if pgt >= 2 else None
    hess = torch.zeros((nt, hk, nd), dtype=cd, device="cuda") if pgt >= 3 else None
    ier = C.c_int(0)
    stream = torch.cuda.current_stream().cuda_stream
    _lib.lib().b2fmm_lap_direct_dev(C.c_int(kind), C.c_int(nd), C.c_int64(ns), _ptr(s), _ptr(q),
                                    _ptr(d), _ptr(v), C.c_int64(nt), _ptr(t), C.c_int(pgt),
                                    _ptr(pot), _ptr(grad), _ptr(hess), C.c_double(thresh),
                                    C.c_void_p(stream), C.byref(ier))
    if ier.value != 0:
        raise RuntimeError(f"direct sum failed, ier={ier.value}")

    def user(a, k):
        if a is None:
            return None
        if k == 1:
            a = a[:, 0, :]
            r = a[:, 0] if nd == 1 else a.T
        else:
            r = a[:, :, 0].T if nd == 1 else a.permute(2, 1, 0)
        return r if torch_mode else r.cpu().numpy()

    potu = pot[:, 0] if nd == 1 else pot.T
    out = Output()
    out.pottarg = potu if torch_mode else potu.cpu().numpy()
    if pgt >= 2:
        out.gradtarg = user(grad, gk)
    if pgt >= 3:
        out.hesstarg = user(hess, hk)
    return out


def _direct_front(kind, sources, targets, charges, dipstr, dipvec, pgt, nd, thresh):
    assert sources.shape[0] == 2, "The first dimension of sources must be 2"
    out = Output()
    if pgt == 0:
        print("Nothing to compute, set either pg or pgt to non-zero")
        return out
    _check_common(sources, charges, dipstr, dipvec, None, nd, need_dipvec=(kind != 0))
    assert targets.shape[0] == 2, "The first dimension of targets must be 2"
    if charges is None and dipstr is None:
        return out
    return _direct_run(kind, sources, targets, charges, dipstr, dipvec, pgt, nd, thresh)


def l2ddir(*, sources, targets, charges=None, dipstr=None, dipvec=None, pgt=0, nd=1,
           thresh=1e-16):
    """Complex Laplace direct sum (fmm2d.py:1493-1614)."""
    return _direct_front(1, sources, targets, charges, dipstr, dipvec, pgt, nd, thresh)


def r2ddir(*, sources, targets, charges=None, dipstr=None, dipvec=None, pgt=0, nd=1,
           thresh=1e-16):
    """Real Laplace direct sum (fmm2d.py:1370-1491)."""
    return _direct_front(2, sources, targets, charges, dipstr, dipvec, pgt, nd, thresh)


def c2ddir(*, sources, targets, charges=None, dipstr=None, pgt=0, nd=1, thresh=1e-16):
    """Cauchy direct sum (fmm2d.py:1616-1740)."""
    return _direct_front(0, sources, targets, charges, dipstr, None, pgt, nd, thresh)


# ---------------------------------------------------------------------------
# Helmholtz (python/fmm2dpy/fmm2d.py:20-199, 1250-1368)
# ---------------------------------------------------------------------------
def _helm_run(eps, zk, sources, charges, dipstr, dipvec, targets, ifpgh, ifpghtarg, nd,
              ndiv=None, timeinfo=None, **_ignored):
    """One Helmholtz FMM call; returns user-shaped outputs and ier."""
    torch_mode = _is_torch(sources)
    B = _TH if torch_mode else _NP
    ns = _ns_of(sources)
    zk = complex(zk)
    dt = np.complex128
    s = B.prep(sources, (2, ns), (1, 0), np.float64)
    q = None if charges is None else B.prep(charges, (nd, ns), (1, 0), dt)
    d = None if dipstr is None else B.prep(dipstr, (nd, ns), (1, 0), dt)
    v = None if dipstr is None else B.prep(dipvec, (nd, 2, ns), (2, 1, 0), np.float64)
    nt = 0
    t = None
    if targets is not None and ifpghtarg > 0:
        nt = _ns_of(targets)
        t = B.prep(targets, (2, nt), (1, 0), np.float64)
    kw = dict(device=sources.device) if torch_mode else {}
    pot = B.empty((ns, nd), dt, **kw) if ifpgh >= 1 else None
    grad = B.empty((ns, 2, nd), dt, **kw) if ifpgh >= 2 else None
    hess = B.empty((ns, 3, nd), dt, **kw) if ifpgh >= 3 else None
    pott = B.empty((nt, nd), dt, **kw) if ifpghtarg >= 1 and nt else None
    gradt = B.empty((nt, 2, nd), dt, **kw) if ifpghtarg >= 2 and nt else None
    hesst = B.empty((nt, 3, nd), dt, **kw) if ifpghtarg >= 3 and nt else None
    ti = np.zeros(8) if timeinfo is None else timeinfo
    ier = C.c_int(0)
    L = _lib.lib()
    head = [C.c_int(nd), C.c_double(eps), C.c_double(zk.real), C.c_double(zk.imag), C.c_int64(ns),
            _ptr(s), C.c_int(q is not None), _ptr(q), C.c_int(d is not None), _ptr(d), _ptr(v)]
    pgh = [C.c_int(ifpgh), _ptr(pot), _ptr(grad), _ptr(hess), C.c_int64(nt), _ptr(t),
           C.c_int(ifpghtarg), _ptr(pott), _ptr(gradt), _ptr(hesst)]
    if torch_mode:
        import torch
        opts = _options("fp64", ndiv)
        stream = torch.cuda.current_stream(sources.device).cuda_stream
        L.b2fmm_hfmm2d_dev(*head, *pgh, C.byref(opts), ti.ctypes.data_as(C.c_void_p),
                           C.c_void_p(stream), C.byref(ier))
    else:
        L.b2fmm_hfmm2d_ndiv(*head, C.c_int(0), *pgh, C.c_int(int(ndiv) if ndiv else 0),
                            C.c_int(0), C.c_int(1), ti.ctypes.data_as(C.c_void_p), C.byref(ier))

    def user(a, kind):
        if a is None:
            return None
        if kind == "p":
            return a[:, 0] if nd == 1 else B.T(a, (1, 0))
        return B.T(a[:, :, 0], (1, 0)) if nd == 1 else B.T(a, (2, 1, 0))

    return dict(pot=user(pot, "p"), grad=user(grad, "g"), hess=user(hess, "h"),
                pottarg=user(pott, "p"), gradtarg=user(gradt, "g"), hesstarg=user(hesst, "h"),
                ier=ier.value)


_HST_MSG = ("if both potential or potential at gradient are requested at sources and targets, "
            "then the same pg must be equal to pgt")


def hfmm2d(*, eps, zk, sources, charges=None, dipstr=None, dipvec=None, targets=None, pg=0,
           pgt=0, nd=1, **ext):
    """Helmholtz FMM (python/fmm2dpy/fmm2d.py:20-199).

    u(x) = (i/4) sum_j c_j H0(k|x - x_j|) + k d_j v_j.(x - x_j)/|x - x_j|
    H1(k|x - x_j|), with gradients; pg / pgt take 1 (potential) or 2
    (potential and gradient) as in the reference front end.  Self
    interactions are omitted.  ``out.ier`` is 20 when some level that
    translates expansions has boxes larger than 16 wavelengths.
    """
    out = Output()
    ns, ifcharge, ifdipole = _check_common(sources, charges, dipstr, dipvec, targets, nd)
    if pg == 0 and pgt == 0:
        print("Nothing to compute, set either pg or pgt to non-zero")
        return out
    if not (ifcharge or ifdipole):
        return out
    q = charges if ifcharge else None
    d = dipstr if ifdipole else None
    v = dipvec if ifdipole else None
    res = None
    if pg in (1, 2) and targets is not None:
        assert pg == pgt, _HST_MSG
        res = _helm_run(eps, zk, sources, q, d, v, targets, pgt, pgt, nd, **ext)
    elif pg in (1, 2):
        res = _helm_run(eps, zk, sources, q, d, v, None, pg, 0, nd, **ext)
    elif targets is not None and pgt in (1, 2):
        res = _helm_run(eps, zk, sources, q, d, v, targets, 0, pgt, nd, **ext)
    if res is not None:
        for k in ("pot", "grad", "pottarg", "gradtarg"):
            if res[k] is not None:
                setattr(out, k, res[k])
        out.ier = res["ier"]
    return out


def h2ddir(*, zk, sources, targets, charges=None, dipstr=None, dipvec=None, pgt=0, nd=1,
           thresh=1e-16):
    """Helmholtz direct sum (python/fmm2dpy/fmm2d.py:1250-1368); pgt 1 or 2.
    A source is skipped at targets where |zk| |x - x_j| is below thresh
    (at or below for the charge potential-only kernel)."""
    import torch
    assert sources.shape[0] == 2, "The first dimension of sources must be 2"
    out = Output()
    if pgt == 0:
        print("Nothing to compute, set either pg or pgt to non-zero")
        return out
    ns, ifcharge, ifdipole = _check_common(sources, charges, dipstr, dipvec, None, nd)
    assert targets.shape[0] == 2, "The first dimension of targets must be 2"
    if pgt not in (1, 2) or not (ifcharge or ifdipole):
        return out
    torch_mode = _is_torch(sources)
    zk = complex(zk)
    nt = _ns_of(targets)
    s = _to_dev(sources, torch.float64).reshape(2, ns).T.contiguous()
    t = _to_dev(targets, torch.float64).reshape(2, nt).T.contiguous()
    cd = torch.complex128
    q = _to_dev(charges, cd).reshape(nd, ns).T.contiguous() if ifcharge else None
    d = _to_dev(dipstr, cd).reshape(nd, ns).T.contiguous() if ifdipole else None
    v = (_to_dev(dipvec, torch.float64).reshape(nd, 2, ns).permute(2, 1, 0).contiguous()
         if ifdipole else None)
    pot = torch.zeros((nt, nd), dtype=cd, device="cuda")
    grad = torch.zeros((nt, 2, nd), dtype=cd, device="cuda") if pgt >= 2 else None
    ier = C.c_int(0)
    stream = torch.cuda.current_stream().cuda_stream
    _lib.lib().b2fmm_h2ddir_dev(C.c_int(nd), C.c_double(zk.real), C.c_double(zk.imag),
                                C.c_int64(ns), _ptr(s), _ptr(q), _ptr(d), _ptr(v),
                                C.c_int64(nt), _ptr(t), C.c_int(pgt), _ptr(pot), _ptr(grad),
                                None, C.c_double(thresh), C.c_void_p(stream), C.byref(ier))
    if ier.value != 0:
        raise RuntimeError(f"direct sum failed, ier={ier.value}")
    potu = pot[:, 0] if nd == 1 else pot.T
    out.pottarg = potu if torch_mode else potu.cpu().numpy()
    if pgt >= 2:
        g = grad[:, :, 0].T if nd == 1 else grad.permute(2, 1, 0)
        out.gradtarg = g if torch_mode else g.cpu().numpy()
    return out


# ---------------------------------------------------------------------------
# relative l2 error of the first ntest values (fmm2d.py:2017-2139)
# ---------------------------------------------------------------------------
def _fortran_dev(a, shape, dtype):
    """A user array of the reference's shape (nd, k, n) as a CUDA tensor in
    column-major (Fortran) element order."""
    import torch
    t = _to_dev(a, dtype).reshape(shape)
    return t.permute(*reversed(range(len(shape)))).contiguous()


def _user(t, torch_mode, squeeze):
    """Device output in column-major order (n, ..., nd) back to the
    reference's (nd, ..., n) shape (without nd when squeeze)."""
    if t is None:
        return None
    r = t.permute(*reversed(range(t.dim())))
    if squeeze:
        r = r[0]
    return r if torch_mode else r.cpu().numpy()


def _bh_check(sources, charges, dipoles, nd, ns):
    """Shape assertions of the reference's bhfmm2d / bh2ddir front ends."""
    if charges is not None:
        if nd == 1 and ns > 1:
            assert charges.shape[0] == 2 and charges.shape[1] == ns, \
                "Charges must be of shape [2, number of source]"
        if nd == 1 and ns == 1:
            assert charges.shape[0] == 2, "Charges must of shape [2, number of sources]"
        if nd > 1:
            assert charges.shape[0] == nd and charges.shape[1] == 2 and charges.shape[2] == ns, \
                "Charges must be of shape [nd,2,ns] where nd is number of densities, and ns " \
                "is number of sources"
    if dipoles is not None:
        if nd == 1 and ns > 1:
            assert dipoles.shape[0] == 3 and dipoles.shape[1] == ns, \
                "Dipole must of shape [3, number of sources]"
        if nd == 1 and ns == 1:
            assert dipoles.shape[0] == 3, "Dipole must of shape [3, number of sources]"
        if nd > 1:
            assert dipoles.shape[0] == nd and dipoles.shape[1] == 3 and dipoles.shape[2] == ns, \
                "Dipole must of shape [nd,2, number of sources]"


def _bh_run(eps, sources, charges, dipoles, targets, pg, pgt, nd, direct=False, thresh=1e-16):
    import torch
    torch_mode = _is_torch(sources)
    ns = _ns_of(sources)
    s = _fortran_dev(sources, (2, ns), torch.float64)
    q = None if charges is None else _fortran_dev(charges, (nd, 2, ns), torch.complex128)
    d = None if dipoles is None else _fortran_dev(dipoles, (nd, 3, ns), torch.complex128)
    nt = 0
    t = None
    if targets is not None and pgt > 0:
        nt = _ns_of(targets)
        t = _fortran_dev(targets, (2, nt), torch.float64)
    z = lambda *sh: torch.zeros(sh, dtype=torch.complex128, device="cuda")
    pot = z(ns, nd) if pg >= 1 else None
    grad = z(ns, 3, nd) if pg >= 2 else None
    pott = z(nt, nd) if pgt >= 1 and nt else None
    gradt = z(nt, 3, nd) if pgt >= 2 and nt else None
    ier = C.c_int(0)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    L = _lib.lib()
    if direct:
        L.b2fmm_bh2ddir_dev(nd, ns, _ptr(s), _ptr(q), _ptr(d), nt, _ptr(t), pgt, _ptr(pott),
                            _ptr(gradt), C.c_double(thresh), stream, C.byref(ier))
    else:
        L.b2fmm_bhfmm2d_dev(nd, C.c_double(eps), ns, _ptr(s), int(q is not None), _ptr(q),
                            int(d is not None), _ptr(d), pg, _ptr(pot), _ptr(grad), nt, _ptr(t),
                            pgt, _ptr(pott), _ptr(gradt), stream, C.byref(ier))
    out = Output()
    out.ier = ier.value
    sq = nd == 1
    out.pot, out.grad = _user(pot, torch_mode, sq), _user(grad, torch_mode, sq)
    out.pottarg, out.gradtarg = _user(pott, torch_mode, sq), _user(gradt, torch_mode, sq)
    return out


def bhfmm2d(*, eps, sources, charges=None, dipoles=None, targets=None, pg=0, pgt=0, nd=1):
    """Biharmonic FMM (python/fmm2dpy/fmm2d.py bhfmm2d, src/biharmonic/bhfmm2d.f):
    u(x) = sum 2 c1 log|x-x_j| + c2 (x-x_j)/conj(x-x_j) + d1/(x-x_j)
    + d3/conj(x-x_j) + d2 (x-x_j)/conj(x-x_j)^2; grad the three derivatives
    (d/dz, its conj(z) part, d/dconj(z)).  charges (nd,2,n), dipoles (nd,3,n)."""
    out = Output()
    assert sources.shape[0] == 2, "The first dimension of sources must be 2"
    ns = _ns_of(sources)
    if pg == 0 and pgt == 0:
        print("Nothing to compute, set either pg or pgt to non-zero")
        return out
    _bh_check(sources, charges, dipoles, nd, ns)
    if targets is not None:
        assert targets.shape[0] == 2, "The first dimension of targets must be 2"
    return _bh_run(eps, sources, charges, dipoles, targets, pg, pgt, nd)


def bh2ddir(*, sources, targets, charges=None, dipoles=None, pgt=0, nd=1, thresh=1e-16):
    """All-pairs biharmonic sums at the targets (fmm2d.py bh2ddir)."""
    out = Output()
    assert sources.shape[0] == 2, "The first dimension of sources must be 2"
    ns = _ns_of(sources)
    if pgt == 0:
        print("Nothing to compute, set either pg or pgt to non-zero")
        return out
    _bh_check(sources, charges, dipoles, nd, ns)
    assert targets.shape[0] == 2, "The first dimension of targets must be 2"
    return _bh_run(0.0, sources, charges, dipoles, targets, 0, pgt, nd, direct=True,
                   thresh=thresh)


def _st_check(stoklet, strslet, strsvec, nd, ns):
    if stoklet is not None:
        if nd == 1 and ns > 1:
            assert stoklet.shape[0] == 2 and stoklet.shape[1] == ns, \
                "stoklet vectors must be of shape [2,number of sources]"
        if nd == 1 and ns == 1:
            assert stoklet.shape[0] == 2, "stoklet vectors must be of shape [2,number of sources]"
        if nd > 1:
            assert stoklet.shape[0] == nd and stoklet.shape[1] == 2 and stoklet.shape[2] == ns, \
                "stoklet vectors must be of shape [nd,2,ns] where nd is number of densities, " \
                "and ns is number of sources"
    if strslet is not None and strsvec is not None:
        if nd == 1 and ns > 1:
            assert strslet.shape[0] == 2 and strslet.shape[1] == ns, \
                "strslet vectors must be of shape [2,number of sources]"
            assert strsvec.shape[0] == 2 and strsvec.shape[1] == ns, \
                "strsvec vectors must be of shape [2,number of sources]"
        if nd == 1 and ns == 1:
            assert strslet.shape[0] == 2, "strslet vectors must be of shape [2,number of sources]"
            assert strsvec.shape[0] == 2, "strsvec vectors must be of shape [2,number of sources]"
        if nd > 1:
            assert strslet.shape[0] == nd and strslet.shape[1] == 2 and strslet.shape[2] == ns, \
                "strslet vectors must be of shape [nd,2,ns] where nd is number of densities, " \
                "and ns is number of sources"
            assert strsvec.shape[0] == nd and strsvec.shape[1] == 2 and strsvec.shape[2] == ns, \
                "strsvec vectors must be of shape [nd,2,ns] where nd is number of densities, " \
                "and ns is number of sources"


def _st_run(eps, sources, stoklet, strslet, strsvec, targets, ifppreg, ifppregtarg, nd,
            direct=False, thresh=1e-16):
    import torch
    torch_mode = _is_torch(sources)
    ns = _ns_of(sources)
    s = _fortran_dev(sources, (2, ns), torch.float64)
    f = lambda a: None if a is None else _fortran_dev(a, (nd, 2, ns), torch.float64)
    sk, sl, sv = f(stoklet), f(strslet), f(strsvec)
    nt = 0
    t = None
    if targets is not None and ifppregtarg > 0:
        nt = _ns_of(targets)
        t = _fortran_dev(targets, (2, nt), torch.float64)
    z = lambda *sh: torch.zeros(sh, dtype=torch.float64, device="cuda")
    bufs = []
    for n, lev in ((ns, ifppreg), (nt, ifppregtarg)):
        bufs.append((z(n, 2, nd) if lev >= 1 and n else None,
                     z(n, nd) if lev >= 2 and n else None,
                     z(n, 2, 2, nd) if lev >= 3 and n else None))
    (pot, pre, grad), (pott, pret, gradt) = bufs
    ier = C.c_int(0)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    L = _lib.lib()
    ist, isl = int(sk is not None), int(sl is not None)
    if direct:
        for tg, n, lev, (po, pr, gr) in ((s, ns, ifppreg, bufs[0]), (t, nt, ifppregtarg, bufs[1])):
            if lev > 0 and n:
                L.b2fmm_st2ddir_dev(nd, ns, _ptr(s), ist, _ptr(sk), isl, _ptr(sl), _ptr(sv), n,
                                    _ptr(tg), lev, _ptr(po), _ptr(pr), _ptr(gr),
                                    C.c_double(thresh), stream, C.byref(ier))
    else:
        L.b2fmm_stfmm2d_dev(nd, C.c_double(eps), ns, _ptr(s), ist, _ptr(sk), isl, _ptr(sl),
                            _ptr(sv), ifppreg, _ptr(pot), _ptr(pre), _ptr(grad), nt, _ptr(t),
                            ifppregtarg, _ptr(pott), _ptr(pret), _ptr(gradt), stream,
                            C.byref(ier))
    out = Output()
    out.ier = ier.value
    out.pot, out.pre, out.grad = (_user(a, torch_mode, False) for a in (pot, pre, grad))
    out.pottarg, out.pretarg, out.gradtarg = (_user(a, torch_mode, False)
                                              for a in (pott, pret, gradt))
    return out


def _st_front(eps, sources, stoklet, strslet, strsvec, targets, ifppreg, ifppregtarg, nd,
              direct, thresh=1e-16):
    out = Output()
    if ifppreg == 0 and ifppregtarg == 0:
        print("Nothing to compute, set either ifppreg or ifppregtarg to non-zero")
        return out
    if stoklet is None and strslet is None and strsvec is None:
        print("Nothing to compute, set either stoklet or strslet+strsvec to non-None")
        return out
    if strslet is not None and strsvec is None:
        print("strslet and strsvec mush be both None or both not None")
        return out
    if strslet is None and strsvec is not None:
        print("strslet and strsvec mush be both None or both not None")
        return out
    assert sources.shape[0] == 2, "The first dimension of sources must be 2"
    ns = _ns_of(sources)
    if targets is not None:
        assert targets.shape[0] == 2, "The first dimension of targets must be 2"
    _st_check(stoklet, strslet, strsvec, nd, ns)
    return _st_run(eps, sources, stoklet, strslet, strsvec, targets, ifppreg, ifppregtarg, nd,
                   direct, thresh)


def stfmm2d(*, eps, sources, stoklet=None, strslet=None, strsvec=None, targets=None, ifppreg=0,
            ifppregtarg=0, nd=1):
    """Stokes FMM (fmm2d.py stfmm2d, src/stokes/stfmm2d.f): velocity (nd,2,n),
    pressure (nd,n) and velocity gradient (nd,2,2,n) of stokeslets and
    stresslets (nd,2,n each)."""
    return _st_front(eps, sources, stoklet, strslet, strsvec, targets, ifppreg, ifppregtarg, nd,
                     False)


def st2ddir(*, eps, sources, stoklet=None, strslet=None, strsvec=None, targets=None, ifppreg=0,
            ifppregtarg=0, nd=1, thresh=1e-16):
    """All-pairs Stokes sums (fmm2d.py st2ddir, stokkernels2d.f)."""
    return _st_front(eps, sources, stoklet, strslet, strsvec, targets, ifppreg, ifppregtarg, nd,
                     True, thresh)


def _np(a):
    if _is_torch(a):
        return a.detach().cpu().numpy()
    return np.asarray(a)


def comperr(*, ntest, out, outex, pg=0, pgt=0, nd=1, cauchy=0, bh=0):
    """sqrt(sum |out - outex|^2 / sum |outex|^2) over pot/grad/hess of the
    first ntest sources (pg) and targets (pgt), as in the reference."""
    r = 0.0
    err = 0.0

    def acc(a, b, real=False):
        nonlocal r, err
        a = _np(a)
        b = _np(b)
        if real:
            a, b = a.real, b.real
        r += la.norm(b.ravel()) ** 2
        err += la.norm((b - a).ravel()) ** 2

    gk = 3 if bh == 1 else 2

    def part(o, ox, level, kind):
        # kind: "pot", "grad", "hess"
        if nd == 1:
            if kind == "pot":
                acc(o[0:ntest], ox[0:ntest], real=(cauchy != 0))
            elif kind == "grad":
                if cauchy == 0:
                    acc(o[:, 0:ntest], ox[:, 0:ntest])
                else:
                    acc(o[0:ntest], ox[0:ntest])
            else:
                if cauchy == 0:
                    acc(o[:, 0:ntest], ox[:, 0:ntest])
                else:
                    acc(o[0:ntest], ox[0:ntest])
        else:
            if kind == "pot":
                acc(o[:, 0:ntest], ox[:, 0:ntest], real=(cauchy != 0))
            elif cauchy == 0:
                acc(o[:, :, 0:ntest], ox[:, :, 0:ntest])
            else:
                acc(o[:, 0:ntest], ox[:, 0:ntest])

    del gk
    if pg > 0:
        part(out.pot, outex.pot, pg, "pot")
    if pg >= 2:
        part(out.grad, outex.grad, pg, "grad")
    if pg >= 3:
        part(out.hess, outex.hess, pg, "hess")
    if pgt > 0:
        part(out.pottarg, outex.pottarg, pgt, "pot")
    if pgt >= 2:
        part(out.gradtarg, outex.gradtarg, pgt, "grad")
    if pgt >= 3:
        part(out.hesstarg, outex.hesstarg, pgt, "hess")
    return np.sqrt(err / r)
