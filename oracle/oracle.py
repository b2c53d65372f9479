"""ctypes front end of the CPU oracle (test infrastructure only).

Loads ``oracle/liboracle_fmm2d.so`` (built from ``fmm2d_oracle.cpp`` by
``oracle/Makefile``) and exposes the oracle's FMM drivers, tree/list export and
direct sums with numpy arrays in the reference's layouts.  Only tests/,
``__graft_entry__.smoke()`` and bench.py's CPU-baseline legs import this.
"""
import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIBPATH = os.path.join(_HERE, "liboracle_fmm2d.so")
_lib = None

MNL = (13, 27, 20, 5)


def build(force=False):
    """Compile the oracle with its Makefile (g++ -O3 -fopenmp)."""
    if force or not os.path.exists(_LIBPATH) or (
        os.path.getmtime(_LIBPATH) < os.path.getmtime(os.path.join(_HERE, "fmm2d_oracle.cpp"))
    ):
        subprocess.check_call(["make", "-s", "-C", _HERE, "CXX=g++"])
    return _LIBPATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIBPATH):
            build()
        _lib = C.CDLL(_LIBPATH)
        _lib.orc_tree_new.restype = C.c_void_p
        _lib.orc_num_threads.restype = C.c_int
        _lib.orc_lap_ndiv.restype = C.c_int
        _lib.orc_lap_ndiv.argtypes = [C.c_double]
        _lib.orc_lap_nterms.restype = C.c_int
        _lib.orc_lap_nterms.argtypes = [C.c_double]
    return _lib


def _p(a):
    if a is None:
        return None
    return a.ctypes.data_as(C.c_void_p)


def _f64(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float64)


def _c128(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.complex128)


def num_threads():
    return lib().orc_num_threads()


def set_num_threads(n):
    lib().orc_set_num_threads(C.c_int(int(n)))


def lap_ndiv(eps):
    return lib().orc_lap_ndiv(eps)


def lap_nterms(eps):
    return lib().orc_lap_nterms(eps)


def tree(sources, targets=None, idivflag=0, ndiv=15, nlmax=51):
    """Reference tree (after level restriction), point sort and lists 1-4."""
    s = _f64(sources.T)  # (n,2) row-major == Fortran (2,n)
    ns = s.shape[0]
    t = _f64(np.zeros((2, 0)) .T if targets is None else targets.T)
    nt = t.shape[0]
    L = lib()
    nl, nb = C.c_int(), C.c_int()
    h = L.orc_tree_new(_p(s), C.c_int(ns), _p(t), C.c_int(nt), C.c_int(idivflag), C.c_int(ndiv),
                       C.c_int(nlmax), C.byref(nl), C.byref(nb))
    nl, nb = nl.value, nb.value
    i32 = lambda *shape: np.zeros(shape, dtype=np.int32)
    out = dict(nlevels=nl, nboxes=nb, laddr=i32(nl + 1, 2), ilevel=i32(nb), iparent=i32(nb),
               nchild=i32(nb), ichild=i32(nb, 4), ncoll=i32(nb), coll=i32(nb, 9),
               centers=np.zeros((nb, 2)), boxsize=np.zeros(nl + 1), isrc=i32(ns),
               isrcse=i32(nb, 2), itarg=i32(nt), itargse=i32(nb, 2))
    L.orc_tree_get(C.c_void_p(h), *[_p(out[k]) for k in (
        "laddr", "ilevel", "iparent", "nchild", "ichild", "ncoll", "coll", "centers", "boxsize",
        "isrc", "isrcse", "itarg", "itargse")])
    lists = dict(nlist1=i32(nb), list1=i32(nb, MNL[0]), nlist2=i32(nb), list2=i32(nb, MNL[1]),
                 nlist3=i32(nb), list3=i32(nb, MNL[2]), nlist4=i32(nb), list4=i32(nb, MNL[3]))
    L.orc_tree_lists(C.c_void_p(h), *[_p(lists[k]) for k in (
        "nlist1", "list1", "nlist2", "list2", "nlist3", "list3", "nlist4", "list4")])
    out.update(lists)
    L.orc_tree_free(C.c_void_p(h))
    return out


def _alloc_c(nd, n, k=1, dtype=np.complex128):
    return np.zeros((n, k, nd), dtype=dtype)


def cfmm2d(eps, sources, charges=None, dipstr=None, targets=None, ifpgh=0, ifpghtarg=0, nd=1,
           ndiv=0, idivflag=0, ifnear=1):
    """Oracle cfmm2d.  Densities (nd, n) complex; returns dict of (nd, n) outputs."""
    s = _f64(sources.T)
    ns = s.shape[0]
    t = _f64(np.zeros((0, 2)) if targets is None else targets.T)
    nt = t.shape[0]
    q = None if charges is None else _c128(np.asarray(charges).reshape(nd, ns).T)
    d = None if dipstr is None else _c128(np.asarray(dipstr).reshape(nd, ns).T)
    pot, grad, hess = (np.zeros((max(ns, 1), nd), np.complex128) for _ in range(3))
    pt, gt, ht = (np.zeros((max(nt, 1), nd), np.complex128) for _ in range(3))
    tinfo = np.zeros(8)
    ier = C.c_int(0)
    lib().orc_cfmm2d(C.c_int(nd), C.c_double(eps), C.c_int(ns), _p(s), C.c_int(q is not None),
                     _p(q), C.c_int(d is not None), _p(d), C.c_int(ifpgh), _p(pot), _p(grad),
                     _p(hess), C.c_int(nt), _p(t), C.c_int(ifpghtarg), _p(pt), _p(gt), _p(ht),
                     C.c_int(ndiv), C.c_int(idivflag), C.c_int(ifnear), _p(tinfo), C.byref(ier))
    return dict(pot=pot[:ns].T, grad=grad[:ns].T, hess=hess[:ns].T, pottarg=pt[:nt].T,
                gradtarg=gt[:nt].T, hesstarg=ht[:nt].T, timeinfo=tinfo, ier=ier.value)


def _lap_common(fn, dt, eps, sources, charges, dipstr, dipvec, targets, ifpgh, ifpghtarg, nd,
                ndiv):
    s = _f64(sources.T)
    ns = s.shape[0]
    t = _f64(np.zeros((0, 2)) if targets is None else targets.T)
    nt = t.shape[0]
    cv = (lambda a: np.ascontiguousarray(np.asarray(a).reshape(nd, ns).T, dtype=dt))
    q = None if charges is None else cv(charges)
    d = None if dipstr is None else cv(dipstr)
    v = None if dipvec is None else _f64(np.asarray(dipvec).reshape(nd, 2, ns).transpose(2, 1, 0))
    pot = np.zeros((max(ns, 1), nd), dt)
    grad = np.zeros((max(ns, 1), 2, nd), dt)
    hess = np.zeros((max(ns, 1), 3, nd), dt)
    pt = np.zeros((max(nt, 1), nd), dt)
    gt = np.zeros((max(nt, 1), 2, nd), dt)
    ht = np.zeros((max(nt, 1), 3, nd), dt)
    tinfo = np.zeros(8)
    ier = C.c_int(0)
    fn(C.c_int(nd), C.c_double(eps), C.c_int(ns), _p(s), C.c_int(q is not None), _p(q),
       C.c_int(d is not None), _p(d), _p(v), C.c_int(ifpgh), _p(pot), _p(grad), _p(hess),
       C.c_int(nt), _p(t), C.c_int(ifpghtarg), _p(pt), _p(gt), _p(ht), C.c_int(ndiv), _p(tinfo),
       C.byref(ier))
    return dict(pot=pot[:ns].T, grad=grad[:ns].transpose(2, 1, 0),
                hess=hess[:ns].transpose(2, 1, 0), pottarg=pt[:nt].T,
                gradtarg=gt[:nt].transpose(2, 1, 0), hesstarg=ht[:nt].transpose(2, 1, 0),
                timeinfo=tinfo, ier=ier.value)


def lfmm2d(eps, sources, charges=None, dipstr=None, dipvec=None, targets=None, ifpgh=0,
           ifpghtarg=0, nd=1, ndiv=0):
    """Oracle lfmm2d; outputs pot (nd,n), grad (nd,2,n), hess (nd,3,n)."""
    return _lap_common(lib().orc_lfmm2d, np.complex128, eps, sources, charges, dipstr, dipvec,
                       targets, ifpgh, ifpghtarg, nd, ndiv)


def rfmm2d(eps, sources, charges=None, dipstr=None, dipvec=None, targets=None, ifpgh=0,
           ifpghtarg=0, nd=1, ndiv=0):
    """Oracle rfmm2d (real densities)."""
    return _lap_common(lib().orc_rfmm2d, np.float64, eps, sources, charges, dipstr, dipvec,
                       targets, ifpgh, ifpghtarg, nd, ndiv)


def c2ddir(sources, targets, charges=None, dipstr=None, ifpgh=1, nd=1, thresh=1e-16):
    s = _f64(sources.T)
    t = _f64(targets.T)
    ns, nt = s.shape[0], t.shape[0]
    q = None if charges is None else _c128(np.asarray(charges).reshape(nd, ns).T)
    d = None if dipstr is None else _c128(np.asarray(dipstr).reshape(nd, ns).T)
    pot, grad, hess = (np.zeros((nt, nd), np.complex128) for _ in range(3))
    lib().orc_c2ddir(C.c_int(nd), _p(s), C.c_int(ns), _p(q), _p(d), _p(t), C.c_int(nt),
                     C.c_int(ifpgh), _p(pot), _p(grad), _p(hess), C.c_double(thresh))
    return dict(pottarg=pot.T, gradtarg=grad.T, hesstarg=hess.T)


def _ldir(fn, dt, sources, targets, charges, dipstr, dipvec, ifpgh, nd, thresh):
    s = _f64(sources.T)
    t = _f64(targets.T)
    ns, nt = s.shape[0], t.shape[0]
    cv = (lambda a: np.ascontiguousarray(np.asarray(a).reshape(nd, ns).T, dtype=dt))
    q = None if charges is None else cv(charges)
    d = None if dipstr is None else cv(dipstr)
    v = None if dipvec is None else _f64(np.asarray(dipvec).reshape(nd, 2, ns).transpose(2, 1, 0))
    pot = np.zeros((nt, nd), dt)
    grad = np.zeros((nt, 2, nd), dt)
    hess = np.zeros((nt, 3, nd), dt)
    fn(C.c_int(nd), _p(s), C.c_int(ns), _p(q), _p(d), _p(v), _p(t), C.c_int(nt), C.c_int(ifpgh),
       _p(pot), _p(grad), _p(hess), C.c_double(thresh))
    return dict(pottarg=pot.T, gradtarg=grad.transpose(2, 1, 0), hesstarg=hess.transpose(2, 1, 0))


def l2ddir(sources, targets, charges=None, dipstr=None, dipvec=None, ifpgh=1, nd=1, thresh=1e-16):
    return _ldir(lib().orc_l2ddir, np.complex128, sources, targets, charges, dipstr, dipvec, ifpgh,
                 nd, thresh)


def r2ddir(sources, targets, charges=None, dipstr=None, dipvec=None, ifpgh=1, nd=1, thresh=1e-16):
    return _ldir(lib().orc_r2ddir, np.float64, sources, targets, charges, dipstr, dipvec, ifpgh,
                 nd, thresh)


def hkrand(n, seed=None):
    """Reference test RNG (hkrand/dlaran); seed=None continues the stream."""
    if seed is not None:
        lib().orc_hkrand_seed(C.c_int(seed))
    out = np.zeros(n)
    lib().orc_hkrand_fill(_p(out), C.c_long(n))
    return out


# ---------------------------------------------------------------- Helmholtz
def hfmm2d(eps, zk, sources, charges=None, dipstr=None, dipvec=None, targets=None, ifpgh=0,
           ifpghtarg=0, nd=1, ndiv=0):
    """Oracle hfmm2d; outputs pot (nd,n), grad (nd,2,n), hess (nd,3,n) complex."""
    s = _f64(sources.T)
    ns = s.shape[0]
    t = _f64(np.zeros((0, 2)) if targets is None else targets.T)
    nt = t.shape[0]
    cv = (lambda a: np.ascontiguousarray(np.asarray(a).reshape(nd, ns).T, dtype=np.complex128))
    q = None if charges is None else cv(charges)
    d = None if dipstr is None else cv(dipstr)
    v = None if dipvec is None else _f64(np.asarray(dipvec).reshape(nd, 2, ns).transpose(2, 1, 0))
    pot = np.zeros((max(ns, 1), nd), np.complex128)
    grad = np.zeros((max(ns, 1), 2, nd), np.complex128)
    hess = np.zeros((max(ns, 1), 3, nd), np.complex128)
    pt = np.zeros((max(nt, 1), nd), np.complex128)
    gt = np.zeros((max(nt, 1), 2, nd), np.complex128)
    ht = np.zeros((max(nt, 1), 3, nd), np.complex128)
    tinfo = np.zeros(8)
    ier = C.c_int(0)
    zk = complex(zk)
    lib().orc_hfmm2d(C.c_int(nd), C.c_double(eps), C.c_double(zk.real), C.c_double(zk.imag),
                     C.c_int(ns), _p(s), C.c_int(q is not None), _p(q), C.c_int(d is not None),
                     _p(d), _p(v), C.c_int(ifpgh), _p(pot), _p(grad), _p(hess), C.c_int(nt), _p(t),
                     C.c_int(ifpghtarg), _p(pt), _p(gt), _p(ht), C.c_int(ndiv), _p(tinfo),
                     C.byref(ier))
    return dict(pot=pot[:ns].T, grad=grad[:ns].transpose(2, 1, 0),
                hess=hess[:ns].transpose(2, 1, 0), pottarg=pt[:nt].T,
                gradtarg=gt[:nt].transpose(2, 1, 0), hesstarg=ht[:nt].transpose(2, 1, 0),
                timeinfo=tinfo, ier=ier.value)


def h2ddir(zk, sources, targets, charges=None, dipstr=None, dipvec=None, ifpgh=1, nd=1,
           thresh=1e-16):
    s = _f64(sources.T)
    t = _f64(targets.T)
    ns, nt = s.shape[0], t.shape[0]
    cv = (lambda a: np.ascontiguousarray(np.asarray(a).reshape(nd, ns).T, dtype=np.complex128))
    q = None if charges is None else cv(charges)
    d = None if dipstr is None else cv(dipstr)
    v = None if dipvec is None else _f64(np.asarray(dipvec).reshape(nd, 2, ns).transpose(2, 1, 0))
    pot = np.zeros((nt, nd), np.complex128)
    grad = np.zeros((nt, 2, nd), np.complex128)
    hess = np.zeros((nt, 3, nd), np.complex128)
    zk = complex(zk)
    lib().orc_h2ddir(C.c_int(nd), C.c_double(zk.real), C.c_double(zk.imag), _p(s), C.c_int(ns),
                     _p(q), _p(d), _p(v), _p(t), C.c_int(nt), C.c_int(ifpgh), _p(pot), _p(grad),
                     _p(hess), C.c_double(thresh))
    return dict(pottarg=pot.T, gradtarg=grad.transpose(2, 1, 0), hesstarg=hess.transpose(2, 1, 0))


def hankel01(z):
    out = np.zeros(4)
    lib().orc_hankel01(C.c_double(complex(z).real), C.c_double(complex(z).imag), _p(out))
    return complex(out[0], out[1]), complex(out[2], out[3])


def jbessel2d(nterms, z, rscale):
    out = np.zeros(nterms + 1, np.complex128)
    z = complex(z)
    lib().orc_jbessel2d(C.c_int(nterms), C.c_double(z.real), C.c_double(z.imag),
                        C.c_double(rscale), _p(out))
    return out


def h2dall(nterms, z, rscale):
    out = np.zeros(nterms + 1, np.complex128)
    z = complex(z)
    lib().orc_h2dall(C.c_int(nterms), C.c_double(z.real), C.c_double(z.imag), C.c_double(rscale),
                     _p(out))
    return out


def h2dterms(bsize, zk, eps):
    zk = complex(zk)
    lib().orc_h2dterms.restype = C.c_int
    return lib().orc_h2dterms(C.c_double(bsize), C.c_double(zk.real), C.c_double(zk.imag),
                              C.c_double(eps))
