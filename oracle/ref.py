"""ctypes front end of the reference itself (test infrastructure only).

``oracle/_ref/libfmm2d_ref.so`` is the reference's own Fortran (src/laplace,
src/helmholtz, src/common), translated to C by ``oracle/f77c.py`` and compiled
with gcc (``make -C oracle ref``; no Fortran compiler exists in this image).
It exports the reference's symbols with gfortran's calling convention, so the
functions below call exactly what a Fortran or f2py caller would:
``lfmm2d_`` (src/laplace/lfmm2d.f:29), ``rfmm2d_`` (rfmm2d.f:27), ``cfmm2d_``
(cfmm2d.f:23), ``hfmm2d_`` (src/helmholtz/hfmm2d.f:19), their ``_ndiv``
variants, the tree routines (src/common/pts_tree2d.f:34,406,1222,
tree_routs2d.f:459,486) and the direct sums.

The library is built in this container, where the reference's sources are;
the built ``.so`` travels with the repository snapshot.  ``available()`` says
whether it is present.  Only tests/, ``__graft_entry__`` and bench.py's
CPU-baseline legs use this module.

Inputs and outputs follow ``oracle/oracle.py``: sources ``(2, n)``, densities
``(nd, n)`` (or ``(n,)``), dipvec ``(nd, 2, n)``; outputs ``pot (nd, n)``,
``grad (nd, 2, n)``, ``hess (nd, 3, n)`` (Cauchy: ``(nd, n)`` each).
"""
import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(_HERE, "_ref", "libfmm2d_ref.so")
REFERENCE = os.environ.get("FMM2D_REFERENCE", "/root/reference")
_lib = None


def build(force=False):
    """Translates and compiles the reference (only where its sources are)."""
    if not os.path.isdir(REFERENCE):
        return LIBPATH if os.path.exists(LIBPATH) else None
    args = ["make", "-s", "-C", _HERE, "ref", f"REF={REFERENCE}"]
    if force:
        args.insert(2, "-B")
    subprocess.check_call(args)
    return LIBPATH


def available():
    return os.path.exists(LIBPATH)


def lib():
    global _lib
    if _lib is None:
        if not available():
            build()
        _lib = C.CDLL(LIBPATH)
        _lib.hkrand_.restype = C.c_double
        _lib.dlaran_.restype = C.c_double
    return _lib


def set_num_threads(n):
    """OpenMP threads of the reference's parallel loops."""
    gomp = C.CDLL("libgomp.so.1")
    gomp.omp_set_num_threads(C.c_int(int(n)))


def num_threads():
    gomp = C.CDLL("libgomp.so.1")
    return gomp.omp_get_max_threads()


def _i(v):
    return C.byref(C.c_int(int(v)))


def _d(v):
    return C.byref(C.c_double(float(v)))


def _z(v):
    v = complex(v)
    return C.byref((C.c_double * 2)(v.real, v.imag))


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def _pts(x):
    """(2, n) points in Fortran layout (2, n): n rows of (x, y)."""
    x = np.zeros((2, 0)) if x is None else np.asarray(x, dtype=np.float64)
    return np.ascontiguousarray(x.T), x.shape[1]


def _dens(a, nd, n, dt):
    if a is None:
        return np.zeros((max(n, 1), nd), dt)
    return np.ascontiguousarray(np.asarray(a).reshape(nd, n).T, dtype=dt)


def _dipvec(v, nd, n):
    if v is None:
        return np.zeros((max(n, 1), 2, nd))
    return np.ascontiguousarray(np.asarray(v, dtype=np.float64).reshape(nd, 2, n).transpose(2, 1, 0))


def _out(nd, n, k, dt):
    return np.zeros((max(n, 1), k, nd), dt)


def _lap(fn, dt, eps, sources, charges, dipstr, dipvec, targets, ifpgh, ifpghtarg, nd, ndiv,
         idivflag, ifnear):
    s, ns = _pts(sources)
    t, nt = _pts(targets)
    q = _dens(charges, nd, ns, dt)
    d = _dens(dipstr, nd, ns, dt)
    v = _dipvec(dipvec, nd, ns)
    pot, grad, hess = _out(nd, ns, 1, dt), _out(nd, ns, 2, dt), _out(nd, ns, 3, dt)
    pt, gt, ht = _out(nd, nt, 1, dt), _out(nd, nt, 2, dt), _out(nd, nt, 3, dt)
    ier = C.c_int(0)
    tinfo = np.zeros(8)
    common = [_i(nd), _d(eps), _i(ns), _p(s), _i(charges is not None), _p(q),
              _i(dipstr is not None), _p(d), _p(v), _i(0), _i(ifpgh), _p(pot), _p(grad), _p(hess),
              _i(nt), _p(t), _i(ifpghtarg), _p(pt), _p(gt), _p(ht)]
    if ndiv:
        getattr(lib(), fn + "_ndiv_")(*common, _i(ndiv), _i(idivflag), _i(ifnear), _p(tinfo),
                                      C.byref(ier))
    else:
        getattr(lib(), fn + "_")(*common, C.byref(ier))
    tr = lambda a, n: a[:n].transpose(2, 1, 0)
    return dict(pot=pot[:ns, 0].T, grad=tr(grad, ns), hess=tr(hess, ns), pottarg=pt[:nt, 0].T,
                gradtarg=tr(gt, nt), hesstarg=tr(ht, nt), timeinfo=tinfo, ier=ier.value)


def lfmm2d(eps, sources, charges=None, dipstr=None, dipvec=None, targets=None, ifpgh=0,
           ifpghtarg=0, nd=1, ndiv=0, idivflag=0, ifnear=1):
    """The reference's lfmm2d (src/laplace/lfmm2d.f:29); ndiv > 0 calls lfmm2d_ndiv."""
    return _lap("lfmm2d", np.complex128, eps, sources, charges, dipstr, dipvec, targets, ifpgh,
                ifpghtarg, nd, ndiv, idivflag, ifnear)


def rfmm2d(eps, sources, charges=None, dipstr=None, dipvec=None, targets=None, ifpgh=0,
           ifpghtarg=0, nd=1, ndiv=0, idivflag=0, ifnear=1):
    """The reference's rfmm2d (src/laplace/rfmm2d.f:27); real densities and outputs."""
    return _lap("rfmm2d", np.float64, eps, sources, charges, dipstr, dipvec, targets, ifpgh,
                ifpghtarg, nd, ndiv, idivflag, ifnear)


def cfmm2d(eps, sources, charges=None, dipstr=None, targets=None, ifpgh=0, ifpghtarg=0, nd=1,
           ndiv=0, idivflag=0, ifnear=1):
    """The reference's cfmm2d (src/laplace/cfmm2d.f:23); outputs (nd, n) complex."""
    s, ns = _pts(sources)
    t, nt = _pts(targets)
    q = _dens(charges, nd, ns, np.complex128)
    d = _dens(dipstr, nd, ns, np.complex128)
    outs = [np.zeros((max(n, 1), nd), np.complex128) for n in (ns, ns, ns, nt, nt, nt)]
    ier = C.c_int(0)
    tinfo = np.zeros(8)
    common = [_i(nd), _d(eps), _i(ns), _p(s), _i(charges is not None), _p(q),
              _i(dipstr is not None), _p(d), _i(0), _i(ifpgh), _p(outs[0]), _p(outs[1]),
              _p(outs[2]), _i(nt), _p(t), _i(ifpghtarg), _p(outs[3]), _p(outs[4]), _p(outs[5])]
    if ndiv:
        lib().cfmm2d_ndiv_(*common, _i(ndiv), _i(idivflag), _i(ifnear), _p(tinfo), C.byref(ier))
    else:
        lib().cfmm2d_(*common, C.byref(ier))
    k = ("pot", "grad", "hess", "pottarg", "gradtarg", "hesstarg")
    r = {name: o[:(ns if i < 3 else nt)].T for i, (name, o) in enumerate(zip(k, outs))}
    r.update(timeinfo=tinfo, ier=ier.value)
    return r


def hfmm2d(eps, zk, sources, charges=None, dipstr=None, dipvec=None, targets=None, ifpgh=0,
           ifpghtarg=0, nd=1, ndiv=0, idivflag=0, ifnear=1):
    """The reference's hfmm2d (src/helmholtz/hfmm2d.f:19), wideband path included."""
    s, ns = _pts(sources)
    t, nt = _pts(targets)
    dt = np.complex128
    q = _dens(charges, nd, ns, dt)
    d = _dens(dipstr, nd, ns, dt)
    v = _dipvec(dipvec, nd, ns)
    pot, grad, hess = _out(nd, ns, 1, dt), _out(nd, ns, 2, dt), _out(nd, ns, 3, dt)
    pt, gt, ht = _out(nd, nt, 1, dt), _out(nd, nt, 2, dt), _out(nd, nt, 3, dt)
    ier = C.c_int(0)
    tinfo = np.zeros(8)
    common = [_i(nd), _d(eps), _z(zk), _i(ns), _p(s), _i(charges is not None), _p(q),
              _i(dipstr is not None), _p(d), _p(v), _i(0), _i(ifpgh), _p(pot), _p(grad),
              _p(hess), _i(nt), _p(t), _i(ifpghtarg), _p(pt), _p(gt), _p(ht)]
    if ndiv:
        lib().hfmm2d_ndiv_(*common, _i(ndiv), _i(idivflag), _i(ifnear), _p(tinfo), C.byref(ier))
    else:
        lib().hfmm2d_(*common, C.byref(ier))
    tr = lambda a, n: a[:n].transpose(2, 1, 0)
    return dict(pot=pot[:ns, 0].T, grad=tr(grad, ns), hess=tr(hess, ns), pottarg=pt[:nt, 0].T,
                gradtarg=tr(gt, nt), hesstarg=tr(ht, nt), timeinfo=tinfo, ier=ier.value)


def lndiv2d(eps, ns, nt, ifcharge, ifdipole, ifpgh, ifpghtarg):
    """ndiv and idivflag of src/laplace/lndiv2d.f."""
    ndiv, idiv = C.c_int(0), C.c_int(0)
    lib().lndiv2d_(_d(eps), _i(ns), _i(nt), _i(ifcharge), _i(ifdipole), _i(ifpgh),
                   _i(ifpghtarg), C.byref(ndiv), C.byref(idiv))
    return ndiv.value, idiv.value


def l2dterms(eps):
    """nterms of src/laplace/l2dterms.f:38."""
    n, ier = C.c_int(0), C.c_int(0)
    lib().l2dterms_(_d(eps), C.byref(n), C.byref(ier))
    return n.value


def tree(sources, targets=None, idivflag=0, ndiv=15, nlmax=51):
    """The reference's adaptive tree, point sort and lists 1-4, in the
    conventions of ``oracle.tree``: 0-based boxes and points, -1 for none,
    half-open point ranges, lists padded with -1 to widths 13/27/20/5.

    Calls pts_tree_mem / pts_tree_build / pts_tree_sort
    (src/common/pts_tree2d.f:34,406,1222) and computemnlists / computelists
    (src/common/tree_routs2d.f:459,486) as cfmm2d does (cfmm2d.f:172-200,
    692-700): nlmin 0, ifunif 0, iper 0."""
    s, ns = _pts(sources)
    t, nt = _pts(targets)
    L = lib()
    nlevels, nboxes, ltree = C.c_int(0), C.c_int(0), C.c_int(0)
    L.pts_tree_mem_(_p(s), _i(ns), _p(t), _i(nt), _i(idivflag), _i(ndiv), _i(0), _i(nlmax),
                    _i(0), _i(0), C.byref(nlevels), C.byref(nboxes), C.byref(ltree))
    nl, nb, lt = nlevels.value, nboxes.value, ltree.value
    itree = np.zeros(lt, np.int32)
    iptr = np.zeros(8, np.int32)
    centers = np.zeros((nb, 2))
    boxsize = np.zeros(nl + 1)
    L.pts_tree_build_(_p(s), _i(ns), _p(t), _i(nt), _i(idivflag), _i(ndiv), _i(0), _i(nlmax),
                      _i(0), _i(0), _i(nl), _i(nb), _i(lt), _p(itree), _p(iptr), _p(centers),
                      _p(boxsize))
    isrc = np.zeros(max(ns, 1), np.int32)
    isrcse = np.zeros((nb, 2), np.int32)
    itarg = np.zeros(max(nt, 1), np.int32)
    itargse = np.zeros((nb, 2), np.int32)
    L.pts_tree_sort_(_i(ns), _p(s), _p(itree), _i(lt), _i(nb), _i(nl), _p(iptr), _p(centers),
                     _p(isrc), _p(isrcse))
    L.pts_tree_sort_(_i(nt), _p(t), _p(itree), _i(lt), _i(nb), _i(nl), _p(iptr), _p(centers),
                     _p(itarg), _p(itargse))
    mn = [C.c_int(0) for _ in range(4)]
    L.computemnlists_(_i(nl), _i(nb), _p(itree), _i(lt), _p(iptr), _p(centers), _p(boxsize),
                      _i(0), *[C.byref(m) for m in mn])
    mn = [m.value for m in mn]
    nls = [np.zeros(nb, np.int32) for _ in range(4)]
    lsts = [np.zeros((nb, max(m, 1)), np.int32) for m in mn]
    args = []
    for k in range(4):
        args += [_i(mn[k]), _p(nls[k]), _p(lsts[k])]
    L.computelists_(_i(nl), _i(nb), _p(itree), _i(lt), _p(iptr), _p(centers), _p(boxsize),
                    _i(0), *args)
    ip = [int(x) - 1 for x in iptr]
    box = lambda k, w=1: itree[ip[k]:ip[k] + w * nb]
    laddr = itree[:2 * (nl + 1)].reshape(nl + 1, 2) - 1
    zb = lambda a: np.where(a > 0, a - 1, -1).astype(np.int32)
    out = dict(nlevels=nl, nboxes=nb, laddr=laddr.astype(np.int32),
               ilevel=box(1).astype(np.int32), iparent=zb(box(2)),
               nchild=box(3).astype(np.int32), ichild=zb(box(4, 4).reshape(nb, 4)),
               ncoll=box(5).astype(np.int32), coll=zb(box(6, 9).reshape(nb, 9)),
               centers=centers, boxsize=boxsize, isrc=(isrc[:ns] - 1).astype(np.int32),
               isrcse=np.stack([isrcse[:, 0] - 1, isrcse[:, 1]], axis=1).astype(np.int32),
               itarg=(itarg[:nt] - 1).astype(np.int32),
               itargse=np.stack([itargse[:, 0] - 1, itargse[:, 1]], axis=1).astype(np.int32))
    widths = (13, 27, 20, 5)
    for k in range(4):
        full = np.full((nb, widths[k]), -1, np.int32)
        w = min(widths[k], lsts[k].shape[1])
        full[:, :w] = zb(lsts[k][:, :w])
        for b in range(nb):
            full[b, nls[k][b]:] = -1
        out[f"nlist{k + 1}"] = nls[k]
        out[f"list{k + 1}"] = full
    return out


def hkrand(n, seed=None):
    """n values of the reference's test generator hkrand (src/common/hkrand.f).
    With ``seed`` the generator restarts from state (0, 0, 0, 2 seed + 1 mod
    4096) first, as ``hkrand(seed)`` does for seed != 0 (seed 0 restarts the
    initial DATA state, which hkrand(2048) reaches)."""
    L = lib()
    out = []
    if seed is not None and n > 0:
        out.append(L.hkrand_(_i(seed if seed != 0 else 2048)))
    while len(out) < n:
        out.append(L.hkrand_(_i(0)))
    return np.array(out)


def direct(kind, sources, targets, charges=None, dipstr=None, dipvec=None, ifpgh=1, nd=1,
           thresh=1e-16, zk=None):
    """The reference's direct sums: kind 'c' (c2d_direct*, cauchykernels2d.f),
    'l' (l2d_direct*, lapkernels2d.f), 'r' (r2d_direct*, rlapkernels2d.f), 'h'
    (h2d_direct*, helmkernels2d.f).  Returns pottarg / gradtarg / hesstarg."""
    s, ns = _pts(sources)
    t, nt = _pts(targets)
    dt = np.float64 if kind == "r" else np.complex128
    q = _dens(charges, nd, ns, dt)
    d = _dens(dipstr, nd, ns, dt)
    v = _dipvec(dipvec, nd, ns)
    cauchy = kind == "c"
    pot = np.zeros((max(nt, 1), nd), dt)
    grad = np.zeros((max(nt, 1), nd) if cauchy else (max(nt, 1), 2, nd), dt)
    hess = np.zeros((max(nt, 1), nd) if cauchy else (max(nt, 1), 3, nd), dt)
    tag = ("c" if charges is not None else "") + ("d" if dipstr is not None else "")
    tag += "pgh"[ifpgh - 1]
    fn = getattr(lib(), f"{kind}2d_direct{tag}_")
    head = [_i(nd)] + ([_z(zk)] if kind == "h" else []) + [_p(s), _i(ns)]
    dens = []
    if charges is not None:
        dens.append(_p(q))
    if dipstr is not None:
        dens.append(_p(d))
        if not cauchy:
            dens.append(_p(v))
    outs = [_p(pot)] + ([_p(grad)] if ifpgh >= 2 else []) + ([_p(hess)] if ifpgh >= 3 else [])
    fn(*head, *dens, _p(t), _i(nt), *outs, _d(thresh))
    if cauchy:
        return dict(pottarg=pot[:nt].T, gradtarg=grad[:nt].T, hesstarg=hess[:nt].T)
    tr = lambda a: a[:nt].transpose(2, 1, 0)
    return dict(pottarg=pot[:nt].T, gradtarg=tr(grad), hesstarg=tr(hess))
