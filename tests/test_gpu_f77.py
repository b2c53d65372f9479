"""libfmm2d.so against the reference library, routine by routine.

Every flag wrapper {c,l,r,h}fmm2d_{s,t,st}_{c,d,cd}_{p,g,h}[_vec] (216), the
core routines, their _ndiv variants and the C function hfmm2d_s_c_p are
called with the same host arrays in both libraries (the reference: its own
Fortran, oracle/_ref).  At eps 1e-9 both run the FP64 algorithm on the same
tree with the same expansion orders, so the outputs agree to round-off.
"""
import ctypes as C
import os

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EPS = 1e-9
TOL = {"c": 1e-11, "l": 1e-11, "r": 1e-11, "h": 1e-10}
ZK = 12.0 + 0.5j
NS, NT = 900, 700


@pytest.fixture(scope="module")
def libs(gpu, ref):
    return C.CDLL(os.path.join(ROOT, "fmm2d_b200", "libfmm2d.so")), ref.lib()


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p)


class Case:
    """Host arrays in the reference's column-major layout (numpy arrays
    with the Fortran index order reversed)."""

    def __init__(self, fam, nd, seed):
        rng = np.random.default_rng(seed)
        real = fam == "r"
        self.fam, self.nd = fam, nd
        cx = (lambda *s: rng.normal(size=s)) if real else (
            lambda *s: rng.normal(size=s) + 1j * rng.normal(size=s))
        self.src = rng.uniform(0, 1, (NS, 2))
        self.trg = rng.uniform(-0.1, 1.1, (NT, 2))
        self.charge = np.ascontiguousarray(cx(NS, nd))
        self.dipstr = np.ascontiguousarray(cx(NS, nd))
        self.dipvec = rng.uniform(-1, 1, (NS, 2, nd))
        self.zk = np.array([ZK.real, ZK.imag])

    def outputs(self, n):
        dt = np.float64 if self.fam == "r" else np.complex128
        g, h = (1, 1) if self.fam == "c" else (2, 3)
        return [np.full((n, self.nd), np.nan, dt), np.full((n, g, self.nd), np.nan, dt),
                np.full((n, h, self.nd), np.nan, dt)]

    def wrapper_args(self, kind, dens, out, vec):
        """Argument list of {fam}fmm2d_{kind}_{dens}_{out}[_vec] and the
        output arrays it writes."""
        lvl = "pgh".index(out) + 1
        a = [C.byref(C.c_int(self.nd))] if vec else []
        a += [C.byref(C.c_double(EPS))]
        if self.fam == "h":
            a.append(_ptr(self.zk))
        a += [C.byref(C.c_int(NS)), _ptr(self.src)]
        if "c" in dens:
            a.append(_ptr(self.charge))
        if "d" in dens:
            a.append(_ptr(self.dipstr))
            if self.fam != "c":
                a.append(_ptr(self.dipvec))
        outs = []
        if kind in ("s", "st"):
            o = self.outputs(NS)[:lvl]
            a += [_ptr(x) for x in o]
            outs += o
        if kind in ("t", "st"):
            o = self.outputs(NT)[:lvl]
            a += [C.byref(C.c_int(NT)), _ptr(self.trg)] + [_ptr(x) for x in o]
            outs += o
        ier = C.c_int(-1)
        a.append(C.byref(ier))
        return a, outs, ier


def _wrappers():
    for fam in "clrh":
        for kind in ("s", "t", "st"):
            for dens in ("c", "d", "cd"):
                for out in "pgh":
                    yield fam, kind, dens, out


@pytest.mark.parametrize("fam", list("clrh"))
@pytest.mark.parametrize("vec", [False, True])
def test_flag_wrappers_match_the_reference(libs, fam, vec):
    ours, theirs = libs
    case = Case(fam, 2 if vec else 1, seed=2 * "clrh".index(fam) + vec)
    bad = []
    for f, kind, dens, out in _wrappers():
        if f != fam:
            continue
        name = f"{fam}fmm2d_{kind}_{dens}_{out}_" + ("vec_" if vec else "")
        a1, o1, ier1 = case.wrapper_args(kind, dens, out, vec)
        a2, o2, ier2 = case.wrapper_args(kind, dens, out, vec)
        getattr(ours, name)(*a1)
        getattr(theirs, name)(*a2)
        assert ier1.value == 0 and ier2.value == 0, name
        for x, y in zip(o1, o2):
            assert np.isfinite(x).all(), name
            e = rel_l2(x, y)
            if not e < TOL[fam]:
                bad.append((name, e))
    assert not bad, bad


def _core_args(case, lib_nd, lvl, with_ndiv):
    fam = case.fam
    a = [C.byref(C.c_int(lib_nd)), C.byref(C.c_double(EPS))]
    if fam == "h":
        a.append(_ptr(case.zk))
    a += [C.byref(C.c_int(NS)), _ptr(case.src), C.byref(C.c_int(1)), _ptr(case.charge),
          C.byref(C.c_int(1)), _ptr(case.dipstr)]
    if fam != "c":
        a.append(_ptr(case.dipvec))
    so, to = case.outputs(NS), case.outputs(NT)
    a += [C.byref(C.c_int(0)), C.byref(C.c_int(lvl))] + [_ptr(x) for x in so]
    a += [C.byref(C.c_int(NT)), _ptr(case.trg), C.byref(C.c_int(lvl))] + [_ptr(x) for x in to]
    t = np.zeros(8)
    if with_ndiv:
        a += [C.byref(C.c_int(25)), C.byref(C.c_int(0)), C.byref(C.c_int(1)), _ptr(t)]
    ier = C.c_int(-1)
    a.append(C.byref(ier))
    return a, so[:lvl] + to[:lvl], ier


@pytest.mark.parametrize("fam", list("clrh"))
@pytest.mark.parametrize("ndiv", [False, True])
def test_core_routines_match_the_reference(libs, fam, ndiv):
    ours, theirs = libs
    case = Case(fam, 3, seed=40 + "clrh".index(fam))
    name = f"{fam}fmm2d_" + ("ndiv_" if ndiv else "")
    a1, o1, ier1 = _core_args(case, 3, 3, ndiv)
    a2, o2, ier2 = _core_args(case, 3, 3, ndiv)
    getattr(ours, name)(*a1)
    getattr(theirs, name)(*a2)
    assert ier1.value == 0 and ier2.value == 0
    for x, y in zip(o1, o2):
        assert rel_l2(x, y) < TOL[fam], name


class Zk(C.Structure):
    """double _Complex passed by value (two doubles, as the x86-64 ABI passes it)."""
    _fields_ = [("re", C.c_double), ("im", C.c_double)]


def test_c_declaration_hfmm2d_s_c_p(libs):
    """include/fmm2d/helmholtz.h:10 of the reference: by-value eps and zk,
    64-bit sizes."""
    ours, theirs = libs
    case = Case("h", 1, seed=77)
    pot = np.full(NS, np.nan, np.complex128)
    ier = C.c_int64(-1)
    f = ours.hfmm2d_s_c_p
    f.argtypes = [C.c_double, Zk, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p,
                  C.POINTER(C.c_int64)]
    f(EPS, Zk(ZK.real, ZK.imag), NS, _ptr(case.src), _ptr(case.charge), _ptr(pot), C.byref(ier))
    a, o, ier2 = case.wrapper_args("s", "c", "p", False)
    theirs.hfmm2d_s_c_p_(*a)
    assert ier.value == 0 and ier2.value == 0
    assert rel_l2(pot, o[0][:, 0]) < TOL["h"]
