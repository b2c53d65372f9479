"""hfmm2d_mps (the FMM over multipole expansions) against the reference.

Inputs follow the reference's own test (test/helmholtz/test_hfmm2d_mps.f90):
sources on a grid, expansion centres shifted by h/100, the multipoles formed
from the sources' charges by the reference's h2dformmpc; here every source
carries a charge and the orders vary from expansion to expansion.  Checks:
  * the local expansions equal the reference's hfmm2d_mps to round-off;
  * evaluated at the sources (h2dtaevalp), they give the potential of all
    the other charges within the requested precision (the reference test's
    criterion, against the reference's hfmm2d);
  * the same through the Fortran entry point of libfmm2d.so;
  * larger irregular sets (uniform and clustered centres), nd 1, 2 and 3.
"""
import ctypes as C
import os

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TOL_REF = 1e-10  # local expansions against the reference's, FP64 both


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


class Mps:
    """Expansions about centres next to sources, formed by the reference."""

    def __init__(self, r, src, nd, zk, orders, shift, seed):
        rng = np.random.default_rng(seed)
        n = src.shape[1]
        self.nd, self.zk, self.n = nd, zk, n
        self.src = np.asfortranarray(src)
        self.cen = np.asfortranarray(src + np.array([[shift], [0.0]]))
        self.charge = np.asfortranarray(rng.normal(size=(nd, n)) + 1j * rng.normal(size=(nd, n)))
        self.mterms = np.asarray(orders, dtype=np.int32)
        sizes = nd * (2 * self.mterms + 1)
        self.impole = (1 + np.concatenate([[0], np.cumsum(sizes)[:-1]])).astype(np.int32)
        self.ntot = int(sizes.sum())
        sc = abs(zk) * shift
        self.rs = np.full(n, sc if sc < 1 else 1.0)
        self.mpole = np.zeros(self.ntot, np.complex128)
        zka = np.array([zk.real, zk.imag])
        for i in range(n):
            o = self.impole[i] - 1
            blk = np.zeros((2 * self.mterms[i] + 1, nd), np.complex128)  # (nd, -m:m) column-major
            q = np.ascontiguousarray(self.charge[:, i])
            r.h2dformmpc_(C.byref(C.c_int(nd)), _p(zka), C.byref(C.c_double(self.rs[i])),
                          _p(np.ascontiguousarray(self.src[:, i])), C.byref(C.c_int(1)), _p(q),
                          _p(np.ascontiguousarray(self.cen[:, i])),
                          C.byref(C.c_int(int(self.mterms[i]))), _p(blk))
            self.mpole[o:o + blk.size] = blk.ravel()

    def ours(self, eps):
        from fmm2d_b200 import _lib
        local = np.zeros(self.ntot, np.complex128)
        ier = C.c_int(-1)
        _lib.lib().b2fmm_hfmm2d_mps(self.nd, eps, self.zk.real, self.zk.imag, self.n, _p(self.cen),
                                    _p(self.rs), _p(self.mterms), self.ntot, _p(self.mpole),
                                    _p(self.impole), _p(local), C.byref(ier))
        return ier.value, local

    def fortran(self, lib, eps):
        local = np.zeros(self.ntot, np.complex128)
        ier = C.c_int(-1)
        zka = np.array([self.zk.real, self.zk.imag])
        lib.hfmm2d_mps_(C.byref(C.c_int(self.nd)), C.byref(C.c_double(eps)), _p(zka),
                        C.byref(C.c_int(self.n)), _p(self.cen), _p(self.rs), _p(self.mterms),
                        C.byref(C.c_int(self.ntot)), _p(self.mpole), _p(self.impole), _p(local),
                        C.byref(ier))
        return ier.value, local

    def evaluate(self, r, local):
        """Each local expansion at its own source (h2dtaevalp)."""
        zka = np.array([self.zk.real, self.zk.imag])
        pot = np.zeros((self.n, self.nd), np.complex128)
        for i in range(self.n):
            o = self.impole[i] - 1
            m = int(self.mterms[i])
            blk = np.ascontiguousarray(local[o:o + self.nd * (2 * m + 1)])
            out = np.zeros(self.nd, np.complex128)
            r.h2dtaevalp_(C.byref(C.c_int(self.nd)), _p(zka), C.byref(C.c_double(self.rs[i])),
                          _p(np.ascontiguousarray(self.cen[:, i])), _p(blk), C.byref(C.c_int(m)),
                          _p(np.ascontiguousarray(self.src[:, i])), C.byref(C.c_int(1)), _p(out))
            pot[i] = out
        return pot.T


def _grid(n1):
    h = 1.0 / (n1 + 1)
    g = np.arange(1, n1 + 1) * h
    x, y = np.meshgrid(g, g, indexing="ij")
    return np.stack([x.ravel(), y.ravel()]), h


@pytest.mark.parametrize("nd", [1, 2, 3])
def test_reference_case_matches_reference(gpu, ref, nd):
    r = ref.lib()
    src, h = _grid(10)
    n = src.shape[1]
    zk = 2 * np.pi + 0j
    orders = 30 + (np.arange(n) % 5) - 2
    m = Mps(r, src, nd, zk, orders, h / 100, seed=nd)
    eps = 0.5e-9
    ier, loc = m.ours(eps)
    ier_r, loc_r = m.fortran(r, eps)
    assert ier == 0 and ier_r == 0
    assert rel_l2(loc, loc_r) < TOL_REF
    # the reference test's check: the local expansions reproduce the FMM
    # potential of all the other charges at the sources
    out = ref.hfmm2d(eps, zk, src, charges=m.charge, ifpgh=1, nd=nd)
    assert rel_l2(m.evaluate(r, loc), out["pot"]) < 1e-8


def test_fortran_entry_point(gpu, ref):
    r = ref.lib()
    f77 = C.CDLL(os.path.join(ROOT, "fmm2d_b200", "libfmm2d.so"))
    src, h = _grid(8)
    m = Mps(r, src, 1, 6.0 + 0.2j, np.full(src.shape[1], 20), h / 50, seed=5)
    ier, loc = m.fortran(f77, 1e-9)
    ier_r, loc_r = m.fortran(r, 1e-9)
    assert ier == 0 and ier_r == 0
    assert rel_l2(loc, loc_r) < TOL_REF


@pytest.mark.parametrize("kind", ["uniform", "clustered"])
def test_irregular_centres(gpu, ref, kind):
    r = ref.lib()
    rng = np.random.default_rng(11)
    n = 1500
    if kind == "uniform":
        src = rng.uniform(0, 1, (2, n))
    else:
        ctr = rng.uniform(0.2, 0.8, (2, 6))
        src = ctr[:, rng.integers(0, 6, n)] + 0.02 * rng.normal(size=(2, n))
    zk = 15.0 + 0.3j
    # centres 1e-6 from their sources, well below the closest pair of
    # sources (~1e-4), so that every expansion converges where it is used
    m = Mps(r, src, 2, zk, 8 + rng.integers(0, 8, n), 1e-6, seed=12)
    ier, loc = m.ours(1e-9)
    ier_r, loc_r = m.fortran(r, 1e-9)
    assert ier == 0 and ier_r == 0
    assert rel_l2(loc, loc_r) < TOL_REF
    out = ref.hfmm2d(1e-9, zk, src, charges=m.charge, ifpgh=1, nd=2)
    assert rel_l2(m.evaluate(r, loc), out["pot"]) < 1e-8


def test_block_outside_array_is_refused(gpu, ref):
    r = ref.lib()
    src, h = _grid(4)
    m = Mps(r, src, 1, 3.0 + 0j, np.full(src.shape[1], 5), h / 100, seed=3)
    m.ntot -= 1  # the last block now ends past the array
    ier, _ = m.ours(1e-9)
    assert ier == 100
