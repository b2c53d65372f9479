"""No-GPU checks of the boundary: the library loads and exports every
symbol include/fmm2d_b200.h declares; the python front end keeps the
reference's argument checks and dispatch."""
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    txt = open(os.path.join(ROOT, "include", "fmm2d_b200.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(b2fmm_\w+)\s*\(", txt)))


def test_library_exports_every_declared_symbol():
    import ctypes
    from fmm2d_b200 import _lib
    lib = ctypes.CDLL(_lib.LIBPATH)
    names = declared_symbols()
    assert len(names) >= 17
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(names) <= set(_lib.SIGNATURES)


def test_library_is_sm100a_build():
    from fmm2d_b200 import _lib
    assert _lib.version().startswith("fmm2d_b200")


def test_nothing_to_compute(capsys):
    import fmm2d_b200 as fmm
    src = np.zeros((2, 4))
    out = fmm.lfmm2d(eps=1e-6, sources=src, charges=np.ones(4, complex))
    assert out.pot is None and out.pottarg is None and out.ier == 0
    assert "Nothing to compute" in capsys.readouterr().out


@pytest.mark.parametrize("fn", ["lfmm2d", "rfmm2d", "cfmm2d"])
def test_shape_assertions(fn):
    import fmm2d_b200 as fmm
    f = getattr(fmm, fn)
    with pytest.raises(AssertionError, match="first dimension of sources must be 2"):
        f(eps=1e-6, sources=np.zeros((3, 5)), charges=np.ones(5), pg=1)
    with pytest.raises(AssertionError, match="Charges must be same length"):
        f(eps=1e-6, sources=np.zeros((2, 5)), charges=np.ones(4), pg=1)
    with pytest.raises(AssertionError, match=r"Charges must be of shape \[nd,ns\]"):
        f(eps=1e-6, sources=np.zeros((2, 5)), charges=np.ones((3, 5)), pg=1, nd=2)
    with pytest.raises(AssertionError, match="first dimension of targets must be 2"):
        f(eps=1e-6, sources=np.zeros((2, 5)), charges=np.ones(5), targets=np.zeros((1, 3)), pg=1)


def test_st_requires_equal_flags():
    import fmm2d_b200 as fmm
    with pytest.raises(AssertionError, match="same pg must be equal to pgt"):
        fmm.lfmm2d(eps=1e-6, sources=np.zeros((2, 5)), charges=np.ones(5, complex),
                   targets=np.zeros((2, 3)), pg=2, pgt=1)


def test_comperr_formula():
    import fmm2d_b200 as fmm
    a, b = fmm.Output(), fmm.Output()
    b.pot = np.array([3.0 + 0j, 4.0])
    a.pot = np.array([3.0 + 0j, 4.3])
    assert abs(fmm.comperr(ntest=2, out=a, outex=b, pg=1) - 0.3 / 5.0) < 1e-15
