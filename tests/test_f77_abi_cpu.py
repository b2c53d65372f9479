"""No-GPU checks of libfmm2d.so, the reference's own entry points served by
the B200 library: it loads, exports every routine include/fmm2d_f77.h
declares (the 4 core routines, their 4 _ndiv variants, 27 + 27 flag
wrappers per family, hfmm2d_mps, bhfmm2d, stfmm2d and the C function
hfmm2d_s_c_p), and every Fortran
name it exports is one the reference library exports too."""
import ctypes
import os
import re
import subprocess


ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "fmm2d_f77.h")
F77LIB = os.path.join(ROOT, "fmm2d_b200", "libfmm2d.so")


def declared():
    """Function names of the header after preprocessing (the flag wrappers
    are declared through macros)."""
    txt = subprocess.run(["gcc", "-E", "-P", "-I", os.path.join(ROOT, "include"), HEADER],
                         capture_output=True, text=True, check=True).stdout
    return sorted(set(re.findall(r"\bvoid\s+(\w+)\s*\(", txt)))


def expected():
    names = []
    for f in "clrh":
        names += [f + "fmm2d_", f + "fmm2d_ndiv_"]
        for k in ("s", "t", "st"):
            for d in ("c", "d", "cd"):
                for o in "pgh":
                    names += [f"{f}fmm2d_{k}_{d}_{o}_", f"{f}fmm2d_{k}_{d}_{o}_vec_"]
    return sorted(names + ["hfmm2d_s_c_p", "hfmm2d_mps_", "bhfmm2d_", "stfmm2d_"])


def test_header_declares_the_reference_surface():
    assert declared() == expected()
    assert len(expected()) == 4 * (2 + 54) + 4


def test_library_exports_every_declared_routine():
    lib = ctypes.CDLL(F77LIB)
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing


def test_names_are_the_reference_library_names(ref):
    """Every Fortran-convention name (trailing underscore) exists in the
    reference library, built from its sources."""
    r = ref.lib()
    fortran = [n for n in declared() if n.endswith("_")]
    absent = [n for n in fortran if not hasattr(r, n)]
    assert not absent, absent
