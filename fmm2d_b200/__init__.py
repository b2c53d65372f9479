"""fmm2d_b200: the fmm2d FMM evaluation path (Laplace / Cauchy / Helmholtz,
biharmonic and Stokes in 2-D) on NVIDIA B200 GPUs, behind the fmm2dpy python
interface.

    import fmm2d_b200 as fmm
    out = fmm.lfmm2d(eps=1e-6, sources=src, charges=q, pg=2)

See fmm2d_b200/fmm2d.py for the entry points; the CUDA library's C ABI is
include/fmm2d_b200.h, the reference library's own Fortran and C entry points
(served by fmm2d_b200/libfmm2d.so) include/fmm2d_f77.h.
"""
from .fmm2d import (Output, bh2ddir, bhfmm2d, c2ddir, cfmm2d, comperr,  # noqa: F401
                    h2ddir, hfmm2d, l2ddir, lfmm2d, r2ddir, rfmm2d, st2ddir, stfmm2d)
from ._lib import version  # noqa: F401

__all__ = ["Output", "hfmm2d", "lfmm2d", "rfmm2d", "cfmm2d", "bhfmm2d", "stfmm2d", "h2ddir",
           "l2ddir", "r2ddir", "c2ddir", "bh2ddir", "st2ddir", "comperr", "version"]
