"""fmm2d_b200: the fmm2d FMM evaluation path (Laplace / Cauchy / Helmholtz in
2-D) on NVIDIA B200 GPUs, behind the fmm2dpy python interface.

    import fmm2d_b200 as fmm
    out = fmm.lfmm2d(eps=1e-6, sources=src, charges=q, pg=2)

See fmm2d_b200/fmm2d.py for the entry points; the CUDA library's C ABI is
include/fmm2d_b200.h.
"""
from .fmm2d import (Output, c2ddir, cfmm2d, comperr, h2ddir, hfmm2d, l2ddir,  # noqa: F401
                    lfmm2d, r2ddir, rfmm2d)
from ._lib import version  # noqa: F401

__all__ = ["Output", "hfmm2d", "lfmm2d", "rfmm2d", "cfmm2d", "h2ddir", "l2ddir", "r2ddir",
           "c2ddir", "comperr", "version"]
