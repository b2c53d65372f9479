"""ctypes binding of ``libfmm2d_b200.so`` (the C ABI of include/fmm2d_b200.h).

The library is built in-tree by ``fmm2d_b200/build.py``.  Loading fails loudly
when it is missing: there is no CPU fallback behind this package.
"""
import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(HERE, "libfmm2d_b200.so")

c_int, c_double, c_int64, c_void_p = C.c_int, C.c_double, C.c_int64, C.c_void_p
P = c_void_p  # all array arguments are raw pointers


class Options(C.Structure):
    """Mirror of ``b2fmm_options``."""
    _fields_ = [("ndiv", c_int), ("idivflag", c_int), ("ifnear", c_int), ("precision", c_int),
                ("async_call", c_int), ("level_balance", c_double)]


PREC = {"auto": 0, "fp64": 1, "mixed": 2}

_LAP_HOST = [c_int, c_double, c_int64, P, c_int, P, c_int, P]
_PGH = [c_int, P, P, P, c_int64, P, c_int, P, P, P]
_HELM_HOST = [c_int, c_double, c_double, c_double, c_int64, P, c_int, P, c_int, P, P]

# name -> argtypes, for every symbol declared in include/fmm2d_b200.h
SIGNATURES = {
    "b2fmm_version": [],
    "b2fmm_cfmm2d": _LAP_HOST + [c_int] + _PGH + [P],
    "b2fmm_lfmm2d": _LAP_HOST + [P, c_int] + _PGH + [P],
    "b2fmm_rfmm2d": _LAP_HOST + [P, c_int] + _PGH + [P],
    "b2fmm_cfmm2d_ndiv": _LAP_HOST + [c_int] + _PGH + [c_int, c_int, c_int, P, P],
    "b2fmm_lfmm2d_ndiv": _LAP_HOST + [P, c_int] + _PGH + [c_int, c_int, c_int, P, P],
    "b2fmm_rfmm2d_ndiv": _LAP_HOST + [P, c_int] + _PGH + [c_int, c_int, c_int, P, P],
    "b2fmm_cfmm2d_ex": _LAP_HOST + _PGH + [P, P, P],
    "b2fmm_lfmm2d_ex": _LAP_HOST + [P] + _PGH + [P, P, P],
    "b2fmm_rfmm2d_ex": _LAP_HOST + [P] + _PGH + [P, P, P],
    "b2fmm_cfmm2d_host_async": _LAP_HOST + _PGH + [P, P, P],
    "b2fmm_lfmm2d_host_async": _LAP_HOST + [P] + _PGH + [P, P, P],
    "b2fmm_rfmm2d_host_async": _LAP_HOST + [P] + _PGH + [P, P, P],
    "b2fmm_cfmm2d_dev": _LAP_HOST + _PGH + [P, P, P, P],
    "b2fmm_lfmm2d_dev": _LAP_HOST + [P] + _PGH + [P, P, P, P],
    "b2fmm_rfmm2d_dev": _LAP_HOST + [P] + _PGH + [P, P, P, P],
    "b2fmm_lap_direct_dev": [c_int, c_int, c_int64, P, P, P, P, c_int64, P, c_int, P, P, P,
                             c_double, P, P],
    "b2fmm_lap_direct_noalloc_dev": [c_int, c_int, c_int64, P, P, P, P, c_int64, P, c_int, P, P,
                                     P, c_double, P, P],
    "b2fmm_hfmm2d": _HELM_HOST + [c_int] + _PGH + [P],
    "b2fmm_hfmm2d_ndiv": _HELM_HOST + [c_int] + _PGH + [c_int, c_int, c_int, P, P],
    "b2fmm_hfmm2d_dev": _HELM_HOST + _PGH + [P, P, P, P],
    "b2fmm_bhfmm2d": [c_int, c_double, c_int64, P, c_int, P, c_int, P, c_int, c_int, P, P, P,
                      c_int64, P, c_int, P, P, P, P],
    "b2fmm_bhfmm2d_dev": [c_int, c_double, c_int64, P, c_int, P, c_int, P, c_int, P, P, c_int64,
                          P, c_int, P, P, P, P],
    "b2fmm_bh2ddir_dev": [c_int, c_int64, P, P, P, c_int64, P, c_int, P, P, c_double, P, P],
    "b2fmm_stfmm2d": [c_int, c_double, c_int64, P, c_int, P, c_int, P, P, c_int, P, P, P, c_int64,
                      P, c_int, P, P, P, P],
    "b2fmm_stfmm2d_dev": [c_int, c_double, c_int64, P, c_int, P, c_int, P, P, c_int, P, P, P,
                          c_int64, P, c_int, P, P, P, P, P],
    "b2fmm_st2ddir_dev": [c_int, c_int64, P, c_int, P, c_int, P, P, c_int64, P, c_int, P, P, P,
                          c_double, P, P],
    "b2fmm_hfmm2d_mps": [c_int, c_double, c_double, c_double, c_int64, P, P, P, c_int64, P, P, P,
                         P],
    "b2fmm_h2ddir_dev": [c_int, c_double, c_double, c_int64, P, P, P, P, c_int64, P, c_int, P,
                         P, P, c_double, P, P],
    "b2fmm_h2dterms": [c_double, c_double, c_double, c_double, P],
    "b2fmm_helm_special": [c_int, c_int, c_double, c_double, c_double, P],
    "b2fmm_tree_build": [P, c_int64, P, c_int64, c_int, c_int, c_int, P, P, P],
    "b2fmm_tree_get": [P] * 23,
    "b2fmm_tree_free": [P],
    "b2fmm_kernel_launches": [],
    "b2fmm_set_stats": [c_int],
    "b2fmm_set_device_ranges": [c_int],
    "b2fmm_async_status": [P, P],
    "b2fmm_test_fail_alloc": [c_int],
    "b2fmm_test_barrier_limit": [C.c_longlong],
    "b2fmm_get_stats": [P, c_int],
    "b2fmm_fma_peak": [c_int],
    "b2fmm_set_m2l_tensor_cores": [c_int],
    "b2fmm_set_p2p_shape": [c_int, c_int],
    "b2fmm_get_p2p_shape": [c_int],
    "b2fmm_mlp_param_count": [c_int, c_int, c_int],
    "b2fmm_mlp_forward": [P, c_int, c_int, c_int, c_int, P, P, P, P],
    "b2fmm_mlp_gradient": [P, P, c_int, c_int, c_int, c_int, P, P, P, P, P],
    "b2fmm_mlp_train": [P, P, c_int, c_int, c_int, c_int, P, c_int, C.c_float, P, P, P],
    "b2fmm_point_stats": [P, c_int64, P, c_int64, P, P, P],
    "b2fmm_tc_gemm_probe": [P, P, c_int, c_int, P, P, P],
    "b2fmm_plan_create": [c_int, c_int, c_double, c_int64, P, c_int, c_int, c_int, c_int64, P,
                          c_int, P, P, P],
    "b2fmm_plan_eval": [P] * 12,
    "b2fmm_plan_status": [P],
    "b2fmm_plan_free": [P],
    "b2fmm_batch_graph_create": [c_int] + [P] * 10 + [c_int, P],
    "b2fmm_batch_graph_launch": [P, P, P],
    "b2fmm_batch_graph_status": [P],
    "b2fmm_batch_graph_nodes": [P],
    "b2fmm_batch_graph_free": [P],
}

_lib = None


class LibraryMissing(RuntimeError):
    pass


def lib():
    """Load the CUDA library (raises LibraryMissing when it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIBPATH):
            raise LibraryMissing(
                f"{LIBPATH} not found: build it with `python -m fmm2d_b200.build` "
                "(there is no CPU fallback)")
        L = C.CDLL(LIBPATH)
        for name, args in SIGNATURES.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = None
        L.b2fmm_version.restype = C.c_char_p
        L.b2fmm_tree_build.restype = c_void_p
        L.b2fmm_kernel_launches.restype = C.c_uint64
        L.b2fmm_fma_peak.restype = c_double
        L.b2fmm_h2dterms.restype = c_int
        L.b2fmm_plan_create.restype = c_void_p
        L.b2fmm_mlp_param_count.restype = c_int
        L.b2fmm_plan_status.restype = c_int
        L.b2fmm_batch_graph_create.restype = c_void_p
        L.b2fmm_batch_graph_status.restype = c_int
        L.b2fmm_batch_graph_nodes.restype = C.c_int64
        L.b2fmm_set_p2p_shape.restype = c_int
        L.b2fmm_get_p2p_shape.restype = c_int
        _lib = L
        # the autotuner's committed near-field tile shapes (fmm2d_b200/autotune.py)
        from . import autotune
        autotune.apply(autotune.load(), L)
    return _lib


STAT_KEYS = ["nboxes", "nlevels", "nleaves", "nterms1", "p2p_pairs", "m2l_pairs", "m2p_evals",
             "p2l_sources", "npts_eval", "tree_ms", "fmm_ms", "nd_cauchy", "m2l_tc_steps",
             "tl_pre", "tl_tree", "tl_setup", "tl_fmm", "tl_post"]


def get_stats():
    import numpy as np
    out = np.zeros(len(STAT_KEYS))
    lib().b2fmm_get_stats(out.ctypes.data_as(c_void_p), len(STAT_KEYS))
    return dict(zip(STAT_KEYS, out.tolist()))


def version():
    return lib().b2fmm_version().decode()
