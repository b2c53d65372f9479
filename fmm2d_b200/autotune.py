"""Autotuner of the mixed-precision near-field tile shapes.

The near-field kernel (k_p2p_leaf, csrc/lap_mixed.cu) is compiled in
B2FMM_P2P_SHAPES tile shapes: staged sources per warp and chunk, unrolling
of the pair loop, resident blocks per SM.  Which is fastest depends on the
leaf size (how many targets share a staged source and how many sources a
warp stages per work item), so the library keeps one shape per leaf-size
class (ndiv <= 20, <= 56, larger).  ``tune`` times every shape on synthetic
problems of each class through the C ABI (lfmm2d, charges and dipoles,
pot + grad, the 16-Gaussian mixture and the uniform square at eps 1e-6,
CUDA events around back-to-back calls) and keeps, per class, the shape with
the smallest total time; ``save`` writes the choice to
fmm2d_b200/autotune.json (committed), which ``_lib.lib()`` applies when the
library loads.

Usage on a GPU:
    python -m fmm2d_b200.autotune [--out fmm2d_b200/autotune.json]
"""
import argparse
import ctypes as C
import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
TABLE = os.path.join(HERE, "autotune.json")
NCLASSES = 3
SHAPES = [  # mirror of P2P_SHAPES in csrc/lap_mixed.cu
    {"chunk": 128, "unroll": 2, "min_blocks": 6},
    {"chunk": 64, "unroll": 2, "min_blocks": 8},
    {"chunk": 128, "unroll": 4, "min_blocks": 5},
]
# representative leaf size of each class and the problems it is timed on
CLASS_NDIV = [15, 40, 112]
PROBLEMS = [("mixture", 1000000, 3), ("uniform", 1000000, 4), ("mixture", 4000000, 5)]


def select(times):
    """Per class, the shape with the smallest total time; times[c][v] is the
    total time of shape v on class c's problems."""
    return [int(np.argmin(np.asarray(t, dtype=np.float64))) for t in times]


def apply(table, L=None):
    """Push a table {"shapes": [one per class]} into the library (None:
    leave the library's defaults)."""
    if not table:
        return
    if L is None:
        from . import _lib
        L = _lib.lib()
    for c, v in enumerate(table["shapes"]):
        if L.b2fmm_set_p2p_shape(c, int(v)) != 0:
            raise ValueError(f"autotune table: bad shape {v} for class {c}")


def load(path=TABLE):
    if not os.path.exists(path):
        return None
    d = json.load(open(path))
    if len(d.get("shapes", [])) != NCLASSES or any(not 0 <= v < len(SHAPES)
                                                  for v in d["shapes"]):
        return None
    return d


def save(table, path=TABLE):
    json.dump(table, open(path, "w"), indent=1)


def _time_lfmm(L, ts, tq, td, tv, ndiv, steps=5):
    """Device ms per call (min over rounds of steps back-to-back calls)."""
    import torch
    from . import _lib
    n = ts.shape[0]
    pot = torch.empty((n, 1), dtype=torch.complex128, device="cuda")
    grad = torch.empty((n, 2, 1), dtype=torch.complex128, device="cuda")
    o = _lib.Options()
    o.ndiv, o.idivflag, o.ifnear, o.precision = int(ndiv), 0, 1, _lib.PREC["mixed"]
    st = torch.cuda.current_stream()
    ier = C.c_int(0)

    def call():
        L.b2fmm_lfmm2d_dev(1, C.c_double(1e-6), C.c_int64(n), C.c_void_p(ts.data_ptr()), 1,
                           C.c_void_p(tq.data_ptr()), 1, C.c_void_p(td.data_ptr()),
                           C.c_void_p(tv.data_ptr()), 2, C.c_void_p(pot.data_ptr()),
                           C.c_void_p(grad.data_ptr()), None, C.c_int64(0), None, 0, None,
                           None, None, C.byref(o), None, C.c_void_p(st.cuda_stream),
                           C.byref(ier))
        if ier.value != 0:
            raise RuntimeError(f"lfmm2d ier={ier.value}")

    call()
    best = float("inf")
    for _ in range(3):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(steps):
            call()
        e1.record(st)
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1) / steps)
    return best


def tune(problems=PROBLEMS, class_ndiv=CLASS_NDIV):
    """Times of every (class, shape) and the chosen table."""
    import torch
    from . import _lib
    from .costmodel import make_problem
    L = _lib.lib()
    saved = [L.b2fmm_get_p2p_shape(c) for c in range(NCLASSES)]
    data = []
    for kind, n, seed in problems:
        src, q = make_problem(kind, n, seed)
        rng = np.random.default_rng(seed)
        d = rng.normal(size=n) + 1j * rng.normal(size=n)
        a = rng.uniform(0, 2 * np.pi, n)
        data.append([torch.as_tensor(np.ascontiguousarray(src.T), device="cuda"),
                     torch.as_tensor((q + 0j).reshape(n, 1), device="cuda"),
                     torch.as_tensor(d.reshape(n, 1), device="cuda"),
                     torch.as_tensor(np.stack([np.cos(a), np.sin(a)], 1).reshape(n, 2, 1),
                                     device="cuda")])
    times = [[0.0] * len(SHAPES) for _ in range(NCLASSES)]
    try:
        for c, nd in enumerate(class_ndiv):
            for v in range(len(SHAPES)):
                L.b2fmm_set_p2p_shape(c, v)
                times[c][v] = sum(_time_lfmm(L, *x, nd) for x in data)
    finally:
        for c, v in enumerate(saved):
            L.b2fmm_set_p2p_shape(c, v)
    table = {"shapes": select(times), "class_ndiv": list(class_ndiv), "shape_list": SHAPES,
             "problems": [list(p) for p in problems], "total_ms": times,
             "device": torch.cuda.get_device_name()}
    return table


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=TABLE)
    args = ap.parse_args()
    table = tune()
    save(table, args.out)
    apply(table)
    print(json.dumps(table))


if __name__ == "__main__":
    main()
