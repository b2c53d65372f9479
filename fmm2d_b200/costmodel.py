"""Learned cost model for the leaf size (ndiv) and the per-level
near-field / expansion balance of the Laplace FMM.

The reference picks ndiv from a fixed table of eps (lndiv2d.f:1-39) and uses
it at every level.  Here a small MLP, trained on timings the FMM itself
produces, predicts the log run time of one rfmm2d / lfmm2d / cfmm2d call from
cheap point-distribution statistics, a candidate ndiv and a candidate level
balance b (the leaf capacity at level l is ndiv 2^(b (lp - l)), lp the level
whose boxes hold ndiv points of a uniform cloud: b > 0 keeps more points in
the leaves above lp, as P2P work, and splits the boxes below it sooner, into
more M2L work; b < 0 the reverse).  ``choose_ndiv`` returns the candidate
ndiv with the smallest prediction at b = 0; ``choose_tree`` keeps it unless
a balance at one of the three best ndiv (where the training timings sample
the balances) is predicted faster by more than 2 %.
The network's forward, backward and Adam kernels are hand-written CUDA
(include/fmm2d_b200.h: b2fmm_mlp_*); the point statistics come from a GPU
histogram (b2fmm_point_stats).  The table stays the fallback when no trained
weights are present, and accuracy is never traded: ndiv and the balance
change only the tree, the expansion order still follows eps, and every
training run is checked against the FP64 direct sum.

Usage on a GPU:
    python -m fmm2d_b200.costmodel train  [--out fmm2d_b200/costmodel_weights.json]
    python -m fmm2d_b200.costmodel train --from-samples   # refit on the committed samples
    python -m fmm2d_b200.costmodel evaluate

``train`` times every candidate ndiv at balance 0 on the training problems,
then the three fastest of them at the other balances, and writes the samples
to fmm2d_b200/costmodel_samples.json (committed, so the fit is reproducible
without re-timing) together with the weights.  Beside the network it records
the best single constant ndiv per eps on the same training timings (the
smallest total time over the training problems).  ``evaluate`` times four
arms on held-out problems: the table, that constant (which separates what the
network learned about the point distribution from "larger leaves than the
table"), the network's ndiv at balance 0, and its (ndiv, balance) pair (the
difference between the last two is what the level balance gains).
"""
import argparse
import ctypes as C
import json
import math
import os
import time

import numpy as np

from . import _lib

NIN, H1, H2 = 10, 32, 32
CANDIDATES = [4, 6, 8, 11, 15, 20, 28, 40, 56, 80, 112]
BALANCES = [-0.5, -0.25, 0.0, 0.25, 0.5]
HERE = os.path.dirname(os.path.abspath(__file__))
WEIGHTS = os.path.join(HERE, "costmodel_weights.json")
SAMPLES = os.path.join(HERE, "costmodel_samples.json")


def table_ndiv(eps):
    """lndiv2d.f:23-38."""
    for lim, nd in ((0.5, 3), (0.5e-1, 5), (0.5e-2, 8), (0.5e-3, 10), (0.5e-6, 15),
                    (0.5e-9, 20), (0.5e-12, 25), (0.5e-15, 45)):
        if eps >= lim:
            return nd
    return None


# ---------------------------------------------------------------------------
# features
# ---------------------------------------------------------------------------
def histogram(src_dev, trg_dev=None):
    """128 x 128 occupancy histogram on the GPU (device inputs (n, 2) f64)."""
    import torch
    h = torch.zeros(128 * 128, dtype=torch.int32, device=src_dev.device)
    ier = C.c_int(0)
    nt = 0 if trg_dev is None else trg_dev.shape[0]
    _lib.lib().b2fmm_point_stats(
        C.c_void_p(src_dev.data_ptr()), C.c_int64(src_dev.shape[0]),
        None if trg_dev is None else C.c_void_p(trg_dev.data_ptr()), C.c_int64(nt),
        C.c_void_p(h.data_ptr()), C.c_void_p(torch.cuda.current_stream().cuda_stream),
        C.byref(ier))
    if ier.value != 0:
        raise RuntimeError(f"b2fmm_point_stats ier={ier.value}")
    return h.cpu().numpy().astype(np.float64).reshape(128, 128)


def features_from_hist(hist, eps):
    """8 distribution features: size, accuracy, occupancy dimensions at four
    grid resolutions, normalised entropy and peak concentration."""
    n = hist.sum()
    f = [math.log10(max(n, 1)) / 7.0, -math.log10(eps) / 12.0]
    for g in (16, 32, 64, 128):
        k = 128 // g
        occ = np.count_nonzero(hist.reshape(g, k, g, k).sum(axis=(1, 3)))
        f.append(math.log(max(occ, 1)) / math.log(g * g))
    p = hist[hist > 0] / max(n, 1)
    f.append(float(-(p * np.log(p)).sum() / math.log(128 * 128)) if p.size else 0.0)
    mean_nz = n / max(np.count_nonzero(hist), 1)
    f.append(math.log10(max(hist.max(), 1) / max(mean_nz, 1e-300)) / 4.0)
    return np.array(f, dtype=np.float32)


def model_inputs(feat, cands=CANDIDATES, balances=None):
    """Network inputs for candidate leaf sizes cands at level balances
    (default 0 for every candidate)."""
    x = np.zeros((len(cands), NIN), dtype=np.float32)
    x[:, :8] = feat
    x[:, 8] = np.log2(np.asarray(cands, dtype=np.float64)) / 7.0
    if balances is not None:
        x[:, 9] = 2.0 * np.asarray(balances, dtype=np.float64)
    return x





# ---------------------------------------------------------------------------
# the model
# ---------------------------------------------------------------------------
class CostModel:
    def __init__(self, params, ymean=0.0, ystd=1.0, best_constant=None):
        self.params = np.asarray(params, dtype=np.float32)
        self.ymean, self.ystd = float(ymean), float(ystd)
        self.best_constant = dict(best_constant or {})  # eps (str) -> ndiv
        assert self.params.size == _lib.lib().b2fmm_mlp_param_count(NIN, H1, H2)

    def constant_ndiv(self, eps):
        """The best constant ndiv of the training timings for eps (the table's
        value when eps was not in the training set)."""
        return self.best_constant.get(repr(float(eps)), table_ndiv(eps))

    @staticmethod
    def init(seed=0):
        """Random weights scaled by 1/sqrt(fan-in), zero biases."""
        rng = np.random.default_rng(seed)
        blocks = [("W", H1, NIN), ("b", H1, 0), ("W", H2, H1), ("b", H2, 0), ("W", 1, H2),
                  ("b", 1, 0)]
        parts = [rng.normal(size=r * c) / math.sqrt(c) if k == "W" else np.zeros(r)
                 for k, r, c in blocks]
        return CostModel(np.concatenate(parts).astype(np.float32))

    def predict(self, X):
        """Predicted log times (model units) for inputs X (B, NIN), on the GPU."""
        import torch
        tx = torch.as_tensor(np.ascontiguousarray(X, dtype=np.float32), device="cuda")
        tp = torch.as_tensor(self.params, device="cuda")
        ty = torch.empty(X.shape[0], dtype=torch.float32, device="cuda")
        ier = C.c_int(0)
        _lib.lib().b2fmm_mlp_forward(C.c_void_p(tx.data_ptr()), X.shape[0], NIN, H1, H2,
                                     C.c_void_p(tp.data_ptr()), C.c_void_p(ty.data_ptr()),
                                     C.c_void_p(torch.cuda.current_stream().cuda_stream),
                                     C.byref(ier))
        if ier.value != 0:
            raise RuntimeError(f"b2fmm_mlp_forward ier={ier.value}")
        return ty.cpu().numpy() * self.ystd + self.ymean

    def choose_ndiv(self, feat):
        """Best predicted ndiv at level balance 0."""
        return CANDIDATES[int(np.argmin(self.predict(model_inputs(feat))))]

    def choose_tree(self, feat, top=3, margin=0.02):
        """(ndiv, level balance): the best predicted ndiv at balance 0 unless
        a balance at one of the `top` best ndiv (the region the training
        timings cover) is predicted faster by more than `margin`."""
        p0 = self.predict(model_inputs(feat))
        best = (CANDIDATES[int(np.argmin(p0))], 0.0)
        g = [(CANDIDATES[i], b) for i in np.argsort(p0)[:top] for b in BALANCES if b != 0.0]
        p = self.predict(model_inputs(feat, [c[0] for c in g], [c[1] for c in g]))
        j = int(np.argmin(p))
        return g[j] if p[j] < float(np.min(p0)) - math.log1p(margin) else best

    def save(self, path=WEIGHTS):
        json.dump({"nin": NIN, "h1": H1, "h2": H2, "candidates": CANDIDATES,
                   "balances": BALANCES,
                   "ymean": self.ymean, "ystd": self.ystd, "best_constant": self.best_constant,
                   "params": [float(v) for v in self.params]}, open(path, "w"))

    @staticmethod
    def load(path=WEIGHTS):
        if not os.path.exists(path):
            return None
        d = json.load(open(path))
        if (d["nin"], d["h1"], d["h2"]) != (NIN, H1, H2):
            return None
        return CostModel(d["params"], d["ymean"], d["ystd"], d.get("best_constant"))


def train(X, y, steps=3000, lr=3e-3, seed=0):
    """Full-batch Adam on the GPU (hand-written kernels); returns the model
    and the loss history."""
    import torch
    ymean, ystd = float(np.mean(y)), float(np.std(y) or 1.0)
    m = CostModel.init(seed)
    m.ymean, m.ystd = ymean, ystd
    tx = torch.as_tensor(np.ascontiguousarray(X, dtype=np.float32), device="cuda")
    tt = torch.as_tensor(((np.asarray(y) - ymean) / ystd).astype(np.float32), device="cuda")
    tp = torch.as_tensor(m.params, device="cuda")
    hist = np.zeros(steps, dtype=np.float32)
    ier = C.c_int(0)
    _lib.lib().b2fmm_mlp_train(C.c_void_p(tx.data_ptr()), C.c_void_p(tt.data_ptr()), X.shape[0],
                               NIN, H1, H2, C.c_void_p(tp.data_ptr()), steps, C.c_float(lr),
                               hist.ctypes.data_as(C.c_void_p),
                               C.c_void_p(torch.cuda.current_stream().cuda_stream), C.byref(ier))
    if ier.value != 0:
        raise RuntimeError(f"b2fmm_mlp_train ier={ier.value}")
    m.params = tp.cpu().numpy()
    return m, hist


_MODEL = None


def auto_tree(src_dev, trg_dev, eps):
    """(ndiv, level balance) chosen by the trained model, or the lndiv2d
    table and balance 0 without one."""
    global _MODEL
    if _MODEL is None:
        _MODEL = CostModel.load() or False
    if not _MODEL:
        return table_ndiv(eps), 0.0
    return _MODEL.choose_tree(features_from_hist(histogram(src_dev, trg_dev), eps))


# ---------------------------------------------------------------------------
# problems and timings
# ---------------------------------------------------------------------------
def make_problem(kind, n, seed):
    """Sources of the cost-model sweep: 'uniform' square, 'mixture' of 16
    Gaussians (sigma log-uniform 1e-4..1e-1), 'curve' r = 0.3 (1 + 0.2 cos 5t)
    with density graded over 1e3 (t with pdf proportional to 10^(3 t / 2 pi))."""
    rng = np.random.default_rng(seed)
    if kind == "uniform":
        src = rng.uniform(0, 1, (2, n))
    elif kind == "mixture":
        c = rng.uniform(0, 1, (2, 16))
        sig = 10 ** rng.uniform(-4, -1, 16)
        k = rng.integers(0, 16, n)
        src = c[:, k] + sig[k] * rng.normal(size=(2, n))
    else:
        u = rng.uniform(0, 1, n)
        t = 2 * np.pi * np.log10(1 + u * (1e3 - 1)) / 3.0  # inverse CDF of 10^(3t/2pi)
        r = 0.3 * (1 + 0.2 * np.cos(5 * t))
        src = np.stack([0.5 + r * np.cos(t), 0.5 + r * np.sin(t)])
    q = rng.normal(size=n)
    return src, q


def time_rfmm(ts, tq, eps, ndiv, reps=2, balance=0.0):
    """Device time (ms, min of reps) of one rfmm2d call (pg = 2) and its
    potential / gradient."""
    import torch
    n = ts.shape[0]
    pot = torch.empty((n, 1), dtype=torch.float64, device="cuda")
    grad = torch.empty((n, 2, 1), dtype=torch.float64, device="cuda")
    o = _lib.Options()
    o.ndiv, o.idivflag, o.ifnear, o.precision = int(ndiv), 0, 1, 0
    o.level_balance = float(balance)
    st = torch.cuda.current_stream()
    best = float("inf")
    for _ in range(reps + 1):
        ier = C.c_int(0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        _lib.lib().b2fmm_rfmm2d_dev(1, C.c_double(eps), C.c_int64(n), C.c_void_p(ts.data_ptr()), 1,
                                    C.c_void_p(tq.data_ptr()), 0, None, None, 2,
                                    C.c_void_p(pot.data_ptr()), C.c_void_p(grad.data_ptr()), None,
                                    C.c_int64(0), None, 0, None, None, None, C.byref(o), None,
                                    C.c_void_p(st.cuda_stream), C.byref(ier))
        e1.record(st)
        torch.cuda.synchronize()
        if ier.value != 0:
            raise RuntimeError(f"rfmm2d ier={ier.value}")
        best = min(best, e0.elapsed_time(e1))
    return best, pot, grad


def direct_error(ts, tq, pot, grad, m=200, seed=0):
    """Relative l2 error of pot+grad at m random sources against the FP64
    direct sum on the GPU (b2fmm_lap_direct_dev, real kernel)."""
    import torch
    n = ts.shape[0]
    idx = torch.as_tensor(np.sort(np.random.default_rng(seed).choice(n, min(m, n), False)),
                          device="cuda")
    tt = ts[idx].contiguous()
    ep = torch.empty((len(idx), 1), dtype=torch.float64, device="cuda")
    eg = torch.empty((len(idx), 2, 1), dtype=torch.float64, device="cuda")
    ier = C.c_int(0)
    _lib.lib().b2fmm_lap_direct_dev(2, 1, C.c_int64(n), C.c_void_p(ts.data_ptr()),
                                    C.c_void_p(tq.data_ptr()), None, None, C.c_int64(len(idx)),
                                    C.c_void_p(tt.data_ptr()), 2, C.c_void_p(ep.data_ptr()),
                                    C.c_void_p(eg.data_ptr()), None, C.c_double(1e-16),
                                    C.c_void_p(torch.cuda.current_stream().cuda_stream),
                                    C.byref(ier))
    a = torch.cat([pot[idx].flatten(), grad[idx].flatten()])
    b = torch.cat([ep.flatten(), eg.flatten()])
    return float(torch.linalg.norm(a - b) / torch.linalg.norm(b))


def collect(problems, cands=CANDIDATES, reps=2, check=True, nbest=3):
    """Rows (features, log2 ndiv, balance), targets (log ms) and the error of
    every (problem, candidate) run: every ndiv at balance 0, then the nbest
    fastest of those at the other balances."""
    import torch
    X, y, rec = [], [], []
    for kind, n, eps, seed in problems:
        src, q = make_problem(kind, n, seed)
        ts = torch.as_tensor(np.ascontiguousarray(src.T), device="cuda")
        tq = torch.as_tensor(q.reshape(n, 1), device="cuda")
        feat = features_from_hist(histogram(ts), eps)
        times = {}

        def run(nd, b):
            ms, pot, grad = time_rfmm(ts, tq, eps, nd, reps, b)
            err = direct_error(ts, tq, pot, grad) if check else None
            X.append(model_inputs(feat, [nd], [b])[0])
            y.append(math.log(ms))
            rec.append({"kind": kind, "n": n, "eps": eps, "ndiv": nd, "balance": b, "ms": ms,
                        "err": err})
            return ms

        for nd in cands:
            times[nd] = run(nd, 0.0)
        for nd in sorted(times, key=times.get)[:nbest]:
            for b in BALANCES:
                if b != 0.0:
                    run(nd, b)
    return np.array(X, dtype=np.float32), np.array(y, dtype=np.float64), rec


def best_constant(rec):
    """Per eps, the candidate with the smallest total time over the problems
    timed in rec at level balance 0 (every problem is timed at every
    candidate there)."""
    out = {}
    for eps in sorted({r["eps"] for r in rec}):
        tot = {}
        for r in rec:
            if r["eps"] == eps and r.get("balance", 0.0) == 0.0:
                tot[r["ndiv"]] = tot.get(r["ndiv"], 0.0) + r["ms"]
        out[repr(float(eps))] = int(min(tot, key=tot.get))
    return out


def save_samples(X, y, rec, path=SAMPLES):
    json.dump({"nin": NIN, "candidates": CANDIDATES, "X": np.asarray(X).tolist(),
               "y": np.asarray(y).tolist(), "runs": rec}, open(path, "w"))


def load_samples(path=SAMPLES):
    """Samples file; rows written before the level balance input read as
    balance 0."""
    d = json.load(open(path))
    X = np.array(d["X"], dtype=np.float32)
    if X.shape[1] < NIN:
        X = np.concatenate([X, np.zeros((X.shape[0], NIN - X.shape[1]), np.float32)], axis=1)
    return X, np.array(d["y"], dtype=np.float64), d["runs"]


def sweep_problems(count, seed0, nmin=1e4, nmax=8e6):
    """count problems: N log-uniform, distribution and eps cycling."""
    rng = np.random.default_rng(seed0)
    out = []
    for i in range(count):
        n = int(round(10 ** rng.uniform(math.log10(nmin), math.log10(nmax))))
        out.append((("uniform", "mixture", "curve")[i % 3], n, (1e-3, 1e-6)[(i // 3) % 2],
                    seed0 + 17 * i))
    return out


def evaluate(model, problems):
    """The network's (ndiv, level balance) against the lndiv2d table, the
    best constant ndiv and the network's ndiv alone (balance 0) on the same
    problems, every run error-checked against the direct sum."""
    import torch
    rows = []
    for kind, n, eps, seed in problems:
        src, q = make_problem(kind, n, seed)
        ts = torch.as_tensor(np.ascontiguousarray(src.T), device="cuda")
        tq = torch.as_tensor(q.reshape(n, 1), device="cuda")
        t0 = time.perf_counter()
        feat = features_from_hist(histogram(ts), eps)
        nd_m, b_m = model.choose_tree(feat)
        choose_ms = (time.perf_counter() - t0) * 1e3
        nd_n = model.choose_ndiv(feat)
        nd_t = table_ndiv(eps)
        nd_c = model.constant_ndiv(eps)
        row = {"kind": kind, "n": n, "eps": eps, "ndiv_table": nd_t, "ndiv_mlp": nd_m,
               "balance_mlp": b_m, "ndiv_mlp_alone": nd_n, "ndiv_constant": nd_c,
               "choose_ms": choose_ms}
        for arm, nd, b in (("table", nd_t, 0.0), ("mlp", nd_m, b_m), ("mlp_ndiv", nd_n, 0.0),
                           ("constant", nd_c, 0.0)):
            ms, p, g = time_rfmm(ts, tq, eps, nd, balance=b)
            row["ms_" + arm] = ms
            row["err_" + arm] = direct_error(ts, tq, p, g)
        rows.append(row)
    tot = {a: sum(r["ms_" + a] for r in rows) for a in ("table", "mlp", "mlp_ndiv", "constant")}
    out = {"problems": len(rows), "best_constant": model.best_constant, "rows": rows}
    for a, v in tot.items():
        out["total_ms_" + a] = v
        out["max_err_over_eps_" + a] = max(r["err_" + a] / r["eps"] for r in rows)
    out["speedup"] = tot["table"] / tot["mlp"]
    out["speedup_vs_constant"] = tot["constant"] / tot["mlp"]
    out["speedup_of_balance"] = tot["mlp_ndiv"] / tot["mlp"]
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("cmd", choices=["train", "evaluate"])
    ap.add_argument("--out", default=WEIGHTS)
    ap.add_argument("--train-problems", type=int, default=60)
    ap.add_argument("--steps", type=int, default=3000)
    ap.add_argument("--samples", default=SAMPLES, help="training samples (written by train)")
    ap.add_argument("--from-samples", action="store_true",
                    help="refit on the samples file instead of timing")
    args = ap.parse_args()
    if args.cmd == "train":
        if args.from_samples:
            X, y, rec = load_samples(args.samples)
        else:
            probs = sweep_problems(args.train_problems, seed0=1000, nmax=2e6)
            X, y, rec = collect(probs)
            save_samples(X, y, rec, args.samples)
        bad = [r for r in rec if r["err"] is not None and r["err"] > r["eps"]]
        m, hist = train(X, y, steps=args.steps)
        m.best_constant = best_constant(rec)
        m.save(args.out)
        print(json.dumps({"samples": len(y), "loss_first": float(hist[0]),
                          "loss_last": float(hist[-1]), "runs_over_eps": len(bad),
                          "best_constant": m.best_constant, "weights": args.out}))
    else:
        m = CostModel.load(args.out)
        print(json.dumps({k: v for k, v in evaluate(m, sweep_problems(40, seed0=5000)).items()
                          if k != "rows"}))


if __name__ == "__main__":
    main()
