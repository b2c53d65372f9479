"""Benchmark: points/sec of the 4M-point nonuniform Laplace FMM (eps 1e-6) on B200.

Workload (the headline configuration): lfmm2d on N = 4,000,000 sources drawn
from a mixture of 16 Gaussians (centres uniform in [0,1]^2, sigma log-uniform
in [1e-4, 1e-1]), complex charges with N(0,1) real/imaginary parts, dipstr
N(0,1) (real), unit dipvec at a uniform angle, eps = 1e-6, pg = 2 (potential
and gradient at the sources); seeded synthetic data (numpy default_rng(1)).

A step is one complete FMM call (tree, lists, all passes, caller-order
results).  ``value`` times it with inputs resident in HBM (device-pointer C
ABI b2fmm_lfmm2d_dev) in the mixed-precision mode; the K timed calls are
queued back to back (options.async_call: no host wait inside or between
them) and their device status is checked after the timing.  ``fp64_value``
is the plain FP64 GPU FMM on the same inputs, timed the same way; ``e2e``
calls the queued host-pointer entry point b2fmm_lfmm2d_host_async with pinned
host buffers on two streams in turn (every step copies its inputs in and its
results out; one step's copies overlap the other's FMM; wall clock from the
first call to both streams finished), ``e2e_blocking`` the blocking
b2fmm_lfmm2d_ex (one wait per call).  Every run reports the
relative l2 error of pot+grad against the FP64 direct sum over 1000 random
sources.  ``--impl reference`` times the reference itself (its Fortran
translated to C by oracle/f77c.py, gcc -O3 -fopenmp; no Fortran compiler
exists here) on a bounded sample of the same workload with all host
threads; ``cpu_baseline`` is the same code on a 1M-point sample.

Lines printed before the headline line: ``lfmm2d_eps_sweep`` (the headline
workload at eps 1e-3, mixed, and 1e-9, FP64, with their errors);
``rfmm2d_c1`` (plain rfmm2d, 100,000 uniform sources, real N(0,1) charges,
eps 1e-6, pg 2: FP64 and mixed GPU time, the reference on the host cores and
the FP64 GPU result against the reference's); ``roofline_detail``.

``helmholtz_c4`` adds the Helmholtz configuration: hfmm2d with zk = 40 on
2,000,000 sources at uniform random angles on the curve
r(t) = 0.3 (1 + 0.2 cos 5t) about (0.5, 0.5) and 1,000,000 uniform targets,
complex charges and dipole strengths CN(0,1), unit dipvec at a uniform angle,
eps = 1e-9, pgt = 2 (FP64 throughout), timed the same way with its relative
l2 error against the FP64 direct sum on 1000 targets.  ``--c4-only`` prints
just that object (``--c4-scale`` shrinks it for profiling).

``batched_c3`` is the batched configuration: 256 independent cfmm2d problems
with N log-uniform in [2e3, 2e5], uniform or single-Gaussian clouds, nd in
{1, 2, 4} complex densities, eps = 1e-6, pg = 1.  It times 256 sequential
plain calls (b2fmm_cfmm2d_dev, tree included in every call) against one
launch of a CUDA graph that evaluates all 256 plans (trees built once,
b2fmm_plan_create; their build time is reported separately), and checks
the graph's results against the sequential ones.

``costmodel_c5`` is the learned-cost-model sweep: 40 rfmm2d problems with N
log-uniform in [1e4, 8e6] over three distributions (uniform; the 16-Gaussian
mixture; the curve above with density graded over 1e3), real N(0,1)
charges, eps in {1e-3, 1e-6}, pg = 2: total time with the leaf size and level
balance chosen by the trained network (fmm2d_b200/costmodel.py) against the
lndiv2d table, the best single constant leaf size per eps of the training
timings, and the network's leaf size alone at balance 0, all four
error-checked against the FP64 direct sum.

Multi-GPU (torchrun): every rank evaluates its own independent problem of the
same size (replicas, no collective in the data path); timings are the max over
ranks (one all_reduce of the step times) and ``value`` counts all ranks' points.
"""
import argparse
import ctypes as C
import json
import math
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "points/sec, 4M nonuniform Laplace eps 1e-6: mixed-prec vs FP64 plain, 1 B200"
WORKLOAD = "lfmm2d 16-Gaussian mixture, complex charges + dipoles, eps=1e-6, pg=2"


def make_inputs(n, seed=1):
    rng = np.random.default_rng(seed)
    c = rng.uniform(0, 1, (2, 16))
    sig = 10 ** rng.uniform(-4, -1, 16)
    k = rng.integers(0, 16, n)
    src = c[:, k] + sig[k] * rng.normal(size=(2, n))
    q = rng.normal(size=n) + 1j * rng.normal(size=n)
    d = rng.normal(size=n) + 0j
    ph = rng.uniform(0, 2 * np.pi, n)
    v = np.stack([np.cos(ph), np.sin(ph)])
    return src, q, d, v


def make_c4_inputs(ns, nt, seed=4):
    """Helmholtz configuration: closed smooth curve + uniform targets."""
    rng = np.random.default_rng(seed)
    th = rng.uniform(0, 2 * np.pi, ns)
    r = 0.3 * (1 + 0.2 * np.cos(5 * th))
    src = np.stack([0.5 + r * np.cos(th), 0.5 + r * np.sin(th)])
    trg = rng.uniform(0, 1, (2, nt))
    q = (rng.normal(size=ns) + 1j * rng.normal(size=ns)) / np.sqrt(2)
    d = (rng.normal(size=ns) + 1j * rng.normal(size=ns)) / np.sqrt(2)
    ph = rng.uniform(0, 2 * np.pi, ns)
    v = np.stack([np.cos(ph), np.sin(ph)])
    return src, trg, q, d, v


def helmholtz_c4(L, dev, stream, scale=1.0, steps=3, warmup=1):
    """hfmm2d, zk=40, 2M curve sources + 1M targets, eps=1e-9, pgt=2."""
    import torch
    from fmm2d_b200 import _lib
    ns, nt = int(2_000_000 * scale), int(1_000_000 * scale)
    src, trg, q, d, v = make_c4_inputs(ns, nt)
    hs, hq, hd, hv = fortran_layout(src, q, d, v)
    ds, dq, dd, dv = (torch.as_tensor(x, device=dev) for x in (hs, hq, hd, hv))
    dt = torch.as_tensor(np.ascontiguousarray(trg.T), device=dev)
    pt = torch.empty((nt, 1), dtype=torch.complex128, device=dev)
    gt = torch.empty((nt, 2, 1), dtype=torch.complex128, device=dev)
    ptr = lambda t: C.c_void_p(t.data_ptr())
    zk, eps = 40.0, 1e-9

    def step(ti=None):
        o = _lib.Options()
        o.ndiv, o.idivflag, o.ifnear, o.precision = 0, 0, 1, 1
        ier = C.c_int(0)
        ti = ti if ti is not None else np.zeros(8)
        L.b2fmm_hfmm2d_dev(1, eps, zk, 0.0, ns, ptr(ds), 1, ptr(dq), 1, ptr(dd), ptr(dv), 0,
                           None, None, None, nt, ptr(dt), 2, ptr(pt), ptr(gt), None, C.byref(o),
                           ti.ctypes.data_as(C.c_void_p), C.c_void_p(stream.cuda_stream),
                           C.byref(ier))
        if ier.value != 0:
            raise RuntimeError(f"b2fmm_hfmm2d_dev ier={ier.value}")

    for _ in range(warmup):
        step()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    tis = np.zeros(8)
    e0.record(stream)
    for _ in range(steps):
        ti = np.zeros(8)
        step(ti)
        tis += ti
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    tis /= steps
    rng = np.random.default_rng(98)
    idx = np.sort(rng.choice(nt, min(1000, nt), replace=False))
    tsel = torch.as_tensor(np.ascontiguousarray(trg[:, idx].T), device=dev)
    m = len(idx)
    ep = torch.empty((m, 1), dtype=torch.complex128, device=dev)
    eg = torch.empty((m, 2, 1), dtype=torch.complex128, device=dev)
    ier = C.c_int(0)
    L.b2fmm_h2ddir_dev(1, zk, 0.0, ns, ptr(ds), ptr(dq), ptr(dd), ptr(dv), m, ptr(tsel), 2,
                       ptr(ep), ptr(eg), None, C.c_double(1e-16),
                       C.c_void_p(stream.cuda_stream), C.byref(ier))
    ia = torch.as_tensor(idx, device=dev)
    a_p, a_g = pt[ia, 0].cpu().numpy(), gt[ia, :, 0].cpu().numpy()
    e_p, e_g = ep[:, 0].cpu().numpy(), eg[:, :, 0].cpu().numpy()
    err = float(np.sqrt((np.linalg.norm(a_p - e_p) ** 2 + np.linalg.norm(a_g - e_g) ** 2)
                        / (np.linalg.norm(e_p) ** 2 + np.linalg.norm(e_g) ** 2)))
    return {"workload": "hfmm2d zk=40, curve r=0.3(1+0.2cos5t) sources + uniform targets, "
                        "charges+dipoles CN(0,1), eps=1e-9, pgt=2, FP64",
            "ns": ns, "nt": nt, "value": (ns + nt) / (ms * 1e-3), "unit": "points/s",
            "ms_per_step": ms, "steps": steps, "rel_l2_err": err,
            "err_ref": f"FP64 direct sum over {m} random targets",
            "phase_ms": {k: round(tis[i] * 1e3, 3) for k, i in
                         (("p2m", 0), ("m2m", 2), ("p2l", 1), ("m2l", 3), ("l2l", 4),
                          ("leaf_eval(l2p+m2p+p2p)", 7))}}


def batched_c3(L, dev, nprob=256, seed=3, nbranch=16, launches=5):
    """256 cfmm2d problems: sequential plain calls vs one captured graph."""
    import torch
    from fmm2d_b200 import _lib
    from fmm2d_b200.plan import BatchGraph, Plan
    rng = np.random.default_rng(seed)
    probs = []
    for i in range(nprob):
        n = int(round(10 ** rng.uniform(np.log10(2e3), np.log10(2e5))))
        nd = int(rng.choice([1, 2, 4]))
        if rng.uniform() < 0.5:
            src = rng.uniform(0, 1, (2, n))
        else:
            c = rng.uniform(0.25, 0.75, 2)
            src = c[:, None] + 10 ** rng.uniform(-3, -1) * rng.normal(size=(2, n))
        q = rng.normal(size=(nd, n)) + 1j * rng.normal(size=(nd, n))
        ts = torch.as_tensor(np.ascontiguousarray(src.T), device=dev)
        tq = torch.as_tensor(np.ascontiguousarray(q.T), device=dev)
        probs.append((n, nd, ts, tq, torch.empty((n, nd), dtype=torch.complex128, device=dev)))
    npts = sum(p[0] for p in probs)
    stream = torch.cuda.current_stream(dev)
    ptr = lambda t: C.c_void_p(t.data_ptr())
    o = _lib.Options()
    o.ndiv, o.idivflag, o.ifnear, o.precision = 0, 0, 1, 0

    def sequential():
        for n, nd, ts, tq, pot in probs:
            ier = C.c_int(0)
            L.b2fmm_cfmm2d_dev(nd, C.c_double(1e-6), C.c_int64(n), ptr(ts), 1, ptr(tq), 0, None, 1,
                               ptr(pot), None, None, C.c_int64(0), None, 0, None, None, None,
                               C.byref(o), None, C.c_void_p(stream.cuda_stream), C.byref(ier))
            if ier.value != 0:
                raise RuntimeError(f"b2fmm_cfmm2d_dev ier={ier.value}")

    sequential()  # warm-up
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    sequential()
    e1.record(stream)
    torch.cuda.synchronize()
    seq_ms = e0.elapsed_time(e1)
    seq_pot = [p[4].clone() for p in probs]

    def make_plans():
        return [Plan("cfmm2d", eps=1e-6, sources=ts, charges=True, pg=1, nd=nd)
                for n, nd, ts, tq, pot in probs]

    # warm-up, as for the sequential calls: the first plans of a process also
    # pay the one-time growth of the stream-ordered memory pool
    for p in make_plans():
        p.close()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    plans = make_plans()
    torch.cuda.synchronize()
    plan_ms = (time.perf_counter() - t0) * 1e3
    t0 = time.perf_counter()
    g = BatchGraph(plans, charges=[p[3] for p in probs], nbranch=nbranch)
    torch.cuda.synchronize()
    graph_build_ms = (time.perf_counter() - t0) * 1e3
    g.launch()
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(launches):
        g.launch(stream.cuda_stream)
    e1.record(stream)
    torch.cuda.synchronize()
    graph_ms = e0.elapsed_time(e1) / launches
    st = g.status()
    err = 0.0
    for (n, nd, ts, tq, pot), ref, out in zip(probs, seq_pot, g.outs):
        a, b = out["pot"], ref
        err = max(err, float(torch.linalg.norm(a - b) / torch.linalg.norm(b)))
    nodes = g.nodes
    g.close()
    for p in plans:
        p.close()
    return {"workload": "256 cfmm2d problems, N log-uniform [2e3, 2e5], uniform or "
                        "single-Gaussian clouds, nd in {1,2,4}, eps=1e-6, pg=1",
            "problems": nprob, "points": npts, "unit": "points/s",
            "sequential_ms": seq_ms, "sequential_value": npts / (seq_ms * 1e-3),
            "graph_ms": graph_ms, "graph_value": npts / (graph_ms * 1e-3),
            "graph_speedup": seq_ms / graph_ms, "graph_branches": nbranch, "graph_nodes": nodes,
            "plan_build_ms": plan_ms, "graph_build_ms": graph_build_ms,
            "graph_plus_plans_value": npts / ((graph_ms + plan_ms) * 1e-3),
            "max_rel_diff_graph_vs_sequential": err, "status": st}


def fortran_layout(src, q, d, v):
    """(2,n)/(n,)/(2,n) user arrays -> the C ABI's column-major layouts."""
    return (np.ascontiguousarray(src.T), np.ascontiguousarray(q.reshape(-1, 1)),
            np.ascontiguousarray(d.reshape(-1, 1)), np.ascontiguousarray(v.T.reshape(-1, 2, 1)))


class ClockSampler:
    """SM clock and clock-event (throttle) reasons of the timed GPU, sampled
    every 200 ms from before the warm-up to after the timed steps.  In-process
    NVML reads (pynvml) in a background thread; the GPU is found by its UUID,
    so the sample is of the device the process runs on whatever
    CUDA_VISIBLE_DEVICES maps.  Falls back to an nvidia-smi subprocess when
    pynvml is missing (its periodic queries hold driver locks for some
    milliseconds, which shows in short timed regions)."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.thread = None
        self.samples = []
        self.path = os.path.join("/tmp", f"b2fmm_clocks_{os.getpid()}.csv")

    def _uuid(self):
        try:
            import torch
            u = torch.cuda.get_device_properties(self.gpu).uuid
            s = str(u)
            return s if s.startswith("GPU-") else "GPU-" + s
        except Exception:
            return None

    def start(self):
        try:
            import threading
            import pynvml as nv
            nv.nvmlInit()
            uid = self._uuid()
            h = (nv.nvmlDeviceGetHandleByUUID(uid) if uid
                 else nv.nvmlDeviceGetHandleByIndex(self.gpu))
            self.nv, self.h = nv, h
            self.max_mhz = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
            bits = {"hw_slowdown": nv.nvmlClocksEventReasonHwSlowdown,
                    "hw_thermal_slowdown": nv.nvmlClocksEventReasonHwThermalSlowdown,
                    "sw_thermal_slowdown": nv.nvmlClocksEventReasonSwThermalSlowdown,
                    "sw_power_cap": nv.nvmlClocksEventReasonSwPowerCap}
            self.stop_flag = threading.Event()

            def loop():
                while not self.stop_flag.is_set():
                    try:
                        mhz = float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM))
                        r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                        self.samples.append((mhz, [k for k, b in bits.items() if r & b]))
                    except Exception:
                        pass
                    self.stop_flag.wait(0.2)

            self.thread = threading.Thread(target=loop, daemon=True)
            self.thread.start()
            return
        except Exception:
            self.thread = None
        try:
            self.f = open(self.path, "w")
            uid = self._uuid()
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-i", uid if uid else str(self.gpu), "-lms", "200"], stdout=self.f,
                stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
            return
        t0 = time.time()
        while time.time() - t0 < 5.0 and self.proc.poll() is None:
            if os.path.getsize(self.path) > 0:
                break
            time.sleep(0.02)

    def stop(self):
        if self.thread is not None:
            self.stop_flag.set()
            self.thread.join(timeout=5)
            try:
                self.nv.nvmlShutdown()
            except Exception:
                pass
            if not self.samples:
                return None
            reasons = sorted({r for _, rs in self.samples for r in rs})
            return {"sm_mhz": statistics.median([m for m, _ in self.samples]),
                    "sm_max_mhz": self.max_mhz, "reasons": reasons,
                    "samples": len(self.samples), "source": "nvml"}
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.f.close()
        sm, mx, reasons = [], [], set()
        for line in open(self.path):
            p = [x.strip() for x in line.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx.append(float(p[2]))
            except ValueError:
                continue
            for nm, val in zip(self.NAMES, p[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx),
                "reasons": sorted(reasons), "samples": len(sm), "source": "nvidia-smi"}


def max_over_ranks(x, dist, device):
    """Largest value of x over the ranks (one all-reduce; x itself when not
    distributed).  The step time of the slowest rank bounds the job."""
    if not dist:
        return x
    import torch
    t = torch.tensor([float(x)], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def dist_info():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


REF_KIND = ("the reference's own Fortran (src/laplace, src/common), translated to C by "
            "oracle/f77c.py and compiled with gcc -O3 -funroll-loops -fopenmp")


def _ref_module():
    """The reference itself (oracle/_ref) when built, else the C++ restatement."""
    from oracle import ref as R
    if R.available():
        return R, "reference"
    from oracle import oracle as O
    O.build()
    return O, "port"


def cpu_baseline(n_sample, reps=1):
    """The reference's lfmm2d on a bounded sample, all host threads."""
    M, kind = _ref_module()
    M.set_num_threads(os.cpu_count() or 1)
    src, q, d, v = make_inputs(n_sample, seed=1)
    M.lfmm2d(1e-6, src[:, :20000], charges=q[:20000], dipstr=d[:20000], dipvec=v[:, :20000],
             ifpgh=2)  # warm-up
    ts = []
    for _ in range(reps):
        t0 = time.perf_counter()
        M.lfmm2d(1e-6, src, charges=q, dipstr=d, dipvec=v, ifpgh=2)
        ts.append(time.perf_counter() - t0)
    t = min(ts)
    return {"value": n_sample / t, "unit": "points/s", "cores": M.num_threads(), "kind": kind,
            "sample": f"{n_sample} points of the same 16-Gaussian mixture (seed 1), one lfmm2d "
                      f"call, eps=1e-6, pg=2; {t:.2f} s"
                      + (f"; {REF_KIND}" if kind == "reference" else "")}


def run_reference(args, rank, world):
    if rank != 0:
        return
    n_sample = args.ref_sample
    M, kind = _ref_module()
    M.set_num_threads(os.cpu_count() or 1)
    src, q, d, v = make_inputs(n_sample, seed=1)
    for _ in range(args.warmup):
        M.lfmm2d(1e-6, src, charges=q, dipstr=d, dipvec=v, ifpgh=2)
    ts = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        M.lfmm2d(1e-6, src, charges=q, dipstr=d, dipvec=v, ifpgh=2)
        ts.append(time.perf_counter() - t0)
    t = sum(ts) / len(ts)
    val = n_sample / t
    line = {"impl": "reference", "metric": METRIC, "value": val, "unit": "points/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": {"workload": WORKLOAD + f"; bounded sample n={n_sample}",
                                            "n_points": n_sample, "eps": 1e-6},
            "cpu_baseline": {"value": val, "unit": "points/s", "cores": M.num_threads(),
                             "kind": kind,
                             "sample": f"{n_sample} points of the same mixture per step"
                                       + (f"; {REF_KIND}" if kind == "reference" else "")},
            "e2e": {"value": val, "unit": "points/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def _lfmm_dev(L, n, ds, dq, dd, dv, pot, grad, stream, eps, precision, async_call=0,
              timeinfo=None):
    from fmm2d_b200 import _lib
    o = _lib.Options()
    o.ndiv, o.idivflag, o.ifnear, o.precision = 0, 0, 1, _lib.PREC[precision]
    o.async_call = async_call
    ier = C.c_int(0)
    ptr = lambda t: C.c_void_p(t.data_ptr())
    ti = timeinfo.ctypes.data_as(C.c_void_p) if timeinfo is not None else None
    L.b2fmm_lfmm2d_dev(1, C.c_double(eps), C.c_int64(n), ptr(ds), 1, ptr(dq), 1, ptr(dd),
                       ptr(dv), 2, ptr(pot), ptr(grad), None, C.c_int64(0), None, 0, None,
                       None, None, C.byref(o), ti, C.c_void_p(stream.cuda_stream), C.byref(ier))
    if ier.value != 0:
        raise RuntimeError(f"b2fmm_lfmm2d_dev ier={ier.value}")


def async_status(L, stream):
    ier = C.c_int(-1)
    L.b2fmm_async_status(C.c_void_p(stream.cuda_stream), C.byref(ier))
    if ier.value != 0:
        raise RuntimeError(f"asynchronous FMM calls failed: ier={ier.value}")


def rel_err_vs_direct(L, ds, dq, dd, dv, src, n, pot, grad, stream, dev, seed=99):
    """comperr-style relative l2 error of pot+grad against the FP64 direct sum
    over 1000 random sources."""
    import torch
    ptr = lambda t: C.c_void_p(t.data_ptr())
    rng = np.random.default_rng(seed)
    idx = np.sort(rng.choice(n, 1000, replace=False))
    tsel = torch.as_tensor(np.ascontiguousarray(src[:, idx].T), device=dev)
    ep = torch.empty((1000, 1), dtype=torch.complex128, device=dev)
    eg = torch.empty((1000, 2, 1), dtype=torch.complex128, device=dev)
    ier = C.c_int(0)
    L.b2fmm_lap_direct_dev(1, 1, C.c_int64(n), ptr(ds), ptr(dq), ptr(dd), ptr(dv),
                           C.c_int64(1000), ptr(tsel), 2, ptr(ep), ptr(eg), None,
                           C.c_double(1e-16), C.c_void_p(stream.cuda_stream), C.byref(ier))
    ia = torch.as_tensor(idx, device=dev)
    a_p, a_g = pot[ia, 0].cpu().numpy(), grad[ia, :, 0].cpu().numpy()
    e_p, e_g = ep[:, 0].cpu().numpy(), eg[:, :, 0].cpu().numpy()
    return float(np.sqrt((np.linalg.norm(a_p - e_p) ** 2 + np.linalg.norm(a_g - e_g) ** 2)
                         / (np.linalg.norm(e_p) ** 2 + np.linalg.norm(e_g) ** 2)))


def c2_eps_sweep(L, n, ds, dq, dd, dv, src, pot, grad, stream, dev, steps=5):
    """The headline workload at eps 1e-3 and 1e-9: mixed (1e-3) and FP64
    (1e-9, below the mixed path's range) device time and error."""
    import torch
    out = {}
    for eps in (1e-3, 1e-9):
        precision = "mixed" if eps >= 1e-6 else "fp64"
        for _ in range(2):
            _lfmm_dev(L, n, ds, dq, dd, dv, pot, grad, stream, eps, precision)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            _lfmm_dev(L, n, ds, dq, dd, dv, pot, grad, stream, eps, precision, async_call=1)
        e1.record(stream)
        torch.cuda.synchronize()
        async_status(L, stream)
        ms = e0.elapsed_time(e1) / steps
        out[f"eps_{eps:g}"] = {"precision": precision, "ms_per_step": ms,
                               "value": n / (ms * 1e-3), "unit": "points/s", "eps": eps,
                               "rel_l2_err": rel_err_vs_direct(L, ds, dq, dd, dv, src, n, pot,
                                                               grad, stream, dev)}
    return out


def rfmm_c1(L, dev, stream, steps=20, cpu=True):
    """Plain rfmm2d: 100,000 uniform sources, real N(0,1) charges, eps 1e-6,
    pg 2, no targets; FP64 and mixed GPU device time, and the reference's own
    CPU code on the same inputs with all host threads."""
    import torch
    from fmm2d_b200 import _lib
    n = 100_000
    rng = np.random.default_rng(0)
    src = rng.uniform(0, 1, (2, n))
    q = rng.normal(size=n)
    ds = torch.as_tensor(np.ascontiguousarray(src.T), device=dev)
    dq = torch.as_tensor(q.reshape(n, 1), device=dev)
    pot = torch.empty((n, 1), dtype=torch.float64, device=dev)
    grad = torch.empty((n, 2, 1), dtype=torch.float64, device=dev)
    ptr = lambda t: C.c_void_p(t.data_ptr())
    res = {"workload": "rfmm2d 100,000 uniform sources, real N(0,1) charges, eps=1e-6, pg=2",
           "n": n, "unit": "points/s"}

    def call(precision, async_call):
        o = _lib.Options()
        o.ndiv, o.idivflag, o.ifnear, o.precision = 0, 0, 1, _lib.PREC[precision]
        o.async_call = async_call
        ier = C.c_int(0)
        L.b2fmm_rfmm2d_dev(1, C.c_double(1e-6), C.c_int64(n), ptr(ds), 1, ptr(dq), 0, None, None,
                           2, ptr(pot), ptr(grad), None, C.c_int64(0), None, 0, None, None, None,
                           C.byref(o), None, C.c_void_p(stream.cuda_stream), C.byref(ier))
        if ier.value != 0:
            raise RuntimeError(f"b2fmm_rfmm2d_dev ier={ier.value}")

    for precision in ("fp64", "mixed"):
        for _ in range(3):
            call(precision, 0)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            call(precision, 1)
        e1.record(stream)
        torch.cuda.synchronize()
        async_status(L, stream)
        ms = e0.elapsed_time(e1) / steps
        res[precision] = {"ms_per_step": ms, "value": n / (ms * 1e-3)}
    if cpu:
        M, kind = _ref_module()
        M.set_num_threads(os.cpu_count() or 1)
        M.rfmm2d(1e-6, src, charges=q, ifpgh=2)
        ts = []
        for _ in range(3):
            t0 = time.perf_counter()
            r = M.rfmm2d(1e-6, src, charges=q, ifpgh=2)
            ts.append(time.perf_counter() - t0)
        t = min(ts)
        res["cpu"] = {"value": n / t, "ms_per_step": t * 1e3, "cores": M.num_threads(),
                      "kind": kind}
        # the FP64 GPU result against the reference's own output
        call("fp64", 0)
        torch.cuda.synchronize()
        a = pot[:, 0].cpu().numpy()
        res["fp64_rel_diff_vs_cpu"] = float(np.linalg.norm(a - r["pot"][0])
                                            / np.linalg.norm(r["pot"][0]))
    return res


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=4_000_000)
    ap.add_argument("--ref-sample", type=int, default=500_000)
    ap.add_argument("--cpu-sample", type=int, default=1_000_000)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--no-c4", action="store_true", help="skip the Helmholtz configuration")
    ap.add_argument("--c4-only", action="store_true", help="run only the Helmholtz configuration")
    ap.add_argument("--c4-scale", type=float, default=1.0)
    ap.add_argument("--no-c3", action="store_true", help="skip the batched configuration")
    ap.add_argument("--no-c5", action="store_true", help="skip the cost-model sweep")
    ap.add_argument("--no-c1", action="store_true", help="skip the plain rfmm2d configuration")
    ap.add_argument("--no-sweep", action="store_true", help="skip the eps 1e-3 / 1e-9 runs")
    ap.add_argument("--c3-only", action="store_true", help="run only the batched configuration")
    args = ap.parse_args()
    rank, world, local = dist_info()
    if args.impl == "reference":
        run_reference(args, rank, world)
        return

    import torch
    from fmm2d_b200 import _lib
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        pg = dist
    L = _lib.lib()
    stream = torch.cuda.current_stream(dev)
    if args.c3_only:
        res = batched_c3(L, dev)
        if rank == 0:
            print(json.dumps({"batched_c3": res}), flush=True)
        return
    if args.c4_only:
        res = helmholtz_c4(L, dev, stream, args.c4_scale, max(1, args.steps), max(1, args.warmup))
        if rank == 0:
            print(json.dumps({"helmholtz_c4": res}), flush=True)
        return
    n = args.n
    src, q, d, v = make_inputs(n, seed=1 + rank)
    hs, hq, hd, hv = fortran_layout(src, q, d, v)
    ds, dq, dd, dv = (torch.as_tensor(x, device=dev) for x in (hs, hq, hd, hv))
    pot = torch.empty((n, 1), dtype=torch.complex128, device=dev)
    grad = torch.empty((n, 2, 1), dtype=torch.complex128, device=dev)
    ptr = lambda t: C.c_void_p(t.data_ptr())

    def step(precision, timeinfo=None, async_call=0):
        _lfmm_dev(L, n, ds, dq, dd, dv, pot, grad, stream, 1e-6, precision, async_call, timeinfo)

    def timed(precision, steps, warmup, with_clocks=False):
        # the clock sampler runs from before the warm-up to after the timed steps
        sampler = ClockSampler(local) if with_clocks else None
        if sampler:
            sampler.start()
        for _ in range(warmup):
            step(precision)
        if pg:
            pg.barrier()
        torch.cuda.synchronize()
        L0 = L.b2fmm_kernel_launches()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        # the steps are queued back to back (asynchronous calls: no host wait
        # inside or between them); their outcome is checked after the timing
        e0.record(stream)
        for _ in range(steps):
            step(precision, async_call=1)
        e1.record(stream)
        torch.cuda.synchronize()
        launches = L.b2fmm_kernel_launches() - L0
        clocks = sampler.stop() if sampler else None
        async_status(L, stream)
        # phase times from three more (untimed, synchronous) calls
        tis = np.zeros(8)
        for _ in range(3):
            ti = np.zeros(8)
            step(precision, ti)
            tis += ti / 3
        ms = max_over_ranks(e0.elapsed_time(e1) / steps, pg, dev)
        return ms, tis, launches, clocks

    prec = args.precision
    # Process warm-up before the first timed loop: in a fresh process the first
    # calls run slower (stream-ordered pool growth, lazily loaded kernels, clock
    # ramp), which W = 3 warm-up calls do not cover.  About one second of
    # untimed calls is spent here; the W warm-up calls of timed() follow.
    prewarm_s = 1.0
    t_end = time.perf_counter() + prewarm_s
    while time.perf_counter() < t_end:
        step(prec)
        torch.cuda.synchronize()
    if pg:
        pg.barrier()
    ms, ti, launches, clocks = timed(prec, args.steps, args.warmup, with_clocks=True)
    ms64, ti64, _, _ = timed("fp64", max(2, args.steps // 2), 1) if prec != "fp64" else (ms, ti, 0, None)
    value = world * n / (ms * 1e-3)
    value64 = world * n / (ms64 * 1e-3)
    # the same mixed step with the M2L on the CUDA cores instead of tcgen05
    ms_cc = None
    if prec == "mixed":
        L.b2fmm_set_m2l_tensor_cores(0)
        ms_cc, _, _, _ = timed(prec, max(2, args.steps // 4), 1)
        L.b2fmm_set_m2l_tensor_cores(1)

    # work counts and roofline of the dominant kernel (from this run)
    L.b2fmm_set_stats(1)
    step(prec)
    L.b2fmm_set_stats(0)
    st = _lib.get_stats()
    phases = {"p2m": ti[0], "p2l": ti[1], "m2m": ti[2], "m2l": ti[3], "l2l": ti[4]}
    if prec == "mixed":
        # two kernels: k_far_mixed (L2P + M2P, FP64), then k_p2p_leaf (FP32)
        phases.update({"far(l2p+m2p)": ti[5], "p2p": ti[7]})
    else:
        phases["leaf_eval(l2p+m2p+p2p)"] = ti[7]
    phases_ms = {k: round(v * 1e3, 4) for k, v in phases.items()}
    dom = max(phases, key=phases.get)
    fma_peak = L.b2fmm_fma_peak(1 if prec == "fp64" else 0)
    nd2 = st["nd_cauchy"]
    P = st["nterms1"]
    # algorithmic flops (FMA = 2): P2P charge+dipole pot+grad per pair 15 + 28*nd2
    # (per pair: 15 real flops for the kernel terms, 28 per density); M2L per
    # translation 2*P*P real MACs x 2 (re,im) x nd2
    far_fl = st["npts_eval"] * 16 * P * nd2 + st["m2p_evals"] * 16 * P * nd2
    p2p_fl = st["p2p_pairs"] * (15 + 28 * nd2)
    flops = {"leaf_eval(l2p+m2p+p2p)": p2p_fl + far_fl, "far(l2p+m2p)": far_fl, "p2p": p2p_fl,
             "m2l": st["m2l_pairs"] * 4 * P * P * nd2}
    t_dom = phases[dom]
    achieved = flops.get(dom, 0.0) / t_dom / 1e12 if t_dom > 0 else 0.0
    counts = {k: st[k] for k in ("nboxes", "nlevels", "nleaves", "nterms1", "p2p_pairs",
                                 "m2l_pairs", "m2p_evals")}
    peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))) \
        if os.path.exists(os.path.join(ROOT, "MEASURED_PEAKS.json")) else {}
    if dom == "m2l" and prec == "mixed":
        # tensor-core M2L: useful flops against the measured dense bf16 peak
        # (MEASURED_PEAKS.json); TF32 issues at half that rate.  Issued work:
        # per tile step, 3 split products x K/8 MMAs of 128 x N x 8
        # (K = 2 KH, N = 2 KH rounded to 16, KH = P rounded to 4)
        KH = (int(P) + 3) // 4 * 4
        K, N = 2 * KH, (2 * KH + 15) // 16 * 16
        mma = st["m2l_tc_steps"] * 3 * (K // 8)
        issued = mma * (128 * N * 8 * 2)
        peak = peaks.get("bf16_tflops", 1590.0)
        roofline = {"bound": "tensor", "kernel": "m2l (k_m2l_tc, tcgen05 kind::tf32)",
                    "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                    "frac": achieved / peak, "traffic": None,
                    "issued_tensor_tflops": issued / t_dom / 1e12,
                    "tile_steps": st["m2l_tc_steps"], "mma_instructions": mma,
                    "issued_frac_of_tf32_peak": issued / t_dom / 1e12 / (peak / 2),
                    "peak_source": ("MEASURED_PEAKS.json bf16_tflops (burst)" if peaks else
                                    "fallback 1590 TFLOP/s bf16")}
    else:
        roofline = {"bound": "fma", "kernel": dom, "achieved": achieved,
                    "peak": fma_peak / 1e12, "unit": "TFLOP/s",
                    "frac": achieved / (fma_peak / 1e12), "traffic": None,
                    "peak_source": ("in-run FMA microbenchmark b2fmm_fma_peak "
                                    f"({'FP64' if prec == 'fp64' else 'FP32'})")}
    t_p2p = phases.get("p2p", phases.get("leaf_eval(l2p+m2p+p2p)", 0.0))
    roofline["near_field"] = {"bound": "fma", "pairs": st["p2p_pairs"],
                              "achieved": p2p_fl / t_p2p / 1e12 if t_p2p > 0 else 0.0,
                              "peak": fma_peak / 1e12, "unit": "TFLOP/s",
                              "note": ("k_p2p_leaf alone (FP32 pair kernel, two-float "
                                       "leaf-relative pair differences)" if "p2p" in phases else
                                       "P2P flops over the whole fused leaf kernel")}
    roofline["near_field"]["frac"] = roofline["near_field"]["achieved"] / (fma_peak / 1e12)
    roofline.update({"phase_ms": phases_ms, "tree_ms": round(st["tree_ms"], 4),
                     "counts": counts})
    prof = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(prof):
        try:
            roofline["traffic"] = json.load(open(prof)).get(dom)
        except ValueError:
            pass

    # accuracy against the FP64 direct sum on 1000 random sources
    step(prec)
    err = rel_err_vs_direct(L, ds, dq, dd, dv, src, n, pot, grad, stream, dev)
    step("fp64")
    err64 = rel_err_vs_direct(L, ds, dq, dd, dv, src, n, pot, grad, stream, dev)

    # end to end through the reference-named host entry point, pinned buffers
    hsrc = torch.as_tensor(hs).pin_memory()
    hq_ = torch.as_tensor(hq).pin_memory()
    hd_ = torch.as_tensor(hd).pin_memory()
    hv_ = torch.as_tensor(hv).pin_memory()
    hpot = torch.empty((n, 1), dtype=torch.complex128).pin_memory()
    hgrad = torch.empty((n, 2, 1), dtype=torch.complex128).pin_memory()

    def e2e_step():
        ier = C.c_int(0)
        o = _lib.Options()
        o.ndiv, o.idivflag, o.ifnear, o.precision = 0, 0, 1, _lib.PREC[prec]
        L.b2fmm_lfmm2d_ex(1, C.c_double(1e-6), C.c_int64(n), ptr(hsrc), 1, ptr(hq_), 1, ptr(hd_),
                          ptr(hv_), 2, ptr(hpot), ptr(hgrad), None, C.c_int64(0), None, 0, None,
                          None, None, C.byref(o), None, C.byref(ier))
        if ier.value != 0:
            raise RuntimeError(f"b2fmm_lfmm2d_ex ier={ier.value}")

    # blocking calls: copies in, FMM, copies out, one wait per call
    for _ in range(max(1, args.warmup - 1)):
        e2e_step()
    if pg:
        pg.barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        e2e_step()
    te_block = max_over_ranks((time.perf_counter() - t0) / args.steps, pg, dev)

    # queued calls (b2fmm_lfmm2d_host_async) on two streams in turn, each
    # with its own pinned result arrays: one call's copies overlap the other's
    # FMM; every step still copies its inputs in and its results out
    streams = [torch.cuda.Stream(dev), torch.cuda.Stream(dev)]
    hpot2 = [hpot, torch.empty_like(hpot).pin_memory()]
    hgrad2 = [hgrad, torch.empty_like(hgrad).pin_memory()]

    def e2e_async(k):
        ier = C.c_int(0)
        o = _lib.Options()
        o.ndiv, o.idivflag, o.ifnear, o.precision = 0, 0, 1, _lib.PREC[prec]
        L.b2fmm_lfmm2d_host_async(1, C.c_double(1e-6), C.c_int64(n), ptr(hsrc), 1, ptr(hq_), 1,
                                  ptr(hd_), ptr(hv_), 2, ptr(hpot2[k % 2]), ptr(hgrad2[k % 2]),
                                  None, C.c_int64(0), None, 0, None, None, None, C.byref(o),
                                  C.c_void_p(streams[k % 2].cuda_stream), C.byref(ier))
        if ier.value != 0:
            raise RuntimeError(f"b2fmm_lfmm2d_host_async ier={ier.value}")

    def queued_status():
        for s_ in streams:
            ier = C.c_int(0)
            L.b2fmm_async_status(C.c_void_p(s_.cuda_stream), C.byref(ier))
            if ier.value != 0:
                raise RuntimeError(f"b2fmm_lfmm2d_host_async: device status {ier.value}")

    for k in range(max(2, args.warmup - 1)):
        e2e_async(k)
    torch.cuda.synchronize()
    queued_status()
    if pg:
        pg.barrier()
    t0 = time.perf_counter()
    for k in range(args.steps):
        e2e_async(k)
    for s_ in streams:
        s_.synchronize()
    te = max_over_ranks((time.perf_counter() - t0) / args.steps, pg, dev)
    queued_status()
    # the queued calls' results against the blocking call's
    e2e_diff = float(torch.linalg.norm((hpot2[(args.steps - 1) % 2] - hpot).flatten()) /
                     torch.linalg.norm(hpot.flatten())) if args.steps > 1 else 0.0
    h2d = hsrc.numel() * 8 + hq_.numel() * 16 + hd_.numel() * 16 + hv_.numel() * 8
    d2h = hpot.numel() * 16 + hgrad.numel() * 16

    # the other configurations, each on a line of its own before the headline
    def emit(key, obj):
        if rank == 0 and obj is not None:
            print(json.dumps({key: obj}), flush=True)

    if not args.no_sweep:
        emit("lfmm2d_eps_sweep", c2_eps_sweep(L, n, ds, dq, dd, dv, src, pot, grad, stream, dev))
    if not args.no_c1:
        emit("rfmm2d_c1", rfmm_c1(L, dev, stream, cpu=(rank == 0 and world == 1
                                                      and not args.no_cpu_baseline)))
    if not args.no_c3:
        emit("batched_c3", batched_c3(L, dev))
    if not args.no_c5:
        from fmm2d_b200 import costmodel as cm
        model = cm.CostModel.load()
        if model is not None:
            res = cm.evaluate(model, cm.sweep_problems(40, seed0=5000))
            c5 = {k: v for k, v in res.items() if k != "rows"}
            c5["workload"] = ("40 rfmm2d problems, N log-uniform [1e4, 8e6], uniform / "
                              "16-Gaussian mixture / graded curve, eps in {1e-3, 1e-6}, pg=2")
            c5["ndiv_mlp"] = [r["ndiv_mlp"] for r in res["rows"]]
            c5["balance_mlp"] = [r["balance_mlp"] for r in res["rows"]]
            c5["ndiv_constant"] = sorted({r["ndiv_constant"] for r in res["rows"]})
            emit("costmodel_c5", c5)
    if not args.no_c4:
        emit("helmholtz_c4", helmholtz_c4(L, dev, stream, args.c4_scale))
    emit("roofline_detail", roofline)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(args.cpu_sample)

    if rank == 0:
        # the headline line last, compact: the sub-configurations are above
        rl = {k: roofline[k] for k in ("bound", "kernel", "achieved", "peak", "unit", "frac",
                                       "traffic", "peak_source")}
        rl["phase_ms"] = phases_ms
        line = {"metric": METRIC, "value": value, "unit": "points/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
                "speedup_vs_fp64": value / value64, "fp64_value": value64,
                "fp64_ms_per_step": ms64, "rel_l2_err": err, "fp64_rel_l2_err": err64,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32+f64" if prec == "mixed" else "f64", "data": "synthetic",
                "config": {"workload": WORKLOAD, "n_points_per_gpu": n, "eps": 1e-6,
                           "precision": prec, "parallelism": f"replicas x{world}",
                           "calls": "queued back to back (asynchronous), checked after",
                           "l2_policy": "inputs (256 MB) and expansions larger than L2"},
                "err_ref": "FP64 direct sum over 1000 random sources",
                "mixed_cuda_core_m2l_ms_per_step": ms_cc,
                "e2e_blocking": {"value": world * n / te_block, "unit": "points/s",
                                 "ms_per_step": te_block * 1e3,
                                 "call": "b2fmm_lfmm2d_ex, one wait per call"},
                "e2e": {"value": world * n / te, "unit": "points/s", "h2d_bytes_per_step": h2d,
                        "d2h_bytes_per_step": d2h, "ms_per_step": te * 1e3,
                        "call": "b2fmm_lfmm2d_host_async on two streams in turn",
                        "rel_diff_vs_blocking_call": e2e_diff},
                "gpu_launches": int(launches),
                "roofline": rl, "cpu_baseline": cpu, "clocks": clocks}
        print(json.dumps(line), flush=True)
    if pg:
        pg.barrier()
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
