"""Reusable FMM plans and batched evaluation in one CUDA graph (extensions;
the reference rebuilds its tree in every call).

``Plan`` keeps everything that depends only on the points (tree, lists,
sorted points, operator tables, work buffers) for repeated evaluations with
new densities, the common case of iterative solvers.  ``BatchGraph`` captures
one evaluation of many plans into a single CUDA graph whose branches run
concurrently.  Arrays are CUDA torch tensors in the C ABI layouts
(include/fmm2d_b200.h): sources (ns, 2) float64; charges / dipstr (n, nd)
complex128 (cfmm2d, lfmm2d) or float64 (rfmm2d); dipvec (n, 2, nd) float64.
"""
import ctypes as C

from . import _lib

KINDS = {"cfmm2d": 0, "lfmm2d": 1, "rfmm2d": 2}


def _p(t):
    return None if t is None else C.c_void_p(t.data_ptr())


class Plan:
    """Plan of a cfmm2d / lfmm2d / rfmm2d call on fixed sources and targets."""

    def __init__(self, kind, *, eps, sources, targets=None, charges=True, dipoles=False, pg=0,
                 pgt=0, nd=1, precision="auto", ndiv=None):
        import torch
        self.kind, self.fe, self.nd = kind, KINDS[kind], nd
        self.pg, self.pgt = pg, (pgt if targets is not None else 0)
        self.charges, self.dipoles = charges, dipoles
        self.sources = sources.contiguous()
        self.targets = None if targets is None else targets.contiguous()
        self.ns = self.sources.shape[0]
        self.nt = 0 if targets is None else self.targets.shape[0]
        o = _lib.Options()
        o.ndiv, o.idivflag, o.ifnear, o.precision = int(ndiv or 0), 0, 1, _lib.PREC[precision]
        ier = C.c_int(0)
        stream = torch.cuda.current_stream(self.sources.device).cuda_stream
        self._h = _lib.lib().b2fmm_plan_create(
            self.fe, nd, C.c_double(eps), C.c_int64(self.ns), _p(self.sources), int(charges),
            int(dipoles), pg, C.c_int64(self.nt), _p(self.targets), self.pgt, C.byref(o),
            C.c_void_p(stream), C.byref(ier))
        if not self._h:
            raise RuntimeError(f"b2fmm_plan_create ier={ier.value}")
        self.dev = self.sources.device

    def outputs(self):
        """Fresh output tensors in the C ABI layouts."""
        import torch
        dt = torch.float64 if self.fe == 2 else torch.complex128
        nd = self.nd
        g = (lambda n: (n, nd)) if self.fe == 0 else (lambda n: (n, 2, nd))
        h = (lambda n: (n, nd)) if self.fe == 0 else (lambda n: (n, 3, nd))
        mk = lambda shape, on: torch.zeros(shape, dtype=dt, device=self.dev) if on else None
        return {"pot": mk((self.ns, nd), self.pg >= 1), "grad": mk(g(self.ns), self.pg >= 2),
                "hess": mk(h(self.ns), self.pg >= 3),
                "pottarg": mk((self.nt, nd), self.pgt >= 1 and self.nt),
                "gradtarg": mk(g(self.nt), self.pgt >= 2 and self.nt),
                "hesstarg": mk(h(self.nt), self.pgt >= 3 and self.nt)}

    def eval(self, charges=None, dipstr=None, dipvec=None, out=None, stream=None):
        """Enqueue one evaluation on `stream` (default: current stream)."""
        import torch
        out = out if out is not None else self.outputs()
        st = stream if stream is not None else torch.cuda.current_stream(self.dev).cuda_stream
        ier = C.c_int(0)
        _lib.lib().b2fmm_plan_eval(self._h, _p(charges), _p(dipstr), _p(dipvec), _p(out["pot"]),
                                   _p(out["grad"]), _p(out["hess"]), _p(out["pottarg"]),
                                   _p(out["gradtarg"]), _p(out["hesstarg"]), C.c_void_p(st),
                                   C.byref(ier))
        if ier.value != 0:
            raise RuntimeError(f"b2fmm_plan_eval ier={ier.value}")
        return out

    def status(self):
        return _lib.lib().b2fmm_plan_status(self._h)

    def close(self):
        if getattr(self, "_h", None):
            _lib.lib().b2fmm_plan_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class BatchGraph:
    """One CUDA graph evaluating every plan once (concurrent branches)."""

    def __init__(self, plans, charges=None, dipstr=None, dipvec=None, outs=None, nbranch=16):
        n = len(plans)
        self.plans = plans
        self.outs = outs if outs is not None else [p.outputs() for p in plans]
        self._keep = [charges, dipstr, dipvec]
        arr = lambda ts: None if ts is None else (C.c_void_p * n)(
            *[None if t is None else t.data_ptr() for t in ts])
        col = lambda k: arr([o[k] for o in self.outs]) if any(o[k] is not None for o in self.outs) \
            else None
        self._arrays = [arr(charges), arr(dipstr), arr(dipvec)] + \
            [col(k) for k in ("pot", "grad", "hess", "pottarg", "gradtarg", "hesstarg")]
        hs = (C.c_void_p * n)(*[p._h for p in plans])
        ier = C.c_int(0)
        self._h = _lib.lib().b2fmm_batch_graph_create(n, hs, *self._arrays, nbranch, C.byref(ier))
        if not self._h:
            raise RuntimeError(f"b2fmm_batch_graph_create ier={ier.value}")

    @property
    def nodes(self):
        return int(_lib.lib().b2fmm_batch_graph_nodes(self._h))

    def launch(self, stream=None):
        import torch
        st = stream if stream is not None else torch.cuda.current_stream().cuda_stream
        ier = C.c_int(0)
        _lib.lib().b2fmm_batch_graph_launch(self._h, C.c_void_p(st), C.byref(ier))
        if ier.value != 0:
            raise RuntimeError(f"b2fmm_batch_graph_launch ier={ier.value}")

    def status(self):
        return _lib.lib().b2fmm_batch_graph_status(self._h)

    def close(self):
        if getattr(self, "_h", None):
            _lib.lib().b2fmm_batch_graph_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
