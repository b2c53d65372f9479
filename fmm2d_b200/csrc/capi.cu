// extern "C" entry points (include/fmm2d_b200.h).
#include <cstring>
#include <vector>

#include "../../include/fmm2d_b200.h"
#include "batch.cuh"
#include "biharmonic.cuh"
#include "direct.cuh"
#include "helm_special.cuh"
#include "helmholtz.cuh"
#include "laplace.cuh"
#include "tree.cuh"
#include "peaks.cuh"
#include "lap_mixed.cuh"
#include "mlp.cuh"
#include "tc_m2l.cuh"

namespace b2 {
std::atomic<unsigned long long> g_launches{0};

// allocation fault injection (b2fmm_test_fail_alloc): -1 off, else the
// number of allocations that still succeed before one fails
std::atomic<int> g_fail_after{-1};
bool alloc_fault_due() {
  int v = g_fail_after.load(std::memory_order_relaxed);
  while (v >= 0) {
    if (g_fail_after.compare_exchange_weak(v, v - 1)) return v == 0;
  }
  return false;
}
}

using namespace b2;

namespace {

template <typename F>
void guarded(int* ier, F&& f) {
  try {
    int r = f();
    if (ier) *ier = r;
  } catch (const CudaError& e) {
    fprintf(stderr, "fmm2d_b200: %s\n", e.what());
    if (ier) *ier = e.ier;
  } catch (const std::bad_alloc&) {
    if (ier) *ier = IER_ALLOC;
  } catch (...) {
    if (ier) *ier = IER_CUDA;
  }
}

LapArgs make_args(int fe, int nd, double eps, int64_t ns, const double* sources, int ifcharge,
                  const double* charge, int ifdipole, const double* dipstr, const double* dipvec,
                  int ifpgh, double* pot, double* grad, double* hess, int64_t nt,
                  const double* targ, int ifpghtarg, double* pottarg, double* gradtarg,
                  double* hesstarg, const b2fmm_options* o, double* timeinfo) {
  LapArgs a;
  a.fe = fe;
  a.nd = nd;
  a.eps = eps;
  a.ns = ns;
  a.src = sources;
  a.charge = ifcharge == 1 ? charge : nullptr;
  a.dipstr = ifdipole == 1 ? dipstr : nullptr;
  a.dipvec = ifdipole == 1 ? dipvec : nullptr;
  a.ifpgh = ifpgh;
  a.pot = pot;
  a.grad = grad;
  a.hess = hess;
  a.nt = nt;
  a.trg = targ;
  a.ifpghtarg = ifpghtarg;
  a.pottarg = pottarg;
  a.gradtarg = gradtarg;
  a.hesstarg = hesstarg;
  if (o) {
    a.ndiv = o->ndiv;
    a.lbal = o->level_balance;
    a.idivflag = o->idivflag;
    a.ifnear = o->ifnear;
    a.precision = o->precision;
    a.async_call = o->async_call == 1;
  }
  a.timeinfo = timeinfo;
  return a;
}

// Second stream of the calling thread for host->device copies that overlap
// the tree build, with the events that order it against the main stream.
struct SideStream {
  cudaStream_t s = nullptr;
  cudaEvent_t alloc_done = nullptr, copies_done = nullptr;
  ~SideStream() {
    if (copies_done) cudaEventDestroy(copies_done);
    if (alloc_done) cudaEventDestroy(alloc_done);
    if (s) cudaStreamDestroy(s);
  }
};

SideStream& side_stream() {
  thread_local SideStream ss;
  if (!ss.s) {
    B2_CHECK(cudaStreamCreateWithFlags(&ss.s, cudaStreamNonBlocking));
    B2_CHECK(cudaEventCreateWithFlags(&ss.alloc_done, cudaEventDisableTiming));
    B2_CHECK(cudaEventCreateWithFlags(&ss.copies_done, cudaEventDisableTiming));
  }
  return ss;
}

// Host-pointer driver: copies inputs to the device, runs, copies results back.
// The point coordinates go first on the main stream (the tree needs them);
// the densities follow on a side stream while the tree is being built, and
// the evaluation waits for them.  async: everything is queued on st and the
// call returns without waiting (device buffers are freed in stream order
// after the copies back; failures go to the device's status word,
// lap_async_status); otherwise one wait at the end.
int lap_host(LapArgs h, cudaStream_t st = cudaStreamPerThread, bool async = false) {
  if (h.timeinfo) async = false;
  const int nd = h.nd;
  const long ns = h.ns, nt = h.nt;
  const int cw = h.fe == FE_REAL ? 1 : 2;
  const int gw = h.fe == FE_CAUCHY ? 1 : 2, hw = h.fe == FE_CAUCHY ? 1 : 3;
  const size_t nq = (size_t)cw * nd;
  DBuf<double> src(st), trg(st), q(st), dp(st), dv(st), po(st), gr(st), he(st), pt(st), gt(st),
      ht(st);
  auto up = [&](DBuf<double>& d, const double* hp, size_t n) {
    if (!hp || n == 0) return (double*)nullptr;
    d.alloc(n, st);
    B2_CHECK(cudaMemcpyAsync(d.p, hp, n * sizeof(double), cudaMemcpyHostToDevice, st));
    return d.p;
  };
  auto mk = [&](DBuf<double>& d, size_t n) {
    if (n == 0) return (double*)nullptr;
    d.alloc(n, st);
    return d.p;
  };
  LapArgs a = h;
  a.src = up(src, h.src, 2 * (size_t)ns);
  a.trg = up(trg, h.ifpghtarg > 0 ? h.trg : nullptr, 2 * (size_t)nt);
  // densities: allocated on the main stream, copied on the side stream
  SideStream& ss = side_stream();
  const double* hq = h.charge;
  const double* hd = h.dipstr;
  const double* hv = h.fe != FE_CAUCHY && h.dipstr ? h.dipvec : nullptr;
  a.charge = hq ? mk(q, nq * ns) : nullptr;
  a.dipstr = hd ? mk(dp, nq * ns) : nullptr;
  a.dipvec = hv ? mk(dv, 2 * (size_t)nd * ns) : nullptr;
  B2_CHECK(cudaEventRecord(ss.alloc_done, st));
  B2_CHECK(cudaStreamWaitEvent(ss.s, ss.alloc_done, 0));
  auto side_up = [&](const double* dst, const double* hp, size_t n) {
    if (dst && hp && n)
      B2_CHECK(cudaMemcpyAsync((void*)dst, hp, n * sizeof(double), cudaMemcpyHostToDevice, ss.s));
  };
  side_up(a.charge, hq, nq * ns);
  side_up(a.dipstr, hd, nq * ns);
  side_up(a.dipvec, hv, 2 * (size_t)nd * ns);
  B2_CHECK(cudaEventRecord(ss.copies_done, ss.s));
  // whatever happens below, the main stream (on which the buffers are freed)
  // waits for the side copies first
  struct WaitOnExit {
    cudaStream_t st;
    cudaEvent_t e;
    ~WaitOnExit() { cudaStreamWaitEvent(st, e, 0); }
  } wait_guard{st, ss.copies_done};
  a.pot = h.ifpgh >= 1 ? mk(po, nq * ns) : nullptr;
  a.grad = h.ifpgh >= 2 ? mk(gr, nq * gw * ns) : nullptr;
  a.hess = h.ifpgh >= 3 ? mk(he, nq * hw * ns) : nullptr;
  a.pottarg = h.ifpghtarg >= 1 ? mk(pt, nq * nt) : nullptr;
  a.gradtarg = h.ifpghtarg >= 2 ? mk(gt, nq * gw * nt) : nullptr;
  a.hesstarg = h.ifpghtarg >= 3 ? mk(ht, nq * hw * nt) : nullptr;
  auto down = [&](double* hp, const double* dpp, size_t n) {
    if (hp && dpp && n) B2_CHECK(cudaMemcpyAsync(hp, dpp, n * sizeof(double), cudaMemcpyDeviceToHost, st));
  };
  auto down_all = [&] {
    down(h.pot, a.pot, nq * ns);
    down(h.grad, a.grad, nq * gw * ns);
    down(h.hess, a.hess, nq * hw * ns);
    down(h.pottarg, a.pottarg, nq * nt);
    down(h.gradtarg, a.gradtarg, nq * gw * nt);
    down(h.hesstarg, a.hesstarg, nq * hw * nt);
  };
  if (async) {
    a.async_call = true;
    a.status_word = nullptr;  // the device's status word
    int r = lap_fmm_device(a, st, ss.copies_done);
    if (r != IER_OK) return r;
    down_all();
    return IER_OK;
  }
  // the whole call (copies in, FMM, copies out) is queued before the one
  // wait; the FMM's outcome comes back in the call's own status word
  DBuf<int> status(st);
  status.alloc(1, st);
  status.zero(1);
  a.async_call = !h.timeinfo;
  a.status_word = status.p;
  int r = lap_fmm_device(a, st, ss.copies_done);
  if (r != IER_OK) return r;
  down_all();
  int* hs = pinned_ints(1);
  B2_CHECK(cudaMemcpyAsync(hs, status.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  B2_CHECK(cudaStreamSynchronize(st));
  const int code = a.async_call ? hs[0] : IER_OK;
  if (code == IER_TREE_LIMIT) {
    // the tree needs the build with read-back: run the FMM again that way
    a.async_call = false;
    a.status_word = nullptr;
    r = lap_fmm_device(a, st, nullptr);
    if (r != IER_OK) return r;
    down_all();
    B2_CHECK(cudaStreamSynchronize(st));
    return IER_OK;
  }
  return code;
}

HelmArgs make_hargs(int nd, double eps, double zkr, double zki, int64_t ns, const double* sources,
                    int ifcharge, const double* charge, int ifdipole, const double* dipstr,
                    const double* dipvec, int ifpgh, double* pot, double* grad, double* hess,
                    int64_t nt, const double* targ, int ifpghtarg, double* pottarg,
                    double* gradtarg, double* hesstarg, const b2fmm_options* o,
                    double* timeinfo) {
  HelmArgs a;
  a.nd = nd;
  a.eps = eps;
  a.zkr = zkr;
  a.zki = zki;
  a.ns = ns;
  a.src = sources;
  a.charge = ifcharge == 1 ? charge : nullptr;
  a.dipstr = ifdipole == 1 ? dipstr : nullptr;
  a.dipvec = ifdipole == 1 ? dipvec : nullptr;
  a.ifpgh = ifpgh;
  a.pot = pot;
  a.grad = grad;
  a.hess = hess;
  a.nt = nt;
  a.trg = targ;
  a.ifpghtarg = ifpghtarg;
  a.pottarg = pottarg;
  a.gradtarg = gradtarg;
  a.hesstarg = hesstarg;
  if (o) {
    a.ndiv = o->ndiv;
    a.ifnear = o->ifnear;
  }
  a.timeinfo = timeinfo;
  return a;
}

// Host-pointer Helmholtz driver (complex values interleaved re/im).
int helm_host(HelmArgs h) {
  cudaStream_t st = cudaStreamPerThread;
  const int nd = h.nd;
  const long ns = h.ns, nt = h.ifpghtarg > 0 ? h.nt : 0;
  const size_t nq = 2 * (size_t)nd;
  DBuf<double> src(st), trg(st), q(st), dp(st), dv(st), po(st), gr(st), he(st), pt(st), gt(st),
      ht(st);
  auto up = [&](DBuf<double>& d, const double* hp, size_t n) {
    if (!hp || n == 0) return (double*)nullptr;
    d.alloc(n, st);
    B2_CHECK(cudaMemcpyAsync(d.p, hp, n * sizeof(double), cudaMemcpyHostToDevice, st));
    return d.p;
  };
  auto mk = [&](DBuf<double>& d, size_t n) {
    if (n == 0) return (double*)nullptr;
    d.alloc(n, st);
    return d.p;
  };
  HelmArgs a = h;
  a.src = up(src, h.src, 2 * (size_t)ns);
  a.trg = up(trg, nt > 0 ? h.trg : nullptr, 2 * (size_t)nt);
  a.charge = up(q, h.charge, nq * ns);
  a.dipstr = up(dp, h.dipstr, nq * ns);
  a.dipvec = up(dv, h.dipstr ? h.dipvec : nullptr, 2 * (size_t)nd * ns);
  a.pot = h.ifpgh >= 1 ? mk(po, nq * ns) : nullptr;
  a.grad = h.ifpgh >= 2 ? mk(gr, nq * 2 * ns) : nullptr;
  a.hess = h.ifpgh >= 3 ? mk(he, nq * 3 * ns) : nullptr;
  a.pottarg = h.ifpghtarg >= 1 ? mk(pt, nq * nt) : nullptr;
  a.gradtarg = h.ifpghtarg >= 2 ? mk(gt, nq * 2 * nt) : nullptr;
  a.hesstarg = h.ifpghtarg >= 3 ? mk(ht, nq * 3 * nt) : nullptr;
  int r = helm_fmm_device(a, st);
  if (r != IER_OK) return r;
  auto down = [&](double* hp, const double* dpp, size_t n) {
    if (hp && dpp && n) B2_CHECK(cudaMemcpyAsync(hp, dpp, n * sizeof(double), cudaMemcpyDeviceToHost, st));
  };
  down(h.pot, a.pot, nq * ns);
  down(h.grad, a.grad, nq * 2 * ns);
  down(h.hess, a.hess, nq * 3 * ns);
  down(h.pottarg, a.pottarg, nq * nt);
  down(h.gradtarg, a.gradtarg, nq * 2 * nt);
  down(h.hesstarg, a.hesstarg, nq * 3 * nt);
  B2_CHECK(cudaStreamSynchronize(st));
  return IER_OK;
}

struct TreeHandle {
  DeviceTree T;
};

}  // namespace

extern "C" {

const char* b2fmm_version(void) { return "fmm2d_b200 0.1 (sm_100a)"; }

void b2fmm_cfmm2d(int nd, double eps, int64_t ns, const double* sources, int ifcharge,
                  const double* charge, int ifdipole, const double* dipstr, int iper, int ifpgh,
                  double* pot, double* grad, double* hess, int64_t nt, const double* targ,
                  int ifpghtarg, double* pottarg, double* gradtarg, double* hesstarg, int* ier) {
  (void)iper;
  guarded(ier, [&] {
    return lap_host(make_args(FE_CAUCHY, nd, eps, ns, sources, ifcharge, charge, ifdipole, dipstr,
                              nullptr, ifpgh, pot, grad, hess, nt, targ, ifpghtarg, pottarg,
                              gradtarg, hesstarg, nullptr, nullptr));
  });
}

void b2fmm_lfmm2d(int nd, double eps, int64_t ns, const double* sources, int ifcharge,
                  const double* charge, int ifdipole, const double* dipstr, const double* dipvec,
                  int iper, int ifpgh, double* pot, double* grad, double* hess, int64_t nt,
                  const double* targ, int ifpghtarg, double* pottarg, double* gradtarg,
                  double* hesstarg, int* ier) {
  (void)iper;
  guarded(ier, [&] {
    return lap_host(make_args(FE_LAPLACE, nd, eps, ns, sources, ifcharge, charge, ifdipole, dipstr,
                              dipvec, ifpgh, pot, grad, hess, nt, targ, ifpghtarg, pottarg,
                              gradtarg, hesstarg, nullptr, nullptr));
  });
}

void b2fmm_rfmm2d(int nd, double eps, int64_t ns, const double* sources, int ifcharge,
                  const double* charge, int ifdipole, const double* dipstr, const double* dipvec,
                  int iper, int ifpgh, double* pot, double* grad, double* hess, int64_t nt,
                  const double* targ, int ifpghtarg, double* pottarg, double* gradtarg,
                  double* hesstarg, int* ier) {
  (void)iper;
  guarded(ier, [&] {
    return lap_host(make_args(FE_REAL, nd, eps, ns, sources, ifcharge, charge, ifdipole, dipstr,
                              dipvec, ifpgh, pot, grad, hess, nt, targ, ifpghtarg, pottarg,
                              gradtarg, hesstarg, nullptr, nullptr));
  });
}

void b2fmm_cfmm2d_ndiv(int nd, double eps, int64_t ns, const double* sources, int ifcharge,
                       const double* charge, int ifdipole, const double* dipstr, int iper,
                       int ifpgh, double* pot, double* grad, double* hess, int64_t nt,
                       const double* targ, int ifpghtarg, double* pottarg, double* gradtarg,
                       double* hesstarg, int ndiv, int idivflag, int ifnear, double* timeinfo,
                       int* ier) {
  (void)iper;
  b2fmm_options o{ndiv, idivflag, ifnear, PREC_AUTO};
  guarded(ier, [&] {
    return lap_host(make_args(FE_CAUCHY, nd, eps, ns, sources, ifcharge, charge, ifdipole, dipstr,
                              nullptr, ifpgh, pot, grad, hess, nt, targ, ifpghtarg, pottarg,
                              gradtarg, hesstarg, &o, timeinfo));
  });
}

void b2fmm_lfmm2d_ndiv(int nd, double eps, int64_t ns, const double* sources, int ifcharge,
                       const double* charge, int ifdipole, const double* dipstr,
                       const double* dipvec, int iper, int ifpgh, double* pot, double* grad,
                       double* hess, int64_t nt, const double* targ, int ifpghtarg,
                       double* pottarg, double* gradtarg, double* hesstarg, int ndiv,
                       int idivflag, int ifnear, double* timeinfo, int* ier) {
  (void)iper;
  b2fmm_options o{ndiv, idivflag, ifnear, PREC_AUTO};
  guarded(ier, [&] {
    return lap_host(make_args(FE_LAPLACE, nd, eps, ns, sources, ifcharge, charge, ifdipole, dipstr,
                              dipvec, ifpgh, pot, grad, hess, nt, targ, ifpghtarg, pottarg,
                              gradtarg, hesstarg, &o, timeinfo));
  });
}

void b2fmm_rfmm2d_ndiv(int nd, double eps, int64_t ns, const double* sources, int ifcharge,
                       const double* charge, int ifdipole, const double* dipstr,
                       const double* dipvec, int iper, int ifpgh, double* pot, double* grad,
                       double* hess, int64_t nt, const double* targ, int ifpghtarg,
                       double* pottarg, double* gradtarg, double* hesstarg, int ndiv,
                       int idivflag, int ifnear, double* timeinfo, int* ier) {
  (void)iper;
  b2fmm_options o{ndiv, idivflag, ifnear, PREC_AUTO};
  guarded(ier, [&] {
    return lap_host(make_args(FE_REAL, nd, eps, ns, sources, ifcharge, charge, ifdipole, dipstr,
                              dipvec, ifpgh, pot, grad, hess, nt, targ, ifpghtarg, pottarg,
                              gradtarg, hesstarg, &o, timeinfo));
  });
}

void b2fmm_cfmm2d_ex(int nd, double eps, int64_t ns, const double* sources, int ifcharge,
                     const double* charge, int ifdipole, const double* dipstr, int ifpgh,
                     double* pot, double* grad, double* hess, int64_t nt, const double* targ,
                     int ifpghtarg, double* pottarg, double* gradtarg, double* hesstarg,
                     const b2fmm_options* opts, double* timeinfo, int* ier) {
  guarded(ier, [&] {
    return lap_host(make_args(FE_CAUCHY, nd, eps, ns, sources, ifcharge, charge, ifdipole, dipstr,
                              nullptr, ifpgh, pot, grad, hess, nt, targ, ifpghtarg, pottarg,
                              gradtarg, hesstarg, opts, timeinfo));
  });
}

void b2fmm_lfmm2d_ex(int nd, double eps, int64_t ns, const double* sources, int ifcharge,
                     const double* charge, int ifdipole, const double* dipstr,
                     const double* dipvec, int ifpgh, double* pot, double* grad, double* hess,
                     int64_t nt, const double* targ, int ifpghtarg, double* pottarg,
                     double* gradtarg, double* hesstarg, const b2fmm_options* opts,
                     double* timeinfo, int* ier) {
  guarded(ier, [&] {
    return lap_host(make_args(FE_LAPLACE, nd, eps, ns, sources, ifcharge, charge, ifdipole, dipstr,
                              dipvec, ifpgh, pot, grad, hess, nt, targ, ifpghtarg, pottarg,
                              gradtarg, hesstarg, opts, timeinfo));
  });
}

void b2fmm_rfmm2d_ex(int nd, double eps, int64_t ns, const double* sources, int ifcharge,
                     const double* charge, int ifdipole, const double* dipstr,
                     const double* dipvec, int ifpgh, double* pot, double* grad, double* hess,
                     int64_t nt, const double* targ, int ifpghtarg, double* pottarg,
                     double* gradtarg, double* hesstarg, const b2fmm_options* opts,
                     double* timeinfo, int* ier) {
  guarded(ier, [&] {
    return lap_host(make_args(FE_REAL, nd, eps, ns, sources, ifcharge, charge, ifdipole, dipstr,
                              dipvec, ifpgh, pot, grad, hess, nt, targ, ifpghtarg, pottarg,
                              gradtarg, hesstarg, opts, timeinfo));
  });
}

void b2fmm_cfmm2d_host_async(int nd, double eps, int64_t ns, const double* sources,
                             int ifcharge, const double* charge, int ifdipole,
                             const double* dipstr, int ifpgh, double* pot, double* grad,
                             double* hess, int64_t nt, const double* targ, int ifpghtarg,
                             double* pottarg, double* gradtarg, double* hesstarg,
                             const b2fmm_options* opts, void* stream, int* ier) {
  guarded(ier, [&] {
    return lap_host(make_args(FE_CAUCHY, nd, eps, ns, sources, ifcharge, charge, ifdipole,
                              dipstr, nullptr, ifpgh, pot, grad, hess, nt, targ, ifpghtarg,
                              pottarg, gradtarg, hesstarg, opts, nullptr),
                    (cudaStream_t)stream, true);
  });
}

void b2fmm_lfmm2d_host_async(int nd, double eps, int64_t ns, const double* sources,
                             int ifcharge, const double* charge, int ifdipole,
                             const double* dipstr, const double* dipvec, int ifpgh, double* pot,
                             double* grad, double* hess, int64_t nt, const double* targ,
                             int ifpghtarg, double* pottarg, double* gradtarg, double* hesstarg,
                             const b2fmm_options* opts, void* stream, int* ier) {
  guarded(ier, [&] {
    return lap_host(make_args(FE_LAPLACE, nd, eps, ns, sources, ifcharge, charge, ifdipole,
                              dipstr, dipvec, ifpgh, pot, grad, hess, nt, targ, ifpghtarg,
                              pottarg, gradtarg, hesstarg, opts, nullptr),
                    (cudaStream_t)stream, true);
  });
}

void b2fmm_rfmm2d_host_async(int nd, double eps, int64_t ns, const double* sources,
                             int ifcharge, const double* charge, int ifdipole,
                             const double* dipstr, const double* dipvec, int ifpgh, double* pot,
                             double* grad, double* hess, int64_t nt, const double* targ,
                             int ifpghtarg, double* pottarg, double* gradtarg, double* hesstarg,
                             const b2fmm_options* opts, void* stream, int* ier) {
  guarded(ier, [&] {
    return lap_host(make_args(FE_REAL, nd, eps, ns, sources, ifcharge, charge, ifdipole, dipstr,
                              dipvec, ifpgh, pot, grad, hess, nt, targ, ifpghtarg, pottarg,
                              gradtarg, hesstarg, opts, nullptr),
                    (cudaStream_t)stream, true);
  });
}

void b2fmm_cfmm2d_dev(int nd, double eps, int64_t ns, const double* sources, int ifcharge,
                      const double* charge, int ifdipole, const double* dipstr, int ifpgh,
                      double* pot, double* grad, double* hess, int64_t nt, const double* targ,
                      int ifpghtarg, double* pottarg, double* gradtarg, double* hesstarg,
                      const b2fmm_options* opts, double* timeinfo, void* stream, int* ier) {
  guarded(ier, [&] {
    return lap_fmm_device(make_args(FE_CAUCHY, nd, eps, ns, sources, ifcharge, charge, ifdipole,
                                    dipstr, nullptr, ifpgh, pot, grad, hess, nt, targ, ifpghtarg,
                                    pottarg, gradtarg, hesstarg, opts, timeinfo),
                          (cudaStream_t)stream);
  });
}

void b2fmm_lfmm2d_dev(int nd, double eps, int64_t ns, const double* sources, int ifcharge,
                      const double* charge, int ifdipole, const double* dipstr,
                      const double* dipvec, int ifpgh, double* pot, double* grad, double* hess,
                      int64_t nt, const double* targ, int ifpghtarg, double* pottarg,
                      double* gradtarg, double* hesstarg, const b2fmm_options* opts,
                      double* timeinfo, void* stream, int* ier) {
  guarded(ier, [&] {
    return lap_fmm_device(make_args(FE_LAPLACE, nd, eps, ns, sources, ifcharge, charge, ifdipole,
                                    dipstr, dipvec, ifpgh, pot, grad, hess, nt, targ, ifpghtarg,
                                    pottarg, gradtarg, hesstarg, opts, timeinfo),
                          (cudaStream_t)stream);
  });
}

void b2fmm_rfmm2d_dev(int nd, double eps, int64_t ns, const double* sources, int ifcharge,
                      const double* charge, int ifdipole, const double* dipstr,
                      const double* dipvec, int ifpgh, double* pot, double* grad, double* hess,
                      int64_t nt, const double* targ, int ifpghtarg, double* pottarg,
                      double* gradtarg, double* hesstarg, const b2fmm_options* opts,
                      double* timeinfo, void* stream, int* ier) {
  guarded(ier, [&] {
    return lap_fmm_device(make_args(FE_REAL, nd, eps, ns, sources, ifcharge, charge, ifdipole,
                                    dipstr, dipvec, ifpgh, pot, grad, hess, nt, targ, ifpghtarg,
                                    pottarg, gradtarg, hesstarg, opts, timeinfo),
                          (cudaStream_t)stream);
  });
}

void b2fmm_lap_direct_dev(int kind, int nd, int64_t ns, const double* sources,
                          const double* charge, const double* dipstr, const double* dipvec,
                          int64_t nt, const double* targ, int ifpgh, double* pot, double* grad,
                          double* hess, double thresh, void* stream, int* ier) {
  guarded(ier, [&] {
    return lap_direct_device(kind, nd, ns, sources, charge, dipstr, dipvec, nt, targ, ifpgh, pot,
                             grad, hess, thresh, (cudaStream_t)stream);
  });
}

void b2fmm_lap_direct_noalloc_dev(int kind, int nd, int64_t ns, const double* sources,
                                  const double* charge, const double* dipstr,
                                  const double* dipvec, int64_t nt, const double* targ,
                                  int ifpgh, double* pot, double* grad, double* hess,
                                  double thresh, void* stream, int* ier) {
  guarded(ier, [&] {
    return lap_direct_device_noalloc(kind, nd, ns, sources, charge, dipstr, dipvec, nt, targ,
                                     ifpgh, pot, grad, hess, thresh, (cudaStream_t)stream);
  });
}

void b2fmm_hfmm2d(int nd, double eps, double zk_re, double zk_im, int64_t ns,
                  const double* sources, int ifcharge, const double* charge, int ifdipole,
                  const double* dipstr, const double* dipvec, int iper, int ifpgh, double* pot,
                  double* grad, double* hess, int64_t nt, const double* targ, int ifpghtarg,
                  double* pottarg, double* gradtarg, double* hesstarg, int* ier) {
  (void)iper;
  guarded(ier, [&] {
    return helm_host(make_hargs(nd, eps, zk_re, zk_im, ns, sources, ifcharge, charge, ifdipole,
                                dipstr, dipvec, ifpgh, pot, grad, hess, nt, targ, ifpghtarg,
                                pottarg, gradtarg, hesstarg, nullptr, nullptr));
  });
}

void b2fmm_hfmm2d_ndiv(int nd, double eps, double zk_re, double zk_im, int64_t ns,
                       const double* sources, int ifcharge, const double* charge, int ifdipole,
                       const double* dipstr, const double* dipvec, int iper, int ifpgh,
                       double* pot, double* grad, double* hess, int64_t nt, const double* targ,
                       int ifpghtarg, double* pottarg, double* gradtarg, double* hesstarg,
                       int ndiv, int idivflag, int ifnear, double* timeinfo, int* ier) {
  (void)iper;
  (void)idivflag;
  b2fmm_options o{ndiv, 0, ifnear, PREC_FP64};
  guarded(ier, [&] {
    return helm_host(make_hargs(nd, eps, zk_re, zk_im, ns, sources, ifcharge, charge, ifdipole,
                                dipstr, dipvec, ifpgh, pot, grad, hess, nt, targ, ifpghtarg,
                                pottarg, gradtarg, hesstarg, &o, timeinfo));
  });
}

void b2fmm_hfmm2d_dev(int nd, double eps, double zk_re, double zk_im, int64_t ns,
                      const double* sources, int ifcharge, const double* charge, int ifdipole,
                      const double* dipstr, const double* dipvec, int ifpgh, double* pot,
                      double* grad, double* hess, int64_t nt, const double* targ, int ifpghtarg,
                      double* pottarg, double* gradtarg, double* hesstarg,
                      const b2fmm_options* opts, double* timeinfo, void* stream, int* ier) {
  guarded(ier, [&] {
    return helm_fmm_device(make_hargs(nd, eps, zk_re, zk_im, ns, sources, ifcharge, charge,
                                      ifdipole, dipstr, dipvec, ifpgh, pot, grad, hess, nt, targ,
                                      ifpghtarg, pottarg, gradtarg, hesstarg, opts, timeinfo),
                           (cudaStream_t)stream);
  });
}

namespace {
// Host arrays in, device copies, a device call, results back: inputs (host
// pointer, doubles) and outputs (host pointer, doubles); null entries skip.
struct HostIO {
  cudaStream_t st = cudaStreamPerThread;
  std::vector<DBuf<double>*> bufs;
  std::vector<std::pair<double*, const double*>> outs;  // host, device
  std::vector<size_t> out_n;
  ~HostIO() {
    for (auto* b : bufs) delete b;
  }
  const double* in(const double* h, size_t n) {
    if (!h || n == 0) return nullptr;
    auto* b = new DBuf<double>(st);
    bufs.push_back(b);
    b->alloc(n, st);
    B2_CHECK(cudaMemcpyAsync(b->p, h, n * sizeof(double), cudaMemcpyHostToDevice, st));
    return b->p;
  }
  double* out(double* h, size_t n) {
    if (!h || n == 0) return nullptr;
    auto* b = new DBuf<double>(st);
    bufs.push_back(b);
    b->alloc(n, st);
    outs.push_back({h, b->p});
    out_n.push_back(n);
    return b->p;
  }
  void finish() {
    for (size_t k = 0; k < outs.size(); k++)
      B2_CHECK(cudaMemcpyAsync(outs[k].first, outs[k].second, out_n[k] * sizeof(double),
                               cudaMemcpyDeviceToHost, st));
    B2_CHECK(cudaStreamSynchronize(st));
  }
};

BhArgs bh_args(int nd, double eps, int64_t ns, const double* sources, int ifcharge,
               const double* charge, int ifdipole, const double* dip, int ifpgh, double* pot,
               double* grad, int64_t nt, const double* targ, int ifpghtarg, double* pottarg,
               double* gradtarg) {
  BhArgs b;
  b.nd = nd;
  b.eps = eps;
  b.ns = ns;
  b.src = sources;
  b.charge = ifcharge == 1 ? charge : nullptr;
  b.dip = ifdipole == 1 ? dip : nullptr;
  b.ifpgh = ifpgh;
  b.pot = pot;
  b.grad = grad;
  b.nt = nt;
  b.trg = targ;
  b.ifpghtarg = ifpghtarg;
  b.pottarg = pottarg;
  b.gradtarg = gradtarg;
  return b;
}

StArgs st_args(int nd, double eps, int64_t ns, const double* sources, int ifstoklet,
               const double* stoklet, int ifstrslet, const double* strslet, const double* strsvec,
               int ifppreg, double* pot, double* pre, double* grad, int64_t nt, const double* targ,
               int ifppregtarg, double* pottarg, double* pretarg, double* gradtarg) {
  StArgs a;
  a.nd = nd;
  a.eps = eps;
  a.ns = ns;
  a.src = sources;
  a.stoklet = ifstoklet == 1 ? stoklet : nullptr;
  a.strslet = ifstrslet == 1 ? strslet : nullptr;
  a.strsvec = ifstrslet == 1 ? strsvec : nullptr;
  a.ifppreg = ifppreg;
  a.pot = pot;
  a.pre = pre;
  a.grad = grad;
  a.nt = nt;
  a.trg = targ;
  a.ifppregtarg = ifppregtarg;
  a.pottarg = pottarg;
  a.pretarg = pretarg;
  a.gradtarg = gradtarg;
  return a;
}
}  // namespace

void b2fmm_bhfmm2d_dev(int nd, double eps, int64_t ns, const double* sources, int ifcharge,
                       const double* charge, int ifdipole, const double* dip, int ifpgh,
                       double* pot, double* grad, int64_t nt, const double* targ, int ifpghtarg,
                       double* pottarg, double* gradtarg, void* stream, int* ier) {
  guarded(ier, [&] {
    return bh_device(bh_args(nd, eps, ns, sources, ifcharge, charge, ifdipole, dip, ifpgh, pot,
                             grad, nt, targ, ifpghtarg, pottarg, gradtarg),
                     (cudaStream_t)stream);
  });
}

void b2fmm_bh2ddir_dev(int nd, int64_t ns, const double* sources, const double* charge,
                       const double* dip, int64_t nt, const double* targ, int ifpgh, double* pot,
                       double* grad, double thresh, void* stream, int* ier) {
  guarded(ier, [&] {
    BhArgs b = bh_args(nd, 0.0, ns, sources, charge ? 1 : 0, charge, dip ? 1 : 0, dip, 0, nullptr,
                       nullptr, nt, targ, ifpgh, pot, grad);
    b.direct = true;
    b.thresh = thresh;
    return bh_device(b, (cudaStream_t)stream);
  });
}

void b2fmm_bhfmm2d(int nd, double eps, int64_t ns, const double* sources, int ifcharge,
                   const double* charge, int ifdipole, const double* dip, int iper, int ifpgh,
                   double* pot, double* grad, double* hess, int64_t nt, const double* targ,
                   int ifpghtarg, double* pottarg, double* gradtarg, double* hesstarg, int* ier) {
  (void)iper;
  (void)hess;
  (void)hesstarg;
  guarded(ier, [&] {
    if (nd < 1 || ns < 0 || nt < 0) return (int)IER_BADARG;
    HostIO io;
    const size_t n2 = 2 * (size_t)nd;  // doubles per complex density
    const int ifs = std::min(ifpgh, 2), ift = std::min(ifpghtarg, 2);
    const long ntt = ift > 0 ? nt : 0;
    BhArgs b = bh_args(
        nd, eps, ns, io.in(sources, 2 * (size_t)ns), ifcharge,
        ifcharge == 1 ? io.in(charge, n2 * 2 * ns) : nullptr, ifdipole,
        ifdipole == 1 ? io.in(dip, n2 * 3 * ns) : nullptr, ifs,
        ifs >= 1 ? io.out(pot, n2 * ns) : nullptr, ifs >= 2 ? io.out(grad, n2 * 3 * ns) : nullptr,
        ntt, io.in(targ, 2 * (size_t)ntt), ift, ift >= 1 ? io.out(pottarg, n2 * ntt) : nullptr,
        ift >= 2 ? io.out(gradtarg, n2 * 3 * ntt) : nullptr);
    int r = bh_device(b, io.st);
    if (r != IER_OK) return r;
    io.finish();
    return (int)IER_OK;
  });
}

void b2fmm_stfmm2d_dev(int nd, double eps, int64_t ns, const double* sources, int ifstoklet,
                       const double* stoklet, int ifstrslet, const double* strslet,
                       const double* strsvec, int ifppreg, double* pot, double* pre, double* grad,
                       int64_t nt, const double* targ, int ifppregtarg, double* pottarg,
                       double* pretarg, double* gradtarg, void* stream, int* ier) {
  guarded(ier, [&] {
    return stokes_device(st_args(nd, eps, ns, sources, ifstoklet, stoklet, ifstrslet, strslet,
                                 strsvec, ifppreg, pot, pre, grad, nt, targ, ifppregtarg, pottarg,
                                 pretarg, gradtarg),
                         (cudaStream_t)stream);
  });
}

void b2fmm_st2ddir_dev(int nd, int64_t ns, const double* sources, int ifstoklet,
                       const double* stoklet, int ifstrslet, const double* strslet,
                       const double* strsvec, int64_t nt, const double* targ, int ifppreg,
                       double* pot, double* pre, double* grad, double thresh, void* stream,
                       int* ier) {
  guarded(ier, [&] {
    StArgs a = st_args(nd, 0.0, ns, sources, ifstoklet, stoklet, ifstrslet, strslet, strsvec, 0,
                       nullptr, nullptr, nullptr, nt, targ, ifppreg, pot, pre, grad);
    a.direct = true;
    a.thresh = thresh;
    return stokes_device(a, (cudaStream_t)stream);
  });
}

void b2fmm_stfmm2d(int nd, double eps, int64_t ns, const double* sources, int ifstoklet,
                   const double* stoklet, int ifstrslet, const double* strslet,
                   const double* strsvec, int ifppreg, double* pot, double* pre, double* grad,
                   int64_t nt, const double* targ, int ifppregtarg, double* pottarg,
                   double* pretarg, double* gradtarg, int* ier) {
  guarded(ier, [&] {
    if (nd < 1 || ns < 0 || nt < 0) return (int)IER_BADARG;
    HostIO io;
    const size_t nn = (size_t)nd;
    const int ifs = std::min(ifppreg, 3), ift = std::min(ifppregtarg, 3);
    const long ntt = ift > 0 ? nt : 0;
    StArgs a = st_args(
        nd, eps, ns, io.in(sources, 2 * (size_t)ns), ifstoklet,
        ifstoklet == 1 ? io.in(stoklet, nn * 2 * ns) : nullptr, ifstrslet,
        ifstrslet == 1 ? io.in(strslet, nn * 2 * ns) : nullptr,
        ifstrslet == 1 ? io.in(strsvec, nn * 2 * ns) : nullptr, ifs,
        ifs >= 1 ? io.out(pot, nn * 2 * ns) : nullptr, ifs >= 2 ? io.out(pre, nn * ns) : nullptr,
        ifs >= 3 ? io.out(grad, nn * 4 * ns) : nullptr, ntt, io.in(targ, 2 * (size_t)ntt), ift,
        ift >= 1 ? io.out(pottarg, nn * 2 * ntt) : nullptr,
        ift >= 2 ? io.out(pretarg, nn * ntt) : nullptr,
        ift >= 3 ? io.out(gradtarg, nn * 4 * ntt) : nullptr);
    int r = stokes_device(a, io.st);
    if (r != IER_OK) return r;
    io.finish();
    return (int)IER_OK;
  });
}

void b2fmm_hfmm2d_mps(int nd, double eps, double zk_re, double zk_im, int64_t nmpole,
                      const double* cmpole, const double* rmpole, const int* mterms,
                      int64_t ntot, const double* mpole, const int* impole, double* local,
                      int* ier) {
  guarded(ier, [&] {
    if (nd < 1 || nmpole < 0 || ntot < 0) return (int)IER_BADARG;
    if (nmpole == 0) return (int)IER_OK;
    if (!cmpole || !rmpole || !mterms || !mpole || !impole || !local) return (int)IER_BADARG;
    // every (nd, -m..m) block inside the coefficient arrays
    int mmax = 0;
    for (int64_t i = 0; i < nmpole; i++) {
      const int64_t m = mterms[i], o = (int64_t)impole[i] - 1;
      if (m < 0 || o < 0 || o + (int64_t)nd * (2 * m + 1) > ntot) return (int)IER_BADARG;
      mmax = std::max(mmax, (int)m);
    }
    cudaStream_t st = cudaStreamPerThread;
    DBuf<double> c(st), r(st), mp(st), lo(st);
    DBuf<int> mt(st), im(st);
    c.alloc(2 * (size_t)nmpole, st);
    r.alloc(nmpole, st);
    mt.alloc(nmpole, st);
    im.alloc(nmpole, st);
    mp.alloc(2 * (size_t)ntot, st);
    lo.alloc(2 * (size_t)ntot, st);
    B2_CHECK(cudaMemcpyAsync(c.p, cmpole, sizeof(double) * 2 * nmpole, cudaMemcpyHostToDevice, st));
    B2_CHECK(cudaMemcpyAsync(r.p, rmpole, sizeof(double) * nmpole, cudaMemcpyHostToDevice, st));
    B2_CHECK(cudaMemcpyAsync(mt.p, mterms, sizeof(int) * nmpole, cudaMemcpyHostToDevice, st));
    B2_CHECK(cudaMemcpyAsync(im.p, impole, sizeof(int) * nmpole, cudaMemcpyHostToDevice, st));
    B2_CHECK(cudaMemcpyAsync(mp.p, mpole, sizeof(double) * 2 * ntot, cudaMemcpyHostToDevice, st));
    // entries outside every block keep the caller's values, as in the reference
    B2_CHECK(cudaMemcpyAsync(lo.p, local, sizeof(double) * 2 * ntot, cudaMemcpyHostToDevice, st));
    int rc = helm_mps_device(nd, eps, zk_re, zk_im, nmpole, c.p, r.p, mt.p, im.p, ntot, mp.p,
                             lo.p, mmax, st);
    if (rc != IER_OK) return rc;
    B2_CHECK(cudaMemcpyAsync(local, lo.p, sizeof(double) * 2 * ntot, cudaMemcpyDeviceToHost, st));
    B2_CHECK(cudaStreamSynchronize(st));
    return (int)IER_OK;
  });
}

void b2fmm_h2ddir_dev(int nd, double zk_re, double zk_im, int64_t ns, const double* sources,
                      const double* charge, const double* dipstr, const double* dipvec,
                      int64_t nt, const double* targ, int ifpgh, double* pot, double* grad,
                      double* hess, double thresh, void* stream, int* ier) {
  guarded(ier, [&] {
    return helm_direct_device(nd, zk_re, zk_im, ns, sources, charge, dipstr, dipvec, nt, targ,
                              ifpgh, pot, grad, hess, thresh, (cudaStream_t)stream);
  });
}

void* b2fmm_plan_create(int fe, int nd, double eps, int64_t ns, const double* sources,
                        int ifcharge, int ifdipole, int ifpgh, int64_t nt, const double* targ,
                        int ifpghtarg, const b2fmm_options* opts, void* stream, int* ier) {
  static const double present = 0.0;  // marks a density kind the evaluations will pass
  LapPlan* p = nullptr;
  guarded(ier, [&] {
    LapArgs a;
    a.fe = fe;
    a.nd = nd;
    a.eps = eps;
    a.ns = ns;
    a.src = sources;
    a.charge = ifcharge == 1 ? &present : nullptr;
    a.dipstr = ifdipole == 1 ? &present : nullptr;
    a.ifpgh = ifpgh;
    a.nt = nt;
    a.trg = targ;
    a.ifpghtarg = ifpghtarg;
    if (opts) {
      a.ndiv = opts->ndiv;
      a.lbal = opts->level_balance;
      a.idivflag = opts->idivflag;
      a.ifnear = opts->ifnear;
      a.precision = opts->precision;
    }
    return lap_plan_create(a, (cudaStream_t)stream, true, &p);
  });
  if (ier && *ier != IER_OK && p) {
    lap_plan_free(p);
    p = nullptr;
  }
  return p;
}

void b2fmm_plan_eval(void* plan, const double* charge, const double* dipstr, const double* dipvec,
                     double* pot, double* grad, double* hess, double* pottarg, double* gradtarg,
                     double* hesstarg, void* stream, int* ier) {
  guarded(ier, [&] {
    return lap_plan_eval((LapPlan*)plan, charge, dipstr, dipvec, pot, grad, hess, pottarg,
                         gradtarg, hesstarg, (cudaStream_t)stream, false, nullptr);
  });
}

int b2fmm_plan_status(void* plan) {
  int ier = 0;
  guarded(&ier, [&] { return lap_plan_status((LapPlan*)plan); });
  return ier;
}

void b2fmm_plan_free(void* plan) { lap_plan_free((LapPlan*)plan); }

void* b2fmm_batch_graph_create(int n, void* const* plans, const double* const* charge,
                               const double* const* dipstr, const double* const* dipvec,
                               double* const* pot, double* const* grad, double* const* hess,
                               double* const* pottarg, double* const* gradtarg,
                               double* const* hesstarg, int nbranch, int* ier) {
  BatchGraph* g = nullptr;
  guarded(ier, [&] {
    BatchIO io;
    io.charge = charge;
    io.dipstr = dipstr;
    io.dipvec = dipvec;
    io.pot = pot;
    io.grad = grad;
    io.hess = hess;
    io.pottarg = pottarg;
    io.gradtarg = gradtarg;
    io.hesstarg = hesstarg;
    return batch_graph_create(n, (LapPlan* const*)plans, io, nbranch, &g);
  });
  return g;
}

void b2fmm_batch_graph_launch(void* graph, void* stream, int* ier) {
  guarded(ier, [&] { return batch_graph_launch((BatchGraph*)graph, (cudaStream_t)stream); });
}

int b2fmm_batch_graph_status(void* graph) {
  int ier = 0;
  guarded(&ier, [&] { return batch_graph_status((BatchGraph*)graph); });
  return ier;
}

int64_t b2fmm_batch_graph_nodes(void* graph) {
  return (int64_t)batch_graph_nodes((const BatchGraph*)graph);
}

void b2fmm_batch_graph_free(void* graph) { batch_graph_free((BatchGraph*)graph); }

int b2fmm_h2dterms(double bsize, double zk_re, double zk_im, double eps, int* ier) {
  int e = 0, p = 0;
  guarded(ier, [&] {
    p = helm_nterms(bsize, zk_re, zk_im, eps, &e);
    return e;
  });
  return p;
}

void b2fmm_helm_special(int kind, int n, double z_re, double z_im, double rscale, double* out) {
  double2 z = make_double2(z_re, z_im);
  if (kind == 0) {
    double2 h0, h1;
    helm::hank01(z, h0, h1);
    out[0] = h0.x;
    out[1] = h0.y;
    out[2] = h1.x;
    out[3] = h1.y;
  } else if (kind == 1) {
    helm::jscaled(n, z, rscale, (double2*)out);
  } else {
    helm::hscaled(n, z, rscale, (double2*)out);
  }
}

void* b2fmm_tree_build(const double* sources_dev, int64_t ns, const double* targ_dev, int64_t nt,
                       int idivflag, int ndiv, int nlmax, int* nlevels, int* nboxes, int* ier) {
  TreeHandle* h = nullptr;
  guarded(ier, [&] {
    if (ns < 1 || nt < 0 || ndiv < 1 || nlmax < 0 || nlmax > NLMAX) return (int)IER_BADARG;
    int dev = 0;
    B2_CHECK(cudaGetDevice(&dev));
    configure_mempool(dev);
    h = new TreeHandle();
    build_device_tree(h->T, sources_dev, ns, targ_dev, nt, idivflag, ndiv, nlmax,
                      cudaStreamPerThread);
    // the lists are still being written on the stream; b2fmm_tree_get copies
    // synchronously
    B2_CHECK(cudaStreamSynchronize(cudaStreamPerThread));
    *nlevels = h->T.nlevels;
    *nboxes = h->T.nboxes;
    return (int)IER_OK;
  });
  if (ier && *ier != IER_OK) {
    delete h;
    return nullptr;
  }
  return h;
}

void b2fmm_tree_get(void* tree, int* laddr, int* ilevel, int* iparent, int* nchild, int* ichild,
                    int* ncoll, int* coll, double* centers, double* boxsize, int* isrc,
                    int* isrcse, int* itarg, int* itargse, int* nlist1, int* list1, int* nlist2,
                    int* list2, int* nlist3, int* list3, int* nlist4, int* list4, int* ier) {
  guarded(ier, [&] {
    TreeHandle* h = (TreeHandle*)tree;
    DeviceTree& T = h->T;
    cudaStream_t st = T.st;
    int nb = T.nboxes;
    for (int l = 0; l <= T.nlevels; l++) {
      laddr[2 * l] = T.lfirst[l];
      laddr[2 * l + 1] = T.llast[l];
      boxsize[l] = T.boxsize[l];
    }
    auto cp = [&](void* dst, const void* src, size_t bytes) {
      if (bytes) B2_CHECK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, st));
    };
    cp(ilevel, T.level.p, sizeof(int) * nb);
    cp(iparent, T.parent.p, sizeof(int) * nb);
    cp(nchild, T.nchild.p, sizeof(int) * nb);
    cp(ichild, T.child.p, sizeof(int) * 4 * nb);
    cp(ncoll, T.ncoll.p, sizeof(int) * nb);
    cp(coll, T.coll.p, sizeof(int) * 9 * nb);
    cp(centers, T.center.p, sizeof(double) * 2 * nb);
    cp(isrc, T.isrc.p, sizeof(int) * T.ns);
    cp(isrcse, T.srng.p, sizeof(int) * 2 * nb);
    cp(itarg, T.itarg.p, sizeof(int) * T.nt);
    cp(itargse, T.trng.p, sizeof(int) * 2 * nb);
    cp(nlist1, T.nlist1.p, sizeof(int) * nb);
    cp(list1, T.list1.p, sizeof(int) * MNLIST1 * nb);
    cp(nlist2, T.nlist2.p, sizeof(int) * nb);
    cp(list2, T.list2.p, sizeof(int) * MNLIST2 * nb);
    cp(nlist3, T.nlist3.p, sizeof(int) * nb);
    cp(list3, T.list3.p, sizeof(int) * MNLIST3 * nb);
    cp(nlist4, T.nlist4.p, sizeof(int) * nb);
    cp(list4, T.list4.p, sizeof(int) * MNLIST4 * nb);
    B2_CHECK(cudaStreamSynchronize(st));
    return (int)IER_OK;
  });
}

void b2fmm_tree_free(void* tree) { delete (TreeHandle*)tree; }

uint64_t b2fmm_kernel_launches(void) { return g_launches.load(); }

void b2fmm_set_stats(int on) { set_stats(on != 0); }

void b2fmm_set_device_ranges(int on) { set_device_ranges(on != 0); }

void b2fmm_test_fail_alloc(int after) { b2::g_fail_after.store(after < 0 ? -1 : after); }

void b2fmm_test_barrier_limit(long long cycles) { set_tree_barrier_limit(cycles); }

void b2fmm_async_status(void* stream, int* ier) {
  guarded(ier, [&] { return lap_async_status((cudaStream_t)stream); });
}

void b2fmm_get_stats(double* out, int n) {
  const LapStats& S = last_stats();
  const double v[18] = {S.nboxes,    S.nlevels,     S.nleaves,   S.nterms1,
                        S.p2p_pairs, S.m2l_pairs,   S.m2p_evals, S.p2l_sources,
                        S.npts_eval, S.tree_ms,     S.fmm_ms,    S.nd_cauchy,
                        S.m2l_tc_steps, S.tl_pre,   S.tl_tree,   S.tl_setup,
                        S.tl_fmm,    S.tl_post};
  for (int i = 0; i < n && i < 18; i++) out[i] = v[i];
}

double b2fmm_fma_peak(int fp64) { return fma_peak_flops(fp64 != 0); }

int b2fmm_mlp_param_count(int nin, int h1, int h2) { return mlp_param_count(nin, h1, h2); }

void b2fmm_mlp_forward(const float* x, int batch, int nin, int h1, int h2, const float* params,
                       float* y, void* stream, int* ier) {
  guarded(ier, [&] { return mlp_forward(x, batch, nin, h1, h2, params, y, (cudaStream_t)stream); });
}

void b2fmm_mlp_gradient(const float* x, const float* target, int batch, int nin, int h1, int h2,
                        const float* params, float* grad, float* loss, void* stream, int* ier) {
  guarded(ier, [&] {
    int r = mlp_gradient(x, target, batch, nin, h1, h2, params, grad, loss, (cudaStream_t)stream);
    if (r == IER_OK) B2_CHECK(cudaStreamSynchronize((cudaStream_t)stream));
    return r;
  });
}

void b2fmm_mlp_train(const float* x, const float* target, int batch, int nin, int h1, int h2,
                     float* params, int steps, float lr, float* loss_history, void* stream,
                     int* ier) {
  guarded(ier, [&] {
    return mlp_train(x, target, batch, nin, h1, h2, params, steps, lr, loss_history,
                     (cudaStream_t)stream);
  });
}

void b2fmm_point_stats(const double* sources, int64_t ns, const double* targ, int64_t nt,
                       unsigned* hist, void* stream, int* ier) {
  guarded(ier, [&] { return point_stats(sources, ns, targ, nt, hist, (cudaStream_t)stream); });
}

void b2fmm_set_m2l_tensor_cores(int on) { set_m2l_tensor_cores(on != 0); }

int b2fmm_set_p2p_shape(int leaf_class, int shape) { return set_p2p_shape(leaf_class, shape); }

int b2fmm_get_p2p_shape(int leaf_class) { return p2p_shape(leaf_class); }

void b2fmm_tc_gemm_probe(const float* a_dev, const float* b_dev, int k, int n, float* d_dev,
                         void* stream, int* ier) {
  guarded(ier, [&] { return tc_gemm_probe(a_dev, b_dev, k, n, d_dev, (cudaStream_t)stream); });
}

}  // extern "C"
