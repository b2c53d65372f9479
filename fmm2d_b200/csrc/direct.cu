// Direct (all-pairs) sums on the device: the c2ddir / l2ddir / r2ddir
// evaluators of the python API (python/fmm2dpy/fmm2d.py:1370-1740) over the
// kernels of src/laplace/cauchykernels2d.f, lapkernels2d.f and
// rlapkernels2d.f.  Each block takes 128 targets and one slice of the
// sources (staged through shared memory); slices write partial sums that a
// second kernel adds in slice order, so the result is deterministic.
#include "direct.cuh"

#include <mutex>

namespace b2 {

namespace {

constexpr int DT = 128;  // targets per block

// Per-pair contributions for one density.
// kind 0 (Cauchy): outputs pot, d/dz, d2/dz2 as complex (3 slots).
// kind 1/2 (Laplace form): pot, (d/dx, d/dy), (xx, xy, yy) (6 slots).
template <int KIND>
__device__ __forceinline__ void pair_terms(double dx, double dy, double rr, double2 q, double2 dp,
                                           const double* v, bool hq, bool hd, int ifpgh,
                                           double2* o) {
  if (KIND == 0) {
    double ir = 1.0 / rr;
    double2 zi = make_double2(dx * ir, -dy * ir);
    double lg = 0.5 * log(rr);
    double2 z2 = make_double2(-(zi.x * zi.x - zi.y * zi.y), -(2 * zi.x * zi.y));
    if (hq) {
      o[0].x += lg * q.x;
      o[0].y += lg * q.y;
      if (ifpgh >= 2) cfma(o[1], zi, q);
      if (ifpgh >= 3) cfma(o[2], z2, q);
    }
    if (hd) {
      cfma(o[0], zi, dp);
      if (ifpgh >= 2) cfma(o[1], z2, dp);
      if (ifpgh >= 3) cfma(o[2], cscale(cmul(z2, zi), -2.0), dp);
    }
  } else {
    double lg = 0.5 * log(rr);
    double r2 = rr * rr, r3 = r2 * rr;
    double gx = dx / rr, gy = dy / rr;
    double hxx = (rr - 2 * dx * dx) / r2, hxy = -2 * dx * dy / r2, hyy = (rr - 2 * dy * dy) / r2;
    if (hq) {
      o[0].x += lg * q.x;
      o[0].y += lg * q.y;
      if (ifpgh >= 2) {
        o[1].x += gx * q.x; o[1].y += gx * q.y;
        o[2].x += gy * q.x; o[2].y += gy * q.y;
      }
      if (ifpgh >= 3) {
        o[3].x += hxx * q.x; o[3].y += hxx * q.y;
        o[4].x += hxy * q.x; o[4].y += hxy * q.y;
        o[5].x += hyy * q.x; o[5].y += hyy * q.y;
      }
    }
    if (hd) {
      // dipole potential -v.grad_x log r (lapkernels2d.f:640-648)
      double2 d1 = cscale(dp, v[0]), d2 = cscale(dp, v[1]);
      o[0].x -= d1.x * gx + d2.x * gy;
      o[0].y -= d1.y * gx + d2.y * gy;
      if (ifpgh >= 2) {
        o[1].x -= d1.x * hxx + d2.x * hxy; o[1].y -= d1.y * hxx + d2.y * hxy;
        o[2].x -= d1.x * hxy + d2.x * hyy; o[2].y -= d1.y * hxy + d2.y * hyy;
      }
      if (ifpgh >= 3) {
        double txxx = (-6 * dx * rr + 8 * dx * dx * dx) / r3;
        double txxy = (-2 * dy * rr + 8 * dx * dx * dy) / r3;
        double txyy = (-2 * dx * rr + 8 * dx * dy * dy) / r3;
        double tyyy = (-6 * dy * rr + 8 * dy * dy * dy) / r3;
        o[3].x -= d1.x * txxx + d2.x * txxy; o[3].y -= d1.y * txxx + d2.y * txxy;
        o[4].x -= d1.x * txxy + d2.x * txyy; o[4].y -= d1.y * txxy + d2.y * txyy;
        o[5].x -= d1.x * txyy + d2.x * tyyy; o[5].y -= d1.y * txyy + d2.y * tyyy;
      }
    }
  }
}

// One density per launch slice d; partial[slice][target][slot].
template <int KIND>
__global__ void __launch_bounds__(DT) k_direct(int nd, int d, long ns, const double* __restrict__ src,
                                              const double* __restrict__ charge,
                                              const double* __restrict__ dipstr,
                                              const double* __restrict__ dipvec, long nt,
                                              const double* __restrict__ trg, int ifpgh,
                                              double th2, int lt, long chunk,
                                              double2* __restrict__ partial) {
  constexpr int NS = KIND == 0 ? 3 : 6;
  __shared__ double sx[DT], sy[DT], sv0[DT], sv1[DT];
  __shared__ double2 sq[DT], sd[DT];
  long t = blockIdx.x * (long)DT + threadIdx.x;
  bool act = t < nt;
  double x = act ? trg[2 * t] : 0, y = act ? trg[2 * t + 1] : 0;
  double2 o[NS];
  for (int k = 0; k < NS; k++) o[k] = make_double2(0, 0);
  long s0 = blockIdx.y * chunk, s1 = min(ns, s0 + chunk);
  bool hq = charge != nullptr, hd = dipstr != nullptr;
  for (long b0 = s0; b0 < s1; b0 += DT) {
    __syncthreads();
    long j = b0 + threadIdx.x;
    if (j < s1) {
      sx[threadIdx.x] = src[2 * j];
      sy[threadIdx.x] = src[2 * j + 1];
      if (KIND == 2) {
        if (hq) sq[threadIdx.x] = make_double2(charge[j * nd + d], 0);
        if (hd) sd[threadIdx.x] = make_double2(dipstr[j * nd + d], 0);
      } else {
        if (hq) sq[threadIdx.x] = ((const double2*)charge)[j * nd + d];
        if (hd) sd[threadIdx.x] = ((const double2*)dipstr)[j * nd + d];
      }
      if (KIND != 0 && hd) {
        sv0[threadIdx.x] = dipvec[(j * 2 + 0) * nd + d];
        sv1[threadIdx.x] = dipvec[(j * 2 + 1) * nd + d];
      }
    }
    __syncthreads();
    int m = (int)min((long)DT, s1 - b0);
    if (act) {
      for (int i = 0; i < m; i++) {
        double dx = x - sx[i], dy = y - sy[i];
        double rr = dx * dx + dy * dy;
        if (lt ? (rr < th2) : (rr <= th2)) continue;
        double v[2] = {KIND != 0 && hd ? sv0[i] : 0.0, KIND != 0 && hd ? sv1[i] : 0.0};
        pair_terms<KIND>(dx, dy, rr, hq ? sq[i] : make_double2(0, 0),
                         hd ? sd[i] : make_double2(0, 0), v, hq, hd, ifpgh, o);
      }
    }
  }
  if (act)
    for (int k = 0; k < NS; k++) partial[((size_t)blockIdx.y * nt + t) * NS + k] = o[k];
}

template <int KIND>
__global__ void k_direct_reduce(int nd, int d, long nt, int nslice, int ifpgh,
                                const double2* __restrict__ partial, double* pot, double* grad,
                                double* hess) {
  constexpr int NS = KIND == 0 ? 3 : 6;
  long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= nt) return;
  double2 o[NS];
  for (int k = 0; k < NS; k++) o[k] = make_double2(0, 0);
  for (int s = 0; s < nslice; s++)
    for (int k = 0; k < NS; k++) o[k] = cadd(o[k], partial[((size_t)s * nt + t) * NS + k]);
  if (KIND == 0) {
    ((double2*)pot)[t * nd + d] = o[0];
    if (ifpgh >= 2) ((double2*)grad)[t * nd + d] = o[1];
    if (ifpgh >= 3) ((double2*)hess)[t * nd + d] = o[2];
  } else if (KIND == 1) {
    ((double2*)pot)[t * nd + d] = o[0];
    if (ifpgh >= 2) {
      ((double2*)grad)[(t * 2 + 0) * nd + d] = o[1];
      ((double2*)grad)[(t * 2 + 1) * nd + d] = o[2];
    }
    if (ifpgh >= 3)
      for (int k = 0; k < 3; k++) ((double2*)hess)[(t * 3 + k) * nd + d] = o[3 + k];
  } else {
    pot[t * nd + d] = o[0].x;
    if (ifpgh >= 2) {
      grad[(t * 2 + 0) * nd + d] = o[1].x;
      grad[(t * 2 + 1) * nd + d] = o[2].x;
    }
    if (ifpgh >= 3)
      for (int k = 0; k < 3; k++) hess[(t * 3 + k) * nd + d] = o[3 + k].x;
  }
}

template <int KIND>
void run_direct(int nd, long ns, const double* src, const double* charge, const double* dipstr,
                const double* dipvec, long nt, const double* trg, int ifpgh, double* pot,
                double* grad, double* hess, double thresh, cudaStream_t st) {
  constexpr int NS = KIND == 0 ? 3 : 6;
  int tb = ceil_div(nt, DT);
  int nslice = std::max(1, std::min(1024, (148 * 16) / std::max(tb, 1)));
  long chunk = (ns + nslice - 1) / nslice;
  chunk = ((chunk + DT - 1) / DT) * DT;
  nslice = (int)std::max(1L, (ns + chunk - 1) / chunk);
  // strict comparison for the charge kernels with derivatives
  // (cauchykernels2d.f / lapkernels2d.f thresholds)
  int lt = (ifpgh >= 2 && (KIND != 0 ? charge != nullptr : true)) ? 1 : 0;
  DBuf<double2> part(st);
  part.alloc((size_t)nslice * nt * NS, st);
  for (int d = 0; d < nd; d++) {
    dim3 grid(tb, nslice);
    k_direct<KIND><<<grid, DT, 0, st>>>(nd, d, ns, src, charge, dipstr, dipvec, nt, trg, ifpgh,
                                        thresh * thresh, lt, chunk, part.p);
    B2_LAUNCH_CHECK();
    k_direct_reduce<KIND><<<ceil_div(nt, 256), 256, 0, st>>>(nd, d, nt, nslice, ifpgh, part.p,
                                                             pot, grad, hess);
    B2_LAUNCH_CHECK();
  }
  B2_CHECK(cudaStreamSynchronize(st));
}

}  // namespace

int lap_direct_device(int kind, int nd, long ns, const double* src, const double* charge,
                      const double* dipstr, const double* dipvec, long nt, const double* trg,
                      int ifpgh, double* pot, double* grad, double* hess, double thresh,
                      cudaStream_t st) {
  if (nd < 1 || ns < 0 || nt < 0 || ifpgh < 1 || ifpgh > 3 || kind < 0 || kind > 2)
    return IER_BADARG;
  if (nt == 0) return IER_OK;
  if (ns == 0 || (!charge && !dipstr)) {
    int cw = kind == 2 ? 1 : 2, gw = kind == 0 ? 1 : 2, hw = kind == 0 ? 1 : 3;
    B2_CHECK(cudaMemsetAsync(pot, 0, sizeof(double) * cw * nd * nt, st));
    if (ifpgh >= 2) B2_CHECK(cudaMemsetAsync(grad, 0, sizeof(double) * cw * gw * nd * nt, st));
    if (ifpgh >= 3) B2_CHECK(cudaMemsetAsync(hess, 0, sizeof(double) * cw * hw * nd * nt, st));
    B2_CHECK(cudaStreamSynchronize(st));
    return IER_OK;
  }
  if (kind != 0 && dipstr && !dipvec) return IER_BADARG;
  if (kind == 0)
    run_direct<0>(nd, ns, src, charge, dipstr, dipvec, nt, trg, ifpgh, pot, grad, hess, thresh, st);
  else if (kind == 1)
    run_direct<1>(nd, ns, src, charge, dipstr, dipvec, nt, trg, ifpgh, pot, grad, hess, thresh, st);
  else
    run_direct<2>(nd, ns, src, charge, dipstr, dipvec, nt, trg, ifpgh, pot, grad, hess, thresh, st);
  return IER_OK;
}

}  // namespace b2

namespace b2 {

// ---------------------------------------------------------------------------
// Allocation-free variant of the direct sum.
//
// Some callers cannot allocate device memory while they call us: code that
// runs inside another framework's memory budget (the whole device already
// reserved by its allocator), latency-critical loops that must not hit a
// synchronising or failing cudaMalloc, or embedded pipelines with a fixed
// memory plan.  lap_direct_device_noalloc() therefore takes its per-slice
// partial sums from the file-scope array below instead of the stream-ordered
// pool.  The array is NOALLOC_SCRATCH_ELEMS complex doubles (4 MiB) and every
// GPU that loads this library keeps it until the process exits.
//
// In host code `g_direct_scratch` only names a host-side stand-in, not the
// device address, so the first call on each device looks the address up with
// cudaGetSymbolAddress (with that device current) and caches it; make that
// first call before the device's memory is handed to another allocator: with
// CUDA's lazy module loading it may be the
// look-up that loads this module and reserves the array (or set
// CUDA_MODULE_LOADING=EAGER).  All calls share the one array and it
// keeps the last call's contents: the first kernel writes every element the
// second one reads, so nothing needs clearing, but calls that overlap on the
// GPU (other streams, other host threads) race on it and must be serialised
// by the caller.
// ---------------------------------------------------------------------------
namespace {

constexpr size_t NOALLOC_SCRATCH_ELEMS = (size_t)1 << 18;  // 4 MiB of double2
static __device__ __align__(256) double2 g_direct_scratch[NOALLOC_SCRATCH_ELEMS];

std::mutex g_scratch_mu;
double2* g_scratch_addr[128] = {nullptr};

double2* scratch_address() {
  int dev = 0;
  B2_CHECK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 128) throw CudaError("device ordinal beyond 127", IER_BADARG);
  std::lock_guard<std::mutex> g(g_scratch_mu);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    // with lazy module loading this first look-up may be what loads the
    // module and reserves the array: out of memory then is IER_ALLOC
    cudaError_t e = cudaGetSymbolAddress(&p, g_direct_scratch);
    if (e != cudaSuccess || !p)
      throw CudaError(std::string("cudaGetSymbolAddress(g_direct_scratch): ") +
                          cudaGetErrorString(e),
                      e == cudaErrorMemoryAllocation ? IER_ALLOC : IER_CUDA);
    g_scratch_addr[dev] = (double2*)p;
  }
  return g_scratch_addr[dev];
}

template <int KIND>
int run_direct_noalloc(int nd, long ns, const double* src, const double* charge,
                       const double* dipstr, const double* dipvec, long nt, const double* trg,
                       int ifpgh, double* pot, double* grad, double* hess, double thresh,
                       cudaStream_t st) {
  constexpr int NS = KIND == 0 ? 3 : 6;
  if ((size_t)nt * NS > NOALLOC_SCRATCH_ELEMS) {
    fprintf(stderr,
            "fmm2d_b200: b2fmm_lap_direct_noalloc_dev: %ld targets need %zu scratch elements, "
            "the static scratch holds %zu (at most %zu targets for this kernel)\n",
            nt, (size_t)nt * NS, NOALLOC_SCRATCH_ELEMS, NOALLOC_SCRATCH_ELEMS / NS);
    return IER_NOALLOC_TOO_LARGE;
  }
  double2* part = scratch_address();
  int tb = ceil_div(nt, DT);
  long fit = (long)(NOALLOC_SCRATCH_ELEMS / ((size_t)nt * NS));
  int nslice = std::max(1, std::min(1024, (148 * 16) / std::max(tb, 1)));
  nslice = (int)std::min<long>(nslice, fit);
  long chunk = (ns + nslice - 1) / nslice;
  chunk = ((chunk + DT - 1) / DT) * DT;
  nslice = (int)std::max(1L, (ns + chunk - 1) / chunk);
  int lt = (ifpgh >= 2 && (KIND != 0 ? charge != nullptr : true)) ? 1 : 0;
  for (int d = 0; d < nd; d++) {
    dim3 grid(tb, nslice);
    k_direct<KIND><<<grid, DT, 0, st>>>(nd, d, ns, src, charge, dipstr, dipvec, nt, trg, ifpgh,
                                        thresh * thresh, lt, chunk, part);
    B2_LAUNCH_CHECK();
    k_direct_reduce<KIND><<<ceil_div(nt, 256), 256, 0, st>>>(nd, d, nt, nslice, ifpgh, part, pot,
                                                             grad, hess);
    B2_LAUNCH_CHECK();
  }
  B2_CHECK(cudaStreamSynchronize(st));
  return IER_OK;
}

}  // namespace

int lap_direct_device_noalloc(int kind, int nd, long ns, const double* src, const double* charge,
                              const double* dipstr, const double* dipvec, long nt,
                              const double* trg, int ifpgh, double* pot, double* grad,
                              double* hess, double thresh, cudaStream_t st) {
  if (nd < 1 || ns < 0 || nt < 0 || ifpgh < 1 || ifpgh > 3 || kind < 0 || kind > 2)
    return IER_BADARG;
  if (nt == 0) return IER_OK;
  if (ns == 0 || (!charge && !dipstr)) {
    int cw = kind == 2 ? 1 : 2, gw = kind == 0 ? 1 : 2, hw = kind == 0 ? 1 : 3;
    B2_CHECK(cudaMemsetAsync(pot, 0, sizeof(double) * cw * nd * nt, st));
    if (ifpgh >= 2) B2_CHECK(cudaMemsetAsync(grad, 0, sizeof(double) * cw * gw * nd * nt, st));
    if (ifpgh >= 3) B2_CHECK(cudaMemsetAsync(hess, 0, sizeof(double) * cw * hw * nd * nt, st));
    B2_CHECK(cudaStreamSynchronize(st));
    return IER_OK;
  }
  if (kind != 0 && dipstr && !dipvec) return IER_BADARG;
  if (kind == 0)
    return run_direct_noalloc<0>(nd, ns, src, charge, dipstr, dipvec, nt, trg, ifpgh, pot, grad,
                                 hess, thresh, st);
  if (kind == 1)
    return run_direct_noalloc<1>(nd, ns, src, charge, dipstr, dipvec, nt, trg, ifpgh, pot, grad,
                                 hess, thresh, st);
  return run_direct_noalloc<2>(nd, ns, src, charge, dipstr, dipvec, nt, trg, ifpgh, pot, grad,
                               hess, thresh, st);
}

}  // namespace b2
