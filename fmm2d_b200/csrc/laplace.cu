// Cauchy/Laplace FMM on B200 (FP64 path).
//
// Follows the step order of cfmm2dmain (src/laplace/cfmm2d.f:442-1341) with
// the operators of src/laplace/laprouts2d.f and the near field of
// src/laplace/cauchykernels2d.f.  Layout in HBM: points and densities are
// gathered once into tree order (sources/targets sorted into leaves), and the
// multipole / local expansions live in two arrays of nboxes x P x ND complex
// doubles (P = nterms + 1 coefficients, ND densities of the current chunk),
// so the coefficients of one box are contiguous.
//
// Kernels (one warp per box unless noted):
//   k_p2m        P2M at leaves (step 1; k_p2m_f32 on the mixed path)
//   k_m2m        upward pass, one launch per level (step 3; a block per
//                chunk of boxes, the quadrant-symmetric operators)
//   k_p2l        list 4 -> local (step 2; k_p2l_f32 on the mixed path)
//   k_m2l        list 2 multipole -> local (step 4)
//   k_l2l        downward pass, one launch per level (step 5; as k_m2m)
//   leaf passes  (steps 6-8, csrc/lap_mixed.cu) on per-tree work items:
//                L2P + M2P one point per thread (k_far_mixed), then the
//                near field one warp per item of up to 32 points of a leaf
//                (k_p2p_leaf64; FP32 k_p2p_leaf on the mixed path)
//   k_unpack     caller layout (cfmm / lfmm / rfmm) and inverse permutation
#include "laplace.cuh"

#include <memory>
#include "lap_common.cuh"
#include "lap_mixed.cuh"

#include <cmath>
#include <mutex>


namespace b2 {

namespace {
std::atomic<bool> g_stats_on{false};
std::atomic<bool> g_device_ranges{true};
thread_local LapStats g_last_stats;
}  // namespace

// src/laplace/lndiv2d.f:1-39
int lap_ndiv(double eps) {
  if (eps >= 0.5e0) return 3;
  if (eps >= 0.5e-1) return 5;
  if (eps >= 0.5e-2) return 8;
  if (eps >= 0.5e-3) return 10;
  if (eps >= 0.5e-6) return 15;
  if (eps >= 0.5e-9) return 20;
  if (eps >= 0.5e-12) return 25;
  if (eps >= 0.5e-15) return 45;
  return -1;  // reference: ns + nt (no refinement)
}

// src/laplace/l2dterms.f:38-82: smallest j >= 2 with
// (sqrt2/2)^j / 1.5^(j+1) < eps (worst-case M2L decay), else 1.
int lap_nterms(double eps) {
  const double z2 = std::sqrt(2.0) / 2.0;
  double h = 1.0, jp = 1.0;
  for (int j = 0; j <= 100; j++) {
    h *= 1.5;
    if (j >= 2 && std::fabs(jp * (1.0 / h)) < eps) return j;
    jp *= z2;
  }
  return 1;
}

void set_stats(bool on) { g_stats_on = on; }
const LapStats& last_stats() { return g_last_stats; }

namespace {
struct DeviceTables {
  double* binom = nullptr;
  double2* shift = nullptr;
};

// The binomials and the M2M / L2L tables of the child (+,+) (the formulas at
// m2m_level), once per device.
const DeviceTables& device_tables() {
  static std::mutex mu;
  static DeviceTables tab[128];
  int dev = 0;
  B2_CHECK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 128) throw CudaError("device ordinal beyond 127", IER_CUDA);
  std::lock_guard<std::mutex> g(mu);
  if (!tab[dev].binom) {
    // Pascal recursion as in init_carray (src/common/fmmcommon2d.f:150-165)
    std::vector<double> c((size_t)BINOM_N * BINOM_N, 0.0);
    for (int l = 0; l < BINOM_N; l++) c[(size_t)l * BINOM_N] = 1.0;
    for (int m = 1; m < BINOM_N; m++) {
      c[(size_t)m * BINOM_N + m] = 1.0;
      for (int l = m + 1; l < BINOM_N; l++)
        c[(size_t)l * BINOM_N + m] = c[(size_t)(l - 1) * BINOM_N + m] + c[(size_t)(l - 1) * BINOM_N + m - 1];
    }
    // (1 + i)^k, Gaussian integers (exact below k = 106)
    std::vector<double2> pw(BINOM_N);
    pw[0] = make_double2(1.0, 0.0);
    for (int k = 1; k < BINOM_N; k++)
      pw[k] = make_double2(pw[k - 1].x - pw[k - 1].y, pw[k - 1].x + pw[k - 1].y);
    std::vector<double2> sh(2 * (size_t)SHIFT_TAB);
    double2* m2m = sh.data();
    double2* l2l = m2m + SHIFT_TAB;
    for (int a = 0; a < BINOM_N; a++)
      for (int b = 0; b <= a; b++) {
        const size_t o = (size_t)a * (a + 1) / 2 + b;
        // M2M B[i = a][j = b]
        double f;
        if (a == 0) f = 1.0;
        else if (b == 0) f = -std::ldexp(1.0, -2 * a) / a;
        else f = c[(size_t)(a - 1) * BINOM_N + (b - 1)] * std::ldexp(1.0, b - 2 * a);
        m2m[o] = make_double2(pw[a - b].x * f, pw[a - b].y * f);
        // L2L E[j = a][i = b]
        const double e = c[(size_t)a * BINOM_N + b] * std::ldexp(1.0, b - 2 * a);
        l2l[o] = make_double2(pw[a - b].x * e, pw[a - b].y * e);
      }
    double* d = nullptr;
    double2* d2 = nullptr;
    B2_CHECK(cudaMalloc(&d, c.size() * sizeof(double)));
    B2_CHECK(cudaMemcpy(d, c.data(), c.size() * sizeof(double), cudaMemcpyHostToDevice));
    B2_CHECK(cudaMalloc(&d2, sh.size() * sizeof(double2)));
    B2_CHECK(cudaMemcpy(d2, sh.data(), sh.size() * sizeof(double2), cudaMemcpyHostToDevice));
    tab[dev].shift = d2;
    tab[dev].binom = d;
  }
  return tab[dev];
}
}  // namespace

const double* device_binomials() { return device_tables().binom; }
const double2* device_shift_tables() { return device_tables().shift; }

void configure_mempool(int device) {
  static std::mutex mu;
  static bool done[128] = {false};
  std::lock_guard<std::mutex> g(mu);
  if (done[device]) return;
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
    uint64_t thr = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
  }
  done[device] = true;
}

// One long-lived non-blocking stream per device for the plans' own work
// (construction, status reads, release).  A stream per plan, kept for the
// plan's lifetime, made each new plan slower with the number of live plans
// (1 ms for the first, ~25 ms after 256 in the stream-ordered allocator).
cudaStream_t plan_stream(int device) {
  static std::mutex mu;
  static cudaStream_t streams[128] = {};
  std::lock_guard<std::mutex> g(mu);
  if (!streams[device]) B2_CHECK(cudaStreamCreateWithFlags(&streams[device], cudaStreamNonBlocking));
  return streams[device];
}

namespace {

using namespace lapk;

// ---------------------------------------------------------------------------
// Shared-memory staging used by P2M and P2L: a chunk of sources at a time,
// one per lane, each lane writing the power table w^0..w^(P-1) of its source
// and its (pre-scaled) densities; then the lanes switch to one coefficient
// each and accumulate over the staged sources.  P2M takes 16 sources (a leaf
// holds at most 15 at eps >= 1e-6) in half the shared memory of 32, and asks
// for at most 64 registers a thread with one or two densities: more warps per
// SM (P2M 0.77 -> 0.67 ms at 4M points).  P2L takes 32 (its sources come
// from up to five leaves).
// ---------------------------------------------------------------------------
constexpr int P2M_CHUNK = 16;
#define P2M_MIN_BLOCKS(ND) ((ND) <= 2 ? 16 : ((ND) == 4 ? 12 : 6))
// step 1: P2M (laprouts2d.f:84-282) at leaves of level >= 2; every other leaf
// gets a zero expansion so that list 2 / list 3 reads are well defined.
// m_0 += q,  m_n += -q w^n / n + (d/r) w^(n-1),  w = (x - c) / r
// A warp takes 32 of its boxes at a time (stride = the grid's warps): each
// lane loads one box's child count, level, sources and centre, ballots mark
// the leaves, and the warp then works through them with the box data
// shuffled from the lane that loaded it (one round of loads per 32 boxes
// instead of a chain of rounds per box).
template <int ND>
__global__ void __launch_bounds__(64, P2M_MIN_BLOCKS(ND)) k_p2m(TV t, int first, int n, const double2* __restrict__ xs,
                                            Dens D, int P, double2* __restrict__ mp) {
  extern __shared__ double2 smem[];
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  resolve_range(t, first, n);
  double2* W = smem + (size_t)wib * (P2M_CHUNK * P + 2 * P2M_CHUNK * ND);
  double2* Q = W + P2M_CHUNK * P;
  double2* Dd = Q + P2M_CHUNK * ND;
  for (int base = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; base < n; base += 32 * nw) {
    const int mine = base + lane * nw;
    int nc = 1, lev = 0;
    int2 sr = make_int2(0, 0);
    double2 cen = make_double2(0, 0);
    if (mine < n) {
      const int b = first + mine;
      nc = t.nchild[b];
      lev = t.level[b];
      sr = t.srng[b];
      cen = t.center[b];
    }
    const bool work = nc == 0 && lev >= 2 && sr.y > sr.x;
    unsigned zm = __ballot_sync(~0u, mine < n && nc == 0 && !work);
    unsigned wm = __ballot_sync(~0u, mine < n && work);
    while (zm) {
      const int src = __ffs(zm) - 1;
      zm &= zm - 1;
      const size_t b = (size_t)first + base + src * nw;
      for (int e = lane; e < P * ND; e += 32) mp[b * P * ND + e] = make_double2(0, 0);
    }
    while (wm) {
      const int src = __ffs(wm) - 1;
      wm &= wm - 1;
      const int b = first + base + src * nw;
      const int2 srb = make_int2(__shfl_sync(~0u, sr.x, src), __shfl_sync(~0u, sr.y, src));
      const double2 c = make_double2(__shfl_sync(~0u, cen.x, src), __shfl_sync(~0u, cen.y, src));
      const double r = t.boxsize[__shfl_sync(~0u, lev, src)];
      const double ri = 1.0 / r;
      double2 acc[2][ND];
#pragma unroll
      for (int s = 0; s < 2; s++)
#pragma unroll
        for (int d = 0; d < ND; d++) acc[s][d] = make_double2(0, 0);
      for (int s0 = srb.x; s0 < srb.y; s0 += P2M_CHUNK) {
        const int m = min(P2M_CHUNK, srb.y - s0);
        __syncwarp();
        if (lane < m) {
          const int j = s0 + lane;
          const double2 x = xs[j];
          const double2 w = make_double2((x.x - c.x) / r, (x.y - c.y) / r);
          double2 pw = make_double2(1.0, 0.0);
          for (int k = 0; k < P; k++) {
            W[lane * P + k] = pw;
            pw = cmul(pw, w);
          }
#pragma unroll
          for (int d = 0; d < ND; d++) {
            Q[lane * ND + d] = D.q ? D.q[(size_t)j * D.ndc + D.d0 + d] : make_double2(0, 0);
            Dd[lane * ND + d] =
                D.d ? cscale(D.d[(size_t)j * D.ndc + D.d0 + d], ri) : make_double2(0, 0);
          }
        }
        __syncwarp();
#pragma unroll
        for (int s = 0; s < 2; s++) {
          const int k = lane + 32 * s;
          if (k >= P) break;
          if (k == 0) {
            for (int j = 0; j < m; j++)
#pragma unroll
              for (int d = 0; d < ND; d++) acc[s][d] = cadd(acc[s][d], Q[j * ND + d]);
          } else {
            const double mik = -1.0 / k;
            for (int j = 0; j < m; j++) {
              const double2 wk = W[j * P + k], wk1 = W[j * P + k - 1];
              const double2 cq = cscale(wk, mik);
#pragma unroll
              for (int d = 0; d < ND; d++) {
                cfma(acc[s][d], Q[j * ND + d], cq);
                cfma(acc[s][d], Dd[j * ND + d], wk1);
              }
            }
          }
        }
      }
#pragma unroll
      for (int s = 0; s < 2; s++) {
        const int k = lane + 32 * s;
        if (k >= P) break;
#pragma unroll
        for (int d = 0; d < ND; d++) mp[((size_t)b * P + k) * ND + d] = acc[s][d];
      }
    }
  }
}

// The mixed path's P2M: the same staging and lane mapping with the
// per-source terms and the sums over a chunk of sources in FP32, each
// chunk's partial sums added to FP64 accumulators; w = (x - c) / r is formed
// in FP64 and rounded once.
template <int ND>
__global__ void __launch_bounds__(64, P2M_MIN_BLOCKS(ND)) k_p2m_f32(TV t, int first, int n, const double2* __restrict__ xs,
                                            Dens D, int P, double2* __restrict__ mp) {
  extern __shared__ float2 fsm1[];
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  resolve_range(t, first, n);
  float2* W = fsm1 + (size_t)wib * (P2M_CHUNK * P + 2 * P2M_CHUNK * ND);
  float2* Q = W + P2M_CHUNK * P;
  float2* Dd = Q + P2M_CHUNK * ND;
  for (int base = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; base < n; base += 32 * nw) {
    const int mine = base + lane * nw;
    int nc = 1, lev = 0;
    int2 sr = make_int2(0, 0);
    double2 cen = make_double2(0, 0);
    if (mine < n) {
      const int b = first + mine;
      nc = t.nchild[b];
      lev = t.level[b];
      sr = t.srng[b];
      cen = t.center[b];
    }
    const bool work = nc == 0 && lev >= 2 && sr.y > sr.x;
    unsigned zm = __ballot_sync(~0u, mine < n && nc == 0 && !work);
    unsigned wm = __ballot_sync(~0u, mine < n && work);
    while (zm) {
      const int src = __ffs(zm) - 1;
      zm &= zm - 1;
      const size_t b = (size_t)first + base + src * nw;
      for (int e = lane; e < P * ND; e += 32) mp[b * P * ND + e] = make_double2(0, 0);
    }
    while (wm) {
      const int src = __ffs(wm) - 1;
      wm &= wm - 1;
      const int b = first + base + src * nw;
      const int2 srb = make_int2(__shfl_sync(~0u, sr.x, src), __shfl_sync(~0u, sr.y, src));
      const double2 c = make_double2(__shfl_sync(~0u, cen.x, src), __shfl_sync(~0u, cen.y, src));
      const double r = t.boxsize[__shfl_sync(~0u, lev, src)];
      const double ri = 1.0 / r;
      double2 acc[2][ND];
#pragma unroll
      for (int s = 0; s < 2; s++)
#pragma unroll
        for (int d = 0; d < ND; d++) acc[s][d] = make_double2(0, 0);
      for (int s0 = srb.x; s0 < srb.y; s0 += P2M_CHUNK) {
        const int m = min(P2M_CHUNK, srb.y - s0);
        __syncwarp();
        if (lane < m) {
          const int j = s0 + lane;
          const double2 x = xs[j];
          const float2 w = make_float2((float)((x.x - c.x) * ri), (float)((x.y - c.y) * ri));
          float2 pw = make_float2(1.0f, 0.0f);
          for (int k = 0; k < P; k++) {
            W[lane * P + k] = pw;
            pw = cmulf(pw, w);
          }
#pragma unroll
          for (int d = 0; d < ND; d++) {
            const double2 q = D.q ? D.q[(size_t)j * D.ndc + D.d0 + d] : make_double2(0, 0);
            const double2 dv =
                D.d ? cscale(D.d[(size_t)j * D.ndc + D.d0 + d], ri) : make_double2(0, 0);
            Q[lane * ND + d] = make_float2((float)q.x, (float)q.y);
            Dd[lane * ND + d] = make_float2((float)dv.x, (float)dv.y);
          }
        }
        __syncwarp();
#pragma unroll
        for (int s = 0; s < 2; s++) {
          const int k = lane + 32 * s;
          if (k >= P) break;
          float2 part[ND];
#pragma unroll
          for (int d = 0; d < ND; d++) part[d] = make_float2(0.0f, 0.0f);
          if (k == 0) {
            for (int j = 0; j < m; j++)
#pragma unroll
              for (int d = 0; d < ND; d++) {
                part[d].x += Q[j * ND + d].x;
                part[d].y += Q[j * ND + d].y;
              }
          } else {
            const float mik = -1.0f / (float)k;
            for (int j = 0; j < m; j++) {
              const float2 wk = W[j * P + k], wk1 = W[j * P + k - 1];
              const float2 cq = make_float2(wk.x * mik, wk.y * mik);
#pragma unroll
              for (int d = 0; d < ND; d++) {
                const float2 q = Q[j * ND + d], dd = Dd[j * ND + d];
                part[d].x += q.x * cq.x - q.y * cq.y + dd.x * wk1.x - dd.y * wk1.y;
                part[d].y += q.x * cq.y + q.y * cq.x + dd.x * wk1.y + dd.y * wk1.x;
              }
            }
          }
#pragma unroll
          for (int d = 0; d < ND; d++) {
            acc[s][d].x += (double)part[d].x;
            acc[s][d].y += (double)part[d].y;
          }
        }
      }
#pragma unroll
      for (int s = 0; s < 2; s++) {
        const int k = lane + 32 * s;
        if (k >= P) break;
#pragma unroll
        for (int d = 0; d < ND; d++) mp[((size_t)b * P + k) * ND + d] = acc[s][d];
      }
    }
  }
}

// ---------------------------------------------------------------------------
// M2M and L2L with the quadrant symmetry.  A child's centre is its parent's
// plus v_c h, h half the child's size, v_c = u_c (1 + i) with u_c = -1, -i,
// i, 1 for the reference's child order (-,-), (+,-), (-,+), (+,+), so that
// with the expansions scaled by the box sizes every translation of the tree
// is one of four operators that differ by the powers u_c^(i-j).  The
// operators of the child (+,+) are level-independent tables (built once, on
// the host, in device_binomials):
//   M2M  B[i][j] = 2^j (1+i)^(i-j) / 4^i * C(i-1, j-1)  (j >= 1),
//        B[i][0] = -(1+i)^i / (i 4^i),  B[0][0] = 1;
//   L2L  E[j][i] = C(j, i) 2^i (1+i)^(j-i) / 4^j  (i <= j),
// both lower-triangular, row a at a (a + 1) / 2, so that the rows below P
// are a prefix.  The M2M of a parent is then one triangular product with
// the children's four-point sums S_m[j] = sum_c u_c^m h_c[j]:
//   H_i = sum_{j <= i} B[i][j] S_{(i-j) mod 4}[j];
// the L2L one triangular product split by (j - i) mod 4,
//   A_q[i] = sum_{j >= i, j - i = q mod 4} E[j][i] l_j,
// and child c adds sum_q u_c^q A_q[i].  This is the reference's recurrence
// (laprouts2d.f:905-1015, 1020-1123) with the powers of z0 / r exact (the
// reference forms z0 from the rounded centres) and a quarter of its work.
// A block scans 2G boxes of the level at a time (G parents make about two
// (parent, coefficient, density) items a thread), compacts the parents
// into shared memory and takes them in groups of up to G: a pass over the
// items stages the inputs, a second one forms the outputs.  Small chunks
// give a level many blocks: with chunks of 256 boxes, levels of mostly
// parents ran a dozen groups one after another per block (M2M 1.37 ms,
// L2L 2.69 ms at 4M points, against 0.82 and 0.83 ms for the warp-per-
// parent recurrence); chunks of 2G boxes take 0.47 and 0.50 ms.
// ---------------------------------------------------------------------------
constexpr int SHIFT_THREADS = 128;

// i^q z
__device__ __forceinline__ double2 mul_ipow(double2 z, int q) {
  double2 r = (q & 1) ? make_double2(-z.y, z.x) : z;
  if (q & 2) r = make_double2(-r.x, -r.y);
  return r;
}

// The parents among the level's boxes [c0, min(c0 + CH, end)) (CH <=
// SHIFT_THREADS), in box order: their numbers and children in shared
// memory; returns their count.  need_eval: only parents with evaluation
// points (L2L).
__device__ __forceinline__ int collect_parents(const TV& t, int c0, int CH, int end,
                                               bool need_eval, int* box, int4* ch, int* wcnt) {
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const int b = c0 + tid;
  bool isp = false;
  int4 c = make_int4(-1, -1, -1, -1);
  if (tid < CH && b < end) {
    // a box has children iff its first child number is set (one round of
    // independent loads, no nchild read before the children)
    c = t.child[b];
    isp = c.x >= 0;
    if (need_eval) {
      int ne = 0;
      if (t.ifpghtarg > 0) ne += t.trng[b].y - t.trng[b].x;
      if (t.ifpgh > 0) ne += t.srng[b].y - t.srng[b].x;
      isp = isp && ne > 0;
    }
  }
  const unsigned m = __ballot_sync(~0u, isp);
  if (lane == 0) wcnt[w] = __popc(m);
  __syncthreads();
  int off = 0, tot = 0;
#pragma unroll
  for (int k = 0; k < SHIFT_THREADS / 32; k++) {
    const int v = wcnt[k];
    off += k < w ? v : 0;
    tot += v;
  }
  if (isp) {
    const int pos = off + __popc(m & ((1u << lane) - 1));
    box[pos] = b;
    ch[pos] = c;
  }
  __syncthreads();
  return tot;
}

// Shared memory of a block of the M2M / L2L kernels: the table prefix, the
// staged inputs of G parents (four sums per item for M2M, one coefficient
// for L2L), the compacted parents.
__host__ __device__ constexpr size_t shift_smem(int P, int ND, int G, bool m2m) {
  return sizeof(double2) * ((size_t)P * (P + 1) / 2 + (size_t)G * P * ND * (m2m ? 4 : 1)) +
         SHIFT_THREADS * (sizeof(int4) + sizeof(int)) + 32 * sizeof(int);
}

// step 3: M2M of the level's parents (every parent is written; a child
// without sources holds a zero expansion and adds nothing).
template <int ND>
__device__ __forceinline__ void m2m_level(const TV& t, int first, int n, int P, int G,
                                          const double2* __restrict__ tab,
                                          double2* __restrict__ mp) {
  extern __shared__ double2 smem[];
  const int PN = P * ND, nt = P * (P + 1) / 2;
  double2* B = smem;
  double2* S = B + nt;  // [parent][j][density][m]
  int4* ch = (int4*)(S + (size_t)G * PN * 4);
  int* box = (int*)(ch + SHIFT_THREADS);
  int* wcnt = box + SHIFT_THREADS;
  for (int e = threadIdx.x; e < nt; e += blockDim.x) B[e] = tab[e];
  const int end = first + n, CH = min(2 * G, SHIFT_THREADS);
  for (int c0 = first + blockIdx.x * CH; c0 < end; c0 += gridDim.x * CH) {
    const int np = collect_parents(t, c0, CH, end, false, box, ch, wcnt);
    for (int g0 = 0; g0 < np; g0 += G) {
      const int ne = min(G, np - g0) * PN;
      for (int e = threadIdx.x; e < ne; e += blockDim.x) {
        const int p = e / PN, r = e - p * PN;
        const int4 c = ch[g0 + p];
        const double2 h0 = mp[(size_t)c.x * PN + r], h1 = mp[(size_t)c.y * PN + r];
        const double2 h2 = mp[(size_t)c.z * PN + r], h3 = mp[(size_t)c.w * PN + r];
        const double2 a = cadd(h3, h0), b = cadd(h1, h2), s = csub(h3, h0), dd = csub(h2, h1);
        double2* o = S + (size_t)e * 4;
        o[0] = cadd(a, b);
        o[1] = make_double2(s.x - dd.y, s.y + dd.x);  // s + i dd
        o[2] = csub(a, b);
        o[3] = make_double2(s.x + dd.y, s.y - dd.x);  // s - i dd
      }
      __syncthreads();
      for (int e = threadIdx.x; e < ne; e += blockDim.x) {
        const int p = e / PN, r = e - p * PN, i = r / ND, d = r - i * ND;
        const double2* Br = B + i * (i + 1) / 2;
        const double2* Sp = S + ((size_t)p * PN + d) * 4;
        double2 acc0 = make_double2(0, 0), acc1 = make_double2(0, 0);
        int j = 0;
        for (; j + 1 <= i; j += 2) {
          cfma(acc0, Br[j], Sp[j * ND * 4 + ((i - j) & 3)]);
          cfma(acc1, Br[j + 1], Sp[(j + 1) * ND * 4 + ((i - j - 1) & 3)]);
        }
        if (j <= i) cfma(acc0, Br[j], Sp[j * ND * 4 + ((i - j) & 3)]);
        mp[(size_t)box[g0 + p] * PN + r] = cadd(acc0, acc1);
      }
      __syncthreads();
    }
  }
}

// ---------------------------------------------------------------------------
// step 2: P2L from list 4 (laprouts2d.f:501-690), z0 = x - c, w = r/z0:
// l_0 += q log|z0| - d/z0,  l_n += -q w^n/n - (d/z0) w^n.
// A warp takes 32 of its boxes at a time (as in P2M) and ballots those with
// a list 4 and evaluation points.  The sources of the (at most 5) list-4
// boxes are taken 32 at a time from their concatenation; each lane computes
// 1/z0, log|z0| and the powers of its source once.  The locals are zero
// before this kernel (each box is written by one warp), so they are stored,
// not updated.
// ---------------------------------------------------------------------------
template <int ND>
__global__ void __launch_bounds__(64) k_p2l(TV t, int first, int n, const double2* __restrict__ xs,
                                            Dens D, int P, double2* __restrict__ lo) {
  extern __shared__ double2 smem[];
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  resolve_range(t, first, n);
  double2* W = smem + (size_t)wib * (32 * P + 64 * ND + 32);
  double2* Q = W + 32 * P;
  double2* Dd = Q + 32 * ND;
  double* LG = (double*)(Dd + 32 * ND);
  for (int base = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; base < n; base += 32 * nw) {
    const int mine = base + lane * nw;
    int n4 = 0, lev = 0;
    double2 cen = make_double2(0, 0);
    if (mine < n) {
      const int b = first + mine;
      n4 = t.nl4[b];
      lev = t.level[b];
      cen = t.center[b];
      int ne = 0;
      if (t.ifpghtarg > 0) ne += t.trng[b].y - t.trng[b].x;
      if (t.ifpgh > 0) ne += t.srng[b].y - t.srng[b].x;
      if (ne == 0) n4 = 0;
    }
    unsigned wm = __ballot_sync(~0u, n4 > 0);
    while (wm) {
      const int src = __ffs(wm) - 1;
      wm &= wm - 1;
      const int b = first + base + src * nw;
      const int nb4 = __shfl_sync(~0u, n4, src);
      const double2 c = make_double2(__shfl_sync(~0u, cen.x, src), __shfl_sync(~0u, cen.y, src));
      const double r = t.boxsize[__shfl_sync(~0u, lev, src)];
      // lanes e < nb4: the list-4 box e, its first source and its offset in
      // the concatenation (exclusive scan of the counts)
      int2 sr = make_int2(0, 0);
      if (lane < nb4) sr = t.srng[t.l4[(size_t)MNLIST4 * b + lane]];
      int cnt = sr.y - sr.x, inc = cnt;
#pragma unroll
      for (int o = 1; o < 8; o <<= 1) {
        const int v = __shfl_up_sync(~0u, inc, o);
        if (lane >= o) inc += v;
      }
      const int tot = __shfl_sync(~0u, inc, MNLIST4 - 1);
      int bs[MNLIST4], be[MNLIST4];
#pragma unroll
      for (int e = 0; e < MNLIST4; e++) {
        bs[e] = __shfl_sync(~0u, sr.x, e);
        be[e] = __shfl_sync(~0u, inc - cnt, e);
      }
      double2 acc[2][ND];
#pragma unroll
      for (int s = 0; s < 2; s++)
#pragma unroll
        for (int d = 0; d < ND; d++) acc[s][d] = make_double2(0, 0);
      for (int g0 = 0; g0 < tot; g0 += 32) {
        const int m = min(32, tot - g0);
        __syncwarp();
        if (lane < m) {
          const int g = g0 + lane;
          int js = bs[0], jb = be[0];
#pragma unroll
          for (int e = 1; e < MNLIST4; e++)
            if (e < nb4 && g >= be[e]) {
              js = bs[e];
              jb = be[e];
            }
          const int j = js + (g - jb);
          const double2 x = xs[j];
          const double2 z0 = make_double2(x.x - c.x, x.y - c.y);
          const double2 zi = crcp(z0);
          const double2 w = make_double2(r * zi.x, r * zi.y);
          double2 pw = make_double2(1.0, 0.0);
          for (int k = 0; k < P; k++) {
            W[lane * P + k] = pw;
            pw = cmul(pw, w);
          }
          LG[lane] = log(hypot(z0.x, z0.y));
          const double2 mzi = cneg(zi);
#pragma unroll
          for (int d = 0; d < ND; d++) {
            Q[lane * ND + d] = D.q ? D.q[(size_t)j * D.ndc + D.d0 + d] : make_double2(0, 0);
            Dd[lane * ND + d] = D.d ? cmul(D.d[(size_t)j * D.ndc + D.d0 + d], mzi) : make_double2(0, 0);
          }
        }
        __syncwarp();
#pragma unroll
        for (int s = 0; s < 2; s++) {
          const int k = lane + 32 * s;
          if (k >= P) break;
          if (k == 0) {
            for (int j = 0; j < m; j++) {
              const double lg = LG[j];
#pragma unroll
              for (int d = 0; d < ND; d++) {
                const double2 q = Q[j * ND + d];
                acc[s][d].x += q.x * lg + Dd[j * ND + d].x;
                acc[s][d].y += q.y * lg + Dd[j * ND + d].y;
              }
            }
          } else {
            const double mik = -1.0 / k;
            for (int j = 0; j < m; j++) {
              const double2 wk = W[j * P + k];
              const double2 cq = cscale(wk, mik);
#pragma unroll
              for (int d = 0; d < ND; d++) {
                cfma(acc[s][d], Q[j * ND + d], cq);
                cfma(acc[s][d], Dd[j * ND + d], wk);
              }
            }
          }
        }
      }
#pragma unroll
      for (int s = 0; s < 2; s++) {
        const int k = lane + 32 * s;
        if (k >= P) break;
#pragma unroll
        for (int d = 0; d < ND; d++) lo[((size_t)b * P + k) * ND + d] = acc[s][d];
      }
    }
  }
}

// The mixed path's P2L: the same staging and lane mapping with the
// per-source terms and the sums over a chunk of 32 sources in FP32, each
// chunk's partial sums added to FP64 accumulators.  The source offset is
// formed in FP64 and scaled by the box size first, u = (x - c) / r (O(1)
// whatever the coordinates' magnitude), so that w = 1/u, d/z0 = (d/r) w and
// log|z0| = log|u| + log r, the last as log r times the chunk's charge sum
// in FP64.
template <int ND>
__global__ void __launch_bounds__(64) k_p2l_f32(TV t, int first, int n,
                                                const double2* __restrict__ xs, Dens D, int P,
                                                double2* __restrict__ lo) {
  extern __shared__ float2 fsm2[];
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  resolve_range(t, first, n);
  float2* W = fsm2 + (size_t)wib * (32 * P + 64 * ND + 16);
  float2* Q = W + 32 * P;
  float2* Dd = Q + 32 * ND;
  float* LG = reinterpret_cast<float*>(Dd + 32 * ND);
  for (int base = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; base < n; base += 32 * nw) {
    const int mine = base + lane * nw;
    int n4 = 0, lev = 0;
    double2 cen = make_double2(0, 0);
    if (mine < n) {
      const int b = first + mine;
      n4 = t.nl4[b];
      lev = t.level[b];
      cen = t.center[b];
      int ne = 0;
      if (t.ifpghtarg > 0) ne += t.trng[b].y - t.trng[b].x;
      if (t.ifpgh > 0) ne += t.srng[b].y - t.srng[b].x;
      if (ne == 0) n4 = 0;
    }
    unsigned wm = __ballot_sync(~0u, n4 > 0);
    while (wm) {
      const int src = __ffs(wm) - 1;
      wm &= wm - 1;
      const int b = first + base + src * nw;
      const int nb4 = __shfl_sync(~0u, n4, src);
      const double2 c = make_double2(__shfl_sync(~0u, cen.x, src), __shfl_sync(~0u, cen.y, src));
      const double r = t.boxsize[__shfl_sync(~0u, lev, src)];
      const double ri = 1.0 / r, lr = log(r);
      int2 sr = make_int2(0, 0);
      if (lane < nb4) sr = t.srng[t.l4[(size_t)MNLIST4 * b + lane]];
      int cnt = sr.y - sr.x, inc = cnt;
#pragma unroll
      for (int o = 1; o < 8; o <<= 1) {
        const int v = __shfl_up_sync(~0u, inc, o);
        if (lane >= o) inc += v;
      }
      const int tot = __shfl_sync(~0u, inc, MNLIST4 - 1);
      int bs[MNLIST4], be[MNLIST4];
#pragma unroll
      for (int e = 0; e < MNLIST4; e++) {
        bs[e] = __shfl_sync(~0u, sr.x, e);
        be[e] = __shfl_sync(~0u, inc - cnt, e);
      }
      double2 acc[2][ND];
#pragma unroll
      for (int s = 0; s < 2; s++)
#pragma unroll
        for (int d = 0; d < ND; d++) acc[s][d] = make_double2(0, 0);
      for (int g0 = 0; g0 < tot; g0 += 32) {
        const int m = min(32, tot - g0);
        __syncwarp();
        if (lane < m) {
          const int g = g0 + lane;
          int js = bs[0], jb = be[0];
#pragma unroll
          for (int e = 1; e < MNLIST4; e++)
            if (e < nb4 && g >= be[e]) {
              js = bs[e];
              jb = be[e];
            }
          const int j = js + (g - jb);
          const double2 x = xs[j];
          const float2 u = make_float2((float)((x.x - c.x) * ri), (float)((x.y - c.y) * ri));
          const float iu2 = 1.0f / (u.x * u.x + u.y * u.y);
          const float2 w = make_float2(u.x * iu2, -u.y * iu2);  // r / z0
          float2 pw = make_float2(1.0f, 0.0f);
          for (int k = 0; k < P; k++) {
            W[lane * P + k] = pw;
            pw = cmulf(pw, w);
          }
          LG[lane] = -0.5f * logf(iu2);  // log|u|
#pragma unroll
          for (int d = 0; d < ND; d++) {
            const double2 q = D.q ? D.q[(size_t)j * D.ndc + D.d0 + d] : make_double2(0, 0);
            Q[lane * ND + d] = make_float2((float)q.x, (float)q.y);
            float2 dd = make_float2(0.0f, 0.0f);
            if (D.d) {
              const double2 dv = D.d[(size_t)j * D.ndc + D.d0 + d];
              dd = cmulf(make_float2((float)(dv.x * ri), (float)(dv.y * ri)), w);
            }
            Dd[lane * ND + d] = make_float2(-dd.x, -dd.y);  // -d / z0
          }
        }
        __syncwarp();
#pragma unroll
        for (int s = 0; s < 2; s++) {
          const int k = lane + 32 * s;
          if (k >= P) break;
          float2 part[ND];
#pragma unroll
          for (int d = 0; d < ND; d++) part[d] = make_float2(0.0f, 0.0f);
          if (k == 0) {
            float qs[2 * ND];
#pragma unroll
            for (int e = 0; e < 2 * ND; e++) qs[e] = 0.0f;
            for (int j = 0; j < m; j++) {
              const float lg = LG[j];
#pragma unroll
              for (int d = 0; d < ND; d++) {
                const float2 q = Q[j * ND + d];
                part[d].x += q.x * lg + Dd[j * ND + d].x;
                part[d].y += q.y * lg + Dd[j * ND + d].y;
                qs[2 * d] += q.x;
                qs[2 * d + 1] += q.y;
              }
            }
#pragma unroll
            for (int d = 0; d < ND; d++) {
              acc[s][d].x += (double)part[d].x + lr * (double)qs[2 * d];
              acc[s][d].y += (double)part[d].y + lr * (double)qs[2 * d + 1];
            }
          } else {
            const float mik = -1.0f / (float)k;
            for (int j = 0; j < m; j++) {
              const float2 wk = W[j * P + k];
              const float2 cq = make_float2(wk.x * mik, wk.y * mik);
#pragma unroll
              for (int d = 0; d < ND; d++) {
                const float2 q = Q[j * ND + d], dd = Dd[j * ND + d];
                part[d].x += q.x * cq.x - q.y * cq.y + dd.x * wk.x - dd.y * wk.y;
                part[d].y += q.x * cq.y + q.y * cq.x + dd.x * wk.y + dd.y * wk.x;
              }
            }
#pragma unroll
            for (int d = 0; d < ND; d++) {
              acc[s][d].x += (double)part[d].x;
              acc[s][d].y += (double)part[d].y;
            }
          }
        }
      }
#pragma unroll
      for (int s = 0; s < 2; s++) {
        const int k = lane + 32 * s;
        if (k >= P) break;
#pragma unroll
        for (int d = 0; d < ND; d++) lo[((size_t)b * P + k) * ND + d] = acc[s][d];
      }
    }
  }
}

// ---------------------------------------------------------------------------
// step 4: M2L over list 2 (laprouts2d.f:1130-1244), z0 = c_src - c_tgt,
// u = r/z0, t_j = h_j (-u)^j:
//   L_0 += t_0 log|z0| + sum_{j>=1} t_j
//   L_i += (-t_0/i + sum_{j>=1} C(i+j-1, j-1) t_j) u^i
// The offset-independent matrix G (G_0j = 1, G_i0 = -1/i, G_ij = C(i+j-1,j-1))
// sits in shared memory; per pair only the power vectors depend on z0.
// ---------------------------------------------------------------------------
template <int ND>
__global__ void __launch_bounds__(128) k_m2l(TV t, int first, int n, int P,
                                             const double* __restrict__ binom,
                                             const double2* __restrict__ mp,
                                             double2* __restrict__ lo) {
  extern __shared__ double2 smem[];
  resolve_range(t, first, n);
  double* G = (double*)smem;  // G[j * P + i]
  for (int e = threadIdx.x; e < P * P; e += blockDim.x) {
    int j = e / P, i = e % P;
    double g;
    if (i == 0)
      g = (j == 0) ? 0.0 : 1.0;
    else if (j == 0)
      g = -1.0 / i;
    else
      g = binom[(size_t)(i + j - 1) * BINOM_N + (j - 1)];
    G[e] = g;
  }
  __syncthreads();
  double2* Tbase = smem + (P * P + 1) / 2;
  WARP_LOOP(n) {
    double2* T = Tbase + (size_t)wib * P * ND;
    int b = first + bi;
    int n2 = t.nl2[b];
    if (n2 == 0 || !t.has_eval_pts(b)) continue;
    double r = t.boxsize[t.level[b]];
    double2 cb = t.center[b];
    double2 acc[2][ND];
#pragma unroll
    for (int s = 0; s < 2; s++)
#pragma unroll
      for (int d = 0; d < ND; d++) acc[s][d] = make_double2(0, 0);
    for (int e = 0; e < n2; e++) {
      int jb = t.l2[(size_t)MNLIST2 * b + e];
      double2 cj = t.center[jb];
      double2 z0 = make_double2(cj.x - cb.x, cj.y - cb.y);
      double2 zi = crcp(z0);
      double2 u = make_double2(zi.x * r, zi.y * r);
      double lg = lane == 0 ? log(hypot(z0.x, z0.y)) : 0.0;
      lg = __shfl_sync(~0u, lg, 0);
      double2 ui[2];
      __syncwarp();
#pragma unroll
      for (int s = 0; s < 2; s++) {
        int j = lane + 32 * s;
        if (j >= P) break;
        double2 uj = cpow_int(u, j);
        ui[s] = uj;
        double2 sj = (j & 1) ? cneg(uj) : uj;
#pragma unroll
        for (int d = 0; d < ND; d++) T[j * ND + d] = cmul(mp[((size_t)jb * P + j) * ND + d], sj);
      }
      __syncwarp();
#pragma unroll
      for (int s = 0; s < 2; s++) {
        int i = lane + 32 * s;
        if (i >= P) break;
        double2 y[ND];
#pragma unroll
        for (int d = 0; d < ND; d++) y[d] = make_double2(0, 0);
        for (int j = 0; j < P; j++) {
          double g = G[j * P + i];
#pragma unroll
          for (int d = 0; d < ND; d++) {
            double2 tj = T[j * ND + d];
            y[d].x += g * tj.x;
            y[d].y += g * tj.y;
          }
        }
        if (i == 0) {
#pragma unroll
          for (int d = 0; d < ND; d++) {
            acc[s][d].x += y[d].x + T[d].x * lg;
            acc[s][d].y += y[d].y + T[d].y * lg;
          }
        } else {
#pragma unroll
          for (int d = 0; d < ND; d++) cfma(acc[s][d], y[d], ui[s]);
        }
      }
    }
#pragma unroll
    for (int s = 0; s < 2; s++) {
      int i = lane + 32 * s;
      if (i >= P) break;
#pragma unroll
      for (int d = 0; d < ND; d++) {
        size_t o = ((size_t)b * P + i) * ND + d;
        lo[o] = cadd(lo[o], acc[s][d]);
      }
    }
  }
}

// ---------------------------------------------------------------------------
// step 5: L2L of the level's parents with evaluation points into their four
// children (the quadrant-symmetric form above).
// ---------------------------------------------------------------------------
template <int ND>
__device__ __forceinline__ void l2l_level(const TV& t, int first, int n, int P, int G,
                                          const double2* __restrict__ tab,
                                          double2* __restrict__ lo) {
  extern __shared__ double2 smem[];
  const int PN = P * ND, nt = P * (P + 1) / 2;
  double2* E = smem;
  double2* L = E + nt;  // [parent][j][density]
  int4* ch = (int4*)(L + (size_t)G * PN);
  int* box = (int*)(ch + SHIFT_THREADS);
  int* wcnt = box + SHIFT_THREADS;
  for (int e = threadIdx.x; e < nt; e += blockDim.x) E[e] = tab[e];
  const int end = first + n, CH = min(2 * G, SHIFT_THREADS);
  for (int c0 = first + blockIdx.x * CH; c0 < end; c0 += gridDim.x * CH) {
    const int np = collect_parents(t, c0, CH, end, true, box, ch, wcnt);
    for (int g0 = 0; g0 < np; g0 += G) {
      const int ne = min(G, np - g0) * PN;
      for (int e = threadIdx.x; e < ne; e += blockDim.x) {
        const int p = e / PN, r = e - p * PN;
        L[e] = lo[(size_t)box[g0 + p] * PN + r];
      }
      __syncthreads();
      for (int e = threadIdx.x; e < ne; e += blockDim.x) {
        const int p = e / PN, r = e - p * PN, i = r / ND, d = r - i * ND;
        const int4 c = ch[g0 + p];
        // the children's locals first: their loads overlap the sums
        double2 cur[4];
#pragma unroll
        for (int k = 0; k < 4; k++) cur[k] = lo[(size_t)child_of(c, k) * PN + r];
        const double2* Lp = L + (size_t)p * PN + d;
        double2 A[4];
#pragma unroll
        for (int q = 0; q < 4; q++) A[q] = make_double2(0, 0);
        for (int j0 = i; j0 < P; j0 += 4) {
#pragma unroll
          for (int q = 0; q < 4; q++) {
            const int j = j0 + q;
            if (j < P) cfma(A[q], E[j * (j + 1) / 2 + i], Lp[j * ND]);
          }
        }
        // child c adds sum_q u_c^q A_q: (+,+) E + F, (-,-) E - F,
        // (-,+) G + iH, (+,-) G - iH
        const double2 Ev = cadd(A[0], A[2]), F = cadd(A[1], A[3]);
        const double2 Gv = csub(A[0], A[2]), H = csub(A[1], A[3]);
        const double2 add[4] = {csub(Ev, F), make_double2(Gv.x + H.y, Gv.y - H.x),
                                make_double2(Gv.x - H.y, Gv.y + H.x), cadd(Ev, F)};
#pragma unroll
        for (int k = 0; k < 4; k++) lo[(size_t)child_of(c, k) * PN + r] = cadd(cur[k], add[k]);
      }
      __syncthreads();
    }
  }
}

// One level of M2M / L2L per launch (the host knows the level's boxes).
// (first = RANGE_LEVEL: the level's boxes from the device level table).
template <int ND>
__global__ void __launch_bounds__(SHIFT_THREADS) k_m2m(TV t, int first, int n, int lev, int P, int G,
                                                       const double2* __restrict__ tab,
                                                       double2* __restrict__ mp) {
  resolve_range(t, first, n, lev);
  m2m_level<ND>(t, first, n, P, G, tab, mp);
}
template <int ND>
__global__ void __launch_bounds__(SHIFT_THREADS) k_l2l(TV t, int first, int n, int lev, int P, int G,
                                                       const double2* __restrict__ tab,
                                                       double2* __restrict__ lo) {
  resolve_range(t, first, n, lev);
  l2l_level<ND>(t, first, n, P, G, tab, lo);
}

// The levels >= lev_min in one cooperative launch, the boxes of every level
// from the tree's device level table and a grid barrier between levels: the
// upward pass finest parents first, the downward pass coarsest first.  The
// host launches the levels below lev_min one by one; this kernel takes the
// part of a tree deeper than the host expected (nothing when the guess was
// right).  A barrier that gives up sets *err (the call reports IER_TIMEOUT).
template <int ND>
__global__ void __launch_bounds__(SHIFT_THREADS) k_m2m_all(TV t, int P, int G,
                                                           const double2* __restrict__ tab,
                                                           double2* __restrict__ mp, GridBar* gb,
                                                           int* err, int lev_min) {
  const TreeCtl* c = t.ctl;
  if (c->status != TB_OK) return;
  const int nl = c->nlevels, lo_lev = max(lev_min, 1);
  for (int lev = nl - 1; lev >= lo_lev; lev--) {
    const int first = c->lfirst[lev];
    m2m_level<ND>(t, first, c->llast[lev] - first + 1, P, G, tab, mp);
    if (lev > lo_lev && !grid_barrier(gb, 1)) {
      if (threadIdx.x == 0) atomicExch(err, 1);
      return;
    }
  }
}
template <int ND>
__global__ void __launch_bounds__(SHIFT_THREADS) k_l2l_all(TV t, int P, int G,
                                                           const double2* __restrict__ tab,
                                                           double2* __restrict__ lo, GridBar* gb,
                                                           int* err, int lev_min) {
  const TreeCtl* c = t.ctl;
  if (c->status != TB_OK) return;
  const int nl = c->nlevels;
  for (int lev = max(lev_min, 1); lev <= nl - 1; lev++) {
    const int first = c->lfirst[lev];
    l2l_level<ND>(t, first, c->llast[lev] - first + 1, P, G, tab, lo);
    if (lev < nl - 1 && !grid_barrier(gb, 1)) {
      if (threadIdx.x == 0) atomicExch(err, 1);
      return;
    }
  }
}
// ---------------------------------------------------------------------------
// gather / unpack
// ---------------------------------------------------------------------------
__global__ void k_gather_pts(const double* __restrict__ xy, const int* __restrict__ perm, long n,
                             double2* __restrict__ out) {
  long k = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (k >= n) return;
  int i = perm[k];
  out[k] = make_double2(xy[2 * (size_t)i], xy[2 * (size_t)i + 1]);
}

// Caller densities -> sorted Cauchy densities (lfmm2d.f:139-156, rfmm2d.f:137-151)
__global__ void k_gather_dens(int fe, int nd, int ndc, const int* __restrict__ perm, long n,
                              const double* __restrict__ charge, const double* __restrict__ dipstr,
                              const double* __restrict__ dipvec, double2* __restrict__ qs,
                              double2* __restrict__ ds) {
  long k = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (k >= n) return;
  size_t i = perm[k];
  for (int j = 0; j < nd; j++) {
    if (fe == FE_CAUCHY) {
      if (qs) qs[k * ndc + j] = ((const double2*)charge)[i * nd + j];
      if (ds) ds[k * ndc + j] = ((const double2*)dipstr)[i * nd + j];
    } else {
      double2 mv = make_double2(0, 0);
      if (ds) mv = make_double2(-dipvec[(i * 2 + 0) * nd + j], -dipvec[(i * 2 + 1) * nd + j]);
      if (fe == FE_LAPLACE) {
        if (qs) {
          double2 q = ((const double2*)charge)[i * nd + j];
          qs[k * ndc + 2 * j] = make_double2(q.x, 0);
          qs[k * ndc + 2 * j + 1] = make_double2(q.y, 0);
        }
        if (ds) {
          double2 dd = ((const double2*)dipstr)[i * nd + j];
          ds[k * ndc + 2 * j] = cscale(mv, dd.x);
          ds[k * ndc + 2 * j + 1] = cscale(mv, dd.y);
        }
      } else {
        if (qs) qs[k * ndc + j] = make_double2(charge[i * nd + j], 0);
        if (ds) ds[k * ndc + j] = cscale(mv, dipstr[i * nd + j]);
      }
    }
  }
}

// Sorted Cauchy results -> caller layout and order (lfmm2d.f:169-223,
// rfmm2d.f:158-212; cfmm2d.f:399-432 for the inverse permutation).
__global__ void k_unpack(int fe, int nd, int ndc, int ifl, const int* __restrict__ inv, long n,
                         const double2* __restrict__ P1, const double2* __restrict__ G1,
                         const double2* __restrict__ H1, double* pot, double* grad, double* hess) {
  // one output point per thread (caller order), read from its tree position:
  // the writes are contiguous, the reads gathered
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const size_t k = inv[i];
  for (int j = 0; j < nd; j++) {
    if (fe == FE_CAUCHY) {
      ((double2*)pot)[i * nd + j] = P1[k * ndc + j];
      if (ifl >= 2) ((double2*)grad)[i * nd + j] = G1[k * ndc + j];
      if (ifl >= 3) ((double2*)hess)[i * nd + j] = H1[k * ndc + j];
    } else if (fe == FE_LAPLACE) {
      double2 a = P1[k * ndc + 2 * j], bb = P1[k * ndc + 2 * j + 1];
      ((double2*)pot)[i * nd + j] = make_double2(a.x, bb.x);
      if (ifl >= 2) {
        double2 ga = G1[k * ndc + 2 * j], gb = G1[k * ndc + 2 * j + 1];
        ((double2*)grad)[(i * 2 + 0) * nd + j] = make_double2(ga.x, gb.x);
        ((double2*)grad)[(i * 2 + 1) * nd + j] = make_double2(-ga.y, -gb.y);
      }
      if (ifl >= 3) {
        double2 ha = H1[k * ndc + 2 * j], hb = H1[k * ndc + 2 * j + 1];
        ((double2*)hess)[(i * 3 + 0) * nd + j] = make_double2(ha.x, hb.x);
        ((double2*)hess)[(i * 3 + 1) * nd + j] = make_double2(-ha.y, -hb.y);
        ((double2*)hess)[(i * 3 + 2) * nd + j] = make_double2(-ha.x, -hb.x);
      }
    } else {
      pot[i * nd + j] = P1[k * ndc + j].x;
      if (ifl >= 2) {
        double2 g = G1[k * ndc + j];
        grad[(i * 2 + 0) * nd + j] = g.x;
        grad[(i * 2 + 1) * nd + j] = -g.y;
      }
      if (ifl >= 3) {
        double2 h = H1[k * ndc + j];
        hess[(i * 3 + 0) * nd + j] = h.x;
        hess[(i * 3 + 1) * nd + j] = -h.y;
        hess[(i * 3 + 2) * nd + j] = -h.x;
      }
    }
  }
}

// inv[perm[k]] = k: tree position of every caller-order point
__global__ void k_inverse_perm(const int* __restrict__ perm, long n, int* __restrict__ inv) {
  const long k = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (k < n) inv[perm[k]] = (int)k;
}

// Work counts for the roofline accounting (enabled by set_stats).
__global__ void k_stats(TV t, int nb, unsigned long long* out) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (nb < 0) {
    int f = RANGE_ALL;
    resolve_range(t, f, nb);
  }
  unsigned long long c[6] = {0, 0, 0, 0, 0, 0};
  if (b < nb) {
    long ne = 0;
    if (t.ifpgh > 0) ne += t.srng[b].y - t.srng[b].x;
    if (t.ifpghtarg > 0) ne += t.trng[b].y - t.trng[b].x;
    if (t.nchild[b] == 0) {
      c[0] = 1;
      long s = 0;
      for (int e = 0; e < t.nl1[b]; e++) {
        int j = t.l1[(size_t)MNLIST1 * b + e];
        s += t.srng[j].y - t.srng[j].x;
      }
      c[1] = (unsigned long long)(ne * s);
      c[3] = (unsigned long long)(ne * t.nl3[b]);
      c[5] = (unsigned long long)ne;
    }
    if (ne > 0 && t.level[b] >= 2) {
      c[2] = t.nl2[b];
      long s4 = 0;
      for (int e = 0; e < t.nl4[b]; e++) {
        int j = t.l4[(size_t)MNLIST4 * b + e];
        s4 += t.srng[j].y - t.srng[j].x;
      }
      c[4] = (unsigned long long)s4;
    }
  }
  for (int k = 0; k < 6; k++) {
    unsigned long long v = c[k];
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(~0u, v, o);
    if ((threadIdx.x & 31) == 0 && v) atomicAdd(&out[k], v);
  }
}

// Outputs are zero when every source and target coincides (a tree of one
// box of size 0): all interactions are omitted self-interactions.  Checked on
// the device for calls that did not read the tree back.
__global__ void k_zero_if_point_tree(const TreeCtl* c, double* a0, long n0, double* a1, long n1,
                                     double* a2, long n2, double* a3, long n3, double* a4,
                                     long n4, double* a5, long n5) {
  if (c->status != TB_OK || c->bs[0] != 0.0) return;
  const long g = blockIdx.x * (long)blockDim.x + threadIdx.x, gs = (long)gridDim.x * blockDim.x;
  double* a[6] = {a0, a1, a2, a3, a4, a5};
  const long n[6] = {n0, n1, n2, n3, n4, n5};
  for (int q = 0; q < 6; q++)
    for (long i = g; i < n[q]; i += gs) a[q][i] = 0.0;
}

// ---------------------------------------------------------------------------
// host driver
// ---------------------------------------------------------------------------
int warp_grid(long nitems, int warps_per_block) {
  long blocks = (nitems + warps_per_block - 1) / warps_per_block;
  return (int)std::max(1L, std::min(blocks, 148L * 64));
}

// Blocks of a cooperative launch of `kernel` (all resident): as many per SM
// as registers and shared memory allow, up to g_coop_blocks_per_sm.
std::atomic<int> g_coop_blocks_per_sm{8};

template <typename K>
int coop_grid(K kernel, int threads, size_t smem) {
  static std::mutex mu;
  static std::vector<std::pair<std::pair<const void*, size_t>, int>> done[128];
  int dev = 0;
  B2_CHECK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 128) throw CudaError("device ordinal beyond 127", IER_CUDA);
  std::lock_guard<std::mutex> g(mu);
  const size_t key = smem * 64 + (size_t)g_coop_blocks_per_sm.load();
  for (auto& e : done[dev])
    if (e.first.first == (const void*)kernel && e.first.second == key) return e.second;
  int nsm = 0, per = 0, coop = 0;
  B2_CHECK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  B2_CHECK(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
  if (!coop) throw CudaError("cooperative launch not supported", IER_CUDA);
  B2_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, threads, smem));
  if (per < 1) throw CudaError("cooperative pass does not fit an SM", IER_CUDA);
  const int grid = std::min(per, g_coop_blocks_per_sm.load()) * nsm;
  done[dev].push_back({{(const void*)kernel, key}, grid});
  return grid;
}

// Launch context of one evaluation: the box count to size grids by (the
// capacity when the host did not read the tree back), whether ranges come
// from the device level table, the grid barrier of the all-level passes and
// the evaluation's error flag.
struct Launch {
  int nb;
  bool dev;
  GridBar* gb;
  int* err;
  int lev_hint;  // levels the host launches one by one (device ranges)
};

template <int ND>
void run_chunk(const TV& tv, DeviceTree& T, const LapArgs& a, const Dens& D, int P,
               const double2* xs, const double2* xt, double2* mp, double2* lo, double2* ps,
               double2* gs, double2* hs, double2* pt, double2* gt, double2* ht, const Launch& X,
               cudaStream_t st, cudaEvent_t* ev, const MixedData* M, const MixedData& LD,
               bool skip_near) {
  const double* binom = device_binomials();
  const int ifnear = skip_near ? 0 : a.ifnear;
  const int nb = X.nb;
  const bool dev = X.dev;
  const int nl = dev ? 0 : T.nlevels;
  const int all = dev ? RANGE_ALL : 0;
  const int from2 = dev ? RANGE_FROM2 : (nl >= 2 ? T.lfirst[2] : 0);
  const int n_from2 = dev ? nb : (nl >= 2 ? nb - T.lfirst[2] : 0);
  B2_CHECK(cudaEventRecord(ev[0], st));
  size_t sm_p2m = sizeof(double2) * 2 * (P2M_CHUNK * (size_t)P + 2 * P2M_CHUNK * ND);
  size_t sm_p2l = sizeof(double2) * 2 * (32 * (size_t)P + 64 * ND + 32);
  set_smem_attr(k_p2m<ND>, sm_p2m);
  set_smem_attr(k_p2l<ND>, sm_p2l);
  if (M) {
    const size_t sm = sizeof(float2) * 2 * (P2M_CHUNK * (size_t)P + 2 * P2M_CHUNK * ND);
    set_smem_attr(k_p2m_f32<ND>, sm);
    k_p2m_f32<ND><<<warp_grid(nb, 2), 64, sm, st>>>(tv, all, nb, xs, D, P, mp);
  } else {
    k_p2m<ND><<<warp_grid(nb, 2), 64, sm_p2m, st>>>(tv, all, nb, xs, D, P, mp);
  }
  B2_LAUNCH_CHECK();
  B2_CHECK(cudaEventRecord(ev[1], st));
  // M2M / L2L: parents per group for about two items a thread
  const double2* tab_m2m = device_shift_tables();
  const double2* tab_l2l = tab_m2m + SHIFT_TAB;
  const int g_m2m = std::max(1, std::min(SHIFT_THREADS / 2, 2 * SHIFT_THREADS / (P * ND)));
  const int g_l2l = g_m2m;
  const size_t sm_m2m = shift_smem(P, ND, g_m2m, true), sm_l2l = shift_smem(P, ND, g_l2l, false);
  set_smem_attr(k_m2m<ND>, sm_m2m);
  set_smem_attr(k_l2l<ND>, sm_l2l);
  // one block per chunk of 2G boxes of a level, at most 64 blocks an SM
  const int shift_ch = std::min(2 * g_m2m, SHIFT_THREADS);
  auto shift_grid = [&](long n) { return (int)std::max(1L, std::min<long>(ceil_div(n, shift_ch), 148L * 64)); };
  TV tvc = tv;
  // boxes at level l: at most 4^l and the capacity (grids of the levels the
  // host launches without knowing their size)
  auto level_bound = [&](int l) { return (int)std::min<long>(nb, l < 15 ? 1L << (2 * l) : nb); };
  if (dev) {
    // the part deeper than the expected depth first, then level by level
    set_smem_attr(k_m2m_all<ND>, sm_m2m);
    const int grid = coop_grid(k_m2m_all<ND>, SHIFT_THREADS, sm_m2m);
    int Pv = P, Gv = g_m2m, lmin = X.lev_hint;
    GridBar* gb = X.gb;
    int* err = X.err;
    void* args[] = {&tvc, &Pv, &Gv, (void*)&tab_m2m, &mp, &gb, &err, &lmin};
    B2_CHECK(cudaLaunchCooperativeKernel((const void*)k_m2m_all<ND>, dim3(grid),
                                         dim3(SHIFT_THREADS), args, sm_m2m, st));
    B2_LAUNCH_CHECK();
    for (int l = X.lev_hint - 1; l >= 1; l--) {
      const int nbl = level_bound(l);
      k_m2m<ND><<<shift_grid(nbl), SHIFT_THREADS, sm_m2m, st>>>(tv, RANGE_LEVEL, nbl, l, P, g_m2m,
                                                                tab_m2m, mp);
      B2_LAUNCH_CHECK();
    }
  } else {
    for (int l = nl - 1; l >= 1; l--) {
      int f = T.lfirst[l], n = T.llast[l] - f + 1;
      k_m2m<ND><<<shift_grid(n), SHIFT_THREADS, sm_m2m, st>>>(tv, f, n, l, P, g_m2m, tab_m2m, mp);
      B2_LAUNCH_CHECK();
    }
  }
  B2_CHECK(cudaEventRecord(ev[2], st));
  B2_CHECK(cudaMemsetAsync(lo, 0, sizeof(double2) * (size_t)nb * P * ND, st));
  if (n_from2 > 0 && M) {
    const size_t sm = sizeof(float2) * 2 * (32 * (size_t)P + 64 * ND + 16);
    set_smem_attr(k_p2l_f32<ND>, sm);
    k_p2l_f32<ND><<<warp_grid(n_from2, 2), 64, sm, st>>>(tv, from2, n_from2, xs, D, P, lo);
    B2_LAUNCH_CHECK();
  } else if (n_from2 > 0) {
    k_p2l<ND><<<warp_grid(n_from2, 2), 64, sm_p2l, st>>>(tv, from2, n_from2, xs, D, P, lo);
    B2_LAUNCH_CHECK();
  }
  B2_CHECK(cudaEventRecord(ev[3], st));
  if (n_from2 > 0 && M) {
    lap_mixed_m2l(ND, tv, from2, n_from2, P, binom, *M, mp, lo, st);
  } else if (n_from2 > 0) {
    size_t sm = sizeof(double) * (P * P + 1) + sizeof(double2) * 4 * P * ND;
    if (sm > 48 * 1024)
      set_smem_attr(k_m2l<ND>, sm);
    k_m2l<ND><<<warp_grid(n_from2, 4), 128, sm, st>>>(tv, from2, n_from2, P, binom, mp, lo);
    B2_LAUNCH_CHECK();
  }
  B2_CHECK(cudaEventRecord(ev[4], st));
  if (dev) {
    for (int l = 1; l <= X.lev_hint - 1; l++) {
      const int nbl = level_bound(l);
      k_l2l<ND><<<shift_grid(nbl), SHIFT_THREADS, sm_l2l, st>>>(tv, RANGE_LEVEL, nbl, l, P, g_l2l,
                                                                tab_l2l, lo);
      B2_LAUNCH_CHECK();
    }
    set_smem_attr(k_l2l_all<ND>, sm_l2l);
    const int grid = coop_grid(k_l2l_all<ND>, SHIFT_THREADS, sm_l2l);
    int Pv = P, Gv = g_l2l, lmin = X.lev_hint;
    GridBar* gb = X.gb;
    int* err = X.err;
    void* args[] = {&tvc, &Pv, &Gv, (void*)&tab_l2l, &lo, &gb, &err, &lmin};
    B2_CHECK(cudaLaunchCooperativeKernel((const void*)k_l2l_all<ND>, dim3(grid),
                                         dim3(SHIFT_THREADS), args, sm_l2l, st));
    B2_LAUNCH_CHECK();
  } else {
    for (int l = 1; l <= nl - 1; l++) {
      int f = T.lfirst[l], n = T.llast[l] - f + 1;
      k_l2l<ND><<<shift_grid(n), SHIFT_THREADS, sm_l2l, st>>>(tv, f, n, l, P, g_l2l, tab_l2l, lo);
      B2_LAUNCH_CHECK();
    }
  }
  B2_CHECK(cudaEventRecord(ev[5], st));
  // near-field threshold boxsize(0) 2^-51, taken on the device from the tree
  const double thresh = -1.0;
  auto leaf = [&](int use_t, int ifl, const double2* xe, double2* po, double2* gr, double2* he) {
    if (ifl <= 0) return;
    if (M) {
      // ev[7]: between the far-field and near-field kernels of the sources
      lap_mixed_leaf(ND, ifl, tv, nb, use_t, *M, xe, D.ndc, D.d0, P, mp, lo, thresh, ifnear, po,
                     gr, he, st, use_t == 0 ? ev[7] : nullptr);
      return;
    }
    lap_fp64_leaf(ND, ifl, tv, use_t, LD, xe, D, P, mp, lo, thresh, ifnear, po, gr, he, st);
  };
  leaf(0, a.ifpgh, xs, ps, gs, hs);
  leaf(1, a.ifpghtarg, xt, pt, gt, ht);
  B2_CHECK(cudaEventRecord(ev[6], st));
}

}  // namespace

struct LapPlan {
  LapArgs a;                      // geometry and flags (density/output pointers unused)
  cudaStream_t st = nullptr;      // stream owning the buffers
  bool own = false;               // st is the shared plan stream (not the caller's)
  bool dev = false;               // box ranges from the device (tree not read back)
  int nd = 1, ndc = 1, P = 0, chunk = 1, ndiv = 0;
  long ns = 0, nt = 0;
  bool fc = false, fd = false, mixed = false;
  bool zero = false;              // nothing interacts: every output is zero
  float tree_ms = 0;
  DeviceTree T;
  DBuf<double2> xs, xt, qs, ds, ps, gs, hs, pt, gt, ht, mp, lo;
  DBuf<int> err;
  DBuf<GridBar> gbar;      // grid barrier of the all-level M2M / L2L passes
  DBuf<int> inv_s, inv_t;  // tree position of every caller-order source / target
  MixedData MD;
  TV tv{};
  cudaEvent_t ev[8] = {};
  cudaEvent_t tree_ev[2] = {};  // start / end of the tree build (plans on the caller's stream)
  ~LapPlan() {
    for (auto& e : ev)
      if (e) cudaEventDestroy(e);
    for (auto& e : tree_ev)
      if (e) cudaEventDestroy(e);
  }
};

namespace {

// Element counts (doubles) of the caller's output arrays.
struct OutSizes {
  size_t pot, grad, hess, pott, gradt, hesst;
};

OutSizes out_sizes(const LapPlan& p) {
  const LapArgs& a = p.a;
  const size_t cw = a.fe == FE_REAL ? 1 : 2;
  const size_t gw = a.fe == FE_CAUCHY ? 1 : 2, hw = a.fe == FE_CAUCHY ? 1 : 3;
  const size_t nd = p.nd, ns = p.ns, nt = p.nt;
  OutSizes o{};
  o.pot = a.ifpgh >= 1 ? cw * nd * ns : 0;
  o.grad = a.ifpgh >= 2 ? cw * gw * nd * ns : 0;
  o.hess = a.ifpgh >= 3 ? cw * hw * nd * ns : 0;
  o.pott = a.ifpghtarg >= 1 ? cw * nd * nt : 0;
  o.gradt = a.ifpghtarg >= 2 ? cw * gw * nd * nt : 0;
  o.hesst = a.ifpghtarg >= 3 ? cw * hw * nd * nt : 0;
  return o;
}

// Levels of the upward and downward passes the host launches one by one
// without reading the tree back (see k_m2m_all): the depth of the last tree
// of this size, else that of a uniform cloud.
int level_hint(long npts, int ndiv) {
  int nb = 0, nl = 0;
  if (tree_shape(npts, ndiv, &nb, &nl)) return nl;
  int l = 1;
  for (double boxes = (double)npts / std::max(ndiv, 1); boxes > 1 && l < NLMAX; boxes /= 4) l++;
  return l;
}

// The end-of-call check, one small readback after `st` has finished: the
// evaluation's error flag and, when the host did not read the tree back, the
// tree's box count and status.  IER_RETRY: the tree needs the build with
// read-back (more boxes than the capacity, or more than 32 levels).
constexpr int IER_RETRY = -1;

int finish(LapPlan& p, cudaStream_t st) {
  int* h = pinned_ints(8);
  B2_CHECK(cudaMemcpyAsync(h, p.err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  const bool dev = p.dev && p.T.ctl.p;
  if (dev)  // nboxes, nlevels, cap, status: the head of the control block
    B2_CHECK(cudaMemcpyAsync(h + 4, p.T.ctl.p, 4 * sizeof(int), cudaMemcpyDeviceToHost, st));
  B2_CHECK(cudaStreamSynchronize(st));
  if (dev) {
    const int status = h[7];
    if (status == TB_OVERFLOW || status == TB_DEEP) return IER_RETRY;
    if (status == TB_BADPTS) return IER_BADARG;
    if (status != TB_OK) return IER_TIMEOUT;
    note_tree_shape(p.ns + p.nt, p.ndiv, h[4], h[5]);
  }
  if (h[0]) {
    B2_CHECK(cudaMemsetAsync(p.err.p, 0, sizeof(int), st));
    B2_CHECK(cudaStreamSynchronize(st));
    return IER_TIMEOUT;
  }
  return IER_OK;
}

}  // namespace

int lap_plan_create(const LapArgs& a, cudaStream_t st_in, bool own_stream, LapPlan** out,
                    bool device_ranges) {
  *out = nullptr;
  if (a.nd < 1 || a.ns < 0 || a.nt < 0 || a.ifpgh < 0 || a.ifpgh > 3 || a.ifpghtarg < 0 ||
      a.ifpghtarg > 3 || a.ns > (1L << 30) || a.nt > (1L << 30) || a.fe < 0 || a.fe > 2)
    return IER_BADARG;
  if (a.ns > 0 && !a.src) return IER_BADARG;
  if (a.nt > 0 && a.ifpghtarg > 0 && !a.trg) return IER_BADARG;
  int dev = 0;
  B2_CHECK(cudaGetDevice(&dev));
  configure_mempool(dev);
  std::unique_ptr<LapPlan> pl(new LapPlan());
  LapPlan& p = *pl;
  p.a = a;
  p.a.charge = p.a.dipstr = p.a.dipvec = nullptr;
  p.a.pot = p.a.grad = p.a.hess = p.a.pottarg = p.a.gradtarg = p.a.hesstarg = nullptr;
  p.a.timeinfo = nullptr;
  p.nd = a.nd;
  p.ndc = a.fe == FE_LAPLACE ? 2 * a.nd : a.nd;
  p.ns = a.ns;
  p.nt = a.ifpghtarg > 0 ? a.nt : 0;
  p.a.nt = p.nt;
  p.fc = a.charge != nullptr;
  p.fd = a.dipstr != nullptr;
  if (own_stream) {
    p.st = plan_stream(dev);
    p.own = true;
    // the plan's stream starts after the work already queued on the caller's
    cudaEvent_t e;
    B2_CHECK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    B2_CHECK(cudaEventRecord(e, st_in));
    B2_CHECK(cudaStreamWaitEvent(p.st, e, 0));
    B2_CHECK(cudaEventDestroy(e));
  } else {
    p.st = st_in;
  }
  cudaStream_t st = p.st;
  for (auto& e : p.ev) B2_CHECK(cudaEventCreate(&e));
  p.err.alloc(1, st);
  p.err.zero(1);
  if (p.ns == 0 || (!p.fc && !p.fd)) {
    p.zero = true;
    if (own_stream) B2_CHECK(cudaStreamSynchronize(st));
    *out = pl.release();
    return IER_OK;
  }
  int ndiv = a.ndiv > 0 ? a.ndiv : lap_ndiv(a.eps);
  if (ndiv <= 0) ndiv = (int)std::min<long>(p.ns + p.nt, 1L << 30);
  p.ndiv = ndiv;
  p.P = lap_nterms(a.eps) + 1;
  if (p.P > 64) return IER_NTERMS;
  p.mixed = a.precision == PREC_MIXED || (a.precision == PREC_AUTO && a.eps >= 1e-6);

  cudaEvent_t e0, e1;
  B2_CHECK(cudaEventCreate(&e0));
  B2_CHECK(cudaEventCreate(&e1));
  B2_CHECK(cudaEventRecord(e0, st));
  // a level-balanced tree has no cached shape to size a one-attempt build:
  // it is built with the host in the loop
  p.dev = device_ranges && !own_stream && a.lbal == 0.0;
  if (p.dev)
    build_device_tree_async(p.T, a.src, p.ns, a.trg, p.nt, a.idivflag, ndiv, NLMAX,
                            tree_capacity_guess(p.ns + p.nt, ndiv, a.async_call ? 1.25 : 1.1),
                            st);
  else
    build_device_tree(p.T, a.src, p.ns, a.trg, p.nt, a.idivflag, ndiv, NLMAX, st, a.lbal);
  B2_CHECK(cudaEventRecord(e1, st));
  DeviceTree& T = p.T;
  if (!p.dev && T.bs0 == 0.0) {
    // every source and target coincides: all interactions are self
    // interactions, which the reference omits, so every output is zero
    p.zero = true;
    if (own_stream) B2_CHECK(cudaStreamSynchronize(st));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    *out = pl.release();
    return IER_OK;
  }
  const int nb = T.nboxes;  // the capacity when the tree was not read back
  p.xs.alloc(p.ns, st);
  k_gather_pts<<<ceil_div(p.ns, 256), 256, 0, st>>>(a.src, T.isrc.p, p.ns, p.xs.p);
  B2_LAUNCH_CHECK();
  p.inv_s.alloc(p.ns, st);
  k_inverse_perm<<<ceil_div(p.ns, 256), 256, 0, st>>>(T.isrc.p, p.ns, p.inv_s.p);
  B2_LAUNCH_CHECK();
  if (p.nt > 0) {
    p.xt.alloc(p.nt, st);
    k_gather_pts<<<ceil_div(p.nt, 256), 256, 0, st>>>(a.trg, T.itarg.p, p.nt, p.xt.p);
    B2_LAUNCH_CHECK();
    p.inv_t.alloc(p.nt, st);
    k_inverse_perm<<<ceil_div(p.nt, 256), 256, 0, st>>>(T.itarg.p, p.nt, p.inv_t.p);
    B2_LAUNCH_CHECK();
  }
  const size_t nsd = (size_t)p.ns * p.ndc, ntd = (size_t)p.nt * p.ndc;
  if (p.fc) p.qs.alloc(nsd, st);
  if (p.fd) p.ds.alloc(nsd, st);
  if (a.ifpgh >= 1) p.ps.alloc(nsd, st);
  if (a.ifpgh >= 2) p.gs.alloc(nsd, st);
  if (a.ifpgh >= 3) p.hs.alloc(nsd, st);
  if (a.ifpghtarg >= 1 && p.nt) p.pt.alloc(ntd, st);
  if (a.ifpghtarg >= 2 && p.nt) p.gt.alloc(ntd, st);
  if (a.ifpghtarg >= 3 && p.nt) p.ht.alloc(ntd, st);
  p.tv = TV{T.center.p, T.level.p, T.nchild.p, T.child.p, T.srng.p, T.trng.p, T.nlist1.p,
            T.list1.p, T.nlist2.p, T.list2.p, T.nlist3.p, T.list3.p, T.nlist4.p, T.list4.p,
            &T.ctl.p->bs[0], a.ifpgh, p.nt > 0 ? a.ifpghtarg : 0, T.ctl.p};
  p.chunk = p.ndc >= 8 ? 8 : (p.ndc >= 4 ? 4 : (p.ndc >= 2 ? 2 : 1));
  p.mp.alloc((size_t)nb * p.P * p.chunk, st);
  p.lo.alloc((size_t)nb * p.P * p.chunk, st);
  p.gbar.alloc(1, st);
  p.gbar.zero(1);
  if (!p.mixed) {
    // the FP64 leaf passes use the same leaf maps and near-field work items
    p.MD.xs64 = p.xs.p;
    lap_mixed_leaves(p.MD, p.tv, nb, p.dev, p.ns, p.nt, p.ndiv, st);
  }
  if (p.mixed) {
    lap_mixed_prepare(p.MD, p.xs.p, p.ns, p.xt.p, p.nt, p.fc, p.fd, p.ndc, 0.0, 0.0, p.P, st);
    p.MD.err = p.err.p;
    lap_mixed_leaves(p.MD, p.tv, nb, p.dev, p.ns, p.nt, p.ndiv, st);
    const bool levels_ok = p.dev || (T.nlevels >= 2 && T.nlevels < 64);
    if (levels_ok && m2l_tensor_cores() && m2l_tc_supported(p.P)) {
      p.MD.tc = true;
      p.MD.nlev = p.dev ? NLMAX + 3 : T.nlevels + 1;
      p.MD.nboxes = nb;
      if (p.dev)
        m2l_tc_build(p.MD.pairs, p.tv, RANGE_FROM2, nb, nb, p.P, p.chunk, st);
      else
        m2l_tc_build(p.MD.pairs, p.tv, T.lfirst[2], nb - T.lfirst[2], nb, p.P, p.chunk, st);
      if (p.MD.pairs.n > 0) p.MD.mp32.alloc(m2l_tc_scratch(p.MD.pairs, nb, p.chunk), st);
    }
  }
  device_binomials();
  device_shift_tables();
  if (p.own) {
    // the plan is evaluated on other streams: finish its construction here
    B2_CHECK(cudaStreamSynchronize(st));
    B2_CHECK(cudaEventElapsedTime(&p.tree_ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
  } else {
    // evaluated on the caller's stream right after: no wait here; the tree
    // time is read when the statistics are
    p.tree_ev[0] = e0;
    p.tree_ev[1] = e1;
  }
  *out = pl.release();
  return IER_OK;
}

int lap_plan_create(const LapArgs& a, cudaStream_t st_in, bool own_stream, LapPlan** out) {
  return lap_plan_create(a, st_in, own_stream, out, false);
}

int lap_plan_eval(LapPlan* pp, const double* charge, const double* dipstr, const double* dipvec,
                  double* pot, double* grad, double* hess, double* pottarg, double* gradtarg,
                  double* hesstarg, cudaStream_t st, bool sync, double* timeinfo) {
  return lap_plan_eval_part(pp, charge, dipstr, dipvec, pot, grad, hess, pottarg, gradtarg,
                            hesstarg, st, sync, timeinfo, 0);
}

int lap_plan_eval_part(LapPlan* pp, const double* charge, const double* dipstr,
                       const double* dipvec, double* pot, double* grad, double* hess,
                       double* pottarg, double* gradtarg, double* hesstarg, cudaStream_t st,
                       bool sync, double* timeinfo, int part) {
  if (!pp || part < 0 || part > 2) return IER_BADARG;
  if (part != 0 && !lap_plan_defers_near(pp)) return IER_BADARG;
  LapPlan& p = *pp;
  const LapArgs& a = p.a;
  if ((charge != nullptr) != p.fc || (dipstr != nullptr) != p.fd) return IER_BADARG;
  if ((a.fe == FE_LAPLACE || a.fe == FE_REAL) && dipstr && !dipvec) return IER_BADARG;
  const OutSizes o = out_sizes(p);
  if ((o.pot && !pot) || (o.grad && !grad) || (o.hess && !hess) || (o.pott && !pottarg) ||
      (o.gradt && !gradtarg) || (o.hesst && !hesstarg))
    return IER_BADARG;
  if (timeinfo)
    for (int i = 0; i < 8; i++) timeinfo[i] = 0;
  if (p.zero) {
    auto z = [&](double* d, size_t n) {
      if (n) B2_CHECK(cudaMemsetAsync(d, 0, sizeof(double) * n, st));
    };
    z(pot, o.pot);
    z(grad, o.grad);
    z(hess, o.hess);
    z(pottarg, o.pott);
    z(gradtarg, o.gradt);
    z(hesstarg, o.hesst);
    if (sync) B2_CHECK(cudaStreamSynchronize(st));
    return IER_OK;
  }
  DeviceTree& T = p.T;
  const long ns = p.ns, nt = p.nt;
  const int nd = p.nd, ndc = p.ndc, P = p.P;
  double tsum[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  // part 2: only the unpack of a near field added by the batched pass
  if (part != 2) {
  k_gather_dens<<<ceil_div(ns, 256), 256, 0, st>>>(a.fe, nd, ndc, T.isrc.p, ns, charge, dipstr,
                                                   dipvec, p.qs.p, p.ds.p);
  B2_LAUNCH_CHECK();
  if (p.mixed) lap_mixed_densities(p.MD, p.qs.p, p.ds.p, ns, ndc, st);
  if (p.dev) B2_CHECK(cudaMemsetAsync(p.gbar.p, 0, sizeof(GridBar), st));
  const MixedData* Mp = p.mixed ? &p.MD : nullptr;
  const Launch X{T.nboxes, p.dev, p.gbar.p, p.err.p,
                 p.dev ? level_hint(p.ns + p.nt, p.ndiv) : 0};
  for (int d0 = 0; d0 < ndc;) {
    int left = ndc - d0;
    int ND = left >= 8 ? 8 : (left >= 4 ? 4 : (left >= 2 ? 2 : 1));
    Dens D{p.fc ? p.qs.p : nullptr, p.fd ? p.ds.p : nullptr, ndc, d0};
    switch (ND) {
      case 8: run_chunk<8>(p.tv, T, a, D, P, p.xs.p, p.xt.p, p.mp.p, p.lo.p, p.ps.p, p.gs.p, p.hs.p, p.pt.p, p.gt.p, p.ht.p, X, st, p.ev, Mp, p.MD, part == 1); break;
      case 4: run_chunk<4>(p.tv, T, a, D, P, p.xs.p, p.xt.p, p.mp.p, p.lo.p, p.ps.p, p.gs.p, p.hs.p, p.pt.p, p.gt.p, p.ht.p, X, st, p.ev, Mp, p.MD, part == 1); break;
      case 2: run_chunk<2>(p.tv, T, a, D, P, p.xs.p, p.xt.p, p.mp.p, p.lo.p, p.ps.p, p.gs.p, p.hs.p, p.pt.p, p.gt.p, p.ht.p, X, st, p.ev, Mp, p.MD, part == 1); break;
      default: run_chunk<1>(p.tv, T, a, D, P, p.xs.p, p.xt.p, p.mp.p, p.lo.p, p.ps.p, p.gs.p, p.hs.p, p.pt.p, p.gt.p, p.ht.p, X, st, p.ev, Mp, p.MD, part == 1); break;
    }
    if (timeinfo) {
      B2_CHECK(cudaEventSynchronize(p.ev[6]));
      float ms[6];
      for (int i = 0; i < 6; i++) B2_CHECK(cudaEventElapsedTime(&ms[i], p.ev[i], p.ev[i + 1]));
      // reference buckets: 1 P2M, 2 P2L, 3 M2M, 4 M2L, 5 L2L, 6 M2P, 7 L2P, 8 P2P;
      // M2P/L2P/P2P run fused in one kernel and are reported in bucket 8.
      tsum[0] += ms[0] * 1e-3;
      tsum[2] += ms[1] * 1e-3;
      tsum[1] += ms[2] * 1e-3;
      tsum[3] += ms[3] * 1e-3;
      tsum[4] += ms[4] * 1e-3;
      if (Mp && a.ifpgh > 0) {
        // mixed path: L2P + M2P of the sources in bucket 6, the rest (their
        // near field, and the targets' far and near field) in bucket 8
        float far = 0.f, rest = 0.f;
        B2_CHECK(cudaEventElapsedTime(&far, p.ev[5], p.ev[7]));
        B2_CHECK(cudaEventElapsedTime(&rest, p.ev[7], p.ev[6]));
        tsum[5] += far * 1e-3;
        tsum[7] += rest * 1e-3;
      } else {
        tsum[7] += ms[5] * 1e-3;
      }
    }
    d0 += ND;
  }
  }
  // part 1: the near field comes from the batched pass, then part 2
  if (part == 1) return IER_OK;
  if (a.ifpgh > 0) {
    k_unpack<<<ceil_div(ns, 256), 256, 0, st>>>(a.fe, nd, ndc, a.ifpgh, p.inv_s.p, ns, p.ps.p,
                                                p.gs.p, p.hs.p, pot, grad, hess);
    B2_LAUNCH_CHECK();
  }
  if (a.ifpghtarg > 0 && nt > 0) {
    k_unpack<<<ceil_div(nt, 256), 256, 0, st>>>(a.fe, nd, ndc, a.ifpghtarg, p.inv_t.p, nt, p.pt.p,
                                                p.gt.p, p.ht.p, pottarg, gradtarg, hesstarg);
    B2_LAUNCH_CHECK();
  }
  if (p.dev) {
    k_zero_if_point_tree<<<148, 256, 0, st>>>(T.ctl.p, pot, (long)o.pot, grad, (long)o.grad,
                                              hess, (long)o.hess, pottarg, (long)o.pott, gradtarg,
                                              (long)o.gradt, hesstarg, (long)o.hesst);
    B2_LAUNCH_CHECK();
  }
  if (timeinfo)
    for (int i = 0; i < 8; i++) timeinfo[i] = tsum[i];
  if (sync) return finish(p, st);
  return IER_OK;
}

bool lap_plan_defers_near(const LapPlan* p) {
  // one density chunk (ndc 1, 2, 4 or 8), mixed precision, with a near field
  return p && p->mixed && !p->zero && p->a.ifnear &&
         (p->ndc == 1 || p->ndc == 2 || p->ndc == 4 || p->ndc == 8);
}

void lap_plan_near_entries(LapPlan* p, std::vector<P2PBatchEntry>& out) {
  if (!lap_plan_defers_near(p)) return;
  if (p->a.ifpgh > 0)
    out.push_back(P2PBatchEntry{&p->tv, &p->MD, p->xs.p, 0, p->ndc, p->ndc, p->a.ifpgh, p->ps.p,
                                p->gs.p, p->hs.p});
  if (p->nt > 0 && p->a.ifpghtarg > 0)
    out.push_back(P2PBatchEntry{&p->tv, &p->MD, p->xt.p, 1, p->ndc, p->ndc, p->a.ifpghtarg,
                                p->pt.p, p->gt.p, p->ht.p});
}

int lap_plan_status(LapPlan* p) {
  if (!p) return IER_BADARG;
  B2_CHECK(cudaDeviceSynchronize());
  return finish(*p, p->st);
}

void lap_plan_free(LapPlan* p) {
  if (!p) return;
  cudaStream_t st = p->st;
  bool own = p->own;
  if (own) cudaDeviceSynchronize();  // evaluations may have run on other streams
  delete p;                          // buffers are released on the plan's stream
  if (own) cudaStreamSynchronize(st);
}

namespace {

// One call: the plan (box ranges taken on the device when device_ranges, so
// the host does not wait for the tree), its evaluation and the end-of-call
// check.
int fmm_once(const LapArgs& a, cudaStream_t st, cudaEvent_t dens_ready, bool device_ranges,
             cudaEvent_t call0) {
  LapPlan* p = nullptr;
  int r = lap_plan_create(a, st, false, &p, device_ranges);
  if (r != IER_OK) return r;
  if (dens_ready) B2_CHECK(cudaStreamWaitEvent(st, dens_ready, 0));
  std::unique_ptr<LapPlan, void (*)(LapPlan*)> guard(p, lap_plan_free);
  const bool want_stats = g_stats_on.load();
  DBuf<unsigned long long> dstat(st);
  if (want_stats && !p->zero) {
    dstat.alloc(6, st);
    dstat.zero(6);
    k_stats<<<ceil_div(p->T.nboxes, 256), 256, 0, st>>>(p->tv, p->dev ? -1 : p->T.nboxes,
                                                        dstat.p);
    B2_LAUNCH_CHECK();
  }
  cudaEvent_t e0, e1;
  B2_CHECK(cudaEventCreate(&e0));
  B2_CHECK(cudaEventCreate(&e1));
  B2_CHECK(cudaEventRecord(e0, st));
  r = lap_plan_eval(p, a.charge, a.dipstr, a.dipvec, a.pot, a.grad, a.hess, a.pottarg, a.gradtarg,
                    a.hesstarg, st, true, a.timeinfo);
  B2_CHECK(cudaEventRecord(e1, st));
  B2_CHECK(cudaEventSynchronize(e1));
  if (want_stats && !p->zero && r == IER_OK) {
    unsigned long long hs6[6];
    B2_CHECK(cudaMemcpy(hs6, dstat.p, sizeof(hs6), cudaMemcpyDeviceToHost));
    int hn[2] = {0, 0};
    B2_CHECK(cudaMemcpy(hn, p->T.ctl.p, sizeof(hn), cudaMemcpyDeviceToHost));
    float t2 = 0;
    B2_CHECK(cudaEventElapsedTime(&t2, e0, e1));
    LapStats& S = g_last_stats;
    S.nboxes = hn[0];
    S.nlevels = hn[1];
    S.nleaves = (double)hs6[0];
    S.nterms1 = p->P;
    S.p2p_pairs = (double)hs6[1];
    S.m2l_pairs = (double)hs6[2];
    S.m2p_evals = (double)hs6[3];
    S.p2l_sources = (double)hs6[4];
    S.npts_eval = (double)hs6[5];
    if (p->tree_ev[1]) {
      B2_CHECK(cudaEventSynchronize(p->tree_ev[1]));
      B2_CHECK(cudaEventElapsedTime(&p->tree_ms, p->tree_ev[0], p->tree_ev[1]));
    }
    S.tree_ms = p->tree_ms;
    S.fmm_ms = t2;
    auto el = [](cudaEvent_t x, cudaEvent_t y) {
      float ms = 0;
      return (x && y && cudaEventElapsedTime(&ms, x, y) == cudaSuccess) ? (double)ms : -1.0;
    };
    S.tl_pre = el(call0, p->tree_ev[0]);
    S.tl_tree = el(p->tree_ev[0], p->tree_ev[1]);
    S.tl_setup = el(p->tree_ev[1], p->ev[0]);
    S.tl_fmm = el(p->ev[0], p->ev[6]);
    S.tl_post = el(p->ev[6], e1);
    S.nd_cauchy = p->ndc;
    S.m2l_tc_steps = 0;
    if (p->mixed && p->MD.tc && p->MD.pairs.steps.p) {
      unsigned long long hsteps = 0;
      B2_CHECK(cudaMemcpy(&hsteps, p->MD.pairs.steps.p, sizeof(hsteps), cudaMemcpyDeviceToHost));
      S.m2l_tc_steps = (double)hsteps;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return r;
}

// Device-wide status word of asynchronous calls: the first failure code.
int* async_word() {
  static std::mutex mu;
  static int* words[128] = {nullptr};
  int dev = 0;
  B2_CHECK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 128) throw CudaError("device ordinal beyond 127", IER_CUDA);
  std::lock_guard<std::mutex> g(mu);
  if (!words[dev]) {
    int* w = nullptr;
    B2_CHECK(cudaMalloc(&w, sizeof(int)));
    B2_CHECK(cudaMemset(w, 0, sizeof(int)));
    words[dev] = w;
  }
  return words[dev];
}

__global__ void k_fold_status(const TreeCtl* c, const int* err, int* word) {
  int code = 0;
  if (c && c->status != TB_OK)
    code = c->status == TB_TIMEOUT ? IER_TIMEOUT
                                   : (c->status == TB_BADPTS ? IER_BADARG : IER_TREE_LIMIT);
  if (!code && *err) code = IER_TIMEOUT;
  if (code) atomicCAS(word, 0, code);
}

// One call queued on `st` without any host wait: box ranges on the device,
// the outcome folded into the device's status word.
int fmm_async(const LapArgs& a, cudaStream_t st, cudaEvent_t dens_ready) {
  LapPlan* p = nullptr;
  int r = lap_plan_create(a, st, false, &p, true);
  if (r != IER_OK) return r;
  if (dens_ready) B2_CHECK(cudaStreamWaitEvent(st, dens_ready, 0));
  std::unique_ptr<LapPlan, void (*)(LapPlan*)> guard(p, lap_plan_free);
  r = lap_plan_eval(p, a.charge, a.dipstr, a.dipvec, a.pot, a.grad, a.hess, a.pottarg, a.gradtarg,
                    a.hesstarg, st, false, nullptr);
  if (r != IER_OK) return r;
  k_fold_status<<<1, 1, 0, st>>>(p->zero ? nullptr : p->T.ctl.p, p->err.p,
                                 a.status_word ? a.status_word : async_word());
  B2_LAUNCH_CHECK();
  return IER_OK;  // the plan's buffers are released stream-ordered after the call
}

}  // namespace

int lap_async_status(cudaStream_t st) {
  int* w = async_word();
  B2_CHECK(cudaStreamSynchronize(st));
  int h = 0;
  B2_CHECK(cudaMemcpy(&h, w, sizeof(int), cudaMemcpyDeviceToHost));
  if (h) B2_CHECK(cudaMemset(w, 0, sizeof(int)));
  return h;
}

// A single call does not wait for its tree on the host: the passes read
// their box ranges on the device and one check at the end of the call reads
// the outcome.  A tree that needed more boxes than the capacity guess, or
// more than 32 levels, makes the call run again with the tree read back.
int lap_fmm_device(const LapArgs& a, cudaStream_t st, cudaEvent_t dens_ready) {
  if ((a.fe == FE_LAPLACE || a.fe == FE_REAL) && a.dipstr && !a.dipvec) return IER_BADARG;
  // phase times and statistics need the host to wait: those calls are synchronous
  if (a.async_call && !a.timeinfo && !g_stats_on.load()) return fmm_async(a, st, dens_ready);
  cudaEvent_t call0 = nullptr;
  if (g_stats_on.load()) {
    B2_CHECK(cudaEventCreate(&call0));
    B2_CHECK(cudaEventRecord(call0, st));
  }
  int r = fmm_once(a, st, dens_ready, g_device_ranges.load(), call0);
  if (r == IER_RETRY) r = fmm_once(a, st, nullptr, false, call0);
  if (call0) cudaEventDestroy(call0);
  return r;
}

void set_device_ranges(bool on) { g_device_ranges.store(on); }

}  // namespace b2
