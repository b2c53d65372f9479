// Mixed-precision Laplace kernels (eps >= 1e-6).
//
// * k_m2l_f32: the M2L of laprouts2d.f:1130-1244 in FP32.  Boxes of one
//   level are translated by integer offsets o (|o|_inf in 2..3) in units of
//   the box size, so u = r/z0 = 1/o and log|z0| = log r + log|o| come from
//   49-entry tables; per translation only the gather of the source
//   multipole (FP64 -> FP32) and the fixed matrix G(i,j) = C(i+j-1, j-1)
//   remain.  Local expansions are accumulated in FP32 per target box and
//   added to the FP64 expansion once.
// * k_far_mixed: L2P and M2P in FP64 (as the FP64 path), one evaluation
//   point per thread.
// * k_p2p_leaf: the near field in FP32, per work item (up to 32 evaluation
//   points of one leaf) over sources staged in shared memory as two-float
//   offsets from the leaf centre, so a pair difference keeps the relative
//   accuracy of an FP64 difference even for nearly coincident points
//   (separations of 1e-12 occur in graded distributions); log and 1/r^2 use
//   the SFU.  Per-pair terms are summed in FP32 over at most 32 sources and
//   the partial sums in FP64.
#include "lap_mixed.cuh"

#include <atomic>
#include <memory>
#include <cstddef>
#include <type_traits>
#include "laplace.cuh"

namespace b2 {

namespace {

using namespace lapk;

__global__ void k_prep_dens(const double2* __restrict__ in, long m, float2* __restrict__ out) {
  long k = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (k < m) out[k] = make_float2((float)in[k].x, (float)in[k].y);
}

// utab[o][k] = (1/o)^k for o = (ox, oy), ox, oy in -3..3; lgtab[o] = log|o|
__global__ void k_utab(int P, float2* utab, float* lgtab) {
  int i = blockIdx.x, k = threadIdx.x;
  int ox = i / 7 - 3, oy = i % 7 - 3;
  if (k >= P) return;
  if (ox == 0 && oy == 0) {
    utab[i * P + k] = make_float2(0.f, 0.f);
    if (k == 0) lgtab[i] = 0.f;
    return;
  }
  double2 u = crcp(make_double2((double)ox, (double)oy));
  double2 p = cpow_int(u, k);
  utab[i * P + k] = make_float2((float)p.x, (float)p.y);
  if (k == 0) lgtab[i] = (float)log(hypot((double)ox, (double)oy));
}

__device__ __forceinline__ float2 cmulf_(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ void cfmaf_(float2& a, float2 b, float2 c) {
  a.x = fmaf(b.x, c.x, fmaf(-b.y, c.y, a.x));
  a.y = fmaf(b.x, c.y, fmaf(b.y, c.x, a.y));
}

// Register-tiled FP32 M2L.  Per target box (one warp) and translation e:
// y = G t_e with t_e(j) = h_j (-u)^j, u = 1/o, followed by L_i += u^i y_i
// (L_0 += y_0 + t_0 log|z0|).  Lane = (row block rb of 4 rows, translation
// group eg): the warp takes EG translations at a time; each lane multiplies
// its 4 rows of G (a float4 per j from shared memory) with the 2*ND real
// columns of its translation (one broadcast load per j), i.e. 8*ND FMAs per
// two shared loads.  Partial locals of the EG groups are summed through
// shared memory at the end of the box.
template <int ND>
__global__ void __launch_bounds__(128) k_m2l_f32(TV t, int first, int n, int P, int RB, int EG,
                                                 const double* __restrict__ binom,
                                                 const float2* __restrict__ utab_g,
                                                 const float* __restrict__ lgtab_g,
                                                 const double2* __restrict__ mp,
                                                 double2* __restrict__ lo) {
  extern __shared__ float4 sm4[];
  const int CW = 2 * ND;  // real columns per translation
  // per-warp scratch first (16-byte aligned blocks), then the tables
  const size_t warp_floats = (size_t)EG * P * CW * 2 + ((2 * EG + 3) & ~3);
  float* wbase = (float*)sm4;
  float4* G4 = (float4*)(wbase + 4 * warp_floats);  // [P][RB]: rows 4rb..4rb+3 of column j
  float2* U = (float2*)(G4 + (size_t)P * RB);      // [49][P]
  float* LG = (float*)(U + 49 * P);                // [49]
  resolve_range(t, first, n);
  for (int e = threadIdx.x; e < P * RB * 4; e += blockDim.x) {
    int j = e / (RB * 4), i = e % (RB * 4);
    float g = 0.f;
    if (i < P) {
      if (i == 0)
        g = (j == 0) ? 0.f : 1.f;
      else if (j == 0)
        g = -1.f / i;
      else
        g = (float)binom[(size_t)(i + j - 1) * BINOM_N + (j - 1)];
    }
    ((float*)G4)[e] = g;
  }
  for (int e = threadIdx.x; e < 49 * P; e += blockDim.x) U[e] = utab_g[e];
  for (int e = threadIdx.x; e < 49; e += blockDim.x) LG[e] = lgtab_g[e];
  __syncthreads();
  WARP_LOOP(n) {
    float* Tw = wbase + (size_t)wib * warp_floats;   // [EG][P][CW]
    float* Rw = Tw + (size_t)EG * P * CW;            // [EG][P][CW] partial locals
    int* OI = (int*)(Rw + (size_t)EG * P * CW);      // [EG] offsets
    float* LGE = (float*)(OI + EG);                  // [EG] log|z0|
    int b = first + bi;
    int n2 = t.nl2[b];
    if (n2 == 0 || !t.has_eval_pts(b)) continue;
    double r = t.boxsize[t.level[b]];
    double2 cb = t.center[b];
    float lgr = (float)log(r);
    double rinv = 1.0 / r;
    const int rb = lane % RB, eg = lane / RB;
    const bool act = eg < EG;
    float acc[4][2 * ND];
#pragma unroll
    for (int q = 0; q < 4; q++)
#pragma unroll
      for (int c = 0; c < 2 * ND; c++) acc[q][c] = 0.f;
    for (int e0 = 0; e0 < n2; e0 += EG) {
      int cnt = min(EG, n2 - e0);
      __syncwarp();
      if (lane < cnt) {
        int jb = t.l2[(size_t)MNLIST2 * b + e0 + lane];
        double2 cj = t.center[jb];
        int ox = __double2int_rn((cj.x - cb.x) * rinv), oy = __double2int_rn((cj.y - cb.y) * rinv);
        int oi = (ox + 3) * 7 + (oy + 3);
        OI[lane] = oi;
        LGE[lane] = lgr + LG[oi];
      }
      __syncwarp();
      // gather t_e(j) = h_j (-u)^j in FP32
      for (int k = lane; k < cnt * P * ND; k += 32) {
        int e = k / (P * ND), rem = k % (P * ND), j = rem / ND, d = rem % ND;
        int jb = t.l2[(size_t)MNLIST2 * b + e0 + e];
        float2 sj = U[OI[e] * P + j];
        if (j & 1) sj = make_float2(-sj.x, -sj.y);
        double2 h = mp[((size_t)jb * P + j) * ND + d];
        float2 v = cmulf_(make_float2((float)h.x, (float)h.y), sj);
        Tw[((size_t)e * P + j) * CW + 2 * d] = v.x;
        Tw[((size_t)e * P + j) * CW + 2 * d + 1] = v.y;
      }
      __syncwarp();
      if (act && eg < cnt) {
        float y[4][2 * ND];
#pragma unroll
        for (int q = 0; q < 4; q++)
#pragma unroll
          for (int c = 0; c < 2 * ND; c++) y[q][c] = 0.f;
        const float* Te = Tw + (size_t)eg * P * CW;
        for (int j = 0; j < P; j++) {
          float4 g = G4[j * RB + rb];
          float tv[2 * ND];
          if (ND % 2 == 0) {
#pragma unroll
            for (int c = 0; c < ND / 2; c++) {
              float4 v4 = ((const float4*)(Te + j * CW))[c];
              tv[4 * c] = v4.x;
              tv[4 * c + 1] = v4.y;
              tv[4 * c + 2] = v4.z;
              tv[4 * c + 3] = v4.w;
            }
          } else {
#pragma unroll
            for (int c = 0; c < ND; c++) {
              float2 v2 = ((const float2*)(Te + j * CW))[c];
              tv[2 * c] = v2.x;
              tv[2 * c + 1] = v2.y;
            }
          }
#pragma unroll
          for (int c = 0; c < 2 * ND; c++) {
            y[0][c] = fmaf(g.x, tv[c], y[0][c]);
            y[1][c] = fmaf(g.y, tv[c], y[1][c]);
            y[2][c] = fmaf(g.z, tv[c], y[2][c]);
            y[3][c] = fmaf(g.w, tv[c], y[3][c]);
          }
        }
        const int oi = OI[eg];
        const float lge = LGE[eg];
#pragma unroll
        for (int q = 0; q < 4; q++) {
          int i = 4 * rb + q;
          if (i >= P) break;
          if (i == 0) {
#pragma unroll
            for (int d = 0; d < ND; d++) {
              acc[q][2 * d] += y[q][2 * d] + Te[2 * d] * lge;
              acc[q][2 * d + 1] += y[q][2 * d + 1] + Te[2 * d + 1] * lge;
            }
          } else {
            float2 ui = U[oi * P + i];
#pragma unroll
            for (int d = 0; d < ND; d++) {
              float yr = y[q][2 * d], yi = y[q][2 * d + 1];
              acc[q][2 * d] += yr * ui.x - yi * ui.y;
              acc[q][2 * d + 1] += yr * ui.y + yi * ui.x;
            }
          }
        }
      }
    }
    // sum the translation groups and add to the FP64 local expansion
    __syncwarp();
    if (act) {
#pragma unroll
      for (int q = 0; q < 4; q++) {
        int i = 4 * rb + q;
        if (i >= P) break;
#pragma unroll
        for (int c = 0; c < 2 * ND; c++) Rw[((size_t)eg * P + i) * CW + c] = acc[q][c];
      }
    }
    __syncwarp();
    for (int k = lane; k < P * ND; k += 32) {
      int i = k / ND, d = k % ND;
      float sr = 0.f, si = 0.f;
      for (int g = 0; g < EG; g++) {
        sr += Rw[((size_t)g * P + i) * CW + 2 * d];
        si += Rw[((size_t)g * P + i) * CW + 2 * d + 1];
      }
      size_t o = ((size_t)b * P + i) * ND + d;
      double2 cur = lo[o];
      lo[o] = make_double2(cur.x + sr, cur.y + si);
    }
  }
}

// Leaf box of every evaluation point (points are in tree order).
__global__ void k_point_leaf(TV t, int nb, int use_targets, int* __restrict__ leaf) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (nb < 0) {
    int f = RANGE_ALL;
    resolve_range(t, f, nb);
  }
  if (b >= nb || t.nchild[b] != 0) return;
  int2 r = use_targets ? t.trng[b] : t.srng[b];
  for (int k = r.x; k < r.y; k++) leaf[k] = b;
}

// Blocks of 128 threads per SM asked of the register allocator for the far
// field: 8 (at most 64 registers a thread) for one or two densities without
// hessians, where the extra warps hide the coefficient loads (leaf phase
// 2.59 -> 2.50 ms at 4M points); the compiler's choice otherwise.
#define FAR_MIN_BLOCKS(ND, IFPGH) ((ND) <= 2 && (IFPGH) <= 2 ? 8 : 1)

// Far field of one evaluation point per thread, FP64: L2P from the local
// expansion of its leaf and M2P from the leaf's list-3 boxes (the
// coefficients of one box are shared by the neighbouring threads of the same
// leaf through the L1 cache).  Writes pot / grad / hess of the point.
template <int ND, int IFPGH>
__global__ void __launch_bounds__(128, FAR_MIN_BLOCKS(ND, IFPGH)) k_far_mixed(
    TV t, long n, const int* __restrict__ leaf, const double2* __restrict__ xe64, int ndc, int d0,
    int P, const double2* __restrict__ mp, const double2* __restrict__ lo,
    double2* __restrict__ pot, double2* __restrict__ grad, double2* __restrict__ hess) {
  long k = blockIdx.x * (long)blockDim.x + threadIdx.x;
  // after a failed tree build the leaf map is not written
  if (k >= n || t.ctl->status != TB_OK) return;
  const int b = leaf[k];
  const int lev = t.level[b];
  const double r = t.boxsize[lev];
  const double2 cb = t.center[b];
  const double2 z = xe64[k];
  double2 pt[ND], gr[ND], hs[ND];
  {
    // L2P: sum_m L_m ((z - c) / r)^m and derivatives (Horner)
    const double2* L = lo + (size_t)b * P * ND;
    double2 zz = make_double2((z.x - cb.x) / r, (z.y - cb.y) / r);
    double2 f[ND], f1[ND], f2[ND];
#pragma unroll
    for (int d = 0; d < ND; d++) {
      f[d] = L[(P - 1) * ND + d];
      f1[d] = f2[d] = make_double2(0, 0);
    }
    // Horner steps in groups of four whose coefficient loads are issued
    // together (one load latency per group instead of per step)
    auto step = [&](const double2 (&c)[ND]) {
#pragma unroll
      for (int d = 0; d < ND; d++) {
        if (IFPGH >= 3) f2[d] = cadd(cmul(f2[d], zz), f1[d]);
        if (IFPGH >= 2) f1[d] = cadd(cmul(f1[d], zz), f[d]);
        f[d] = cadd(cmul(f[d], zz), c[d]);
      }
    };
    int m = P - 2;
    for (; m >= 3; m -= 4) {
      double2 c0[ND], c1[ND], c2[ND], c3[ND];
#pragma unroll
      for (int d = 0; d < ND; d++) {
        c0[d] = L[m * ND + d];
        c1[d] = L[(m - 1) * ND + d];
        c2[d] = L[(m - 2) * ND + d];
        c3[d] = L[(m - 3) * ND + d];
      }
      step(c0);
      step(c1);
      step(c2);
      step(c3);
    }
    for (; m >= 0; m--) {
      double2 c0[ND];
#pragma unroll
      for (int d = 0; d < ND; d++) c0[d] = L[m * ND + d];
      step(c0);
    }
    double ri = 1.0 / r;
#pragma unroll
    for (int d = 0; d < ND; d++) {
      pt[d] = f[d];
      gr[d] = IFPGH >= 2 ? cscale(f1[d], ri) : make_double2(0, 0);
      hs[d] = IFPGH >= 3 ? cscale(f2[d], 2.0 * ri * ri) : make_double2(0, 0);
    }
  }
  const int n3 = t.nl3[b];
  for (int e = 0; e < n3; e++) {
    // M2P: c_0 log(z - c) + sum_{m>=1} c_m (r_j / (z - c))^m
    int jb = t.l3[(size_t)MNLIST3 * b + e];
    const double2* M = mp + (size_t)jb * P * ND;
    double rj = t.boxsize[lev + 1];
    double2 cj = t.center[jb];
    double2 zc = make_double2(z.x - cj.x, z.y - cj.y);
    double2 zi = crcp(zc);
    double2 w = make_double2(rj * zi.x, rj * zi.y);
    double lg = log(hypot(zc.x, zc.y));
    double2 f[ND], f1[ND], f2[ND];
#pragma unroll
    for (int d = 0; d < ND; d++) {
      f[d] = M[(P - 1) * ND + d];
      f1[d] = f2[d] = make_double2(0, 0);
    }
    auto mstep = [&](const double2 (&c)[ND]) {
#pragma unroll
      for (int d = 0; d < ND; d++) {
        if (IFPGH >= 3) f2[d] = cadd(cmul(f2[d], w), f1[d]);
        if (IFPGH >= 2) f1[d] = cadd(cmul(f1[d], w), f[d]);
        f[d] = cadd(cmul(f[d], w), c[d]);
      }
    };
    int m = P - 2;
    for (; m >= 4; m -= 4) {
      double2 c0[ND], c1[ND], c2[ND], c3[ND];
#pragma unroll
      for (int d = 0; d < ND; d++) {
        c0[d] = M[m * ND + d];
        c1[d] = M[(m - 1) * ND + d];
        c2[d] = M[(m - 2) * ND + d];
        c3[d] = M[(m - 3) * ND + d];
      }
      mstep(c0);
      mstep(c1);
      mstep(c2);
      mstep(c3);
    }
    for (; m >= 1; m--) {
      double2 c0[ND];
#pragma unroll
      for (int d = 0; d < ND; d++) c0[d] = M[m * ND + d];
      mstep(c0);
    }
    double2 w2 = cmul(w, w);
#pragma unroll
    for (int d = 0; d < ND; d++) {
      double2 c0 = M[d];
      double2 Sv = cmul(w, f[d]);
      double2 S1 = cadd(f[d], cmul(w, f1[d]));
      pt[d].x += Sv.x + c0.x * lg;
      pt[d].y += Sv.y + c0.y * lg;
      if (IFPGH >= 2) {
        double2 gg = cmul(S1, w2);
        gg = make_double2(-gg.x / rj, -gg.y / rj);
        gr[d] = cadd(gr[d], cadd(gg, cmul(c0, zi)));
      }
      if (IFPGH >= 3) {
        double2 S2 = cscale(cadd(f1[d], cmul(w, f2[d])), 2.0);
        double2 w3 = cmul(w2, w), w4 = cmul(w2, w2);
        double2 h = cadd(cmul(S2, w4), cscale(cmul(S1, w3), 2.0));
        h = cscale(h, 1.0 / (rj * rj));
        hs[d] = cadd(hs[d], csub(h, cmul(c0, cmul(zi, zi))));
      }
    }
  }
#pragma unroll
  for (int d = 0; d < ND; d++) {
    size_t o = (size_t)k * ndc + d0 + d;
    pot[o] = pt[d];
    if (IFPGH >= 2) grad[o] = gr[d];
    if (IFPGH >= 3) hess[o] = hs[d];
  }
}

// Tile shapes of the near-field pass (k_p2p_leaf), chosen per leaf-size
// class by the autotuner (fmm2d_b200/autotune.py, b2fmm_set_p2p_shape):
// sources staged per warp and chunk, unrolling of the pair loop, and the
// resident blocks of 128 threads per SM asked of the register allocator
// (for one or two densities without hessians; the compiler's choice and
// shape 0 otherwise).
struct P2PShape {
  int chunk, unroll, min_blocks;
};
constexpr P2PShape P2P_SHAPES[] = {{128, 2, 6}, {64, 2, 8}, {128, 4, 5}};
constexpr int P2P_NSHAPES = 3;
static_assert(P2P_NSHAPES == B2FMM_P2P_SHAPES, "shape table and C ABI agree");
constexpr bool p2p_tuned(int ND, int IFPGH) { return ND <= 2 && IFPGH <= 2; }
#define P2P_MIN_BLOCKS(ND, IFPGH, V) (p2p_tuned(ND, IFPGH) ? P2P_SHAPES[V].min_blocks : 1)

// Far field of the mixed path in FP32, one evaluation point per thread:
// L2P from the leaf's local expansion (FP64, rounded to FP32 on load) and
// M2P from the FP32 copy of the multipoles that the tensor-core M2L makes
// (mp32: [box][ND][KH] complex, zero beyond P).  Point-to-centre
// differences are formed in FP64 and rounded once; Horner, the complex
// reciprocal and log|z - c| (SFU) in FP32; the sums go to FP64 outputs.
// Relative error ~1e-7 of the far field, below the eps >= 1e-6 the mixed
// path serves.  Writes pot / grad / hess of the point.
__device__ __forceinline__ float2 f2_(double2 a) { return make_float2((float)a.x, (float)a.y); }
__device__ __forceinline__ float2 caddf_(float2 a, float2 b) {
  return make_float2(a.x + b.x, a.y + b.y);
}
__device__ __forceinline__ float2 cmaf_(float2 a, float2 b, float2 c) {  // a b + c
  return make_float2(fmaf(a.x, b.x, fmaf(-a.y, b.y, c.x)), fmaf(a.x, b.y, fmaf(a.y, b.x, c.y)));
}

template <int ND, int IFPGH>
__global__ void __launch_bounds__(128, FAR_MIN_BLOCKS(ND, IFPGH)) k_far_f32(
    TV t, long n, const int* __restrict__ leaf, const double2* __restrict__ xe64, int ndc, int d0,
    int P, int KH, const float2* __restrict__ mp32, const double2* __restrict__ lo,
    double2* __restrict__ pot, double2* __restrict__ grad, double2* __restrict__ hess) {
  long k = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (k >= n || t.ctl->status != TB_OK) return;
  const int b = leaf[k];
  const int lev = t.level[b];
  const double r = t.boxsize[lev];
  const double2 cb = t.center[b];
  const double2 z = xe64[k];
  float2 pt[ND], gr[ND], hs[ND];
  {
    const double2* L = lo + (size_t)b * P * ND;
    const double ri = 1.0 / r;
    const float2 zz = make_float2((float)((z.x - cb.x) * ri), (float)((z.y - cb.y) * ri));
    float2 f[ND], f1[ND], f2[ND];
#pragma unroll
    for (int d = 0; d < ND; d++) {
      f[d] = f2_(L[(P - 1) * ND + d]);
      f1[d] = f2[d] = make_float2(0.f, 0.f);
    }
    auto step = [&](const float2 (&c)[ND]) {
#pragma unroll
      for (int d = 0; d < ND; d++) {
        if (IFPGH >= 3) f2[d] = cmaf_(f2[d], zz, f1[d]);
        if (IFPGH >= 2) f1[d] = cmaf_(f1[d], zz, f[d]);
        f[d] = cmaf_(f[d], zz, c[d]);
      }
    };
    int m = P - 2;
    for (; m >= 3; m -= 4) {
      float2 c0[ND], c1[ND], c2[ND], c3[ND];
#pragma unroll
      for (int d = 0; d < ND; d++) {
        c0[d] = f2_(L[m * ND + d]);
        c1[d] = f2_(L[(m - 1) * ND + d]);
        c2[d] = f2_(L[(m - 2) * ND + d]);
        c3[d] = f2_(L[(m - 3) * ND + d]);
      }
      step(c0);
      step(c1);
      step(c2);
      step(c3);
    }
    for (; m >= 0; m--) {
      float2 c0[ND];
#pragma unroll
      for (int d = 0; d < ND; d++) c0[d] = f2_(L[m * ND + d]);
      step(c0);
    }
    const float rif = (float)ri;
#pragma unroll
    for (int d = 0; d < ND; d++) {
      pt[d] = f[d];
      gr[d] = IFPGH >= 2 ? make_float2(f1[d].x * rif, f1[d].y * rif) : make_float2(0.f, 0.f);
      hs[d] = IFPGH >= 3 ? make_float2(f2[d].x * 2.f * rif * rif, f2[d].y * 2.f * rif * rif)
                         : make_float2(0.f, 0.f);
    }
  }
  const int n3 = t.nl3[b];
  const float rj = (float)t.boxsize[lev + 1], irj = 1.f / rj;
  for (int e = 0; e < n3; e++) {
    // M2P: c_0 log(z - c) + sum_{m>=1} c_m (r_j / (z - c))^m
    const int jb = t.l3[(size_t)MNLIST3 * b + e];
    const double2 cj = t.center[jb];
    const float2 zc = make_float2((float)(z.x - cj.x), (float)(z.y - cj.y));
    const float q2 = fmaf(zc.x, zc.x, zc.y * zc.y);
    const float iq = __fdividef(1.f, q2);
    const float2 zi = make_float2(zc.x * iq, -zc.y * iq);
    const float2 w = make_float2(rj * zi.x, rj * zi.y);
    const float lg = 0.5f * __logf(q2);
    const float2* M = mp32 + (size_t)jb * ND * KH;
    float2 f[ND], f1[ND], f2[ND];
#pragma unroll
    for (int d = 0; d < ND; d++) {
      f[d] = M[d * KH + P - 1];
      f1[d] = f2[d] = make_float2(0.f, 0.f);
    }
    auto mstep = [&](const float2 (&c)[ND]) {
#pragma unroll
      for (int d = 0; d < ND; d++) {
        if (IFPGH >= 3) f2[d] = cmaf_(f2[d], w, f1[d]);
        if (IFPGH >= 2) f1[d] = cmaf_(f1[d], w, f[d]);
        f[d] = cmaf_(f[d], w, c[d]);
      }
    };
    int m = P - 2;
    for (; m >= 4; m -= 4) {
      float2 c0[ND], c1[ND], c2[ND], c3[ND];
#pragma unroll
      for (int d = 0; d < ND; d++) {
        c0[d] = M[d * KH + m];
        c1[d] = M[d * KH + m - 1];
        c2[d] = M[d * KH + m - 2];
        c3[d] = M[d * KH + m - 3];
      }
      mstep(c0);
      mstep(c1);
      mstep(c2);
      mstep(c3);
    }
    for (; m >= 1; m--) {
      float2 c0[ND];
#pragma unroll
      for (int d = 0; d < ND; d++) c0[d] = M[d * KH + m];
      mstep(c0);
    }
    const float2 w2 = cmulf_(w, w);
#pragma unroll
    for (int d = 0; d < ND; d++) {
      const float2 c0 = M[d * KH];
      const float2 Sv = cmulf_(w, f[d]);
      const float2 S1 = caddf_(f[d], cmulf_(w, f1[d]));
      pt[d].x += Sv.x + c0.x * lg;
      pt[d].y += Sv.y + c0.y * lg;
      if (IFPGH >= 2) {
        const float2 gg = cmulf_(S1, w2);
        gr[d] = caddf_(gr[d], caddf_(make_float2(-gg.x * irj, -gg.y * irj), cmulf_(c0, zi)));
      }
      if (IFPGH >= 3) {
        const float2 S2p = caddf_(f1[d], cmulf_(w, f2[d]));
        const float2 S2 = make_float2(2.f * S2p.x, 2.f * S2p.y);
        const float2 w3 = cmulf_(w2, w), w4 = cmulf_(w2, w2);
        const float2 S1w3 = cmulf_(S1, w3);
        float2 hh = caddf_(cmulf_(S2, w4), make_float2(2.f * S1w3.x, 2.f * S1w3.y));
        hh = make_float2(hh.x * irj * irj, hh.y * irj * irj);
        const float2 c0zz = cmulf_(c0, cmulf_(zi, zi));
        hs[d] = caddf_(hs[d], make_float2(hh.x - c0zz.x, hh.y - c0zz.y));
      }
    }
  }
#pragma unroll
  for (int d = 0; d < ND; d++) {
    const size_t o = (size_t)k * ndc + d0 + d;
    pot[o] = make_double2(pt[d].x, pt[d].y);
    if (IFPGH >= 2) grad[o] = make_double2(gr[d].x, gr[d].y);
    if (IFPGH >= 3) hess[o] = make_double2(hs[d].x, hs[d].y);
  }
}

// Grid of a persistent pass: every SM filled with as many blocks as fit.
template <typename K>
int resident_grid(K kernel, int threads, size_t smem) {
  static std::mutex mu;
  static std::vector<std::pair<std::pair<const void*, int>, int>> done;
  int dev = 0;
  B2_CHECK(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> g(mu);
  for (auto& e : done)
    if (e.first.first == (const void*)kernel && e.first.second == dev) return e.second;
  int nsm = 0, per = 0;
  B2_CHECK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  B2_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, threads, smem));
  const int grid = std::max(1, per) * nsm;
  done.push_back({{(const void*)kernel, dev}, grid});
  return grid;
}

// Near field of the mixed path, FP32 (cauchykernels2d.f c2d_directcdg and
// relatives), one warp per work item of up to 32 evaluation points of one
// leaf box (the item list is built once per tree by k_p2p_items; warps take
// items in turn).  The warp stages the union of the item's list-1 sources in
// shared memory, up to 128 at a time, as offsets from the leaf
// centre scaled by a power of two 2^-e close to 1/(box size): x = hi + lo,
// two floats (48 significant bits of an offset of a few box sizes).  A pair
// difference is (zh - sh) + (zl - sl), with an absolute error of ~2^-46 in
// these units.  Pairs closer than 2^-20 box sizes (rare, but graded
// distributions have them) add nothing in the branch-free pass; the target's
// lane forms them after it as an FP64 difference of the input coordinates
// rounded once, so nearly coincident points keep the relative accuracy of
// the FP64 difference, and skips the pair of a point with itself by index.
// Lane = (target ti, source phase ph): the warp takes
// the item's ntc targets, 32 / ntc phases each, and the phases of one
// target are summed by shuffles at the end.
// Terms use the scaled geometry: log r = log r' + e ln 2, 1/z = 2^-e / z'
// (dipole strengths are staged times 2^-e, gradients and hessians scaled
// once per target).
// Per-pair terms are summed in FP32 over at most 32 sources, those partial
// sums in FP64, and added to the far field already in the outputs.  KIND: 1
// charges, 2 dipoles, 3 both.
static_assert(MNLIST1 <= 16, "list-1 search below covers 16 boxes");

__device__ __forceinline__ void split_hilo(double x, float& hi, float& lo) {
  hi = __double2float_rn(x);
  lo = __double2float_rn(x - (double)hi);
}

// One staged source: scaled offset (hi x, hi y, lo x, lo y), then its
// charges and dipole strengths (KIND decides which are present).
template <int ND, int KIND>
struct P2PSrc {
  float4 p;
  float2 c[ND * ((KIND & 1) + ((KIND >> 1) & 1))];
};

// A near-field work item (see k_p2p_items).
struct P2PItem {
  int b, k0, meta, ex;  // box, first point, points | list-1 length << 8, exponent
  int S, pad0, pad1, pad2;  // sources in the list-1 boxes
  double2 c;            // box centre
  int lst[16];          // list-1 source range starts
  int lpre[16];         // exclusive prefix of the range lengths
};

static_assert(offsetof(P2PItem, lpre) == offsetof(P2PItem, lst) + 16 * sizeof(int),
              "lst and lpre are read as 32 consecutive ints");

// Shared memory of one warp: staged sources and one leaf's list-1 ranges.
template <int ND, int KIND, int CH>
struct P2PWarp {
  P2PSrc<ND, KIND> s[CH];
  int lst[16];   // list-1 source range starts
  int lpre[16];  // exclusive prefix of the list-1 range lengths (follows lst)
};
using P2PWarp11 = P2PWarp<1, 1, 64>;
static_assert(offsetof(P2PWarp11, lpre) == offsetof(P2PWarp11, lst) + 16 * sizeof(int),
              "lst and lpre are written as 32 consecutive ints");

// Near-field work items of one tree, ceil(n / 32) per leaf box with n
// evaluation points, written once per tree (appended in any order; count[0]
// ends as the number of items).  An item holds everything the pass needs
// before it stages sources: the box, its first point and point count, the
// list-1 length, the binary exponent of the box size, the centre, and the
// source ranges of the list-1 boxes with their exclusive prefix.
__global__ void k_p2p_items(TV t, int nb, int use_targets, P2PItem* __restrict__ items,
                            int* __restrict__ count) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (nb < 0) {
    int f = RANGE_ALL;
    resolve_range(t, f, nb);
  }
  int ni = 0;
  int2 tr = make_int2(0, 0);
  if (b < nb && t.nchild[b] == 0) {
    tr = use_targets ? t.trng[b] : t.srng[b];
    ni = tr.y > tr.x ? (tr.y - tr.x + 31) / 32 : 0;
  }
  // one atomic per warp
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  int inc = ni;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int v = __shfl_up_sync(FULL, inc, o);
    if (lane >= o) inc += v;
  }
  int base = 0;
  if (lane == 31 && inc > 0) base = atomicAdd(count, inc);
  base = __shfl_sync(FULL, base, 31) + inc - ni;
  if (ni == 0) return;
  P2PItem it;
  int ex = 0;
  frexp(t.boxsize[t.level[b]], &ex);
  const int n1 = t.nl1[b];
  it.b = b;
  it.ex = ex;
  it.c = t.center[b];
  int S = 0;
  for (int e = 0; e < 16; e++) {
    int2 r = make_int2(0, 0);
    if (e < n1) r = t.srng[t.l1[(size_t)MNLIST1 * b + e]];
    it.lst[e] = r.x;
    it.lpre[e] = S;
    S += r.y - r.x;
  }
  it.S = S;
  it.pad0 = it.pad1 = it.pad2 = 0;
  const int nt = tr.y - tr.x;
  for (int i = 0; i < ni; i++) {
    it.k0 = tr.x + 32 * i;
    it.meta = min(32, nt - 32 * i) | (n1 << 8);
    items[base + i] = it;
  }
}

// One near-field job: the work items of one tree with the arrays they read
// and the outputs they add to (k_p2p_leaf takes one, k_p2p_batch many).
struct P2PJob {
  const TreeCtl* ctl;     // tree status (no items after a failed build)
  const double* bs;       // box sizes (bs[0]: the root, for the default threshold)
  const double2* xs64;    // sorted sources
  const double2* xe64;    // sorted evaluation points
  const float2* q32;      // FP32 charges, ndc per point, or null
  const float2* d32;      // FP32 dipole strengths or null
  const P2PItem* items;
  const int* nitems;
  double2 *pot, *grad, *hess;  // tree-order outputs (added to)
  double thresh;          // < 0: boxsize(0) 2^-51
  int ndc, d0, self_pairs, pad;
};

// The near field of one work item (the body of k_p2p_leaf and k_p2p_batch).
template <int ND, int IFPGH, int KIND, int V>
__device__ __forceinline__ void p2p_item(const P2PJob& J, const P2PItem& I,
                                         P2PWarp<ND, KIND, P2P_SHAPES[V].chunk>& W, int lane) {
  constexpr bool HQ = KIND & 1, HD = (KIND >> 1) & 1;
  constexpr int DOFF = HQ ? ND : 0;  // first dipole entry of a staged source
  constexpr unsigned FULL = 0xffffffffu;
  constexpr int CH = P2P_SHAPES[V].chunk, UNROLL = P2P_SHAPES[V].unroll;
  const double thr = J.thresh >= 0 ? J.thresh : J.bs[0] * 0x1p-51;
  // the previous item's lanes are done with the list-1 ranges (its close
  // pairs read them after the last chunk)
  __syncwarp();
  // the list-1 ranges and their prefix: 32 consecutive ints, one a lane
  ((int*)W.lst)[lane] = ((const int*)I.lst)[lane];
  const int4 h = *(const int4*)&I;
  const int n1 = h.z >> 8, ntc = h.z & 255, ex = h.w;
  const int S = I.S;
  const double2 c = I.c;
  // 32 / ntc and lane / ntc by a float reciprocal (exact: the quotients
  // are at least 1/64 away from the next integer)
  const float rn = __frcp_rn((float)ntc);
  const int nph = __float2int_rz(32.5f * rn);
  const int ph = __float2int_rz(((float)lane + 0.5f) * rn), ti = lane - ph * ntc;
  const bool act = ph < nph;
  const long k = (long)h.y + ti;
  const double sc = __hiloint2double((1023 - ex) << 20, 0);  // 2^-ex
  const float scf = (float)sc;
  const double ts = thr * sc;
  const float th2 = (float)(ts * ts);
  // pairs below this squared distance take the careful path (FP64
  // difference, exclusion test)
  const float rslow = fmaxf(0x1p-40f, 2.f * th2);
  const float lsc = (float)((double)ex * 0.69314718055994530942);
  __syncwarp();
  // at most 32 sources per lane and chunk: one FP32 partial sum each
  const int cap = min(CH, 32 * nph);
  float2 zh, zl;
  {
    const double2 z = J.xe64[k];
    split_hilo((z.x - c.x) * sc, zh.x, zl.x);
    split_hilo((z.y - c.y) * sc, zh.y, zl.y);
  }
  double2 pt[ND], gr[ND], hs[ND];
#pragma unroll
  for (int d = 0; d < ND; d++) pt[d] = gr[d] = hs[d] = make_double2(0, 0);
  int nslow = 0;
  for (int u0 = 0; u0 < S; u0 += cap) {
    const int m = min(cap, S - u0);
    for (int i = lane; i < m; i += 32) {
      // the list-1 box of source u: the last e with lpre[e] <= u
      const int u = u0 + i;
      int e = 0;
#pragma unroll
      for (int step = 8; step > 0; step >>= 1)
        if (e + step < n1 && W.lpre[e + step] <= u) e += step;
      const int j = W.lst[e] + (u - W.lpre[e]);
      const double2 sxy = J.xs64[j];
      P2PSrc<ND, KIND>& R = W.s[i];
      float4 p;
      split_hilo((sxy.x - c.x) * sc, p.x, p.z);
      split_hilo((sxy.y - c.y) * sc, p.y, p.w);
      R.p = p;
      const size_t o = (size_t)j * J.ndc + J.d0;
#pragma unroll
      for (int d = 0; d < ND; d++) {
        if (HQ) R.c[d] = J.q32[o + d];
        if (HD) {
          const float2 v = J.d32[o + d];
          R.c[DOFF + d] = make_float2(v.x * scf, v.y * scf);
        }
      }
    }
    __syncwarp();
    if (act) {
      float2 fp[ND], fg[ND], fh[ND];
#pragma unroll
      for (int d = 0; d < ND; d++) fp[d] = fg[d] = fh[d] = make_float2(0.f, 0.f);
      // branch-free pairs: a pair closer than rslow (the pair of a point
      // with itself, nearly coincident or excluded pairs) adds nothing
      // here and is counted; such pairs are formed after the item
      const P2PSrc<ND, KIND>* const Rend = W.s + m;
#pragma unroll UNROLL
      for (const P2PSrc<ND, KIND>* R = W.s + ph; R < Rend; R += nph) {
        const float4 p = R->p;
        const float dx = (zh.x - p.x) + (zl.x - p.z);
        const float dy = (zh.y - p.y) + (zl.y - p.w);
        const float rr = fmaf(dx, dx, dy * dy);
        const bool fast = rr >= rslow;
        nslow += fast ? 0 : 1;
        const float ir = fast ? __fdividef(1.0f, rr) : 0.f;
        const float2 zi = make_float2(dx * ir, -dy * ir);
        const float2 z2 = make_float2(-(zi.x * zi.x - zi.y * zi.y), -2.f * zi.x * zi.y);
        if (HQ) {
          const float lg = fast ? fmaf(0.5f, __logf(rr), lsc) : 0.f;
#pragma unroll
          for (int d = 0; d < ND; d++) {
            const float2 v = R->c[d];
            fp[d].x = fmaf(lg, v.x, fp[d].x);
            fp[d].y = fmaf(lg, v.y, fp[d].y);
            if (IFPGH >= 2) cfmaf_(fg[d], zi, v);
            if (IFPGH >= 3) cfmaf_(fh[d], z2, v);
          }
        }
        if (HD) {
          float2 z3 = make_float2(0.f, 0.f);
          if (IFPGH >= 3) {
            z3 = cmulf_(z2, zi);
            z3 = make_float2(-2.f * z3.x, -2.f * z3.y);
          }
#pragma unroll
          for (int d = 0; d < ND; d++) {
            const float2 v = R->c[DOFF + d];
            cfmaf_(fp[d], zi, v);
            if (IFPGH >= 2) cfmaf_(fg[d], z2, v);
            if (IFPGH >= 3) cfmaf_(fh[d], z3, v);
          }
        }
      }
#pragma unroll
      for (int d = 0; d < ND; d++) {
        pt[d].x += fp[d].x;
        pt[d].y += fp[d].y;
        if (IFPGH >= 2) {
          gr[d].x += fg[d].x;
          gr[d].y += fg[d].y;
        }
        if (IFPGH >= 3) {
          hs[d].x += fh[d].x;
          hs[d].y += fh[d].y;
        }
      }
    }
    __syncwarp();
  }
  // sum the phases of every target: a tree over ph by shuffles at strides
  // ntc, 2 ntc, 4 ntc, ... (a lane adds its partner only if that phase
  // exists)
  for (int hh = 1; hh < nph; hh <<= 1) {
    const bool take = (ph & (2 * hh - 1)) == 0 && ph + hh < nph;
    const int off = hh * ntc;
    {
      const int v = __shfl_down_sync(FULL, nslow, off);
      if (take) nslow += v;
    }
#pragma unroll
    for (int d = 0; d < ND; d++) {
      double2 v;
      v.x = __shfl_down_sync(FULL, pt[d].x, off);
      v.y = __shfl_down_sync(FULL, pt[d].y, off);
      if (take) {
        pt[d].x += v.x;
        pt[d].y += v.y;
      }
      if (IFPGH >= 2) {
        v.x = __shfl_down_sync(FULL, gr[d].x, off);
        v.y = __shfl_down_sync(FULL, gr[d].y, off);
        if (take) {
          gr[d].x += v.x;
          gr[d].y += v.y;
        }
      }
      if (IFPGH >= 3) {
        v.x = __shfl_down_sync(FULL, hs[d].x, off);
        v.y = __shfl_down_sync(FULL, hs[d].y, off);
        if (take) {
          hs[d].x += v.x;
          hs[d].y += v.y;
        }
      }
    }
  }
  // the close pairs: beyond the pair of a point with itself (one per
  // target when the evaluation points are the sources) they are rare; the
  // target's lane walks its sources again and forms them one by one
  const bool redo = act && ph == 0 && nslow > (J.self_pairs ? 1 : 0);
  if (__any_sync(FULL, redo) && redo) {
    const double2 z = J.xe64[k];
    for (int e = 0; e < n1; e++) {
      const int j0 = W.lst[e], len = (e + 1 < n1 ? W.lpre[e + 1] : S) - W.lpre[e];
      for (int j = j0; j < j0 + len; j++) {
        const double2 sxy = J.xs64[j];
        float4 p;
        split_hilo((sxy.x - c.x) * sc, p.x, p.z);
        split_hilo((sxy.y - c.y) * sc, p.y, p.w);
        float dx = (zh.x - p.x) + (zl.x - p.z);
        float dy = (zh.y - p.y) + (zl.y - p.w);
        float rr = fmaf(dx, dx, dy * dy);
        if (rr >= rslow) continue;  // formed in the pass above
        if (J.self_pairs && j == k) continue;  // a point and itself: r = 0
        if (rr < 0x1p-40f) {
          // nearly coincident: the FP64 difference, rounded once
          dx = __double2float_rn((z.x - sxy.x) * sc);
          dy = __double2float_rn((z.y - sxy.y) * sc);
          rr = fmaf(dx, dx, dy * dy);
        }
        // cauchykernels2d.f: <= for potential-only, < otherwise
        if (IFPGH == 1 ? (rr <= th2) : (rr < th2)) continue;
        const float ir = __fdividef(1.0f, rr);
        const float2 zi = make_float2(dx * ir, -dy * ir);
        const float2 z2 = make_float2(-(zi.x * zi.x - zi.y * zi.y), -2.f * zi.x * zi.y);
        const float2 z3 = IFPGH >= 3 ? cmulf_(z2, zi) : make_float2(0.f, 0.f);
        const size_t o = (size_t)j * J.ndc + J.d0;
#pragma unroll
        for (int d = 0; d < ND; d++) {
          float2 fp = make_float2(0.f, 0.f), fg = fp, fh = fp;
          if (HQ) {
            const float lg = fmaf(0.5f, __logf(rr), lsc);
            const float2 v = J.q32[o + d];
            fp = make_float2(lg * v.x, lg * v.y);
            if (IFPGH >= 2) cfmaf_(fg, zi, v);
            if (IFPGH >= 3) cfmaf_(fh, z2, v);
          }
          if (HD) {
            const float2 v0 = J.d32[o + d];
            const float2 v = make_float2(v0.x * scf, v0.y * scf);
            cfmaf_(fp, zi, v);
            if (IFPGH >= 2) cfmaf_(fg, z2, v);
            if (IFPGH >= 3) cfmaf_(fh, make_float2(-2.f * z3.x, -2.f * z3.y), v);
          }
          pt[d].x += fp.x;
          pt[d].y += fp.y;
          if (IFPGH >= 2) {
            gr[d].x += fg.x;
            gr[d].y += fg.y;
          }
          if (IFPGH >= 3) {
            hs[d].x += fh.x;
            hs[d].y += fh.y;
          }
        }
      }
    }
  }
  if (lane < ntc) {
#pragma unroll
    for (int d = 0; d < ND; d++) {
      const size_t o = (size_t)k * J.ndc + J.d0 + d;
      double2 w = J.pot[o];
      J.pot[o] = make_double2(w.x + pt[d].x, w.y + pt[d].y);
      if (IFPGH >= 2) {
        w = J.grad[o];
        J.grad[o] = make_double2(w.x + sc * gr[d].x, w.y + sc * gr[d].y);
      }
      if (IFPGH >= 3) {
        w = J.hess[o];
        const double s2 = sc * sc;
        J.hess[o] = make_double2(w.x + s2 * hs[d].x, w.y + s2 * hs[d].y);
      }
    }
  }
}

template <int ND, int IFPGH, int KIND, int V>
__global__ void __launch_bounds__(128, P2P_MIN_BLOCKS(ND, IFPGH, V)) k_p2p_leaf(P2PJob J) {
  extern __shared__ float4 p2p_sm[];
  constexpr int CH = P2P_SHAPES[V].chunk;
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  P2PWarp<ND, KIND, CH>& W = ((P2PWarp<ND, KIND, CH>*)p2p_sm)[wib];
  // after a failed tree build the item list is empty
  const int ni = J.ctl->status == TB_OK ? *J.nitems : 0;
  const int nw = gridDim.x * (blockDim.x >> 5);
  for (int it = blockIdx.x * (blockDim.x >> 5) + wib; it < ni; it += nw)
    p2p_item<ND, IFPGH, KIND, V>(J, J.items[it], W, lane);
}

// Item offsets of the jobs of a batch (jobs of failed trees count none);
// one block of 256 threads.
__global__ void k_p2p_batch_prefix(const P2PJob* __restrict__ jobs, int njobs,
                                   int* __restrict__ prefix) {
  __shared__ int cnt[256];
  __shared__ int carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int base = 0; base < njobs; base += 256) {
    const int j = base + threadIdx.x;
    cnt[threadIdx.x] = j < njobs && jobs[j].ctl->status == TB_OK ? *jobs[j].nitems : 0;
    __syncthreads();
    if (threadIdx.x == 0) {
      int s = carry;
      for (int q = 0; q < 256 && base + q < njobs; q++) {
        prefix[base + q] = s;
        s += cnt[q];
      }
      carry = s;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) prefix[njobs] = carry;
}

// The near field of many trees in one persistent launch: warps take the
// items of all jobs in turn (the job of an item by a binary search of the
// prefix).
template <int ND, int IFPGH, int KIND, int V>
__global__ void __launch_bounds__(128, P2P_MIN_BLOCKS(ND, IFPGH, V)) k_p2p_batch(
    const P2PJob* __restrict__ jobs, int njobs, const int* __restrict__ prefix) {
  extern __shared__ float4 p2p_sm[];
  constexpr int CH = P2P_SHAPES[V].chunk;
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  P2PWarp<ND, KIND, CH>& W = ((P2PWarp<ND, KIND, CH>*)p2p_sm)[wib];
  const int ni = prefix[njobs];
  const int nw = gridDim.x * (blockDim.x >> 5);
  for (int it = blockIdx.x * (blockDim.x >> 5) + wib; it < ni; it += nw) {
    int lo = 0, hi = njobs - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (prefix[mid] <= it) lo = mid; else hi = mid - 1;
    }
    const P2PJob J = jobs[lo];
    p2p_item<ND, IFPGH, KIND, V>(J, J.items[it - prefix[lo]], W, lane);
  }
}

// Near field of the FP64 path (cauchykernels2d.f), on the same work items
// and lane mapping as k_p2p_leaf: sources staged as FP64 coordinates and
// densities, pair differences, terms and sums in FP64 as the reference, the
// pairs at r <= thresh (r < thresh with gradients) left out by a select,
// not a branch.  Adds to the far field already in the outputs.
template <int ND, int KIND>
struct P2PSrc64 {
  double2 p;
  double2 c[ND * ((KIND & 1) + ((KIND >> 1) & 1))];
};

template <int ND, int KIND>
struct P2PWarp64 {
  P2PSrc64<ND, KIND> s[64];
  int lst[16];
  int lpre[16];
};

template <int ND, int IFPGH, int KIND>
__global__ void __launch_bounds__(128) k_p2p_leaf64(
    TV t, const double2* __restrict__ xs64, const double2* __restrict__ xe64,
    const double2* __restrict__ q64, const double2* __restrict__ d64, int ndc, int d0,
    double thresh, const P2PItem* __restrict__ items, const int* __restrict__ nitems,
    double2* __restrict__ pot, double2* __restrict__ grad, double2* __restrict__ hess) {
  constexpr bool HQ = KIND & 1, HD = (KIND >> 1) & 1;
  constexpr int DOFF = HQ ? ND : 0;
  constexpr int CH = 64;
  extern __shared__ float4 p2p_sm[];
  constexpr unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  P2PWarp64<ND, KIND>& W = ((P2PWarp64<ND, KIND>*)p2p_sm)[wib];
  const int ni = t.ctl->status == TB_OK ? *nitems : 0;
  const double thr = near_thresh(t, thresh);
  const double th2 = thr * thr;
  const int nw = gridDim.x * (blockDim.x >> 5);
  for (int it = blockIdx.x * (blockDim.x >> 5) + wib; it < ni; it += nw) {
    const P2PItem& I = items[it];
    ((int*)W.lst)[lane] = ((const int*)I.lst)[lane];
    const int4 h = *(const int4*)&I;
    const int n1 = h.z >> 8, ntc = h.z & 255;
    const int S = I.S;
    const float rn = __frcp_rn((float)ntc);
    const int nph = __float2int_rz(32.5f * rn);
    const int ph = __float2int_rz(((float)lane + 0.5f) * rn), ti = lane - ph * ntc;
    const bool act = ph < nph;
    const long k = (long)h.y + ti;
    __syncwarp();
    const double2 z = xe64[k];
    double2 pt[ND], gr[ND], hs[ND];
#pragma unroll
    for (int d = 0; d < ND; d++) pt[d] = gr[d] = hs[d] = make_double2(0, 0);
    for (int u0 = 0; u0 < S; u0 += CH) {
      const int m = min(CH, S - u0);
      for (int i = lane; i < m; i += 32) {
        const int u = u0 + i;
        int e = 0;
#pragma unroll
        for (int step = 8; step > 0; step >>= 1)
          if (e + step < n1 && W.lpre[e + step] <= u) e += step;
        const int j = W.lst[e] + (u - W.lpre[e]);
        P2PSrc64<ND, KIND>& R = W.s[i];
        R.p = xs64[j];
        const size_t o = (size_t)j * ndc + d0;
#pragma unroll
        for (int d = 0; d < ND; d++) {
          if (HQ) R.c[d] = q64[o + d];
          if (HD) R.c[DOFF + d] = d64[o + d];
        }
      }
      __syncwarp();
      if (act) {
        for (int u = ph; u < m; u += nph) {
          const P2PSrc64<ND, KIND>& R = W.s[u];
          const double dx = z.x - R.p.x, dy = z.y - R.p.y;
          const double rr = dx * dx + dy * dy;
          // cauchykernels2d.f: <= for potential-only, < otherwise
          const bool inc = IFPGH == 1 ? !(rr <= th2) : !(rr < th2);
          const double ir = inc ? 1.0 / rr : 0.0;
          const double2 zi = make_double2(dx * ir, -dy * ir);
          const double2 z2 = cneg(cmul(zi, zi));
          if (HQ) {
            const double lg = inc ? 0.5 * log(rr) : 0.0;
#pragma unroll
            for (int d = 0; d < ND; d++) {
              const double2 c = R.c[d];
              pt[d].x += lg * c.x;
              pt[d].y += lg * c.y;
              if (IFPGH >= 2) cfma(gr[d], zi, c);
              if (IFPGH >= 3) cfma(hs[d], z2, c);
            }
          }
          if (HD) {
            const double2 z3 = IFPGH >= 3 ? cscale(cmul(z2, zi), -2.0) : make_double2(0, 0);
#pragma unroll
            for (int d = 0; d < ND; d++) {
              const double2 c = R.c[DOFF + d];
              cfma(pt[d], zi, c);
              if (IFPGH >= 2) cfma(gr[d], z2, c);
              if (IFPGH >= 3) cfma(hs[d], z3, c);
            }
          }
        }
      }
      __syncwarp();
    }
    for (int hh = 1; hh < nph; hh <<= 1) {
      const bool take = (ph & (2 * hh - 1)) == 0 && ph + hh < nph;
      const int off = hh * ntc;
#pragma unroll
      for (int d = 0; d < ND; d++) {
        double2 v;
        v.x = __shfl_down_sync(FULL, pt[d].x, off);
        v.y = __shfl_down_sync(FULL, pt[d].y, off);
        if (take) pt[d] = cadd(pt[d], v);
        if (IFPGH >= 2) {
          v.x = __shfl_down_sync(FULL, gr[d].x, off);
          v.y = __shfl_down_sync(FULL, gr[d].y, off);
          if (take) gr[d] = cadd(gr[d], v);
        }
        if (IFPGH >= 3) {
          v.x = __shfl_down_sync(FULL, hs[d].x, off);
          v.y = __shfl_down_sync(FULL, hs[d].y, off);
          if (take) hs[d] = cadd(hs[d], v);
        }
      }
    }
    if (lane < ntc) {
#pragma unroll
      for (int d = 0; d < ND; d++) {
        const size_t o = (size_t)k * ndc + d0 + d;
        pot[o] = cadd(pot[o], pt[d]);
        if (IFPGH >= 2) grad[o] = cadd(grad[o], gr[d]);
        if (IFPGH >= 3) hess[o] = cadd(hess[o], hs[d]);
      }
    }
  }
}

template <int ND, int IFPGH, int KIND>
void p2p64_launch(const TV& t, const MixedData& M, const double2* xe64, const Dens& D,
                  double thresh, const P2PItem* items, const int* nitems, double2* pot,
                  double2* grad, double2* hess, cudaStream_t st) {
  constexpr size_t sm = 4 * sizeof(P2PWarp64<ND, KIND>);
  auto kern = k_p2p_leaf64<ND, IFPGH, KIND>;
  set_smem_attr(kern, sm);
  kern<<<resident_grid(kern, 128, sm), 128, sm, st>>>(t, M.xs64, xe64, D.q, D.d, D.ndc, D.d0,
                                                     thresh, items, nitems, pot, grad, hess);
  B2_LAUNCH_CHECK();
}

template <int ND, int IFPGH>
void leaf64_launch(const TV& t, int use_targets, const MixedData& M, const double2* xe64,
                   const Dens& D, int P, const double2* mp, const double2* lo, double thresh,
                   int ifnear, double2* pot, double2* grad, double2* hess, cudaStream_t st) {
  const long n = use_targets ? M.nt : M.ns;
  if (n <= 0) return;
  const int* leaf = use_targets ? M.leaf_t.p : M.leaf_s.p;
  k_far_mixed<ND, IFPGH><<<ceil_div(n, 128), 128, 0, st>>>(t, n, leaf, xe64, D.ndc, D.d0, P, mp,
                                                          lo, pot, grad, hess);
  B2_LAUNCH_CHECK();
  const int kind = (D.q ? 1 : 0) | (D.d ? 2 : 0);
  if (!ifnear || kind == 0) return;
  const P2PItem* items = (const P2PItem*)(use_targets ? M.items_t.p : M.items_s.p);
  const int* nitems = M.nitems.p + (use_targets ? 1 : 0);
  if (kind == 3)
    p2p64_launch<ND, IFPGH, 3>(t, M, xe64, D, thresh, items, nitems, pot, grad, hess, st);
  else if (kind == 2)
    p2p64_launch<ND, IFPGH, 2>(t, M, xe64, D, thresh, items, nitems, pot, grad, hess, st);
  else
    p2p64_launch<ND, IFPGH, 1>(t, M, xe64, D, thresh, items, nitems, pot, grad, hess, st);
}

std::atomic<int> g_p2p_shape[B2FMM_P2P_CLASSES] = {};

template <int ND, int IFPGH, int KIND, int V>
void p2p_launch_v(const TV& t, const MixedData& M, const double2* xe64, int ndc, int d0,
                  double thresh, const P2PItem* items, const int* nitems, double2* pot,
                  double2* grad, double2* hess, cudaStream_t st) {
  constexpr size_t sm = 4 * sizeof(P2PWarp<ND, KIND, P2P_SHAPES[V].chunk>);
  auto kern = k_p2p_leaf<ND, IFPGH, KIND, V>;
  set_smem_attr(kern, sm);
  const P2PJob J{t.ctl, t.boxsize, M.xs64, xe64, M.q.p, M.d.p, items, nitems, pot, grad, hess,
                 thresh, ndc, d0, xe64 == M.xs64 ? 1 : 0, 0};
  kern<<<resident_grid(kern, 128, sm), 128, sm, st>>>(J);
  B2_LAUNCH_CHECK();
}

template <int ND, int IFPGH, int KIND>
void p2p_launch(const TV& t, const MixedData& M, const double2* xe64, int ndc, int d0,
                double thresh, const P2PItem* items, const int* nitems, double2* pot,
                double2* grad, double2* hess, cudaStream_t st) {
  const int v = p2p_tuned(ND, IFPGH) ? g_p2p_shape[p2p_leaf_class(M.ndiv)].load() : 0;
  if constexpr (p2p_tuned(ND, IFPGH)) {
    if (v == 1) {
      p2p_launch_v<ND, IFPGH, KIND, 1>(t, M, xe64, ndc, d0, thresh, items, nitems, pot, grad,
                                       hess, st);
      return;
    }
    if (v == 2) {
      p2p_launch_v<ND, IFPGH, KIND, 2>(t, M, xe64, ndc, d0, thresh, items, nitems, pot, grad,
                                       hess, st);
      return;
    }
  }
  p2p_launch_v<ND, IFPGH, KIND, 0>(t, M, xe64, ndc, d0, thresh, items, nitems, pot, grad, hess,
                                   st);
}

int grid_for(long nitems, int wpb) {
  long blocks = (nitems + wpb - 1) / wpb;
  return (int)std::max(1L, std::min(blocks, 148L * 32));
}

template <int ND>
void m2l_launch(const TV& t, int first, int n, int P, const double* binom, const MixedData& M,
                const double2* mp, double2* lo, cudaStream_t st) {
  const int RB = (P + 3) / 4, EG = 32 / RB;
  const size_t warp_floats = (size_t)EG * P * 2 * ND * 2 + ((2 * EG + 3) & ~3);
  size_t sm = sizeof(float) * 4 * warp_floats + sizeof(float4) * (size_t)P * RB +
              sizeof(float2) * 49 * P + sizeof(float) * 52;
  set_smem_attr(k_m2l_f32<ND>, sm);
  k_m2l_f32<ND><<<grid_for(n, 4), 128, sm, st>>>(t, first, n, P, RB, EG, binom, M.utab.p,
                                                  M.lgtab.p, mp, lo);
  B2_LAUNCH_CHECK();
}

template <int ND, int IFPGH>
void leaf_launch(const TV& t, int use_targets, const MixedData& M, const double2* xe64, int ndc,
                 int d0, int P, const double2* mp, const double2* lo, double thresh, int ifnear,
                 double2* pot, double2* grad, double2* hess, cudaStream_t st,
                 cudaEvent_t far_done) {
  const long n = use_targets ? M.nt : M.ns;
  if (n <= 0) return;
  const int* leaf = use_targets ? M.leaf_t.p : M.leaf_s.p;
  if (M.tc && M.pairs.usable && M.pairs.P == P && M.err && M.pairs.n > 0 && M.mp32.p) {
    // the FP32 multipoles of this chunk, from the tensor-core M2L
    k_far_f32<ND, IFPGH><<<ceil_div(n, 128), 128, 0, st>>>(t, n, leaf, xe64, ndc, d0, P,
                                                          m2l_kh(P), M.mp32.p, lo, pot, grad,
                                                          hess);
  } else {
    k_far_mixed<ND, IFPGH><<<ceil_div(n, 128), 128, 0, st>>>(t, n, leaf, xe64, ndc, d0, P, mp, lo,
                                                            pot, grad, hess);
  }
  B2_LAUNCH_CHECK();
  if (far_done) B2_CHECK(cudaEventRecord(far_done, st));
  const int kind = (M.q.p ? 1 : 0) | (M.d.p ? 2 : 0);
  if (!ifnear || kind == 0) return;
  const P2PItem* items = (const P2PItem*)(use_targets ? M.items_t.p : M.items_s.p);
  const int* nitems = M.nitems.p + (use_targets ? 1 : 0);
  if (kind == 3)
    p2p_launch<ND, IFPGH, 3>(t, M, xe64, ndc, d0, thresh, items, nitems, pot, grad, hess, st);
  else if (kind == 2)
    p2p_launch<ND, IFPGH, 2>(t, M, xe64, ndc, d0, thresh, items, nitems, pot, grad, hess, st);
  else
    p2p_launch<ND, IFPGH, 1>(t, M, xe64, ndc, d0, thresh, items, nitems, pot, grad, hess, st);
}

template <int ND>
void leaf_dispatch(int ifl, const TV& t, int use_targets, const MixedData& M,
                   const double2* xe64, int ndc, int d0, int P, const double2* mp,
                   const double2* lo, double thresh, int ifnear, double2* pot, double2* grad,
                   double2* hess, cudaStream_t st, cudaEvent_t far_done) {
  if (ifl == 1)
    leaf_launch<ND, 1>(t, use_targets, M, xe64, ndc, d0, P, mp, lo, thresh, ifnear, pot, grad, hess, st, far_done);
  else if (ifl == 2)
    leaf_launch<ND, 2>(t, use_targets, M, xe64, ndc, d0, P, mp, lo, thresh, ifnear, pot, grad, hess, st, far_done);
  else
    leaf_launch<ND, 3>(t, use_targets, M, xe64, ndc, d0, P, mp, lo, thresh, ifnear, pot, grad, hess, st, far_done);
}

template <int ND, int IFPGH, int KIND, int V>
void p2p_batch_group(const P2PJob* jobs, int njobs, int* prefix, cudaStream_t st) {
  constexpr size_t sm = 4 * sizeof(P2PWarp<ND, KIND, P2P_SHAPES[V].chunk>);
  auto kern = k_p2p_batch<ND, IFPGH, KIND, V>;
  set_smem_attr(kern, sm);
  k_p2p_batch_prefix<<<1, 256, 0, st>>>(jobs, njobs, prefix);
  B2_LAUNCH_CHECK();
  kern<<<resident_grid(kern, 128, sm), 128, sm, st>>>(jobs, njobs, prefix);
  B2_LAUNCH_CHECK();
}

template <int ND, int IFPGH, int KIND>
void p2p_batch_shape(int v, const P2PJob* jobs, int njobs, int* prefix, cudaStream_t st) {
  if constexpr (p2p_tuned(ND, IFPGH)) {
    if (v == 1) return p2p_batch_group<ND, IFPGH, KIND, 1>(jobs, njobs, prefix, st);
    if (v == 2) return p2p_batch_group<ND, IFPGH, KIND, 2>(jobs, njobs, prefix, st);
  }
  p2p_batch_group<ND, IFPGH, KIND, 0>(jobs, njobs, prefix, st);
}

template <int ND, int IFPGH>
void p2p_batch_kind(int kind, int v, const P2PJob* jobs, int njobs, int* prefix,
                    cudaStream_t st) {
  if (kind == 3) p2p_batch_shape<ND, IFPGH, 3>(v, jobs, njobs, prefix, st);
  else if (kind == 2) p2p_batch_shape<ND, IFPGH, 2>(v, jobs, njobs, prefix, st);
  else p2p_batch_shape<ND, IFPGH, 1>(v, jobs, njobs, prefix, st);
}

template <int ND>
void p2p_batch_ifl(int ifl, int kind, int v, const P2PJob* jobs, int njobs, int* prefix,
                   cudaStream_t st) {
  if (ifl == 1) p2p_batch_kind<ND, 1>(kind, v, jobs, njobs, prefix, st);
  else if (ifl == 2) p2p_batch_kind<ND, 2>(kind, v, jobs, njobs, prefix, st);
  else p2p_batch_kind<ND, 3>(kind, v, jobs, njobs, prefix, st);
}

}  // namespace

void lap_mixed_prepare(MixedData& M, const double2* xs, long ns, const double2* xt, long nt,
                       bool has_q, bool has_d, int ndc, double cx0, double cy0, int P,
                       cudaStream_t st) {
  (void)xt;
  (void)cx0;
  (void)cy0;
  M.xs64 = xs;
  long m = ns * (long)ndc;
  if (has_q) M.q.alloc(m, st);
  if (has_d) M.d.alloc(m, st);
  M.utab.alloc(49 * (size_t)P, st);
  M.lgtab.alloc(49, st);
  k_utab<<<49, 64, 0, st>>>(P, M.utab.p, M.lgtab.p);
  B2_LAUNCH_CHECK();
}

void lap_mixed_leaves(MixedData& M, const TV& t, int nb, bool dev, long ns, long nt, int ndiv,
                      cudaStream_t st) {
  M.ns = ns;
  M.nt = nt;
  M.ndiv = ndiv;
  M.leaf_s.alloc(ns, st);
  k_point_leaf<<<ceil_div(nb, 128), 128, 0, st>>>(t, dev ? -1 : nb, 0, M.leaf_s.p);
  B2_LAUNCH_CHECK();
  M.nitems.alloc(2, st);
  B2_CHECK(cudaMemsetAsync(M.nitems.p, 0, 2 * sizeof(int), st));
  // at most one item per leaf plus one per 32 points
  M.items_s.alloc(((size_t)nb + ns / 32 + 1) * sizeof(P2PItem), st);
  k_p2p_items<<<ceil_div(nb, 128), 128, 0, st>>>(t, dev ? -1 : nb, 0, (P2PItem*)M.items_s.p,
                                                  M.nitems.p);
  B2_LAUNCH_CHECK();
  if (nt > 0) {
    M.leaf_t.alloc(nt, st);
    k_point_leaf<<<ceil_div(nb, 128), 128, 0, st>>>(t, dev ? -1 : nb, 1, M.leaf_t.p);
    B2_LAUNCH_CHECK();
    M.items_t.alloc(((size_t)nb + nt / 32 + 1) * sizeof(P2PItem), st);
    k_p2p_items<<<ceil_div(nb, 128), 128, 0, st>>>(t, dev ? -1 : nb, 1, (P2PItem*)M.items_t.p,
                                                    M.nitems.p + 1);
    B2_LAUNCH_CHECK();
  }
}

void lap_mixed_densities(MixedData& M, const double2* qs, const double2* ds, long ns, int ndc,
                         cudaStream_t st) {
  long m = ns * (long)ndc;
  if (qs && M.q.p) {
    k_prep_dens<<<ceil_div(m, 256), 256, 0, st>>>(qs, m, M.q.p);
    B2_LAUNCH_CHECK();
  }
  if (ds && M.d.p) {
    k_prep_dens<<<ceil_div(m, 256), 256, 0, st>>>(ds, m, M.d.p);
    B2_LAUNCH_CHECK();
  }
}

namespace {
std::atomic<bool> g_m2l_tc{true};
}

int p2p_leaf_class(int ndiv) { return ndiv <= 20 ? 0 : (ndiv <= 56 ? 1 : 2); }

int set_p2p_shape(int leaf_class, int shape) {
  if (leaf_class < 0 || leaf_class >= B2FMM_P2P_CLASSES || shape < 0 || shape >= P2P_NSHAPES)
    return IER_BADARG;
  g_p2p_shape[leaf_class].store(shape);
  return IER_OK;
}

int p2p_shape(int leaf_class) {
  return leaf_class < 0 || leaf_class >= B2FMM_P2P_CLASSES ? -1 : g_p2p_shape[leaf_class].load();
}

void set_m2l_tensor_cores(bool on) { g_m2l_tc.store(on); }
bool m2l_tensor_cores() { return g_m2l_tc.load(); }

void lap_mixed_m2l(int ND, const TV& t, int first, int n, int P, const double* binom,
                   const MixedData& M, const double2* mp, double2* lo, cudaStream_t st) {
  if (M.tc && M.pairs.usable && M.pairs.P == P && M.err) {
    int r = m2l_tc_run(ND, M.pairs, mp, M.mp32.p, (long)M.mp32.n, M.nboxes, t.ctl, lo, t.boxsize,
                       M.nlev, M.err, st);
    if (r != IER_OK) throw CudaError("tensor-core M2L: invalid arguments", r);
    return;
  }
  switch (ND) {
    case 8: m2l_launch<8>(t, first, n, P, binom, M, mp, lo, st); break;
    case 4: m2l_launch<4>(t, first, n, P, binom, M, mp, lo, st); break;
    case 2: m2l_launch<2>(t, first, n, P, binom, M, mp, lo, st); break;
    default: m2l_launch<1>(t, first, n, P, binom, M, mp, lo, st); break;
  }
}

void lap_fp64_leaf(int ND, int ifl, const TV& t, int use_targets, const MixedData& M,
                   const double2* xe64, const Dens& D, int P, const double2* mp,
                   const double2* lo, double thresh, int ifnear, double2* pot, double2* grad,
                   double2* hess, cudaStream_t st) {
  auto run = [&](auto nd_tag) {
    constexpr int N = decltype(nd_tag)::value;
    if (ifl == 1)
      leaf64_launch<N, 1>(t, use_targets, M, xe64, D, P, mp, lo, thresh, ifnear, pot, grad, hess, st);
    else if (ifl == 2)
      leaf64_launch<N, 2>(t, use_targets, M, xe64, D, P, mp, lo, thresh, ifnear, pot, grad, hess, st);
    else
      leaf64_launch<N, 3>(t, use_targets, M, xe64, D, P, mp, lo, thresh, ifnear, pot, grad, hess, st);
  };
  switch (ND) {
    case 8: run(std::integral_constant<int, 8>()); break;
    case 4: run(std::integral_constant<int, 4>()); break;
    case 2: run(std::integral_constant<int, 2>()); break;
    default: run(std::integral_constant<int, 1>()); break;
  }
}

struct P2PBatch {
  struct Group {
    int ND, ifl, kind, shape, njobs;
    P2PJob* jobs;  // device
    int* prefix;   // device, njobs + 1
  };
  std::vector<Group> groups;
  ~P2PBatch() {
    for (auto& g : groups) {
      cudaFree(g.jobs);
      cudaFree(g.prefix);
    }
  }
};

P2PBatch* p2p_batch_create(const std::vector<P2PBatchEntry>& E) {
  std::unique_ptr<P2PBatch> B(new P2PBatch());
  std::vector<int> done(E.size(), 0);
  for (size_t i = 0; i < E.size(); i++) {
    if (done[i]) continue;
    const P2PBatchEntry& e = E[i];
    const int kind = (e.M->q.p ? 1 : 0) | (e.M->d.p ? 2 : 0);
    if (kind == 0) {
      done[i] = 1;
      continue;
    }
    // the tile shape each plan's own near field would use
    auto shape_of = [](const P2PBatchEntry& x) {
      return x.ND <= 2 && x.ifl <= 2 ? g_p2p_shape[p2p_leaf_class(x.M->ndiv)].load() : 0;
    };
    const int shape = shape_of(e);
    std::vector<P2PJob> jobs;
    for (size_t k = i; k < E.size(); k++) {
      const P2PBatchEntry& f = E[k];
      const int fk = (f.M->q.p ? 1 : 0) | (f.M->d.p ? 2 : 0);
      if (done[k] || f.ND != e.ND || f.ifl != e.ifl || fk != kind || shape_of(f) != shape)
        continue;
      done[k] = 1;
      jobs.push_back(P2PJob{f.tv->ctl, f.tv->boxsize, f.M->xs64, f.xe64, f.M->q.p, f.M->d.p,
                            (const P2PItem*)(f.use_targets ? f.M->items_t.p : f.M->items_s.p),
                            f.M->nitems.p + (f.use_targets ? 1 : 0), f.pot, f.grad, f.hess,
                            -1.0, f.ndc, 0, f.xe64 == f.M->xs64 ? 1 : 0, 0});
    }
    P2PBatch::Group g{e.ND, e.ifl, kind, shape, (int)jobs.size(), nullptr, nullptr};
    B2_CHECK(cudaMalloc(&g.jobs, sizeof(P2PJob) * jobs.size()));
    B2_CHECK(cudaMalloc(&g.prefix, sizeof(int) * (jobs.size() + 1)));
    B->groups.push_back(g);
    B2_CHECK(cudaMemcpy(g.jobs, jobs.data(), sizeof(P2PJob) * jobs.size(),
                        cudaMemcpyHostToDevice));
  }
  return B.release();
}

void p2p_batch_launch(const P2PBatch* B, cudaStream_t st) {
  for (const auto& g : B->groups) {
    switch (g.ND) {
      case 8: p2p_batch_ifl<8>(g.ifl, g.kind, g.shape, g.jobs, g.njobs, g.prefix, st); break;
      case 4: p2p_batch_ifl<4>(g.ifl, g.kind, g.shape, g.jobs, g.njobs, g.prefix, st); break;
      case 2: p2p_batch_ifl<2>(g.ifl, g.kind, g.shape, g.jobs, g.njobs, g.prefix, st); break;
      default: p2p_batch_ifl<1>(g.ifl, g.kind, g.shape, g.jobs, g.njobs, g.prefix, st); break;
    }
  }
}

void p2p_batch_free(P2PBatch* B) { delete B; }

void lap_mixed_leaf(int ND, int ifl, const TV& t, int nb, int use_targets, const MixedData& M,
                    const double2* xe64, int ndc, int d0, int P, const double2* mp,
                    const double2* lo, double thresh, int ifnear, double2* pot, double2* grad,
                    double2* hess, cudaStream_t st, cudaEvent_t far_done) {
  (void)nb;
  switch (ND) {
    case 8: leaf_dispatch<8>(ifl, t, use_targets, M, xe64, ndc, d0, P, mp, lo, thresh, ifnear, pot, grad, hess, st, far_done); break;
    case 4: leaf_dispatch<4>(ifl, t, use_targets, M, xe64, ndc, d0, P, mp, lo, thresh, ifnear, pot, grad, hess, st, far_done); break;
    case 2: leaf_dispatch<2>(ifl, t, use_targets, M, xe64, ndc, d0, P, mp, lo, thresh, ifnear, pot, grad, hess, st, far_done); break;
    default: leaf_dispatch<1>(ifl, t, use_targets, M, xe64, ndc, d0, P, mp, lo, thresh, ifnear, pot, grad, hess, st, far_done); break;
  }
}

}  // namespace b2
