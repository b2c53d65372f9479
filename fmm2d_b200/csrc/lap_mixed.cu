// Mixed-precision Laplace kernels (eps >= 1e-6).
//
// * k_m2l_f32: the M2L of laprouts2d.f:1130-1244 in FP32.  Boxes of one
//   level are translated by integer offsets o (|o|_inf in 2..3) in units of
//   the box size, so u = r/z0 = 1/o and log|z0| = log r + log|o| come from
//   49-entry tables; per translation only the gather of the source
//   multipole (FP64 -> FP32) and the fixed matrix G(i,j) = C(i+j-1, j-1)
//   remain.  Local expansions are accumulated in FP32 per target box and
//   added to the FP64 expansion once.
// * k_far_mixed / k_p2p_mixed: one evaluation point per thread.  L2P and M2P
//   in FP64 (as the FP64 path), then the near field in FP32.  The coordinate
//   difference of a pair is formed in FP64 and rounded once to FP32, so it
//   keeps the relative accuracy of the FP64 path's difference even for nearly
//   coincident points (separations of 1e-12 occur in graded distributions);
//   log and 1/r^2 use the SFU.  Per-pair terms are summed in FP32 over at
//   most 32 sources and the partial sums in FP64.
#include "lap_mixed.cuh"

#include <atomic>
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

// The same for the near field: 10 blocks (at most 48 registers a thread) for
// one or two densities without hessians (leaf phase 2.50 -> 2.43 ms at 4M).
#define P2P_MIN_BLOCKS(ND, IFPGH) ((ND) <= 2 && (IFPGH) <= 2 ? 10 : 1)

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

// Near field of one evaluation point per thread, FP32 (cauchykernels2d.f):
// all sources of the leaf's list-1 boxes; coordinate differences from the
// hi/lo float pairs, per-pair terms summed in FP32 over at most 32 sources,
// the partial sums in FP64, added to the far field already in the outputs.
template <int ND, int IFPGH>
__global__ void __launch_bounds__(128, P2P_MIN_BLOCKS(ND, IFPGH)) k_p2p_mixed(
    TV t, long n, const int* __restrict__ leaf, const double2* __restrict__ xs64,
    const double2* __restrict__ xe64, const float2* __restrict__ q32,
    const float2* __restrict__ d32, int ndc, int d0, float th2, double2* __restrict__ pot,
    double2* __restrict__ grad, double2* __restrict__ hess) {
  long k = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (k >= n || t.ctl->status != TB_OK) return;
  if (th2 < 0.f) {
    const double thr = near_thresh(t, -1.0);
    th2 = (float)(thr * thr);
  }
  const bool hq = q32 != nullptr, hd = d32 != nullptr;
  const int b = leaf[k];
  const double2 z = xe64[k];
  double2 pt[ND], gr[ND], hs[ND];
#pragma unroll
  for (int d = 0; d < ND; d++) pt[d] = gr[d] = hs[d] = make_double2(0, 0);
  float2 fp[ND], fg[ND], fh[ND];
#pragma unroll
  for (int d = 0; d < ND; d++) fp[d] = fg[d] = fh[d] = make_float2(0.f, 0.f);
  int cnt = 0;
  const int n1 = t.nl1[b];
  for (int e = 0; e < n1; e++) {
    int2 sr = t.srng[t.l1[(size_t)MNLIST1 * b + e]];
    for (int j = sr.x; j < sr.y; j++) {
      // the difference in FP64 (as the FP64 path forms it), the kernel in FP32:
      // sources closer than ~1e-15 of the coordinates keep their relative accuracy
      double2 s = xs64[j];
      float dx = (float)(z.x - s.x);
      float dy = (float)(z.y - s.y);
      float rr = fmaf(dx, dx, dy * dy);
      // cauchykernels2d.f: <= for potential-only, < otherwise
      if (!(IFPGH == 1 ? (rr <= th2) : (rr < th2))) {
        float ir = __fdividef(1.0f, rr);
        float2 zi = make_float2(dx * ir, -dy * ir);
        float2 z2 = make_float2(-(zi.x * zi.x - zi.y * zi.y), -2.f * zi.x * zi.y);
        if (hq) {
          float lg = 0.5f * __logf(rr);
#pragma unroll
          for (int d = 0; d < ND; d++) {
            float2 c = q32[(size_t)j * ndc + d0 + d];
            fp[d].x = fmaf(lg, c.x, fp[d].x);
            fp[d].y = fmaf(lg, c.y, fp[d].y);
            if (IFPGH >= 2) cfmaf_(fg[d], zi, c);
            if (IFPGH >= 3) cfmaf_(fh[d], z2, c);
          }
        }
        if (hd) {
          float2 z3 = make_float2(0.f, 0.f);
          if (IFPGH >= 3) {
            z3 = cmulf_(z2, zi);
            z3 = make_float2(-2.f * z3.x, -2.f * z3.y);
          }
#pragma unroll
          for (int d = 0; d < ND; d++) {
            float2 c = d32[(size_t)j * ndc + d0 + d];
            cfmaf_(fp[d], zi, c);
            if (IFPGH >= 2) cfmaf_(fg[d], z2, c);
            if (IFPGH >= 3) cfmaf_(fh[d], z3, c);
          }
        }
      }
      if (++cnt == 32) {
        cnt = 0;
#pragma unroll
        for (int d = 0; d < ND; d++) {
          pt[d].x += fp[d].x;
          pt[d].y += fp[d].y;
          fp[d] = make_float2(0.f, 0.f);
          if (IFPGH >= 2) {
            gr[d].x += fg[d].x;
            gr[d].y += fg[d].y;
            fg[d] = make_float2(0.f, 0.f);
          }
          if (IFPGH >= 3) {
            hs[d].x += fh[d].x;
            hs[d].y += fh[d].y;
            fh[d] = make_float2(0.f, 0.f);
          }
        }
      }
    }
  }
#pragma unroll
  for (int d = 0; d < ND; d++) {
    size_t o = (size_t)k * ndc + d0 + d;
    double2 v = pot[o];
    pot[o] = make_double2(v.x + pt[d].x + fp[d].x, v.y + pt[d].y + fp[d].y);
    if (IFPGH >= 2) {
      v = grad[o];
      grad[o] = make_double2(v.x + gr[d].x + fg[d].x, v.y + gr[d].y + fg[d].y);
    }
    if (IFPGH >= 3) {
      v = hess[o];
      hess[o] = make_double2(v.x + hs[d].x + fh[d].x, v.y + hs[d].y + fh[d].y);
    }
  }
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
void leaf_launch(const TV& t, int nb, int use_targets, const MixedData& M, const double2* xe64,
                 int ndc, int d0, int P, const double2* mp, const double2* lo, double thresh,
                 int ifnear, double2* pot, double2* grad, double2* hess, cudaStream_t st,
                 cudaEvent_t far_done) {
  (void)nb;
  const long n = use_targets ? M.nt : M.ns;
  if (n <= 0) return;
  const int* leaf = use_targets ? M.leaf_t.p : M.leaf_s.p;
  k_far_mixed<ND, IFPGH><<<ceil_div(n, 128), 128, 0, st>>>(t, n, leaf, xe64, ndc, d0, P, mp, lo,
                                                          pot, grad, hess);
  B2_LAUNCH_CHECK();
  if (far_done) B2_CHECK(cudaEventRecord(far_done, st));
  if (!ifnear) return;
  k_p2p_mixed<ND, IFPGH><<<ceil_div(n, 128), 128, 0, st>>>(
      t, n, leaf, M.xs64, xe64, M.q.p, M.d.p, ndc, d0,
      thresh >= 0 ? (float)(thresh * thresh) : -1.f, pot, grad, hess);
  B2_LAUNCH_CHECK();
}

template <int ND>
void leaf_dispatch(int ifl, const TV& t, int nb, int use_targets, const MixedData& M,
                   const double2* xe64, int ndc, int d0, int P, const double2* mp,
                   const double2* lo, double thresh, int ifnear, double2* pot, double2* grad,
                   double2* hess, cudaStream_t st, cudaEvent_t far_done) {
  if (ifl == 1)
    leaf_launch<ND, 1>(t, nb, use_targets, M, xe64, ndc, d0, P, mp, lo, thresh, ifnear, pot, grad, hess, st, far_done);
  else if (ifl == 2)
    leaf_launch<ND, 2>(t, nb, use_targets, M, xe64, ndc, d0, P, mp, lo, thresh, ifnear, pot, grad, hess, st, far_done);
  else
    leaf_launch<ND, 3>(t, nb, use_targets, M, xe64, ndc, d0, P, mp, lo, thresh, ifnear, pot, grad, hess, st, far_done);
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

void lap_mixed_leaves(MixedData& M, const TV& t, int nb, bool dev, long ns, long nt,
                      cudaStream_t st) {
  M.ns = ns;
  M.nt = nt;
  M.leaf_s.alloc(ns, st);
  k_point_leaf<<<ceil_div(nb, 128), 128, 0, st>>>(t, dev ? -1 : nb, 0, M.leaf_s.p);
  B2_LAUNCH_CHECK();
  if (nt > 0) {
    M.leaf_t.alloc(nt, st);
    k_point_leaf<<<ceil_div(nb, 128), 128, 0, st>>>(t, dev ? -1 : nb, 1, M.leaf_t.p);
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

void lap_mixed_leaf(int ND, int ifl, const TV& t, int nb, int use_targets, const MixedData& M,
                    const double2* xe64, int ndc, int d0, int P, const double2* mp,
                    const double2* lo, double thresh, int ifnear, double2* pot, double2* grad,
                    double2* hess, cudaStream_t st, cudaEvent_t far_done) {
  switch (ND) {
    case 8: leaf_dispatch<8>(ifl, t, nb, use_targets, M, xe64, ndc, d0, P, mp, lo, thresh, ifnear, pot, grad, hess, st, far_done); break;
    case 4: leaf_dispatch<4>(ifl, t, nb, use_targets, M, xe64, ndc, d0, P, mp, lo, thresh, ifnear, pot, grad, hess, st, far_done); break;
    case 2: leaf_dispatch<2>(ifl, t, nb, use_targets, M, xe64, ndc, d0, P, mp, lo, thresh, ifnear, pot, grad, hess, st, far_done); break;
    default: leaf_dispatch<1>(ifl, t, nb, use_targets, M, xe64, ndc, d0, P, mp, lo, thresh, ifnear, pot, grad, hess, st, far_done); break;
  }
}

}  // namespace b2
