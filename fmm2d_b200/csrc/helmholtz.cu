// Helmholtz FMM on B200 (FP64): hfmm2dmain (src/helmholtz/hfmm2d.f:456-1580)
// with the operators of src/helmholtz/helmrouts2d.f, the wideband
// translations of wideband2d.f and the near field of helmkernels2d.f; and
// the FMM over multipole sources hfmm2d_mps (hfmm2d_mps.f).
//
// Expansions have 2p_l+1 coefficients (n = -p_l..p_l) per density, with a
// per-level order p_l (h2dterms) and scale rs_l = min(|zk bs_l / 2pi|, 1);
// box b of level l stores them at off_l + (b - lfirst_l) (2p_l+1) ND.
// Centres of boxes of one level differ by multiples of the box size, so the
// translation kernels of M2L (per integer offset) and of M2M / L2L (per
// child slot) are tabulated once per level; M2L and the shifts then become
// Toeplitz convolutions with per-lane rscale factors:
//   M2M: H2(i) += sum_j H1(j) T(i-j) (rs1/rs2)^|i| rs1^(2e),
//        e = max(0,|j|-|i|) for j of the sign of i, else |j|   (h2dmpmp)
//   L2L: J2(i) += sum_j J1(j) T(i-j) F(i,j)                     (h2dlocloc)
//   M2L: L(i)  += sum_j H(j) T(i-j) rs^(2 min(|j|,|i|)) [same sign] (h2dmploc)
#include "helmholtz.cuh"

#include <algorithm>
#include <cmath>
#include <mutex>

#include "fft235.cuh"
#include "helm_special.cuh"
#include "lap_common.cuh"
#include "laplace.cuh"
#include "tree.cuh"

namespace b2 {

namespace helm {
const SerTab& helm_tables() {
  static SerTab T;
  static std::once_flag once;
  std::call_once(once, [] {
    double f = 1.0;  // k!
    double hk = 0.0;
    const double eg = 0.57721566490153286061;
    for (int k = 0; k < NSER; k++) {
      if (k > 0) {
        f *= k;
        hk += 1.0 / k;
      }
      double fk1 = f * (k + 1);
      T.c0[k] = 1.0 / (f * f);
      T.c1[k] = 1.0 / (f * fk1);
      T.cy0[k] = hk / (f * f);
      T.cy1[k] = (2.0 * (hk - eg) + 1.0 / (k + 1)) / (f * fk1);
    }
    T.a0[0] = T.a1[0] = 1.0;
    for (int k = 1; k < NSER; k++) {
      double m = (2.0 * k - 1) * (2.0 * k - 1);
      T.a0[k] = T.a0[k - 1] * (0.0 - m) / (8.0 * k);
      T.a1[k] = T.a1[k - 1] * (4.0 - m) / (8.0 * k);
    }
  });
  return T;
}
}  // namespace helm

namespace {

using namespace lapk;
using helm::hscaled;
using helm::jscaled;

void ensure_device_tables() {
  static std::mutex mu;
  static bool done[128] = {false};
  int dev = 0;
  B2_CHECK(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> g(mu);
  if (done[dev]) return;
  const helm::SerTab& T = helm::helm_tables();
  B2_CHECK(cudaMemcpyToSymbol(helm::c_ser, &T, sizeof(T)));
  done[dev] = true;
}

constexpr int HMAXP = 63;      // largest order of the coefficient-per-lane translations
constexpr int HF_MAXSIG = 7000;  // longest signature (2 x 7000 x 16 B of shared memory)

struct HLev {
  int lfirst, p, P, ok;  // ok: expansions formed at this level (zkiupbound test)
  double rs, bs;
  long off;              // expansion offset (double2 units, times ND inside kernels)
  int nsh;               // half width of the M2M/L2L tables towards level l+1
  long tm2l, tm2m, tl2l; // table offsets (double2 units)
  // wideband: translations of this level (M2L, and the shifts between it
  // and level l+1) run on signatures, FFTs of the expansions
  int wide;
  int nsig, nsig_sh;      // signature lengths: M2L, shifts towards l+1
  long sig_off;           // per-box M2L signatures (double2 units, times ND)
  long tv_m2l, tv_mm, tv_ll;  // diagonal translation operators (double2 units)
};

__device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }

// T[k], k = -nt..nt: T(0) = Z_0, T(j) = e^j Z_j, T(-j) = (-conj e)^j Z_j with
// e = exp(-i theta) (the jtemp/htemp tables of h2dmpmp / h2dmploc).
__device__ void phase_table(int nt, double theta, const double2* Z, double2* T) {
  double2 e = make_double2(cos(theta), -sin(theta));
  double2 ec = cconj(e);
  T[nt] = Z[0];
  double2 a = e, b = make_double2(-ec.x, -ec.y);
  for (int j = 1; j <= nt; j++) {
    T[nt + j] = cmul(a, Z[j]);
    T[nt - j] = cmul(b, Z[j]);
    a = cmul(a, e);
    b = cmul(b, make_double2(-ec.x, -ec.y));
  }
}

// One thread per (level, table): M2L tables for 49 offsets at levels >= 2,
// M2M and L2L tables for the 4 child slots below every level.
__global__ void k_h_tables(const HLev* __restrict__ lv, int nl, double zkr, double zki,
                           double2* __restrict__ tabs, double2* __restrict__ scratch,
                           int scratch_stride) {
  int tid = blockIdx.x * blockDim.x + threadIdx.x;
  const double pi = 3.14159265358979323846;
  int nper = 49 + 8;
  int l = tid / nper, k = tid % nper;
  if (l > nl) return;
  double2 zk = make_double2(zkr, zki);
  double2* Z = scratch + (size_t)tid * scratch_stride;
  HLev L = lv[l];
  if (k < 49) {
    if (l < 2 || !L.ok || L.wide) return;
    int ox = k / 7 - 3, oy = k % 7 - 3;
    if (ox >= -1 && ox <= 1 && oy >= -1 && oy <= 1) return;
    // z0 = c_tgt - c_src = o bs; theta - pi as in h2dmploc
    double x = ox * L.bs, y = oy * L.bs;
    double r = sqrt(x * x + y * y), th = atan2(y, x) - pi;
    int nt = 2 * L.p;
    hscaled(nt + 1, make_double2(zk.x * r, zk.y * r), L.rs, Z);
    phase_table(nt, th, Z, tabs + L.tm2l + (size_t)k * (2 * nt + 1));
    return;
  }
  if (l >= nl || l < 2 || L.wide) return;  // shifts run between levels >= 2
  HLev C = lv[l + 1];
  int slot = (k - 49) % 4, kind = (k - 49) / 4;  // kind 0: M2M, 1: L2L
  if (!(kind == 0 ? C.ok : L.ok)) return;
  double h = C.bs / 2;
  double cx = (slot & 1) ? h : -h, cy = (slot < 2) ? -h : h;  // child - parent
  int nt = L.nsh;
  // M2M: z0 = parent - child, scaled by rs(child); L2L: child - parent, rs(parent)
  double x = kind == 0 ? -cx : cx, y = kind == 0 ? -cy : cy;
  double r = sqrt(x * x + y * y), th = atan2(y, x) - pi;
  double rs1 = kind == 0 ? C.rs : L.rs;
  jscaled(nt + 3, make_double2(zk.x * r, zk.y * r), rs1, Z);
  phase_table(nt, th, Z, tabs + (kind == 0 ? L.tm2m : L.tl2l) + (size_t)slot * (2 * nt + 1));
}

struct HDens {
  const double2* q;   // sorted charges (nd per point)
  const double2* d;   // sorted dipole strengths
  const double* v;    // sorted dipvec (2*nd per point)
  int nd, d0;
};

// Per-source expansion terms (ctompole / dtompole, helmrouts2d.f:1383-1492)
// for coefficient n of one density: Z = scaled J (multipole) or H (local),
// E = powers of e = exp(-i theta) of the source, q, dipole d with (v1, v2).
__device__ __forceinline__ double2 src_term(int n, const double2* Z, const double2* E, double2 q,
                                            double2 d, double v1, double v2, bool hq, bool hd,
                                            double2 zk, double rs) {
  int m = n < 0 ? -n : n;
  double2 res = make_double2(0, 0);
  double2 em = E[m];
  double2 eneg = cconj(em);  // e^{+i m theta}
  if (hq) {
    if (n == 0)
      res = cmul(q, Z[0]);
    else if (n > 0)
      res = cmul(cmul(Z[m], em), q);
    else {
      double2 t = cmul(Z[m], eneg);
      if (m & 1) t = make_double2(-t.x, -t.y);
      res = cmul(t, q);
    }
  }
  if (hd) {
    double2 e1 = E[1], ei = cconj(E[1]);  // zmul, zinv
    double2 hzk = make_double2(0.5 * zk.x, 0.5 * zk.y);
    if (n == 0) {
      double2 sp = cadd(e1, ei), sm = csub(e1, ei);
      double2 u = cadd(cscale(sp, v1), cscale(make_double2(-sm.y, sm.x), v2));  // (e+ei) v1 + (e-ei) i v2
      double2 t = cmul(cmul(cscale(Z[1], rs), hzk), u);
      res = csub(res, cmul(d, t));
    } else if (n > 0) {
      double2 z7 = cmul(cscale(ei, 1.0 / rs), make_double2(-v1, v2));
      double2 z8 = cmul(cscale(e1, rs), make_double2(v1, v2));
      double2 t1 = cmul(make_double2(-hzk.x, -hzk.y), E[m]);  // -(zk/2) e^m
      double2 s = cadd(cmul(Z[m - 1], z7), cmul(Z[m + 1], z8));
      res = cadd(res, cmul(cmul(s, t1), d));
    } else {
      double2 z9 = cmul(cscale(e1, 1.0 / rs), make_double2(-v1, -v2));
      double2 z10 = cmul(cscale(ei, rs), make_double2(v1, -v2));
      double2 t2 = cmul(hzk, eneg);  // (zk/2) zinv^m (-1)^(m-1)
      if (!(m & 1)) t2 = make_double2(-t2.x, -t2.y);
      double2 s = cadd(cmul(Z[m - 1], z9), cmul(Z[m + 1], z10));
      res = cadd(res, cmul(cmul(s, t2), d));
    }
  }
  return res;
}

// Form expansions from sources (P2M with J, P2L with H).  Warp per box;
// 16 sources staged at a time (tables Z and E in shared memory), then lanes
// take coefficients n = -p..p.
template <int ND>
__device__ void form_from_sources(int lane, double2* Zs, double2* Es, double* Ps, int sbeg,
                                  int send, const double2* __restrict__ xs, const HDens& D,
                                  double2 c, double2 zk, double rs, int p, bool mpole, int n0,
                                  int SB, double2 acc[4][ND]) {
  const int W = p + 3;  // table width (orders 0..p+2)
  const bool hq = D.q != nullptr, hd = D.d != nullptr;
  for (int s0 = sbeg; s0 < send; s0 += SB) {
    int m = min(SB, send - s0);
    __syncwarp();
    if (lane < m) {
      int j = s0 + lane;
      double2 x = xs[j];
      double dx = x.x - c.x, dy = x.y - c.y;
      double r = sqrt(dx * dx + dy * dy);
      double th = (dx == 0 && dy == 0) ? 0.0 : atan2(dy, dx);
      double2 z = make_double2(zk.x * r, zk.y * r);
      double2* Z = Zs + lane * W;
      if (mpole)
        jscaled(p + 1, z, rs, Z);
      else
        hscaled(p + 2, z, rs, Z);
      double2 e = make_double2(cos(th), -sin(th));
      double2* E = Es + lane * W;
      E[0] = make_double2(1, 0);
      for (int k = 1; k <= p + 1; k++) E[k] = cmul(E[k - 1], e);
      double* Pp = Ps + lane * (4 * ND + 2 * ND);
      for (int d = 0; d < ND; d++) {
        double2 q = hq ? D.q[(size_t)j * D.nd + D.d0 + d] : make_double2(0, 0);
        double2 dd = hd ? D.d[(size_t)j * D.nd + D.d0 + d] : make_double2(0, 0);
        Pp[4 * d] = q.x;
        Pp[4 * d + 1] = q.y;
        Pp[4 * d + 2] = dd.x;
        Pp[4 * d + 3] = dd.y;
        Pp[4 * ND + 2 * d] = hd ? D.v[((size_t)j * 2 + 0) * D.nd + D.d0 + d] : 0.0;
        Pp[4 * ND + 2 * d + 1] = hd ? D.v[((size_t)j * 2 + 1) * D.nd + D.d0 + d] : 0.0;
      }
    }
    __syncwarp();
    double rsd = mpole ? rs : 1.0 / rs;
#pragma unroll
    for (int sl = 0; sl < 4; sl++) {
      int n = n0 + lane + 32 * sl;
      if (n > p) break;
      for (int jj = 0; jj < m; jj++) {
        const double* Pp = Ps + jj * (4 * ND + 2 * ND);
#pragma unroll
        for (int d = 0; d < ND; d++) {
          double2 q = make_double2(Pp[4 * d], Pp[4 * d + 1]);
          double2 dd = make_double2(Pp[4 * d + 2], Pp[4 * d + 3]);
          acc[sl][d] = cadd(acc[sl][d],
                            src_term(n, Zs + jj * W, Es + jj * W, q, dd, Pp[4 * ND + 2 * d],
                                     Pp[4 * ND + 2 * d + 1], hq, hd, zk, rsd));
        }
      }
    }
  }
}

#define HLOOP(n)                                                                      \
  const int lane = threadIdx.x & 31;                                                  \
  const int wib = threadIdx.x >> 5;                                                   \
  const int nwarps = (gridDim.x * blockDim.x) >> 5;                                   \
  for (int bi = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; bi < (n); bi += nwarps)

__device__ __forceinline__ double2* hexp(double2* base, const HLev& L, int b, int ND) {
  return base + (L.off + (size_t)(b - L.lfirst) * L.P) * ND;
}

// Shared memory of one warp of the expansion-forming kernels: tables of SB
// sources (Z and E, orders 0..maxp+2) and their densities.
__device__ __forceinline__ double2* form_smem(double2* base, int wib, int maxp, int SB, int ND) {
  return base + (size_t)wib * SB * (2 * (maxp + 3) + 3 * ND);
}

// step 1: P2M at leaves of levels >= 2 (zero expansions elsewhere), 128
// coefficients at a time
template <int ND>
__global__ void __launch_bounds__(64) k_h_p2m(TV t, const HLev* __restrict__ lv, int nb,
                                              const double2* __restrict__ xs, HDens D, double zkr,
                                              double zki, double2* __restrict__ mp, int maxp,
                                              int SB) {
  extern __shared__ double2 hsm[];
  HLOOP(nb) {
    int b = bi;
    if (t.nchild[b] != 0) continue;
    int lev = t.level[b];
    if (lev < 2) continue;  // multipoles of levels 0 and 1 are never used
    HLev L = lv[lev];
    int W = L.p + 3;
    double2* Zs = form_smem(hsm, wib, maxp, SB, ND);
    double2* Es = Zs + SB * W;
    double* Ps = (double*)(Es + SB * W);
    int2 sr = t.srng[b];
    double2* M = hexp(mp, L, b, ND);
    for (int n0 = -L.p; n0 <= L.p; n0 += 128) {
      double2 acc[4][ND];
#pragma unroll
      for (int s = 0; s < 4; s++)
#pragma unroll
        for (int d = 0; d < ND; d++) acc[s][d] = make_double2(0, 0);
      if (L.ok && sr.y > sr.x)
        form_from_sources<ND>(lane, Zs, Es, Ps, sr.x, sr.y, xs, D, t.center[b],
                              make_double2(zkr, zki), L.rs, L.p, true, n0, SB, acc);
#pragma unroll
      for (int s = 0; s < 4; s++) {
        int n = n0 + lane + 32 * s;
        if (n > L.p) break;
#pragma unroll
        for (int d = 0; d < ND; d++) M[(n + L.p) * ND + d] = acc[s][d];
      }
    }
  }
}

// step 2: P2L from list 4
template <int ND>
__global__ void __launch_bounds__(64) k_h_p2l(TV t, const HLev* __restrict__ lv, int first, int n,
                                              const double2* __restrict__ xs, HDens D, double zkr,
                                              double zki, double2* __restrict__ lo, int maxp,
                                              int SB) {
  extern __shared__ double2 hsm[];
  HLOOP(n) {
    int b = first + bi;
    int n4 = t.nl4[b];
    if (n4 == 0 || !t.has_eval_pts(b)) continue;
    int lev = t.level[b];
    HLev L = lv[lev];
    if (!L.ok) continue;
    int W = L.p + 3;
    double2* Zs = form_smem(hsm, wib, maxp, SB, ND);
    double2* Es = Zs + SB * W;
    double* Ps = (double*)(Es + SB * W);
    double2* Lo = hexp(lo, L, b, ND);
    for (int n0 = -L.p; n0 <= L.p; n0 += 128) {
      double2 acc[4][ND];
#pragma unroll
      for (int s = 0; s < 4; s++)
#pragma unroll
        for (int d = 0; d < ND; d++) acc[s][d] = make_double2(0, 0);
      for (int e = 0; e < n4; e++) {
        int2 sr = t.srng[t.l4[(size_t)MNLIST4 * b + e]];
        form_from_sources<ND>(lane, Zs, Es, Ps, sr.x, sr.y, xs, D, t.center[b],
                              make_double2(zkr, zki), L.rs, L.p, false, n0, SB, acc);
      }
#pragma unroll
      for (int s = 0; s < 4; s++) {
        int nn = n0 + lane + 32 * s;
        if (nn > L.p) break;
#pragma unroll
        for (int d = 0; d < ND; d++)
          Lo[(nn + L.p) * ND + d] = cadd(Lo[(nn + L.p) * ND + d], acc[s][d]);
      }
    }
  }
}

// step 3: M2M, parents of one level.  One block per parent, one thread per
// output coefficient i; each child's multipole (plain and scaled by
// rs1^(2|j|)) and its child-slot kernel table are staged in shared memory:
//   H2(i) += (rs1/rs2)^|i| sum_j H1(j) T(i-j) rs1^(2e),
//   e = max(0, |j| - |i|) for j of the sign of i, else |j|   (h2dmpmp)
template <int ND>
__global__ void __launch_bounds__(128) k_h_m2m(TV t, const HLev* __restrict__ lv, int lev, int first,
                                               int n, const double2* __restrict__ tabs,
                                               double2* __restrict__ mp) {
  extern __shared__ double2 hsm[];
  const HLev L = lv[lev], C = lv[lev + 1];
  const int p1 = C.p, p2 = L.p, nt = L.nsh, np1 = 2 * p1 + 1;
  double2* Hs = hsm;                    // [np1 ND]
  double2* Hsc = Hs + np1 * ND;         // H1(j) rs1^(2|j|)
  double2* Ts = Hsc + np1 * ND;         // [2 nt + 1]
  double* R1 = reinterpret_cast<double*>(Ts + 2 * nt + 1);  // rs1^(2k), k <= max(p1, p2)
  const int tid = threadIdx.x, i = tid - p2;
  const bool act = tid < 2 * p2 + 1;
  const int ai = i < 0 ? -i : i;
  const int kmax = p1 > p2 ? p1 : p2;
  for (int k = tid; k <= kmax; k += blockDim.x) R1[k] = pow(C.rs, 2.0 * k);
  const double fi = pow(C.rs / L.rs, (double)ai);
  for (int bi = blockIdx.x; bi < n; bi += gridDim.x) {
    const int b = first + bi;
    if (t.nchild[b] == 0) continue;
    double2 acc[ND];
#pragma unroll
    for (int d = 0; d < ND; d++) acc[d] = make_double2(0, 0);
    const int4 ch = t.child[b];
    const int cc[4] = {ch.x, ch.y, ch.z, ch.w};
    for (int q = 0; q < 4; q++) {
      const int k = cc[q];
      if (t.srng[k].y <= t.srng[k].x) continue;  // block-uniform
      const double2* H1 = hexp(mp, C, k, ND);
      const double2* Tg = tabs + L.tm2m + (size_t)q * (2 * nt + 1);
      __syncthreads();  // R1 ready / the previous child is consumed
      for (int e = tid; e < np1 * ND; e += blockDim.x) {
        double2 h = H1[e];
        int jj = e / ND - p1;
        Hs[e] = h;
        Hsc[e] = cscale(h, R1[jj < 0 ? -jj : jj]);
      }
      for (int e = tid; e <= 2 * nt; e += blockDim.x) Ts[e] = Tg[e];
      __syncthreads();
      if (!act) continue;
      const double2* T = Ts + nt;
      if (i == 0) {
        for (int jj = -p1; jj <= p1; jj++) {
#pragma unroll
          for (int d = 0; d < ND; d++) cfma(acc[d], Hsc[(jj + p1) * ND + d], T[-jj]);
        }
        continue;
      }
      // opposite sign or j = 0: rs1^(2|j|); same sign, |j| <= |i|: 1;
      // same sign, |j| > |i|: rs1^(2(|j| - |i|))
      const int sg = i > 0 ? 1 : -1;
      for (int aj = 0; aj <= p1; aj++) {
        int jj = -sg * aj;
#pragma unroll
        for (int d = 0; d < ND; d++) cfma(acc[d], Hsc[(jj + p1) * ND + d], T[i - jj]);
      }
      for (int aj = 1; aj <= p1; aj++) {
        int jj = sg * aj;
        double2 tt = T[i - jj];
        if (aj > ai) tt = cscale(tt, R1[aj - ai]);
#pragma unroll
        for (int d = 0; d < ND; d++) cfma(acc[d], Hs[(jj + p1) * ND + d], tt);
      }
    }
    if (act) {
      double2* M = hexp(mp, L, b, ND);
#pragma unroll
      for (int d = 0; d < ND; d++) M[(i + p2) * ND + d] = cscale(acc[d], fi);
    }
    __syncthreads();
  }
}

// The same M2M with the child slots folded together.  The slots' tables
// differ only by the phases of their offsets' angles, multiples of pi/2
// apart: T_q(m) = T_3(m) (-i)^(m k_q), k_q = 2, 3, 1, 0 for the slots (-,-),
// (+,-), (-,+), (+,+).  So sum_q sum_j T_q(i-j) H_q(j) = sum_j T_3(i-j)
// S_((i-j) mod 4)(j) with the four-point sums S_m = sum_q (-i)^(m k_q) H_q
// (and their rs1^(2|j|)-scaled copies): one staging round and one pass over
// j per parent instead of four (a child without sources adds nothing: it
// is left out of the sums).  For one or two densities (the staged sums take
// four times the shared memory of one child).
template <int ND>
__global__ void __launch_bounds__(128) k_h_m2m_sym(TV t, const HLev* __restrict__ lv, int lev,
                                                   int first, int n,
                                                   const double2* __restrict__ tabs,
                                                   double2* __restrict__ mp) {
  extern __shared__ double2 hsm[];
  const HLev L = lv[lev], C = lv[lev + 1];
  const int p1 = C.p, p2 = L.p, nt = L.nsh, np1 = 2 * p1 + 1, NS = np1 * ND;
  double2* Sh = hsm;            // [m][np1 ND]
  double2* Sc = Sh + 4 * NS;    // the same, times rs1^(2|j|)
  double2* Ts = Sc + 4 * NS;    // slot (+,+)'s table [2 nt + 1]
  double* R1 = reinterpret_cast<double*>(Ts + 2 * nt + 1);  // rs1^(2k), k <= max(p1, p2)
  const int tid = threadIdx.x, i = tid - p2;
  const bool act = tid < 2 * p2 + 1;
  const int ai = i < 0 ? -i : i;
  const int kmax = p1 > p2 ? p1 : p2;
  for (int k = tid; k <= kmax; k += blockDim.x) R1[k] = pow(C.rs, 2.0 * k);
  for (int e = tid; e <= 2 * nt; e += blockDim.x) Ts[e] = tabs[L.tm2m + 3 * (2 * nt + 1) + e];
  const double fi = pow(C.rs / L.rs, (double)ai);
  const double2 z = make_double2(0, 0);
  for (int bi = blockIdx.x; bi < n; bi += gridDim.x) {
    const int b = first + bi;
    if (t.nchild[b] == 0) continue;
    const int4 ch = t.child[b];
    const bool h0 = t.srng[ch.x].y > t.srng[ch.x].x, h1 = t.srng[ch.y].y > t.srng[ch.y].x;
    const bool h2 = t.srng[ch.z].y > t.srng[ch.z].x, h3 = t.srng[ch.w].y > t.srng[ch.w].x;
    const double2* H0 = hexp(mp, C, ch.x, ND);
    const double2* H1 = hexp(mp, C, ch.y, ND);
    const double2* H2 = hexp(mp, C, ch.z, ND);
    const double2* H3 = hexp(mp, C, ch.w, ND);
    __syncthreads();  // tables ready / the previous parent is consumed
    for (int e = tid; e < NS; e += blockDim.x) {
      const double2 x0 = h0 ? H0[e] : z, x1 = h1 ? H1[e] : z;
      const double2 x2 = h2 ? H2[e] : z, x3 = h3 ? H3[e] : z;
      const double2 a = cadd(x3, x0), bb = cadd(x1, x2), c = csub(x3, x0), dd = csub(x1, x2);
      const double2 s0 = cadd(a, bb), s2 = csub(a, bb);
      const double2 s1 = make_double2(c.x - dd.y, c.y + dd.x);  // c + i dd
      const double2 s3 = make_double2(c.x + dd.y, c.y - dd.x);  // c - i dd
      const int jj = e / ND - p1;
      const double r = R1[jj < 0 ? -jj : jj];
      Sh[e] = s0;
      Sh[NS + e] = s1;
      Sh[2 * NS + e] = s2;
      Sh[3 * NS + e] = s3;
      Sc[e] = cscale(s0, r);
      Sc[NS + e] = cscale(s1, r);
      Sc[2 * NS + e] = cscale(s2, r);
      Sc[3 * NS + e] = cscale(s3, r);
    }
    __syncthreads();
    if (!act) continue;
    const double2* T = Ts + nt;
    double2 acc[ND];
#pragma unroll
    for (int d = 0; d < ND; d++) acc[d] = make_double2(0, 0);
    if (i == 0) {
      for (int jj = -p1; jj <= p1; jj++) {
        const double2* S = Sc + ((-jj) & 3) * NS + (jj + p1) * ND;
#pragma unroll
        for (int d = 0; d < ND; d++) cfma(acc[d], S[d], T[-jj]);
      }
    } else {
      // opposite sign or j = 0: rs1^(2|j|); same sign, |j| <= |i|: 1;
      // same sign, |j| > |i|: rs1^(2(|j| - |i|))
      const int sg = i > 0 ? 1 : -1;
      for (int aj = 0; aj <= p1; aj++) {
        const int jj = -sg * aj;
        const double2* S = Sc + ((i - jj) & 3) * NS + (jj + p1) * ND;
#pragma unroll
        for (int d = 0; d < ND; d++) cfma(acc[d], S[d], T[i - jj]);
      }
      for (int aj = 1; aj <= p1; aj++) {
        const int jj = sg * aj;
        double2 tt = T[i - jj];
        if (aj > ai) tt = cscale(tt, R1[aj - ai]);
        const double2* S = Sh + ((i - jj) & 3) * NS + (jj + p1) * ND;
#pragma unroll
        for (int d = 0; d < ND; d++) cfma(acc[d], S[d], tt);
      }
    }
    double2* M = hexp(mp, L, b, ND);
#pragma unroll
    for (int d = 0; d < ND; d++) M[(i + p2) * ND + d] = cscale(acc[d], fi);
  }
}

// step 4: M2L over list 2 (same level: rs1 = rs2, (rs2/rs1)^|i| = 1).
// One block per target box, one thread per output coefficient i; for every
// list-2 source the block stages its multipole (plain and scaled by
// rs^(2|j|)) and the (level, offset) kernel table in shared memory, then
//   L(i) += sum_j H(j) T(i-j) rs^(2 min(|i|,|j|)) [i, j of the same sign]
// with the rscale factor folded into three j ranges (h2dmploc).
template <int ND>
__global__ void __launch_bounds__(128) k_h_m2l(TV t, const HLev* __restrict__ lv, int first, int n,
                                               const double2* __restrict__ tabs,
                                               const double2* __restrict__ mp,
                                               double2* __restrict__ lo, int maxp) {
  extern __shared__ double2 hsm[];
  double2* Hs = hsm;                               // [(2 maxp + 1) ND]
  double2* Hsc = Hs + (2 * maxp + 1) * ND;         // H(j) rs^(2|j|)
  double2* Ts = Hsc + (2 * maxp + 1) * ND;         // [4 maxp + 1]
  double* RS2 = reinterpret_cast<double*>(Ts + 4 * maxp + 1);  // rs^(2k), k <= maxp
  const int tid = threadIdx.x;
  for (int bi = blockIdx.x; bi < n; bi += gridDim.x) {
    const int b = first + bi;
    const int n2 = t.nl2[b];
    if (n2 == 0 || !t.has_eval_pts(b)) continue;
    const int lev = t.level[b];
    const HLev L = lv[lev];
    if (!L.ok || L.wide) continue;
    const int p = L.p, np = 2 * p + 1, nt = 2 * p;
    const int i = tid - p;
    const bool act = tid < np;
    __syncthreads();  // the previous box is done with the shared arrays
    for (int k = tid; k <= p; k += blockDim.x) RS2[k] = pow(L.rs, 2.0 * k);
    double2 acc1[ND], acc2[ND];
#pragma unroll
    for (int d = 0; d < ND; d++) acc1[d] = acc2[d] = make_double2(0, 0);
    const double2 cb = t.center[b];
    const double rinv = 1.0 / L.bs;
    for (int e = 0; e < n2; e++) {
      const int jb = t.l2[(size_t)MNLIST2 * b + e];
      const double2 cj = t.center[jb];
      const int ox = __double2int_rn((cb.x - cj.x) * rinv);
      const int oy = __double2int_rn((cb.y - cj.y) * rinv);
      const double2* Tg = tabs + L.tm2l + (size_t)((ox + 3) * 7 + (oy + 3)) * (2 * nt + 1);
      const double2* H = hexp(const_cast<double2*>(mp), L, jb, ND);
      __syncthreads();  // RS2 written / previous source consumed
      for (int k = tid; k < np * ND; k += blockDim.x) {
        double2 h = H[k];
        int jj = k / ND - p;
        Hs[k] = h;
        Hsc[k] = cscale(h, RS2[jj < 0 ? -jj : jj]);
      }
      for (int k = tid; k <= 2 * nt; k += blockDim.x) Ts[k] = Tg[k];
      __syncthreads();
      if (act) {
        const double2* T = Ts + nt;  // T[k], k = -nt..nt
        int a0, a1, b0, b1, c0, c1;  // plain, scaled, constant-factor j ranges
        if (i >= 0) {
          a0 = -p; a1 = 0; b0 = 1; b1 = i; c0 = i + 1; c1 = p;
        } else {
          a0 = 0; a1 = p; b0 = i; b1 = -1; c0 = -p; c1 = i - 1;
        }
        for (int jj = a0; jj <= a1; jj++) {
          double2 tt = T[i - jj];
#pragma unroll
          for (int d = 0; d < ND; d++) cfma(acc1[d], Hs[(jj + p) * ND + d], tt);
        }
        for (int jj = b0; jj <= b1; jj++) {
          double2 tt = T[i - jj];
#pragma unroll
          for (int d = 0; d < ND; d++) cfma(acc1[d], Hsc[(jj + p) * ND + d], tt);
        }
        for (int jj = c0; jj <= c1; jj++) {
          double2 tt = T[i - jj];
#pragma unroll
          for (int d = 0; d < ND; d++) cfma(acc2[d], Hs[(jj + p) * ND + d], tt);
        }
      }
    }
    if (act) {
      double2* Lo = hexp(lo, L, b, ND);
      const double f = RS2[i < 0 ? -i : i];
#pragma unroll
      for (int d = 0; d < ND; d++)
        Lo[(i + p) * ND + d] = cadd(Lo[(i + p) * ND + d], cadd(acc1[d], cscale(acc2[d], f)));
    }
  }
}

// step 5: L2L from the parents of one level.  One block per parent, one
// thread per output coefficient i of the children; the parent's local
// expansion is staged once, each child slot's kernel table per child:
//   J2(i) += sum_j J1(j) T(i-j) F(i, j),  F = 1 for i = 0,
//   (rs1 rs2)^|i| for j of the other sign or j = 0,
//   (rs2/rs1)^|i| rs1^(2 max(0, |i| - |j|)) for j of the sign of i  (h2dlocloc)
template <int ND>
__global__ void __launch_bounds__(128) k_h_l2l(TV t, const HLev* __restrict__ lv, int lev, int first,
                                               int n, const double2* __restrict__ tabs,
                                               double2* __restrict__ lo) {
  extern __shared__ double2 hsm[];
  const HLev L = lv[lev], C = lv[lev + 1];
  const int p1 = L.p, p2 = C.p, nt = L.nsh, np1 = 2 * p1 + 1;
  double2* Js = hsm;                    // [np1 ND]
  double2* Ts = Js + np1 * ND;          // [4][2 nt + 1]
  double* R1 = reinterpret_cast<double*>(Ts + 4 * (2 * nt + 1));  // rs1^(2k), k <= p2
  const int tid = threadIdx.x, i = tid - p2;
  const bool act = tid < 2 * p2 + 1;
  const int ai = i < 0 ? -i : i;
  const double rs1 = L.rs, rs2 = C.rs;
  for (int k = tid; k <= p2; k += blockDim.x) R1[k] = pow(rs1, 2.0 * k);
  for (int e = tid; e < 4 * (2 * nt + 1); e += blockDim.x) Ts[e] = tabs[L.tl2l + e];
  const double A = pow(rs2 / rs1, (double)ai), Cf = pow(rs1 * rs2, (double)ai);
  for (int bi = blockIdx.x; bi < n; bi += gridDim.x) {
    const int b = first + bi;
    if (t.nchild[b] == 0 || !t.has_eval_pts(b)) continue;
    const double2* J1 = hexp(lo, L, b, ND);
    __syncthreads();  // tables ready / the previous parent is consumed
    for (int e = tid; e < np1 * ND; e += blockDim.x) Js[e] = J1[e];
    __syncthreads();
    if (!act) continue;
    const int4 ch = t.child[b];
    const int cc[4] = {ch.x, ch.y, ch.z, ch.w};
    for (int q = 0; q < 4; q++) {
      const double2* T = Ts + (size_t)q * (2 * nt + 1) + nt;
      double2 acc[ND], accc[ND], acca[ND];
#pragma unroll
      for (int d = 0; d < ND; d++) acc[d] = accc[d] = acca[d] = make_double2(0, 0);
      if (i == 0) {
        for (int jj = -p1; jj <= p1; jj++) {
#pragma unroll
          for (int d = 0; d < ND; d++) cfma(acc[d], Js[(jj + p1) * ND + d], T[-jj]);
        }
      } else {
        const int sg = i > 0 ? 1 : -1;
        for (int aj = 0; aj <= p1; aj++) {  // other sign and j = 0
          int jj = -sg * aj;
#pragma unroll
          for (int d = 0; d < ND; d++) cfma(accc[d], Js[(jj + p1) * ND + d], T[i - jj]);
        }
        for (int aj = 1; aj <= p1; aj++) {  // same sign
          int jj = sg * aj;
          double2 tt = T[i - jj];
          if (aj < ai) tt = cscale(tt, R1[ai - aj]);
#pragma unroll
          for (int d = 0; d < ND; d++) cfma(acca[d], Js[(jj + p1) * ND + d], tt);
        }
      }
      double2* J2 = hexp(lo, C, cc[q], ND);
#pragma unroll
      for (int d = 0; d < ND; d++) {
        double2 v = cadd(acc[d], cadd(cscale(accc[d], Cf), cscale(acca[d], A)));
        J2[(i + p2) * ND + d] = cadd(J2[(i + p2) * ND + d], v);
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Wideband levels (src/helmholtz/wideband2d.f, hfmm2d.f:1051-1097,
// 1124-1208, 1279-1285).  With unit scales every translation is the linear
// convolution out(i) = sum_j in(j) T(i-j) of the expansion with the shift's
// table T(k), k = -nt..nt.  An expansion placed at indices k mod nsig
// (nsig >= 2 nt + 1, 5-smooth) and Fourier transformed is its signature;
// the translation is then a pointwise product with the transformed table
// (divided by nsig), and the backward transform gives the expansion back.
// ---------------------------------------------------------------------------
struct TvJob {
  long out;
  int nsig, nt, bessel;  // bessel: J tables (shifts), else H (M2L)
  double x, y;           // centre shift c2 - c1
};

// One block per operator (h2d_mkm2ltrans / h2d_mkmpshift).
__global__ void __launch_bounds__(256) k_hf_transvec(const TvJob* __restrict__ jobs, double zkr,
                                                     double zki, double2* __restrict__ tabs) {
  extern __shared__ __align__(16) double2 fsm[];
  const TvJob J = jobs[blockIdx.x];
  fft::Plan P;
  fft::plan(J.nsig, P);
  double2* X = fsm;
  double2* Y = X + J.nsig;  // holds the values Z_k first (nt + 2 <= nsig)
  const double pi = 3.14159265358979323846;
  if (threadIdx.x == 0) {
    const double r = sqrt(J.x * J.x + J.y * J.y);
    const double2 z = make_double2(zkr * r, zki * r);
    if (J.bessel)
      jscaled(J.nt, z, 1.0, Y);
    else
      hscaled(J.nt + 1, z, 1.0, Y);
  }
  const double th = atan2(J.y, J.x) - pi;
  const double inv = 1.0 / J.nsig;
  for (int k = threadIdx.x; k < J.nsig; k += blockDim.x) X[k] = make_double2(0, 0);
  __syncthreads();
  for (int j = threadIdx.x; j <= J.nt; j += blockDim.x) {
    double sn, cs;
    sincos(j * th, &sn, &cs);
    const double2 zj = cscale(Y[j], inv);
    X[j] = cmul(make_double2(cs, -sn), zj);  // exp(-i theta)^j Z_j
    if (j > 0) {
      double2 t = cmul(make_double2(cs, sn), zj);  // (-conj e)^j Z_j
      if (j & 1) t = make_double2(-t.x, -t.y);
      X[J.nsig - j] = t;
    }
  }
  const double2* R = fft::block_fft(P, X, Y, -1);
  for (int k = threadIdx.x; k < J.nsig; k += blockDim.x) tabs[J.out + k] = R[k];
}

// x[k mod nsig] = E(k), k = -p..p (density d), zero elsewhere.
__device__ __forceinline__ void hf_pack(const double2* __restrict__ E, int p, int ND, int d,
                                        double2* x, int nsig) {
  for (int k = threadIdx.x; k < nsig; k += blockDim.x) {
    int i = k <= p ? k : (k >= nsig - p ? k - nsig : p + 1);
    x[k] = i <= p ? E[(size_t)(i + p) * ND + d] : make_double2(0, 0);
  }
}

// E(i) += x[i mod nsig], i = -p..p (density d).
__device__ __forceinline__ void hf_unpack_add(const double2* x, int nsig, double2* E, int p,
                                              int ND, int d) {
  for (int i = (int)threadIdx.x - p; i <= p; i += blockDim.x) {
    const int k = i >= 0 ? i : nsig + i;
    double2* e = E + (size_t)(i + p) * ND + d;
    *e = cadd(*e, x[k]);
  }
}

// Signatures of the multipoles of one wideband level (h2d_mptosig).
template <int ND>
__global__ void __launch_bounds__(256) k_hf_tosig(const HLev* __restrict__ lv, int lev, int first,
                                                  int n, const double2* __restrict__ mp,
                                                  double2* __restrict__ sig) {
  extern __shared__ __align__(16) double2 fsm[];
  const HLev L = lv[lev];
  fft::Plan P;
  fft::plan(L.nsig, P);
  double2* X = fsm;
  double2* Y = X + L.nsig;
  for (int bi = blockIdx.x; bi < n; bi += gridDim.x) {
    const int b = first + bi;
    const double2* E = hexp(const_cast<double2*>(mp), L, b, ND);
    double2* S = sig + (L.sig_off + (size_t)(b - L.lfirst) * L.nsig) * ND;
    for (int d = 0; d < ND; d++) {
      hf_pack(E, L.p, ND, d, X, L.nsig);
      const double2* R = fft::block_fft(P, X, Y, -1);
      for (int k = threadIdx.x; k < L.nsig; k += blockDim.x) S[(size_t)k * ND + d] = R[k];
      __syncthreads();
    }
  }
}

// M2L of one wideband level: products of the list-2 signatures with the
// offset's operator, summed, transformed back and added to the local
// expansion (h2d_diagtrans, h2d_sig2exp).
template <int ND>
__global__ void __launch_bounds__(256) k_hf_m2l(TV t, const HLev* __restrict__ lv, int lev, int first,
                                                int n, const double2* __restrict__ sig,
                                                const double2* __restrict__ tabs,
                                                double2* __restrict__ lo) {
  extern __shared__ __align__(16) double2 fsm[];
  const HLev L = lv[lev];
  fft::Plan P;
  fft::plan(L.nsig, P);
  double2* X = fsm;
  double2* Y = X + L.nsig;
  const double rinv = 1.0 / L.bs;
  for (int bi = blockIdx.x; bi < n; bi += gridDim.x) {
    const int b = first + bi;
    const int n2 = t.nl2[b];
    if (n2 == 0 || !t.has_eval_pts(b)) continue;
    const double2 cb = t.center[b];
    for (int d = 0; d < ND; d++) {
      for (int k = threadIdx.x; k < L.nsig; k += blockDim.x) {
        double2 acc = make_double2(0, 0);
        for (int e = 0; e < n2; e++) {
          const int jb = t.l2[(size_t)MNLIST2 * b + e];
          const double2 cj = t.center[jb];
          const int ox = __double2int_rn((cb.x - cj.x) * rinv);
          const int oy = __double2int_rn((cb.y - cj.y) * rinv);
          const double2 tv = tabs[L.tv_m2l + (size_t)((ox + 3) * 7 + (oy + 3)) * L.nsig + k];
          const double2 sj = sig[(L.sig_off + (size_t)(jb - L.lfirst) * L.nsig + k) * ND + d];
          cfma(acc, tv, sj);
        }
        X[k] = acc;
      }
      const double2* R = fft::block_fft(P, X, Y, +1);
      hf_unpack_add(R, L.nsig, hexp(lo, L, b, ND), L.p, ND, d);
      __syncthreads();
    }
  }
}

// One shift between a wideband level and the next through signatures:
// dst(-p2..p2) += backward(op * forward(src(-p1..p1))).
template <int ND>
__device__ void hf_shift(const fft::Plan& P, const double2* src, int p1, const double2* op,
                         double2* dst, int p2, double2* X, double2* Y) {
  for (int d = 0; d < ND; d++) {
    hf_pack(src, p1, ND, d, X, P.n);
    double2* R = fft::block_fft(P, X, Y, -1);
    double2* W = R == X ? Y : X;
    for (int k = threadIdx.x; k < P.n; k += blockDim.x) R[k] = cmul(R[k], op[k]);
    const double2* B = fft::block_fft(P, R, W, +1);
    hf_unpack_add(B, P.n, dst, p2, ND, d);
    __syncthreads();
  }
}

// M2M into the parents of one wideband level (h2dmpmphf + h2d_sig2exp).
template <int ND>
__global__ void __launch_bounds__(256) k_hf_m2m(TV t, const HLev* __restrict__ lv, int lev, int first,
                                                int n, const double2* __restrict__ tabs,
                                                double2* __restrict__ mp) {
  extern __shared__ __align__(16) double2 fsm[];
  const HLev L = lv[lev], C = lv[lev + 1];
  fft::Plan P;
  fft::plan(L.nsig_sh, P);
  double2* X = fsm;
  double2* Y = X + L.nsig_sh;
  for (int bi = blockIdx.x; bi < n; bi += gridDim.x) {
    const int b = first + bi;
    if (t.nchild[b] == 0) continue;
    double2* M = hexp(mp, L, b, ND);
    for (int e = threadIdx.x; e < L.P * ND; e += blockDim.x) M[e] = make_double2(0, 0);
    __syncthreads();
    const int4 ch = t.child[b];
    const int cc[4] = {ch.x, ch.y, ch.z, ch.w};
    for (int q = 0; q < 4; q++) {
      const int k = cc[q];
      if (k < 0 || t.srng[k].y <= t.srng[k].x) continue;
      hf_shift<ND>(P, hexp(mp, C, k, ND), C.p, tabs + L.tv_mm + (size_t)q * L.nsig_sh, M, L.p, X,
                   Y);
    }
  }
}

// L2L from the parents of one wideband level (h2dloclochf).
template <int ND>
__global__ void __launch_bounds__(256) k_hf_l2l(TV t, const HLev* __restrict__ lv, int lev, int first,
                                                int n, const double2* __restrict__ tabs,
                                                double2* __restrict__ lo) {
  extern __shared__ __align__(16) double2 fsm[];
  const HLev L = lv[lev], C = lv[lev + 1];
  fft::Plan P;
  fft::plan(L.nsig_sh, P);
  double2* X = fsm;
  double2* Y = X + L.nsig_sh;
  for (int bi = blockIdx.x; bi < n; bi += gridDim.x) {
    const int b = first + bi;
    if (t.nchild[b] == 0 || !t.has_eval_pts(b)) continue;
    const double2* J1 = hexp(lo, L, b, ND);
    const int4 ch = t.child[b];
    const int cc[4] = {ch.x, ch.y, ch.z, ch.w};
    for (int q = 0; q < 4; q++) {
      if (cc[q] < 0) continue;
      hf_shift<ND>(P, J1, L.p, tabs + L.tv_ll + (size_t)q * L.nsig_sh, hexp(lo, C, cc[q], ND), C.p,
                   X, Y);
    }
  }
}

// Pair term of the near field (helmkernels2d.f h2d_directcdh, cdg, ...).
template <int ND, int IFPGH>
__device__ __forceinline__ void h_pair(double xd, double yd, double2 zk, const double2* q,
                                       const double2* dd, const double* v, bool hq, bool hd,
                                       double2 pot[ND], double2 g1[ND], double2 g2[ND],
                                       double2 hh[ND][3]) {
  double rr = xd * xd + yd * yd, r = sqrt(rr);
  double2 z = make_double2(zk.x * r, zk.y * r);
  double2 h0, h1;
  helm::hank01(z, h0, h1);
  const double2 i4 = make_double2(0, 0.25);
  double ir = 1.0 / r;
  double ct = xd * ir, st = yd * ir;
  double2 zki4 = cmul(zk, i4);
  if (hq) {
    double2 cdd = cscale(cmul(h1, zki4), -ir);  // -h1 zk i/4 / r
    double2 h2z = csub(cscale(h1, 2.0), cmul(z, h0));
    double2 chs = cscale(zki4, ir / rr);
#pragma unroll
    for (int d = 0; d < ND; d++) {
      pot[d] = cadd(pot[d], cmul(cmul(h0, i4), q[d]));
      if (IFPGH >= 2) {
        double2 c = cmul(cdd, q[d]);
        g1[d] = cadd(g1[d], cscale(c, xd));
        g2[d] = cadd(g2[d], cscale(c, yd));
      }
      if (IFPGH >= 3) {
        double2 c = cmul(chs, q[d]);
        hh[d][0] = cadd(hh[d][0], cmul(c, csub(cscale(h2z, xd * xd), cscale(h1, rr))));
        hh[d][1] = cadd(hh[d][1], cmul(c, cscale(h2z, xd * yd)));
        hh[d][2] = cadd(hh[d][2], cmul(c, csub(cscale(h2z, yd * yd), cscale(h1, rr))));
      }
    }
  }
  if (hd) {
    double2 zi = crcp(z);
    double2 h2 = csub(cscale(cmul(h1, zi), 2.0), h0);
    double2 cdd = cscale(cmul(h1, zki4), ir);      // h1 / r zk i/4
    double2 cdd2 = cmul(cmul(zk, zk), make_double2(0, -0.25));  // -zk^2 i/4
    double2 f1 = csub(cscale(h2, ct * ct - 0.5), cscale(h0, 0.5));
    double2 f2 = cscale(h2, ct * st);
    double2 f3 = csub(cscale(h2, st * st - 0.5), cscale(h0, 0.5));
#pragma unroll
    for (int d = 0; d < ND; d++) {
      double v1 = v[2 * d], v2 = v[2 * d + 1];
      pot[d] = cadd(pot[d], cscale(cmul(cdd, dd[d]), xd * v1 + yd * v2));
      if (IFPGH >= 2) {
        double2 c = cmul(cdd2, dd[d]);
        double2 hxx = cmul(c, f1), hxy = cmul(c, f2), hyy = cmul(c, f3);
        g1[d] = cadd(g1[d], cadd(cscale(hxx, v1), cscale(hxy, v2)));
        g2[d] = cadd(g2[d], cadd(cscale(hxy, v1), cscale(hyy, v2)));
      }
      if (IFPGH >= 3) {
        double2 h3 = csub(cscale(cmul(h2, zi), 4.0), h1);
        double2 a1 = cscale(csub(cscale(h1, 0.75), cscale(h3, 0.5 * (ct * ct - 0.5 - st * st))), ct);
        double2 a2 = cscale(csub(cscale(h1, 0.25), cscale(h3, 0.5 * (1.5 * ct * ct - 0.5 * st * st))), st);
        double2 a3 = cscale(csub(cscale(h1, 0.25), cscale(h3, 0.5 * (1.5 * st * st - 0.5 * ct * ct))), ct);
        double2 a4 = cscale(csub(cscale(h1, 0.75), cscale(h3, 0.5 * (st * st - 0.5 - ct * ct))), st);
        double2 c3 = cmul(cmul(cmul(zk, zk), zk), make_double2(0, -0.25));
        double2 c = cmul(c3, dd[d]);
        hh[d][0] = cadd(hh[d][0], cmul(c, cadd(cscale(a1, v1), cscale(a2, v2))));
        hh[d][1] = cadd(hh[d][1], cmul(c, cadd(cscale(a2, v1), cscale(a3, v2))));
        hh[d][2] = cadd(hh[d][2], cmul(c, cadd(cscale(a3, v1), cscale(a4, v2))));
      }
    }
  }
}

// Leaf box of every evaluation point (points are in tree order).
__global__ void k_h_point_leaf(TV t, int nb, int use_targets, int* __restrict__ leaf) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nb || t.nchild[b] != 0) return;
  int2 r = use_targets ? t.trng[b] : t.srng[b];
  for (int k = r.x; k < r.y; k++) leaf[k] = b;
}

// Coefficient n of the derivative expansions of mk_mpoleg / mk_mpoleh
// (helmrouts2d.f): with s1 = zk/(2s), s2 = zk s/2, s3 = i s1, s4 = i s2,
//   X(n) = [n+1 >= 1 ? s2 : s1] F(n+1) - [n-1 >= 0 ? s1 : s2] F(n-1),
//   Y(n) = [n+1 >= 1 ? s4 : s3] F(n+1) + [n-1 >= 0 ? s3 : s4] F(n-1);
// XX, XY come from X and YY from Y by the same rules.
struct DerivCoef {
  double2 s1, s2, s3, s4;
};

template <typename F>
__device__ __forceinline__ double2 rule_x(F f, int n, const DerivCoef& c) {
  double2 a = f(n + 1), b = f(n - 1);
  return csub(cmul(n + 1 >= 1 ? c.s2 : c.s1, a), cmul(n - 1 >= 0 ? c.s1 : c.s2, b));
}
template <typename F>
__device__ __forceinline__ double2 rule_y(F f, int n, const DerivCoef& c) {
  double2 a = f(n + 1), b = f(n - 1);
  return cadd(cmul(n + 1 >= 1 ? c.s4 : c.s3, a), cmul(n - 1 >= 0 ? c.s3 : c.s4, b));
}

// Adds sum_n V(n) mt(n) for V = E (and its derivative expansions) at one
// point, mt(0) = (i/4) Z_0, mt(n) = (i/4) Z_n e^{i n th}, mt(-n) = (i/4) Z_n
// (-e^{-i th})^n (mpole_evalp / h2dtaevalp, helmrouts2d.f:274-966), with the
// scaled Bessel (local, mpole = false) or Hankel (multipole) sequence Z of
// argument zz = zk r generated by its recurrence on the fly, no tables.
template <int ND, int IFPGH>
__device__ void eval_at_point(const double2* __restrict__ E, int p, double2 zk, double rs,
                              bool mpole, double2 zz, double2 ep, double2 po[ND], double2 g1[ND],
                              double2 g2[ND], double2 hh[ND][3]) {
  const int q = p + IFPGH - 1;  // highest order that contributes
  const double s = mpole ? rs : 1.0 / rs;
  DerivCoef c;
  c.s1 = cscale(zk, 0.5 / s);
  c.s2 = cscale(zk, 0.5 * s);
  c.s3 = make_double2(-c.s1.y, c.s1.x);
  c.s4 = make_double2(-c.s2.y, c.s2.x);
  const double2 i4 = make_double2(0.0, 0.25);
  auto contribute = [&](int m, double2 Zm, double2 epm) {
    // orders +m and -m share Z_m
    double2 base = cmul(Zm, i4);
    for (int sgn = 1; sgn >= -1; sgn -= 2) {
      if (m == 0 && sgn < 0) break;
      int n = sgn * m;
      double2 ph = sgn > 0 ? epm : cconj(epm);
      if (sgn < 0 && (m & 1)) ph = make_double2(-ph.x, -ph.y);
      double2 mt = cmul(base, ph);
#pragma unroll
      for (int d = 0; d < ND; d++) {
        auto Ef = [&](int k) {
          return (k >= -p && k <= p) ? E[(size_t)(k + p) * ND + d] : make_double2(0, 0);
        };
        if (m <= p) po[d] = cadd(po[d], cmul(Ef(n), mt));
        if (IFPGH >= 2) {
          g1[d] = cadd(g1[d], cmul(rule_x(Ef, n, c), mt));
          g2[d] = cadd(g2[d], cmul(rule_y(Ef, n, c), mt));
        }
        if (IFPGH >= 3) {
          auto Xf = [&](int k) { return rule_x(Ef, k, c); };
          auto Yf = [&](int k) { return rule_y(Ef, k, c); };
          hh[d][0] = cadd(hh[d][0], cmul(rule_x(Xf, n, c), mt));
          hh[d][1] = cadd(hh[d][1], cmul(rule_y(Xf, n, c), mt));
          hh[d][2] = cadd(hh[d][2], cmul(rule_y(Yf, n, c), mt));
        }
      }
    }
  };
  if (!mpole) {
    // scaled J, downward from the series start
    int M = 0;
    double2 f_hi, f_lo;
    if (!helm::jstart(q, zz, rs, M, f_hi, f_lo)) {
      contribute(0, make_double2(1, 0), make_double2(1, 0));
      return;
    }
    const int mtop = min(M, q);
    double2 epm = make_double2(1, 0);
    for (int k = 0; k < mtop; k++) epm = cmul(epm, ep);
    const double2 epc = cconj(ep);
    auto visit = [&](int m, double2 Zm) {
      if (m > q) return;
      contribute(m, Zm, epm);
      epm = cmul(epm, epc);
    };
    visit(M, f_hi);
    visit(M - 1, f_lo);
    const double2 cz = cscale(crcp(zz), 2.0 * rs);
    const double s2r = rs * rs;
    for (int n = M - 1; n >= 1; n--) {
      double2 nx = csub(cmul(cscale(cz, (double)n), f_lo), cscale(f_hi, s2r));
      f_hi = f_lo;
      f_lo = nx;
      visit(n - 1, nx);
    }
  } else {
    // scaled H, upward from H0, H1
    if (hypot(zz.x, zz.y) < 1e-200) return;
    double2 h0, h1;
    helm::hank01(zz, h0, h1);
    double2 zm1 = h0, zm = cscale(h1, rs);  // Z_0, Z_1
    contribute(0, h0, make_double2(1, 0));
    double2 epm = ep;
    if (q >= 1) contribute(1, zm, epm);
    const double2 cz = cscale(crcp(zz), 2.0 * rs);
    const double s2r = rs * rs;
    for (int m = 1; m < q; m++) {
      double2 nx = csub(cmul(cscale(cz, (double)m), zm), cscale(zm1, s2r));
      zm1 = zm;
      zm = nx;
      epm = cmul(epm, ep);
      contribute(m + 1, zm, epm);
    }
  }
}

// steps 6 and 7, one evaluation point per thread: L2P from its leaf's local
// expansion and M2P from the leaf's list-3 boxes; writes the outputs.
template <int ND, int IFPGH>
__global__ void __launch_bounds__(128) k_h_far(TV t, const HLev* __restrict__ lv, long n,
                                               const int* __restrict__ leaf,
                                               const double2* __restrict__ xe, HDens D, double zkr,
                                               double zki, const double2* __restrict__ mp,
                                               const double2* __restrict__ lo,
                                               double2* __restrict__ pot,
                                               double2* __restrict__ grad,
                                               double2* __restrict__ hess) {
  long k = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (k >= n) return;
  const double2 zk = make_double2(zkr, zki);
  const double azk = hypot(zkr, zki);
  const int b = leaf[k];
  const int lev = t.level[b];
  const double2 z = xe[k];
  double2 po[ND], g1[ND], g2[ND], hh[ND][3];
#pragma unroll
  for (int d = 0; d < ND; d++) {
    po[d] = g1[d] = g2[d] = make_double2(0, 0);
    hh[d][0] = hh[d][1] = hh[d][2] = make_double2(0, 0);
  }
  auto polar = [&](double2 c, double2& zz, double2& ep) {
    double dx = z.x - c.x, dy = z.y - c.y;
    double r = sqrt(dx * dx + dy * dy);
    double th = (dx == 0 && dy == 0) ? 0.0 : atan2(dy, dx);
    zz = make_double2(zk.x * r, zk.y * r);
    double sn, cs;
    sincos(th, &sn, &cs);
    ep = make_double2(cs, sn);
  };
  (void)azk;
  const HLev L = lv[lev];
  if (L.ok && lev >= 2) {
    double2 zz, ep;
    polar(t.center[b], zz, ep);
    eval_at_point<ND, IFPGH>(hexp(const_cast<double2*>(lo), L, b, ND), L.p, zk, L.rs, false, zz,
                             ep, po, g1, g2, hh);
  }
  const int n3 = t.nl3[b];
  for (int e = 0; e < n3; e++) {
    const HLev C = lv[lev + 1];
    if (!C.ok) break;
    int jb = t.l3[(size_t)MNLIST3 * b + e];
    double2 zz, ep;
    polar(t.center[jb], zz, ep);
    eval_at_point<ND, IFPGH>(hexp(const_cast<double2*>(mp), C, jb, ND), C.p, zk, C.rs, true, zz,
                             ep, po, g1, g2, hh);
  }
#pragma unroll
  for (int d = 0; d < ND; d++) {
    size_t o = (size_t)k * D.nd + D.d0 + d;
    pot[o] = po[d];
    if (IFPGH >= 2) {
      grad[((size_t)k * 2 + 0) * D.nd + D.d0 + d] = g1[d];
      grad[((size_t)k * 2 + 1) * D.nd + D.d0 + d] = g2[d];
    }
    if (IFPGH >= 3)
      for (int c = 0; c < 3; c++) hess[((size_t)k * 3 + c) * D.nd + D.d0 + d] = hh[d][c];
  }
}

// step 8, one evaluation point per thread: the sources of its leaf's list-1
// boxes (h2d_direct*), added to the far field already in the outputs.
template <int ND, int IFPGH>
__global__ void __launch_bounds__(128) k_h_p2p(TV t, long n, const int* __restrict__ leaf,
                                               const double2* __restrict__ xs,
                                               const double2* __restrict__ xe, HDens D,
                                               double zkr, double zki, double thresh,
                                               double2* __restrict__ pot,
                                               double2* __restrict__ grad,
                                               double2* __restrict__ hess) {
  long k = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (k >= n) return;
  const double2 zk = make_double2(zkr, zki);
  const double azk = hypot(zkr, zki);
  const bool hq = D.q != nullptr, hd = D.d != nullptr;
  const int b = leaf[k];
  const double2 z = xe[k];
  double2 po[ND], g1[ND], g2[ND], hh[ND][3];
#pragma unroll
  for (int d = 0; d < ND; d++) {
    po[d] = g1[d] = g2[d] = make_double2(0, 0);
    hh[d][0] = hh[d][1] = hh[d][2] = make_double2(0, 0);
  }
  // helmkernels2d.f: <= for the charge potential-only kernel, < otherwise
  const bool le = (IFPGH == 1) && hq && !hd;
  const int n1 = t.nl1[b];
  for (int e = 0; e < n1; e++) {
    int2 sr = t.srng[t.l1[(size_t)MNLIST1 * b + e]];
    for (int j = sr.x; j < sr.y; j++) {
      double2 y = xs[j];
      double xd = z.x - y.x, yd = z.y - y.y;
      double az = azk * sqrt(xd * xd + yd * yd);
      if (le ? (az <= thresh) : (az < thresh)) continue;
      double2 qv[ND], dv[ND];
      double vv[2 * ND];
#pragma unroll
      for (int d = 0; d < ND; d++) {
        qv[d] = hq ? D.q[(size_t)j * D.nd + D.d0 + d] : make_double2(0, 0);
        dv[d] = hd ? D.d[(size_t)j * D.nd + D.d0 + d] : make_double2(0, 0);
        vv[2 * d] = hd ? D.v[((size_t)j * 2 + 0) * D.nd + D.d0 + d] : 0.0;
        vv[2 * d + 1] = hd ? D.v[((size_t)j * 2 + 1) * D.nd + D.d0 + d] : 0.0;
      }
      h_pair<ND, IFPGH>(xd, yd, zk, qv, dv, vv, hq, hd, po, g1, g2, hh);
    }
  }
#pragma unroll
  for (int d = 0; d < ND; d++) {
    size_t o = (size_t)k * D.nd + D.d0 + d;
    pot[o] = cadd(pot[o], po[d]);
    if (IFPGH >= 2) {
      size_t o1 = ((size_t)k * 2 + 0) * D.nd + D.d0 + d, o2 = ((size_t)k * 2 + 1) * D.nd + D.d0 + d;
      grad[o1] = cadd(grad[o1], g1[d]);
      grad[o2] = cadd(grad[o2], g2[d]);
    }
    if (IFPGH >= 3)
      for (int c = 0; c < 3; c++) {
        size_t oc = ((size_t)k * 3 + c) * D.nd + D.d0 + d;
        hess[oc] = cadd(hess[oc], hh[d][c]);
      }
  }
}

__global__ void k_h_gather(const double* __restrict__ xy, const int* __restrict__ perm, long n,
                           int nd, const double* __restrict__ charge,
                           const double* __restrict__ dipstr, const double* __restrict__ dipvec,
                           double2* __restrict__ xs, double2* __restrict__ qs,
                           double2* __restrict__ ds, double* __restrict__ vs) {
  long k = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (k >= n) return;
  size_t i = perm[k];
  xs[k] = make_double2(xy[2 * i], xy[2 * i + 1]);
  for (int d = 0; d < nd; d++) {
    if (qs) qs[k * nd + d] = ((const double2*)charge)[i * nd + d];
    if (ds) {
      ds[k * nd + d] = ((const double2*)dipstr)[i * nd + d];
      vs[(k * 2 + 0) * nd + d] = dipvec[(i * 2 + 0) * nd + d];
      vs[(k * 2 + 1) * nd + d] = dipvec[(i * 2 + 1) * nd + d];
    }
  }
}

__global__ void k_h_unpack(const int* __restrict__ perm, long n, int w,
                           const double2* __restrict__ in, double2* __restrict__ out) {
  long k = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (k >= n) return;
  size_t i = perm[k];
  for (int c = 0; c < w; c++) out[i * w + c] = in[k * w + c];
}

// direct sums
template <int IFPGH>
__global__ void __launch_bounds__(128) k_h_direct(int nd, int d, long ns, const double* __restrict__ src,
                                                 const double* __restrict__ charge,
                                                 const double* __restrict__ dipstr,
                                                 const double* __restrict__ dipvec, long nt,
                                                 const double* __restrict__ trg, double zkr,
                                                 double zki, double thresh, long chunk,
                                                 double2* __restrict__ part) {
  __shared__ double sx[128], sy[128], sv[256];
  __shared__ double2 sq[128], sd[128];
  long tix = blockIdx.x * 128L + threadIdx.x;
  bool act = tix < nt;
  double x = act ? trg[2 * tix] : 0, y = act ? trg[2 * tix + 1] : 0;
  double2 po[1] = {make_double2(0, 0)}, g1[1] = {make_double2(0, 0)}, g2[1] = {make_double2(0, 0)};
  double2 hh[1][3] = {{make_double2(0, 0), make_double2(0, 0), make_double2(0, 0)}};
  long s0 = blockIdx.y * chunk, s1 = min(ns, s0 + chunk);
  bool hq = charge != nullptr, hd = dipstr != nullptr;
  double2 zk = make_double2(zkr, zki);
  double azk = hypot(zkr, zki);
  for (long b0 = s0; b0 < s1; b0 += 128) {
    __syncthreads();
    long j = b0 + threadIdx.x;
    if (j < s1) {
      sx[threadIdx.x] = src[2 * j];
      sy[threadIdx.x] = src[2 * j + 1];
      if (hq) sq[threadIdx.x] = ((const double2*)charge)[j * nd + d];
      if (hd) {
        sd[threadIdx.x] = ((const double2*)dipstr)[j * nd + d];
        sv[2 * threadIdx.x] = dipvec[(j * 2 + 0) * nd + d];
        sv[2 * threadIdx.x + 1] = dipvec[(j * 2 + 1) * nd + d];
      }
    }
    __syncthreads();
    int m = (int)min(128L, s1 - b0);
    if (act)
      for (int i = 0; i < m; i++) {
        double xd = x - sx[i], yd = y - sy[i];
        double az = azk * sqrt(xd * xd + yd * yd);
        bool le = (IFPGH == 1) && hq && !hd;
        if (le ? (az <= thresh) : (az < thresh)) continue;
        h_pair<1, IFPGH>(xd, yd, zk, &sq[i], &sd[i], &sv[2 * i], hq, hd, po, g1, g2, hh);
      }
  }
  if (act) {
    double2* o = part + ((size_t)blockIdx.y * nt + tix) * 6;
    o[0] = po[0];
    o[1] = g1[0];
    o[2] = g2[0];
    o[3] = hh[0][0];
    o[4] = hh[0][1];
    o[5] = hh[0][2];
  }
}

__global__ void k_h_direct_reduce(int nd, int d, long nt, int nslice, int ifpgh,
                                  const double2* __restrict__ part, double2* pot, double2* grad,
                                  double2* hess) {
  long tix = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (tix >= nt) return;
  double2 o[6];
  for (int c = 0; c < 6; c++) o[c] = make_double2(0, 0);
  for (int s = 0; s < nslice; s++)
    for (int c = 0; c < 6; c++) o[c] = cadd(o[c], part[((size_t)s * nt + tix) * 6 + c]);
  pot[tix * nd + d] = o[0];
  if (ifpgh >= 2) {
    grad[(tix * 2 + 0) * nd + d] = o[1];
    grad[(tix * 2 + 1) * nd + d] = o[2];
  }
  if (ifpgh >= 3)
    for (int c = 0; c < 3; c++) hess[(tix * 3 + c) * nd + d] = o[3 + c];
}

template <typename K>
void set_smem(K kernel, size_t bytes) {
  if (bytes > 48 * 1024)
    set_smem_attr(kernel, bytes);
}

int grid_w(long nitems, int wpb) {
  long blocks = (nitems + wpb - 1) / wpb;
  return (int)std::max(1L, std::min(blocks, 148L * 32));
}

// Per-level expansion orders and scales, the expansion layout and the
// translation tables of one tree (hfmm2d.f:317-326 for orders and scales).
struct HelmLevels {
  std::vector<HLev> hl;
  int maxp = 0;      // largest order at levels >= 2 of the coefficient-per-lane kernels
  int maxp_all = 0;  // largest order at levels >= 2
  long off = 0;      // expansion storage per density (double2 units)
  long sig_total = 0;  // M2L signatures of the wideband levels per density
  int maxsig = 0;      // longest signature
  DBuf<HLev> dlv;
  DBuf<double2> tabs;
  DBuf<double> dbs;  // box sizes, one level past the deepest
  explicit HelmLevels(cudaStream_t st) : dlv(st), tabs(st), dbs(st) {}
};

// ier 13: an order the kernels do not support (above HMAXP with a scale
// below 1, or a signature longer than HF_MAXSIG).
int helm_levels(const DeviceTree& T, double zkr, double zki, double eps, HelmLevels& H,
                cudaStream_t st) {
  const int nl = T.nlevels;
  const double pi = 4 * std::atan(1.0);
  const double zkabs = std::hypot(zkr, zki);
  std::vector<HLev>& hl = H.hl;
  hl.assign(nl + 1, HLev{});
  int maxp = 0, maxp_all = 0, ier = 0;
  for (int l = 0; l <= nl; l++) {
    double bs = T.boxsize[l];
    hl[l].lfirst = T.lfirst[l];
    hl[l].rs = std::min(zkabs * bs / (2.0 * pi), 1.0);
    hl[l].bs = bs;
    hl[l].p = helm_nterms(bs, zkr, zki, eps, &ier);
    hl[l].P = 2 * hl[l].p + 1;
    hl[l].ok = (zki * bs < 40.0) ? 1 : 0;
    // boxes above 16 wavelengths take the diagonal (signature) translations
    // (hfmm2d.f:1001-1013, 1124-1208); so do orders beyond the
    // coefficient-per-lane kernels, where the scale is 1 as well and the two
    // forms are the same convolution
    const bool hf = bs / (1.0 / (zkr / (2.0 * pi))) > 16.0;
    hl[l].wide = (l >= 2 && hl[l].ok && (hf || hl[l].p > HMAXP)) ? 1 : 0;
    if (l >= 2 && hl[l].ok) {
      if (hl[l].wide)
        maxp_all = std::max(maxp_all, hl[l].p);
      else
        maxp = std::max(maxp, hl[l].p);
    }
  }
  if (ier) return ier;
  if (maxp > HMAXP) return IER_NTERMS;
  maxp_all = std::max(maxp_all, maxp);
  for (int l = 2; l <= nl; l++) {
    HLev& L = hl[l];
    if (!L.wide) continue;
    // the signature form holds for unit scales only (rscale = 1 in
    // wideband2d.f); shifts also need the child level's scale to be 1
    if (L.rs != 1.0 || (l < nl && hl[l + 1].ok && hl[l + 1].rs != 1.0)) return IER_NTERMS;
    L.nsig = fft::next235(2 * (L.p + L.p) + 1);
    L.nsig_sh = l < nl ? fft::next235(2 * (L.p + hl[l + 1].p) + 1) : 0;
    if (L.nsig > HF_MAXSIG || L.nsig_sh > HF_MAXSIG) return IER_NTERMS;
  }
  H.maxp = maxp;
  H.maxp_all = maxp_all;
  // expansion and table layout
  long off = 0, toff = 0, soff = 0;
  for (int l = 0; l <= nl; l++) {
    HLev& L = hl[l];
    const long nbl = (long)(T.llast[l] - T.lfirst[l] + 1);
    L.off = off;
    off += nbl * L.P;
    L.nsh = l < nl ? L.p + hl[l + 1].p : 0;
    L.tm2l = toff;
    if (l >= 2 && !L.wide) toff += 49L * (4 * L.p + 1);
    L.tm2m = toff;
    if (l < nl && !L.wide) toff += 4L * (2 * L.nsh + 1);
    L.tl2l = toff;
    if (l < nl && !L.wide) toff += 4L * (2 * L.nsh + 1);
    if (L.wide) {
      L.tv_m2l = toff;
      toff += 49L * L.nsig;
      L.tv_mm = toff;
      if (l < nl) toff += 4L * L.nsig_sh;
      L.tv_ll = toff;
      if (l < nl) toff += 4L * L.nsig_sh;
      L.sig_off = soff;
      soff += nbl * L.nsig;
    }
  }
  H.sig_total = soff;
  H.off = off;
  H.dlv.alloc(nl + 1, st);
  B2_CHECK(cudaMemcpyAsync(H.dlv.p, hl.data(), sizeof(HLev) * (nl + 1), cudaMemcpyHostToDevice, st));
  DBuf<double2> scratch(st);
  H.tabs.alloc(std::max(toff, 1L), st);
  const int nthreads = (nl + 1) * 57, sstride = 2 * (2 * HMAXP) + 8;
  scratch.alloc((size_t)nthreads * sstride, st);
  k_h_tables<<<ceil_div(nthreads, 64), 64, 0, st>>>(H.dlv.p, nl, zkr, zki, H.tabs.p, scratch.p,
                                                    sstride);
  B2_LAUNCH_CHECK();
  // diagonal operators of the wideband levels: M2L per offset (target -
  // source = o bs), M2M per child slot (parent - child), L2L (child - parent)
  std::vector<TvJob> jobs;
  int maxsig = 0;
  for (int l = 2; l <= nl; l++) {
    const HLev& L = hl[l];
    if (!L.wide) continue;
    for (int k = 0; k < 49; k++) {
      const int ox = k / 7 - 3, oy = k % 7 - 3;
      if (ox >= -1 && ox <= 1 && oy >= -1 && oy <= 1) continue;
      jobs.push_back(TvJob{L.tv_m2l + (long)k * L.nsig, L.nsig, 2 * L.p, 0, ox * L.bs, oy * L.bs});
    }
    maxsig = std::max(maxsig, L.nsig);
    if (l < nl) {
      const double h = L.bs / 4;  // child centre - parent centre
      for (int q = 0; q < 4; q++) {
        const double cx = (q & 1) ? h : -h, cy = (q < 2) ? -h : h;
        const int nt = L.p + hl[l + 1].p;
        jobs.push_back(TvJob{L.tv_mm + (long)q * L.nsig_sh, L.nsig_sh, nt, 1, -cx, -cy});
        jobs.push_back(TvJob{L.tv_ll + (long)q * L.nsig_sh, L.nsig_sh, nt, 1, cx, cy});
      }
      maxsig = std::max(maxsig, L.nsig_sh);
    }
  }
  if (!jobs.empty()) {
    DBuf<TvJob> dj(st);
    dj.alloc(jobs.size(), st);
    B2_CHECK(cudaMemcpyAsync(dj.p, jobs.data(), sizeof(TvJob) * jobs.size(), cudaMemcpyHostToDevice,
                             st));
    const size_t sm = 2 * sizeof(double2) * (size_t)maxsig;
    set_smem(k_hf_transvec, sm);
    k_hf_transvec<<<(int)jobs.size(), 256, sm, st>>>(dj.p, zkr, zki, H.tabs.p);
    B2_LAUNCH_CHECK();
  }
  H.maxsig = maxsig;
  std::vector<double> bsx(T.boxsize);
  bsx.push_back(T.boxsize.back() / 2);
  H.dbs.alloc(bsx.size(), st);
  B2_CHECK(cudaMemcpyAsync(H.dbs.p, bsx.data(), sizeof(double) * bsx.size(), cudaMemcpyHostToDevice,
                           st));
  return IER_OK;
}

// Source batch of the expansion-forming kernels (2 warps per block) and
// their shared memory: 16 sources at a time, fewer for high orders.
int form_batch(int maxp, int ND, size_t* bytes) {
  int SB = 16;
  auto need = [&](int sb) { return sizeof(double2) * 2 * (size_t)sb * (2 * (maxp + 3) + 3 * ND); };
  while (SB > 1 && need(SB) > 200 * 1024) SB /= 2;
  *bytes = need(SB);
  return SB;
}

// M2M into levels nl-1 .. 2; signature form at the wideband levels.
template <int ND>
void upward_pass(const TV& tv, const DeviceTree& T, const HelmLevels& H, double2* mp,
                 cudaStream_t st) {
  const std::vector<HLev>& hl = H.hl;
  for (int l = T.nlevels - 1; l >= 2; l--) {
    if (!hl[l].ok) continue;
    int f = T.lfirst[l], n = T.llast[l] - f + 1;
    if (hl[l].wide) {
      const size_t sm = 2 * sizeof(double2) * (size_t)hl[l].nsig_sh;
      set_smem(k_hf_m2m<ND>, sm);
      k_hf_m2m<ND><<<(int)std::min<long>(n, 148L * 4), 256, sm, st>>>(tv, H.dlv.p, l, f, n,
                                                                      H.tabs.p, mp);
    } else {
      if (ND <= 2) {
        size_t sm = sizeof(double2) * (8 * (2 * hl[l + 1].p + 1) * ND + 2 * hl[l].nsh + 1) +
                    sizeof(double) * (HMAXP + 1);
        set_smem(k_h_m2m_sym<ND>, sm);
        k_h_m2m_sym<ND><<<(int)std::min<long>(n, 148L * 16), 128, sm, st>>>(tv, H.dlv.p, l, f, n,
                                                                           H.tabs.p, mp);
      } else {
        size_t sm = sizeof(double2) * (2 * (2 * hl[l + 1].p + 1) * ND + 2 * hl[l].nsh + 1) +
                    sizeof(double) * (HMAXP + 1);
        set_smem(k_h_m2m<ND>, sm);
        k_h_m2m<ND><<<(int)std::min<long>(n, 148L * 16), 128, sm, st>>>(tv, H.dlv.p, l, f, n,
                                                                       H.tabs.p, mp);
      }
    }
    B2_LAUNCH_CHECK();
  }
}

// M2L at levels >= 2: tabulated kernels, and signatures at the wideband levels.
template <int ND>
void m2l_pass(const TV& tv, const DeviceTree& T, const HelmLevels& H, const double2* mp,
              double2* lo, double2* sig, cudaStream_t st) {
  const int nb = T.nboxes, nl = T.nlevels;
  if (nl < 2) return;
  const int maxp = H.maxp;
  {
    int f = T.lfirst[2], n = nb - f;
    size_t sm = sizeof(double2) * (2 * (2 * maxp + 1) * ND + 4 * maxp + 1) +
                sizeof(double) * (maxp + 1);
    set_smem(k_h_m2l<ND>, sm);
    k_h_m2l<ND><<<(int)std::min<long>(n, 148L * 16), 128, sm, st>>>(tv, H.dlv.p, f, n, H.tabs.p,
                                                                   mp, lo, maxp);
    B2_LAUNCH_CHECK();
  }
  for (int l = 2; l <= nl; l++) {
    const HLev& L = H.hl[l];
    if (!L.wide) continue;
    int f = T.lfirst[l], n = T.llast[l] - f + 1;
    const size_t sm = 2 * sizeof(double2) * (size_t)L.nsig;
    set_smem(k_hf_tosig<ND>, sm);
    k_hf_tosig<ND><<<(int)std::min<long>(n, 148L * 4), 256, sm, st>>>(H.dlv.p, l, f, n, mp, sig);
    B2_LAUNCH_CHECK();
    set_smem(k_hf_m2l<ND>, sm);
    k_hf_m2l<ND><<<(int)std::min<long>(n, 148L * 4), 256, sm, st>>>(tv, H.dlv.p, l, f, n, sig,
                                                                    H.tabs.p, lo);
    B2_LAUNCH_CHECK();
  }
}

// L2L from levels 2 .. nl-1; signature form at the wideband levels.
template <int ND>
void downward_pass(const TV& tv, const DeviceTree& T, const HelmLevels& H, double2* lo,
                   cudaStream_t st) {
  const std::vector<HLev>& hl = H.hl;
  for (int l = 2; l <= T.nlevels - 1; l++) {
    if (!hl[l].ok) continue;
    int f = T.lfirst[l], n = T.llast[l] - f + 1;
    if (hl[l].wide) {
      const size_t sm = 2 * sizeof(double2) * (size_t)hl[l].nsig_sh;
      set_smem(k_hf_l2l<ND>, sm);
      k_hf_l2l<ND><<<(int)std::min<long>(n, 148L * 4), 256, sm, st>>>(tv, H.dlv.p, l, f, n,
                                                                      H.tabs.p, lo);
    } else {
      size_t sm = sizeof(double2) * ((2 * hl[l].p + 1) * ND + 4 * (2 * hl[l].nsh + 1)) +
                  sizeof(double) * (HMAXP + 1);
      set_smem(k_h_l2l<ND>, sm);
      k_h_l2l<ND><<<(int)std::min<long>(n, 148L * 16), 128, sm, st>>>(tv, H.dlv.p, l, f, n,
                                                                     H.tabs.p, lo);
    }
    B2_LAUNCH_CHECK();
  }
}

template <int ND>
void helm_chunk(const TV& tv, DeviceTree& T, const HelmArgs& a, const HDens& D,
                const HelmLevels& H, const double2* xs, const double2* xt, double2* mp,
                double2* lo, double2* sig, double2* ps, double2* gs, double2* hs, double2* pt,
                double2* gt, double2* ht, double thresh, const int* leaf_s, const int* leaf_t,
                long ns_pts, long nt_pts, cudaStream_t st, cudaEvent_t* ev) {
  const int nb = T.nboxes, nl = T.nlevels;
  const HLev* dlv = H.dlv.p;
  B2_CHECK(cudaEventRecord(ev[0], st));
  size_t sm_form = 0;
  const int SB = form_batch(H.maxp_all, ND, &sm_form);
  set_smem(k_h_p2m<ND>, sm_form);
  set_smem(k_h_p2l<ND>, sm_form);
  k_h_p2m<ND><<<grid_w(nb, 2), 64, sm_form, st>>>(tv, dlv, nb, xs, D, a.zkr, a.zki, mp,
                                                  H.maxp_all, SB);
  B2_LAUNCH_CHECK();
  B2_CHECK(cudaEventRecord(ev[1], st));
  upward_pass<ND>(tv, T, H, mp, st);
  B2_CHECK(cudaEventRecord(ev[2], st));
  if (nl >= 2) {
    int f = T.lfirst[2], n = nb - f;
    k_h_p2l<ND><<<grid_w(n, 2), 64, sm_form, st>>>(tv, dlv, f, n, xs, D, a.zkr, a.zki, lo,
                                                   H.maxp_all, SB);
    B2_LAUNCH_CHECK();
  }
  B2_CHECK(cudaEventRecord(ev[3], st));
  m2l_pass<ND>(tv, T, H, mp, lo, sig, st);
  B2_CHECK(cudaEventRecord(ev[4], st));
  downward_pass<ND>(tv, T, H, lo, st);
  B2_CHECK(cudaEventRecord(ev[5], st));
  auto leaf = [&](int use_t, int ifl, const double2* xe, double2* po, double2* gr, double2* he) {
    const long n = use_t ? nt_pts : ns_pts;
    if (ifl <= 0 || n <= 0) return;
    const int* lf = use_t ? leaf_t : leaf_s;
    const int g = ceil_div(n, 128);
#define B2_H_LEAF(IFL)                                                                        \
  k_h_far<ND, IFL><<<g, 128, 0, st>>>(tv, dlv, n, lf, xe, D, a.zkr, a.zki, mp, lo, po, gr, he); \
  B2_LAUNCH_CHECK();                                                                          \
  if (a.ifnear) {                                                                             \
    k_h_p2p<ND, IFL><<<g, 128, 0, st>>>(tv, n, lf, xs, xe, D, a.zkr, a.zki, thresh, po, gr,   \
                                        he);                                                  \
    B2_LAUNCH_CHECK();                                                                        \
  }
    if (ifl == 1) {
      B2_H_LEAF(1)
    } else if (ifl == 2) {
      B2_H_LEAF(2)
    } else {
      B2_H_LEAF(3)
    }
#undef B2_H_LEAF
  };
  leaf(0, a.ifpgh, xs, ps, gs, hs);
  leaf(1, a.ifpghtarg, xt, pt, gt, ht);
  B2_CHECK(cudaEventRecord(ev[6], st));
}


// ---------------------------------------------------------------------------
// FMM over multipole sources (hfmm2d_mps, src/helmholtz/hfmm2d_mps.f:19-1025).
// The tree is built on the expansion centres (ndiv 1).  Box-to-box steps are
// the kernels above; the steps that start or end at an expansion of its own
// centre, scale and order translate one expansion at a time:
//   step 1  expansion -> leaf multipole (h2dmpmp)       k_mps_boxes
//   step 2  list-4 expansions -> box local (h2dmploc)   k_mps_boxes
//   step 6  list-3 multipoles -> expansion (h2dmploc)   k_mps_locals
//   step 7  leaf local -> expansion (h2dlocloc)         k_mps_locals
//   step 8  list-1 expansions -> expansion (h2dmploc)   k_mps_locals
// ---------------------------------------------------------------------------
enum { X_MPMP = 0, X_MPLOC = 1, X_LOCLOC = 2 };

// Expansions in tree order: centre, scale, order, offset of (nd, -m..m) in
// the caller's coefficient arrays.
struct MpsExp {
  const double2* c;
  const double* rs;
  const int* m;
  const long* off;
};

// Warp-private shared scratch of the translations: Z[nt + 4], T[2 nt + 1],
// R[max order + 1].
struct XScr {
  double2* Z;
  double2* T;
  double* R;
};

// dst(i) += sum_j src(j) T(i-j) f(i,j), i = -n2..n2, j = -n1..n1, with the
// (value, phase) table T of the centre shift c2 - c1 (J_n(zk r)/rs1^n for the
// shifts, H_n(zk r) rs1^n for multipole to local; theta - pi as in
// h2dmpmp / h2dmploc / h2dlocloc, helmrouts2d.f:967-1378) and the rscale
// factors of each operator:
//   mpmp:   (rs1/rs2)^|i| rs1^(2e), e = max(0,|j|-|i|) for j of the sign of i, else |j|
//   mploc:  (rs2/rs1)^|i| rs1^(2 min(|i|,|j|)) for j of the sign of i, else (rs2/rs1)^|i|
//   locloc: 1 for i = 0; (rs1 rs2)^|i| for j = 0 or of the other sign;
//           (rs2/rs1)^|i| rs1^(2 max(0,|i|-|j|)) for j of the sign of i.
// src and dst hold ND densities per coefficient at strides ss and ds.
template <int ND>
__device__ void warp_xlate(int kind, double2 zk, double rs1, double2 c1, const double2* src, int ss,
                           int n1, double rs2, double2 c2, double2* dst, int ds, int n2,
                           const XScr& S, int lane) {
  const int nt = n1 + n2;
  const double pi = 3.14159265358979323846;
  const double x = c2.x - c1.x, y = c2.y - c1.y;
  const double th = atan2(y, x) - pi;
  if (lane == 0) {
    const double r = sqrt(x * x + y * y);
    const double2 z = make_double2(zk.x * r, zk.y * r);
    if (kind == X_MPLOC)
      hscaled(nt + 1, z, rs1, S.Z);
    else
      jscaled(nt + 3, z, rs1, S.Z);
  }
  const int mx = n1 > n2 ? n1 : n2;
  for (int k = lane; k <= mx; k += 32) S.R[k] = pow(rs1, 2.0 * k);
  __syncwarp();
  for (int j = lane; j <= nt; j += 32) {
    double sn, cs;
    sincos(j * th, &sn, &cs);
    const double2 e = make_double2(cs, -sn);  // exp(-i theta)^j
    const double2 zj = S.Z[j];
    S.T[nt + j] = cmul(e, zj);
    if (j > 0) {
      double2 t = cmul(make_double2(cs, sn), zj);  // conj(e)^j Z_j
      if (j & 1) t = make_double2(-t.x, -t.y);
      S.T[nt - j] = t;
    }
  }
  __syncwarp();
  const double2* T = S.T + nt;
  for (int i = lane - n2; i <= n2; i += 32) {
    const int ai = i < 0 ? -i : i;
    double2 a0[ND], a1[ND];  // a0: unit factor, a1: the second factor class
#pragma unroll
    for (int d = 0; d < ND; d++) a0[d] = a1[d] = make_double2(0, 0);
    for (int j = -n1; j <= n1; j++) {
      const int aj = j < 0 ? -j : j;
      const bool same = i != 0 && j != 0 && ((i > 0) == (j > 0));
      double f = 1.0;
      bool second = false;
      if (kind == X_MPMP) {
        f = S.R[same ? (aj > ai ? aj - ai : 0) : aj];
      } else if (kind == X_MPLOC) {
        if (same) f = S.R[ai < aj ? ai : aj];
      } else if (i != 0) {
        if (same)
          f = S.R[ai > aj ? ai - aj : 0];
        else
          second = true;
      }
      const double2 t = cscale(T[i - j], f);
      const double2* sj = src + (size_t)(j + n1) * ss;
#pragma unroll
      for (int d = 0; d < ND; d++) {
        if (second)
          cfma(a1[d], sj[d], t);
        else
          cfma(a0[d], sj[d], t);
      }
    }
    double g0 = 1.0, g1 = 0.0;
    if (kind == X_MPMP) {
      g0 = pow(rs1 / rs2, (double)ai);
    } else if (kind == X_MPLOC) {
      g0 = pow(rs2 / rs1, (double)ai);
    } else if (i != 0) {
      g0 = pow(rs2 / rs1, (double)ai);
      g1 = pow(rs1 * rs2, (double)ai);
    }
    double2* di = dst + (size_t)(i + n2) * ds;
#pragma unroll
    for (int d = 0; d < ND; d++)
      di[d] = cadd(di[d], cadd(cscale(a0[d], g0), cscale(a1[d], g1)));
  }
  __syncwarp();
}

__device__ __forceinline__ XScr warp_scratch(char* base, int maxnt, int wib) {
  const size_t zn = (size_t)maxnt + 4, tn = 2 * (size_t)maxnt + 1, rn = (size_t)maxnt + 2;
  const size_t per = (zn + tn) * sizeof(double2) + rn * sizeof(double);
  char* w = base + per * wib;
  XScr S;
  S.Z = reinterpret_cast<double2*>(w);
  S.T = S.Z + zn;
  S.R = reinterpret_cast<double*>(S.T + tn);
  return S;
}

// Steps 1 and 2, one warp per box of levels >= 2 (boxes first .. first+n-1).
template <int ND>
__global__ void __launch_bounds__(128) k_mps_boxes(TV t, const HLev* __restrict__ lv, int first,
                                                   int n, MpsExp E, const double2* __restrict__ mpole,
                                                   int nd, int d0, double2 zk, double2* mp,
                                                   double2* lo, int maxnt) {
  extern __shared__ __align__(16) char xsm[];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const XScr S = warp_scratch(xsm, maxnt, wib);
  const int nw = gridDim.x * (blockDim.x >> 5);
  for (int w = blockIdx.x * (blockDim.x >> 5) + wib; w < n; w += nw) {
    const int b = first + w;
    const HLev L = lv[t.level[b]];
    if (!L.ok) continue;
    const double2 cb = t.center[b];
    if (t.nchild[b] == 0) {
      const int2 r = t.srng[b];
      double2* M = hexp(mp, L, b, ND);
      for (int k = r.x; k < r.y; k++)
        warp_xlate<ND>(X_MPMP, zk, E.rs[k], E.c[k], mpole + E.off[k] + d0, nd, E.m[k], L.rs, cb,
                       M, ND, L.p, S, lane);
    }
    double2* Lo = hexp(lo, L, b, ND);
    const int n4 = t.nl4[b];
    for (int e = 0; e < n4; e++) {
      const int jb = t.l4[(size_t)MNLIST4 * b + e];
      const int2 r = t.srng[jb];
      for (int k = r.x; k < r.y; k++)
        warp_xlate<ND>(X_MPLOC, zk, E.rs[k], E.c[k], mpole + E.off[k] + d0, nd, E.m[k], L.rs, cb,
                       Lo, ND, L.p, S, lane);
    }
  }
}

// Steps 6-8, one warp per expansion (tree order), accumulating into the
// caller's local array (zeroed here first, as hfmm2dmain_mps zeroes it).
template <int ND>
__global__ void __launch_bounds__(128) k_mps_locals(TV t, const HLev* __restrict__ lv, int nlev,
                                                    const int* __restrict__ leaf, long nexp,
                                                    MpsExp E, const double2* __restrict__ mpole,
                                                    int nd, int d0, double2 zk,
                                                    const double2* __restrict__ mp,
                                                    const double2* __restrict__ lo,
                                                    double2* __restrict__ local, double thresh,
                                                    int maxnt) {
  extern __shared__ __align__(16) char xsm[];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const XScr S = warp_scratch(xsm, maxnt, wib);
  const long nw = (long)gridDim.x * (blockDim.x >> 5);
  for (long j = blockIdx.x * (long)(blockDim.x >> 5) + wib; j < nexp; j += nw) {
    const int m2 = E.m[j];
    const double rs2 = E.rs[j];
    const double2 c2 = E.c[j];
    double2* dst = local + E.off[j] + d0;
    for (int e = lane; e < 2 * m2 + 1; e += 32)
#pragma unroll
      for (int d = 0; d < ND; d++) dst[(size_t)e * nd + d] = make_double2(0, 0);
    __syncwarp();
    const int B = leaf[j];
    const int lb = t.level[B];
    // step 6: multipoles of list-3 boxes (one level down)
    const int n3 = t.nl3[B];
    for (int e = 0; e < n3; e++) {
      const int jb = t.l3[(size_t)MNLIST3 * B + e];
      const HLev LJ = lv[t.level[jb]];
      if (!LJ.ok) continue;
      warp_xlate<ND>(X_MPLOC, zk, LJ.rs, t.center[jb], hexp(const_cast<double2*>(mp), LJ, jb, ND),
                     ND, LJ.p, rs2, c2, dst, nd, m2, S, lane);
    }
    // step 7: the leaf's local expansion (zero above level 2, where no
    // translation reaches)
    const HLev L = lv[lb];
    if (L.ok && lb >= 2)
      warp_xlate<ND>(X_LOCLOC, zk, L.rs, t.center[B], hexp(const_cast<double2*>(lo), L, B, ND), ND,
                     L.p, rs2, c2, dst, nd, m2, S, lane);
    // step 8: expansions of list-1 boxes, except coincident centres
    const int n1 = t.nl1[B];
    for (int e = 0; e < n1; e++) {
      const int jb = t.l1[(size_t)MNLIST1 * B + e];
      const int2 r = t.srng[jb];
      for (int k = r.x; k < r.y; k++) {
        const double2 ck = E.c[k];
        const double dx = ck.x - c2.x, dy = ck.y - c2.y;
        if (!(sqrt(dx * dx + dy * dy) > thresh)) continue;
        warp_xlate<ND>(X_MPLOC, zk, E.rs[k], ck, mpole + E.off[k] + d0, nd, E.m[k], rs2, c2, dst,
                       nd, m2, S, lane);
      }
    }
  }
  (void)nlev;
}

// Expansion data in tree order; off = (impole - 1) / 1 in double2 units.
__global__ void k_mps_gather(const double* __restrict__ cen, const double* __restrict__ rsc,
                             const int* __restrict__ mt, const int* __restrict__ impole,
                             const int* __restrict__ perm, long n, double2* c, double* rs, int* m,
                             long* off) {
  const long k = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (k >= n) return;
  const long i = perm[k];
  c[k] = make_double2(cen[2 * i], cen[2 * i + 1]);
  rs[k] = rsc[i];
  m[k] = mt[i];
  off[k] = (long)impole[i] - 1;
}

size_t mps_smem(int maxnt, int warps) {
  const size_t zn = (size_t)maxnt + 4, tn = 2 * (size_t)maxnt + 1, rn = (size_t)maxnt + 2;
  return ((zn + tn) * sizeof(double2) + rn * sizeof(double)) * warps;
}

template <int ND>
void mps_chunk(const TV& tv, const DeviceTree& T, const HelmLevels& H, const MpsExp& E,
               const double2* mpole, int nd, int d0, double2 zk, double2* mp, double2* lo,
               double2* sig, const int* leaf, long nc, double2* local, double thresh, int maxnt,
               int warps, cudaStream_t st) {
  const int nb = T.nboxes, nl = T.nlevels;
  const size_t xs = mps_smem(maxnt, warps);
  const int thr = 32 * warps;
  B2_CHECK(cudaMemsetAsync(mp, 0, sizeof(double2) * (size_t)H.off * ND, st));
  B2_CHECK(cudaMemsetAsync(lo, 0, sizeof(double2) * (size_t)H.off * ND, st));
  if (nl >= 2) {
    const int f = T.lfirst[2], n = nb - f;
    set_smem(k_mps_boxes<ND>, xs);
    k_mps_boxes<ND><<<(int)std::min<long>(ceil_div(n, warps), 148L * 8), thr, xs, st>>>(
        tv, H.dlv.p, f, n, E, mpole, nd, d0, zk, mp, lo, maxnt);
    B2_LAUNCH_CHECK();
  }
  upward_pass<ND>(tv, T, H, mp, st);
  m2l_pass<ND>(tv, T, H, mp, lo, sig, st);
  downward_pass<ND>(tv, T, H, lo, st);
  set_smem(k_mps_locals<ND>, xs);
  k_mps_locals<ND><<<(int)std::min<long>(ceil_div(nc, warps), 148L * 8), thr, xs, st>>>(
      tv, H.dlv.p, nl, leaf, nc, E, mpole, nd, d0, zk, mp, lo, local, thresh, maxnt);
  B2_LAUNCH_CHECK();
}
}  // namespace

int helm_nterms(double bsize, double zkr, double zki, double eps, int* ier) {
  // h2dterms: first j with (|J_j H_j| + |J_(j-1) H_(j-1)|) |H_0| < eps (|J_0 H_0| + |J_1 H_1|)
  const double pi2 = 8 * std::atan(1.0);
  double2 zb = make_double2(zkr * bsize, zki * bsize);
  double rscale = 1.0;
  if (std::hypot(zb.x, zb.y) < pi2) rscale = std::hypot(zb.x, zb.y);
  // the criterion is met near order 1.5 |zk bsize| + (digits); the
  // reference scans up to 50000 orders
  const int NT = (int)std::min(50000.0, std::max(400.0, 2.0 * std::hypot(zb.x, zb.y) + 200.0));
  std::vector<double2> hf(NT + 1), jf(NT + 1);
  helm::hscaled(NT, make_double2(1.5 * zb.x, 1.5 * zb.y), rscale, hf.data());
  double c = std::sqrt(2.0) / 2.0;
  helm::jscaled(NT, make_double2(c * zb.x, c * zb.y), rscale, jf.data());
  auto ab = [](double2 a, double2 b) { double2 m = cmul(a, b); return std::hypot(m.x, m.y); };
  double x0 = ab(jf[0], hf[0]) + ab(jf[1], hf[1]);
  double h0 = std::hypot(hf[0].x, hf[0].y);
  for (int j = 2; j <= NT; j++) {
    double v = (ab(jf[j], hf[j]) + ab(jf[j - 1], hf[j - 1])) * h0;
    if (v < eps * x0) return j + 1;
  }
  *ier = IER_NTERMS;
  return 10001;
}

int helm_fmm_device(const HelmArgs& a, cudaStream_t st) {
  if (a.nd < 1 || a.ns < 0 || a.nt < 0 || a.ifpgh < 0 || a.ifpgh > 3 || a.ifpghtarg < 0 ||
      a.ifpghtarg > 3 || a.ns > (1L << 30) || a.nt > (1L << 30))
    return IER_BADARG;
  if (a.ns > 0 && !a.src) return IER_BADARG;
  if (a.nt > 0 && a.ifpghtarg > 0 && !a.trg) return IER_BADARG;
  if (a.dipstr && !a.dipvec) return IER_BADARG;
  int dev = 0;
  B2_CHECK(cudaGetDevice(&dev));
  configure_mempool(dev);
  ensure_device_tables();
  const int nd = a.nd;
  const long ns = a.ns, nt = a.ifpghtarg > 0 ? a.nt : 0;
  const bool fc = a.charge != nullptr, fd = a.dipstr != nullptr;
  if (a.timeinfo)
    for (int i = 0; i < 8; i++) a.timeinfo[i] = 0;
  auto zero_outputs = [&]() {
    if (a.ifpgh >= 1 && ns) B2_CHECK(cudaMemsetAsync(a.pot, 0, sizeof(double2) * nd * ns, st));
    if (a.ifpgh >= 2 && ns) B2_CHECK(cudaMemsetAsync(a.grad, 0, sizeof(double2) * 2 * nd * ns, st));
    if (a.ifpgh >= 3 && ns) B2_CHECK(cudaMemsetAsync(a.hess, 0, sizeof(double2) * 3 * nd * ns, st));
    if (a.ifpghtarg >= 1 && nt) B2_CHECK(cudaMemsetAsync(a.pottarg, 0, sizeof(double2) * nd * nt, st));
    if (a.ifpghtarg >= 2 && nt) B2_CHECK(cudaMemsetAsync(a.gradtarg, 0, sizeof(double2) * 2 * nd * nt, st));
    if (a.ifpghtarg >= 3 && nt) B2_CHECK(cudaMemsetAsync(a.hesstarg, 0, sizeof(double2) * 3 * nd * nt, st));
    B2_CHECK(cudaStreamSynchronize(st));
  };
  if (ns == 0 || (!fc && !fd)) {
    zero_outputs();
    return IER_OK;
  }
  int ndiv = a.ndiv > 0 ? a.ndiv : lap_ndiv(a.eps);  // hndiv2d.f: same table as lndiv2d
  if (ndiv <= 0) ndiv = (int)std::min<long>(ns + nt, 1L << 30);
  DeviceTree T;
  build_device_tree(T, a.src, ns, a.trg, nt, 0, ndiv, NLMAX, st);
  if (T.bs0 == 0.0) {
    zero_outputs();
    return IER_OK;
  }
  const double zkabs = std::hypot(a.zkr, a.zki);
  HelmLevels H(st);
  if (int r = helm_levels(T, a.zkr, a.zki, a.eps, H, st)) return r;
  const long off = H.off;
  DBuf<double>& dbs = H.dbs;
  // sorted inputs
  DBuf<double2> xs(st), xt(st), qs(st), ds(st);
  DBuf<double> vs(st);
  xs.alloc(ns, st);
  if (fc) qs.alloc((size_t)ns * nd, st);
  if (fd) {
    ds.alloc((size_t)ns * nd, st);
    vs.alloc((size_t)ns * 2 * nd, st);
  }
  k_h_gather<<<ceil_div(ns, 256), 256, 0, st>>>(a.src, T.isrc.p, ns, nd, a.charge, a.dipstr,
                                               a.dipvec, xs.p, qs.p, ds.p, vs.p);
  B2_LAUNCH_CHECK();
  if (nt > 0) {
    xt.alloc(nt, st);
    k_h_gather<<<ceil_div(nt, 256), 256, 0, st>>>(a.trg, T.itarg.p, nt, 0, nullptr, nullptr,
                                                 nullptr, xt.p, nullptr, nullptr, nullptr);
    B2_LAUNCH_CHECK();
  }
  DBuf<double2> ps(st), gs(st), hs(st), pt(st), gt(st), ht(st);
  if (a.ifpgh >= 1) ps.alloc((size_t)ns * nd, st);
  if (a.ifpgh >= 2) gs.alloc((size_t)ns * 2 * nd, st);
  if (a.ifpgh >= 3) hs.alloc((size_t)ns * 3 * nd, st);
  if (a.ifpghtarg >= 1 && nt) pt.alloc((size_t)nt * nd, st);
  if (a.ifpghtarg >= 2 && nt) gt.alloc((size_t)nt * 2 * nd, st);
  if (a.ifpghtarg >= 3 && nt) ht.alloc((size_t)nt * 3 * nd, st);
  TV tv{T.center.p, T.level.p, T.nchild.p, T.child.p, T.srng.p, T.trng.p, T.nlist1.p, T.list1.p,
        T.nlist2.p, T.list2.p, T.nlist3.p, T.list3.p, T.nlist4.p, T.list4.p, dbs.p, a.ifpgh,
        nt > 0 ? a.ifpghtarg : 0, T.ctl.p};
  const double thresh = zkabs * T.bs0 * std::ldexp(1.0, -51);
  // leaf box of every sorted point, for the one-point-per-thread leaf kernels
  DBuf<int> leafs(st), leaft(st);
  leafs.alloc(ns, st);
  k_h_point_leaf<<<ceil_div(T.nboxes, 128), 128, 0, st>>>(tv, T.nboxes, 0, leafs.p);
  B2_LAUNCH_CHECK();
  if (nt > 0) {
    leaft.alloc(nt, st);
    k_h_point_leaf<<<ceil_div(T.nboxes, 128), 128, 0, st>>>(tv, T.nboxes, 1, leaft.p);
    B2_LAUNCH_CHECK();
  }
  int chunk = nd >= 4 ? 4 : (nd >= 2 ? 2 : 1);
  DBuf<double2> mp(st), lo(st), sig(st);
  mp.alloc((size_t)off * chunk, st);
  lo.alloc((size_t)off * chunk, st);
  if (H.sig_total > 0) sig.alloc((size_t)H.sig_total * chunk, st);
  cudaEvent_t ev[8];
  for (int i = 0; i < 8; i++) B2_CHECK(cudaEventCreate(&ev[i]));
  double tsum[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int d0 = 0; d0 < nd;) {
    int left = nd - d0;
    int ND = left >= 4 ? 4 : (left >= 2 ? 2 : 1);
    HDens D{fc ? qs.p : nullptr, fd ? ds.p : nullptr, fd ? vs.p : nullptr, nd, d0};
    B2_CHECK(cudaMemsetAsync(lo.p, 0, sizeof(double2) * (size_t)off * ND, st));
    switch (ND) {
      case 4: helm_chunk<4>(tv, T, a, D, H, xs.p, xt.p, mp.p, lo.p, sig.p, ps.p, gs.p, hs.p, pt.p, gt.p, ht.p, thresh, leafs.p, leaft.p, ns, nt, st, ev); break;
      case 2: helm_chunk<2>(tv, T, a, D, H, xs.p, xt.p, mp.p, lo.p, sig.p, ps.p, gs.p, hs.p, pt.p, gt.p, ht.p, thresh, leafs.p, leaft.p, ns, nt, st, ev); break;
      default: helm_chunk<1>(tv, T, a, D, H, xs.p, xt.p, mp.p, lo.p, sig.p, ps.p, gs.p, hs.p, pt.p, gt.p, ht.p, thresh, leafs.p, leaft.p, ns, nt, st, ev); break;
    }
    if (a.timeinfo) {
      B2_CHECK(cudaEventSynchronize(ev[6]));
      float ms[6];
      for (int i = 0; i < 6; i++) B2_CHECK(cudaEventElapsedTime(&ms[i], ev[i], ev[i + 1]));
      tsum[0] += ms[0] * 1e-3;
      tsum[2] += ms[1] * 1e-3;
      tsum[1] += ms[2] * 1e-3;
      tsum[3] += ms[3] * 1e-3;
      tsum[4] += ms[4] * 1e-3;
      tsum[7] += ms[5] * 1e-3;
    }
    d0 += ND;
  }
  auto unpack = [&](const int* perm, long n, int w, const double2* in, double* out) {
    if (!out || !n) return;
    k_h_unpack<<<ceil_div(n, 256), 256, 0, st>>>(perm, n, w, in, (double2*)out);
    B2_LAUNCH_CHECK();
  };
  if (a.ifpgh >= 1) unpack(T.isrc.p, ns, nd, ps.p, a.pot);
  if (a.ifpgh >= 2) unpack(T.isrc.p, ns, 2 * nd, gs.p, a.grad);
  if (a.ifpgh >= 3) unpack(T.isrc.p, ns, 3 * nd, hs.p, a.hess);
  if (a.ifpghtarg >= 1) unpack(T.itarg.p, nt, nd, pt.p, a.pottarg);
  if (a.ifpghtarg >= 2) unpack(T.itarg.p, nt, 2 * nd, gt.p, a.gradtarg);
  if (a.ifpghtarg >= 3) unpack(T.itarg.p, nt, 3 * nd, ht.p, a.hesstarg);
  B2_CHECK(cudaStreamSynchronize(st));
  if (a.timeinfo)
    for (int i = 0; i < 8; i++) a.timeinfo[i] = tsum[i];
  for (int i = 0; i < 8; i++) cudaEventDestroy(ev[i]);
  return IER_OK;
}

int helm_mps_device(int nd, double eps, double zkr, double zki, long nc, const double* centers,
                    const double* rscales, const int* mterms, const int* impole, long ntot,
                    const double* mpole, double* local, int max_mterms, cudaStream_t st) {
  if (nd < 1 || nc < 0 || ntot < 0 || nc > (1L << 30) || max_mterms < 0) return IER_BADARG;
  if (max_mterms > HMAXP) return IER_NTERMS;
  if (nc == 0) return IER_OK;
  if (!centers || !rscales || !mterms || !impole || !mpole || !local) return IER_BADARG;
  int dev = 0;
  B2_CHECK(cudaGetDevice(&dev));
  configure_mempool(dev);
  ensure_device_tables();
  // tree on the centres, one per leaf (hfmm2d_mps.f:106-143: idivflag 0, ndiv 1)
  DeviceTree T;
  build_device_tree(T, centers, nc, nullptr, 0, 0, 1, NLMAX, st);
  HelmLevels H(st);
  if (int r = helm_levels(T, zkr, zki, eps, H, st)) return r;
  const int maxnt = 2 * std::max(H.maxp_all, max_mterms);
  // warps per block of the per-expansion kernels (their translation scratch)
  int warps = 4;
  while (warps > 1 && mps_smem(maxnt, warps) > 200 * 1024) warps /= 2;
  if (mps_smem(maxnt, warps) > 200 * 1024) return IER_NTERMS;
  DBuf<double2> ec(st);
  DBuf<double> ers(st);
  DBuf<int> em(st), leaf(st);
  DBuf<long> eoff(st);
  ec.alloc(nc, st);
  ers.alloc(nc, st);
  em.alloc(nc, st);
  eoff.alloc(nc, st);
  k_mps_gather<<<ceil_div(nc, 256), 256, 0, st>>>(centers, rscales, mterms, impole, T.isrc.p, nc,
                                                  ec.p, ers.p, em.p, eoff.p);
  B2_LAUNCH_CHECK();
  TV tv{T.center.p, T.level.p, T.nchild.p, T.child.p, T.srng.p, T.trng.p, T.nlist1.p, T.list1.p,
        T.nlist2.p, T.list2.p, T.nlist3.p, T.list3.p, T.nlist4.p, T.list4.p, H.dbs.p, 1, 0,
        T.ctl.p};
  leaf.alloc(nc, st);
  k_h_point_leaf<<<ceil_div(T.nboxes, 128), 128, 0, st>>>(tv, T.nboxes, 0, leaf.p);
  B2_LAUNCH_CHECK();
  // interactions closer than this are skipped (hfmm2d_mps.f:960)
  const double thresh = std::hypot(zkr, zki) * T.bs0 * std::ldexp(1.0, -51);
  // the offsets count complex entries of (nd, -m..m) blocks
  MpsExp E{ec.p, ers.p, em.p, eoff.p};
  const double2 zk = make_double2(zkr, zki);
  const int chunk = nd >= 4 ? 4 : (nd >= 2 ? 2 : 1);
  DBuf<double2> mp(st), lo(st), sig(st);
  mp.alloc((size_t)H.off * chunk, st);
  lo.alloc((size_t)H.off * chunk, st);
  if (H.sig_total > 0) sig.alloc((size_t)H.sig_total * chunk, st);
  auto* mpc = reinterpret_cast<const double2*>(mpole);
  auto* loc = reinterpret_cast<double2*>(local);
  for (int d0 = 0; d0 < nd;) {
    const int left = nd - d0;
    const int ND = left >= 4 ? 4 : (left >= 2 ? 2 : 1);
    switch (ND) {
      case 4: mps_chunk<4>(tv, T, H, E, mpc, nd, d0, zk, mp.p, lo.p, sig.p, leaf.p, nc, loc, thresh, maxnt, warps, st); break;
      case 2: mps_chunk<2>(tv, T, H, E, mpc, nd, d0, zk, mp.p, lo.p, sig.p, leaf.p, nc, loc, thresh, maxnt, warps, st); break;
      default: mps_chunk<1>(tv, T, H, E, mpc, nd, d0, zk, mp.p, lo.p, sig.p, leaf.p, nc, loc, thresh, maxnt, warps, st); break;
    }
    d0 += ND;
  }
  B2_CHECK(cudaStreamSynchronize(st));
  return IER_OK;
}

int helm_direct_device(int nd, double zkr, double zki, long ns, const double* src,
                       const double* charge, const double* dipstr, const double* dipvec, long nt,
                       const double* trg, int ifpgh, double* pot, double* grad, double* hess,
                       double thresh, cudaStream_t st) {
  if (nd < 1 || ns < 0 || nt < 0 || ifpgh < 1 || ifpgh > 3) return IER_BADARG;
  if (nt == 0) return IER_OK;
  if (dipstr && !dipvec) return IER_BADARG;
  int dev = 0;
  B2_CHECK(cudaGetDevice(&dev));
  configure_mempool(dev);
  ensure_device_tables();
  if (ns == 0 || (!charge && !dipstr)) {
    B2_CHECK(cudaMemsetAsync(pot, 0, sizeof(double2) * nd * nt, st));
    if (ifpgh >= 2) B2_CHECK(cudaMemsetAsync(grad, 0, sizeof(double2) * 2 * nd * nt, st));
    if (ifpgh >= 3) B2_CHECK(cudaMemsetAsync(hess, 0, sizeof(double2) * 3 * nd * nt, st));
    B2_CHECK(cudaStreamSynchronize(st));
    return IER_OK;
  }
  int tb = ceil_div(nt, 128);
  int nslice = std::max(1, std::min(1024, (148 * 16) / std::max(tb, 1)));
  long chunk = (ns + nslice - 1) / nslice;
  chunk = ((chunk + 127) / 128) * 128;
  nslice = (int)std::max(1L, (ns + chunk - 1) / chunk);
  DBuf<double2> part(st);
  part.alloc((size_t)nslice * nt * 6, st);
  for (int d = 0; d < nd; d++) {
    dim3 grid(tb, nslice);
    if (ifpgh == 1)
      k_h_direct<1><<<grid, 128, 0, st>>>(nd, d, ns, src, charge, dipstr, dipvec, nt, trg, zkr, zki, thresh, chunk, part.p);
    else if (ifpgh == 2)
      k_h_direct<2><<<grid, 128, 0, st>>>(nd, d, ns, src, charge, dipstr, dipvec, nt, trg, zkr, zki, thresh, chunk, part.p);
    else
      k_h_direct<3><<<grid, 128, 0, st>>>(nd, d, ns, src, charge, dipstr, dipvec, nt, trg, zkr, zki, thresh, chunk, part.p);
    B2_LAUNCH_CHECK();
    k_h_direct_reduce<<<ceil_div(nt, 256), 256, 0, st>>>(nd, d, nt, nslice, ifpgh, part.p,
                                                         (double2*)pot, (double2*)grad,
                                                         (double2*)hess);
    B2_LAUNCH_CHECK();
  }
  B2_CHECK(cudaStreamSynchronize(st));
  return IER_OK;
}

}  // namespace b2
