// Biharmonic and Stokes sums on the Cauchy FMM.
//
// The biharmonic velocity of src/biharmonic/bhkernels2d.f (bh2d_directcdg),
// with w = z - z_j,
//   vel   = sum 2 c1 log|w| + c2 w/conj(w) + d1/w + d3/conj(w) + d2 w/conj(w)^2
//   grad1 = sum c1/w - d1/w^2
//   grad2 = sum c2/conj(w) + d2/conj(w)^2
//   grad3 = sum c1/conj(w) - c2 w/conj(w)^2 - d3/conj(w)^2 - 2 d2 w/conj(w)^3
// is a combination of four Cauchy sums (cauchykernels2d.f c2d_directcdh:
// P = sum q log|w| + dl/w, G = sum q/w - dl/w^2, H = sum -q/w^2 + 2 dl/w^3).
// With r_j = z_j - z0 and r = z - z0 for a fixed origin z0 (the first source):
//   problem 1: q = c1,        dl = d1
//   problem 2: q = conj(c1),  dl = conj(d3) - conj(c2) conj(r_j)
//   problem 3: q = conj(c2),  dl = -conj(d2)
//   problem 4: q = 0,         dl = conj(d2) conj(r_j)
//   vel   = P1 + conj(P2) + r conj(G3) + conj(G4)
//   grad1 = G1,  grad2 = conj(G3),  grad3 = conj(G2) + r conj(H3) + conj(H4)
// The terms in 1/conj(w) are conjugates of Cauchy sums; a factor w = r - r_j
// in front of them splits into r, applied after the sum, and -r_j, folded
// into the densities (e.g. c2 w/conj(w) = r conj(conj(c2)/w) -
// conj(conj(c2) conj(r_j)/w)).
// The four problems run as one Cauchy FMM with 4 nd densities, in FP64.
//
// Stokes (src/stokes/stfmm2d.f:100-330): stokeslets and stresslets become
// biharmonic charges and dipoles, and velocity, pressure and velocity
// gradient are read off the biharmonic velocity and its derivatives.
#include "biharmonic.cuh"

#include <algorithm>

#include "direct.cuh"
#include "laplace.cuh"

namespace b2 {
namespace {

__device__ __forceinline__ double2 cj(double2 a) { return make_double2(a.x, -a.y); }

// Densities of the four Cauchy problems; problem k of density d of source i
// at (i, k nd + d).
__global__ void k_bh_dens(const double* __restrict__ src, long ns, int nd,
                          const double2* __restrict__ charge, const double2* __restrict__ dip,
                          double2* __restrict__ q, double2* __restrict__ dl) {
  const long e = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (e >= ns * nd) return;
  const long i = e / nd;
  const int d = (int)(e % nd);
  const double2 z0 = make_double2(src[0], src[1]);
  const double2 crj = make_double2(src[2 * i] - z0.x, -(src[2 * i + 1] - z0.y));  // conj(r_j)
  const double2 zero = make_double2(0, 0);
  const double2 c1 = charge ? charge[(i * 2 + 0) * nd + d] : zero;
  const double2 c2 = charge ? charge[(i * 2 + 1) * nd + d] : zero;
  const double2 d1 = dip ? dip[(i * 3 + 0) * nd + d] : zero;
  const double2 d2 = dip ? dip[(i * 3 + 1) * nd + d] : zero;
  const double2 d3 = dip ? dip[(i * 3 + 2) * nd + d] : zero;
  const long b = i * 4 * nd + d;
  q[b] = c1;
  dl[b] = d1;
  q[b + nd] = cj(c1);
  dl[b + nd] = csub(cj(d3), cmul(cj(c2), crj));
  q[b + 2 * nd] = cj(c2);
  dl[b + 2 * nd] = make_double2(-d2.x, d2.y);  // -conj(d2)
  q[b + 3 * nd] = zero;
  dl[b + 3 * nd] = cmul(cj(d2), crj);
}

// Velocity and derivatives at n points from the four problems' P, G, H.
__global__ void k_bh_combine(const double* __restrict__ pts, long n, int nd,
                             const double* __restrict__ src, const double2* __restrict__ P,
                             const double2* __restrict__ G, const double2* __restrict__ H,
                             int ifl, double2* __restrict__ pot, double2* __restrict__ grad) {
  const long e = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (e >= n * nd) return;
  const long i = e / nd;
  const int d = (int)(e % nd);
  const double2 r = make_double2(pts[2 * i] - src[0], pts[2 * i + 1] - src[1]);
  const long b = i * 4 * nd + d;
  const double2 g3 = G[b + 2 * nd], g4 = G[b + 3 * nd];
  pot[i * nd + d] = cadd(cadd(P[b], cj(P[b + nd])), cadd(cmul(r, cj(g3)), cj(g4)));
  if (ifl >= 2) {
    grad[(i * 3 + 0) * nd + d] = G[b];
    grad[(i * 3 + 1) * nd + d] = cj(g3);
    grad[(i * 3 + 2) * nd + d] =
        cadd(cj(G[b + nd]), cadd(cmul(r, cj(H[b + 2 * nd])), cj(H[b + 3 * nd])));
  }
}

// Stokeslets and stresslets as biharmonic charges and dipoles
// (stfmm2d.f:145-190): c1 = (-i s1 + s2)/4, c2 = conj(c1);
// z1 = -(-l2 + i l1)/2, z2 = -v2 + i v1, d1 = -i z1 z2, d2 = -conj(d1),
// d3 = i (z1 conj(z2) + conj(z1) z2).
__global__ void k_st_to_bh(long ns, int nd, const double* __restrict__ stoklet,
                           const double* __restrict__ strslet, const double* __restrict__ strsvec,
                           double2* __restrict__ charge, double2* __restrict__ dip) {
  const long e = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (e >= ns * nd) return;
  const long i = e / nd;
  const int d = (int)(e % nd);
  const double2 zero = make_double2(0, 0);
  double2 c1 = zero;
  if (stoklet) {
    const double s1 = stoklet[(i * 2 + 0) * nd + d], s2 = stoklet[(i * 2 + 1) * nd + d];
    c1 = make_double2(s2 / 4, -s1 / 4);
  }
  charge[(i * 2 + 0) * nd + d] = c1;
  charge[(i * 2 + 1) * nd + d] = cj(c1);
  double2 d1 = zero, d2 = zero, d3 = zero;
  if (strslet) {
    const double l1 = strslet[(i * 2 + 0) * nd + d], l2 = strslet[(i * 2 + 1) * nd + d];
    const double v1 = strsvec[(i * 2 + 0) * nd + d], v2 = strsvec[(i * 2 + 1) * nd + d];
    const double2 z1 = make_double2(l2 / 2, -l1 / 2);
    const double2 z2 = make_double2(-v2, v1);
    const double2 p = cmul(z1, z2);
    d1 = make_double2(p.y, -p.x);  // -i p
    d2 = make_double2(-d1.x, d1.y);
    const double2 s = cadd(cmul(z1, cj(z2)), cmul(cj(z1), z2));
    d3 = make_double2(-s.y, s.x);  // i s
  }
  dip[(i * 3 + 0) * nd + d] = d1;
  dip[(i * 3 + 1) * nd + d] = d2;
  dip[(i * 3 + 2) * nd + d] = d3;
}

// zsum(d) = -sum_i c1(d, i), one block per density (fixed summation order).
__global__ void __launch_bounds__(256) k_st_zsum(const double2* __restrict__ charge, long ns,
                                                 int nd, double2* __restrict__ zsum) {
  __shared__ double2 part[256];
  const int d = blockIdx.x;
  double2 acc = make_double2(0, 0);
  for (long i = threadIdx.x; i < ns; i += blockDim.x) acc = cadd(acc, charge[(i * 2) * nd + d]);
  part[threadIdx.x] = acc;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) part[threadIdx.x] = cadd(part[threadIdx.x], part[threadIdx.x + s]);
    __syncthreads();
  }
  if (threadIdx.x == 0) zsum[d] = make_double2(-part[0].x, -part[0].y);
}

// Stokes outputs from the biharmonic ones (stfmm2d.f:222-330); at the
// sources the point's own c1 is added to the velocity as there.
__global__ void k_st_post(long n, int nd, const double2* __restrict__ vel,
                          const double2* __restrict__ bgrad, const double2* __restrict__ zsum,
                          const double2* __restrict__ self_charge, int ifl,
                          double* __restrict__ pot, double* __restrict__ pre,
                          double* __restrict__ grad) {
  const long e = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (e >= n * nd) return;
  const long i = e / nd;
  const int d = (int)(e % nd);
  double2 t = cadd(vel[i * nd + d], zsum[d]);
  if (self_charge) t = cadd(t, self_charge[(i * 2) * nd + d]);
  pot[(i * 2 + 0) * nd + d] = t.y;
  pot[(i * 2 + 1) * nd + d] = -t.x;
  if (ifl >= 2) {
    const double2 g1 = bgrad[(i * 3 + 0) * nd + d];
    pre[i * nd + d] = -4 * g1.y;
    if (ifl >= 3) {
      const double2 g3 = bgrad[(i * 3 + 2) * nd + d];
      auto at = [&](int a, int b) -> double& { return grad[((i * 2 + b) * 2 + a) * nd + d]; };
      at(0, 0) = g3.y;
      at(1, 1) = -g3.y;
      at(1, 0) = 2 * g1.x - g3.x;
      at(0, 1) = -(2 * g1.x + g3.x);
    }
  }
}

}  // namespace

int bh_device(const BhArgs& a, cudaStream_t st) {
  if (a.nd < 1 || a.ns < 0 || a.nt < 0 || a.ifpgh < 0 || a.ifpghtarg < 0 || a.ns > (1L << 30) ||
      a.nt > (1L << 30))
    return IER_BADARG;
  const int nd = a.nd, nd4 = 4 * nd;
  const long ns = a.ns, nt = a.ifpghtarg > 0 ? a.nt : 0;
  const int ifs = std::min(a.ifpgh, 2), ift = std::min(a.ifpghtarg, 2);
  if (ns > 0 && !a.src) return IER_BADARG;
  if (nt > 0 && !a.trg) return IER_BADARG;
  if ((ifs >= 1 && ns && !a.pot) || (ifs >= 2 && ns && !a.grad) || (ift >= 1 && !a.pottarg) ||
      (ift >= 2 && !a.gradtarg))
    return IER_BADARG;
  if (ns == 0 || (!a.charge && !a.dip)) {
    if (ifs >= 1 && ns) B2_CHECK(cudaMemsetAsync(a.pot, 0, sizeof(double2) * nd * ns, st));
    if (ifs >= 2 && ns) B2_CHECK(cudaMemsetAsync(a.grad, 0, sizeof(double2) * 3 * nd * ns, st));
    if (ift >= 1 && nt) B2_CHECK(cudaMemsetAsync(a.pottarg, 0, sizeof(double2) * nd * nt, st));
    if (ift >= 2 && nt) B2_CHECK(cudaMemsetAsync(a.gradtarg, 0, sizeof(double2) * 3 * nd * nt, st));
    B2_CHECK(cudaStreamSynchronize(st));
    return IER_OK;
  }
  DBuf<double2> q(st), dl(st), Ps(st), Gs(st), Hs(st), Pt(st), Gt(st), Ht(st);
  q.alloc((size_t)nd4 * ns, st);
  dl.alloc((size_t)nd4 * ns, st);
  k_bh_dens<<<ceil_div(ns * nd, 256), 256, 0, st>>>(a.src, ns, nd,
                                                    reinterpret_cast<const double2*>(a.charge),
                                                    reinterpret_cast<const double2*>(a.dip), q.p,
                                                    dl.p);
  B2_LAUNCH_CHECK();
  // G of problems 3 and 4 enter the velocity; H for the derivatives
  const int ls = ifs == 0 ? 0 : (ifs >= 2 ? 3 : 2), lt = ift == 0 ? 0 : (ift >= 2 ? 3 : 2);
  auto mk = [&](DBuf<double2>& b, int lev, int need, long n) {
    if (lev < need || n == 0) return (double2*)nullptr;
    b.alloc((size_t)nd4 * n, st);
    return b.p;
  };
  double2 *ps = mk(Ps, ls, 1, ns), *gs = mk(Gs, ls, 2, ns), *hs = mk(Hs, ls, 3, ns);
  double2 *pt = mk(Pt, lt, 1, nt), *gt = mk(Gt, lt, 2, nt), *ht = mk(Ht, lt, 3, nt);
  const double* qd = reinterpret_cast<const double*>(q.p);
  const double* dd = reinterpret_cast<const double*>(dl.p);
  if (a.direct) {
    if (ls) {
      int r = lap_direct_device(0, nd4, ns, a.src, qd, dd, nullptr, ns, a.src, ls, (double*)ps,
                                (double*)gs, (double*)hs, a.thresh, st);
      if (r != IER_OK) return r;
    }
    if (lt) {
      int r = lap_direct_device(0, nd4, ns, a.src, qd, dd, nullptr, nt, a.trg, lt, (double*)pt,
                                (double*)gt, (double*)ht, a.thresh, st);
      if (r != IER_OK) return r;
    }
  } else {
    LapArgs la;
    la.fe = FE_CAUCHY;
    la.nd = nd4;
    la.eps = a.eps;
    la.ns = ns;
    la.src = a.src;
    la.charge = qd;
    la.dipstr = dd;
    la.ifpgh = ls;
    la.pot = (double*)ps;
    la.grad = (double*)gs;
    la.hess = (double*)hs;
    la.nt = nt;
    la.trg = a.trg;
    la.ifpghtarg = lt;
    la.pottarg = (double*)pt;
    la.gradtarg = (double*)gt;
    la.hesstarg = (double*)ht;
    la.ndiv = a.ndiv;
    la.precision = PREC_FP64;  // the combination cancels: keep every sum in FP64
    int r = lap_fmm_device(la, st);
    if (r != IER_OK) return r;
  }
  if (ifs && ns) {
    k_bh_combine<<<ceil_div(ns * nd, 256), 256, 0, st>>>(a.src, ns, nd, a.src, ps, gs, hs, ifs,
                                                         (double2*)a.pot, (double2*)a.grad);
    B2_LAUNCH_CHECK();
  }
  if (ift && nt) {
    k_bh_combine<<<ceil_div(nt * nd, 256), 256, 0, st>>>(a.trg, nt, nd, a.src, pt, gt, ht, ift,
                                                         (double2*)a.pottarg,
                                                         (double2*)a.gradtarg);
    B2_LAUNCH_CHECK();
  }
  B2_CHECK(cudaStreamSynchronize(st));
  return IER_OK;
}

int stokes_device(const StArgs& a, cudaStream_t st) {
  if (a.nd < 1 || a.ns < 0 || a.nt < 0 || a.ifppreg < 0 || a.ifppregtarg < 0) return IER_BADARG;
  if (a.strslet && !a.strsvec) return IER_BADARG;
  const int nd = a.nd;
  const long ns = a.ns, nt = a.ifppregtarg > 0 ? a.nt : 0;
  const int ifs = std::min(a.ifppreg, 3), ift = std::min(a.ifppregtarg, 3);
  if ((ifs >= 1 && ns && !a.pot) || (ifs >= 2 && ns && !a.pre) || (ifs >= 3 && ns && !a.grad) ||
      (ift >= 1 && nt && !a.pottarg) || (ift >= 2 && nt && !a.pretarg) ||
      (ift >= 3 && nt && !a.gradtarg))
    return IER_BADARG;
  if (ns > 0 && !a.src) return IER_BADARG;
  if (nt > 0 && !a.trg) return IER_BADARG;
  DBuf<double2> ch(st), dp(st), zs(st), vs(st), gs(st), vt(st), gt(st);
  const long nb = std::max(ns, 1L);
  ch.alloc((size_t)nd * 2 * nb, st);
  dp.alloc((size_t)nd * 3 * nb, st);
  zs.alloc(nd, st);
  if (ns > 0) {
    k_st_to_bh<<<ceil_div(ns * nd, 256), 256, 0, st>>>(ns, nd, a.stoklet, a.strslet, a.strsvec,
                                                       ch.p, dp.p);
    B2_LAUNCH_CHECK();
  }
  k_st_zsum<<<nd, 256, 0, st>>>(ch.p, ns, nd, zs.p);
  B2_LAUNCH_CHECK();
  BhArgs b;
  b.nd = nd;
  b.eps = a.eps;
  b.ns = ns;
  b.src = a.src;
  b.charge = a.stoklet ? reinterpret_cast<const double*>(ch.p) : nullptr;
  b.dip = a.strslet ? reinterpret_cast<const double*>(dp.p) : nullptr;
  b.ifpgh = std::min(ifs, 2);
  b.nt = nt;
  b.trg = a.trg;
  b.ifpghtarg = std::min(ift, 2);
  b.direct = a.direct;
  b.thresh = a.thresh;
  if (ifs && ns) {
    vs.alloc((size_t)nd * ns, st);
    if (ifs >= 2) gs.alloc((size_t)nd * 3 * ns, st);
    b.pot = (double*)vs.p;
    b.grad = ifs >= 2 ? (double*)gs.p : nullptr;
  }
  if (ift && nt) {
    vt.alloc((size_t)nd * nt, st);
    if (ift >= 2) gt.alloc((size_t)nd * 3 * nt, st);
    b.pottarg = (double*)vt.p;
    b.gradtarg = ift >= 2 ? (double*)gt.p : nullptr;
  }
  int r = bh_device(b, st);
  if (r != IER_OK) return r;
  if (ifs && ns) {
    k_st_post<<<ceil_div(ns * nd, 256), 256, 0, st>>>(ns, nd, vs.p, gs.p, zs.p,
                                                      a.stoklet ? ch.p : nullptr, ifs, a.pot,
                                                      a.pre, a.grad);
    B2_LAUNCH_CHECK();
  }
  if (ift && nt) {
    k_st_post<<<ceil_div(nt * nd, 256), 256, 0, st>>>(nt, nd, vt.p, gt.p, zs.p, nullptr, ift,
                                                      a.pottarg, a.pretarg, a.gradtarg);
    B2_LAUNCH_CHECK();
  }
  B2_CHECK(cudaStreamSynchronize(st));
  return IER_OK;
}

}  // namespace b2
