// Bessel and Hankel functions for the Helmholtz FMM (host and device, FP64).
//
//  * hank01(z): H0^(1)(z), H1^(1)(z) for complex z off the negative real
//    axis, in three regions: |z| <= 4 the ascending series of J0, J1, Y0,
//    Y1 (DLMF 10.2.2, 10.8.1) as polynomials in q = -z^2/4 with precomputed
//    coefficients; 4 < |z| <= 20 J_n by Miller's backward recurrence from
//    order |z| + 32, normalised by J0 + 2 sum J_2k = 1 (DLMF 10.23.E7 /
//    10.12.4), with Y0 and Y1 from Neumann's series (DLMF 10.23.E16 and its
//    derivative); |z| > 20 Hankel's asymptotic expansion (DLMF 10.17.5)
//    truncated at its smallest term.  Relative error ~3e-15 on the real axis,
//    growing like exp(2 Im z) inside |z| <= 20 (2e-14 at Im z = 1.5).
//  * jscaled(N, z, rs, out): out[n] = J_n(z) / rs^n, n = 0..N (the scaled
//    Bessel sequence of jbessel2d, src/common/cdjseval2d.f:5-204), from the
//    series of the two highest retained orders and the backward recurrence
//    F_{n-1} = (2 n rs / z) F_n - rs^2 F_{n+1}; orders whose value is below
//    1e-250 are set to 0.
//  * hscaled(N, z, rs, out): out[n] = H_n(z) rs^n by upward recurrence from
//    H0, H1 (h2dall, src/helmholtz/h2dcommon.f:71-178).
#pragma once
#include <math.h>

#include "common.cuh"

namespace b2 {
namespace helm {

constexpr int NSER = 40;  // series terms available

struct SerTab {
  double c0[NSER];   // 1 / (k!)^2
  double c1[NSER];   // 1 / (k! (k+1)!)
  double cy0[NSER];  // H_k / (k!)^2
  double cy1[NSER];  // (psi(k+1) + psi(k+2)) / (k! (k+1)!)
  double a0[NSER];   // Hankel asymptotic a_k(0)
  double a1[NSER];   // a_k(1)
};

// Filled once per process on the host (helm_tables()) and copied to the
// device constant bank of every translation unit that includes this header
// (c_ser has internal linkage: each such unit uploads its own copy).
const SerTab& helm_tables();
#ifdef __CUDACC__
static __constant__ SerTab c_ser;
#endif

__host__ __device__ __forceinline__ const SerTab& ser_tab() {
#ifdef __CUDA_ARCH__
  return c_ser;
#else
  return helm_tables();
#endif
}

__host__ __device__ __forceinline__ double2 cexp_i(double2 z) {
  // exp(i z)
  double s, c;
  sincos(z.x, &s, &c);
  double m = exp(-z.y);
  return make_double2(m * c, m * s);
}

__host__ __device__ __forceinline__ double2 csqrt_(double2 z) {
  double r = hypot(z.x, z.y);
  double a = sqrt(0.5 * (r + fabs(z.x)));
  if (a == 0.0) return make_double2(0.0, 0.0);
  double b = z.y / (2.0 * a);
  if (z.x >= 0) return make_double2(a, b);
  return make_double2(fabs(b), z.y >= 0 ? a : -a);
}

__host__ __device__ __forceinline__ double2 clog_(double2 z) {
  return make_double2(log(hypot(z.x, z.y)), atan2(z.y, z.x));
}

// Number of series terms that reach ~1e-17 for |q| = |z|^2/4.
__host__ __device__ __forceinline__ int nser_for(double aq) {
  if (aq < 1e-8) return 4;
  if (aq < 1e-3) return 7;
  if (aq < 0.25) return 12;
  if (aq < 4.0) return 18;
  if (aq < 16.0) return 25;
  if (aq < 25.0) return 29;
  return NSER - 1;
}

// Miller + Neumann evaluation for 4 < |z| <= 20.  f_n (unnormalised J_n)
// is produced downwards; the sums over even orders 2k use f_2k and the odd
// neighbours f_2k-1, f_2k+1, so the loop keeps the last three values.
__host__ __device__ inline void hank01_neumann(double2 z, bool real_z, double2& h0,
                                               double2& h1) {
  const double pi = 3.14159265358979323846, eg = 0.57721566490153286061;
  double az = hypot(z.x, z.y);
  int n0 = (int)az + 32;
  n0 += n0 & 1;  // even start
  double2 zi2 = cscale(crcp(z), 2.0);
  if (real_z) zi2 = make_double2(2.0 / z.x, 0.0);
  double2 fa = make_double2(0, 0);      // f_{n+1}
  double2 fb = make_double2(1e-30, 0);  // f_n, n = n0
  double2 nrm = make_double2(0, 0), sy0 = make_double2(0, 0), sy1 = make_double2(0, 0);
  // f_{n0+1} = 0 and f_{n0} enter the sums: n0 is even, k = n0 / 2
  {
    int k = n0 >> 1;
    double sg = (k & 1) ? -1.0 : 1.0;
    nrm = cadd(nrm, fb);
    sy0 = cadd(sy0, cscale(fb, sg / k));
  }
  double2 f_odd_above = fa;  // f_{2k+1} of the pending even order 2k
  int k_even = n0 >> 1;
  double2 j1 = make_double2(0, 0);
  for (int n = n0; n >= 1; n--) {
    double2 t = real_z ? make_double2(zi2.x * n * fb.x - fa.x, 0.0)
                       : csub(cscale(cmul(zi2, fb), (double)n), fa);
    fa = fb;
    fb = t;  // fb = f_{n-1}
    int m = n - 1;
    if (m & 1) {
      // odd order m = 2k - 1 closes the pending even order 2k = m + 1
      if (k_even >= 1) {
        double sg = (k_even & 1) ? -1.0 : 1.0;
        sy1 = cadd(sy1, cscale(csub(fb, f_odd_above), sg / k_even));
      }
      f_odd_above = fb;  // becomes f_{2k+1} for the even order m - 1
      if (m == 1) j1 = fb;
    } else if (m >= 2) {
      int k = m >> 1;
      double sg = (k & 1) ? -1.0 : 1.0;
      nrm = cadd(nrm, fb);
      sy0 = cadd(sy0, cscale(fb, sg / k));
      k_even = k;
    }
  }
  double2 f0 = fb;
  double2 s = cadd(f0, cscale(nrm, 2.0));
  double2 is = crcp(s);
  double2 J0 = cmul(f0, is), J1 = cmul(j1, is);
  double2 Sy0 = cmul(sy0, is), Sy1 = cmul(sy1, is);
  double2 L = clog_(make_double2(0.5 * z.x, 0.5 * z.y));
  L.x += eg;
  double2 Y0 = csub(cscale(cmul(L, J0), 2.0 / pi), cscale(Sy0, 4.0 / pi));
  double2 Y1 = cscale(cmul(J0, crcp(z)), -2.0 / pi);
  Y1 = cadd(Y1, cscale(cmul(L, J1), 2.0 / pi));
  Y1 = cadd(Y1, cscale(Sy1, 2.0 / pi));
  h0 = make_double2(J0.x - Y0.y, J0.y + Y0.x);  // J + i Y
  h1 = make_double2(J1.x - Y1.y, J1.y + Y1.x);
}

__host__ __device__ inline void hank01_real(double x, double2& h0, double2& h1) {
  const double pi = 3.14159265358979323846, eg = 0.57721566490153286061;
  const SerTab& T = ser_tab();
  if (x > 4.0 && x <= 20.0) {
    hank01_neumann(make_double2(x, 0.0), true, h0, h1);
    return;
  }
  if (x <= 4.0) {
    double q = -0.25 * x * x;
    int K = nser_for(fabs(q));
    double p0 = T.c0[K], p1 = T.c1[K], py0 = T.cy0[K], py1 = T.cy1[K];
    for (int k = K - 1; k >= 0; k--) {
      p0 = fma(p0, q, T.c0[k]);
      p1 = fma(p1, q, T.c1[k]);
      py0 = fma(py0, q, T.cy0[k]);
      py1 = fma(py1, q, T.cy1[k]);
    }
    double lz = log(0.5 * x);
    double j0 = p0, j1 = 0.5 * x * p1;
    double y0 = (2.0 / pi) * (lz + eg) * j0 - (2.0 / pi) * py0;
    double y1 = -2.0 / (pi * x) + (2.0 / pi) * lz * j1 - (x / (2.0 * pi)) * py1;
    h0 = make_double2(j0, y0);
    h1 = make_double2(j1, y1);
    return;
  }
  // asymptotic: H_nu = sqrt(2/(pi x)) e^{i(x - nu pi/2 - pi/4)} sum i^k a_k / x^k
  double ix = 1.0 / x;
  double2 s0 = make_double2(1.0, 0.0), s1 = make_double2(1.0, 0.0);
  double p = 1.0, last0 = 1e300, last1 = 1e300;
  bool go0 = true, go1 = true;
  for (int k = 1; k < NSER && (go0 || go1); k++) {
    p *= ix;
    // i^k
    double re = (k % 4 == 0) ? 1.0 : (k % 4 == 2 ? -1.0 : 0.0);
    double im = (k % 4 == 1) ? 1.0 : (k % 4 == 3 ? -1.0 : 0.0);
    double t0 = T.a0[k] * p, t1 = T.a1[k] * p;
    if (go0) {
      if (fabs(t0) > last0) {
        go0 = false;
      } else {
        s0.x += re * t0;
        s0.y += im * t0;
        last0 = fabs(t0);
        if (last0 < 1e-18) go0 = false;
      }
    }
    if (go1) {
      if (fabs(t1) > last1) {
        go1 = false;
      } else {
        s1.x += re * t1;
        s1.y += im * t1;
        last1 = fabs(t1);
        if (last1 < 1e-18) go1 = false;
      }
    }
  }
  double amp = sqrt(2.0 / (pi * x));
  double s, c;
  sincos(x - 0.25 * pi, &s, &c);
  double2 e0 = make_double2(amp * c, amp * s);     // e^{i(x - pi/4)}
  double2 e1 = make_double2(amp * s, -amp * c);    // e^{i(x - 3pi/4)} = -i e0
  h0 = cmul(e0, s0);
  h1 = cmul(e1, s1);
}

__host__ __device__ inline void hank01(double2 z, double2& h0, double2& h1) {
  if (z.y == 0.0 && z.x > 0.0) {
    hank01_real(z.x, h0, h1);
    return;
  }
  const double pi = 3.14159265358979323846, eg = 0.57721566490153286061;
  const SerTab& T = ser_tab();
  double az = hypot(z.x, z.y);
  if (az > 4.0 && az <= 20.0) {
    hank01_neumann(z, false, h0, h1);
    return;
  }
  if (az <= 4.0) {
    double2 q = cmul(z, z);
    q = make_double2(-0.25 * q.x, -0.25 * q.y);
    int K = nser_for(0.25 * az * az);
    double2 p0 = make_double2(T.c0[K], 0), p1 = make_double2(T.c1[K], 0);
    double2 py0 = make_double2(T.cy0[K], 0), py1 = make_double2(T.cy1[K], 0);
    for (int k = K - 1; k >= 0; k--) {
      p0 = cadd(cmul(p0, q), make_double2(T.c0[k], 0));
      p1 = cadd(cmul(p1, q), make_double2(T.c1[k], 0));
      py0 = cadd(cmul(py0, q), make_double2(T.cy0[k], 0));
      py1 = cadd(cmul(py1, q), make_double2(T.cy1[k], 0));
    }
    double2 lz = clog_(make_double2(0.5 * z.x, 0.5 * z.y));
    double2 j0 = p0, j1 = cmul(make_double2(0.5 * z.x, 0.5 * z.y), p1);
    double2 y0 = csub(cscale(cmul(make_double2(lz.x + eg, lz.y), j0), 2.0 / pi), cscale(py0, 2.0 / pi));
    double2 y1 = cscale(crcp(z), -2.0 / pi);
    y1 = cadd(y1, cscale(cmul(lz, j1), 2.0 / pi));
    y1 = csub(y1, cscale(cmul(z, py1), 1.0 / (2.0 * pi)));
    h0 = make_double2(j0.x - y0.y, j0.y + y0.x);  // J + i Y
    h1 = make_double2(j1.x - y1.y, j1.y + y1.x);
    return;
  }
  double2 iz = crcp(z);
  double2 s0 = make_double2(1.0, 0.0), s1 = make_double2(1.0, 0.0);
  double2 p = make_double2(1.0, 0.0);
  double last0 = 1e300, last1 = 1e300;
  bool go0 = true, go1 = true;
  for (int k = 1; k < NSER && (go0 || go1); k++) {
    p = cmul(p, make_double2(-iz.y, iz.x));  // (i/z)^k
    double2 t0 = cscale(p, T.a0[k]), t1 = cscale(p, T.a1[k]);
    double m0 = hypot(t0.x, t0.y), m1 = hypot(t1.x, t1.y);
    if (go0) {
      if (m0 > last0) go0 = false;
      else {
        s0 = cadd(s0, t0);
        last0 = m0;
        if (m0 < 1e-18) go0 = false;
      }
    }
    if (go1) {
      if (m1 > last1) go1 = false;
      else {
        s1 = cadd(s1, t1);
        last1 = m1;
        if (m1 < 1e-18) go1 = false;
      }
    }
  }
  double2 amp = csqrt_(cscale(iz, 2.0 / pi));
  double2 e0 = cmul(amp, cexp_i(make_double2(z.x - 0.25 * pi, z.y)));
  double2 e1 = make_double2(e0.y, -e0.x);  // times -i
  h0 = cmul(e0, s0);
  h1 = cmul(e1, s1);
}

// out[n] = H_n(z) rs^n, n = 0..N (zero for |z| < 1e-200).
__host__ __device__ inline void hscaled(int N, double2 z, double rs, double2* out) {
  if (hypot(z.x, z.y) < 1e-200) {
    for (int i = 0; i <= N; i++) out[i] = make_double2(0, 0);
    return;
  }
  double2 h0, h1;
  hank01(z, h0, h1);
  out[0] = h0;
  if (N >= 1) out[1] = cscale(h1, rs);
  double s2 = rs * rs;
  double2 zinv = cscale(crcp(z), rs);
  for (int i = 1; i < N; i++) {
    double2 a = cmul(cscale(zinv, 2.0 * i), out[i]);
    out[i + 1] = csub(a, cscale(out[i - 1], s2));
  }
}

// Start of the downward recurrence for F_n = J_n(z) / rs^n, n <= N: the
// highest order M kept (S >= max(N, |z| + 10, |z|^2 / 10), where the series of
// F_S has little cancellation, or the highest order whose leading factor
// (|z| / 2 rs)^n / n! is above 1e-250; orders above M are 0) and F_M, F_{M-1}
// from their power series.  False for |z| < 1e-200 (F_0 = 1, the rest 0).
// The caller continues with F_{n-1} = (2 n rs / z) F_n - rs^2 F_{n+1}.
__host__ __device__ inline bool jstart(int N, double2 z, double rs, int& M, double2& f_hi,
                                       double2& f_lo) {
  double az = hypot(z.x, z.y);
  if (az < 1e-200) return false;
  double2 w = cscale(z, 0.5 / rs);
  double aw = 0.5 * az / rs;
  // the series of F_S sums terms up to ~exp(|z|^2 / 4S) times its value:
  // S >= |z|^2 / 10 keeps that factor below e^2.5
  int S = N > (int)az + 10 ? N : (int)az + 10;
  if (az < 200.0 && S < (int)(0.1 * az * az) + 1) S = (int)(0.1 * az * az) + 1;
  if (S < 1) S = 1;
  M = S;
  {
    double lt = 1.0;  // the leading factor (|z| / 2 rs)^n / n!
    for (int n = 1; n <= S; n++) {
      lt *= aw / n;
      if (lt < 1e-250) {
        M = n - 1;
        break;
      }
    }
  }
  if (M < 1) M = 1;
  // F_m = t_m sum_k (-z^2/4)^k m! / (k! (m+k)!), t_m = w^m / m!, m = M, M-1
  double2 q = cmul(z, z);
  q = make_double2(-0.25 * q.x, -0.25 * q.y);
  double2 tM = make_double2(1, 0);
  for (int n = 1; n <= M; n++) tM = cscale(cmul(tM, w), 1.0 / n);
  double2 sr[2];
  for (int s = 0; s < 2; s++) {
    int m = M - s;
    double2 term = make_double2(1, 0), sum = make_double2(1, 0);
    for (int k = 1; k < 400; k++) {
      term = cscale(cmul(term, q), 1.0 / ((double)k * (double)(m + k)));
      sum = cadd(sum, term);
      if (hypot(term.x, term.y) < 1e-17 * hypot(sum.x, sum.y)) break;
    }
    sr[s] = sum;
  }
  f_hi = cmul(tM, sr[0]);                                   // F_M
  f_lo = cmul(cscale(cmul(tM, crcp(w)), (double)M), sr[1]);  // F_{M-1}
  return true;
}

// out[n] = J_n(z) / rs^n, n = 0..N (jstart + the downward recurrence).
__host__ __device__ inline void jscaled(int N, double2 z, double rs, double2* out) {
  int M = 0;
  double2 f_hi, f_lo;
  if (!jstart(N, z, rs, M, f_hi, f_lo)) {
    out[0] = make_double2(1, 0);
    for (int i = 1; i <= N; i++) out[i] = make_double2(0, 0);
    return;
  }
  for (int n = M + 1; n <= N; n++) out[n] = make_double2(0, 0);
  if (M <= N) out[M] = f_hi;
  if (M - 1 <= N) out[M - 1] = f_lo;
  double2 c = cscale(crcp(z), 2.0 * rs);
  double s2 = rs * rs;
  for (int n = M - 1; n >= 1; n--) {
    // F_{n-1} = (2 n rs / z) F_n - rs^2 F_{n+1}
    double2 nx = csub(cmul(cscale(c, (double)n), f_lo), cscale(f_hi, s2));
    f_hi = f_lo;
    f_lo = nx;
    if (n - 1 <= N) out[n - 1] = nx;
  }
}

}  // namespace helm
}  // namespace b2
