// Complex FFT of a 5-smooth length (2^a 3^b 5^c), one thread block per
// transform, in shared memory: the signatures of the wideband Helmholtz
// translations (src/helmholtz/wideband2d.f h2d_mptosig / h2d_sig2exp call
// FFTPACK's zfftf / zfftb on lengths next235(...)).
//
// Conventions as FFTPACK, unnormalised:
//   forward  (dir = -1): X_k = sum_j x_j exp(-2 pi i j k / n)
//   backward (dir = +1): x_j = sum_k X_k exp(+2 pi i j k / n)
//
// Algorithm: self-sorting Stockham, decimation in frequency.  A stage of
// radix r on a sub-length nc (stride s, nc s = n) maps
//   y[q + s (r p + v)] = w^(p v) sum_u x[q + s (p + u m)] e^(dir 2 pi i u v / r),
//   m = nc / r, w = e^(dir 2 pi i / nc), p < m, q < s,
// then continues on nc / r with stride s r; the output ends in natural order.
#pragma once
#include "common.cuh"

namespace b2 {
namespace fft {

constexpr int MAXF = 32;  // factors of a length (2^a 3^b 5^c, n < 2^31)

struct Plan {
  int n, nf;
  int f[MAXF];  // radices, 4s first, then 2, 3, 5
};

// Factorisation of a 5-smooth n (false otherwise).
__host__ __device__ inline bool plan(int n, Plan& P) {
  P.n = n;
  P.nf = 0;
  if (n < 1) return false;
  int m = n;
  while (m % 4 == 0 && P.nf < MAXF) { P.f[P.nf++] = 4; m /= 4; }
  while (m % 2 == 0 && P.nf < MAXF) { P.f[P.nf++] = 2; m /= 2; }
  while (m % 3 == 0 && P.nf < MAXF) { P.f[P.nf++] = 3; m /= 3; }
  while (m % 5 == 0 && P.nf < MAXF) { P.f[P.nf++] = 5; m /= 5; }
  return m == 1;
}

// Smallest even 5-smooth integer >= n (src/common/next235.f: the search
// starts at 2 ceil(n / 2) and steps by 2).
__host__ __device__ inline int next235(int n) {
  int k = 2 * ((n + 1) / 2);
  if (k <= 0) k = 2;
  for (;; k += 2) {
    int m = k;
    while (m % 2 == 0) m /= 2;
    while (m % 3 == 0) m /= 3;
    while (m % 5 == 0) m /= 5;
    if (m == 1) return k;
  }
}

// e^(dir 2 pi i a / b)
__device__ __forceinline__ double2 unit(long a, long b, int dir) {
  double s, c;
  sincospi(2.0 * (double)(a % b) / (double)b, &s, &c);
  return make_double2(c, dir * s);
}

// One transform of P.n points held in x (shared memory), y of the same
// size as scratch; all threads of the block take part.  Returns the buffer
// that holds the result (x or y).
__device__ inline double2* block_fft(const Plan& P, double2* x, double2* y, int dir) {
  const int n = P.n;
  int nc = n, s = 1;
  for (int st = 0; st < P.nf; st++) {
    const int r = P.f[st], m = nc / r;
    __syncthreads();
    for (int t = threadIdx.x; t < m * s; t += blockDim.x) {
      const int p = t / s, q = t - p * s;
      double2 a[5];
      for (int u = 0; u < r; u++) a[u] = x[q + s * (p + u * m)];
      for (int v = 0; v < r; v++) {
        double2 acc = a[0];
        for (int u = 1; u < r; u++) cfma(acc, a[u], unit((long)u * v, r, dir));
        if (v > 0 && p > 0) acc = cmul(acc, unit((long)p * v, nc, dir));
        y[q + s * (r * p + v)] = acc;
      }
    }
    double2* tmp = x;
    x = y;
    y = tmp;
    nc = m;
    s *= r;
  }
  __syncthreads();
  return x;
}

}  // namespace fft
}  // namespace b2
