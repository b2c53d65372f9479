// Learned cost model: a small MLP (nin -> H1 -> H2 -> 1, tanh hidden layers,
// linear output) with hand-written forward, backward and Adam kernels, and
// the point-distribution statistics it reads.
//
// Parameters are one flat FP32 array:
//   W1 [H1][nin], b1 [H1], W2 [H2][H1], b2 [H2], w3 [H2], b3 [1].
// Training minimises the mean squared error over a batch of B samples.
#include "mlp.cuh"

namespace b2 {

namespace {

constexpr int MLP_MAXH = 64;
constexpr int MLP_MAXIN = 32;

struct Off {
  int W1, b1, W2, b2, w3, b3, n;
};

__host__ __device__ inline Off offsets(int nin, int H1, int H2) {
  Off o;
  o.W1 = 0;
  o.b1 = o.W1 + H1 * nin;
  o.W2 = o.b1 + H1;
  o.b2 = o.W2 + H2 * H1;
  o.w3 = o.b2 + H2;
  o.b3 = o.w3 + H2;
  o.n = o.b3 + 1;
  return o;
}

// One sample per thread: activations A1 [B][H1], A2 [B][H2] (kept for the
// backward pass when non-null) and the output Y [B].
__global__ void k_mlp_fwd(const float* __restrict__ X, int B, int nin, int H1, int H2,
                          const float* __restrict__ prm, float* __restrict__ A1,
                          float* __restrict__ A2, float* __restrict__ Y) {
  extern __shared__ float sp[];
  const Off o = offsets(nin, H1, H2);
  for (int e = threadIdx.x; e < o.n; e += blockDim.x) sp[e] = prm[e];
  __syncthreads();
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= B) return;
  float x[MLP_MAXIN], a1[MLP_MAXH];
  for (int i = 0; i < nin; i++) x[i] = X[(size_t)s * nin + i];
  for (int h = 0; h < H1; h++) {
    float z = sp[o.b1 + h];
    for (int i = 0; i < nin; i++) z = fmaf(sp[o.W1 + h * nin + i], x[i], z);
    a1[h] = tanhf(z);
    if (A1) A1[(size_t)s * H1 + h] = a1[h];
  }
  float y = sp[o.b3];
  for (int h = 0; h < H2; h++) {
    float z = sp[o.b2 + h];
    for (int i = 0; i < H1; i++) z = fmaf(sp[o.W2 + h * H1 + i], a1[i], z);
    float a2 = tanhf(z);
    if (A2) A2[(size_t)s * H2 + h] = a2;
    y = fmaf(sp[o.w3 + h], a2, y);
  }
  Y[s] = y;
}

// Per-sample error signals: dY = 2 (Y - T) / B, dZ2 = dY w3 (1 - A2^2),
// dZ1 = (W2^T dZ2) (1 - A1^2).
__global__ void k_mlp_bwd_sample(const float* __restrict__ Y, const float* __restrict__ T, int B,
                                 int nin, int H1, int H2, const float* __restrict__ prm,
                                 const float* __restrict__ A1, const float* __restrict__ A2,
                                 float* __restrict__ dY, float* __restrict__ dZ1,
                                 float* __restrict__ dZ2) {
  extern __shared__ float sp[];
  const Off o = offsets(nin, H1, H2);
  for (int e = threadIdx.x; e < o.n; e += blockDim.x) sp[e] = prm[e];
  __syncthreads();
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= B) return;
  float dy = 2.f * (Y[s] - T[s]) / (float)B;
  dY[s] = dy;
  float dz2[MLP_MAXH];
  for (int h = 0; h < H2; h++) {
    float a = A2[(size_t)s * H2 + h];
    dz2[h] = dy * sp[o.w3 + h] * (1.f - a * a);
    dZ2[(size_t)s * H2 + h] = dz2[h];
  }
  for (int i = 0; i < H1; i++) {
    float g = 0.f;
    for (int h = 0; h < H2; h++) g = fmaf(sp[o.W2 + h * H1 + i], dz2[h], g);
    float a = A1[(size_t)s * H1 + i];
    dZ1[(size_t)s * H1 + i] = g * (1.f - a * a);
  }
}

// One parameter per thread: its gradient summed over the batch.
__global__ void k_mlp_bwd_reduce(const float* __restrict__ X, int B, int nin, int H1, int H2,
                                 const float* __restrict__ A1, const float* __restrict__ A2,
                                 const float* __restrict__ dY, const float* __restrict__ dZ1,
                                 const float* __restrict__ dZ2, float* __restrict__ grad) {
  const Off o = offsets(nin, H1, H2);
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= o.n) return;
  float g = 0.f;
  if (e < o.b1) {
    int h = e / nin, i = e % nin;
    for (int s = 0; s < B; s++) g = fmaf(dZ1[(size_t)s * H1 + h], X[(size_t)s * nin + i], g);
  } else if (e < o.W2) {
    int h = e - o.b1;
    for (int s = 0; s < B; s++) g += dZ1[(size_t)s * H1 + h];
  } else if (e < o.b2) {
    int h = (e - o.W2) / H1, i = (e - o.W2) % H1;
    for (int s = 0; s < B; s++) g = fmaf(dZ2[(size_t)s * H2 + h], A1[(size_t)s * H1 + i], g);
  } else if (e < o.w3) {
    int h = e - o.b2;
    for (int s = 0; s < B; s++) g += dZ2[(size_t)s * H2 + h];
  } else if (e < o.b3) {
    int h = e - o.w3;
    for (int s = 0; s < B; s++) g = fmaf(dY[s], A2[(size_t)s * H2 + h], g);
  } else {
    for (int s = 0; s < B; s++) g += dY[s];
  }
  grad[e] = g;
}

__global__ void k_mlp_loss(const float* __restrict__ Y, const float* __restrict__ T, int B,
                           float* __restrict__ loss) {
  __shared__ float red[256];
  float v = 0.f;
  for (int s = threadIdx.x; s < B; s += blockDim.x) {
    float d = Y[s] - T[s];
    v += d * d;
  }
  red[threadIdx.x] = v;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) *loss = red[0] / (float)B;
}

// Adam (Kingma & Ba 2015) with bias correction; t >= 1.
__global__ void k_adam(float* __restrict__ prm, const float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, int n, float lr, float b1, float b2, float eps,
                       int t) {
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  float gm = b1 * m[e] + (1.f - b1) * g[e];
  float gv = b2 * v[e] + (1.f - b2) * g[e] * g[e];
  m[e] = gm;
  v[e] = gv;
  float mh = gm / (1.f - powf(b1, (float)t)), vh = gv / (1.f - powf(b2, (float)t));
  prm[e] -= lr * mh / (sqrtf(vh) + eps);
}

// Bounding box of the points: per-block partial (xmin, -xmax, ymin, -ymax).
__global__ void k_stats_bbox(const double* __restrict__ src, long ns, const double* __restrict__ trg,
                             long nt, double4* __restrict__ part) {
  __shared__ double r[4][256];
  double x0 = 1e300, x1 = 1e300, y0 = 1e300, y1 = 1e300;
  for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < ns + nt;
       k += (long)gridDim.x * blockDim.x) {
    const double* p = k < ns ? src + 2 * k : trg + 2 * (k - ns);
    x0 = fmin(x0, p[0]);
    x1 = fmin(x1, -p[0]);
    y0 = fmin(y0, p[1]);
    y1 = fmin(y1, -p[1]);
  }
  r[0][threadIdx.x] = x0;
  r[1][threadIdx.x] = x1;
  r[2][threadIdx.x] = y0;
  r[3][threadIdx.x] = y1;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w)
      for (int c = 0; c < 4; c++) r[c][threadIdx.x] = fmin(r[c][threadIdx.x], r[c][threadIdx.x + w]);
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = make_double4(r[0][0], r[1][0], r[2][0], r[3][0]);
}

__global__ void k_stats_bbox_final(const double4* __restrict__ part, int n,
                                   double* __restrict__ bb) {
  if (threadIdx.x != 0) return;
  double4 a = make_double4(1e300, 1e300, 1e300, 1e300);
  for (int i = 0; i < n; i++) {
    a.x = fmin(a.x, part[i].x);
    a.y = fmin(a.y, part[i].y);
    a.z = fmin(a.z, part[i].z);
    a.w = fmin(a.w, part[i].w);
  }
  bb[0] = a.x;
  bb[1] = -a.y;
  bb[2] = a.z;
  bb[3] = -a.w;
}

// Occupancy histogram of the points on a 128 x 128 grid over the square
// that holds them (the FMM's root box): per-block counts in shared memory,
// then the non-empty bins are added to the global histogram.
__global__ void k_stats_hist(const double* __restrict__ src, long ns, const double* __restrict__ trg,
                             long nt, const double* __restrict__ bb, unsigned* __restrict__ hist) {
  extern __shared__ unsigned sh[];
  for (int e = threadIdx.x; e < 128 * 128; e += blockDim.x) sh[e] = 0;
  __syncthreads();
  double w = fmax(bb[1] - bb[0], bb[3] - bb[2]);
  double cx = 0.5 * (bb[0] + bb[1]), cy = 0.5 * (bb[2] + bb[3]);
  double inv = w > 0 ? 128.0 / w : 0.0;
  for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < ns + nt;
       k += (long)gridDim.x * blockDim.x) {
    const double* p = k < ns ? src + 2 * k : trg + 2 * (k - ns);
    int ix = min(127, max(0, (int)floor((p[0] - (cx - 0.5 * w)) * inv)));
    int iy = min(127, max(0, (int)floor((p[1] - (cy - 0.5 * w)) * inv)));
    atomicAdd(&sh[iy * 128 + ix], 1u);
  }
  __syncthreads();
  for (int e = threadIdx.x; e < 128 * 128; e += blockDim.x)
    if (sh[e]) atomicAdd(&hist[e], sh[e]);
}

}  // namespace

int mlp_param_count(int nin, int H1, int H2) { return offsets(nin, H1, H2).n; }

static bool mlp_shape_ok(int nin, int H1, int H2) {
  return nin >= 1 && nin <= MLP_MAXIN && H1 >= 1 && H1 <= MLP_MAXH && H2 >= 1 && H2 <= MLP_MAXH;
}

int mlp_forward(const float* X, int B, int nin, int H1, int H2, const float* prm, float* Y,
                cudaStream_t st) {
  if (!mlp_shape_ok(nin, H1, H2) || B < 0) return IER_BADARG;
  if (B == 0) return IER_OK;
  size_t sm = sizeof(float) * mlp_param_count(nin, H1, H2);
  k_mlp_fwd<<<ceil_div(B, 128), 128, sm, st>>>(X, B, nin, H1, H2, prm, nullptr, nullptr, Y);
  B2_LAUNCH_CHECK();
  return IER_OK;
}

int mlp_gradient(const float* X, const float* T, int B, int nin, int H1, int H2,
                 const float* prm, float* grad, float* loss, cudaStream_t st) {
  if (!mlp_shape_ok(nin, H1, H2) || B < 1) return IER_BADARG;
  const int np = mlp_param_count(nin, H1, H2);
  size_t sm = sizeof(float) * np;
  DBuf<float> A1(st), A2(st), Y(st), dY(st), dZ1(st), dZ2(st);
  A1.alloc((size_t)B * H1, st);
  A2.alloc((size_t)B * H2, st);
  Y.alloc(B, st);
  dY.alloc(B, st);
  dZ1.alloc((size_t)B * H1, st);
  dZ2.alloc((size_t)B * H2, st);
  k_mlp_fwd<<<ceil_div(B, 128), 128, sm, st>>>(X, B, nin, H1, H2, prm, A1.p, A2.p, Y.p);
  B2_LAUNCH_CHECK();
  if (loss) {
    k_mlp_loss<<<1, 256, 0, st>>>(Y.p, T, B, loss);
    B2_LAUNCH_CHECK();
  }
  k_mlp_bwd_sample<<<ceil_div(B, 128), 128, sm, st>>>(Y.p, T, B, nin, H1, H2, prm, A1.p, A2.p,
                                                      dY.p, dZ1.p, dZ2.p);
  B2_LAUNCH_CHECK();
  k_mlp_bwd_reduce<<<ceil_div(np, 128), 128, 0, st>>>(X, B, nin, H1, H2, A1.p, A2.p, dY.p, dZ1.p,
                                                      dZ2.p, grad);
  B2_LAUNCH_CHECK();
  return IER_OK;
}

int mlp_train(const float* X, const float* T, int B, int nin, int H1, int H2, float* prm,
              int steps, float lr, float* loss_hist, cudaStream_t st) {
  if (!mlp_shape_ok(nin, H1, H2) || B < 1 || steps < 0) return IER_BADARG;
  const int np = mlp_param_count(nin, H1, H2);
  DBuf<float> g(st), m(st), v(st), loss(st);
  g.alloc(np, st);
  m.alloc(np, st);
  v.alloc(np, st);
  loss.alloc(std::max(steps, 1), st);
  m.zero(np);
  v.zero(np);
  for (int t = 1; t <= steps; t++) {
    int r = mlp_gradient(X, T, B, nin, H1, H2, prm, g.p, loss.p + (t - 1), st);
    if (r != IER_OK) return r;
    k_adam<<<ceil_div(np, 128), 128, 0, st>>>(prm, g.p, m.p, v.p, np, lr, 0.9f, 0.999f, 1e-8f, t);
    B2_LAUNCH_CHECK();
  }
  if (loss_hist && steps > 0)
    B2_CHECK(cudaMemcpyAsync(loss_hist, loss.p, sizeof(float) * steps, cudaMemcpyDeviceToHost, st));
  B2_CHECK(cudaStreamSynchronize(st));
  return IER_OK;
}

int point_stats(const double* src, long ns, const double* trg, long nt, unsigned* hist,
                cudaStream_t st) {
  if (ns < 0 || nt < 0 || (ns > 0 && !src) || (nt > 0 && !trg)) return IER_BADARG;
  B2_CHECK(cudaMemsetAsync(hist, 0, sizeof(unsigned) * 128 * 128, st));
  if (ns + nt == 0) {
    B2_CHECK(cudaStreamSynchronize(st));
    return IER_OK;
  }
  const int nblk = (int)std::min<long>(296, (ns + nt + 255) / 256);
  DBuf<double4> part(st);
  DBuf<double> bb(st);
  part.alloc(nblk, st);
  bb.alloc(4, st);
  k_stats_bbox<<<nblk, 256, 0, st>>>(src, ns, trg, nt, part.p);
  B2_LAUNCH_CHECK();
  k_stats_bbox_final<<<1, 32, 0, st>>>(part.p, nblk, bb.p);
  B2_LAUNCH_CHECK();
  const size_t sm = sizeof(unsigned) * 128 * 128;
  set_smem_attr(k_stats_hist, sm);
  k_stats_hist<<<nblk, 256, sm, st>>>(src, ns, trg, nt, bb.p, hist);
  B2_LAUNCH_CHECK();
  B2_CHECK(cudaStreamSynchronize(st));
  return IER_OK;
}

}  // namespace b2
