// Learned cost model kernels (small MLP) and point-distribution statistics.
#pragma once
#include "common.cuh"

namespace b2 {

int mlp_param_count(int nin, int H1, int H2);

// Y [B] = MLP(X [B][nin]) for the flat parameter array prm (device pointers).
int mlp_forward(const float* X, int B, int nin, int H1, int H2, const float* prm, float* Y,
                cudaStream_t st);

// Gradient of the mean squared error mean_b (Y_b - T_b)^2 with respect to
// every parameter (grad has mlp_param_count entries); *loss (device) gets
// the loss at prm when loss is non-null.
int mlp_gradient(const float* X, const float* T, int B, int nin, int H1, int H2,
                 const float* prm, float* grad, float* loss, cudaStream_t st);

// `steps` full-batch Adam steps (lr, betas 0.9 / 0.999) on prm in place;
// loss_hist (host, `steps` entries, may be null) receives the loss before
// each step.  Synchronises the stream.
int mlp_train(const float* X, const float* T, int B, int nin, int H1, int H2, float* prm,
              int steps, float lr, float* loss_hist, cudaStream_t st);

// 128 x 128 occupancy histogram of sources and targets over the square that
// holds them (device hist, row-major, iy * 128 + ix).  Synchronises.
int point_stats(const double* src, long ns, const double* trg, long nt, unsigned* hist,
                cudaStream_t st);

}  // namespace b2
