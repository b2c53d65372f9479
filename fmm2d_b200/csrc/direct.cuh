// All-pairs sums on the device (c2ddir / l2ddir / r2ddir of the python API).
#pragma once
#include "common.cuh"

namespace b2 {

// kind 0: Cauchy (cauchykernels2d.f), 1: complex Laplace (lapkernels2d.f),
// 2: real Laplace (rlapkernels2d.f).  Device pointers; outputs overwritten.
int lap_direct_device(int kind, int nd, long ns, const double* src, const double* charge,
                      const double* dipstr, const double* dipvec, long nt, const double* trg,
                      int ifpgh, double* pot, double* grad, double* hess, double thresh,
                      cudaStream_t st);

// Same sums with the partial-sum scratch taken from a static device array
// instead of the memory pool (no device allocation at all); rejects target
// counts whose partials do not fit (IER_NOALLOC_TOO_LARGE).
int lap_direct_device_noalloc(int kind, int nd, long ns, const double* src, const double* charge,
                              const double* dipstr, const double* dipvec, long nt,
                              const double* trg, int ifpgh, double* pot, double* grad,
                              double* hess, double thresh, cudaStream_t st);

}  // namespace b2
