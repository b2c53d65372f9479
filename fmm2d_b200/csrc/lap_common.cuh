// Device-side views and helpers shared by the Laplace kernels
// (laplace.cu: FP64 path, lap_mixed.cu: mixed-precision path).
#pragma once
#include "common.cuh"
#include "tree.cuh"

namespace b2 {
namespace lapk {

// ---------------------------------------------------------------------------
// device helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ double2 cpow_int(double2 w, int e) {
  double2 r = make_double2(1.0, 0.0);
  double2 b = w;
  while (e > 0) {
    if (e & 1) r = cmul(r, b);
    e >>= 1;
    if (e) b = cmul(b, b);
  }
  return r;
}

__device__ __forceinline__ double2 cneg(double2 a) { return make_double2(-a.x, -a.y); }

// Asynchronous 16-byte copy global -> shared (both 16-byte aligned); the
// issuing thread's copies are complete after cp_async_wait_all().
__device__ __forceinline__ void cp_async16(void* sdst, const void* gsrc) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(sdst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

__device__ __forceinline__ int child_of(int4 ch, int c) {
  return c == 0 ? ch.x : (c == 1 ? ch.y : (c == 2 ? ch.z : ch.w));
}

// Box and list arrays of the device tree, passed by value to kernels.
struct TV {
  const double2* center;
  const int* level;
  const int* nchild;
  const int4* child;
  const int2* srng;
  const int2* trng;
  const int* nl1;
  const int* l1;
  const int* nl2;
  const int* l2;
  const int* nl3;
  const int* l3;
  const int* nl4;
  const int* l4;
  const double* boxsize;  // nlevels + 2 entries
  int ifpgh, ifpghtarg;
  __device__ __forceinline__ bool has_eval_pts(int b) const {
    int n = 0;
    if (ifpghtarg > 0) n += trng[b].y - trng[b].x;
    if (ifpgh > 0) n += srng[b].y - srng[b].x;
    return n > 0;
  }
};

struct Dens {
  const double2* q;  // sorted charges (ndc per point) or null
  const double2* d;  // sorted dipole strengths or null
  int ndc;           // Cauchy densities per point
  int d0;            // first density of the current chunk
};

#define WARP_LOOP(n)                                                                  \
  const int lane = threadIdx.x & 31;                                                  \
  const int wib = threadIdx.x >> 5;                                                   \
  const int nwarps = (gridDim.x * blockDim.x) >> 5;                                   \
  for (int bi = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; bi < (n); bi += nwarps)

}  // namespace lapk
}  // namespace b2
