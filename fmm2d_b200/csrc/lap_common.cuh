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
  const TreeCtl* ctl;     // the tree's device control block (level table)
  __device__ __forceinline__ bool has_eval_pts(int b) const {
    int n = 0;
    if (ifpghtarg > 0) n += trng[b].y - trng[b].x;
    if (ifpgh > 0) n += srng[b].y - srng[b].x;
    return n > 0;
  }
};

// Box range of a pass.  first >= 0: [first, first + n) as the host knows
// it.  The negative codes read the range from the tree's device control
// block instead (calls that do not wait for the tree on the host): all
// boxes, the boxes of levels >= 2, or the boxes of level `lev`.  After a
// failed build every range is empty.
constexpr int RANGE_ALL = -1, RANGE_FROM2 = -2, RANGE_LEVEL = -3;

__device__ __forceinline__ void resolve_range(const TV& t, int& first, int& n, int lev = 0) {
  if (first >= 0) return;
  const TreeCtl* c = t.ctl;
  const int code = first;
  first = 0;
  n = 0;
  if (c->status != TB_OK) return;
  const int nb = c->nboxes, nl = c->nlevels;
  if (code == RANGE_ALL) {
    n = nb;
  } else if (code == RANGE_FROM2) {
    if (nl >= 2) {
      first = c->lfirst[2];
      n = nb - first;
    }
  } else if (lev >= 0 && lev <= nl) {
    first = c->lfirst[lev];
    n = c->llast[lev] - first + 1;
  }
}

// The self-interaction threshold of the near field, boxsize(0) 2^-51
// (cfmm2d.f:1276), when the host passes a negative value.
__device__ __forceinline__ double near_thresh(const TV& t, double thresh) {
  return thresh >= 0 ? thresh : t.boxsize[0] * 0x1p-51;
}

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
