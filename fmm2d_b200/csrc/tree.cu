// Device quadtree build.  The reference grows the tree level by level,
// stably partitioning the points of every refined box into its four children
// by comparing against the box centre (pts_tree2d.f:406-755).  Here every
// point instead computes, once, its full 51-level path through the virtual
// complete tree with exactly the same FP64 centre recurrence (centre of a
// child = centre of the parent +/- half the child size), packed into a
// 2-bit-per-level key; one radix sort then makes the points of every box of
// every level contiguous, and box point counts/ranges come from binary
// searches of the sorted keys.  Box creation, level restriction and the
// interaction lists follow the reference's own passes and box numbering so
// that the resulting tree is identical to the reference's, array for array.
// All passes from the root to the final point ranges run in one persistent
// (cooperative) kernel whose blocks step through the levels together behind
// bounded grid barriers; box creation order comes from grid-wide exclusive
// scans over the boxes in number order.  The host reads the level table back
// once, then builds the lists with one more kernel.
#include "tree.cuh"

#include <cmath>

#include <cub/cub.cuh>

#include <algorithm>
#include <cfloat>
#include <mutex>

namespace b2 {

namespace {

// ---------------------------------------------------------------------------
// pinned readback scratch
// ---------------------------------------------------------------------------
thread_local void* g_pinned = nullptr;
thread_local size_t g_pinned_bytes = 0;

std::atomic<long long> g_tree_bar_cycles{0};

void* pinned_bytes(size_t b) {
  if (b > g_pinned_bytes) {
    if (g_pinned) cudaFreeHost(g_pinned);
    g_pinned_bytes = std::max(b, (size_t)1 << 16);
    B2_CHECK(cudaMallocHost(&g_pinned, g_pinned_bytes));
  }
  return g_pinned;
}

// ---------------------------------------------------------------------------
// bounding box of sources and targets (pts_tree2d.f:475-500)
// ---------------------------------------------------------------------------
__device__ __forceinline__ void minmax4(double4& a, const double4 b) {
  a.x = fmin(a.x, b.x);
  a.y = fmax(a.y, b.y);
  a.z = fmin(a.z, b.z);
  a.w = fmax(a.w, b.w);
}

__device__ double4 block_minmax(double4 v) {
  __shared__ double4 sh[32];
  for (int o = 16; o; o >>= 1) {
    double4 w;
    w.x = __shfl_xor_sync(~0u, v.x, o);
    w.y = __shfl_xor_sync(~0u, v.y, o);
    w.z = __shfl_xor_sync(~0u, v.z, o);
    w.w = __shfl_xor_sync(~0u, v.w, o);
    minmax4(v, w);
  }
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) sh[wid] = v;
  __syncthreads();
  if (wid == 0) {
    int nw = blockDim.x >> 5;
    v = lane < nw ? sh[lane] : make_double4(DBL_MAX, -DBL_MAX, DBL_MAX, -DBL_MAX);
    for (int o = 16; o; o >>= 1) {
      double4 w;
      w.x = __shfl_xor_sync(~0u, v.x, o);
      w.y = __shfl_xor_sync(~0u, v.y, o);
      w.z = __shfl_xor_sync(~0u, v.z, o);
      w.w = __shfl_xor_sync(~0u, v.w, o);
      minmax4(v, w);
    }
  }
  return v;
}

__global__ void k_bbox(const double* __restrict__ src, long ns, const double* __restrict__ trg,
                       long nt, double4* part) {
  double4 v = make_double4(DBL_MAX, -DBL_MAX, DBL_MAX, -DBL_MAX);
  long stride = (long)gridDim.x * blockDim.x;
  // a coordinate that is not finite widens the box to infinity, which
  // k_init_root reports as TB_BADPTS
  const double4 bad = make_double4(-INFINITY, INFINITY, -INFINITY, INFINITY);
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < ns; i += stride) {
    double x = src[2 * i], y = src[2 * i + 1];
    minmax4(v, isfinite(x) && isfinite(y) ? make_double4(x, x, y, y) : bad);
  }
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < nt; i += stride) {
    double x = trg[2 * i], y = trg[2 * i + 1];
    minmax4(v, isfinite(x) && isfinite(y) ? make_double4(x, x, y, y) : bad);
  }
  v = block_minmax(v);
  if (threadIdx.x == 0) part[blockIdx.x] = v;
}

// Root box: side max(x-range, y-range), centred on the bounding box.
__global__ void k_bbox_final(const double4* part, int np, double* root) {
  double4 v = make_double4(DBL_MAX, -DBL_MAX, DBL_MAX, -DBL_MAX);
  for (int i = threadIdx.x; i < np; i += blockDim.x) minmax4(v, part[i]);
  v = block_minmax(v);
  if (threadIdx.x == 0) {
    double bs = v.y - v.x, sizey = v.w - v.z;
    if (sizey > bs) bs = sizey;
    root[0] = (v.x + v.y) / 2;
    root[1] = (v.z + v.w) / 2;
    root[2] = bs;
  }
}

// ---------------------------------------------------------------------------
// point keys: the path of a point through the virtual complete tree.
// At each level the point is compared with the centre of its current box
// (x - cx < 0, y - cy < 0; pts_tree2d.f:683,711,729) and the centre moves to
// the child's, cx +/- bs_child/2 (tree_routs2d.f:33-39).
// ---------------------------------------------------------------------------
__global__ void k_keys(const double* __restrict__ xy, long n, const double* __restrict__ root,
                       int nkey, uint64_t* khi, uint64_t* klo, int* idx) {
  long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  double x = xy[2 * i], y = xy[2 * i + 1];
  double cx = root[0], cy = root[1], bs = root[2];
  uint64_t hi = 0, lo = 0;
  for (int lev = 1; lev <= nkey; lev++) {
    bs = bs / 2;  // boxsize(lev) = boxsize(lev-1)/2
    double h = bs / 2;
    int sx = (x - cx < 0) ? 0 : 1;
    int sy = (y - cy < 0) ? 0 : 1;
    uint64_t dg = (uint64_t)(2 * sy + sx);
    cx = cx + (sx ? h : -h);
    cy = cy + (sy ? h : -h);
    if (lev <= 32)
      hi |= dg << (64 - 2 * lev);
    else
      lo |= dg << (64 - 2 * (lev - 32));
  }
  khi[i] = hi;
  klo[i] = lo;
  idx[i] = (int)i;
}

__global__ void k_gather_u64(const uint64_t* __restrict__ in, const int* __restrict__ idx, long n,
                             uint64_t* out) {
  long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i < n) out[i] = in[idx[i]];
}

// Sort points by key: by the first 32 levels, or (deep) lexicographically
// by all 51 levels with a stable least-significant-word-first pass.
void sort_by_key(const double* xy, long n, const double* root, bool deep, DBuf<uint64_t>& khi_out,
                 DBuf<uint64_t>& klo_out, DBuf<int>& idx_out, cudaStream_t st) {
  khi_out.alloc(n, st);
  klo_out.alloc(n, st);
  idx_out.alloc(n, st);
  if (n == 0) return;
  DBuf<uint64_t> khi(st), klo(st), tmpk(st);
  DBuf<int> idx(st), tmpi(st);
  khi.alloc(n, st);
  klo.alloc(n, st);
  idx.alloc(n, st);
  // a tree of at most 32 levels reads only the first key word; deeper trees
  // are rebuilt with deep = true
  k_keys<<<ceil_div(n, 256), 256, 0, st>>>(xy, n, root, deep ? NLMAX : 32, khi.p, klo.p, idx.p);
  B2_LAUNCH_CHECK();
  size_t tb = 0;
  DBuf<char> tmp(st);
  if (!deep) {
    B2_CHECK(cub::DeviceRadixSort::SortPairs(nullptr, tb, khi.p, khi_out.p, idx.p, idx_out.p,
                                             (int)n, 0, 64, st));
    tmp.alloc(tb, st);
    B2_CHECK(cub::DeviceRadixSort::SortPairs(tmp.p, tb, khi.p, khi_out.p, idx.p, idx_out.p,
                                             (int)n, 0, 64, st));
  } else {
    tmpk.alloc(n, st);
    tmpi.alloc(n, st);
    B2_CHECK(cub::DeviceRadixSort::SortPairs(nullptr, tb, klo.p, tmpk.p, idx.p, tmpi.p, (int)n, 0,
                                             64, st));
    tmp.alloc(tb, st);
    B2_CHECK(cub::DeviceRadixSort::SortPairs(tmp.p, tb, klo.p, tmpk.p, idx.p, tmpi.p, (int)n, 0,
                                             64, st));
    k_gather_u64<<<ceil_div(n, 256), 256, 0, st>>>(khi.p, tmpi.p, n, tmpk.p);
    B2_LAUNCH_CHECK();
    B2_CHECK(cub::DeviceRadixSort::SortPairs(tmp.p, tb, tmpk.p, khi_out.p, tmpi.p, idx_out.p,
                                             (int)n, 0, 64, st));
  }
  if (deep) {
    k_gather_u64<<<ceil_div(n, 256), 256, 0, st>>>(klo.p, idx_out.p, n, klo_out.p);
  } else {
    B2_CHECK(cudaMemsetAsync(klo_out.p, 0, sizeof(uint64_t) * n, st));
  }
  B2_LAUNCH_CHECK();
}

// ---------------------------------------------------------------------------
// box data
// ---------------------------------------------------------------------------
struct BoxPtrs {
  double2* center;
  int* level;
  int* parent;
  int* nchild;
  int4* child;
  int* iflag;
  uint64_t* pkey;  // path from the root, 2 bits per level (build scratch)
  int* ncoll;
  int* coll;
  int2* srng;
  int2* trng;
};

BoxPtrs ptrs(DeviceTree& T) {
  return BoxPtrs{T.center.p, T.level.p, T.parent.p, T.nchild.p, T.child.p, T.iflag.p,
                 nullptr,    T.ncoll.p, T.coll.p,   T.srng.p,   T.trng.p};
}

constexpr int TB_BIG = 16384;    // points of a refined box split by a warp

// Create the four children of parent b as boxes base..base+3 with the
// reference's child order (-,-), (+,-), (-,+), (+,+).
__device__ __forceinline__ void create_children(BoxPtrs& B, int b, int base, double bs_child,
                                                int lev_child, int child_flag) {
  double2 c = B.center[b];
  double h = bs_child / 2;
  const uint64_t pk = B.pkey[b];
  for (int j = 0; j < 4; j++) {
    int k = base + j;
    B.center[k] = make_double2(c.x + ((j & 1) ? h : -h), c.y + ((j < 2) ? -h : h));
    B.level[k] = lev_child;
    B.parent[k] = b;
    B.nchild[k] = 0;
    B.child[k] = make_int4(-1, -1, -1, -1);
    B.iflag[k] = child_flag;
    B.pkey[k] = pk * 4 + (uint64_t)j;
    B.srng[k] = make_int2(0, 0);
    B.trng[k] = make_int2(0, 0);
  }
  B.nchild[b] = 4;
  B.child[b] = make_int4(base, base + 1, base + 2, base + 3);
}

__global__ void k_init_root(BoxPtrs B, const double* root, int ns, int nt, TreeCtl* C, int cap,
                            long long bar_cycles) {
  B.center[0] = make_double2(root[0], root[1]);
  B.level[0] = 0;
  B.parent[0] = -1;
  B.nchild[0] = 0;
  B.child[0] = make_int4(-1, -1, -1, -1);
  B.iflag[0] = 0;
  B.pkey[0] = 0;
  B.srng[0] = make_int2(0, ns);
  B.trng[0] = make_int2(0, nt);
  B.ncoll[0] = 1;
  B.coll[0] = 0;
  for (int q = 1; q < 9; q++) B.coll[q] = -1;
  C->nboxes = 1;
  C->nlevels = 0;
  C->cap = cap;
  C->status = isfinite(root[2]) ? TB_OK : TB_BADPTS;
  C->bar_cycles = bar_cycles;
  C->lfirst[0] = 0;
  C->llast[0] = 0;
  C->bs[0] = root[2];
  for (int q = 0; q < TB_GROUPS * 32; q++) C->bar_sub[q] = 0;
  C->bar_top = 0;
  C->bar_gen = 0;
}

// ---------------------------------------------------------------------------
// per-box steps of the build (pts_tree2d.f, tree_routs2d.f)
// ---------------------------------------------------------------------------
// Leaf capacity at level lev: ndiv (pts_tree2d.f), or, with a level balance
// lbal != 0, ndiv 2^(lbal (lpiv - lev)) rounded (at least 1), lpiv the level
// whose boxes would hold ndiv points of a uniform cloud: lbal > 0 lets
// leaves above that level hold more points and splits boxes below it
// sooner (more M2L, less P2P deep down), lbal < 0 the reverse.
__device__ __forceinline__ int level_ndiv(int ndiv, float lbal, float lpiv, int lev) {
  if (lbal == 0.f) return ndiv;
  const float v = (float)ndiv * exp2f(lbal * (lpiv - (float)lev));
  return v >= 2e9f ? 2000000000 : max(1, (int)(v + 0.5f));
}

// refine if the relevant count exceeds ndiv (pts_tree2d.f:538-560)
__device__ __forceinline__ int refine_flag(const BoxPtrs& B, int b, int idivflag, int ndiv) {
  int nss = B.srng[b].y - B.srng[b].x, ntt = B.trng[b].y - B.trng[b].x;
  int nn = idivflag == 0 ? nss : (idivflag == 1 ? ntt : max(nss, ntt));
  return nn > ndiv ? 1 : 0;
}

// Colleagues from the parent's colleagues' children (tree_routs2d.f:160-206).
__device__ void colleagues(BoxPtrs& B, int b, double tol) {
  int* cl = B.coll + 9 * (size_t)b;
  int cnt = 0;
  if (B.level[b] == 0) {
    cl[0] = b;
    cnt = 1;
  } else {
    int dad = B.parent[b];
    double2 cb = B.center[b];
    int nd = B.ncoll[dad];
    for (int q = 0; q < nd; q++) {
      int j = B.coll[9 * (size_t)dad + q];
      int4 ch = B.child[j];
      int cc[4] = {ch.x, ch.y, ch.z, ch.w};
      for (int t = 0; t < 4; t++) {
        int k = cc[t];
        if (k < 0) continue;
        double2 ck = B.center[k];
        if (fabs(ck.x - cb.x) <= tol && fabs(ck.y - cb.y) <= tol) {
          if (cnt < 9) cl[cnt] = k;
          cnt++;
        }
      }
    }
  }
  for (int q = cnt; q < 9; q++) cl[q] = -1;
  B.ncoll[b] = min(cnt, 9);
}

// Level restriction, pass 1 ("flag"): a leaf colleague of a box's
// grandparent that touches the box's parent (pts_tree2d.f:805-842).
__device__ void flag_pass(BoxPtrs& B, int b, double dt) {
  int dad = B.parent[b], gd = B.parent[dad];
  double2 cd = B.center[dad];
  int ng = B.ncoll[gd];
  for (int q = 0; q < ng; q++) {
    int j = B.coll[9 * (size_t)gd + q];
    if (B.nchild[j] != 0 || B.iflag[j] != 0) continue;
    double2 cj = B.center[j];
    if (fabs(cj.x - cd.x) <= dt && fabs(cj.y - cd.y) <= dt) B.iflag[j] = 1;
  }
}

// Pass 2 ("flag+"): a leaf colleague of the parent of a flagged or flag+
// box that touches that box (pts_tree2d.f:852-890).
__device__ void flagplus(BoxPtrs& B, int b, double dt) {
  int f = B.iflag[b];
  if (f != 1 && f != 2) return;
  int dad = B.parent[b];
  double2 cb = B.center[b];
  int nd = B.ncoll[dad];
  for (int q = 0; q < nd; q++) {
    int j = B.coll[9 * (size_t)dad + q];
    if (B.nchild[j] != 0 || B.iflag[j] != 0) continue;
    double2 cj = B.center[j];
    if (fabs(cj.x - cb.x) <= dt && fabs(cj.y - cb.y) <= dt) B.iflag[j] = 2;
  }
}

// A flag++ box is refined if a child (with children) of one of its
// colleagues touches it (tree_routs2d.f:217-326).
__device__ int update_flag(BoxPtrs& B, int b, double dt) {
  int f = B.iflag[b];
  if (f == 3) {
    f = 0;
    double2 cb = B.center[b];
    int nc = B.ncoll[b];
    for (int q = 0; q < nc && !f; q++) {
      int j = B.coll[9 * (size_t)b + q];
      int4 ch = B.child[j];
      int cc[4] = {ch.x, ch.y, ch.z, ch.w};
      for (int t = 0; t < 4; t++) {
        int k = cc[t];
        if (k < 0 || B.nchild[k] <= 0) continue;
        double2 ck = B.center[k];
        if (fabs(ck.x - cb.x) <= dt && fabs(ck.y - cb.y) <= dt) {
          f = 1;
          break;
        }
      }
    }
    B.iflag[b] = f;
  }
  return f == 1 ? 1 : 0;
}

// Point ranges of the four children of refined box b: the three digit
// boundaries in the source range and the three in the target range are six
// independent binary searches, stepped together so that their loads overlap.
__device__ void split_children(BoxPtrs& B, int b, int lev_child, const uint64_t* skhi,
                               const uint64_t* sklo, const uint64_t* tkhi, const uint64_t* tklo) {
  const int2 rs = B.srng[b], rt = B.trng[b];
  int lo[6], hi[6];
#pragma unroll
  for (int q = 0; q < 6; q++) {
    lo[q] = q < 3 ? rs.x : rt.x;
    hi[q] = q < 3 ? rs.y : rt.y;
  }
  for (;;) {
    bool any = false;
#pragma unroll
    for (int q = 0; q < 6; q++) {
      if (lo[q] < hi[q]) {
        any = true;
        const int m = (lo[q] + hi[q]) >> 1;
        const int dg = q < 3 ? key_digit(skhi[m], sklo[m], lev_child)
                             : key_digit(tkhi[m], tklo[m], lev_child);
        if (dg < (q % 3) + 1)
          lo[q] = m + 1;
        else
          hi[q] = m;
      }
    }
    if (!any) break;
  }
  const int4 ch = B.child[b];
  const int cc[4] = {ch.x, ch.y, ch.z, ch.w};
  const int bs_[5] = {rs.x, lo[0], lo[1], lo[2], rs.y};
  const int bt_[5] = {rt.x, lo[3], lo[4], lo[5], rt.y};
#pragma unroll
  for (int j = 0; j < 4; j++) {
    B.srng[cc[j]] = make_int2(bs_[j], bs_[j + 1]);
    B.trng[cc[j]] = make_int2(bt_[j], bt_[j + 1]);
  }
}

// split_children by one warp, for refined boxes with many points: lanes
// 0..29 run the six searches as 6-way searches (5 probes per search and
// round, combined by a ballot), log_6 instead of log_2 rounds of dependent
// loads.  Each search ends at the same boundary as the binary search.
__device__ void split_children_warp(BoxPtrs& B, int b, int lev_child, const uint64_t* skhi,
                                    const uint64_t* sklo, const uint64_t* tkhi,
                                    const uint64_t* tklo) {
  const int lane = threadIdx.x & 31, q = lane / 5, k = lane % 5;
  const int2 rs = B.srng[b], rt = B.trng[b];
  int lo = 0, hi = 0;
  if (q < 6) {
    lo = q < 3 ? rs.x : rt.x;
    hi = q < 3 ? rs.y : rt.y;
  }
  const int t = (q % 3) + 1;
  for (;;) {
    const int n = hi - lo;
    const bool active = n > 0;
    if (!__any_sync(~0u, active)) break;
    bool pred = false;
    if (active) {
      const int p = lo + (int)(((long long)n * (k + 1)) / 6);  // in [lo, hi)
      const int dg = q < 3 ? key_digit(skhi[p], sklo[p], lev_child)
                           : key_digit(tkhi[p], tklo[p], lev_child);
      pred = dg >= t;
    }
    const unsigned m = __ballot_sync(~0u, pred);
    if (active) {
      const unsigned gm = (m >> (q * 5)) & 0x1Fu;
      const int ks = gm ? __ffs(gm) - 1 : 5;  // first probe at or past the boundary
      const int nhi = ks < 5 ? lo + (int)(((long long)n * (ks + 1)) / 6) : hi;
      const int nlo = ks > 0 ? lo + (int)(((long long)n * ks) / 6) + 1 : lo;
      lo = nlo;
      hi = nhi;
    }
  }
  int bd[6];
#pragma unroll
  for (int j = 0; j < 6; j++) bd[j] = __shfl_sync(~0u, lo, j * 5);
  if (lane == 0) {
    const int4 ch = B.child[b];
    const int cc[4] = {ch.x, ch.y, ch.z, ch.w};
    const int bs_[5] = {rs.x, bd[0], bd[1], bd[2], rs.y};
    const int bt_[5] = {rt.x, bd[3], bd[4], bd[5], rt.y};
#pragma unroll
    for (int j = 0; j < 4; j++) {
      B.srng[cc[j]] = make_int2(bs_[j], bs_[j + 1]);
      B.trng[cc[j]] = make_int2(bt_[j], bt_[j + 1]);
    }
  }
}

// Ranges of the sorted source and target keys (first 32 levels) whose top
// 2*lev bits equal the box path pk: the points of the box.  The four binary
// searches (first key with prefix >= pk, first with prefix > pk, in both
// arrays) are stepped together.
__device__ void prefix_ranges(const uint64_t* __restrict__ skhi, int ns,
                              const uint64_t* __restrict__ tkhi, int nt, uint64_t pk, int lev,
                              int2& rs, int2& rt) {
  const int sh = 64 - 2 * lev;
  int lo[4] = {0, 0, 0, 0}, hi[4] = {ns, ns, nt, nt};
  for (;;) {
    bool any = false;
#pragma unroll
    for (int q = 0; q < 4; q++) {
      if (lo[q] < hi[q]) {
        any = true;
        const int m = (lo[q] + hi[q]) >> 1;
        const uint64_t v = (q < 2 ? skhi[m] : tkhi[m]) >> sh;
        if ((q & 1) ? v <= pk : v < pk)
          lo[q] = m + 1;
        else
          hi[q] = m;
      }
    }
    if (!any) break;
  }
  rs = make_int2(lo[0], lo[1]);
  rt = make_int2(lo[2], lo[3]);
}

// ---------------------------------------------------------------------------
// grid-wide primitives of the persistent build kernel (cooperative launch:
// all blocks are resident).  Every wait is bounded; a barrier that gives up
// sets TB_TIMEOUT, which releases the other blocks too.
// ---------------------------------------------------------------------------
__device__ __forceinline__ int ctl_status(const TreeCtl* C) {
  return *reinterpret_cast<const volatile int*>(&C->status);
}

__device__ __forceinline__ bool gbar(TreeCtl* C) { return grid_barrier(C, TB_TIMEOUT); }

// Item i of one box range [f1, f1+n1) or of two concatenated ranges.
struct Items {
  int f1, n1, f2, n;
  __device__ __forceinline__ int box(int i) const { return i < n1 ? f1 + i : f2 + (i - n1); }
};

// The block's contiguous chunk of n items (item order = box order).
struct Chunk {
  int c0, c1;
};
__device__ __forceinline__ Chunk chunk_of(int n) {
  const int G = gridDim.x, ch = (n + G - 1) / G;
  const int c0 = min(n, (int)blockIdx.x * ch);
  return Chunk{c0, min(n, c0 + ch)};
}

// Block-level exclusive scan of one 0/1 flag per thread; returns the
// thread's exclusive rank and sets *sum to the block total.
__device__ __forceinline__ int block_excl_scan(int f, int* wsum, int* sum) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const unsigned bal = __ballot_sync(~0u, f);
  const int in_warp = __popc(bal & ((1u << lane) - 1u));
  __syncthreads();
  if (lane == 0) wsum[w] = __popc(bal);
  __syncthreads();
  int pre = 0, tot = 0;
  for (int q = 0; q < nw; q++) {
    const int v = wsum[q];
    if (q < w) pre += v;
    tot += v;
  }
  *sum = tot;
  return pre + in_warp;
}

// After the barrier that follows the block counts in tot[buf]: the number
// of flagged items in the chunks before this block's, and in all chunks.
__device__ void block_prefix(const TreeCtl* C, int buf, int* red, int& pre, int& total) {
  if (threadIdx.x == 0) red[0] = red[1] = 0;
  __syncthreads();
  int p = 0, a = 0;
  for (int q = threadIdx.x; q < (int)gridDim.x; q += blockDim.x) {
    const int v = C->tot[buf][q];
    if (q < (int)blockIdx.x) p += v;
    a += v;
  }
  atomicAdd(&red[0], p);
  atomicAdd(&red[1], a);
  __syncthreads();
  pre = red[0];
  total = red[1];
  __syncthreads();
}

struct TreeKeys {
  const uint64_t *skhi, *sklo, *tkhi, *tklo;
};

// Renumber the boxes: per level, the level's current range, then its tail
// [tf, tl] (pts_tree2d.f:1066-1215).  The permuted arrays are written into
// the alternate buffers `alt`, which then become current.
__device__ bool reorganize(TreeCtl* C, BoxPtrs& cur, BoxPtrs& alt, int* map, int nl, int nb,
                           int* newf) {
  const int gt = blockIdx.x * blockDim.x + threadIdx.x, gs = gridDim.x * blockDim.x;
  if (threadIdx.x == 0) {
    int c = 0;
    for (int l = 0; l <= nl; l++) {
      newf[l] = c;
      c += (C->llast[l] - C->lfirst[l] + 1) + max(C->tl[l] - C->tf[l] + 1, 0);
    }
  }
  __syncthreads();
  for (int b = gt; b < nb; b += gs) {
    const int l = cur.level[b];
    const int lf = C->lfirst[l], ll = C->llast[l];
    map[b] = (b >= lf && b <= ll) ? newf[l] + (b - lf) : newf[l] + (ll - lf + 1) + (b - C->tf[l]);
  }
  if (!gbar(C)) return false;
  for (int b = gt; b < nb; b += gs) {
    const int m = map[b];
    alt.center[m] = cur.center[b];
    alt.level[m] = cur.level[b];
    alt.nchild[m] = cur.nchild[b];
    alt.iflag[m] = cur.iflag[b];
    alt.pkey[m] = cur.pkey[b];
    const int p = cur.parent[b];
    alt.parent[m] = p < 0 ? -1 : map[p];
    const int4 c = cur.child[b];
    alt.child[m] = make_int4(c.x < 0 ? -1 : map[c.x], c.y < 0 ? -1 : map[c.y],
                             c.z < 0 ? -1 : map[c.z], c.w < 0 ? -1 : map[c.w]);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    for (int l = 0; l <= nl; l++) {
      const int no = C->llast[l] - C->lfirst[l] + 1, nt = max(C->tl[l] - C->tf[l] + 1, 0);
      C->lfirst[l] = newf[l];
      C->llast[l] = newf[l] + no + nt - 1;
    }
  }
  if (!gbar(C)) return false;
  // the permuted arrays become current (the others are recomputed later)
  BoxPtrs t = cur;
  cur.center = alt.center;
  cur.level = alt.level;
  cur.parent = alt.parent;
  cur.nchild = alt.nchild;
  cur.child = alt.child;
  cur.iflag = alt.iflag;
  cur.pkey = alt.pkey;
  alt.center = t.center;
  alt.level = t.level;
  alt.parent = t.parent;
  alt.nchild = t.nchild;
  alt.child = t.child;
  alt.iflag = t.iflag;
  alt.pkey = t.pkey;
  return true;
}

// Colleagues through a hash table of (level, path key) -> box.  The
// colleagues of a box are the existing boxes of its level in its 3x3
// neighbourhood; the reference collects them from the children of the
// parent's colleagues (tree_routs2d.f:160-206), parent colleagues in their
// own order and children in child order, which is the order of the path
// keys (Morton order), so the neighbours are sorted by key.  Paths of at
// most 31 levels fit the 64-bit table key (a sentinel bit above the path).
struct BoxHash {
  unsigned long long* key;  // 0 = empty
  int* box;
  unsigned mask;            // capacity - 1 (power of two)
};

__device__ __forceinline__ unsigned long long hash_key(int lev, uint64_t pk) {
  return (1ull << (2 * lev)) | pk;
}
__device__ __forceinline__ unsigned hash_slot(unsigned long long k, unsigned mask) {
  return (unsigned)((k * 0x9E3779B97F4A7C15ull) >> 32) & mask;
}
__device__ __forceinline__ uint64_t spread_bits(uint32_t x) {
  uint64_t v = x;
  v = (v | (v << 16)) & 0x0000FFFF0000FFFFull;
  v = (v | (v << 8)) & 0x00FF00FF00FF00FFull;
  v = (v | (v << 4)) & 0x0F0F0F0F0F0F0F0Full;
  v = (v | (v << 2)) & 0x3333333333333333ull;
  v = (v | (v << 1)) & 0x5555555555555555ull;
  return v;
}
__device__ __forceinline__ uint32_t compact_bits(uint64_t v) {
  v &= 0x5555555555555555ull;
  v = (v | (v >> 1)) & 0x3333333333333333ull;
  v = (v | (v >> 2)) & 0x0F0F0F0F0F0F0F0Full;
  v = (v | (v >> 4)) & 0x00FF00FF00FF00FFull;
  v = (v | (v >> 8)) & 0x0000FFFF0000FFFFull;
  v = (v | (v >> 16)) & 0x00000000FFFFFFFFull;
  return (uint32_t)v;
}

__device__ void hash_insert(const BoxHash& H, unsigned long long k, int b) {
  unsigned h = hash_slot(k, H.mask);
  for (unsigned it = 0; it <= H.mask; it++) {
    const unsigned long long prev = atomicCAS(&H.key[h], 0ull, k);
    if (prev == 0ull || prev == k) {
      H.box[h] = b;
      return;
    }
    h = (h + 1) & H.mask;
  }
}

__device__ int hash_find(const BoxHash& H, unsigned long long k) {
  unsigned h = hash_slot(k, H.mask);
  for (unsigned it = 0; it <= H.mask; it++) {
    const unsigned long long v = H.key[h];
    if (v == k) return H.box[h];
    if (v == 0ull) return -1;
    h = (h + 1) & H.mask;
  }
  return -1;
}

// Colleagues of every box of the current tree (levels <= 31): clear the
// table, insert every box, look up the 3x3 neighbourhoods; three phases.
// `extra` runs over all boxes in the first phase.
template <class F>
__device__ bool colleagues_hashed(TreeCtl* C, BoxPtrs& B, const BoxHash& H, int nb, F extra) {
  const int gt = blockIdx.x * blockDim.x + threadIdx.x, gs = gridDim.x * blockDim.x;
  for (unsigned h = gt; h <= H.mask; h += gs) H.key[h] = 0ull;
  for (int b = gt; b < nb; b += gs) extra(b);
  if (!gbar(C)) return false;
  for (int b = gt; b < nb; b += gs) hash_insert(H, hash_key(B.level[b], B.pkey[b]), b);
  if (!gbar(C)) return false;
  for (int b = gt; b < nb; b += gs) {
    int* cl = B.coll + 9 * (size_t)b;
    const int l = B.level[b];
    if (l == 0) {
      cl[0] = b;
      for (int q = 1; q < 9; q++) cl[q] = -1;
      B.ncoll[b] = 1;
      continue;
    }
    const uint64_t pk = B.pkey[b];
    const long ix = compact_bits(pk), iy = compact_bits(pk >> 1), side = 1L << l;
    // the 3x3 neighbourhood (q = 3 (dy + 1) + dx + 1): the eight lookups are
    // independent, so their probes advance together, one round of loads at a
    // time (st: 0 probing, 1 found at slot hs, 2 absent; q = 4 is b itself)
    uint64_t nk[9], hk[9];
    unsigned hs[9];
    int st[9];
#pragma unroll
    for (int q = 0; q < 9; q++) {
      const long x = ix + q % 3 - 1, y = iy + q / 3 - 1;
      const bool in = !(x < 0 || y < 0 || x >= side || y >= side);
      nk[q] = in ? ((spread_bits((uint32_t)y) << 1) | spread_bits((uint32_t)x)) : 0;
      hk[q] = hash_key(l, nk[q]);
      hs[q] = hash_slot(hk[q], H.mask);
      st[q] = !in ? 2 : (q == 4 ? 1 : 0);
    }
    for (unsigned it = 0; it <= H.mask; it++) {
      unsigned long long v[9];
#pragma unroll
      for (int q = 0; q < 9; q++) v[q] = st[q] == 0 ? H.key[hs[q]] : 0ull;
      bool more = false;
#pragma unroll
      for (int q = 0; q < 9; q++) {
        if (st[q] != 0) continue;
        if (v[q] == hk[q]) {
          st[q] = 1;
        } else if (v[q] == 0ull) {
          st[q] = 2;
        } else {
          hs[q] = (hs[q] + 1) & H.mask;
          more = true;
        }
      }
      if (!more) break;
    }
    int fbx[9];
#pragma unroll
    for (int q = 0; q < 9; q++) fbx[q] = q == 4 ? b : (st[q] == 1 ? H.box[hs[q]] : -1);
    // the found neighbours in key order
    uint64_t fk[9];
    int fb[9], cnt = 0;
#pragma unroll
    for (int q = 0; q < 9; q++) {
      if (st[q] != 1) continue;
      int r = cnt++;
      while (r > 0 && fk[r - 1] > nk[q]) {
        fk[r] = fk[r - 1];
        fb[r] = fb[r - 1];
        r--;
      }
      fk[r] = nk[q];
      fb[r] = fbx[q];
    }
    for (int q = 0; q < 9; q++) cl[q] = q < cnt ? fb[q] : -1;
    B.ncoll[b] = cnt;
  }
  return gbar(C);
}

// Colleagues of all levels, top down; the first level's pass also runs
// `extra` over all boxes (work that only has to precede the next phase).
template <class F>
__device__ bool colleagues_all(TreeCtl* C, BoxPtrs& B, int nl, int nb, F extra) {
  const int gt = blockIdx.x * blockDim.x + threadIdx.x, gs = gridDim.x * blockDim.x;
  for (int b = gt; b < nb; b += gs) extra(b);
  for (int l = 0; l <= nl; l++) {
    const double tol = (double)1.05f * C->bs[l];
    for (int b = C->lfirst[l] + gt; b <= C->llast[l]; b += gs) colleagues(B, b, tol);
    if (!gbar(C)) return false;
  }
  return true;
}

// The whole level-restricted tree on the device: adaptive refinement level by
// level (pts_tree2d.f:538-755), level restriction (pts_tree2d.f:760-1060,
// tree_routs2d.f:217-388), renumbering and the point ranges of every box, with
// the reference's box numbering.  A refinement step is two phases: every
// block flags the boxes of its contiguous chunk of the level, then after one
// barrier every block knows the
// flagged counts of all chunks and creates the children of its own chunk in
// box order.  Scratch: flag (cap ints; also the renumbering map) and the
// alternate box arrays S.  Outcome in C->status (TB_OVERFLOW: more than
// C->cap boxes; TB_DEEP: levels beyond 32 need the 51-level keys).
__global__ void __launch_bounds__(TB_THREADS, 1)
    k_tree_build(BoxPtrs B, BoxPtrs S, TreeCtl* C, int* flag, TreeKeys K, BoxHash H, int ns,
                 int nt, int idivflag, int ndiv, int nlmax, int deep, float lbal, float lpiv) {
  __shared__ int wsum[32];
  __shared__ int red[2];
  __shared__ int newf[NLMAX + 2];
  __shared__ int bigl[TB_THREADS];  // refined boxes of the chunk split by warps
  __shared__ int nbig;
  const int gt = blockIdx.x * blockDim.x + threadIdx.x, gs = gridDim.x * blockDim.x;
  const int cap = C->cap;
  BoxPtrs cur = B, alt = S;
  int buf = 0;  // tot[] buffer of the next scan
  if (C->status != TB_OK) return;  // non-finite coordinates (every block sees it)
  // A zero-size root (all points coincide) cannot be subdivided: the
  // children would coincide with it forever.  Keep the root as the only box.
  if (C->bs[0] == 0.0) nlmax = 0;
  // --- adaptive refinement ---------------------------------------------
  int f = 0, n = 1, nb = 1, lev = 0;
  for (;; lev++) {
    // phase A: refine flags and counts of own chunk
    const bool more = lev < nlmax;
    const Chunk ch = chunk_of(n);
    const int ndl = level_ndiv(ndiv, lbal, lpiv, lev);
    int cnt = 0;
    if (more)
      for (int i0 = ch.c0; i0 < ch.c1; i0 += blockDim.x) {
        const int i = i0 + threadIdx.x;
        const int fl = i < ch.c1 ? refine_flag(cur, f + i, idivflag, ndl) : 0;
        if (i < ch.c1) flag[i] = fl;
        cnt += __syncthreads_count(fl);
      }
    if (threadIdx.x == 0) C->tot[buf][blockIdx.x] = cnt;
    if (!gbar(C)) return;
    if (!more) break;
    // phase B: children of the flagged boxes of own chunk, in box order
    int pre, tot;
    block_prefix(C, buf, red, pre, tot);
    buf ^= 1;
    if (tot == 0) break;
    if (lev + 1 > 32 && !deep) {
      if (gt == 0) C->status = TB_DEEP;
      return;
    }
    if (nb + 4 * tot > cap) {
      if (gt == 0) C->status = TB_OVERFLOW;
      return;
    }
    const double bsc = C->bs[lev] / 2;
    // boxes with many points are split by a warp each after the loop (their
    // binary searches would be long chains of dependent loads)
    if (threadIdx.x == 0) nbig = 0;
    __syncthreads();
    int run = pre;
    for (int i0 = ch.c0; i0 < ch.c1; i0 += blockDim.x) {
      const int i = i0 + threadIdx.x;
      const int fl = i < ch.c1 ? flag[i] : 0;
      int s;
      const int r = block_excl_scan(fl, wsum, &s);
      if (fl) {
        const int b = f + i;
        create_children(cur, b, nb + 4 * (run + r), bsc, lev + 1, 0);
        const int2 rs = cur.srng[b], rt = cur.trng[b];
        int slot = -1;
        if (rs.y - rs.x + rt.y - rt.x > TB_BIG) {
          slot = atomicAdd(&nbig, 1);
          if (slot < TB_THREADS) bigl[slot] = b;
        }
        if (slot < 0 || slot >= TB_THREADS)
          split_children(cur, b, lev + 1, K.skhi, K.sklo, K.tkhi, K.tklo);
      }
      run += s;
    }
    __syncthreads();
    {
      const int nw = min(nbig, TB_THREADS);
      for (int w = threadIdx.x >> 5; w < nw; w += TB_THREADS / 32)
        split_children_warp(cur, bigl[w], lev + 1, K.skhi, K.sklo, K.tkhi, K.tklo);
    }
    if (gt == 0) {
      C->bs[lev + 1] = bsc;
      C->lfirst[lev + 1] = nb;
      C->llast[lev + 1] = nb + 4 * tot - 1;
      C->nboxes = nb + 4 * tot;
    }
    f = nb;
    n = 4 * tot;
    nb += 4 * tot;
    if (!gbar(C)) return;
  }
  const int nl = lev;
  if (gt == 0) {
    C->nlevels = nl;
    C->bs[nl + 1] = C->bs[nl] / 2;
  }
  // colleagues of the refined tree (the level restriction and the lists use them)
  const bool hashed = nl <= 31;
  if (!(hashed ? colleagues_hashed(C, cur, H, nb, [](int) {})
               : colleagues_all(C, cur, nl, nb, [](int) {})))
    return;
  if (nl >= 2) {
    // --- level restriction ---------------------------------------------
    // pass 1: flag (levels >= 2, one pass); zero the per-level counts and tails
    if (gt == 0)
      for (int l = 0; l <= nl; l++) {
        C->lcnt[l] = 0;
        C->tf[l] = 0;
        C->tl[l] = -1;
      }
    for (int b = C->lfirst[2] + gt; b < nb; b += gs) {
      const int l = cur.level[b];
      flag_pass(cur, b, 1.05 * (C->bs[l - 1] + C->bs[l - 2]) / 2.0);
    }
    if (!gbar(C)) return;
    // pass 2: flag+, finest level first
    for (int l = nl; l >= 1; l--) {
      const double dt = 1.05 * (C->bs[l] + C->bs[l - 1]) / 2.0;
      for (int b = C->lfirst[l] + gt; b <= C->llast[l]; b += gs) flagplus(cur, b, dt);
      if (!gbar(C)) return;
    }
    // subdivide the flag and flag+ boxes of levels 1..nl-2
    if (nl - 2 >= 1) {
      const int f1 = C->lfirst[1], n1 = C->llast[nl - 2] - f1 + 1;
      const Chunk ch = chunk_of(n1);
      int cnt = 0;
      for (int i0 = ch.c0; i0 < ch.c1; i0 += blockDim.x) {
        const int i = i0 + threadIdx.x;
        const int fl = i < ch.c1 ? (cur.iflag[f1 + i] > 0 ? 1 : 0) : 0;
        if (i < ch.c1) flag[i] = fl;
        if (fl) atomicAdd(&C->lcnt[cur.level[f1 + i]], 1);
        cnt += __syncthreads_count(fl);
      }
      if (threadIdx.x == 0) C->tot[buf][blockIdx.x] = cnt;
      if (!gbar(C)) return;
      int pre, tot;
      block_prefix(C, buf, red, pre, tot);
      buf ^= 1;
      if (tot > 0) {
        if (nb + 4 * tot > cap) {
          if (gt == 0) C->status = TB_OVERFLOW;
          return;
        }
        int run = pre;
        for (int i0 = ch.c0; i0 < ch.c1; i0 += blockDim.x) {
          const int i = i0 + threadIdx.x;
          const int fl = i < ch.c1 ? flag[i] : 0;
          int s;
          const int r = block_excl_scan(fl, wsum, &s);
          if (fl) {
            const int b = f1 + i, lc = cur.level[b] + 1;
            create_children(cur, b, nb + 4 * (run + r), C->bs[lc], lc, cur.iflag[b] == 1 ? 3 : 0);
          }
          run += s;
        }
        if (gt == 0) {
          int base = nb;
          for (int l = 1; l <= nl - 2; l++) {
            const int c = C->lcnt[l];
            C->tf[l + 1] = base;
            C->tl[l + 1] = base + 4 * c - 1;
            base += 4 * c;
          }
          C->nboxes = nb + 4 * tot;
        }
        nb += 4 * tot;
        if (!gbar(C)) return;
      }
    }
    if (!reorganize(C, cur, alt, flag, nl, nb, newf)) return;
    // colleagues of the renumbered tree; flag++ boxes keep their flag (3),
    // all others are cleared; the tails are cleared for pass 3
    auto keep3 = [&](int b) {
      if (cur.iflag[b] != 3) cur.iflag[b] = 0;
      if (b <= nl) {
        C->tf[b] = 0;
        C->tl[b] = -1;
      }
    };
    if (!(hashed ? colleagues_hashed(C, cur, H, nb, keep3) : colleagues_all(C, cur, nl, nb, keep3)))
      return;
    // pass 3: flag++ boxes, coarsest level first, refining as needed; the
    // colleagues of a level's new boxes (its tail) are computed in the same
    // phase as the level's flags, by the thread that then flags the box
    for (int l = 2; l <= nl - 2; l++) {
      const int lf = C->lfirst[l], n1 = C->llast[l] - lf + 1, tf = C->tf[l];
      const Items it{lf, n1, tf, n1 + max(C->tl[l] - tf + 1, 0)};
      const double dt = 1.05 * (C->bs[l] + C->bs[l + 1]) / 2.0;
      const double ctol = (double)1.05f * C->bs[l];
      const Chunk ch = chunk_of(it.n);
      int cnt = 0;
      for (int i0 = ch.c0; i0 < ch.c1; i0 += blockDim.x) {
        const int i = i0 + threadIdx.x;
        int fl = 0;
        if (i < ch.c1) {
          const int b = it.box(i);
          if (i >= n1) colleagues(cur, b, ctol);
          fl = update_flag(cur, b, dt);
          flag[i] = fl;
        }
        cnt += __syncthreads_count(fl);
      }
      if (threadIdx.x == 0) C->tot[buf][blockIdx.x] = cnt;
      if (!gbar(C)) return;
      int pre, tot;
      block_prefix(C, buf, red, pre, tot);
      buf ^= 1;
      if (tot == 0) continue;
      if (nb + 4 * tot > cap) {
        if (gt == 0) C->status = TB_OVERFLOW;
        return;
      }
      int run = pre;
      for (int i0 = ch.c0; i0 < ch.c1; i0 += blockDim.x) {
        const int i = i0 + threadIdx.x;
        const int fl = i < ch.c1 ? flag[i] : 0;
        int s;
        const int r = block_excl_scan(fl, wsum, &s);
        if (fl) {
          const int b = it.box(i), lc = cur.level[b] + 1;
          create_children(cur, b, nb + 4 * (run + r), C->bs[lc], lc, cur.iflag[b] == 1 ? 3 : 0);
        }
        run += s;
      }
      if (gt == 0) {
        C->tf[l + 1] = nb;
        C->tl[l + 1] = nb + 4 * tot - 1;
        C->nboxes = nb + 4 * tot;
      }
      nb += 4 * tot;
      if (!gbar(C)) return;
    }
    if (!reorganize(C, cur, alt, flag, nl, nb, newf)) return;
    if (!(hashed ? colleagues_hashed(C, cur, H, nb, [](int) {})
                 : colleagues_all(C, cur, nl, nb, [](int) {})))
      return;
  }
  // --- point ranges of every box of the final tree ----------------------
  if (nl <= 32) {
    // a box's points are the keys with its path as prefix (one pass)
    for (int b = gt + 1; b < nb; b += gs) {
      const int l = cur.level[b];
      int2 rs, rt;
      prefix_ranges(K.skhi, ns, K.tkhi, nt, cur.pkey[b], l, rs, rt);
      cur.srng[b] = rs;
      cur.trng[b] = rt;
    }
  } else {
    for (int l = 0; l < nl; l++) {
      for (int b = C->lfirst[l] + gt; b <= C->llast[l]; b += gs)
        if (cur.nchild[b] != 0) split_children(cur, b, l + 1, K.skhi, K.sklo, K.tkhi, K.tklo);
      if (!gbar(C)) return;
    }
  }
}

// Lists 1-4 of every box (tree_routs2d.f:486-710), as a gather: a box's
// list 1 starts with the coarser adjacent leaves (which the reference
// appends while visiting the coarser level, in increasing box number), then
// its own entries; its list 4 holds the coarser non-adjacent leaves.
__global__ void k_lists(BoxPtrs B, const TreeCtl* C, int* nl1, int* l1, int* nl2, int* l2,
                        int* nl3, int* l3, int* nl4, int* l4) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (C->status != TB_OK || b >= C->nboxes) return;
  const double* boxsize = C->bs;
  int n1 = 0, n2 = 0, n3 = 0, n4 = 0;
  int* L1 = l1 + (size_t)MNLIST1 * b;
  int* L2 = l2 + (size_t)MNLIST2 * b;
  int* L3 = l3 + (size_t)MNLIST3 * b;
  int* L4 = l4 + (size_t)MNLIST4 * b;
  int lev = B.level[b];
  double2 cb = B.center[b];
  bool leaf = B.nchild[b] == 0;
  if (lev == 0) {
    if (leaf) L1[n1++] = b;
  } else {
    int dad = B.parent[b];
    const int* cd = B.coll + 9 * (size_t)dad;
    int ncd = B.ncoll[dad];
    // coarser leaves adjacent to the parent, in increasing box number
    if (lev >= 2) {
      int cand[9], nc = 0;
      for (int q = 0; q < ncd; q++) {
        int j = cd[q];
        if (B.nchild[j] == 0) {
          int t = nc++;
          while (t > 0 && cand[t - 1] > j) {
            cand[t] = cand[t - 1];
            t--;
          }
          cand[t] = j;
        }
      }
      double dt = 1.05 * (boxsize[lev - 1] + boxsize[lev]) / 2.0;
      for (int q = 0; q < nc; q++) {
        int j = cand[q];
        double2 cj = B.center[j];
        double xd = fabs(cb.x - cj.x), yd = fabs(cb.y - cj.y);
        if (xd < dt && yd < dt) {
          if (n1 < MNLIST1) L1[n1] = j;
          n1++;
        } else {
          if (n4 < MNLIST4) L4[n4] = j;
          n4++;
        }
      }
    }
    // list 2: well-separated children of the parent's colleagues
    double tol = (double)1.05f * boxsize[lev];
    for (int q = 0; q < ncd; q++) {
      int j = cd[q];
      int nc = B.nchild[j];
      int4 ch = B.child[j];
      int cc[4] = {ch.x, ch.y, ch.z, ch.w};
      for (int t = 0; t < nc; t++) {
        int k = cc[t];
        double2 ck = B.center[k];
        if (fabs(ck.x - cb.x) >= tol || fabs(ck.y - cb.y) >= tol) {
          if (n2 < MNLIST2) L2[n2] = k;
          n2++;
        }
      }
    }
    if (leaf) {
      const int* cl = B.coll + 9 * (size_t)b;
      int ncl = B.ncoll[b];
      double dt = 1.05 * (boxsize[lev] + boxsize[lev + 1]) / 2.0;
      for (int q = 0; q < ncl; q++) {
        int j = cl[q];
        int nc = B.nchild[j];
        if (nc == 0) {
          if (n1 < MNLIST1) L1[n1] = j;
          n1++;
          continue;
        }
        int4 ch = B.child[j];
        int cc[4] = {ch.x, ch.y, ch.z, ch.w};
        for (int t = 0; t < nc; t++) {
          int k = cc[t];
          double2 ck = B.center[k];
          double xd = fabs(ck.x - cb.x), yd = fabs(ck.y - cb.y);
          if (xd < dt && yd < dt) {
            if (n1 < MNLIST1) L1[n1] = k;
            n1++;
          } else {
            if (n3 < MNLIST3) L3[n3] = k;
            n3++;
          }
        }
      }
    }
  }
  nl1[b] = min(n1, MNLIST1);
  nl2[b] = min(n2, MNLIST2);
  nl3[b] = min(n3, MNLIST3);
  nl4[b] = min(n4, MNLIST4);
  for (int q = n1; q < MNLIST1; q++) L1[q] = -1;
  for (int q = n2; q < MNLIST2; q++) L2[q] = -1;
  for (int q = n3; q < MNLIST3; q++) L3[q] = -1;
  for (int q = n4; q < MNLIST4; q++) L4[q] = -1;
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
void alloc_boxes(DeviceTree& T, int cap) {
  cudaStream_t st = T.st;
  T.center.alloc(cap, st);
  T.level.alloc(cap, st);
  T.parent.alloc(cap, st);
  T.nchild.alloc(cap, st);
  T.child.alloc(cap, st);
  T.iflag.alloc(cap, st);
  T.ncoll.alloc(cap, st);
  T.coll.alloc((size_t)9 * cap, st);
  T.srng.alloc(cap, st);
  T.trng.alloc(cap, st);
  T.cap = cap;
}

// Resident blocks of the persistent build kernel on this device.
int tree_grid() {
  static std::mutex mu;
  static int grid[128] = {0};
  int dev = 0;
  B2_CHECK(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> g(mu);
  if (!grid[dev]) {
    int nsm = 0, per = 0, coop = 0;
    B2_CHECK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    B2_CHECK(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
    if (!coop) throw CudaError("tree build: cooperative launch not supported", IER_CUDA);
    B2_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_tree_build, TB_THREADS, 0));
    grid[dev] = std::max(1, std::min(per * nsm, TB_MAXG));
  }
  return grid[dev];
}

}  // namespace

int* pinned_ints(int n) { return (int*)pinned_bytes(sizeof(int) * (size_t)n); }
double* pinned_doubles(int n) { return (double*)pinned_bytes(sizeof(double) * (size_t)n); }

namespace {

// One build attempt on st with capacity cap: box arrays, hash table and
// scratch, the root, the persistent build kernel.  Outcome in T.ctl.
void launch_tree_attempt(DeviceTree& T, long ns, long nt, int idivflag, int ndiv, int nlmax,
                         int cap, cudaStream_t st, double lbal) {
  alloc_boxes(T, cap);
  DBuf<double2> sc(st);
  DBuf<int> sl(st), sp(st), sn(st), sf(st), flag(st);
  DBuf<int4> sch(st);
  DBuf<uint64_t> pk1(st), pk2(st);
  DBuf<unsigned long long> hkey(st);
  DBuf<int> hbox(st);
  unsigned hcap = 1;
  while (hcap < 2u * (unsigned)cap) hcap <<= 1;
  hkey.alloc(hcap, st);
  hbox.alloc(hcap, st);
  BoxHash H{hkey.p, hbox.p, hcap - 1};
  sc.alloc(cap, st);
  sl.alloc(cap, st);
  sp.alloc(cap, st);
  sn.alloc(cap, st);
  sf.alloc(cap, st);
  sch.alloc(cap, st);
  flag.alloc(cap, st);
  pk1.alloc(cap, st);
  pk2.alloc(cap, st);
  BoxPtrs B = ptrs(T);
  B.pkey = pk1.p;
  BoxPtrs S{sc.p, sl.p, sp.p, sn.p, sch.p, sf.p, pk2.p, nullptr, nullptr, nullptr, nullptr};
  k_init_root<<<1, 1, 0, st>>>(B, T.root.p, (int)ns, (int)nt, T.ctl.p, cap,
                               g_tree_bar_cycles.load());
  B2_LAUNCH_CHECK();
  TreeKeys K{T.skhi.p, T.sklo.p, T.tkhi.p, T.tklo.p};
  TreeCtl* C = T.ctl.p;
  int* fp = flag.p;
  int nsi = (int)ns, nti = (int)nt;
  int deep = T.deep_sorted ? 1 : 0;
  // pivot level of the level balance: where boxes of a uniform cloud of the
  // counted points hold ndiv of them
  const long npiv = idivflag == 0 ? ns : (idivflag == 1 ? nt : std::max(ns, nt));
  float fl_bal = (float)lbal;
  float fl_piv = (float)(0.5 * std::log2(std::max(1.0, (double)npiv / std::max(ndiv, 1))));
  void* args[] = {&B, &S, &C, &fp, &K, &H, &nsi, &nti, &idivflag, &ndiv, &nlmax, &deep,
                  &fl_bal, &fl_piv};
  B2_CHECK(cudaLaunchCooperativeKernel((const void*)k_tree_build, dim3(tree_grid()),
                                       dim3(TB_THREADS), args, 0, st));
  // the scratch above is released stream-ordered after the kernel
}

// Root box (bounding square of sources and targets) and the point sort by
// the first 32 key levels.
void tree_prologue(DeviceTree& T, const double* src, long ns, const double* trg, long nt,
                   cudaStream_t st) {
  T.st = st;
  T.ns = ns;
  T.nt = nt;
  T.deep_sorted = false;
  T.host_known = false;
  int nblk = std::max(1, std::min(ceil_div(std::max(ns, nt), 256), 1184));
  DBuf<double4> part(st);
  part.alloc(nblk, st);
  T.root.alloc(3, st);
  T.ctl.alloc(1, st);
  k_bbox<<<nblk, 256, 0, st>>>(src, ns, trg, nt, part.p);
  B2_LAUNCH_CHECK();
  k_bbox_final<<<1, 256, 0, st>>>(part.p, nblk, T.root.p);
  B2_LAUNCH_CHECK();
  sort_by_key(src, ns, T.root.p, false, T.skhi, T.sklo, T.isrc, st);
  sort_by_key(trg, nt, T.root.p, false, T.tkhi, T.tklo, T.itarg, st);
}

// Lists 1-4 for at most nb_alloc boxes; the kernel takes the box count from
// the control block (nothing after a failed build).
void launch_lists(DeviceTree& T, int nb_alloc, cudaStream_t st) {
  const int nb = nb_alloc;
  T.nlist1.alloc(nb, st);
  T.list1.alloc((size_t)MNLIST1 * nb, st);
  T.nlist2.alloc(nb, st);
  T.list2.alloc((size_t)MNLIST2 * nb, st);
  T.nlist3.alloc(nb, st);
  T.list3.alloc((size_t)MNLIST3 * nb, st);
  T.nlist4.alloc(nb, st);
  T.list4.alloc((size_t)MNLIST4 * nb, st);
  k_lists<<<ceil_div(nb, 128), 128, 0, st>>>(ptrs(T), T.ctl.p, T.nlist1.p, T.list1.p,
                                             T.nlist2.p, T.list2.p, T.nlist3.p, T.list3.p,
                                             T.nlist4.p, T.list4.p);
  B2_LAUNCH_CHECK();
}

std::mutex g_shape_mu;
double g_cap_ratio = 3.0;  // boxes per (points / ndiv) of the largest tree seen
struct Shape {
  long npts;
  int ndiv, nboxes, nlevels;
};
std::vector<Shape> g_shapes;  // most recent last, at most 64

}  // namespace

void note_tree_shape(long npts, int ndiv, int nboxes, int nlevels) {
  if (npts <= 0) return;
  const double r = (double)nboxes / ((double)npts / std::max(ndiv, 1));
  std::lock_guard<std::mutex> g(g_shape_mu);
  g_cap_ratio = std::max(g_cap_ratio, std::min(r, 64.0));
  for (auto& e : g_shapes)
    if (e.npts == npts && e.ndiv == ndiv) {
      e.nboxes = nboxes;
      e.nlevels = nlevels;
      return;
    }
  if (g_shapes.size() >= 64) g_shapes.erase(g_shapes.begin());
  g_shapes.push_back({npts, ndiv, nboxes, nlevels});
}

bool tree_shape(long npts, int ndiv, int* nboxes, int* nlevels) {
  std::lock_guard<std::mutex> g(g_shape_mu);
  for (auto& e : g_shapes)
    if (e.npts == npts && e.ndiv == ndiv) {
      *nboxes = e.nboxes;
      *nlevels = e.nlevels;
      return true;
    }
  return false;
}

void set_tree_barrier_limit(long long cycles) { g_tree_bar_cycles.store(cycles); }

int tree_capacity_guess(long npts, int ndiv, double margin) {
  int nb = 0, nl = 0;
  double c;
  if (tree_shape(npts, ndiv, &nb, &nl)) {
    c = margin * nb + 64;
  } else {
    double r;
    {
      std::lock_guard<std::mutex> g(g_shape_mu);
      r = g_cap_ratio;
    }
    c = std::max(4.0, 1.15 * r) * ((double)npts / std::max(ndiv, 1)) + 64;
  }
  return (int)std::min(c, (double)(1 << 29));
}

void build_device_tree_async(DeviceTree& T, const double* src, long ns, const double* trg,
                             long nt, int idivflag, int ndiv, int nlmax, int cap,
                             cudaStream_t st, double lbal) {
  tree_prologue(T, src, ns, trg, nt, st);
  cap = std::max(cap, 64);
  launch_tree_attempt(T, ns, nt, idivflag, ndiv, nlmax, cap, st, lbal);
  T.nboxes = cap;  // an upper bound until read back
  T.nlevels = -1;
  launch_lists(T, cap, st);
}

void build_device_tree(DeviceTree& T, const double* src, long ns, const double* trg, long nt,
                       int idivflag, int ndiv, int nlmax, cudaStream_t st, double lbal) {
  tree_prologue(T, src, ns, trg, nt, st);
  // one persistent kernel builds the whole tree; it is re-run with more
  // capacity (or with the 51-level keys) when it reports that need
  int cap = (int)std::min<long>(8 + 3 * (ns + nt) / std::max(ndiv, 1), 1L << 30);
  cap = std::max(cap, 64);
  // control block and root box read back together after each build attempt
  char* hbuf = (char*)pinned_bytes(sizeof(TreeCtl) + 4 * sizeof(double));
  TreeCtl* hc = (TreeCtl*)hbuf;
  double* hr = (double*)(hbuf + sizeof(TreeCtl));
  static_assert(sizeof(TreeCtl) % sizeof(double) == 0, "root after the control block");
  for (;;) {
    launch_tree_attempt(T, ns, nt, idivflag, ndiv, nlmax, cap, st, lbal);
    B2_CHECK(cudaMemcpyAsync(hc, T.ctl.p, sizeof(TreeCtl), cudaMemcpyDeviceToHost, st));
    B2_CHECK(cudaMemcpyAsync(hr, T.root.p, 3 * sizeof(double), cudaMemcpyDeviceToHost, st));
    B2_CHECK(cudaStreamSynchronize(st));
    if (hc->status == TB_DEEP && !T.deep_sorted) {
      // levels beyond 32 need the points ordered by all key digits
      sort_by_key(src, ns, T.root.p, true, T.skhi, T.sklo, T.isrc, st);
      sort_by_key(trg, nt, T.root.p, true, T.tkhi, T.tklo, T.itarg, st);
      T.deep_sorted = true;
      continue;
    }
    if (hc->status == TB_OVERFLOW) {
      if (cap >= (1 << 29)) throw CudaError("tree build: too many boxes", IER_ALLOC);
      cap = (int)std::min<long>(2L * cap, 1L << 30);
      continue;
    }
    if (hc->status == TB_BADPTS)
      throw CudaError("a source or target coordinate is not finite", IER_BADARG);
    if (hc->status != TB_OK) throw CudaError("tree build: grid barrier timed out", IER_TIMEOUT);
    break;
  }
  T.host_known = true;
  T.nlevels = hc->nlevels;
  T.nboxes = hc->nboxes;
  T.lfirst.assign(hc->lfirst, hc->lfirst + T.nlevels + 1);
  T.llast.assign(hc->llast, hc->llast + T.nlevels + 1);
  T.boxsize.assign(hc->bs, hc->bs + T.nlevels + 1);
  T.bs0 = hc->bs[0];
  T.cx0 = hr[0];
  T.cy0 = hr[1];
  // the shape cache is keyed by (points, ndiv): level-balanced trees stay out
  if (lbal == 0.0) note_tree_shape(ns + nt, ndiv, T.nboxes, T.nlevels);
  launch_lists(T, T.nboxes, st);
}

}  // namespace b2
