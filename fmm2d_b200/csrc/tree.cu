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
#include "tree.cuh"

#include <cub/cub.cuh>

#include <algorithm>
#include <cfloat>

namespace b2 {

namespace {

// ---------------------------------------------------------------------------
// pinned readback scratch
// ---------------------------------------------------------------------------
thread_local void* g_pinned = nullptr;
thread_local size_t g_pinned_bytes = 0;

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
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < ns; i += stride) {
    double x = src[2 * i], y = src[2 * i + 1];
    minmax4(v, make_double4(x, x, y, y));
  }
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < nt; i += stride) {
    double x = trg[2 * i], y = trg[2 * i + 1];
    minmax4(v, make_double4(x, x, y, y));
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
                       uint64_t* khi, uint64_t* klo, int* idx) {
  long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  double x = xy[2 * i], y = xy[2 * i + 1];
  double cx = root[0], cy = root[1], bs = root[2];
  uint64_t hi = 0, lo = 0;
  for (int lev = 1; lev <= NLMAX; lev++) {
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
  k_keys<<<ceil_div(n, 256), 256, 0, st>>>(xy, n, root, khi.p, klo.p, idx.p);
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
  k_gather_u64<<<ceil_div(n, 256), 256, 0, st>>>(klo.p, idx_out.p, n, klo_out.p);
  B2_LAUNCH_CHECK();
}

// Split the sorted range r of a box at level lev-1 into its four children
// at level lev (digit 0..3 is non-decreasing inside the range).
__device__ __forceinline__ void split_range(int2 r, const uint64_t* __restrict__ khi,
                                            const uint64_t* __restrict__ klo, int lev,
                                            int2 out[4]) {
  int b[5];
  b[0] = r.x;
  b[4] = r.y;
  for (int d = 1; d <= 3; d++) {
    int lo = b[d - 1], hi = r.y;
    while (lo < hi) {
      int m = (lo + hi) >> 1;
      if (key_digit(khi[m], klo[m], lev) < d)
        lo = m + 1;
      else
        hi = m;
    }
    b[d] = lo;
  }
  for (int d = 0; d < 4; d++) out[d] = make_int2(b[d], b[d + 1]);
}

// ---------------------------------------------------------------------------
// box kernels
// ---------------------------------------------------------------------------
struct BoxPtrs {
  double2* center;
  int* level;
  int* parent;
  int* nchild;
  int4* child;
  int* iflag;
  int* ncoll;
  int* coll;
  int2* srng;
  int2* trng;
};

BoxPtrs ptrs(DeviceTree& T) {
  return BoxPtrs{T.center.p, T.level.p, T.parent.p, T.nchild.p, T.child.p,
                 T.iflag.p,  T.ncoll.p, T.coll.p,   T.srng.p,   T.trng.p};
}

__global__ void k_init_root(BoxPtrs B, const double* root, int ns, int nt) {
  B.center[0] = make_double2(root[0], root[1]);
  B.level[0] = 0;
  B.parent[0] = -1;
  B.nchild[0] = 0;
  B.child[0] = make_int4(-1, -1, -1, -1);
  B.iflag[0] = 0;
  B.srng[0] = make_int2(0, ns);
  B.trng[0] = make_int2(0, nt);
}

// refine if the relevant count exceeds ndiv (pts_tree2d.f:538-560)
__global__ void k_refine_flags(BoxPtrs B, int first, int n, int idivflag, int ndiv, int* flags) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int b = first + i;
  int nss = B.srng[b].y - B.srng[b].x, ntt = B.trng[b].y - B.trng[b].x;
  int nn = idivflag == 0 ? nss : (idivflag == 1 ? ntt : max(nss, ntt));
  flags[i] = nn > ndiv ? 1 : 0;
}

__global__ void k_total(const int* flags, const int* scan, int n, int* out) {
  out[0] = n > 0 ? scan[n - 1] + flags[n - 1] : 0;
}

// Create the four children of parent b as boxes base..base+3 with the
// reference's child order (-,-), (+,-), (-,+), (+,+).
__device__ __forceinline__ void create_children(BoxPtrs& B, int b, int base, double bs_child,
                                                int lev_child, int child_flag) {
  double2 c = B.center[b];
  double h = bs_child / 2;
  for (int j = 0; j < 4; j++) {
    int k = base + j;
    B.center[k] = make_double2(c.x + ((j & 1) ? h : -h), c.y + ((j < 2) ? -h : h));
    B.level[k] = lev_child;
    B.parent[k] = b;
    B.nchild[k] = 0;
    B.child[k] = make_int4(-1, -1, -1, -1);
    B.iflag[k] = child_flag;
    B.srng[k] = make_int2(0, 0);
    B.trng[k] = make_int2(0, 0);
  }
  B.nchild[b] = 4;
  B.child[b] = make_int4(base, base + 1, base + 2, base + 3);
}

// Adaptive refinement of one level, with the children's point ranges.
__global__ void k_make_children_t0(BoxPtrs B, int first, int n, const int* flags, const int* scan,
                                   int child_base, double bs_child, int lev_child,
                                   const uint64_t* skhi, const uint64_t* sklo,
                                   const uint64_t* tkhi, const uint64_t* tklo) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || !flags[i]) return;
  int b = first + i;
  int base = child_base + 4 * scan[i];
  int2 sr = B.srng[b], tr = B.trng[b];
  create_children(B, b, base, bs_child, lev_child, 0);
  int2 r[4];
  split_range(sr, skhi, sklo, lev_child, r);
  for (int j = 0; j < 4; j++) B.srng[base + j] = r[j];
  split_range(tr, tkhi, tklo, lev_child, r);
  for (int j = 0; j < 4; j++) B.trng[base + j] = r[j];
}

// Colleagues from the parent's colleagues' children (tree_routs2d.f:160-206).
__global__ void k_colleagues(BoxPtrs B, int first, int n, double tol) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int b = first + i;
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
// The outcome does not depend on the order of the boxes, so all levels >= 2
// run in one launch.
__global__ void k_flag_pass(BoxPtrs B, int first, int n, const double* distest) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int b = first + i;
  int lev = B.level[b];
  if (lev < 2) return;
  double dt = distest[lev];
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
// box that touches that box (pts_tree2d.f:852-890); one level per launch.
__global__ void k_flagplus(BoxPtrs B, int first, int n, double dt) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int b = first + i;
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

// Mark boxes (over one contiguous range, or two concatenated ranges) whose
// flag is > 0.
__global__ void k_mark2(const int* iflag, int f1, int n1, int f2, int n2, int* flags) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n1 + n2) return;
  int b = i < n1 ? f1 + i : f2 + (i - n1);
  flags[i] = iflag[b] > 0 ? 1 : 0;
}

// Refine flagged boxes of one or two concatenated ranges; children of flag-1
// boxes become flag++ (3), of flag+ boxes 0 (tree_routs2d.f:355-385).
__global__ void k_make_children_flag(BoxPtrs B, int f1, int n1, int f2, int n2, const int* flags,
                                     const int* scan, int child_base, const double* boxsize) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n1 + n2 || !flags[i]) return;
  int b = i < n1 ? f1 + i : f2 + (i - n1);
  int lev_child = B.level[b] + 1;
  int pf = B.iflag[b];
  create_children(B, b, child_base + 4 * scan[i], boxsize[lev_child], lev_child, pf == 1 ? 3 : 0);
}

// Per-level counts of flagged boxes inside [lf[l], ll[l]] (T0 layout).
__global__ void k_level_counts(const int* flags, const int* scan, int base, const int* lf,
                               const int* ll, int l0, int l1, int* cnt) {
  int l = l0 + blockIdx.x * blockDim.x + threadIdx.x;
  if (l > l1) return;
  int a = lf[l] - base, e = ll[l] - base;
  cnt[l] = scan[e] + flags[e] - scan[a];
}

__global__ void k_keep_flag3(int* iflag, int n) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n && iflag[i] != 3) iflag[i] = 0;
}

// A flag++ box is refined if a child (with children) of one of its
// colleagues touches it (tree_routs2d.f:217-326).
__global__ void k_update_flags(BoxPtrs B, int f1, int n1, int f2, int n2, double dt, int* flags) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n1 + n2) return;
  int b = i < n1 ? f1 + i : f2 + (i - n1);
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
  flags[i] = (f == 1) ? 1 : 0;
}

// Renumbering: per level, the level's current range, then its tail
// (pts_tree2d.f:1066-1215).  lv = [lf, ll, tf, tl, newf] x (nl+1).
__global__ void k_reorg_map(const int* level, int n, const int* lv, int nl1, int* map) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= n) return;
  int l = level[b];
  int lf = lv[l], ll = lv[nl1 + l], tf = lv[2 * nl1 + l], newf = lv[4 * nl1 + l];
  map[b] = (b >= lf && b <= ll) ? newf + (b - lf) : newf + (ll - lf + 1) + (b - tf);
}

__global__ void k_reorg_apply(BoxPtrs S, BoxPtrs D, const int* map, int n) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= n) return;
  int m = map[b];
  D.center[m] = S.center[b];
  D.level[m] = S.level[b];
  D.nchild[m] = S.nchild[b];
  D.iflag[m] = S.iflag[b];
  int p = S.parent[b];
  D.parent[m] = p < 0 ? -1 : map[p];
  int4 c = S.child[b];
  D.child[m] = make_int4(c.x < 0 ? -1 : map[c.x], c.y < 0 ? -1 : map[c.y],
                         c.z < 0 ? -1 : map[c.z], c.w < 0 ? -1 : map[c.w]);
}

// Point ranges of the children of every refined box of one level.
__global__ void k_split_ranges(BoxPtrs B, int first, int n, int lev_child, const uint64_t* skhi,
                               const uint64_t* sklo, const uint64_t* tkhi, const uint64_t* tklo) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int b = first + i;
  if (B.nchild[b] == 0) return;
  int4 ch = B.child[b];
  int cc[4] = {ch.x, ch.y, ch.z, ch.w};
  int2 r[4];
  split_range(B.srng[b], skhi, sklo, lev_child, r);
  for (int j = 0; j < 4; j++) B.srng[cc[j]] = r[j];
  split_range(B.trng[b], tkhi, tklo, lev_child, r);
  for (int j = 0; j < 4; j++) B.trng[cc[j]] = r[j];
}

__global__ void k_set_root_range(BoxPtrs B, int ns, int nt) {
  B.srng[0] = make_int2(0, ns);
  B.trng[0] = make_int2(0, nt);
}

// Lists 1-4 of every box (tree_routs2d.f:486-710), as a gather: a box's
// list 1 starts with the coarser adjacent leaves (which the reference
// appends while visiting the coarser level, in increasing box number), then
// its own entries; its list 4 holds the coarser non-adjacent leaves.
__global__ void k_lists(BoxPtrs B, int nb, const double* boxsize, int* nl1, int* l1, int* nl2,
                        int* l2, int* nl3, int* l3, int* nl4, int* l4) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nb) return;
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
// host helpers
// ---------------------------------------------------------------------------
struct Scanner {
  DBuf<char> tmp;
  size_t bytes = 0;
  DBuf<int> total;
  // exclusive scan of flags[0..n) into scan; returns the total (synchronises)
  int run(const int* flags, int* scan, int n, cudaStream_t st) {
    if (n <= 0) return 0;
    size_t need = 0;
    B2_CHECK(cub::DeviceScan::ExclusiveSum(nullptr, need, flags, scan, n, st));
    if (need > bytes) {
      tmp.alloc(need, st);
      bytes = need;
    }
    B2_CHECK(cub::DeviceScan::ExclusiveSum(tmp.p, need, flags, scan, n, st));
    if (!total.p) total.alloc(1, st);
    k_total<<<1, 1, 0, st>>>(flags, scan, n, total.p);
    B2_LAUNCH_CHECK();
    int* h = (int*)pinned_bytes(sizeof(int));
    B2_CHECK(cudaMemcpyAsync(h, total.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    B2_CHECK(cudaStreamSynchronize(st));
    return h[0];
  }
};

void ensure_cap(DeviceTree& T, int need) {
  if (need <= T.cap) return;
  int nc = std::max(need, T.cap * 2);
  size_t keep = T.nboxes;
  T.center.grow(nc, keep);
  T.level.grow(nc, keep);
  T.parent.grow(nc, keep);
  T.nchild.grow(nc, keep);
  T.child.grow(nc, keep);
  T.iflag.grow(nc, keep);
  T.ncoll.grow(nc, keep);
  T.coll.grow((size_t)9 * nc, (size_t)9 * keep);
  T.srng.grow(nc, keep);
  T.trng.grow(nc, keep);
  T.cap = nc;
}

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

void colleagues_level(DeviceTree& T, int lev, int first, int n) {
  if (n <= 0) return;
  double tol = (double)1.05f * T.boxsize[lev];
  k_colleagues<<<ceil_div(n, 128), 128, 0, T.st>>>(ptrs(T), first, n, tol);
  B2_LAUNCH_CHECK();
}

void colleagues_all(DeviceTree& T) {
  for (int l = 0; l <= T.nlevels; l++)
    colleagues_level(T, l, T.lfirst[l], T.llast[l] - T.lfirst[l] + 1);
}

void reorganize(DeviceTree& T, const std::vector<int>& tf, const std::vector<int>& tl) {
  int nl1 = T.nlevels + 1;
  std::vector<int> lv(5 * nl1);
  int cur = 0;
  for (int l = 0; l < nl1; l++) {
    int no = T.llast[l] - T.lfirst[l] + 1;
    int nt = tl[l] - tf[l] + 1;
    lv[l] = T.lfirst[l];
    lv[nl1 + l] = T.llast[l];
    lv[2 * nl1 + l] = tf[l];
    lv[3 * nl1 + l] = tl[l];
    lv[4 * nl1 + l] = cur;
    cur += no + std::max(nt, 0);
  }
  cudaStream_t st = T.st;
  int* hp = (int*)pinned_bytes(sizeof(int) * lv.size());
  B2_CHECK(cudaStreamSynchronize(st));  // the pinned scratch may still be in flight
  std::copy(lv.begin(), lv.end(), hp);
  DBuf<int> dlv(st), map(st);
  dlv.alloc(lv.size(), st);
  B2_CHECK(cudaMemcpyAsync(dlv.p, hp, sizeof(int) * lv.size(), cudaMemcpyHostToDevice, st));
  int nb = T.nboxes;
  map.alloc(nb, st);
  k_reorg_map<<<ceil_div(nb, 256), 256, 0, st>>>(T.level.p, nb, dlv.p, nl1, map.p);
  B2_LAUNCH_CHECK();
  DeviceTree N;
  N.st = st;
  alloc_boxes(N, T.cap);
  k_reorg_apply<<<ceil_div(nb, 256), 256, 0, st>>>(ptrs(T), ptrs(N), map.p, nb);
  B2_LAUNCH_CHECK();
  std::swap(T.center, N.center);
  std::swap(T.level, N.level);
  std::swap(T.parent, N.parent);
  std::swap(T.nchild, N.nchild);
  std::swap(T.child, N.child);
  std::swap(T.iflag, N.iflag);
  for (int l = 0; l < nl1; l++) {
    int no = T.llast[l] - T.lfirst[l] + 1;
    int nt = std::max(tl[l] - tf[l] + 1, 0);
    T.lfirst[l] = lv[4 * nl1 + l];
    T.llast[l] = lv[4 * nl1 + l] + no + nt - 1;
  }
  B2_CHECK(cudaStreamSynchronize(st));  // keep `hp` valid until the upload is done
}

DBuf<double> upload_doubles(const std::vector<double>& v, cudaStream_t st) {
  DBuf<double> d(st);
  d.alloc(v.size(), st);
  double* hp = (double*)pinned_bytes(sizeof(double) * v.size());
  B2_CHECK(cudaStreamSynchronize(st));
  std::copy(v.begin(), v.end(), hp);
  B2_CHECK(cudaMemcpyAsync(d.p, hp, sizeof(double) * v.size(), cudaMemcpyHostToDevice, st));
  B2_CHECK(cudaStreamSynchronize(st));
  return d;
}

void fix_level_restriction(DeviceTree& T, Scanner& sc) {
  cudaStream_t st = T.st;
  const int nl = T.nlevels;
  std::vector<double> dflag(nl + 1, 0.0);
  for (int l = 2; l <= nl; l++) dflag[l] = 1.05 * (T.boxsize[l - 1] + T.boxsize[l - 2]) / 2.0;
  DBuf<double> ddflag = upload_doubles(dflag, st);
  DBuf<double> dbs = upload_doubles(T.boxsize, st);
  // pass 1: flag
  {
    int f = T.lfirst[2], n = T.nboxes - f;
    k_flag_pass<<<ceil_div(n, 128), 128, 0, st>>>(ptrs(T), f, n, ddflag.p);
    B2_LAUNCH_CHECK();
  }
  // pass 2: flag+, finest level first
  for (int l = nl; l >= 1; l--) {
    double dt = 1.05 * (T.boxsize[l] + T.boxsize[l - 1]) / 2.0;
    int n = T.llast[l] - T.lfirst[l] + 1;
    k_flagplus<<<ceil_div(n, 128), 128, 0, st>>>(ptrs(T), T.lfirst[l], n, dt);
    B2_LAUNCH_CHECK();
  }
  std::vector<int> tf(nl + 1, 0), tl(nl + 1, -1);
  // subdivide flag and flag+ boxes of levels 1..nl-2
  if (nl - 2 >= 1) {
    int f = T.lfirst[1], n = T.llast[nl - 2] - f + 1;
    DBuf<int> flags(st), scan(st), cnt(st);
    flags.alloc(n, st);
    scan.alloc(n, st);
    k_mark2<<<ceil_div(n, 256), 256, 0, st>>>(T.iflag.p, f, n, 0, 0, flags.p);
    B2_LAUNCH_CHECK();
    int tot = sc.run(flags.p, scan.p, n, st);
    if (tot > 0) {
      std::vector<int> lfl(nl + 1), lll(nl + 1);
      for (int l = 0; l <= nl; l++) {
        lfl[l] = T.lfirst[l];
        lll[l] = T.llast[l];
      }
      DBuf<int> dlf(st), dll(st);
      dlf.alloc(nl + 1, st);
      dll.alloc(nl + 1, st);
      int* hp = (int*)pinned_bytes(sizeof(int) * 2 * (nl + 1));
      std::copy(lfl.begin(), lfl.end(), hp);
      std::copy(lll.begin(), lll.end(), hp + nl + 1);
      B2_CHECK(cudaMemcpyAsync(dlf.p, hp, sizeof(int) * (nl + 1), cudaMemcpyHostToDevice, st));
      B2_CHECK(cudaMemcpyAsync(dll.p, hp + nl + 1, sizeof(int) * (nl + 1), cudaMemcpyHostToDevice,
                               st));
      cnt.alloc(nl + 1, st);
      cnt.zero(nl + 1);
      k_level_counts<<<1, 64, 0, st>>>(flags.p, scan.p, f, dlf.p, dll.p, 1, nl - 2, cnt.p);
      B2_LAUNCH_CHECK();
      int* hc = (int*)pinned_bytes(sizeof(int) * (nl + 1) * 3);
      B2_CHECK(cudaStreamSynchronize(st));
      B2_CHECK(cudaMemcpyAsync(hc, cnt.p, sizeof(int) * (nl + 1), cudaMemcpyDeviceToHost, st));
      B2_CHECK(cudaStreamSynchronize(st));
      std::vector<int> c(hc, hc + nl + 1);
      ensure_cap(T, T.nboxes + 4 * tot);
      k_make_children_flag<<<ceil_div(n, 128), 128, 0, st>>>(ptrs(T), f, n, 0, 0, flags.p, scan.p,
                                                              T.nboxes, dbs.p);
      B2_LAUNCH_CHECK();
      int base = T.nboxes;
      for (int l = 1; l <= nl - 2; l++) {
        tf[l + 1] = base;
        tl[l + 1] = base + 4 * c[l] - 1;
        base += 4 * c[l];
      }
      T.nboxes += 4 * tot;
    }
  }
  reorganize(T, tf, tl);
  colleagues_all(T);
  k_keep_flag3<<<ceil_div(T.nboxes, 256), 256, 0, st>>>(T.iflag.p, T.nboxes);
  B2_LAUNCH_CHECK();
  std::fill(tf.begin(), tf.end(), 0);
  std::fill(tl.begin(), tl.end(), -1);
  // pass 3: flag++ boxes, coarsest level first, refining as needed
  DBuf<int> flags(st), scan(st);
  for (int l = 2; l <= nl - 2; l++) {
    int f1 = T.lfirst[l], n1 = T.llast[l] - f1 + 1;
    int f2 = tf[l], n2 = std::max(tl[l] - tf[l] + 1, 0);
    int n = n1 + n2;
    if (n <= 0) continue;
    flags.grow(n, 0);
    scan.grow(n, 0);
    double dt = 1.05 * (T.boxsize[l] + T.boxsize[l + 1]) / 2.0;
    k_update_flags<<<ceil_div(n, 128), 128, 0, st>>>(ptrs(T), f1, n1, f2, n2, dt, flags.p);
    B2_LAUNCH_CHECK();
    int tot = sc.run(flags.p, scan.p, n, st);
    if (tot == 0) continue;
    ensure_cap(T, T.nboxes + 4 * tot);
    k_make_children_flag<<<ceil_div(n, 128), 128, 0, st>>>(ptrs(T), f1, n1, f2, n2, flags.p,
                                                            scan.p, T.nboxes, dbs.p);
    B2_LAUNCH_CHECK();
    tf[l + 1] = T.nboxes;
    tl[l + 1] = T.nboxes + 4 * tot - 1;
    T.nboxes += 4 * tot;
    colleagues_level(T, l + 1, tf[l + 1], 4 * tot);
  }
  reorganize(T, tf, tl);
  colleagues_all(T);
}

}  // namespace

int* pinned_ints(int n) { return (int*)pinned_bytes(sizeof(int) * (size_t)n); }
double* pinned_doubles(int n) { return (double*)pinned_bytes(sizeof(double) * (size_t)n); }

void build_device_tree(DeviceTree& T, const double* src, long ns, const double* trg, long nt,
                       int idivflag, int ndiv, int nlmax, cudaStream_t st) {
  T.st = st;
  T.ns = ns;
  T.nt = nt;
  T.deep_sorted = false;
  // root box
  int nblk = std::max(1, std::min(ceil_div(std::max(ns, nt), 256), 1184));
  DBuf<double4> part(st);
  part.alloc(nblk, st);
  T.root.alloc(3, st);
  k_bbox<<<nblk, 256, 0, st>>>(src, ns, trg, nt, part.p);
  B2_LAUNCH_CHECK();
  k_bbox_final<<<1, 256, 0, st>>>(part.p, nblk, T.root.p);
  B2_LAUNCH_CHECK();
  // sort points along the virtual complete tree
  sort_by_key(src, ns, T.root.p, false, T.skhi, T.sklo, T.isrc, st);
  sort_by_key(trg, nt, T.root.p, false, T.tkhi, T.tklo, T.itarg, st);
  // boxes
  int cap0 = (int)std::min<long>(8 + 3 * (ns + nt) / std::max(ndiv, 1), 1L << 30);
  alloc_boxes(T, std::max(cap0, 64));
  k_init_root<<<1, 1, 0, st>>>(ptrs(T), T.root.p, (int)ns, (int)nt);
  B2_LAUNCH_CHECK();
  double* hr = (double*)pinned_bytes(3 * sizeof(double));
  B2_CHECK(cudaMemcpyAsync(hr, T.root.p, 3 * sizeof(double), cudaMemcpyDeviceToHost, st));
  B2_CHECK(cudaStreamSynchronize(st));
  T.cx0 = hr[0];
  T.cy0 = hr[1];
  T.bs0 = hr[2];
  T.boxsize.assign(1, T.bs0);
  T.lfirst.assign(1, 0);
  T.llast.assign(1, 0);
  T.nboxes = 1;
  Scanner sc;
  DBuf<int> flags(st), scan(st);
  int lev;
  // A zero-size root (all points coincide) cannot be subdivided: the
  // children would coincide with it forever.  Keep the root as the only box.
  if (T.bs0 == 0.0) nlmax = 0;
  for (lev = 0; lev < nlmax; lev++) {
    int f = T.lfirst[lev], n = T.llast[lev] - f + 1;
    flags.grow(n, 0);
    scan.grow(n, 0);
    k_refine_flags<<<ceil_div(n, 256), 256, 0, st>>>(ptrs(T), f, n, idivflag, ndiv, flags.p);
    B2_LAUNCH_CHECK();
    int nref = sc.run(flags.p, scan.p, n, st);
    if (nref == 0) break;
    if (lev + 1 > 32 && !T.deep_sorted) {
      // levels beyond 32 need the points ordered by all key digits
      sort_by_key(src, ns, T.root.p, true, T.skhi, T.sklo, T.isrc, st);
      sort_by_key(trg, nt, T.root.p, true, T.tkhi, T.tklo, T.itarg, st);
      T.deep_sorted = true;
    }
    T.boxsize.push_back(T.boxsize[lev] / 2);
    ensure_cap(T, T.nboxes + 4 * nref);
    k_make_children_t0<<<ceil_div(n, 128), 128, 0, st>>>(
        ptrs(T), f, n, flags.p, scan.p, T.nboxes, T.boxsize[lev + 1], lev + 1, T.skhi.p, T.sklo.p,
        T.tkhi.p, T.tklo.p);
    B2_LAUNCH_CHECK();
    T.lfirst.push_back(T.nboxes);
    T.nboxes += 4 * nref;
    T.llast.push_back(T.nboxes - 1);
  }
  T.nlevels = lev;
  colleagues_all(T);
  if (T.nlevels >= 2) fix_level_restriction(T, sc);
  // point ranges of every box of the final tree
  k_set_root_range<<<1, 1, 0, st>>>(ptrs(T), (int)ns, (int)nt);
  B2_LAUNCH_CHECK();
  for (int l = 0; l < T.nlevels; l++) {
    int n = T.llast[l] - T.lfirst[l] + 1;
    k_split_ranges<<<ceil_div(n, 128), 128, 0, st>>>(ptrs(T), T.lfirst[l], n, l + 1, T.skhi.p,
                                                     T.sklo.p, T.tkhi.p, T.tklo.p);
    B2_LAUNCH_CHECK();
  }
  // interaction lists
  int nb = T.nboxes;
  T.nlist1.alloc(nb, st);
  T.list1.alloc((size_t)MNLIST1 * nb, st);
  T.nlist2.alloc(nb, st);
  T.list2.alloc((size_t)MNLIST2 * nb, st);
  T.nlist3.alloc(nb, st);
  T.list3.alloc((size_t)MNLIST3 * nb, st);
  T.nlist4.alloc(nb, st);
  T.list4.alloc((size_t)MNLIST4 * nb, st);
  std::vector<double> bsx(T.boxsize);
  bsx.push_back(T.boxsize.back() / 2);  // boxsize(nlevels+1) for the leaf tests
  DBuf<double> dbs = upload_doubles(bsx, st);
  k_lists<<<ceil_div(nb, 128), 128, 0, st>>>(ptrs(T), nb, dbs.p, T.nlist1.p, T.list1.p,
                                             T.nlist2.p, T.list2.p, T.nlist3.p, T.list3.p,
                                             T.nlist4.p, T.list4.p);
  B2_LAUNCH_CHECK();
  B2_CHECK(cudaStreamSynchronize(st));
}

}  // namespace b2
