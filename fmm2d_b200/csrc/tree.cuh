// Device quadtree: adaptive build, level restriction, point sort and
// interaction lists, reproducing the reference tree box for box
// (src/common/pts_tree2d.f, src/common/tree_routs2d.f).
#pragma once
#include "common.cuh"

namespace b2 {

constexpr int MNLIST1 = 13, MNLIST2 = 27, MNLIST3 = 20, MNLIST4 = 5;  // tree_routs2d.f:473-476
constexpr int NLMAX = 51;                                               // cfmm2d.f:148

struct DeviceTree {
  cudaStream_t st = 0;
  long ns = 0, nt = 0;
  int nlevels = 0, nboxes = 0, cap = 0;
  double cx0 = 0, cy0 = 0, bs0 = 0;
  bool deep_sorted = false;  // keys sorted on all 51 levels (else on the first 32)
  std::vector<int> lfirst, llast;  // box range of every level (inclusive)
  std::vector<double> boxsize;     // boxsize[l] = bs0 / 2^l

  // boxes (structure of arrays, capacity `cap`)
  DBuf<double2> center;
  DBuf<int> level, parent, nchild, iflag, ncoll, coll;  // coll: 9 per box
  DBuf<int4> child;
  DBuf<int2> srng, trng;  // half-open ranges in the sorted source / target arrays

  // points sorted into tree order: isrc[k] = caller index of sorted source k
  DBuf<uint64_t> skhi, sklo, tkhi, tklo;
  DBuf<int> isrc, itarg;

  // interaction lists (fixed widths 13/27/20/5 per box)
  DBuf<int> nlist1, list1, nlist2, list2, nlist3, list3, nlist4, list4;

  // device scratch
  DBuf<double> root;  // cx, cy, bs0
};

// Build the level-restricted tree of sources `src` (2*ns doubles, x/y
// interleaved) and targets `trg` on stream `st`.  idivflag 0/1/2 subdivides
// on sources / targets / max of both, as in the reference.
void build_device_tree(DeviceTree& T, const double* src, long ns, const double* trg, long nt,
                       int idivflag, int ndiv, int nlmax, cudaStream_t st);

// Per-thread pinned scratch used for small device->host readbacks.
int* pinned_ints(int n);
double* pinned_doubles(int n);

}  // namespace b2
