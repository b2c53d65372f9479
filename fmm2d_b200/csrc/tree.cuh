// Device quadtree: adaptive build, level restriction, point sort and
// interaction lists, reproducing the reference tree box for box
// (src/common/pts_tree2d.f, src/common/tree_routs2d.f).
#pragma once
#include "common.cuh"

namespace b2 {

constexpr int MNLIST1 = 13, MNLIST2 = 27, MNLIST3 = 20, MNLIST4 = 5;  // tree_routs2d.f:473-476
constexpr int NLMAX = 51;                                               // cfmm2d.f:148

constexpr int TB_MAXG = 1024;    // most blocks of the persistent build kernel
constexpr int TB_THREADS = 512;  // threads per block (one block per SM)
constexpr int TB_GROUPS = 8;     // first-level arrival counters of a grid barrier
// TB_BADPTS: a source or target coordinate is not finite
enum : int { TB_OK = 0, TB_OVERFLOW = 1, TB_DEEP = 2, TB_TIMEOUT = 3, TB_BADPTS = 4 };

// Device control block of the tree build: box count, level table (box range
// of every level), box sizes and status, followed by the grid barrier and
// scan scratch of the persistent build kernel.  It stays on the device for
// the life of the tree: the FMM passes read their box ranges from it, so a
// call need not wait for the tree on the host.  bs[l] = boxsize(l) for
// l = 0 .. nlevels + 1.
struct TreeCtl {
  int nboxes, nlevels, cap, status;
  int lfirst[NLMAX + 2], llast[NLMAX + 2];
  int tf[NLMAX + 2], tl[NLMAX + 2], lcnt[NLMAX + 2];
  double bs[NLMAX + 3];
  unsigned bar_sub[TB_GROUPS * 32];  // one 128-byte line per group
  unsigned bar_top, bar_gen;
  long long bar_cycles;  // wait limit of the grid barrier (<= 0: GRID_BAR_CYCLES)
  int tot[2][TB_MAXG];  // per-block counts of the scans, alternating
};

// Grid barrier state of a cooperative kernel other than the tree build.
struct GridBar {
  unsigned bar_sub[TB_GROUPS * 32];
  unsigned bar_top, bar_gen;
  long long bar_cycles;  // wait limit (<= 0: GRID_BAR_CYCLES)
  int status;  // 0, or the timeout code once a barrier gave up
};

constexpr long long GRID_BAR_CYCLES = 1LL << 30;  // about half a second at 2 GHz

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ unsigned atom_add_acqrel_u32(unsigned* p, unsigned v) {
  unsigned old;
  asm volatile("atom.add.acq_rel.gpu.global.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v)
               : "memory");
  return old;
}

// Two-level grid barrier of a cooperative launch (all blocks resident) with
// acquire-release ordering at GPU scope: a block arrives on its group
// counter, the last arrival of a group on the top counter, and the last
// arrival there advances the generation word the blocks wait on, so every
// write made before the barrier by any block is visible to every block after
// it.  Every wait is bounded: a barrier that gives up stores `timeout_code`
// in C->status, which releases the other blocks too.  Returns false then.
template <class Ctl>
__device__ bool grid_barrier(Ctl* C, int timeout_code) {
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned g0 = ld_acquire_u32(&C->bar_gen);
    const int G = gridDim.x, ng = min(TB_GROUPS, G), grp = blockIdx.x % ng;
    const unsigned members = (unsigned)((G - grp + ng - 1) / ng);
    unsigned* sub = &C->bar_sub[grp * 32];
    if (atom_add_acqrel_u32(sub, 1u) + 1 == members) {
      *sub = 0;
      if (atom_add_acqrel_u32(&C->bar_top, 1u) + 1 == (unsigned)ng) {
        C->bar_top = 0;
        atom_add_acqrel_u32(&C->bar_gen, 1u);
      }
    }
    if (ld_acquire_u32(&C->bar_gen) == g0) {
      const long long lim = C->bar_cycles > 0 ? C->bar_cycles : GRID_BAR_CYCLES;
      const long long t0 = clock64();
      while (ld_acquire_u32(&C->bar_gen) == g0) {
        if (clock64() - t0 > lim ||
            *reinterpret_cast<const volatile int*>(&C->status) == timeout_code) {
          atomicExch(&C->status, timeout_code);
          break;
        }
      }
    }
  }
  __syncthreads();
  return *reinterpret_cast<const volatile int*>(&C->status) != timeout_code;
}

struct DeviceTree {
  cudaStream_t st = 0;
  long ns = 0, nt = 0;
  // host_known: nlevels, nboxes, lfirst, llast, boxsize, cx0, cy0, bs0 were
  // read back.  Otherwise (a tree enqueued without waiting) only `cap` is
  // known on the host: box arrays and lists hold `cap` boxes and the
  // passes read the ranges from `ctl`.
  bool host_known = false;
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
  DBuf<TreeCtl> ctl;  // level table, box count, status (see TreeCtl)
};

// Build the level-restricted tree of sources `src` (2*ns doubles, x/y
// interleaved) and targets `trg` on stream `st`.  idivflag 0/1/2 subdivides
// on sources / targets / max of both, as in the reference.
// lbal: level balance of the leaf capacity (0: ndiv at every level, as the
// reference; otherwise ndiv 2^(lbal (lpiv - level)), lpiv the level whose
// boxes hold ndiv points of a uniform cloud of the counted points).
void build_device_tree(DeviceTree& T, const double* src, long ns, const double* trg, long nt,
                       int idivflag, int ndiv, int nlmax, cudaStream_t st, double lbal = 0.0);

// The same build enqueued on `st` without any host synchronisation: one
// attempt with capacity `cap` boxes and the first 32 key levels.  The tree
// is valid when T.ctl->status ends as TB_OK; TB_OVERFLOW (more boxes) and
// TB_DEEP (more than 32 levels) need build_device_tree instead, and every
// pass that reads its ranges from T.ctl does nothing after such a failure.
void build_device_tree_async(DeviceTree& T, const double* src, long ns, const double* trg,
                             long nt, int idivflag, int ndiv, int nlmax, int cap, cudaStream_t st,
                             double lbal = 0.0);

// Shapes of earlier trees by (points, leaf size): the box count and depth a
// call can expect without reading its tree back.  note_tree_shape records a
// tree read back (or checked at the end of a call); tree_capacity_guess
// gives the box capacity for a build that is not read back: `margin` times
// the remembered count for a size seen before, else a generous multiple of
// points / ndiv (raised by the largest ratio seen).
void note_tree_shape(long npts, int ndiv, int nboxes, int nlevels);

// Test hook: wait limit (clock cycles) of the tree build's grid barrier for
// later builds; <= 0 restores the default of about half a second.
void set_tree_barrier_limit(long long cycles);
bool tree_shape(long npts, int ndiv, int* nboxes, int* nlevels);
int tree_capacity_guess(long npts, int ndiv, double margin);

// Per-thread pinned scratch used for small device->host readbacks.
int* pinned_ints(int n);
double* pinned_doubles(int n);

}  // namespace b2
