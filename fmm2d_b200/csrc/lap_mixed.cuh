// Leaf and M2L kernels of the Laplace FMM.  Mixed precision (eps >= 1e-6 or
// when requested): M2L on the tensor cores (or FP32 CUDA cores), L2P / M2P
// in FP32, an FP32 near field over leaf-relative two-float offsets; the
// expansion coefficients and shifts stay FP64.  The FP64 path's leaf passes
// (far field, FP64 near field on the same work items) live here too.
#pragma once
#include <vector>
#include "lap_common.cuh"
#include "../../include/fmm2d_b200.h"
#include "tc_m2l.cuh"

namespace b2 {

// Data of the mixed-precision kernels: FP32 copies of the sorted densities,
// offset tables, the tensor-core M2L pair list, per-point leaf maps and
// near-field work items.
struct MixedData {
  const double2* xs64 = nullptr;  // sorted sources (FP64, owned by the caller)
  DBuf<float2> q, d;    // all Cauchy densities, ndc per point
  DBuf<float2> utab;    // (1/o)^k for the 7x7 integer offsets o, k < P
  DBuf<float> lgtab;    // log|o|
  M2LPairs pairs;       // list-2 targets and entries for the tensor-core M2L
  DBuf<float2> mp32;    // FP32 copy of one chunk's multipoles (tensor-core M2L)
  bool tc = false;      // run M2L on the tensor cores
  int nlev = 0;         // tree levels + 1
  int nboxes = 0;
  long ns = 0, nt = 0;
  int ndiv = 0;         // leaf capacity of the tree (selects the near-field tile shape)
  DBuf<int> leaf_s, leaf_t;     // leaf box of every sorted source / target
  DBuf<char> items_s, items_t;  // near-field work items (sources, targets)
  DBuf<int> nitems;              // their counts
  int* err = nullptr;   // device flag set by a tensor-core wait that gave up
};

// Tensor-core M2L switch (default on); off selects the FP32 CUDA-core M2L.
void set_m2l_tensor_cores(bool on);
bool m2l_tensor_cores();

// Geometry part (source pointer, offset tables) and allocation of the FP32
// density copies for ndc densities per source.
void lap_mixed_prepare(MixedData& M, const double2* xs, long ns, const double2* xt, long nt,
                       bool has_q, bool has_d, int ndc, double cx0, double cy0, int P,
                       cudaStream_t st);

// Leaf box of every sorted evaluation point and the near-field work items
// (once per tree); nb boxes at most, the box count read from the tree's
// device control block when dev.
void lap_mixed_leaves(MixedData& M, const lapk::TV& t, int nb, bool dev, long ns, long nt,
                      int ndiv, cudaStream_t st);

// Leaf evaluation of the FP64 path on the same work items: L2P + M2P
// (k_far_mixed, FP64) then the FP64 near field (k_p2p_leaf64) for one
// density chunk D (sorted FP64 densities).
void lap_fp64_leaf(int ND, int ifl, const lapk::TV& t, int use_targets, const MixedData& M,
                   const double2* xe64, const lapk::Dens& D, int P, const double2* mp,
                   const double2* lo, double thresh, int ifnear, double2* pot, double2* grad,
                   double2* hess, cudaStream_t st);

// The mixed near field of many trees in one persistent launch per group of
// (ND, pot/grad/hess level, density kind): every entry is the deferred
// near-field pass of one tree (its far field already in pot / grad / hess,
// tree order, a single density chunk of ndc <= 8).  create builds the
// device job tables (outside any capture); launch is stream work only.
struct P2PBatchEntry {
  const lapk::TV* tv;
  const MixedData* M;
  const double2* xe64;  // sorted evaluation points (M->xs64 for the sources)
  int use_targets, ndc, ND, ifl;
  double2 *pot, *grad, *hess;
};
struct P2PBatch;
P2PBatch* p2p_batch_create(const std::vector<P2PBatchEntry>& entries);
void p2p_batch_launch(const P2PBatch* b, cudaStream_t st);
void p2p_batch_free(P2PBatch* b);

// Near-field tile shape per leaf-size class (0: ndiv <= 20, 1: <= 56,
// 2: larger); set_p2p_shape returns IER_BADARG for an unknown class or shape.
int p2p_leaf_class(int ndiv);
int set_p2p_shape(int leaf_class, int shape);
int p2p_shape(int leaf_class);

// FP32 copies of the sorted densities (every evaluation).
void lap_mixed_densities(MixedData& M, const double2* qs, const double2* ds, long ns, int ndc,
                         cudaStream_t st);

// M2L over list 2 for boxes [first, first+n) of one density chunk (FP32).
void lap_mixed_m2l(int ND, const lapk::TV& t, int first, int n, int P, const double* binom,
                   const MixedData& M, const double2* mp, double2* lo, cudaStream_t st);

// Leaf evaluation (L2P + M2P in FP64, then P2P in FP32) for one density
// chunk; far_done (optional) is recorded between the two kernels.
void lap_mixed_leaf(int ND, int ifl, const lapk::TV& t, int nb, int use_targets,
                    const MixedData& M, const double2* xe64, int ndc, int d0, int P,
                    const double2* mp, const double2* lo, double thresh, int ifnear,
                    double2* pot, double2* grad, double2* hess, cudaStream_t st,
                    cudaEvent_t far_done = nullptr);

}  // namespace b2
