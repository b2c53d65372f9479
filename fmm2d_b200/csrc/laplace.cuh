// Cauchy/Laplace FMM engine (the path of src/laplace/cfmm2d.f, lfmm2d.f,
// rfmm2d.f) on device memory.
#pragma once
#include <vector>

#include "common.cuh"
#include "tree.cuh"

namespace b2 {

// How caller densities map onto Cauchy densities and how results map back.
enum FrontEnd {
  FE_CAUCHY = 0,   // cfmm2d: complex charge/dipstr, outputs pot, d/dz, d2/dz2 (nd, n)
  FE_LAPLACE = 1,  // lfmm2d: complex densities split into 2 Cauchy densities each
  FE_REAL = 2      // rfmm2d: real densities
};

enum Precision { PREC_AUTO = 0, PREC_FP64 = 1, PREC_MIXED = 2 };

struct LapArgs {
  int fe = FE_CAUCHY;
  int nd = 1;  // caller's number of densities
  double eps = 1e-6;
  long ns = 0;
  const double* src = nullptr;  // (2, ns)
  const double* charge = nullptr;  // complex (nd, ns) or real (nd, ns)
  const double* dipstr = nullptr;  // complex or real (nd, ns)
  const double* dipvec = nullptr;  // (nd, 2, ns) real, lfmm/rfmm only
  int ifpgh = 0;
  double *pot = nullptr, *grad = nullptr, *hess = nullptr;
  long nt = 0;
  const double* trg = nullptr;  // (2, nt)
  int ifpghtarg = 0;
  double *pottarg = nullptr, *gradtarg = nullptr, *hesstarg = nullptr;
  // tuning (cfmm2d_ndiv.f:23-26)
  int ndiv = 0;  // <= 0: lndiv2d table
  double lbal = 0.0;  // level balance of the leaf capacity (0: ndiv at every level)
  int idivflag = 0;
  int ifnear = 1;
  int precision = PREC_AUTO;
  double* timeinfo = nullptr;  // 8 phase times (s), host memory, may be null
  // return once the call is queued on the stream (no host wait at all);
  // device-side failures go to the device's status word (lap_async_status)
  bool async_call = false;
  int* status_word = nullptr;  // async: fold the outcome here instead of the device's word
};

// Waits for `st` and returns (and clears) the first failure of the
// asynchronous calls queued on this device since the last query (IER_OK,
// IER_TIMEOUT or IER_TREE_LIMIT).
int lap_async_status(cudaStream_t st);

// Runs the FMM on device pointers on stream `st`; returns an ier code.
// dens_ready (optional): an event the evaluation waits for before it reads
// the densities (they may still be arriving on another stream while the tree
// is built).
int lap_fmm_device(const LapArgs& a, cudaStream_t st, cudaEvent_t dens_ready = nullptr);

// A plan holds everything of an FMM call that depends only on the points:
// the tree and lists, the sorted points, the operator tables and every work
// buffer.  lap_plan_eval then runs the density-dependent part (gather, the
// eight FMM steps, unsort) as stream work only: no allocation, no host
// synchronisation unless `sync` is set, so it can be captured in a CUDA
// graph.  One plan must not be evaluated on two streams at the same time.
// `a` gives the geometry and flags; its charge / dipstr pointers only mark
// which densities later evaluations pass (non-null = present).
struct LapPlan;
int lap_plan_create(const LapArgs& a, cudaStream_t st, bool own_stream, LapPlan** out);
// device_ranges: the tree is not read back; the passes take their box ranges
// from its device control block (a single call on the caller's stream; the
// end-of-call check reports a tree that needs the read-back build).
int lap_plan_create(const LapArgs& a, cudaStream_t st, bool own_stream, LapPlan** out,
                    bool device_ranges);

// Single calls take their box ranges on the device (default on); off makes
// every call wait for its tree on the host and launch the passes level by
// level.
void set_device_ranges(bool on);
int lap_plan_eval(LapPlan* p, const double* charge, const double* dipstr, const double* dipvec,
                  double* pot, double* grad, double* hess, double* pottarg, double* gradtarg,
                  double* hesstarg, cudaStream_t st, bool sync, double* timeinfo);
// The same in parts, for batches whose mixed near fields run as one pass
// (p2p_batch_launch over lap_plan_near_entries): part 1 runs everything up
// to the far field of the leaves, part 2 only the unsort into the caller's
// outputs; part 0 is the whole evaluation.  Parts 1 and 2 are for plans
// with lap_plan_defers_near (IER_BADARG otherwise).
int lap_plan_eval_part(LapPlan* p, const double* charge, const double* dipstr,
                       const double* dipvec, double* pot, double* grad, double* hess,
                       double* pottarg, double* gradtarg, double* hesstarg, cudaStream_t st,
                       bool sync, double* timeinfo, int part);
bool lap_plan_defers_near(const LapPlan* p);
// The plan's deferred near-field passes (sources, targets) as batch entries
// (P2PBatchEntry: csrc/lap_mixed.cuh).
struct P2PBatchEntry;
void lap_plan_near_entries(LapPlan* p, std::vector<P2PBatchEntry>& out);
// IER_TIMEOUT when a bounded tensor-core wait of an earlier evaluation gave
// up, else IER_OK; clears the flag.  Synchronises the device.
int lap_plan_status(LapPlan* p);
void lap_plan_free(LapPlan* p);

int lap_nterms(double eps);
int lap_ndiv(double eps);

// Work counts of the last FMM run on this thread (filled when enabled with
// set_stats(true); costs one extra reduction kernel per call).
struct LapStats {
  double nboxes, nlevels, nleaves, nterms1;  // nterms1 = P = nterms + 1
  double p2p_pairs;                          // sum over leaves: evals x list-1 sources
  double m2l_pairs;                          // list-2 translations applied
  double m2p_evals;                          // points x list-3 boxes
  double p2l_sources;                        // list-4 sources applied
  double npts_eval;                          // evaluation points (sources + targets)
  double tree_ms;                            // tree + lists build time (device events)
  double fmm_ms;                             // everything after the tree
  double nd_cauchy;                          // Cauchy densities
  double m2l_tc_steps;                       // tensor-core M2L: offset steps of all tiles (0: not used)
  // device timeline of the call (ms): start -> tree start, tree, tree end ->
  // first FMM pass, FMM passes, last pass -> end of the call
  double tl_pre, tl_tree, tl_setup, tl_fmm, tl_post;
};
void set_stats(bool on);
const LapStats& last_stats();

// Device binomial table C(l, m), 0 <= m <= l < BINOM_N, row-major (BINOM_N^2).
constexpr int BINOM_N = 128;
const double* device_binomials();
// Device tables of the M2M and L2L operators of the child (+,+), each
// lower-triangular over 0 <= b <= a < BINOM_N at a (a + 1) / 2 + b: M2M
// first, L2L at + SHIFT_TAB.
constexpr int SHIFT_TAB = BINOM_N * (BINOM_N + 1) / 2;
const double2* device_shift_tables();

}  // namespace b2
