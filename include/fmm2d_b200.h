/*
 * fmm2d_b200 -- C ABI of the B200 (sm_100a) implementation of the fmm2d FMM
 * evaluation path.  Every entry point replaces one routine of the reference
 * (flatironinstitute/fmm2d); the citation above each declaration names it.
 *
 * Conventions (same as the reference's Fortran arrays):
 *   sources(2,ns), targ(2,nt)          : x/y interleaved doubles
 *   complex arrays                     : interleaved (re, im) doubles
 *   charge/dipstr/pot/grad/hess (nd,n) : density index fastest
 *   lfmm2d/rfmm2d grad (nd,2,n), hess (nd,3,n); dipvec (nd,2,n)
 *   cfmm2d grad = d/dz, hess = d2/dz2, both (nd,n) complex
 * Host entry points take host pointers and block until the results are in
 * the caller's arrays.  The `_dev` entry points take device pointers, run on
 * the given CUDA stream (NULL = legacy default stream) and return after the
 * stream has finished the call.
 * ier: 0 ok, 4 device allocation failure, 13 expansion order too large,
 *      100 invalid argument (a non-finite coordinate included), 101 CUDA
 *      error, 102 a bounded device wait gave up, 103 problem larger than a
 *      fixed static scratch array, 104 (asynchronous calls) the tree needs a
 *      synchronous call.
 */
#ifndef FMM2D_B200_H
#define FMM2D_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Tuning knobs of the *_ndiv drivers (src/laplace/cfmm2d_ndiv.f:23-26) plus
 * the arithmetic mode. */
typedef struct b2fmm_options {
  int ndiv;      /* leaf capacity; <= 0 selects the lndiv2d/hndiv2d table  */
  int idivflag;  /* 0: subdivide on sources, 1: targets, 2: max of both    */
  int ifnear;    /* 1: include list-1 near field (P2P), 0: far field only  */
  int precision; /* 0 auto (mixed when eps >= 1e-6), 1 FP64, 2 mixed        */
  int async_call; /* b2fmm_{c,l,r}fmm2d_dev only (no counterpart in the
                     reference): 1 returns once the whole call is queued on
                     the stream, with no host wait; device-side failures are
                     reported by b2fmm_async_status.  Ignored (synchronous)
                     when timeinfo or statistics are requested. */
  double level_balance; /* Laplace only (no counterpart in the reference):
                     0 keeps the leaf capacity ndiv at every level; otherwise
                     a box of level l is split above ndiv 2^(b (lp - l))
                     points (rounded, at least 1), lp the level whose boxes
                     hold ndiv points of a uniform cloud of the counted
                     points: b > 0 lets leaves above lp hold more points and
                     splits boxes below it sooner, b < 0 the reverse. */
} b2fmm_options;

/* Library version string. */
const char* b2fmm_version(void);

/* ---------------------------------------------------------------- Laplace */

/* cfmm2d: src/laplace/cfmm2d.f:23-26 (Cauchy kernel, complex densities). */
void b2fmm_cfmm2d(int nd, double eps, int64_t ns, const double* sources, int ifcharge,
                  const double* charge, int ifdipole, const double* dipstr, int iper, int ifpgh,
                  double* pot, double* grad, double* hess, int64_t nt, const double* targ,
                  int ifpghtarg, double* pottarg, double* gradtarg, double* hesstarg, int* ier);

/* lfmm2d: src/laplace/lfmm2d.f:29-32 (complex Laplace, dipvec orientations). */
void b2fmm_lfmm2d(int nd, double eps, int64_t ns, const double* sources, int ifcharge,
                  const double* charge, int ifdipole, const double* dipstr, const double* dipvec,
                  int iper, int ifpgh, double* pot, double* grad, double* hess, int64_t nt,
                  const double* targ, int ifpghtarg, double* pottarg, double* gradtarg,
                  double* hesstarg, int* ier);

/* rfmm2d: src/laplace/rfmm2d.f:27-30 (real densities, real outputs). */
void b2fmm_rfmm2d(int nd, double eps, int64_t ns, const double* sources, int ifcharge,
                  const double* charge, int ifdipole, const double* dipstr, const double* dipvec,
                  int iper, int ifpgh, double* pot, double* grad, double* hess, int64_t nt,
                  const double* targ, int ifpghtarg, double* pottarg, double* gradtarg,
                  double* hesstarg, int* ier);

/* cfmm2d_ndiv / lfmm2d_ndiv / rfmm2d_ndiv: src/laplace/cfmm2d_ndiv.f:23-26,
 * lfmm2d_ndiv.f:29, rfmm2d_ndiv.f:27.  timeinfo[8] receives the per-step
 * device times in seconds (P2M, P2L, M2M, M2L, L2L, M2P, L2P, P2P; the
 * fused leaf kernel reports M2P+L2P+P2P in slot 8). */
void b2fmm_cfmm2d_ndiv(int nd, double eps, int64_t ns, const double* sources, int ifcharge,
                       const double* charge, int ifdipole, const double* dipstr, int iper,
                       int ifpgh, double* pot, double* grad, double* hess, int64_t nt,
                       const double* targ, int ifpghtarg, double* pottarg, double* gradtarg,
                       double* hesstarg, int ndiv, int idivflag, int ifnear, double* timeinfo,
                       int* ier);
void b2fmm_lfmm2d_ndiv(int nd, double eps, int64_t ns, const double* sources, int ifcharge,
                       const double* charge, int ifdipole, const double* dipstr,
                       const double* dipvec, int iper, int ifpgh, double* pot, double* grad,
                       double* hess, int64_t nt, const double* targ, int ifpghtarg,
                       double* pottarg, double* gradtarg, double* hesstarg, int ndiv,
                       int idivflag, int ifnear, double* timeinfo, int* ier);
void b2fmm_rfmm2d_ndiv(int nd, double eps, int64_t ns, const double* sources, int ifcharge,
                       const double* charge, int ifdipole, const double* dipstr,
                       const double* dipvec, int iper, int ifpgh, double* pot, double* grad,
                       double* hess, int64_t nt, const double* targ, int ifpghtarg,
                       double* pottarg, double* gradtarg, double* hesstarg, int ndiv,
                       int idivflag, int ifnear, double* timeinfo, int* ier);

/* Host-pointer variants with options and per-step timings (no reference
 * counterpart beyond the *_ndiv drivers; used by the python front end). */
void b2fmm_cfmm2d_ex(int nd, double eps, int64_t ns, const double* sources, int ifcharge,
                     const double* charge, int ifdipole, const double* dipstr, int ifpgh,
                     double* pot, double* grad, double* hess, int64_t nt, const double* targ,
                     int ifpghtarg, double* pottarg, double* gradtarg, double* hesstarg,
                     const b2fmm_options* opts, double* timeinfo, int* ier);
void b2fmm_lfmm2d_ex(int nd, double eps, int64_t ns, const double* sources, int ifcharge,
                     const double* charge, int ifdipole, const double* dipstr,
                     const double* dipvec, int ifpgh, double* pot, double* grad, double* hess,
                     int64_t nt, const double* targ, int ifpghtarg, double* pottarg,
                     double* gradtarg, double* hesstarg, const b2fmm_options* opts,
                     double* timeinfo, int* ier);
void b2fmm_rfmm2d_ex(int nd, double eps, int64_t ns, const double* sources, int ifcharge,
                     const double* charge, int ifdipole, const double* dipstr,
                     const double* dipvec, int ifpgh, double* pot, double* grad, double* hess,
                     int64_t nt, const double* targ, int ifpghtarg, double* pottarg,
                     double* gradtarg, double* hesstarg, const b2fmm_options* opts,
                     double* timeinfo, int* ier);

/* Host-pointer calls that return once queued (no counterpart in the
 * reference, whose calls are all blocking): the copies in, the FMM and the
 * copies back are enqueued on `stream` and the call returns; the results are
 * in the host arrays once the stream has finished (b2fmm_async_status waits
 * for it and returns the first failure, 104 meaning the call's tree needed
 * the synchronous build: repeat it with b2fmm_{c,l,r}fmm2d_ex).  The host
 * arrays must stay valid until then and should be pinned (page-locked), or
 * the copies run synchronously.  Calls on different streams overlap: one
 * call's copies with another's FMM.  Same arguments as the _ex calls,
 * without timeinfo. */
void b2fmm_cfmm2d_host_async(int nd, double eps, int64_t ns, const double* sources,
                             int ifcharge, const double* charge, int ifdipole,
                             const double* dipstr, int ifpgh, double* pot, double* grad,
                             double* hess, int64_t nt, const double* targ, int ifpghtarg,
                             double* pottarg, double* gradtarg, double* hesstarg,
                             const b2fmm_options* opts, void* stream, int* ier);
void b2fmm_lfmm2d_host_async(int nd, double eps, int64_t ns, const double* sources,
                             int ifcharge, const double* charge, int ifdipole,
                             const double* dipstr, const double* dipvec, int ifpgh, double* pot,
                             double* grad, double* hess, int64_t nt, const double* targ,
                             int ifpghtarg, double* pottarg, double* gradtarg, double* hesstarg,
                             const b2fmm_options* opts, void* stream, int* ier);
void b2fmm_rfmm2d_host_async(int nd, double eps, int64_t ns, const double* sources,
                             int ifcharge, const double* charge, int ifdipole,
                             const double* dipstr, const double* dipvec, int ifpgh, double* pot,
                             double* grad, double* hess, int64_t nt, const double* targ,
                             int ifpghtarg, double* pottarg, double* gradtarg, double* hesstarg,
                             const b2fmm_options* opts, void* stream, int* ier);

/* Device-pointer variants of cfmm2d / lfmm2d / rfmm2d (same argument meaning;
 * opts may be NULL for the reference defaults; timeinfo may be NULL). */
void b2fmm_cfmm2d_dev(int nd, double eps, int64_t ns, const double* sources, int ifcharge,
                      const double* charge, int ifdipole, const double* dipstr, int ifpgh,
                      double* pot, double* grad, double* hess, int64_t nt, const double* targ,
                      int ifpghtarg, double* pottarg, double* gradtarg, double* hesstarg,
                      const b2fmm_options* opts, double* timeinfo, void* stream, int* ier);
void b2fmm_lfmm2d_dev(int nd, double eps, int64_t ns, const double* sources, int ifcharge,
                      const double* charge, int ifdipole, const double* dipstr,
                      const double* dipvec, int ifpgh, double* pot, double* grad, double* hess,
                      int64_t nt, const double* targ, int ifpghtarg, double* pottarg,
                      double* gradtarg, double* hesstarg, const b2fmm_options* opts,
                      double* timeinfo, void* stream, int* ier);
void b2fmm_rfmm2d_dev(int nd, double eps, int64_t ns, const double* sources, int ifcharge,
                      const double* charge, int ifdipole, const double* dipstr,
                      const double* dipvec, int ifpgh, double* pot, double* grad, double* hess,
                      int64_t nt, const double* targ, int ifpghtarg, double* pottarg,
                      double* gradtarg, double* hesstarg, const b2fmm_options* opts,
                      double* timeinfo, void* stream, int* ier);

/* Direct sums on the device (the python API's c2ddir / l2ddir / r2ddir:
 * python/fmm2dpy/fmm2d.py:1493-1740 over src/laplace/cauchykernels2d.f,
 * lapkernels2d.f, rlapkernels2d.f).  Outputs are overwritten.  kind selects
 * the kernel: 0 Cauchy, 1 complex Laplace, 2 real Laplace. */
void b2fmm_lap_direct_dev(int kind, int nd, int64_t ns, const double* sources,
                          const double* charge, const double* dipstr, const double* dipvec,
                          int64_t nt, const double* targ, int ifpgh, double* pot, double* grad,
                          double* hess, double thresh, void* stream, int* ier);

/* Allocation-free variant of b2fmm_lap_direct_dev.  This entry point has no
 * counterpart in the reference.  It is for callers that cannot allocate
 * device memory during the call (a device already reserved by another
 * framework's allocator, latency-critical loops, fixed memory plans): it
 * calls no cudaMalloc/cudaFree or allocating library routine and takes its
 * scratch from a 4 MiB static device array instead, which every GPU that
 * loads the library holds until exit.  Limit: nt*3 (kind 0) or nt*6
 * (kinds 1, 2) <= 262144, i.e. at most 87381 / 43690 targets per call;
 * larger nt returns ier = 103 without computing.  The first call on a device
 * looks up the array's device address, so make it before the device's memory
 * is handed to another allocator: with lazy
 * module loading that look-up may be what reserves the array (ier = 4 when
 * the device has no room left; CUDA_MODULE_LOADING=EAGER reserves it at
 * load).  All calls share the array: calls that overlap on the GPU race on
 * it and must be serialised by the caller. */
void b2fmm_lap_direct_noalloc_dev(int kind, int nd, int64_t ns, const double* sources,
                                  const double* charge, const double* dipstr,
                                  const double* dipvec, int64_t nt, const double* targ,
                                  int ifpgh, double* pot, double* grad, double* hess,
                                  double thresh, void* stream, int* ier);

/* -------------------------------------------------------------- Helmholtz */

/* hfmm2d: src/helmholtz/hfmm2d.f:19-22.  zk is passed as (zk_re, zk_im);
 * charge, dipstr and all outputs are complex, grad (nd,2,n), hess (nd,3,n),
 * dipvec (nd,2,n) real.  Levels whose boxes exceed 16 wavelengths
 * (hfmm2d.f:1001-1013) translate in the diagonal (signature) form of
 * src/helmholtz/wideband2d.f. */
void b2fmm_hfmm2d(int nd, double eps, double zk_re, double zk_im, int64_t ns,
                  const double* sources, int ifcharge, const double* charge, int ifdipole,
                  const double* dipstr, const double* dipvec, int iper, int ifpgh, double* pot,
                  double* grad, double* hess, int64_t nt, const double* targ, int ifpghtarg,
                  double* pottarg, double* gradtarg, double* hesstarg, int* ier);

/* hfmm2d_ndiv: src/helmholtz/hfmm2d_ndiv.f:19-22 (idivflag is accepted and
 * ignored, as hfmm2dmain always subdivides on sources). */
void b2fmm_hfmm2d_ndiv(int nd, double eps, double zk_re, double zk_im, int64_t ns,
                       const double* sources, int ifcharge, const double* charge, int ifdipole,
                       const double* dipstr, const double* dipvec, int iper, int ifpgh,
                       double* pot, double* grad, double* hess, int64_t nt, const double* targ,
                       int ifpghtarg, double* pottarg, double* gradtarg, double* hesstarg,
                       int ndiv, int idivflag, int ifnear, double* timeinfo, int* ier);

/* Device-pointer hfmm2d (FP64; opts->precision is ignored). */
void b2fmm_hfmm2d_dev(int nd, double eps, double zk_re, double zk_im, int64_t ns,
                      const double* sources, int ifcharge, const double* charge, int ifdipole,
                      const double* dipstr, const double* dipvec, int ifpgh, double* pot,
                      double* grad, double* hess, int64_t nt, const double* targ, int ifpghtarg,
                      double* pottarg, double* gradtarg, double* hesstarg,
                      const b2fmm_options* opts, double* timeinfo, void* stream, int* ier);

/* ------------------------------------------------- biharmonic and Stokes */

/* bhfmm2d: src/biharmonic/bhfmm2d.f:1-4.  Host arrays: charge complex
 * (nd,2,ns) = (c1, c2), dip complex (nd,3,ns) = (d1, d2, d3); pot complex
 * (nd,n), grad complex (nd,3,n) (d/dz, its conj(z) part, d/dconj(z)); the
 * kernel of bhkernels2d.f bh2d_directcdg.  hess and hesstarg are not
 * computed (as in the reference).  Runs as one FP64 Cauchy FMM over 4 nd
 * densities. */
void b2fmm_bhfmm2d(int nd, double eps, int64_t ns, const double* sources, int ifcharge,
                   const double* charge, int ifdipole, const double* dip, int iper, int ifpgh,
                   double* pot, double* grad, double* hess, int64_t nt, const double* targ,
                   int ifpghtarg, double* pottarg, double* gradtarg, double* hesstarg, int* ier);

/* Device-pointer form of b2fmm_bhfmm2d on `stream` (blocking). */
void b2fmm_bhfmm2d_dev(int nd, double eps, int64_t ns, const double* sources, int ifcharge,
                       const double* charge, int ifdipole, const double* dip, int ifpgh,
                       double* pot, double* grad, int64_t nt, const double* targ, int ifpghtarg,
                       double* pottarg, double* gradtarg, void* stream, int* ier);

/* All-pairs biharmonic sums at nt targets (bh2ddir of the python API,
 * bhkernels2d.f bh2d_direct*); charge or dip may be null; pairs closer than
 * thresh are skipped. */
void b2fmm_bh2ddir_dev(int nd, int64_t ns, const double* sources, const double* charge,
                       const double* dip, int64_t nt, const double* targ, int ifpgh, double* pot,
                       double* grad, double thresh, void* stream, int* ier);

/* stfmm2d: src/stokes/stfmm2d.f:3-7.  Host arrays: stoklet, strslet,
 * strsvec real (nd,2,ns); pot (nd,2,n), pre (nd,n), grad (nd,2,2,n) real;
 * ifppreg 1 velocity, 2 + pressure, 3 + velocity gradient. */
void b2fmm_stfmm2d(int nd, double eps, int64_t ns, const double* sources, int ifstoklet,
                   const double* stoklet, int ifstrslet, const double* strslet,
                   const double* strsvec, int ifppreg, double* pot, double* pre, double* grad,
                   int64_t nt, const double* targ, int ifppregtarg, double* pottarg,
                   double* pretarg, double* gradtarg, int* ier);

/* Device-pointer form of b2fmm_stfmm2d on `stream` (blocking). */
void b2fmm_stfmm2d_dev(int nd, double eps, int64_t ns, const double* sources, int ifstoklet,
                       const double* stoklet, int ifstrslet, const double* strslet,
                       const double* strsvec, int ifppreg, double* pot, double* pre, double* grad,
                       int64_t nt, const double* targ, int ifppregtarg, double* pottarg,
                       double* pretarg, double* gradtarg, void* stream, int* ier);

/* All-pairs Stokes sums at nt targets (st2ddir of the python API,
 * src/stokes/stokkernels2d.f st2ddirectstokstrsg). */
void b2fmm_st2ddir_dev(int nd, int64_t ns, const double* sources, int ifstoklet,
                       const double* stoklet, int ifstrslet, const double* strslet,
                       const double* strsvec, int64_t nt, const double* targ, int ifppreg,
                       double* pot, double* pre, double* grad, double thresh, void* stream,
                       int* ier);

/* hfmm2d_mps: src/helmholtz/hfmm2d_mps.f:19-22.  Host arrays: cmpole (2,
 * nmpole), rmpole (nmpole), mterms (nmpole), impole (nmpole, 1-based
 * offsets into the complex arrays), mpole and local complex (ntot).
 * Expansion i is the (nd, -m..m) block at impole(i) with m = mterms(i) <= 63.
 * On return local holds, at each block, the local expansion about that
 * centre due to all the other expansions.  ier 100 when a block lies
 * outside ntot, 13 for an order above 63. */
void b2fmm_hfmm2d_mps(int nd, double eps, double zk_re, double zk_im, int64_t nmpole,
                      const double* cmpole, const double* rmpole, const int* mterms,
                      int64_t ntot, const double* mpole, const int* impole, double* local,
                      int* ier);

/* h2d_direct{c,d,cd}{p,g,h}: src/helmholtz/helmkernels2d.f:3-904.  Device
 * pointers; charge / dipstr NULL when absent; pairs with |zk r| < thresh
 * (<= for the charge potential-only kernel) are skipped.  Outputs are
 * overwritten (the reference adds into them). */
void b2fmm_h2ddir_dev(int nd, double zk_re, double zk_im, int64_t ns, const double* sources,
                      const double* charge, const double* dipstr, const double* dipvec,
                      int64_t nt, const double* targ, int ifpgh, double* pot, double* grad,
                      double* hess, double thresh, void* stream, int* ier);

/* h2dterms: src/helmholtz/h2dterms.f:35-97 (expansion order of a box). */
int b2fmm_h2dterms(double bsize, double zk_re, double zk_im, double eps, int* ier);

/* Host evaluation of the special functions the Helmholtz kernels use (the
 * same source is compiled for the device): kind 0 writes H0, H1 of z
 * (hank103, src/common/hank103.f:116) as 4 doubles; kind 1 writes
 * J_k(z)/rscale^k, k = 0..n (jbessel2d, src/common/cdjseval2d.f:5-204);
 * kind 2 writes H_k(z) rscale^k (h2dall, src/helmholtz/h2dcommon.f:71-178).
 * out holds 2(n+1) doubles for kinds 1 and 2. */
void b2fmm_helm_special(int kind, int n, double z_re, double z_im, double rscale, double* out);

/* ------------------------------------------- plans and batches (no reference counterpart) */

/* A plan is the point-dependent part of a Laplace / Cauchy FMM call (fe: 0
 * cfmm2d, 1 lfmm2d, 2 rfmm2d): tree, lists, sorted points and every work
 * buffer, built once for fixed sources / targets / flags (the reference
 * rebuilds them in every call of cfmm2d.f:23-436).  Device pointers;
 * ifcharge / ifdipole fix which densities the evaluations pass.  The plan
 * has its own stream; NULL is returned (and *ier set) on error. */
void* b2fmm_plan_create(int fe, int nd, double eps, int64_t ns, const double* sources,
                        int ifcharge, int ifdipole, int ifpgh, int64_t nt, const double* targ,
                        int ifpghtarg, const b2fmm_options* opts, void* stream, int* ier);

/* Enqueue one evaluation of a plan for new densities on `stream` (device
 * pointers, the layouts of the matching b2fmm_*fmm2d_dev call).  Stream work
 * only: no allocation and no host synchronisation, so it may be captured in a
 * CUDA graph; *ier reports argument errors.  A plan must not run on two
 * streams at once. */
void b2fmm_plan_eval(void* plan, const double* charge, const double* dipstr, const double* dipvec,
                     double* pot, double* grad, double* hess, double* pottarg, double* gradtarg,
                     double* hesstarg, void* stream, int* ier);

/* Synchronises the device; 102 if a bounded tensor-core wait of an earlier
 * evaluation gave up (clears the flag), else 0. */
int b2fmm_plan_status(void* plan);
void b2fmm_plan_free(void* plan);

/* One CUDA graph holding one evaluation of each of n plans, spread over
 * nbranch concurrent branches.  The arrays hold one device pointer per plan
 * (NULL array = argument absent for all).  Every plan is evaluated once,
 * synchronously, before the capture.  Plans and pointers must outlive the
 * graph. */
void* b2fmm_batch_graph_create(int n, void* const* plans, const double* const* charge,
                               const double* const* dipstr, const double* const* dipvec,
                               double* const* pot, double* const* grad, double* const* hess,
                               double* const* pottarg, double* const* gradtarg,
                               double* const* hesstarg, int nbranch, int* ier);
void b2fmm_batch_graph_launch(void* graph, void* stream, int* ier);
int b2fmm_batch_graph_status(void* graph);
int64_t b2fmm_batch_graph_nodes(void* graph);
void b2fmm_batch_graph_free(void* graph);

/* -------------------------------------- learned cost model (no reference counterpart) */

/* The reference picks the leaf size from a fixed table (lndiv2d.f:1-39);
 * these entry points carry the small MLP that predicts the FMM's time from
 * point-distribution statistics and the leaf size, with hand-written
 * forward, backward and Adam kernels.  Parameters are one flat FP32 array
 * W1 [h1][nin], b1 [h1], W2 [h2][h1], b2 [h2], w3 [h2], b3; tanh hidden
 * layers, linear output; nin <= 32, h1, h2 <= 64.  Device pointers. */
int b2fmm_mlp_param_count(int nin, int h1, int h2);
void b2fmm_mlp_forward(const float* x, int batch, int nin, int h1, int h2, const float* params,
                       float* y, void* stream, int* ier);
/* Gradient of mean_b (y_b - target_b)^2; loss (device, may be NULL). */
void b2fmm_mlp_gradient(const float* x, const float* target, int batch, int nin, int h1, int h2,
                        const float* params, float* grad, float* loss, void* stream, int* ier);
/* `steps` full-batch Adam steps in place; loss_history: host, may be NULL. */
void b2fmm_mlp_train(const float* x, const float* target, int batch, int nin, int h1, int h2,
                     float* params, int steps, float lr, float* loss_history, void* stream,
                     int* ier);
/* 128 x 128 occupancy histogram (device, row-major) of sources and targets
 * over the square that holds them, the input of the cost-model features. */
void b2fmm_point_stats(const double* sources, int64_t ns, const double* targ, int64_t nt,
                       unsigned* hist, void* stream, int* ier);

/* ------------------------------------------------ near-field tile shapes (no reference counterpart) */

/* The mixed-precision near-field kernel comes in B2FMM_P2P_SHAPES tile
 * shapes (0: 128 staged sources per warp, pair loop unrolled twice, 6 blocks
 * per SM; 1: 64 sources, twice, 8 blocks; 2: 128 sources, four times, 5
 * blocks), one chosen per leaf-size class (0: ndiv <= 20, 1: ndiv <= 56, 2:
 * larger).  Shape 0 everywhere until set; fmm2d_b200/autotune.py times the
 * shapes and the Python package applies its committed choice at load.
 * Results of different shapes agree to FP32 round-off (the staged chunk
 * bounds the FP32 partial sums).  Process-wide; set returns 0 or 100 (an
 * unknown class or shape), get returns the shape or -1. */
#define B2FMM_P2P_SHAPES 3
#define B2FMM_P2P_CLASSES 3
int b2fmm_set_p2p_shape(int leaf_class, int shape);
int b2fmm_get_p2p_shape(int leaf_class);

/* ------------------------------------------------- tensor-core M2L (no reference counterpart) */

/* Mixed-precision Laplace M2L engine switch: 1 (default) runs the list-2
 * translations (laprouts2d.f:1130-1244) as split-TF32 tcgen05 tensor-core
 * tiles; 0 runs the FP32 CUDA-core kernel.  Process-wide. */
void b2fmm_set_m2l_tensor_cores(int on);

/* Check of the tensor-core tile path: D = A B^T for A 128 x k and B n x k
 * (row-major FP32 device arrays; k in {8,16,24,32}, n in {16,32}) through the
 * same shared-memory layout, split-TF32 tcgen05.mma and tcgen05.ld read-back
 * as the M2L kernel.  D is 128 x n row-major.  ier 102 if the bounded wait
 * for the tensor cores expired. */
void b2fmm_tc_gemm_probe(const float* a_dev, const float* b_dev, int k, int n, float* d_dev,
                         void* stream, int* ier);

/* ------------------------------------------------------------------- tree */

/* Level-restricted tree and lists for (sources, targets), exported for
 * structural comparison (src/common/pts_tree2d.f:34-655 tree,
 * pts_tree2d.f:1222-1246 sort, tree_routs2d.f:486-710 lists).
 * b2fmm_tree_build returns a handle and the sizes; b2fmm_tree_get copies the
 * arrays to host memory (0-based box/point indices, -1 = none, half-open
 * point ranges; laddr (nlevels+1, 2) inclusive box ranges per level). */
void* b2fmm_tree_build(const double* sources_dev, int64_t ns, const double* targ_dev, int64_t nt,
                       int idivflag, int ndiv, int nlmax, int* nlevels, int* nboxes, int* ier);
void b2fmm_tree_get(void* tree, int* laddr, int* ilevel, int* iparent, int* nchild, int* ichild,
                    int* ncoll, int* coll, double* centers, double* boxsize, int* isrc,
                    int* isrcse, int* itarg, int* itargse, int* nlist1, int* list1, int* nlist2,
                    int* list2, int* nlist3, int* list3, int* nlist4, int* list4, int* ier);
void b2fmm_tree_free(void* tree);

/* ----------------------------------------------------------- diagnostics */
/* These have no counterpart in the reference; they serve the benchmark's
 * roofline accounting. */

/* Number of kernels this library has launched in the process. */
uint64_t b2fmm_kernel_launches(void);

/* Enable (1) / disable (0) work counting of subsequent FMM calls on this
 * thread; b2fmm_get_stats copies up to n of: nboxes, nlevels, nleaves,
 * nterms+1, P2P pairs, M2L translations, M2P evaluations, P2L sources,
 * evaluation points, tree build ms, FMM ms after the tree, Cauchy densities,
 * tensor-core M2L steps (128-row MMA steps over all super-tiles; 0 when not
 * used), then the device timeline of the call in ms: start to tree start,
 * tree, tree end to the first FMM pass, the FMM passes, last pass to the end
 * of the call. */
void b2fmm_set_stats(int on);
void b2fmm_get_stats(double* out, int n);

/* Waits for `stream` and returns in *ier the first failure of the
 * asynchronous calls (options.async_call = 1) queued on the current device
 * since the last query, then clears it: 0, 102 (a bounded device wait gave
 * up) or 104 (a call's tree needed more boxes or levels than a call without
 * read-back allows: repeat it synchronously).  No counterpart in the
 * reference, whose calls are all blocking. */
void b2fmm_async_status(void* stream, int* ier);

/* Test hooks for the error paths (no counterpart in the reference; they
 * inject failures on the host side only).  b2fmm_test_fail_alloc(k): the
 * (k+1)-th device allocation of the library from now on fails as if the
 * device were out of memory, so the call in progress returns ier = 4; k < 0
 * switches the injection off.  b2fmm_test_barrier_limit(c): later tree
 * builds give up a grid-barrier wait after c clock cycles instead of about
 * half a second, and their calls return ier = 102 (c <= 0 restores the
 * default); the device stays usable. */
void b2fmm_test_fail_alloc(int after);
void b2fmm_test_barrier_limit(long long cycles);

/* Laplace / Cauchy calls take their box ranges from the tree's device
 * level table, so the host does not wait for the tree in the middle of a
 * call (1, the default); 0 reads every tree back first and launches the
 * upward and downward passes level by level.  Results are the same. */
void b2fmm_set_device_ranges(int on);

/* Measured fused-multiply-add throughput of this GPU in flop/s (FP64 when
 * fp64 != 0, else FP32), from a dependent-free FMA loop over all SMs. */
double b2fmm_fma_peak(int fp64);

#ifdef __cplusplus
}
#endif

#endif /* FMM2D_B200_H */
