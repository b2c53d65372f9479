// Helmholtz FMM engine (src/helmholtz/hfmm2d.f, wideband levels included).
#pragma once
#include "common.cuh"

namespace b2 {

struct HelmArgs {
  int nd = 1;
  double eps = 1e-9;
  double zkr = 1.0, zki = 0.0;  // zk
  long ns = 0;
  const double* src = nullptr;     // (2, ns)
  const double* charge = nullptr;  // complex (nd, ns)
  const double* dipstr = nullptr;  // complex (nd, ns)
  const double* dipvec = nullptr;  // (nd, 2, ns)
  int ifpgh = 0;
  double *pot = nullptr, *grad = nullptr, *hess = nullptr;  // complex (nd,n),(nd,2,n),(nd,3,n)
  long nt = 0;
  const double* trg = nullptr;
  int ifpghtarg = 0;
  double *pottarg = nullptr, *gradtarg = nullptr, *hesstarg = nullptr;
  int ndiv = 0;
  int ifnear = 1;
  double* timeinfo = nullptr;
};

// ier: 0 ok, 13 expansion order too large (or one the kernels do not
// support: above 63 with a scale below 1, a signature above 7000 points).
int helm_fmm_device(const HelmArgs& a, cudaStream_t st);

// All-pairs Helmholtz sums (h2d_direct*, src/helmholtz/helmkernels2d.f).
int helm_direct_device(int nd, double zkr, double zki, long ns, const double* src,
                       const double* charge, const double* dipstr, const double* dipvec, long nt,
                       const double* trg, int ifpgh, double* pot, double* grad, double* hess,
                       double thresh, cudaStream_t st);

// FMM over multipole expansions (hfmm2d_mps, src/helmholtz/hfmm2d_mps.f:19-286):
// the local expansion at each of nc centres due to all the other
// expansions.  Device pointers: centers (2, nc), rscales (nc), mterms (nc),
// impole (nc, 1-based offsets into the complex arrays as in the
// reference), mpole and local complex (ntot); expansion i is the (nd,
// -m..m) block at impole(i), m = mterms(i) <= max_mterms.  ier 13 when
// max_mterms exceeds the supported order (63).
int helm_mps_device(int nd, double eps, double zkr, double zki, long nc, const double* centers,
                    const double* rscales, const int* mterms, const int* impole, long ntot,
                    const double* mpole, double* local, int max_mterms, cudaStream_t st);

// Expansion order of a box of size bsize (h2dterms, src/helmholtz/h2dterms.f:35-97).
int helm_nterms(double bsize, double zkr, double zki, double eps, int* ier);

}  // namespace b2
