// Biharmonic and Stokes sums (src/biharmonic/bhfmm2d.f, src/stokes/stfmm2d.f)
// evaluated through the Cauchy FMM.
#pragma once
#include "common.cuh"

namespace b2 {

struct BhArgs {
  int nd = 1;
  double eps = 1e-9;
  long ns = 0;
  const double* src = nullptr;     // (2, ns)
  const double* charge = nullptr;  // complex (nd, 2, ns): c1, c2
  const double* dip = nullptr;     // complex (nd, 3, ns): d1, d2, d3
  int ifpgh = 0;                   // 1 velocity, 2 and its three derivatives
  double *pot = nullptr, *grad = nullptr;  // complex (nd, n), (nd, 3, n)
  long nt = 0;
  const double* trg = nullptr;
  int ifpghtarg = 0;
  double *pottarg = nullptr, *gradtarg = nullptr;
  bool direct = false;  // all pairs (bh2d_direct*) instead of the FMM
  double thresh = 1e-16;  // direct: pairs closer than this are skipped
  int ndiv = 0;
};

// Device pointers on stream st; blocks until the outputs are written.
int bh_device(const BhArgs& a, cudaStream_t st);

struct StArgs {
  int nd = 1;
  double eps = 1e-9;
  long ns = 0;
  const double* src = nullptr;      // (2, ns)
  const double* stoklet = nullptr;  // real (nd, 2, ns), or null
  const double* strslet = nullptr;  // real (nd, 2, ns), or null (with strsvec)
  const double* strsvec = nullptr;  // real (nd, 2, ns)
  int ifppreg = 0;                  // 1 velocity, 2 + pressure, 3 + gradient
  double *pot = nullptr, *pre = nullptr, *grad = nullptr;  // (nd,2,n), (nd,n), (nd,2,2,n)
  long nt = 0;
  const double* trg = nullptr;
  int ifppregtarg = 0;
  double *pottarg = nullptr, *pretarg = nullptr, *gradtarg = nullptr;
  bool direct = false;
  double thresh = 1e-16;
};

int stokes_device(const StArgs& a, cudaStream_t st);

}  // namespace b2
