/* libfmm2d.so: the reference library's Fortran entry points and its C
 * declaration, each a forward to the B200 library's host entry points
 * (b2fmm_cfmm2d ... b2fmm_hfmm2d_ndiv, which copy the host arrays to the
 * device, run the FMM there and copy the results back).  Declarations and
 * the calling convention: include/fmm2d_f77.h.
 *
 * The flag wrappers restate what src/laplace/lfmm2dwrap.f (and its
 * rfmm2d, cfmm2d, hfmm2d and _vec siblings) do: fix ifcharge/ifdipole from
 * the density letters, ifpgh/ifpghtarg from the output letter and the
 * s/t/st prefix (st_ sets both to the same level, e.g.
 * lfmm2dwrap.f lfmm2d_st_c_g: ifpgh = 2, ifpghtarg = 2), nd = 1 unless
 * _vec, and call the core routine.  Outputs the wrapper does not take are
 * passed as null pointers, which the core entry points accept for levels
 * below them. */
#include <complex.h>
#include <stddef.h>
#include <stdint.h>

#include "fmm2d_b200.h"
#include "fmm2d_f77.h"

enum { FAM_c, FAM_l, FAM_r, FAM_h };

static void call_core(int fam, int nd, double eps, const double* zk, int64_t ns,
                      const double* sources, int ifcharge, const double* charge, int ifdipole,
                      const double* dipstr, const double* dipvec, int ifpgh, double* pot,
                      double* grad, double* hess, int64_t nt, const double* targ, int ifpghtarg,
                      double* pottarg, double* gradtarg, double* hesstarg, int* ier) {
  switch (fam) {
    case FAM_c:
      b2fmm_cfmm2d(nd, eps, ns, sources, ifcharge, charge, ifdipole, dipstr, 0, ifpgh, pot, grad,
                   hess, nt, targ, ifpghtarg, pottarg, gradtarg, hesstarg, ier);
      break;
    case FAM_l:
      b2fmm_lfmm2d(nd, eps, ns, sources, ifcharge, charge, ifdipole, dipstr, dipvec, 0, ifpgh,
                   pot, grad, hess, nt, targ, ifpghtarg, pottarg, gradtarg, hesstarg, ier);
      break;
    case FAM_r:
      b2fmm_rfmm2d(nd, eps, ns, sources, ifcharge, charge, ifdipole, dipstr, dipvec, 0, ifpgh,
                   pot, grad, hess, nt, targ, ifpghtarg, pottarg, gradtarg, hesstarg, ier);
      break;
    default:
      b2fmm_hfmm2d(nd, eps, zk[0], zk[1], ns, sources, ifcharge, charge, ifdipole, dipstr,
                   dipvec, 0, ifpgh, pot, grad, hess, nt, targ, ifpghtarg, pottarg, gradtarg,
                   hesstarg, ier);
      break;
  }
}

/* ------------------------------------------------------------ core routines */

void cfmm2d_(const int* nd, const double* eps, const int* ns, const double* sources,
             const int* ifcharge, const double* charge, const int* ifdipole, const double* dipstr,
             const int* iper, const int* ifpgh, double* pot, double* grad, double* hess,
             const int* nt, const double* targ, const int* ifpghtarg, double* pottarg,
             double* gradtarg, double* hesstarg, int* ier) {
  (void)iper;
  b2fmm_cfmm2d(*nd, *eps, *ns, sources, *ifcharge, charge, *ifdipole, dipstr, 0, *ifpgh, pot,
               grad, hess, *nt, targ, *ifpghtarg, pottarg, gradtarg, hesstarg, ier);
}

void lfmm2d_(const int* nd, const double* eps, const int* ns, const double* sources,
             const int* ifcharge, const double* charge, const int* ifdipole, const double* dipstr,
             const double* dipvec, const int* iper, const int* ifpgh, double* pot, double* grad,
             double* hess, const int* nt, const double* targ, const int* ifpghtarg,
             double* pottarg, double* gradtarg, double* hesstarg, int* ier) {
  (void)iper;
  b2fmm_lfmm2d(*nd, *eps, *ns, sources, *ifcharge, charge, *ifdipole, dipstr, dipvec, 0, *ifpgh,
               pot, grad, hess, *nt, targ, *ifpghtarg, pottarg, gradtarg, hesstarg, ier);
}

void rfmm2d_(const int* nd, const double* eps, const int* ns, const double* sources,
             const int* ifcharge, const double* charge, const int* ifdipole, const double* dipstr,
             const double* dipvec, const int* iper, const int* ifpgh, double* pot, double* grad,
             double* hess, const int* nt, const double* targ, const int* ifpghtarg,
             double* pottarg, double* gradtarg, double* hesstarg, int* ier) {
  (void)iper;
  b2fmm_rfmm2d(*nd, *eps, *ns, sources, *ifcharge, charge, *ifdipole, dipstr, dipvec, 0, *ifpgh,
               pot, grad, hess, *nt, targ, *ifpghtarg, pottarg, gradtarg, hesstarg, ier);
}

void hfmm2d_(const int* nd, const double* eps, const double* zk, const int* ns,
             const double* sources, const int* ifcharge, const double* charge,
             const int* ifdipole, const double* dipstr, const double* dipvec, const int* iper,
             const int* ifpgh, double* pot, double* grad, double* hess, const int* nt,
             const double* targ, const int* ifpghtarg, double* pottarg, double* gradtarg,
             double* hesstarg, int* ier) {
  (void)iper;
  b2fmm_hfmm2d(*nd, *eps, zk[0], zk[1], *ns, sources, *ifcharge, charge, *ifdipole, dipstr,
               dipvec, 0, *ifpgh, pot, grad, hess, *nt, targ, *ifpghtarg, pottarg, gradtarg,
               hesstarg, ier);
}

void cfmm2d_ndiv_(const int* nd, const double* eps, const int* ns, const double* sources,
                  const int* ifcharge, const double* charge, const int* ifdipole,
                  const double* dipstr, const int* iper, const int* ifpgh, double* pot,
                  double* grad, double* hess, const int* nt, const double* targ,
                  const int* ifpghtarg, double* pottarg, double* gradtarg, double* hesstarg,
                  const int* ndiv, const int* idivflag, const int* ifnear, double* timeinfo,
                  int* ier) {
  (void)iper;
  b2fmm_cfmm2d_ndiv(*nd, *eps, *ns, sources, *ifcharge, charge, *ifdipole, dipstr, 0, *ifpgh,
                    pot, grad, hess, *nt, targ, *ifpghtarg, pottarg, gradtarg, hesstarg, *ndiv,
                    *idivflag, *ifnear, timeinfo, ier);
}

void lfmm2d_ndiv_(const int* nd, const double* eps, const int* ns, const double* sources,
                  const int* ifcharge, const double* charge, const int* ifdipole,
                  const double* dipstr, const double* dipvec, const int* iper, const int* ifpgh,
                  double* pot, double* grad, double* hess, const int* nt, const double* targ,
                  const int* ifpghtarg, double* pottarg, double* gradtarg, double* hesstarg,
                  const int* ndiv, const int* idivflag, const int* ifnear, double* timeinfo,
                  int* ier) {
  (void)iper;
  b2fmm_lfmm2d_ndiv(*nd, *eps, *ns, sources, *ifcharge, charge, *ifdipole, dipstr, dipvec, 0,
                    *ifpgh, pot, grad, hess, *nt, targ, *ifpghtarg, pottarg, gradtarg, hesstarg,
                    *ndiv, *idivflag, *ifnear, timeinfo, ier);
}

void rfmm2d_ndiv_(const int* nd, const double* eps, const int* ns, const double* sources,
                  const int* ifcharge, const double* charge, const int* ifdipole,
                  const double* dipstr, const double* dipvec, const int* iper, const int* ifpgh,
                  double* pot, double* grad, double* hess, const int* nt, const double* targ,
                  const int* ifpghtarg, double* pottarg, double* gradtarg, double* hesstarg,
                  const int* ndiv, const int* idivflag, const int* ifnear, double* timeinfo,
                  int* ier) {
  (void)iper;
  b2fmm_rfmm2d_ndiv(*nd, *eps, *ns, sources, *ifcharge, charge, *ifdipole, dipstr, dipvec, 0,
                    *ifpgh, pot, grad, hess, *nt, targ, *ifpghtarg, pottarg, gradtarg, hesstarg,
                    *ndiv, *idivflag, *ifnear, timeinfo, ier);
}

void hfmm2d_ndiv_(const int* nd, const double* eps, const double* zk, const int* ns,
                  const double* sources, const int* ifcharge, const double* charge,
                  const int* ifdipole, const double* dipstr, const double* dipvec,
                  const int* iper, const int* ifpgh, double* pot, double* grad, double* hess,
                  const int* nt, const double* targ, const int* ifpghtarg, double* pottarg,
                  double* gradtarg, double* hesstarg, const int* ndiv, const int* idivflag,
                  const int* ifnear, double* timeinfo, int* ier) {
  (void)iper;
  b2fmm_hfmm2d_ndiv(*nd, *eps, zk[0], zk[1], *ns, sources, *ifcharge, charge, *ifdipole, dipstr,
                    dipvec, 0, *ifpgh, pot, grad, hess, *nt, targ, *ifpghtarg, pottarg, gradtarg,
                    hesstarg, *ndiv, *idivflag, *ifnear, timeinfo, ier);
}

void hfmm2d_mps_(const int* nd, const double* eps, const double* zk, const int* nmpole,
                 const double* cmpole, const double* rmpole, const int* mterms, const int* ntot,
                 const double* mpole, const int* impole, double* local, int* ier) {
  b2fmm_hfmm2d_mps(*nd, *eps, zk[0], zk[1], *nmpole, cmpole, rmpole, mterms, *ntot, mpole,
                   impole, local, ier);
}

void bhfmm2d_(const int* nd, const double* eps, const int* ns, const double* sources,
              const int* ifcharge, const double* charge, const int* ifdipole, const double* dip,
              const int* iper, const int* ifpgh, double* pot, double* grad, double* hess,
              const int* nt, const double* targ, const int* ifpghtarg, double* pottarg,
              double* gradtarg, double* hesstarg, int* ier) {
  b2fmm_bhfmm2d(*nd, *eps, *ns, sources, *ifcharge, charge, *ifdipole, dip, *iper, *ifpgh, pot,
                grad, hess, *nt, targ, *ifpghtarg, pottarg, gradtarg, hesstarg, ier);
}

void stfmm2d_(const int* nd, const double* eps, const int* nsource, const double* source,
              const int* ifstoklet, const double* stoklet, const int* ifstrslet,
              const double* strslet, const double* strsvec, const int* ifppreg, double* pot,
              double* pre, double* grad, const int* ntarg, const double* targ,
              const int* ifppregtarg, double* pottarg, double* pretarg, double* gradtarg,
              int* ier) {
  b2fmm_stfmm2d(*nd, *eps, *nsource, source, *ifstoklet, stoklet, *ifstrslet, strslet, strsvec,
                *ifppreg, pot, pre, grad, *ntarg, targ, *ifppregtarg, pottarg, pretarg, gradtarg,
                ier);
}

/* ------------------------------------------------------------ flag wrappers */

#define ZK_c NULL
#define ZK_l NULL
#define ZK_r NULL
#define ZK_h zk
#define IFC_c 1
#define IFC_d 0
#define IFC_cd 1
#define IFD_c 0
#define IFD_d 1
#define IFD_cd 1
#define Q_c charge
#define Q_d NULL
#define Q_cd charge
#define DS_c NULL
#define DS_d dipstr
#define DS_cd dipstr
#define DV_c_c NULL
#define DV_c_d NULL
#define DV_c_cd NULL
#define DV_l_c NULL
#define DV_l_d dipvec
#define DV_l_cd dipvec
#define DV_r_c NULL
#define DV_r_d dipvec
#define DV_r_cd dipvec
#define DV_h_c NULL
#define DV_h_d dipvec
#define DV_h_cd dipvec
#define LVL_p 1
#define LVL_g 2
#define LVL_h 3
#define OS_p pot, NULL, NULL
#define OS_g pot, grad, NULL
#define OS_h pot, grad, hess
#define OT_p pottarg, NULL, NULL
#define OT_g pottarg, gradtarg, NULL
#define OT_h pottarg, gradtarg, hesstarg
#define NONE3 NULL, NULL, NULL

#define DENS(F, D) IFC_##D, Q_##D, IFD_##D, DS_##D, DV_##F##_##D
#define CALL_s(F, D, O)                                                                      \
  call_core(FAM_##F, nd, *eps, ZK_##F, *ns, sources, DENS(F, D), LVL_##O, OS_##O, 0, NULL, 0, \
            NONE3, ier)
#define CALL_t(F, D, O)                                                                         \
  call_core(FAM_##F, nd, *eps, ZK_##F, *ns, sources, DENS(F, D), 0, NONE3, *nt, targ, LVL_##O, \
            OT_##O, ier)
#define CALL_st(F, D, O)                                                                   \
  call_core(FAM_##F, nd, *eps, ZK_##F, *ns, sources, DENS(F, D), LVL_##O, OS_##O, *nt, targ, \
            LVL_##O, OT_##O, ier)

#define DEFINE(F, K, D, O)                                                          \
  void F##fmm2d_##K##_##D##_##O##_(B2F77_SIG_##K(F, D, O)) {                        \
    const int nd = 1;                                                               \
    CALL_##K(F, D, O);                                                              \
  }                                                                                 \
  void F##fmm2d_##K##_##D##_##O##_vec_(const int* ndp, B2F77_SIG_##K(F, D, O)) {    \
    const int nd = *ndp;                                                            \
    CALL_##K(F, D, O);                                                              \
  }

B2F77_EACH(DEFINE, c)
B2F77_EACH(DEFINE, l)
B2F77_EACH(DEFINE, r)
B2F77_EACH(DEFINE, h)

/* ------------------------------------------------------------ C declaration */

void hfmm2d_s_c_p(double eps, double _Complex zk, int64_t ns, double const* sources,
                  double _Complex const* charge, double _Complex* pot, int64_t* ier) {
  const double z[2] = {creal(zk), cimag(zk)};
  int ierr = 0;
  call_core(FAM_h, 1, eps, z, ns, sources, 1, (const double*)charge, 0, NULL, NULL, 1,
            (double*)pot, NULL, NULL, 0, NULL, 0, NONE3, &ierr);
  *ier = ierr;
}
