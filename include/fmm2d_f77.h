/* The reference library's own entry points (libfmm2d), served by the B200
 * library: a program built against the reference links libfmm2d.so from
 * this package instead and runs unchanged.
 *
 * Fortran ABI (gfortran): lower-case name + trailing underscore, every
 * argument by address, INTEGER = 32-bit int, COMPLEX*16 = two doubles.
 * Arrays are column-major exactly as in the reference: sources(2,ns),
 * charge/dipstr/pot(nd,n) (complex, or real for rfmm2d), dipvec(nd,2,n),
 * grad(nd,2,n) and hess(nd,3,n) (cfmm2d: grad(nd,n), hess(nd,n)).
 *
 *   core      cfmm2d_, lfmm2d_, rfmm2d_, hfmm2d_       src/laplace/cfmm2d.f:23-26,
 *             lfmm2d.f:29-32, rfmm2d.f:27-30, src/helmholtz/hfmm2d.f:19-22
 *   tuning    cfmm2d_ndiv_ ... hfmm2d_ndiv_            cfmm2d_ndiv.f:23-26 etc.
 *   sources   hfmm2d_mps_ (multipole expansions)       src/helmholtz/hfmm2d_mps.f:19-22
 *   kernels   bhfmm2d_, stfmm2d_                       src/biharmonic/bhfmm2d.f:1-4,
 *                                                      src/stokes/stfmm2d.f:3-7
 *   flags     {c,l,r,h}fmm2d_{s,t,st}_{c,d,cd}_{p,g,h}[_vec]_   (27 + 27 per family)
 *             src/laplace/{l,r,c}fmm2dwrap.f, {l,r,c}fmm2dwrap_vec.f,
 *             src/helmholtz/hfmm2dwrap.f, hfmm2dwrap_vec.f
 *   C         hfmm2d_s_c_p (by value)                  include/fmm2d/helmholtz.h:10
 *
 * Flag wrappers set the core flags as the reference's wrappers do: s_ at
 * the sources only (ifpgh = level, nt = 0), t_ at the targets only
 * (ifpgh = 0), st_ at both with the same level; c/d/cd select charges,
 * dipoles or both; p/g/h the level 1/2/3.  _vec variants take nd first.
 * Each call blocks until its results are in the caller's host arrays;
 * ier as the core routine reports it (0 ok, 4 allocation failure, 100 and
 * up the B200 library's own codes, see fmm2d_b200.h). */
#ifndef FMM2D_F77_H
#define FMM2D_F77_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- core routines */
void cfmm2d_(const int* nd, const double* eps, const int* ns, const double* sources,
             const int* ifcharge, const double* charge, const int* ifdipole, const double* dipstr,
             const int* iper, const int* ifpgh, double* pot, double* grad, double* hess,
             const int* nt, const double* targ, const int* ifpghtarg, double* pottarg,
             double* gradtarg, double* hesstarg, int* ier);
void lfmm2d_(const int* nd, const double* eps, const int* ns, const double* sources,
             const int* ifcharge, const double* charge, const int* ifdipole, const double* dipstr,
             const double* dipvec, const int* iper, const int* ifpgh, double* pot, double* grad,
             double* hess, const int* nt, const double* targ, const int* ifpghtarg,
             double* pottarg, double* gradtarg, double* hesstarg, int* ier);
void rfmm2d_(const int* nd, const double* eps, const int* ns, const double* sources,
             const int* ifcharge, const double* charge, const int* ifdipole, const double* dipstr,
             const double* dipvec, const int* iper, const int* ifpgh, double* pot, double* grad,
             double* hess, const int* nt, const double* targ, const int* ifpghtarg,
             double* pottarg, double* gradtarg, double* hesstarg, int* ier);
void hfmm2d_(const int* nd, const double* eps, const double* zk, const int* ns,
             const double* sources, const int* ifcharge, const double* charge,
             const int* ifdipole, const double* dipstr, const double* dipvec, const int* iper,
             const int* ifpgh, double* pot, double* grad, double* hess, const int* nt,
             const double* targ, const int* ifpghtarg, double* pottarg, double* gradtarg,
             double* hesstarg, int* ier);

/* ---- tuning variants: ndiv, idivflag, ifnear in; timeinfo(8) out (seconds) */
void cfmm2d_ndiv_(const int* nd, const double* eps, const int* ns, const double* sources,
                  const int* ifcharge, const double* charge, const int* ifdipole,
                  const double* dipstr, const int* iper, const int* ifpgh, double* pot,
                  double* grad, double* hess, const int* nt, const double* targ,
                  const int* ifpghtarg, double* pottarg, double* gradtarg, double* hesstarg,
                  const int* ndiv, const int* idivflag, const int* ifnear, double* timeinfo,
                  int* ier);
void lfmm2d_ndiv_(const int* nd, const double* eps, const int* ns, const double* sources,
                  const int* ifcharge, const double* charge, const int* ifdipole,
                  const double* dipstr, const double* dipvec, const int* iper, const int* ifpgh,
                  double* pot, double* grad, double* hess, const int* nt, const double* targ,
                  const int* ifpghtarg, double* pottarg, double* gradtarg, double* hesstarg,
                  const int* ndiv, const int* idivflag, const int* ifnear, double* timeinfo,
                  int* ier);
void rfmm2d_ndiv_(const int* nd, const double* eps, const int* ns, const double* sources,
                  const int* ifcharge, const double* charge, const int* ifdipole,
                  const double* dipstr, const double* dipvec, const int* iper, const int* ifpgh,
                  double* pot, double* grad, double* hess, const int* nt, const double* targ,
                  const int* ifpghtarg, double* pottarg, double* gradtarg, double* hesstarg,
                  const int* ndiv, const int* idivflag, const int* ifnear, double* timeinfo,
                  int* ier);
void hfmm2d_ndiv_(const int* nd, const double* eps, const double* zk, const int* ns,
                  const double* sources, const int* ifcharge, const double* charge,
                  const int* ifdipole, const double* dipstr, const double* dipvec,
                  const int* iper, const int* ifpgh, double* pot, double* grad, double* hess,
                  const int* nt, const double* targ, const int* ifpghtarg, double* pottarg,
                  double* gradtarg, double* hesstarg, const int* ndiv, const int* idivflag,
                  const int* ifnear, double* timeinfo, int* ier);

/* ---- biharmonic (src/biharmonic/bhfmm2d.f:1-4) and Stokes
 * (src/stokes/stfmm2d.f:3-7) FMMs: charge(nd,2,ns), dip(nd,3,ns) complex;
 * stoklet, strslet, strsvec (nd,2,ns) real; see fmm2d_b200.h. */
void bhfmm2d_(const int* nd, const double* eps, const int* ns, const double* sources,
              const int* ifcharge, const double* charge, const int* ifdipole, const double* dip,
              const int* iper, const int* ifpgh, double* pot, double* grad, double* hess,
              const int* nt, const double* targ, const int* ifpghtarg, double* pottarg,
              double* gradtarg, double* hesstarg, int* ier);
void stfmm2d_(const int* nd, const double* eps, const int* nsource, const double* source,
              const int* ifstoklet, const double* stoklet, const int* ifstrslet,
              const double* strslet, const double* strsvec, const int* ifppreg, double* pot,
              double* pre, double* grad, const int* ntarg, const double* targ,
              const int* ifppregtarg, double* pottarg, double* pretarg, double* gradtarg,
              int* ier);

/* ---- FMM over multipole expansions (src/helmholtz/hfmm2d_mps.f:19-22):
 * cmpole(2,nmpole), rmpole(nmpole), mterms(nmpole), mpole/local(ntot)
 * complex, impole(nmpole) 1-based offsets of the (nd,-m:m) blocks. */
void hfmm2d_mps_(const int* nd, const double* eps, const double* zk, const int* nmpole,
                 const double* cmpole, const double* rmpole, const int* mterms, const int* ntot,
                 const double* mpole, const int* impole, double* local, int* ier);

/* ---- flag wrappers.  Argument lists, in order:
 *   [nd,] eps, [zk,] ns, sources, <densities>, <source outputs>, [nt, targ, <target outputs>,] ier
 * densities: c = charge; d = dipstr[, dipvec]; cd = charge, dipstr[, dipvec]
 *   (dipvec for lfmm2d, rfmm2d and hfmm2d, not cfmm2d);
 * outputs: p = pot; g = pot, grad; h = pot, grad, hess (target: pottarg, ...);
 * s_ has only source outputs, t_ only nt, targ and target outputs, st_ both. */
#define B2F77_HEAD_c const double *eps, const int *ns, const double *sources
#define B2F77_HEAD_l B2F77_HEAD_c
#define B2F77_HEAD_r B2F77_HEAD_c
#define B2F77_HEAD_h const double *eps, const double *zk, const int *ns, const double *sources
#define B2F77_DENS_c_c const double *charge
#define B2F77_DENS_c_d const double *dipstr
#define B2F77_DENS_c_cd const double *charge, const double *dipstr
#define B2F77_DENS_l_c const double *charge
#define B2F77_DENS_l_d const double *dipstr, const double *dipvec
#define B2F77_DENS_l_cd const double *charge, const double *dipstr, const double *dipvec
#define B2F77_DENS_r_c B2F77_DENS_l_c
#define B2F77_DENS_r_d B2F77_DENS_l_d
#define B2F77_DENS_r_cd B2F77_DENS_l_cd
#define B2F77_DENS_h_c B2F77_DENS_l_c
#define B2F77_DENS_h_d B2F77_DENS_l_d
#define B2F77_DENS_h_cd B2F77_DENS_l_cd
#define B2F77_OUT_S_p double *pot
#define B2F77_OUT_S_g double *pot, double *grad
#define B2F77_OUT_S_h double *pot, double *grad, double *hess
#define B2F77_OUT_T_p double *pottarg
#define B2F77_OUT_T_g double *pottarg, double *gradtarg
#define B2F77_OUT_T_h double *pottarg, double *gradtarg, double *hesstarg
#define B2F77_SIG_s(F, D, O) B2F77_HEAD_##F, B2F77_DENS_##F##_##D, B2F77_OUT_S_##O, int *ier
#define B2F77_SIG_t(F, D, O) \
  B2F77_HEAD_##F, B2F77_DENS_##F##_##D, const int *nt, const double *targ, B2F77_OUT_T_##O, int *ier
#define B2F77_SIG_st(F, D, O)                                                            \
  B2F77_HEAD_##F, B2F77_DENS_##F##_##D, B2F77_OUT_S_##O, const int *nt, const double *targ, \
      B2F77_OUT_T_##O, int *ier

/* X(F, kind, densities, outputs) for the 27 combinations of family F */
#define B2F77_EACH_OF(X, F, K, D) X(F, K, D, p) X(F, K, D, g) X(F, K, D, h)
#define B2F77_EACH_K(X, F, K) \
  B2F77_EACH_OF(X, F, K, c) B2F77_EACH_OF(X, F, K, d) B2F77_EACH_OF(X, F, K, cd)
#define B2F77_EACH(X, F) B2F77_EACH_K(X, F, s) B2F77_EACH_K(X, F, t) B2F77_EACH_K(X, F, st)

#define B2F77_DECL(F, K, D, O)                                       \
  void F##fmm2d_##K##_##D##_##O##_(B2F77_SIG_##K(F, D, O));           \
  void F##fmm2d_##K##_##D##_##O##_vec_(const int *nd, B2F77_SIG_##K(F, D, O));
B2F77_EACH(B2F77_DECL, c)
B2F77_EACH(B2F77_DECL, l)
B2F77_EACH(B2F77_DECL, r)
B2F77_EACH(B2F77_DECL, h)

/* ---- the reference's C declaration (include/fmm2d/helmholtz.h:10): Helmholtz
 * potential of charges at the sources, arguments by value, 64-bit sizes. */
#ifndef __cplusplus
void hfmm2d_s_c_p(double eps, double _Complex zk, int64_t ns, double const *sources,
                  double _Complex const *charge, double _Complex *pot, int64_t *ier);
#endif

#ifdef __cplusplus
}
#endif

#endif /* FMM2D_F77_H */
