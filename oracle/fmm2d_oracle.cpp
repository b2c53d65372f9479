// TEST INFRASTRUCTURE ONLY -- the oracle.
//
// CPU restatement (C++17 + OpenMP) of the FMM evaluation path of
// flatironinstitute/fmm2d, which is written in Fortran.  It is used
//   * by tests/ as the parity checker of the CUDA library fmm2d_b200, and
//   * by bench.py (cpu_baseline and `--impl reference`) as the timed CPU
//     baseline, because no Fortran compiler exists in this image.
// The product path (fmm2d_b200/) never links, loads or calls this file.
//
// Parity pin.  The reference is Fortran and no Fortran compiler exists in
// this image, so oracle/f77c.py translates the reference's own source files
// to C and gcc compiles them (make -C oracle ref -> _ref/libfmm2d_ref.so,
// front end oracle/ref.py).  tests/test_ref_pin.py requires this restatement
// to equal that build of the reference: trees, point sorts and lists 1-4
// array for array (uniform, 16-Gaussian, graded-curve, target and duplicate
// point cases, idivflag 0-2), lfmm2d / rfmm2d / cfmm2d / hfmm2d outputs
// within 1e-12 relative l2 on the reference's test inputs
// (test/laplace/test_lfmm2d.f:30-101, test/helmholtz/test_hfmm2d.f:19-51,
// with hkrand/dlaran restated below), the direct sums and the ndiv / nterms
// tables.  Independent checks: mpmath direct sums (tests/golden/).
//
// Conventions: 0-based box and point indices, -1 for "none"; complex arrays
// are interleaved (re, im) doubles in the reference's column-major (nd, n)
// order, i.e. element (d, i) lives at [(i*nd + d)*2].  Point ranges are
// half-open [start, end).

#include <algorithm>
#include <chrono>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef std::complex<double> cdbl;

namespace {

double wtime() {
  using namespace std::chrono;
  return duration<double>(steady_clock::now().time_since_epoch()).count();
}

// ---------------------------------------------------------------------------
// Leaf size and expansion order tables
// ---------------------------------------------------------------------------

// src/laplace/lndiv2d.f:1-39 (idivflag = 0: subdivide on sources only)
int lap_ndiv(double eps, long ns, long nt) {
  if (eps >= 0.5e0) return 3;
  if (eps >= 0.5e-1) return 5;
  if (eps >= 0.5e-2) return 8;
  if (eps >= 0.5e-3) return 10;
  if (eps >= 0.5e-6) return 15;
  if (eps >= 0.5e-9) return 20;
  if (eps >= 0.5e-12) return 25;
  if (eps >= 0.5e-15) return 45;
  return (int)(ns + nt);
}

// src/laplace/l2dterms.f:38-82: first j in [2,100] with
// |(sqrt2/2)^j / 1.5^(j+1)| < eps, else 1.
int lap_nterms(double eps) {
  const double z2 = std::sqrt(2.0) / 2.0;
  cdbl z1(1.5, 0.0);
  cdbl hp = 1.0, jp = 1.0;
  for (int j = 0; j <= 100; j++) {
    // hfun(j) = 1/z1^(j+1), jfun(j) = z2^j, both by repeated products
    hp *= z1;
    if (j >= 2) {
      double x = std::abs(jp * (1.0 / hp));
      if (x < eps) return j;
    }
    jp *= z2;
  }
  return 1;
}

// src/common/fmmcommon2d.f:150-165 (binomial table, Pascal recursion)
struct Binom {
  int ldc = 100;
  std::vector<double> c;  // c[l*(ldc+1)+m] = C(l,m)
  Binom() {
    c.assign((ldc + 1) * (ldc + 1), 0.0);
    for (int l = 0; l <= ldc; l++) c[l * (ldc + 1)] = 1.0;
    for (int m = 1; m <= ldc; m++) {
      c[m * (ldc + 1) + m] = 1.0;
      for (int l = m + 1; l <= ldc; l++)
        c[l * (ldc + 1) + m] = c[(l - 1) * (ldc + 1) + m] + c[(l - 1) * (ldc + 1) + m - 1];
    }
  }
  double operator()(int l, int m) const { return c[l * (ldc + 1) + m]; }
};

// ---------------------------------------------------------------------------
// Quadtree
// ---------------------------------------------------------------------------

struct Tree {
  int nlevels = 0;
  std::vector<int> lfirst, llast;  // per level, inclusive box range
  std::vector<int> ilevel, iparent, nchild, ichild, ncoll, coll;
  std::vector<double> centers, boxsize;
  // point sort (filled by sort_points)
  std::vector<int> isrc, isrcse, itarg, itargse;
  // interaction lists
  std::vector<int> nl1, l1, nl2, l2, nl3, l3, nl4, l4;

  int nboxes() const { return (int)ilevel.size(); }
  int add_box(double cx, double cy, int lev, int par) {
    int b = nboxes();
    centers.push_back(cx);
    centers.push_back(cy);
    ilevel.push_back(lev);
    iparent.push_back(par);
    nchild.push_back(0);
    for (int j = 0; j < 4; j++) ichild.push_back(-1);
    return b;
  }
};

const int MNL1 = 13, MNL2 = 27, MNL3 = 20, MNL4 = 5;  // tree_routs2d.f:473-476
const double F105 = (double)1.05f;  // Fortran default-real literal 1.05

// Child j (0..3) of a box of centre c: (-,-), (+,-), (-,+), (+,+) offsets of
// half the child size (tree_routs2d.f:33-47).
void make_children(Tree& T, int ibox, double bs_child, int child_level) {
  double cx = T.centers[2 * ibox], cy = T.centers[2 * ibox + 1];
  double h = bs_child / 2;
  T.nchild[ibox] = 4;
  for (int j = 0; j < 4; j++) {
    double sx = (j % 2 == 0) ? -h : h;
    double sy = (j < 2) ? -h : h;
    int c = T.add_box(cx + sx, cy + sy, child_level, ibox);
    T.ichild[4 * ibox + j] = c;
  }
}

// Stable 4-way partition of perm[se[2b] .. se[2b+1]) into the children of b:
// first on y - cy < 0, then on x - cx < 0 (pts_tree2d.f:659-754).
void split_points(const Tree& T, int b, const double* xy, std::vector<int>& perm,
                  std::vector<int>& se) {
  int s = se[2 * b], e = se[2 * b + 1];
  double cx = T.centers[2 * b], cy = T.centers[2 * b + 1];
  int cnt[4] = {0, 0, 0, 0};
  std::vector<int> tmp(perm.begin() + s, perm.begin() + e);
  std::vector<unsigned char> slot(e - s);
  for (int k = 0; k < e - s; k++) {
    int i = tmp[k];
    int sy = (xy[2 * i + 1] - cy < 0) ? 0 : 1;
    int sx = (xy[2 * i] - cx < 0) ? 0 : 1;
    slot[k] = (unsigned char)(2 * sy + sx);
    cnt[slot[k]]++;
  }
  int off[4];
  off[0] = s;
  for (int j = 1; j < 4; j++) off[j] = off[j - 1] + cnt[j - 1];
  for (int j = 0; j < 4; j++) {
    int c = T.ichild[4 * b + j];
    se[2 * c] = off[j];
    se[2 * c + 1] = off[j] + cnt[j];
  }
  int pos[4] = {off[0], off[1], off[2], off[3]};
  for (int k = 0; k < e - s; k++) perm[pos[slot[k]]++] = tmp[k];
}

// Colleagues (same-level boxes sharing an edge or vertex, self included)
// from the parent's colleagues' children (tree_routs2d.f:100-211).
void colleagues_of(Tree& T, int ibox) {
  int lev = T.ilevel[ibox];
  T.ncoll[ibox] = 0;
  for (int j = 0; j < 9; j++) T.coll[9 * ibox + j] = -1;
  if (lev == 0) {
    T.ncoll[ibox] = 1;
    T.coll[9 * ibox] = ibox;
    return;
  }
  int dad = T.iparent[ibox];
  double tol = F105 * T.boxsize[lev];
  for (int i = 0; i < T.ncoll[dad]; i++) {
    int jbox = T.coll[9 * dad + i];
    for (int j = 0; j < 4; j++) {
      int kbox = T.ichild[4 * jbox + j];
      if (kbox < 0) continue;
      if (std::fabs(T.centers[2 * kbox] - T.centers[2 * ibox]) <= tol &&
          std::fabs(T.centers[2 * kbox + 1] - T.centers[2 * ibox + 1]) <= tol &&
          T.ncoll[ibox] < 9) {
        T.coll[9 * ibox + T.ncoll[ibox]] = kbox;
        T.ncoll[ibox]++;
      }
    }
  }
}

void compute_colleagues(Tree& T) {
  int nb = T.nboxes();
  T.ncoll.assign(nb, 0);
  T.coll.assign(9 * (size_t)nb, -1);
  for (int lev = 0; lev <= T.nlevels; lev++) {
#pragma omp parallel for schedule(static)
    for (int b = T.lfirst[lev]; b <= T.llast[lev]; b++) colleagues_of(T, b);
  }
}

// Renumber so that each level >= 2 holds its original boxes followed by the
// appended ("tail") boxes of that level (pts_tree2d.f:1066-1215).
void reorganize(Tree& T, const std::vector<int>& tfirst, const std::vector<int>& tlast,
                std::vector<int>& iflag) {
  int nb = T.nboxes();
  std::vector<int> map(nb, -1);
  for (int lev = 0; lev <= std::min(1, T.nlevels); lev++)
    for (int b = T.lfirst[lev]; b <= T.llast[lev]; b++) map[b] = b;
  if (T.nlevels >= 2) {
    int cur = T.lfirst[2];
    for (int lev = 2; lev <= T.nlevels; lev++) {
      int f = cur;
      for (int b = T.lfirst[lev]; b <= T.llast[lev]; b++) map[b] = cur++;
      for (int b = tfirst[lev]; b <= tlast[lev]; b++) map[b] = cur++;
      T.lfirst[lev] = f;
      T.llast[lev] = cur - 1;
    }
  }
  Tree o = T;
  std::vector<int> of = iflag;
  for (int b = 0; b < nb; b++) {
    int n = map[b];
    T.centers[2 * n] = o.centers[2 * b];
    T.centers[2 * n + 1] = o.centers[2 * b + 1];
    T.ilevel[n] = o.ilevel[b];
    T.nchild[n] = o.nchild[b];
    iflag[n] = of[b];
    T.iparent[n] = o.iparent[b] < 0 ? -1 : map[o.iparent[b]];
    for (int j = 0; j < 4; j++) {
      int c = o.ichild[4 * b + j];
      T.ichild[4 * n + j] = c < 0 ? -1 : map[c];
    }
  }
}

// Refine the boxes of [first,last] whose flag is > 0 (tree_routs2d.f:334-388);
// children of flag-1 boxes become flag++ (3), of flag+ boxes 0.
void refine_flagged(Tree& T, int first, int last, int child_level, std::vector<int>& iflag) {
  for (int b = first; b <= last; b++) {
    if (iflag[b] <= 0) continue;
    make_children(T, b, T.boxsize[child_level], child_level);
    for (int j = 0; j < 4; j++) {
      int c = T.ichild[4 * b + j];
      iflag.push_back(iflag[b] == 1 ? 3 : 0);
      (void)c;
    }
  }
}

// A flag++ box stays a leaf unless a child of one of its colleagues has
// children and touches it (tree_routs2d.f:217-326).
void update_flags(Tree& T, int lev, int first, int last, std::vector<int>& iflag) {
  double distest = 1.05 * (T.boxsize[lev] + T.boxsize[lev + 1]) / 2.0;
#pragma omp parallel for schedule(static)
  for (int b = first; b <= last; b++) {
    if (iflag[b] != 3) continue;
    int f = 0;
    for (int i = 0; i < T.ncoll[b] && !f; i++) {
      int jbox = T.coll[9 * b + i];
      for (int j = 0; j < 4; j++) {
        int k = T.ichild[4 * jbox + j];
        if (k < 0 || T.nchild[k] <= 0) continue;
        double xd = T.centers[2 * k] - T.centers[2 * b];
        double yd = T.centers[2 * k + 1] - T.centers[2 * b + 1];
        if (std::fabs(xd) <= distest && std::fabs(yd) <= distest) {
          f = 1;
          break;
        }
      }
    }
    iflag[b] = f;
  }
}

// Level restriction (pts_tree2d.f:758-1061).
void fix_level_restriction(Tree& T) {
  int nl = T.nlevels;
  std::vector<int> iflag(T.nboxes(), 0);
  // flag: leaf colleagues of a grandparent that touch the parent
  for (int lev = nl; lev >= 2; lev--) {
    double distest = 1.05 * (T.boxsize[lev - 1] + T.boxsize[lev - 2]) / 2.0;
    for (int b = T.lfirst[lev]; b <= T.llast[lev]; b++) {
      int dad = T.iparent[b], gd = T.iparent[dad];
      for (int i = 0; i < T.ncoll[gd]; i++) {
        int j = T.coll[9 * gd + i];
        if (T.nchild[j] != 0 || iflag[j] != 0) continue;
        double xd = T.centers[2 * j] - T.centers[2 * dad];
        double yd = T.centers[2 * j + 1] - T.centers[2 * dad + 1];
        if (std::fabs(xd) <= distest && std::fabs(yd) <= distest) iflag[j] = 1;
      }
    }
  }
  // flag+: leaf colleagues of the parent of a flagged/flag+ box that touch it
  for (int lev = nl; lev >= 1; lev--) {
    double distest = 1.05 * (T.boxsize[lev] + T.boxsize[lev - 1]) / 2.0;
    for (int b = T.lfirst[lev]; b <= T.llast[lev]; b++) {
      if (iflag[b] != 1 && iflag[b] != 2) continue;
      int dad = T.iparent[b];
      for (int i = 0; i < T.ncoll[dad]; i++) {
        int j = T.coll[9 * dad + i];
        if (T.nchild[j] != 0 || iflag[j] != 0) continue;
        double xd = T.centers[2 * j] - T.centers[2 * b];
        double yd = T.centers[2 * j + 1] - T.centers[2 * b + 1];
        if (std::fabs(xd) <= distest && std::fabs(yd) <= distest) iflag[j] = 2;
      }
    }
  }
  std::vector<int> tfirst(nl + 1, 0), tlast(nl + 1, -1);
  for (int lev = 1; lev <= nl - 2; lev++) {
    tfirst[lev + 1] = T.nboxes();
    refine_flagged(T, T.lfirst[lev], T.llast[lev], lev + 1, iflag);
    tlast[lev + 1] = T.nboxes() - 1;
  }
  reorganize(T, tfirst, tlast, iflag);
  compute_colleagues(T);
  for (int b = 0; b < T.nboxes(); b++)
    if (iflag[b] != 3) iflag[b] = 0;
  std::fill(tfirst.begin(), tfirst.end(), 0);
  std::fill(tlast.begin(), tlast.end(), -1);
  for (int lev = 2; lev <= nl - 2; lev++) {
    update_flags(T, lev, T.lfirst[lev], T.llast[lev], iflag);
    update_flags(T, lev, tfirst[lev], tlast[lev], iflag);
    tfirst[lev + 1] = T.nboxes();
    refine_flagged(T, T.lfirst[lev], T.llast[lev], lev + 1, iflag);
    refine_flagged(T, tfirst[lev], tlast[lev], lev + 1, iflag);
    tlast[lev + 1] = T.nboxes() - 1;
    // colleagues of the new boxes from their parents' current lists
    T.ncoll.resize(T.nboxes(), 0);
    T.coll.resize(9 * (size_t)T.nboxes(), -1);
    for (int b = tfirst[lev + 1]; b <= tlast[lev + 1]; b++) colleagues_of(T, b);
  }
  reorganize(T, tfirst, tlast, iflag);
  compute_colleagues(T);
}

// Adaptive tree on sources (idivflag 0), targets (1) or max of both (2),
// then level restriction (pts_tree2d.f:406-655).
void build_tree(const double* src, int ns, const double* targ, int nt, int idivflag, int ndiv,
                int nlmax, Tree& T) {
  double xmin, xmax, ymin, ymax;
  if (ns > 0) {
    xmin = xmax = src[0];
    ymin = ymax = src[1];
  } else {
    xmin = xmax = targ[0];
    ymin = ymax = targ[1];
  }
  for (int i = 0; i < ns; i++) {
    xmin = std::min(xmin, src[2 * i]);
    xmax = std::max(xmax, src[2 * i]);
    ymin = std::min(ymin, src[2 * i + 1]);
    ymax = std::max(ymax, src[2 * i + 1]);
  }
  for (int i = 0; i < nt; i++) {
    xmin = std::min(xmin, targ[2 * i]);
    xmax = std::max(xmax, targ[2 * i]);
    ymin = std::min(ymin, targ[2 * i + 1]);
    ymax = std::max(ymax, targ[2 * i + 1]);
  }
  double bs0 = xmax - xmin, sizey = ymax - ymin;
  if (sizey > bs0) bs0 = sizey;
  T = Tree();
  T.boxsize.push_back(bs0);
  T.add_box((xmin + xmax) / 2, (ymin + ymax) / 2, 0, -1);
  T.lfirst.push_back(0);
  T.llast.push_back(0);
  std::vector<int> isrc(ns), itarg(nt), sse(2, 0), tse(2, 0);
  for (int i = 0; i < ns; i++) isrc[i] = i;
  for (int i = 0; i < nt; i++) itarg[i] = i;
  sse[1] = ns;
  tse[1] = nt;
  int lev;
  // all points coincide (zero-size root): no subdivision is possible
  if (bs0 == 0.0) nlmax = 0;
  for (lev = 0; lev < nlmax; lev++) {
    int f = T.lfirst[lev], l = T.llast[lev];
    std::vector<char> ref(l - f + 1, 0);
    bool any = false;
    for (int b = f; b <= l; b++) {
      int nss = sse[2 * b + 1] - sse[2 * b], ntt = tse[2 * b + 1] - tse[2 * b];
      int nn = idivflag == 0 ? nss : (idivflag == 1 ? ntt : std::max(nss, ntt));
      if (nn > ndiv) {
        ref[b - f] = 1;
        any = true;
      }
    }
    if (!any) break;
    T.boxsize.push_back(T.boxsize[lev] / 2);
    T.lfirst.push_back(T.nboxes());
    for (int b = f; b <= l; b++)
      if (ref[b - f]) make_children(T, b, T.boxsize[lev + 1], lev + 1);
    T.llast.push_back(T.nboxes() - 1);
    sse.resize(2 * (size_t)T.nboxes(), 0);
    tse.resize(2 * (size_t)T.nboxes(), 0);
    for (int b = f; b <= l; b++)
      if (ref[b - f]) {
        split_points(T, b, src, isrc, sse);
        split_points(T, b, targ, itarg, tse);
      }
  }
  T.nlevels = lev;
  compute_colleagues(T);
  if (T.nlevels >= 2) fix_level_restriction(T);
}

// Final stable sort of points into the leaves of the final tree
// (pts_tree2d.f:1222-1246).
void sort_points(const Tree& T, const double* xy, int n, std::vector<int>& perm,
                 std::vector<int>& se) {
  perm.resize(n);
  for (int i = 0; i < n; i++) perm[i] = i;
  se.assign(2 * (size_t)T.nboxes(), 0);
  se[1] = n;
  for (int lev = 0; lev < T.nlevels; lev++)
    for (int b = T.lfirst[lev]; b <= T.llast[lev]; b++)
      if (T.nchild[b] > 0) split_points(T, b, xy, perm, se);
}

// Lists 1-4 (tree_routs2d.f:486-710).
void compute_lists(Tree& T) {
  int nb = T.nboxes();
  T.nl1.assign(nb, 0);
  T.nl2.assign(nb, 0);
  T.nl3.assign(nb, 0);
  T.nl4.assign(nb, 0);
  T.l1.assign((size_t)MNL1 * nb, -1);
  T.l2.assign((size_t)MNL2 * nb, -1);
  T.l3.assign((size_t)MNL3 * nb, -1);
  T.l4.assign((size_t)MNL4 * nb, -1);
  if (T.nchild[0] == 0) {
    T.nl1[0] = 1;
    T.l1[0] = 0;
  }
  for (int lev = 1; lev <= T.nlevels; lev++) {
    double tol = F105 * T.boxsize[lev];
    for (int b = T.lfirst[lev]; b <= T.llast[lev]; b++) {
      int dad = T.iparent[b];
      for (int i = 0; i < T.ncoll[dad]; i++) {
        int j = T.coll[9 * dad + i];
        for (int c = 0; c < T.nchild[j]; c++) {
          int k = T.ichild[4 * j + c];
          if (std::fabs(T.centers[2 * k] - T.centers[2 * b]) >= tol ||
              std::fabs(T.centers[2 * k + 1] - T.centers[2 * b + 1]) >= tol) {
            T.l2[(size_t)MNL2 * b + T.nl2[b]++] = k;
          }
        }
      }
      if (T.nchild[b] != 0) continue;
      for (int i = 0; i < T.ncoll[b]; i++) {
        int j = T.coll[9 * b + i];
        if (T.nchild[j] == 0) {
          T.l1[(size_t)MNL1 * b + T.nl1[b]++] = j;
          continue;
        }
        double distest = 1.05 * (T.boxsize[lev] + T.boxsize[lev + 1]) / 2.0;
        for (int c = 0; c < T.nchild[j]; c++) {
          int k = T.ichild[4 * j + c];
          double xd = std::fabs(T.centers[2 * k] - T.centers[2 * b]);
          double yd = std::fabs(T.centers[2 * k + 1] - T.centers[2 * b + 1]);
          if (xd < distest && yd < distest) {
            T.l1[(size_t)MNL1 * b + T.nl1[b]++] = k;
            T.l1[(size_t)MNL1 * k + T.nl1[k]++] = b;
          } else {
            T.l3[(size_t)MNL3 * b + T.nl3[b]++] = k;
            T.l4[(size_t)MNL4 * k + T.nl4[k]++] = b;
          }
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Cauchy expansion operators (src/laplace/laprouts2d.f).  Expansions are
// (nd, 0:p) complex arrays scaled by rscale = box size.
// ---------------------------------------------------------------------------

// P2M, charges and/or dipoles (laprouts2d.f:84-282):
// m_0 += q ; m_n += -q w^n / n + d w^(n-1) / r,  w = (x - c)/r
void p2m(int nd, double r, const double* src, int ns, const cdbl* q, const cdbl* dp,
         const double* c, int p, cdbl* mp) {
  std::vector<cdbl> wc(p + 1), wd(p + 1);
  for (int j = 0; j < ns; j++) {
    cdbl z(src[2 * j] - c[0], src[2 * j + 1] - c[1]);
    cdbl w = z / r;
    cdbl pw = 1.0;
    wc[0] = 1.0;
    wd[0] = 0.0;
    for (int n = 1; n <= p; n++) {
      wd[n] = pw / r;
      pw *= w;
      wc[n] = -pw / (double)n;
    }
    for (int n = 0; n <= p; n++)
      for (int d = 0; d < nd; d++) {
        cdbl a = 0.0;
        if (q) a += q[(size_t)j * nd + d] * wc[n];
        if (dp) a += dp[(size_t)j * nd + d] * wd[n];
        mp[n * nd + d] += a;
      }
  }
}

// P2L (laprouts2d.f:501-690): l_0 += q log|z0|; l_n += -q w^n/n - (d/z0) w^n,
// w = r/z0, z0 = x - c
void p2l(int nd, double r, const double* src, int ns, const cdbl* q, const cdbl* dp,
         const double* c, int p, cdbl* lo) {
  std::vector<cdbl> wc(p + 1), wd(p + 1);
  for (int j = 0; j < ns; j++) {
    cdbl z0(src[2 * j] - c[0], src[2 * j + 1] - c[1]);
    cdbl w = r / z0;
    cdbl zi = 1.0 / z0;
    cdbl pw = 1.0;
    wc[0] = std::log(std::abs(z0));
    wd[0] = -zi;
    for (int n = 1; n <= p; n++) {
      pw *= w;
      wc[n] = -pw / (double)n;
      wd[n] = -zi * pw;
    }
    for (int n = 0; n <= p; n++)
      for (int d = 0; d < nd; d++) {
        cdbl a = 0.0;
        if (q) a += q[(size_t)j * nd + d] * wc[n];
        if (dp) a += dp[(size_t)j * nd + d] * wd[n];
        lo[n * nd + d] += a;
      }
  }
}

// M2P (laprouts2d.f:289-500): pot += m_0 log|z| + sum m_n (r/z)^n, with
// d/dz and d2/dz2.
void m2p(int nd, double r, const double* c, const cdbl* mp, int p, const double* xy, int nt,
         int ifpgh, cdbl* pot, cdbl* grad, cdbl* hess) {
  std::vector<cdbl> zp(p + 3);
  for (int k = 0; k < nt; k++) {
    cdbl z(xy[2 * k] - c[0], xy[2 * k + 1] - c[1]);
    cdbl w = r / z;
    zp[0] = 1.0;
    for (int n = 1; n <= p + 2; n++) zp[n] = zp[n - 1] * w;
    double lg = std::log(std::abs(z));
    for (int d = 0; d < nd; d++) {
      cdbl pt = mp[d] * lg, g = mp[d] * (zp[1] / r), h = -mp[d] * (zp[2] / (r * r));
      for (int n = 1; n <= p; n++) {
        cdbl m = mp[n * nd + d];
        pt += m * zp[n];
        g += m * (-(double)n * zp[n + 1] / r);
        h += m * ((double)n * (n + 1) * zp[n + 2] / (r * r));
      }
      pot[(size_t)k * nd + d] += pt;
      if (ifpgh >= 2) grad[(size_t)k * nd + d] += g;
      if (ifpgh >= 3) hess[(size_t)k * nd + d] += h;
    }
  }
}

// L2P (laprouts2d.f:696-897): pot += sum l_n z^n, z = (x - c)/r.
void l2p(int nd, double r, const double* c, const cdbl* lo, int p, const double* xy, int nt,
         int ifpgh, cdbl* pot, cdbl* grad, cdbl* hess) {
  std::vector<cdbl> zp(p + 1);
  for (int k = 0; k < nt; k++) {
    cdbl z = cdbl(xy[2 * k] - c[0], xy[2 * k + 1] - c[1]) / r;
    zp[0] = 1.0;
    for (int n = 1; n <= p; n++) zp[n] = zp[n - 1] * z;
    for (int d = 0; d < nd; d++) {
      cdbl pt = 0.0, g = 0.0, h = 0.0;
      for (int n = 0; n <= p; n++) {
        cdbl l = lo[n * nd + d];
        pt += l * zp[n];
        if (n >= 1) g += l * (zp[n - 1] * ((double)n / r));
        if (n >= 2) h += l * (zp[n - 2] * ((double)n * (n - 1) / (r * r)));
      }
      pot[(size_t)k * nd + d] += pt;
      if (ifpgh >= 2) grad[(size_t)k * nd + d] += g;
      if (ifpgh >= 3) hess[(size_t)k * nd + d] += h;
    }
  }
}

// M2M (laprouts2d.f:905-1015), z0 = child - parent centre.
void m2m(int nd, double r1, const double* c1, const cdbl* h1, int p1, double r2,
         const double* c2, cdbl* h2, int p2, const Binom& C) {
  cdbl z0(c1[0] - c2[0], c1[1] - c2[1]);
  int nmax = std::max(p1, p2);
  std::vector<cdbl> a(nmax + 1), b(nmax + 1), t(p1 + 1);
  cdbl w1 = 1.0 / (z0 / r1), w2 = z0 / r2;
  a[0] = b[0] = 1.0;
  for (int i = 1; i <= nmax; i++) {
    a[i] = a[i - 1] * w1;
    b[i] = b[i - 1] * w2;
  }
  for (int d = 0; d < nd; d++) {
    for (int j = 0; j <= p1; j++) t[j] = h1[j * nd + d] * a[j];
    h2[d] += h1[d];
    for (int i = 1; i <= p2; i++) {
      cdbl s = -t[0] / (double)i;
      for (int j = 1; j <= std::min(i, p1); j++) s += t[j] * C(i - 1, j - 1);
      h2[i * nd + d] += s * b[i];
    }
  }
}

// L2L (laprouts2d.f:1020-1123), z0 = child - parent centre.
void l2l(int nd, double r1, const double* c1, const cdbl* j1, int p1, double r2,
         const double* c2, cdbl* j2, int p2, const Binom& C) {
  cdbl z0(c2[0] - c1[0], c2[1] - c1[1]);
  int nmax = std::max(p1, p2);
  std::vector<cdbl> a(nmax + 1), b(nmax + 1), t(p1 + 1);
  cdbl w1 = z0 / r1, w2 = 1.0 / (z0 / r2);
  a[0] = b[0] = 1.0;
  for (int i = 1; i <= nmax; i++) {
    a[i] = a[i - 1] * w1;
    b[i] = b[i - 1] * w2;
  }
  for (int d = 0; d < nd; d++) {
    for (int j = 0; j <= p1; j++) t[j] = j1[j * nd + d] * a[j];
    for (int i = 0; i <= p2; i++) {
      cdbl s = 0.0;
      for (int j = i; j <= p1; j++) s += t[j] * C(j, i);
      j2[i * nd + d] += s * b[i];
    }
  }
}

// M2L (laprouts2d.f:1130-1244), z0 = source - target centre.
void m2l(int nd, double r1, const double* c1, const cdbl* h1, int p1, double r2,
         const double* c2, cdbl* j2, int p2, const Binom& C) {
  cdbl z0(c1[0] - c2[0], c1[1] - c2[1]);
  int nmax = std::max(p1, p2);
  std::vector<cdbl> a(nmax + 1), b(nmax + 1), t(p1 + 1);
  cdbl zi = 1.0 / z0;
  a[0] = b[0] = 1.0;
  for (int i = 1; i <= nmax; i++) {
    a[i] = a[i - 1] * (-zi * r1);
    b[i] = b[i - 1] * (zi * r2);
  }
  double lg = std::log(std::abs(z0));
  for (int d = 0; d < nd; d++) {
    for (int j = 0; j <= p1; j++) t[j] = h1[j * nd + d] * a[j];
    cdbl s0 = t[0] * lg;
    for (int j = 1; j <= p1; j++) s0 += t[j];
    j2[d] += s0;
    for (int i = 1; i <= p2; i++) {
      cdbl s = -t[0] / (double)i;
      for (int j = 1; j <= p1; j++) s += t[j] * C(i + j - 1, j - 1);
      j2[i * nd + d] += s * b[i];
    }
  }
}

// ---------------------------------------------------------------------------
// Cauchy direct interactions (src/laplace/cauchykernels2d.f:3-683)
//   pot  += q log|z| + d/z ; grad += q/z - d/z^2 ; hess += -q/z^2 + 2d/z^3
// Pairs with |z| below thresh are skipped; the comparison is <= for the
// potential-only variants and < otherwise, as in the reference.
// ---------------------------------------------------------------------------
void c2d_direct(int nd, const double* src, int ns, const cdbl* q, const cdbl* dp,
                const double* trg, int nt, int ifpgh, cdbl* pot, cdbl* grad, cdbl* hess,
                double thresh) {
  double th2 = thresh * thresh;
  bool le = (ifpgh == 1);
  for (int j = 0; j < nt; j++) {
    for (int i = 0; i < ns; i++) {
      double dx = trg[2 * j] - src[2 * i], dy = trg[2 * j + 1] - src[2 * i + 1];
      double rr = dx * dx + dy * dy;
      if (!q) {
        // dipole-only variants compare |z| against thresh
        double az = std::abs(cdbl(dx, dy));
        if (le ? (az <= thresh) : (az < thresh)) continue;
      } else {
        if (le ? (rr <= th2) : (rr < th2)) continue;
      }
      double lg = std::log(rr) / 2;
      cdbl zi = 1.0 / cdbl(dx, dy);
      cdbl z2 = -zi * zi;
      cdbl z3 = -2.0 * z2 * zi;
      for (int d = 0; d < nd; d++) {
        cdbl pt = 0.0, g = 0.0, h = 0.0;
        if (q) {
          cdbl c = q[(size_t)i * nd + d];
          pt += lg * c;
          g += zi * c;
          h += z2 * c;
        }
        if (dp) {
          cdbl c = dp[(size_t)i * nd + d];
          pt += zi * c;
          g += z2 * c;
          h += z3 * c;
        }
        pot[(size_t)j * nd + d] += pt;
        if (ifpgh >= 2) grad[(size_t)j * nd + d] += g;
        if (ifpgh >= 3) hess[(size_t)j * nd + d] += h;
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Cauchy FMM driver (src/laplace/cfmm2d.f:23-436) and main loop
// (cfmm2d.f:442-1341).  Inputs in caller order; outputs overwritten.
// ---------------------------------------------------------------------------
struct CfmmArgs {
  int nd;
  double eps;
  int ns;
  const double* src;
  int ifcharge;
  const cdbl* charge;
  int ifdipole;
  const cdbl* dipstr;
  int ifpgh;
  cdbl *pot, *grad, *hess;
  int nt;
  const double* targ;
  int ifpghtarg;
  cdbl *pottarg, *gradtarg, *hesstarg;
  int ndiv;  // <= 0: from lndiv2d
  int idivflag;
  int ifnear;
  double* timeinfo;  // 8 entries or null
};

int run_cfmm(const CfmmArgs& A, Tree* keep_tree) {
  const int nd = A.nd;
  double tinfo[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  if (A.ns <= 0) {
    // no sources: every requested output is zero
    if (A.ifpghtarg >= 1) std::fill(A.pottarg, A.pottarg + (size_t)nd * A.nt, cdbl(0));
    if (A.ifpghtarg >= 2) std::fill(A.gradtarg, A.gradtarg + (size_t)nd * A.nt, cdbl(0));
    if (A.ifpghtarg >= 3) std::fill(A.hesstarg, A.hesstarg + (size_t)nd * A.nt, cdbl(0));
    return 0;
  }
  int ndiv = A.ndiv > 0 ? A.ndiv : lap_ndiv(A.eps, A.ns, A.nt);
  Tree T;
  build_tree(A.src, A.ns, A.targ, A.nt, A.idivflag, ndiv, 51, T);
  if (T.boxsize[0] == 0.0) {
    // every point coincides: only self interactions, which are omitted
    auto z = [&](cdbl* p, long n, int on) {
      if (on) std::fill(p, p + (size_t)nd * n, cdbl(0));
    };
    z(A.pot, A.ns, A.ifpgh >= 1);
    z(A.grad, A.ns, A.ifpgh >= 2);
    z(A.hess, A.ns, A.ifpgh >= 3);
    z(A.pottarg, A.nt, A.ifpghtarg >= 1);
    z(A.gradtarg, A.nt, A.ifpghtarg >= 2);
    z(A.hesstarg, A.nt, A.ifpghtarg >= 3);
    return 0;
  }
  sort_points(T, A.src, A.ns, T.isrc, T.isrcse);
  sort_points(T, A.targ, A.nt, T.itarg, T.itargse);
  compute_lists(T);
  const int p = lap_nterms(A.eps);
  const int P = p + 1;
  const int nb = T.nboxes();
  const int ns = A.ns, nt = A.nt;
  const bool fc = A.ifcharge == 1, fd = A.ifdipole == 1;
  // gather into tree order (fmmcommon2d.f:30-54)
  std::vector<double> ss(2 * (size_t)ns), ts(2 * (size_t)nt);
  std::vector<cdbl> qs(fc ? (size_t)nd * ns : 0), ds(fd ? (size_t)nd * ns : 0);
  for (int k = 0; k < ns; k++) {
    int i = T.isrc[k];
    ss[2 * k] = A.src[2 * i];
    ss[2 * k + 1] = A.src[2 * i + 1];
    for (int d = 0; d < nd; d++) {
      if (fc) qs[(size_t)k * nd + d] = A.charge[(size_t)i * nd + d];
      if (fd) ds[(size_t)k * nd + d] = A.dipstr[(size_t)i * nd + d];
    }
  }
  for (int k = 0; k < nt; k++) {
    int i = T.itarg[k];
    ts[2 * k] = A.targ[2 * i];
    ts[2 * k + 1] = A.targ[2 * i + 1];
  }
  const cdbl* qp = fc ? qs.data() : nullptr;
  const cdbl* dpp = fd ? ds.data() : nullptr;
  std::vector<cdbl> pot((size_t)nd * ns), grad((size_t)nd * ns), hess((size_t)nd * ns);
  std::vector<cdbl> pott((size_t)nd * nt), gradt((size_t)nd * nt), hesst((size_t)nd * nt);
  std::vector<cdbl> mp((size_t)nb * P * nd), lo((size_t)nb * P * nd);
  Binom C;
  const int nl = T.nlevels;
  auto npts_src = [&](int b) { return T.isrcse[2 * b + 1] - T.isrcse[2 * b]; };
  auto npts_trg = [&](int b) { return T.itargse[2 * b + 1] - T.itargse[2 * b]; };
  auto has_eval_pts = [&](int b) {
    int n = 0;
    if (A.ifpghtarg > 0) n += npts_trg(b);
    if (A.ifpgh > 0) n += npts_src(b);
    return n > 0;
  };
  auto MP = [&](int b) { return &mp[(size_t)b * P * nd]; };
  auto LO = [&](int b) { return &lo[(size_t)b * P * nd]; };
  auto CEN = [&](int b) { return &T.centers[2 * (size_t)b]; };

  // step 1: P2M at leaves, levels 2..nl
  double t0 = wtime();
  for (int lev = 2; lev <= nl; lev++) {
#pragma omp parallel for schedule(dynamic)
    for (int b = T.lfirst[lev]; b <= T.llast[lev]; b++) {
      int s = T.isrcse[2 * b], n = npts_src(b);
      if (T.nchild[b] == 0 && n > 0)
        p2m(nd, T.boxsize[lev], &ss[2 * (size_t)s], n, qp ? qp + (size_t)s * nd : nullptr,
            dpp ? dpp + (size_t)s * nd : nullptr, CEN(b), p, MP(b));
    }
  }
  tinfo[0] = wtime() - t0;
  // step 2: P2L from list 4
  t0 = wtime();
  for (int lev = 2; lev <= nl; lev++) {
#pragma omp parallel for schedule(dynamic)
    for (int b = T.lfirst[lev]; b <= T.llast[lev]; b++) {
      if (!has_eval_pts(b)) continue;
      for (int i = 0; i < T.nl4[b]; i++) {
        int j = T.l4[(size_t)MNL4 * b + i];
        int s = T.isrcse[2 * j], n = npts_src(j);
        p2l(nd, T.boxsize[lev], &ss[2 * (size_t)s], n, qp ? qp + (size_t)s * nd : nullptr,
            dpp ? dpp + (size_t)s * nd : nullptr, CEN(b), p, LO(b));
      }
    }
  }
  tinfo[1] = wtime() - t0;
  // step 3: M2M upward
  t0 = wtime();
  for (int lev = nl - 1; lev >= 1; lev--) {
#pragma omp parallel for schedule(dynamic)
    for (int b = T.lfirst[lev]; b <= T.llast[lev]; b++) {
      for (int i = 0; i < T.nchild[b]; i++) {
        int c = T.ichild[4 * b + i];
        if (npts_src(c) > 0)
          m2m(nd, T.boxsize[lev + 1], CEN(c), MP(c), p, T.boxsize[lev], CEN(b), MP(b), p, C);
      }
    }
  }
  tinfo[2] = wtime() - t0;
  // step 4: M2L over list 2
  t0 = wtime();
  for (int lev = 2; lev <= nl; lev++) {
#pragma omp parallel for schedule(dynamic)
    for (int b = T.lfirst[lev]; b <= T.llast[lev]; b++) {
      if (!has_eval_pts(b)) continue;
      for (int i = 0; i < T.nl2[b]; i++) {
        int j = T.l2[(size_t)MNL2 * b + i];
        m2l(nd, T.boxsize[lev], CEN(j), MP(j), p, T.boxsize[lev], CEN(b), LO(b), p, C);
      }
    }
  }
  tinfo[3] = wtime() - t0;
  // step 5: L2L downward
  t0 = wtime();
  for (int lev = 1; lev <= nl - 1; lev++) {
#pragma omp parallel for schedule(dynamic)
    for (int b = T.lfirst[lev]; b <= T.llast[lev]; b++) {
      if (!has_eval_pts(b)) continue;
      for (int i = 0; i < T.nchild[b]; i++) {
        int c = T.ichild[4 * b + i];
        l2l(nd, T.boxsize[lev], CEN(b), LO(b), p, T.boxsize[lev + 1], CEN(c), LO(c), p, C);
      }
    }
  }
  tinfo[4] = wtime() - t0;
  // step 6: M2P from list 3
  t0 = wtime();
  for (int lev = 1; lev <= nl - 1; lev++) {
#pragma omp parallel for schedule(dynamic)
    for (int b = T.lfirst[lev]; b <= T.llast[lev]; b++) {
      for (int i = 0; i < T.nl3[b]; i++) {
        int j = T.l3[(size_t)MNL3 * b + i];
        double r = T.boxsize[lev + 1];
        if (A.ifpghtarg > 0) {
          int s = T.itargse[2 * b], n = npts_trg(b);
          m2p(nd, r, CEN(j), MP(j), p, &ts[2 * (size_t)s], n, A.ifpghtarg, &pott[(size_t)s * nd],
              &gradt[(size_t)s * nd], &hesst[(size_t)s * nd]);
        }
        if (A.ifpgh > 0) {
          int s = T.isrcse[2 * b], n = npts_src(b);
          m2p(nd, r, CEN(j), MP(j), p, &ss[2 * (size_t)s], n, A.ifpgh, &pot[(size_t)s * nd],
              &grad[(size_t)s * nd], &hess[(size_t)s * nd]);
        }
      }
    }
  }
  tinfo[5] = wtime() - t0;
  // step 7: L2P at leaves
  t0 = wtime();
  for (int lev = 0; lev <= nl; lev++) {
#pragma omp parallel for schedule(dynamic)
    for (int b = T.lfirst[lev]; b <= T.llast[lev]; b++) {
      if (T.nchild[b] != 0) continue;
      double r = T.boxsize[lev];
      if (A.ifpghtarg > 0) {
        int s = T.itargse[2 * b], n = npts_trg(b);
        l2p(nd, r, CEN(b), LO(b), p, &ts[2 * (size_t)s], n, A.ifpghtarg, &pott[(size_t)s * nd],
            &gradt[(size_t)s * nd], &hesst[(size_t)s * nd]);
      }
      if (A.ifpgh > 0) {
        int s = T.isrcse[2 * b], n = npts_src(b);
        l2p(nd, r, CEN(b), LO(b), p, &ss[2 * (size_t)s], n, A.ifpgh, &pot[(size_t)s * nd],
            &grad[(size_t)s * nd], &hess[(size_t)s * nd]);
      }
    }
  }
  tinfo[6] = wtime() - t0;
  // step 8: P2P over list 1, thresh = boxsize(0) 2^-51
  t0 = wtime();
  double thresh = T.boxsize[0] * std::pow(2.0, -51);
  if (A.ifnear) {
    for (int lev = 0; lev <= nl; lev++) {
#pragma omp parallel for schedule(dynamic)
      for (int b = T.lfirst[lev]; b <= T.llast[lev]; b++) {
        for (int i = 0; i < T.nl1[b]; i++) {
          int j = T.l1[(size_t)MNL1 * b + i];
          int s = T.isrcse[2 * j], n = npts_src(j);
          const double* sp = &ss[2 * (size_t)s];
          const cdbl* qj = qp ? qp + (size_t)s * nd : nullptr;
          const cdbl* dj = dpp ? dpp + (size_t)s * nd : nullptr;
          if (A.ifpghtarg > 0) {
            int t = T.itargse[2 * b], m = npts_trg(b);
            c2d_direct(nd, sp, n, qj, dj, &ts[2 * (size_t)t], m, A.ifpghtarg,
                       &pott[(size_t)t * nd], &gradt[(size_t)t * nd], &hesst[(size_t)t * nd],
                       thresh);
          }
          if (A.ifpgh > 0) {
            int t = T.isrcse[2 * b], m = npts_src(b);
            c2d_direct(nd, sp, n, qj, dj, &ss[2 * (size_t)t], m, A.ifpgh, &pot[(size_t)t * nd],
                       &grad[(size_t)t * nd], &hess[(size_t)t * nd], thresh);
          }
        }
      }
    }
  }
  tinfo[7] = wtime() - t0;
  // scatter back to caller order (fmmcommon2d.f:56-84)
  for (int k = 0; k < ns; k++) {
    int i = T.isrc[k];
    for (int d = 0; d < nd; d++) {
      if (A.ifpgh >= 1) A.pot[(size_t)i * nd + d] = pot[(size_t)k * nd + d];
      if (A.ifpgh >= 2) A.grad[(size_t)i * nd + d] = grad[(size_t)k * nd + d];
      if (A.ifpgh >= 3) A.hess[(size_t)i * nd + d] = hess[(size_t)k * nd + d];
    }
  }
  for (int k = 0; k < nt; k++) {
    int i = T.itarg[k];
    for (int d = 0; d < nd; d++) {
      if (A.ifpghtarg >= 1) A.pottarg[(size_t)i * nd + d] = pott[(size_t)k * nd + d];
      if (A.ifpghtarg >= 2) A.gradtarg[(size_t)i * nd + d] = gradt[(size_t)k * nd + d];
      if (A.ifpghtarg >= 3) A.hesstarg[(size_t)i * nd + d] = hesst[(size_t)k * nd + d];
    }
  }
  if (A.timeinfo)
    for (int i = 0; i < 8; i++) A.timeinfo[i] = tinfo[i];
  if (keep_tree) *keep_tree = std::move(T);
  return 0;
}

// ===========================================================================
// Helmholtz (src/helmholtz/): hfmm2d low-frequency path
// ===========================================================================

// H0^(1)(z), H1^(1)(z).  The oracle evaluates them independently of the
// CUDA library: real arguments with libstdc++'s cylindrical Bessel functions,
// complex arguments with the ascending series (DLMF 10.2.2, 10.8.1) in long
// double for |z| <= 17 and the Hankel asymptotic expansion (DLMF 10.17.5)
// beyond.  (The reference uses its own hank103, src/common/hank103.f.)
typedef std::complex<long double> cld;

void hankel01_series(cld z, cld& h0, cld& h1) {
  const long double pi = 3.141592653589793238462643383279502884L;
  const long double eg = 0.577215664901532860606512090082402431L;
  cld q = -(z * z) / 4.0L;
  cld t0 = 1.0L, t1 = 1.0L;  // (-z^2/4)^k / (k!)^2 and / (k!(k+1)!)
  cld j0 = 0.0L, j1s = 0.0L, y0s = 0.0L, y1s = 0.0L;
  long double hk = 0.0L;  // harmonic number H_k
  for (int k = 0; k < 200; k++) {
    if (k > 0) {
      t0 *= q / ((long double)k * k);
      t1 *= q / ((long double)k * (k + 1));
      hk += 1.0L / k;
    }
    j0 += t0;
    j1s += t1;
    y0s += hk * t0;                               // sum H_k (-z^2/4)^k/(k!)^2
    y1s += (2 * (hk - eg) + 1.0L / (k + 1)) * t1;  // psi(k+1)+psi(k+2)
    if (k > 5 && std::abs(t0) < 1e-30L * std::abs(j0) && std::abs(t1) < 1e-30L) break;
  }
  cld lz = std::log(z / 2.0L);
  cld j1 = (z / 2.0L) * j1s;
  cld y0 = (2.0L / pi) * (lz + eg) * j0 - (2.0L / pi) * y0s;
  cld y1 = -2.0L / (pi * z) + (2.0L / pi) * lz * j1 - (z / (2.0L * pi)) * y1s;
  cld I(0.0L, 1.0L);
  h0 = j0 + I * y0;
  h1 = j1 + I * y1;
}

void hankel01_asym(cld z, cld& h0, cld& h1) {
  const long double pi = 3.141592653589793238462643383279502884L;
  cld I(0.0L, 1.0L);
  cld pre = std::sqrt(2.0L / (pi * z));
  cld out[2];
  for (int nu = 0; nu <= 1; nu++) {
    long double m = 4.0L * nu * nu;
    cld sum = 1.0L, term = 1.0L;
    long double last = 1e300L;
    for (int k = 1; k < 200; k++) {
      long double a = (m - (2.0L * k - 1) * (2.0L * k - 1)) / (k * 8.0L);
      cld nt = term * (I * a / z);
      if (std::abs(nt) > last) break;  // optimal truncation
      last = std::abs(nt);
      term = nt;
      sum += term;
      if (last < 1e-21L) break;
    }
    out[nu] = pre * std::exp(I * (z - nu * pi / 2.0L - pi / 4.0L)) * sum;
  }
  h0 = out[0];
  h1 = out[1];
}

void hankel01(cdbl z, cdbl& h0, cdbl& h1) {
  if (z.imag() == 0.0 && z.real() > 0.0) {
    double x = z.real();
    h0 = cdbl(std::cyl_bessel_j(0.0, x), std::cyl_neumann(0.0, x));
    h1 = cdbl(std::cyl_bessel_j(1.0, x), std::cyl_neumann(1.0, x));
    return;
  }
  cld zl((long double)z.real(), (long double)z.imag()), a, b;
  if (std::abs(zl) <= 17.0L)
    hankel01_series(zl, a, b);
  else
    hankel01_asym(zl, a, b);
  h0 = cdbl((double)a.real(), (double)a.imag());
  h1 = cdbl((double)b.real(), (double)b.imag());
}

// h2dall (src/helmholtz/h2dcommon.f:71-178): hvec(n) = H_n(z) rscale^n,
// n = 0..nterms, by upward recurrence from H0, H1 (zero for |z| < 1e-200).
void h2dall(int nterms, cdbl z, double rscale, cdbl* hv) {
  if (std::abs(z) < 1e-200) {
    for (int i = 0; i <= nterms; i++) hv[i] = 0.0;
    return;
  }
  cdbl h0, h1;
  hankel01(z, h0, h1);
  hv[0] = h0;
  if (nterms >= 1) hv[1] = h1 * rscale;
  double s2 = rscale * rscale;
  cdbl zinv = rscale / z;
  for (int i = 1; i < nterms; i++) hv[i + 1] = (zinv * (2.0 * i)) * hv[i] - s2 * hv[i - 1];
}

// jbessel2d (src/common/cdjseval2d.f:5-204): fjs(n) = J_n(z) / rscale^n,
// n = 0..nterms, by Miller's backward recurrence started where the forward
// recurrence exceeds 1e20, normalised with exp(-/+ i z) = sum (-/+i)^n ...
void jbessel2d(int nterms, cdbl z, double rscale, cdbl* fjs) {
  if (std::abs(z) < 1e-200) {
    fjs[0] = 1.0;
    for (int i = 1; i <= nterms; i++) fjs[i] = 0.0;
    return;
  }
  const double upb2 = 1e40, upb2inv = 1e-40;
  cdbl zinv = 1.0 / z;
  cdbl fn = 1.0, fnm1 = 0.0;
  int ntop = nterms + 10000;
  for (int i = nterms; i <= nterms + 10000; i++) {
    cdbl t = (2.0 * i) * zinv * fn - fnm1;
    if (std::norm(t) > upb2) {
      ntop = i + 1;
      break;
    }
    fnm1 = fn;
    fn = t;
  }
  std::vector<cdbl> f(ntop + 1, 0.0);
  std::vector<char> isc(ntop + 1, 0);
  f[ntop] = 0.0;
  f[ntop - 1] = 1.0;
  for (int i = ntop - 1; i >= 1; i--) {
    cdbl t = (2.0 * i) * zinv * f[i] - f[i + 1];
    f[i - 1] = t;
    if (std::norm(t) > upb2) {
      f[i] *= upb2inv;
      f[i - 1] *= upb2inv;
      isc[i] = 1;
    }
  }
  double sinv = 1.0 / rscale, sctot = 1.0;
  for (int i = 1; i <= ntop; i++) {
    sctot *= sinv;
    if (isc[i - 1]) sctot *= upb2inv;
    f[i] *= sctot;
  }
  cdbl I(0, 1);
  cdbl zmul = z.imag() < 0 ? I : -I;
  cdbl zsn = std::pow(zmul, ntop % 4);
  cdbl zmi = 1.0 / zmul;
  cdbl psi = 0.0;
  for (int i = ntop; i >= 1; i--) {
    psi = rscale * psi + f[i] * zsn;
    zsn *= zmi;
  }
  psi = 2.0 * psi * rscale + f[0];
  cdbl zs = (z.imag() < 0 ? std::exp(I * z) : std::exp(-I * z)) / psi;
  for (int i = 0; i <= nterms; i++) fjs[i] = f[i] * zs;
}

// h2dterms (src/helmholtz/h2dterms.f:35-97): first j with
// (|J_j H_j| + |J_(j-1) H_(j-1)|) |H_0| < eps (|J_0 H_0| + |J_1 H_1|).
int h2dterms(double bsize, cdbl zk, double eps, int* ier) {
  const double pi2 = 8 * std::atan(1.0);
  cdbl z1 = (zk * bsize) * 1.5;
  double rscale = 1.0;
  if (std::abs(zk * bsize) < pi2) rscale = std::abs(zk * bsize);
  const int nt = 2000;
  std::vector<cdbl> hf(nt + 1), jf(nt + 1);
  h2dall(nt, z1, rscale, hf.data());
  cdbl z2 = (zk * bsize) * (std::sqrt(2.0) / 2.0);
  jbessel2d(nt, z2, rscale, jf.data());
  double x0 = std::abs(jf[0] * hf[0]) + std::abs(jf[1] * hf[1]);
  for (int j = 2; j <= nt; j++) {
    double x1 = std::abs(jf[j] * hf[j]), x2 = std::abs(jf[j - 1] * hf[j - 1]);
    if ((x1 + x2) * std::abs(hf[0]) < eps * x0) return j + 1;
  }
  *ier = 13;
  return 10001;
}

int helm_ndiv(double eps, long ns, long nt) { return lap_ndiv(eps, ns, nt); }  // hndiv2d.f

inline void polar(double x, double y, double& r, double& th) {  // h2cart2polar
  r = std::sqrt(x * x + y * y);
  th = (x == 0 && y == 0) ? 0.0 : std::atan2(y, x);
}

// Expansions are (nd, -p:p): element (d, n) at [(n + p) * nd + d].
struct HExp {
  int p, nd;
  cdbl* a;
  cdbl& at(int n, int d) { return a[(size_t)(n + p) * nd + d]; }
};

// ctompole / dtompole (helmrouts2d.f:1383-1492): add one source's charge and
// dipole terms given jv(n) = Z_n (J or H, scaled) and zmul = exp(-i theta).
void add_src_terms(int nd, cdbl zk, double rs, cdbl zmul, const cdbl* jv, const cdbl* q,
                   const cdbl* dst, const double* dv, int ldv, HExp E) {
  cdbl I(0, 1), zinv = std::conj(zmul);
  if (q) {
    for (int d = 0; d < nd; d++) E.at(0, d) += q[d] * jv[0];
    cdbl t1 = zmul, t2 = -zinv;
    for (int n = 1; n <= E.p; n++) {
      for (int d = 0; d < nd; d++) {
        E.at(n, d) += jv[n] * t1 * q[d];
        E.at(-n, d) += jv[n] * t2 * q[d];
      }
      t1 *= zmul;
      t2 = -t2 * zinv;
    }
  }
  if (dst) {
    cdbl z3 = zinv / rs, z4 = zmul * rs, z5 = zmul / rs, z6 = zinv * rs;
    for (int d = 0; d < nd; d++) {
      double v1 = dv[d], v2 = dv[ldv + d];
      E.at(0, d) -= dst[d] * jv[1] * zk / 2.0 * rs * ((zmul + zinv) * v1 + (zmul - zinv) * I * v2);
    }
    cdbl t1 = -zmul * zk / 2.0, t2 = zinv * zk / 2.0;
    for (int n = 1; n <= E.p; n++) {
      for (int d = 0; d < nd; d++) {
        double v1 = dv[d], v2 = dv[ldv + d];
        cdbl a7 = z3 * cdbl(-v1, v2), a8 = z4 * cdbl(v1, v2), a9 = z5 * cdbl(-v1, -v2),
             a10 = z6 * cdbl(v1, -v2);
        E.at(n, d) += (jv[n - 1] * a7 + jv[n + 1] * a8) * t1 * dst[d];
        E.at(-n, d) += (jv[n - 1] * a9 + jv[n + 1] * a10) * t2 * dst[d];
      }
      t1 *= zmul;
      t2 = -t2 * zinv;
    }
  }
}

// mk_mpoleg (helmrouts2d.f): derivative expansions (x and y) of order p+1.
void mk_grad_exp(int nd, cdbl zk, double rs, HExp M, HExp X, HExp Y) {
  cdbl I(0, 1);
  cdbl s1 = zk / 2.0 / rs, s2 = zk / 2.0 * rs, s3 = zk / 2.0 / rs * I, s4 = zk / 2.0 * rs * I;
  for (int n = -X.p; n <= X.p; n++)
    for (int d = 0; d < nd; d++) X.at(n, d) = Y.at(n, d) = 0.0;
  for (int d = 0; d < nd; d++) {
    X.at(-1, d) += s1 * M.at(0, d);
    Y.at(-1, d) += s3 * M.at(0, d);
    X.at(1, d) -= s1 * M.at(0, d);
    Y.at(1, d) += s3 * M.at(0, d);
  }
  for (int i = 1; i <= M.p; i++)
    for (int d = 0; d < nd; d++) {
      X.at(i - 1, d) += s2 * M.at(i, d);
      Y.at(i - 1, d) += s4 * M.at(i, d);
      X.at(i + 1, d) -= s1 * M.at(i, d);
      Y.at(i + 1, d) += s3 * M.at(i, d);
    }
  for (int i = -M.p; i <= -1; i++)
    for (int d = 0; d < nd; d++) {
      X.at(i - 1, d) += s1 * M.at(i, d);
      Y.at(i - 1, d) += s3 * M.at(i, d);
      X.at(i + 1, d) -= s2 * M.at(i, d);
      Y.at(i + 1, d) += s4 * M.at(i, d);
    }
}

// mk_mpoleh: second derivatives (xx from x, xy from x, yy from y), order p+2.
void mk_hess_exp(int nd, cdbl zk, double rs, HExp X, HExp Y, HExp XX, HExp XY, HExp YY) {
  cdbl I(0, 1);
  cdbl s1 = zk / 2.0 / rs, s2 = zk / 2.0 * rs, s3 = zk / 2.0 / rs * I, s4 = zk / 2.0 * rs * I;
  for (int n = -XX.p; n <= XX.p; n++)
    for (int d = 0; d < nd; d++) XX.at(n, d) = XY.at(n, d) = YY.at(n, d) = 0.0;
  for (int d = 0; d < nd; d++) {
    XX.at(-1, d) += s1 * X.at(0, d);
    XY.at(-1, d) += s3 * X.at(0, d);
    YY.at(-1, d) += s3 * Y.at(0, d);
    XX.at(1, d) -= s1 * X.at(0, d);
    XY.at(1, d) += s3 * X.at(0, d);
    YY.at(1, d) += s3 * Y.at(0, d);
  }
  for (int i = 1; i <= X.p; i++)
    for (int d = 0; d < nd; d++) {
      XX.at(i - 1, d) += s2 * X.at(i, d);
      XY.at(i - 1, d) += s4 * X.at(i, d);
      YY.at(i - 1, d) += s4 * Y.at(i, d);
      XX.at(i + 1, d) -= s1 * X.at(i, d);
      XY.at(i + 1, d) += s3 * X.at(i, d);
      YY.at(i + 1, d) += s3 * Y.at(i, d);
    }
  for (int i = -X.p; i <= -1; i++)
    for (int d = 0; d < nd; d++) {
      XX.at(i - 1, d) += s1 * X.at(i, d);
      XY.at(i - 1, d) += s3 * X.at(i, d);
      YY.at(i - 1, d) += s3 * Y.at(i, d);
      XX.at(i + 1, d) -= s2 * X.at(i, d);
      XY.at(i + 1, d) += s4 * X.at(i, d);
      YY.at(i + 1, d) += s4 * Y.at(i, d);
    }
}

// mpole_evalp: sum_n E(n) mt(n) with mt(n) = (i/4) Z_|n| exp(i n theta) (-1)^... 
void eval_exp(int nd, HExp E, const cdbl* mt, int mtoff, cdbl* out) {
  cdbl I4(0, 0.25);
  for (int d = 0; d < nd; d++) out[d] += mt[mtoff] * E.at(0, d) * I4;
  for (int n = 1; n <= E.p; n++)
    for (int d = 0; d < nd; d++) out[d] += E.at(n, d) * mt[mtoff + n] + E.at(-n, d) * mt[mtoff - n];
}

// table mt(-m..m): mt(0) = Z_0, mt(+-n) = (i/4) Z_n zmul^n, (-i/4)(-zinv)^.. as mpole_evalp
void make_mt(int m, cdbl zmul, const cdbl* zv, std::vector<cdbl>& mt) {
  cdbl I4(0, 0.25);
  mt.assign(2 * m + 1, 0.0);
  mt[m] = zv[0];
  cdbl t1 = zmul * I4, t2 = -std::conj(zmul) * I4;
  for (int j = 1; j <= m; j++) {
    mt[m + j] = t1 * zv[j];
    mt[m - j] = t2 * zv[j];
    t1 *= zmul;
    t2 = -t2 * std::conj(zmul);
  }
}

// Evaluate an expansion (multipole with H, local with J) at points with
// derivatives (h2dmpeval*, h2dtaeval*; helmrouts2d.f:274-966).
void helm_eval(int nd, cdbl zk, double rs, const double* c, HExp E, bool mpole, const double* xy,
               int n, int ifpgh, cdbl* pot, cdbl* grad, cdbl* hess) {
  int p = E.p;
  double rsg = mpole ? rs : 1.0 / rs;  // mk_mpoleg scale: rscale for H, 1/rscale for J
  std::vector<cdbl> bx((2 * p + 3) * nd), by((2 * p + 3) * nd), bxx((2 * p + 5) * nd),
      bxy((2 * p + 5) * nd), byy((2 * p + 5) * nd);
  HExp X{p + 1, nd, bx.data()}, Y{p + 1, nd, by.data()};
  HExp XX{p + 2, nd, bxx.data()}, XY{p + 2, nd, bxy.data()}, YY{p + 2, nd, byy.data()};
  if (ifpgh >= 2) mk_grad_exp(nd, zk, rsg, E, X, Y);
  if (ifpgh >= 3) mk_hess_exp(nd, zk, rsg, X, Y, XX, XY, YY);
  std::vector<cdbl> zv(p + 12), mt;
  cdbl I(0, 1);
  for (int k = 0; k < n; k++) {
    double r, th;
    polar(xy[2 * k] - c[0], xy[2 * k + 1] - c[1], r, th);
    cdbl z = zk * r;
    if (mpole)
      h2dall(p + 3, z, rs, zv.data());
    else
      jbessel2d(p + 3, z, rs, zv.data());
    cdbl zmul = std::exp(I * th);
    make_mt(p + 2, zmul, zv.data(), mt);
    eval_exp(nd, E, mt.data(), p + 2, pot + (size_t)k * nd);
    if (ifpgh >= 2) {
      std::vector<cdbl> g(nd, 0.0), h(nd, 0.0);
      eval_exp(nd, X, mt.data(), p + 2, g.data());
      eval_exp(nd, Y, mt.data(), p + 2, h.data());
      for (int d = 0; d < nd; d++) {
        grad[((size_t)k * 2 + 0) * nd + d] += g[d];
        grad[((size_t)k * 2 + 1) * nd + d] += h[d];
      }
    }
    if (ifpgh >= 3) {
      std::vector<cdbl> a(nd, 0.0), b(nd, 0.0), e(nd, 0.0);
      eval_exp(nd, XX, mt.data(), p + 2, a.data());
      eval_exp(nd, XY, mt.data(), p + 2, b.data());
      eval_exp(nd, YY, mt.data(), p + 2, e.data());
      for (int d = 0; d < nd; d++) {
        hess[((size_t)k * 3 + 0) * nd + d] += a[d];
        hess[((size_t)k * 3 + 1) * nd + d] += b[d];
        hess[((size_t)k * 3 + 2) * nd + d] += e[d];
      }
    }
  }
}

// Form an expansion from sources: multipole (J, h2dformmp*) or local
// (H, h2dformta*) about c.
void helm_form(int nd, cdbl zk, double rs, const double* src, int ns, const cdbl* q,
               const cdbl* dst, const double* dv, const double* c, HExp E, bool mpole) {
  cdbl I(0, 1);
  std::vector<cdbl> zv(E.p + 12);
  for (int j = 0; j < ns; j++) {
    double r, th;
    polar(src[2 * j] - c[0], src[2 * j + 1] - c[1], r, th);
    cdbl z = zk * r;
    if (mpole)
      jbessel2d(E.p + 1, z, rs, zv.data());
    else
      h2dall(E.p + 2, z, rs, zv.data());
    cdbl zmul = std::exp(-I * th);
    add_src_terms(nd, zk, mpole ? rs : 1.0 / rs, zmul, zv.data(), q ? q + (size_t)j * nd : nullptr,
                  dst ? dst + (size_t)j * nd : nullptr, dv ? dv + (size_t)j * 2 * nd : nullptr, nd,
                  E);
  }
}

// Translation kernels table ztab(-m..m) = Z_|j| * exp(-i j theta) with the
// (-1)^j sign on negative indices (h2dmpmp / h2dlocloc / h2dmploc).
void shift_table(int m, cdbl zmul, const cdbl* zv, std::vector<cdbl>& t) {
  t.assign(2 * m + 1, 0.0);
  t[m] = zv[0];
  cdbl a = zmul, b = -std::conj(zmul);
  for (int j = 1; j <= m; j++) {
    t[m + j] = a * zv[j];
    t[m - j] = b * zv[j];
    a *= zmul;
    b = -b * std::conj(zmul);
  }
}

// h2dmpmp (helmrouts2d.f:967-1095)
void h2dmpmp(int nd, cdbl zk, double rs1, const double* c1, HExp H1, double rs2, const double* c2,
             HExp H2) {
  const double pi = 4 * std::atan(1.0);
  int p1 = H1.p, p2 = H2.p, nt = p1 + p2;
  double r, th;
  polar(c2[0] - c1[0], c2[1] - c1[1], r, th);
  th -= pi;
  std::vector<cdbl> jv(nt + 12), T;
  jbessel2d(nt + 3, zk * r, rs1, jv.data());
  cdbl I(0, 1);
  shift_table(nt, std::exp(-I * th), jv.data(), T);
  auto J = [&](int j) { return T[nt + j]; };
  for (int d = 0; d < nd; d++) H2.at(0, d) += H1.at(0, d) * J(0);
  double rsj2 = rs1 * rs1, rsj = rsj2;
  for (int j = 1; j <= p1; j++) {
    for (int d = 0; d < nd; d++) {
      H2.at(0, d) += (H1.at(j, d) * J(-j)) * rsj;
      H2.at(0, d) += (H1.at(-j, d) * J(j)) * rsj;
    }
    rsj *= rsj2;
  }
  double rsi5 = rs1 / rs2;
  for (int i = 1; i <= p2; i++) {
    for (int d = 0; d < nd; d++) {
      H2.at(i, d) += H1.at(0, d) * J(i) * rsi5;
      H2.at(-i, d) += H1.at(0, d) * J(-i) * rsi5;
    }
    rsi5 *= rs1 / rs2;
  }
  rsi5 = rs1 / rs2;
  for (int i = 1; i <= p2; i++) {
    rsj = rsj2;
    for (int j = 1; j <= std::min(p1, i); j++) {
      double fs3 = rsi5 * rsj;
      for (int d = 0; d < nd; d++) {
        H2.at(i, d) += (H1.at(j, d) * J(i - j)) * rsi5;
        H2.at(i, d) += (H1.at(-j, d) * J(i + j)) * fs3;
        H2.at(-i, d) += (H1.at(j, d) * J(-i - j)) * fs3;
        H2.at(-i, d) += (H1.at(-j, d) * J(-i + j)) * rsi5;
      }
      rsj *= rsj2;
    }
    rsj = std::pow(rsj2, i + 1);
    double fs2 = rsi5 * rsj2, fs3 = rsi5 * rsj;
    for (int j = i + 1; j <= p1; j++) {
      for (int d = 0; d < nd; d++) {
        H2.at(i, d) += (H1.at(j, d) * J(i - j)) * fs2;
        H2.at(i, d) += (H1.at(-j, d) * J(i + j)) * fs3;
        H2.at(-i, d) += (H1.at(j, d) * J(-i - j)) * fs3;
        H2.at(-i, d) += (H1.at(-j, d) * J(-i + j)) * fs2;
      }
      fs3 *= rsj2;
      fs2 *= rsj2;
    }
    rsi5 *= rs1 / rs2;
  }
}

// h2dlocloc (helmrouts2d.f:1096-1220)
void h2dlocloc(int nd, cdbl zk, double rs1, const double* c1, HExp J1, double rs2,
               const double* c2, HExp J2) {
  const double pi = 4 * std::atan(1.0);
  int p1 = J1.p, p2 = J2.p, nt = p1 + p2;
  double r, th;
  polar(c2[0] - c1[0], c2[1] - c1[1], r, th);
  th -= pi;
  std::vector<cdbl> jv(nt + 12), T;
  jbessel2d(nt + 3, zk * r, rs1, jv.data());
  cdbl I(0, 1);
  shift_table(nt, std::exp(-I * th), jv.data(), T);
  auto J = [&](int j) { return T[nt + j]; };
  for (int d = 0; d < nd; d++) J2.at(0, d) += J1.at(0, d) * J(0);
  for (int j = 1; j <= p1; j++)
    for (int d = 0; d < nd; d++) {
      J2.at(0, d) += J1.at(j, d) * J(-j);
      J2.at(0, d) += J1.at(-j, d) * J(j);
    }
  double rsi = rs1, rsi7 = rs2;
  for (int i = 1; i <= p2; i++) {
    for (int d = 0; d < nd; d++) {
      J2.at(i, d) += J1.at(0, d) * J(i) * rsi7 * rsi;
      J2.at(-i, d) += J1.at(0, d) * J(-i) * rsi7 * rsi;
    }
    rsi *= rs1;
    rsi7 *= rs2;
  }
  rsi = rs1;
  rsi7 = rs2;
  double rsi5 = rs2 / rs1;
  for (int i = 1; i <= p2; i++) {
    double fs2 = rsi5;
    if (p1 <= i) fs2 = fs2 * std::pow(rs1, 2 * (i - p1));
    for (int j = std::min(p1, i); j >= 1; j--) {
      for (int d = 0; d < nd; d++) {
        J2.at(i, d) += (J1.at(j, d) * J(i - j)) * fs2;
        J2.at(i, d) += (J1.at(-j, d) * J(i + j)) * rsi7 * rsi;
        J2.at(-i, d) += (J1.at(j, d) * J(-i - j)) * rsi7 * rsi;
        J2.at(-i, d) += (J1.at(-j, d) * J(-i + j)) * fs2;
      }
      fs2 *= rs1 * rs1;
    }
    for (int j = i + 1; j <= p1; j++) {
      for (int d = 0; d < nd; d++) {
        J2.at(i, d) += (J1.at(j, d) * J(i - j)) * rsi5;
        J2.at(i, d) += (J1.at(-j, d) * J(i + j)) * rsi7 * rsi;
        J2.at(-i, d) += (J1.at(j, d) * J(-i - j)) * rsi7 * rsi;
        J2.at(-i, d) += (J1.at(-j, d) * J(-i + j)) * rsi5;
      }
    }
    rsi *= rs1;
    rsi7 *= rs2;
    rsi5 *= rs2 / rs1;
  }
}

// h2dmploc (helmrouts2d.f:1221-1382)
void h2dmploc(int nd, cdbl zk, double rs1, const double* c1, HExp H, double rs2,
              const double* c2, HExp L) {
  const double pi = 4 * std::atan(1.0);
  int p1 = H.p, p2 = L.p, nt = p1 + p2;
  double r, th;
  polar(c2[0] - c1[0], c2[1] - c1[1], r, th);
  th -= pi;
  std::vector<cdbl> hv(nt + 12), T;
  h2dall(nt + 1, zk * r, rs1, hv.data());
  cdbl I(0, 1);
  shift_table(nt, std::exp(-I * th), hv.data(), T);
  auto Hh = [&](int j) { return T[nt + j]; };
  std::vector<cdbl> tmp((2 * p2 + 1) * nd, 0.0);
  HExp Tm{p2, nd, tmp.data()};
  std::vector<double> rs2pow(p2 + 1);
  double rfac = rs1 * rs1;
  if (p2 >= 1) rs2pow[1] = rfac;
  for (int i = 2; i <= p2; i++) rs2pow[i] = rs2pow[i - 1] * rfac;
  for (int d = 0; d < nd; d++) Tm.at(0, d) += H.at(0, d) * Hh(0);
  for (int j = 1; j <= p1; j++)
    for (int d = 0; d < nd; d++) {
      Tm.at(0, d) += H.at(j, d) * Hh(-j);
      Tm.at(0, d) += H.at(-j, d) * Hh(j);
    }
  for (int i = 1; i <= p2; i++) {
    for (int d = 0; d < nd; d++) {
      Tm.at(i, d) += H.at(0, d) * Hh(i);
      Tm.at(-i, d) += H.at(0, d) * Hh(-i);
    }
    for (int j = 1; j <= std::min(p1, i); j++)
      for (int d = 0; d < nd; d++) {
        Tm.at(i, d) += (H.at(j, d) * Hh(i - j)) * rs2pow[j];
        Tm.at(i, d) += H.at(-j, d) * Hh(i + j);
        Tm.at(-i, d) += H.at(j, d) * Hh(-i - j);
        Tm.at(-i, d) += (H.at(-j, d) * Hh(-i + j)) * rs2pow[j];
      }
    for (int j = i + 1; j <= p1; j++)
      for (int d = 0; d < nd; d++) {
        Tm.at(i, d) += (H.at(j, d) * Hh(i - j)) * rs2pow[i];
        Tm.at(i, d) += H.at(-j, d) * Hh(i + j);
        Tm.at(-i, d) += H.at(j, d) * Hh(-i - j);
        Tm.at(-i, d) += (H.at(-j, d) * Hh(-i + j)) * rs2pow[i];
      }
  }
  double f = rs2 / rs1, rs12 = f;
  for (int d = 0; d < nd; d++) L.at(0, d) += Tm.at(0, d);
  for (int i = 1; i <= p2; i++) {
    for (int d = 0; d < nd; d++) {
      L.at(i, d) += Tm.at(i, d) * rs12;
      L.at(-i, d) += Tm.at(-i, d) * rs12;
    }
    rs12 *= f;
  }
}

// Helmholtz direct interaction (helmkernels2d.f:3-904): pot += (i/4)[H0 q
// + k H1 (v.r)/r d]; gradients and Hessians as h2d_directcdh.  Pairs with
// |k r| below thresh are skipped (<= for the charge potential-only variant).
void h2d_direct(int nd, cdbl zk, const double* src, int ns, const cdbl* q, const cdbl* dst,
                const double* dv, const double* trg, int nt, int ifpgh, cdbl* pot, cdbl* grad,
                cdbl* hess, double thresh) {
  cdbl I4(0, 0.25);
  bool le = (ifpgh == 1 && q && !dst);
  for (int j = 0; j < nt; j++)
    for (int i = 0; i < ns; i++) {
      double xd = trg[2 * j] - src[2 * i], yd = trg[2 * j + 1] - src[2 * i + 1];
      double rr = xd * xd + yd * yd, r = std::sqrt(rr);
      cdbl z = zk * r;
      if (le ? (std::abs(z) <= thresh) : (std::abs(z) < thresh)) continue;
      cdbl h0, h1;
      hankel01(z, h0, h1);
      double ct = xd / r, st = yd / r;
      cdbl h2 = 2.0 * h1 / z - h0, h3 = 4.0 * h2 / z - h1;
      for (int d = 0; d < nd; d++) {
        cdbl P = 0.0, gx = 0.0, gy = 0.0, hxx = 0.0, hxy = 0.0, hyy = 0.0;
        if (q) {
          cdbl c = q[(size_t)i * nd + d];
          P += h0 * c * I4;
          cdbl cd = -h1 * (zk * c * I4 / r);
          gx += cd * xd;
          gy += cd * yd;
          cdbl ch = (zk * c * I4 / r) / rr;
          cdbl h2z = -z * h0 + 2.0 * h1;
          hxx += ch * (h2z * xd * xd - rr * h1);
          hxy += ch * (h2z * xd * yd);
          hyy += ch * (h2z * yd * yd - rr * h1);
        }
        if (dst) {
          cdbl c = dst[(size_t)i * nd + d];
          double v1 = dv[((size_t)i * 2 + 0) * nd + d], v2 = dv[((size_t)i * 2 + 1) * nd + d];
          P += h1 / r * zk * I4 * c * (xd * v1 + yd * v2);
          cdbl c2 = -zk * zk * I4 * c;
          cdbl f1 = h2 * (ct * ct - 0.5) - h0 / 2.0, f2 = h2 * ct * st,
               f3 = h2 * (st * st - 0.5) - h0 / 2.0;
          gx += c2 * f1 * v1 + c2 * f2 * v2;
          gy += c2 * f2 * v1 + c2 * f3 * v2;
          cdbl a1 = (-h1 / 2.0 * (-1.5) - h3 / 2.0 * (ct * ct - 0.5 - st * st)) * ct;
          cdbl a2 = (-h1 / 2.0 * (-0.5) - h3 / 2.0 * (1.5 * ct * ct - 0.5 * st * st)) * st;
          cdbl a3 = (-h1 / 2.0 * (-0.5) - h3 / 2.0 * (1.5 * st * st - 0.5 * ct * ct)) * ct;
          cdbl a4 = (-h1 / 2.0 * (-1.5) - h3 / 2.0 * (st * st - 0.5 - ct * ct)) * st;
          cdbl c3 = -zk * zk * zk * c * I4;
          hxx += c3 * a1 * v1 + c3 * a2 * v2;
          hxy += c3 * a2 * v1 + c3 * a3 * v2;
          hyy += c3 * a3 * v1 + c3 * a4 * v2;
        }
        pot[(size_t)j * nd + d] += P;
        if (ifpgh >= 2) {
          grad[((size_t)j * 2 + 0) * nd + d] += gx;
          grad[((size_t)j * 2 + 1) * nd + d] += gy;
        }
        if (ifpgh >= 3) {
          hess[((size_t)j * 3 + 0) * nd + d] += hxx;
          hess[((size_t)j * 3 + 1) * nd + d] += hxy;
          hess[((size_t)j * 3 + 2) * nd + d] += hyy;
        }
      }
    }
}

// hfmm2d (src/helmholtz/hfmm2d.f:19-450) and hfmm2dmain (456-1580), low
// frequency: every level where M2L runs has box size <= 16 wavelengths.
// Returns 13 if an expansion order exceeds the table, 20 when the
// high-frequency (wideband) branch would be needed.
int run_hfmm(int nd, double eps, cdbl zk, int ns, const double* src, const cdbl* charge,
             const cdbl* dipstr, const double* dipvec, int ifpgh, cdbl* pot, cdbl* grad,
             cdbl* hess, int nt, const double* targ, int ifpghtarg, cdbl* pottarg,
             cdbl* gradtarg, cdbl* hesstarg, int ndiv_in, double* timeinfo) {
  const double pi = 4 * std::atan(1.0);
  double tinfo[8] = {0};
  auto zero_out = [&]() {
    if (ifpgh >= 1) std::fill(pot, pot + (size_t)nd * ns, cdbl(0));
    if (ifpgh >= 2) std::fill(grad, grad + (size_t)2 * nd * ns, cdbl(0));
    if (ifpgh >= 3) std::fill(hess, hess + (size_t)3 * nd * ns, cdbl(0));
    if (ifpghtarg >= 1) std::fill(pottarg, pottarg + (size_t)nd * nt, cdbl(0));
    if (ifpghtarg >= 2) std::fill(gradtarg, gradtarg + (size_t)2 * nd * nt, cdbl(0));
    if (ifpghtarg >= 3) std::fill(hesstarg, hesstarg + (size_t)3 * nd * nt, cdbl(0));
  };
  if (ns <= 0) {
    zero_out();
    return 0;
  }
  int ndiv = ndiv_in > 0 ? ndiv_in : helm_ndiv(eps, ns, nt);
  Tree T;
  build_tree(src, ns, targ, nt, 0, ndiv, 51, T);
  if (T.boxsize[0] == 0.0) {
    zero_out();
    return 0;
  }
  sort_points(T, src, ns, T.isrc, T.isrcse);
  sort_points(T, targ, nt, T.itarg, T.itargse);
  compute_lists(T);
  const int nl = T.nlevels, nb = T.nboxes();
  std::vector<double> rsc(nl + 1);
  std::vector<int> nterms(nl + 1);
  int ier = 0;
  for (int l = 0; l <= nl; l++) {
    rsc[l] = std::min(std::abs(zk * T.boxsize[l] / (2.0 * pi)), 1.0);
    nterms[l] = h2dterms(T.boxsize[l], zk, eps, &ier);
  }
  if (ier) return ier;
  double zi = zk.imag();
  const double zkiup = 40.0;
  // high-frequency levels are not restated: the M2L/M2M levels must be
  // at most 16 wavelengths (hfmm2d.f:1001-1013, 1119-1124)
  for (int l = 1; l <= nl; l++) {
    double dlam = 1.0 / std::real(zk / (2 * pi));
    if (zi * T.boxsize[l] < zkiup && T.boxsize[l] / dlam > 16.0) return 20;
  }
  // expansion storage: per box (2p+1) nd complex
  std::vector<size_t> off(nb);
  size_t tot = 0;
  for (int l = 0; l <= nl; l++)
    for (int b = T.lfirst[l]; b <= T.llast[l]; b++) {
      off[b] = tot;
      tot += (size_t)(2 * nterms[l] + 1) * nd;
    }
  std::vector<cdbl> mp(tot, 0.0), lo(tot, 0.0);
  auto MP = [&](int b) { return HExp{nterms[T.ilevel[b]], nd, &mp[off[b]]}; };
  auto LO = [&](int b) { return HExp{nterms[T.ilevel[b]], nd, &lo[off[b]]}; };
  auto CEN = [&](int b) { return &T.centers[2 * (size_t)b]; };
  // sorted copies
  std::vector<double> ss(2 * (size_t)ns), ts(2 * (size_t)nt), dvs(dipstr ? 2 * (size_t)nd * ns : 0);
  std::vector<cdbl> qs(charge ? (size_t)nd * ns : 0), ds(dipstr ? (size_t)nd * ns : 0);
  for (int k = 0; k < ns; k++) {
    int i = T.isrc[k];
    ss[2 * k] = src[2 * i];
    ss[2 * k + 1] = src[2 * i + 1];
    for (int d = 0; d < nd; d++) {
      if (charge) qs[(size_t)k * nd + d] = charge[(size_t)i * nd + d];
      if (dipstr) {
        ds[(size_t)k * nd + d] = dipstr[(size_t)i * nd + d];
        dvs[((size_t)k * 2 + 0) * nd + d] = dipvec[((size_t)i * 2 + 0) * nd + d];
        dvs[((size_t)k * 2 + 1) * nd + d] = dipvec[((size_t)i * 2 + 1) * nd + d];
      }
    }
  }
  for (int k = 0; k < nt; k++) {
    int i = T.itarg[k];
    ts[2 * k] = targ[2 * i];
    ts[2 * k + 1] = targ[2 * i + 1];
  }
  const cdbl* qp = charge ? qs.data() : nullptr;
  const cdbl* dpp = dipstr ? ds.data() : nullptr;
  const double* dvp = dipstr ? dvs.data() : nullptr;
  std::vector<cdbl> po((size_t)nd * ns), gr((size_t)2 * nd * ns), he((size_t)3 * nd * ns);
  std::vector<cdbl> pt((size_t)nd * nt), gt((size_t)2 * nd * nt), ht((size_t)3 * nd * nt);
  auto nsrc = [&](int b) { return T.isrcse[2 * b + 1] - T.isrcse[2 * b]; };
  auto ntrg = [&](int b) { return T.itargse[2 * b + 1] - T.itargse[2 * b]; };
  auto has_eval = [&](int b) {
    return (ifpghtarg > 0 ? ntrg(b) : 0) + (ifpgh > 0 ? nsrc(b) : 0) > 0;
  };
  auto lev_ok = [&](int l) { return zi * T.boxsize[l] < zkiup; };
  double t0 = wtime();
  // step 1: P2M at leaves
  for (int l = 2; l <= nl; l++) {
    if (!lev_ok(l)) continue;
#pragma omp parallel for schedule(dynamic)
    for (int b = T.lfirst[l]; b <= T.llast[l]; b++) {
      int s = T.isrcse[2 * b];
      if (T.nchild[b] == 0 && nsrc(b) > 0)
        helm_form(nd, zk, rsc[l], &ss[2 * (size_t)s], nsrc(b), qp ? qp + (size_t)s * nd : nullptr,
                  dpp ? dpp + (size_t)s * nd : nullptr, dvp ? dvp + (size_t)s * 2 * nd : nullptr,
                  CEN(b), MP(b), true);
    }
  }
  tinfo[0] = wtime() - t0;
  // step 2: P2L from list 4
  t0 = wtime();
  for (int l = 2; l <= nl; l++) {
    if (!lev_ok(l)) continue;
#pragma omp parallel for schedule(dynamic)
    for (int b = T.lfirst[l]; b <= T.llast[l]; b++) {
      if (!has_eval(b)) continue;
      for (int i = 0; i < T.nl4[b]; i++) {
        int j = T.l4[(size_t)MNL4 * b + i];
        int s = T.isrcse[2 * j];
        helm_form(nd, zk, rsc[l], &ss[2 * (size_t)s], nsrc(j), qp ? qp + (size_t)s * nd : nullptr,
                  dpp ? dpp + (size_t)s * nd : nullptr, dvp ? dvp + (size_t)s * 2 * nd : nullptr,
                  CEN(b), LO(b), false);
      }
    }
  }
  tinfo[1] = wtime() - t0;
  // step 3: M2M
  t0 = wtime();
  for (int l = nl - 1; l >= 1; l--) {
    if (!lev_ok(l)) continue;
#pragma omp parallel for schedule(dynamic)
    for (int b = T.lfirst[l]; b <= T.llast[l]; b++)
      for (int i = 0; i < T.nchild[b]; i++) {
        int c = T.ichild[4 * b + i];
        if (nsrc(c) > 0) h2dmpmp(nd, zk, rsc[l + 1], CEN(c), MP(c), rsc[l], CEN(b), MP(b));
      }
  }
  tinfo[2] = wtime() - t0;
  // step 4: M2L
  t0 = wtime();
  for (int l = 2; l <= nl; l++) {
    if (!lev_ok(l)) continue;
#pragma omp parallel for schedule(dynamic)
    for (int b = T.lfirst[l]; b <= T.llast[l]; b++) {
      if (!has_eval(b)) continue;
      for (int i = 0; i < T.nl2[b]; i++) {
        int j = T.l2[(size_t)MNL2 * b + i];
        h2dmploc(nd, zk, rsc[l], CEN(j), MP(j), rsc[l], CEN(b), LO(b));
      }
    }
  }
  tinfo[3] = wtime() - t0;
  // step 5: L2L
  t0 = wtime();
  for (int l = 1; l <= nl - 1; l++) {
    if (!lev_ok(l)) continue;
#pragma omp parallel for schedule(dynamic)
    for (int b = T.lfirst[l]; b <= T.llast[l]; b++) {
      if (!has_eval(b)) continue;
      for (int i = 0; i < T.nchild[b]; i++) {
        int c = T.ichild[4 * b + i];
        h2dlocloc(nd, zk, rsc[l], CEN(b), LO(b), rsc[l + 1], CEN(c), LO(c));
      }
    }
  }
  tinfo[4] = wtime() - t0;
  // step 6: M2P from list 3
  t0 = wtime();
  for (int l = 1; l <= nl - 1; l++) {
    if (!lev_ok(l + 1)) continue;
#pragma omp parallel for schedule(dynamic)
    for (int b = T.lfirst[l]; b <= T.llast[l]; b++)
      for (int i = 0; i < T.nl3[b]; i++) {
        int j = T.l3[(size_t)MNL3 * b + i];
        if (ifpghtarg > 0) {
          int s = T.itargse[2 * b];
          helm_eval(nd, zk, rsc[l + 1], CEN(j), MP(j), true, &ts[2 * (size_t)s], ntrg(b),
                    ifpghtarg, &pt[(size_t)s * nd], &gt[(size_t)s * 2 * nd], &ht[(size_t)s * 3 * nd]);
        }
        if (ifpgh > 0) {
          int s = T.isrcse[2 * b];
          helm_eval(nd, zk, rsc[l + 1], CEN(j), MP(j), true, &ss[2 * (size_t)s], nsrc(b), ifpgh,
                    &po[(size_t)s * nd], &gr[(size_t)s * 2 * nd], &he[(size_t)s * 3 * nd]);
        }
      }
  }
  tinfo[5] = wtime() - t0;
  // step 7: L2P at leaves
  t0 = wtime();
  for (int l = 0; l <= nl; l++) {
    if (!lev_ok(l)) continue;
#pragma omp parallel for schedule(dynamic)
    for (int b = T.lfirst[l]; b <= T.llast[l]; b++) {
      if (T.nchild[b] != 0) continue;
      if (ifpghtarg > 0) {
        int s = T.itargse[2 * b];
        helm_eval(nd, zk, rsc[l], CEN(b), LO(b), false, &ts[2 * (size_t)s], ntrg(b), ifpghtarg,
                  &pt[(size_t)s * nd], &gt[(size_t)s * 2 * nd], &ht[(size_t)s * 3 * nd]);
      }
      if (ifpgh > 0) {
        int s = T.isrcse[2 * b];
        helm_eval(nd, zk, rsc[l], CEN(b), LO(b), false, &ss[2 * (size_t)s], nsrc(b), ifpgh,
                  &po[(size_t)s * nd], &gr[(size_t)s * 2 * nd], &he[(size_t)s * 3 * nd]);
      }
    }
  }
  tinfo[6] = wtime() - t0;
  // step 8: P2P
  t0 = wtime();
  double thresh = std::abs(zk) * T.boxsize[0] * std::pow(2.0, -51);
  for (int l = 0; l <= nl; l++) {
#pragma omp parallel for schedule(dynamic)
    for (int b = T.lfirst[l]; b <= T.llast[l]; b++)
      for (int i = 0; i < T.nl1[b]; i++) {
        int j = T.l1[(size_t)MNL1 * b + i];
        int s = T.isrcse[2 * j], n = nsrc(j);
        const cdbl* qj = qp ? qp + (size_t)s * nd : nullptr;
        const cdbl* dj = dpp ? dpp + (size_t)s * nd : nullptr;
        const double* vj = dvp ? dvp + (size_t)s * 2 * nd : nullptr;
        if (ifpghtarg > 0) {
          int t = T.itargse[2 * b];
          h2d_direct(nd, zk, &ss[2 * (size_t)s], n, qj, dj, vj, &ts[2 * (size_t)t], ntrg(b),
                     ifpghtarg, &pt[(size_t)t * nd], &gt[(size_t)t * 2 * nd],
                     &ht[(size_t)t * 3 * nd], thresh);
        }
        if (ifpgh > 0) {
          int t = T.isrcse[2 * b];
          h2d_direct(nd, zk, &ss[2 * (size_t)s], n, qj, dj, vj, &ss[2 * (size_t)t], nsrc(b), ifpgh,
                     &po[(size_t)t * nd], &gr[(size_t)t * 2 * nd], &he[(size_t)t * 3 * nd],
                     thresh);
        }
      }
  }
  tinfo[7] = wtime() - t0;
  for (int k = 0; k < ns; k++) {
    int i = T.isrc[k];
    for (int d = 0; d < nd; d++) {
      if (ifpgh >= 1) pot[(size_t)i * nd + d] = po[(size_t)k * nd + d];
      for (int c = 0; c < 2 && ifpgh >= 2; c++)
        grad[((size_t)i * 2 + c) * nd + d] = gr[((size_t)k * 2 + c) * nd + d];
      for (int c = 0; c < 3 && ifpgh >= 3; c++)
        hess[((size_t)i * 3 + c) * nd + d] = he[((size_t)k * 3 + c) * nd + d];
    }
  }
  for (int k = 0; k < nt; k++) {
    int i = T.itarg[k];
    for (int d = 0; d < nd; d++) {
      if (ifpghtarg >= 1) pottarg[(size_t)i * nd + d] = pt[(size_t)k * nd + d];
      for (int c = 0; c < 2 && ifpghtarg >= 2; c++)
        gradtarg[((size_t)i * 2 + c) * nd + d] = gt[((size_t)k * 2 + c) * nd + d];
      for (int c = 0; c < 3 && ifpghtarg >= 3; c++)
        hesstarg[((size_t)i * 3 + c) * nd + d] = ht[((size_t)k * 3 + c) * nd + d];
    }
  }
  if (timeinfo)
    for (int i = 0; i < 8; i++) timeinfo[i] = tinfo[i];
  return 0;
}

// Output unpacking shared by lfmm2d / rfmm2d:
// pot = Re, grad = (Re g, -Im g), hess = (Re h, -Im h, -Re h)
// (lfmm2d.f:169-223, rfmm2d.f:158-212)

}  // namespace

// ===========================================================================
// C ABI of the oracle (used only by tests/ and bench.py via ctypes)
// ===========================================================================
extern "C" {

int orc_num_threads() {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

void orc_set_num_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

int orc_lap_ndiv(double eps) { return lap_ndiv(eps, 0, 0); }
int orc_lap_nterms(double eps) { return lap_nterms(eps); }

// Tree handle for structural parity tests.
void* orc_tree_new(const double* src, int ns, const double* targ, int nt, int idivflag, int ndiv,
                   int nlmax, int* nlevels, int* nboxes) {
  Tree* T = new Tree();
  build_tree(src, ns, targ, nt, idivflag, ndiv, nlmax, *T);
  sort_points(*T, src, ns, T->isrc, T->isrcse);
  sort_points(*T, targ, nt, T->itarg, T->itargse);
  compute_lists(*T);
  *nlevels = T->nlevels;
  *nboxes = T->nboxes();
  return T;
}

void orc_tree_get(void* h, int* laddr, int* ilevel, int* iparent, int* nchild, int* ichild,
                  int* ncoll, int* coll, double* centers, double* boxsize, int* isrc, int* isrcse,
                  int* itarg, int* itargse) {
  Tree* T = (Tree*)h;
  int nb = T->nboxes();
  for (int l = 0; l <= T->nlevels; l++) {
    laddr[2 * l] = T->lfirst[l];
    laddr[2 * l + 1] = T->llast[l];
  }
  std::memcpy(ilevel, T->ilevel.data(), sizeof(int) * nb);
  std::memcpy(iparent, T->iparent.data(), sizeof(int) * nb);
  std::memcpy(nchild, T->nchild.data(), sizeof(int) * nb);
  std::memcpy(ichild, T->ichild.data(), sizeof(int) * 4 * nb);
  std::memcpy(ncoll, T->ncoll.data(), sizeof(int) * nb);
  std::memcpy(coll, T->coll.data(), sizeof(int) * 9 * nb);
  std::memcpy(centers, T->centers.data(), sizeof(double) * 2 * nb);
  std::memcpy(boxsize, T->boxsize.data(), sizeof(double) * (T->nlevels + 1));
  std::memcpy(isrc, T->isrc.data(), sizeof(int) * T->isrc.size());
  std::memcpy(isrcse, T->isrcse.data(), sizeof(int) * 2 * nb);
  std::memcpy(itarg, T->itarg.data(), sizeof(int) * T->itarg.size());
  std::memcpy(itargse, T->itargse.data(), sizeof(int) * 2 * nb);
}

void orc_tree_lists(void* h, int* nl1, int* l1, int* nl2, int* l2, int* nl3, int* l3, int* nl4,
                    int* l4) {
  Tree* T = (Tree*)h;
  int nb = T->nboxes();
  std::memcpy(nl1, T->nl1.data(), sizeof(int) * nb);
  std::memcpy(l1, T->l1.data(), sizeof(int) * MNL1 * nb);
  std::memcpy(nl2, T->nl2.data(), sizeof(int) * nb);
  std::memcpy(l2, T->l2.data(), sizeof(int) * MNL2 * nb);
  std::memcpy(nl3, T->nl3.data(), sizeof(int) * nb);
  std::memcpy(l3, T->l3.data(), sizeof(int) * MNL3 * nb);
  std::memcpy(nl4, T->nl4.data(), sizeof(int) * nb);
  std::memcpy(l4, T->l4.data(), sizeof(int) * MNL4 * nb);
}

void orc_tree_free(void* h) { delete (Tree*)h; }

// cfmm2d (cfmm2d.f:23-26) with the *_ndiv tuning arguments
// (cfmm2d_ndiv.f:23-26); ndiv <= 0 selects the lndiv2d table.
void orc_cfmm2d(int nd, double eps, int ns, const double* sources, int ifcharge,
                const double* charge, int ifdipole, const double* dipstr, int ifpgh, double* pot,
                double* grad, double* hess, int nt, const double* targ, int ifpghtarg,
                double* pottarg, double* gradtarg, double* hesstarg, int ndiv, int idivflag,
                int ifnear, double* timeinfo, int* ier) {
  CfmmArgs A{nd, eps, ns, sources, ifcharge, (const cdbl*)charge, ifdipole, (const cdbl*)dipstr,
             ifpgh, (cdbl*)pot, (cdbl*)grad, (cdbl*)hess, nt, targ, ifpghtarg, (cdbl*)pottarg,
             (cdbl*)gradtarg, (cdbl*)hesstarg, ndiv, idivflag, ifnear, timeinfo};
  *ier = run_cfmm(A, nullptr);
}

// lfmm2d (lfmm2d.f:29-226): complex densities split into two Cauchy
// densities, dipole -> -(v1 + i v2) dipstr.  grad (nd,2,n), hess (nd,3,n).
void orc_lfmm2d(int nd, double eps, int ns, const double* sources, int ifcharge,
                const double* charge, int ifdipole, const double* dipstr, const double* dipvec,
                int ifpgh, double* pot, double* grad, double* hess, int nt, const double* targ,
                int ifpghtarg, double* pottarg, double* gradtarg, double* hesstarg, int ndiv,
                double* timeinfo, int* ier) {
  const cdbl* q = (const cdbl*)charge;
  const cdbl* dps = (const cdbl*)dipstr;
  int nd2 = 2 * nd;
  std::vector<cdbl> q1(ifcharge ? (size_t)nd2 * ns : 0), d1(ifdipole ? (size_t)nd2 * ns : 0);
  for (int i = 0; i < ns; i++)
    for (int j = 0; j < nd; j++) {
      if (ifcharge) {
        q1[(size_t)i * nd2 + 2 * j] = q[(size_t)i * nd + j].real();
        q1[(size_t)i * nd2 + 2 * j + 1] = q[(size_t)i * nd + j].imag();
      }
      if (ifdipole) {
        cdbl v(dipvec[((size_t)i * 2 + 0) * nd + j], dipvec[((size_t)i * 2 + 1) * nd + j]);
        cdbl zt = -v;
        d1[(size_t)i * nd2 + 2 * j] = dps[(size_t)i * nd + j].real() * zt;
        d1[(size_t)i * nd2 + 2 * j + 1] = dps[(size_t)i * nd + j].imag() * zt;
      }
    }
  std::vector<cdbl> p1((size_t)nd2 * ns), g1((size_t)nd2 * ns), h1((size_t)nd2 * ns);
  std::vector<cdbl> pt1((size_t)nd2 * nt), gt1((size_t)nd2 * nt), ht1((size_t)nd2 * nt);
  CfmmArgs A{nd2, eps, ns, sources, ifcharge, q1.data(), ifdipole, d1.data(), ifpgh, p1.data(),
             g1.data(), h1.data(), nt, targ, ifpghtarg, pt1.data(), gt1.data(), ht1.data(), ndiv,
             0, 1, timeinfo};
  *ier = run_cfmm(A, nullptr);
  cdbl I(0, 1);
  auto unpack = [&](int n, int ifl, const std::vector<cdbl>& P1, const std::vector<cdbl>& G1,
                    const std::vector<cdbl>& H1, double* po, double* gr, double* he) {
    cdbl* P = (cdbl*)po;
    cdbl* G = (cdbl*)gr;
    cdbl* H = (cdbl*)he;
    for (int i = 0; i < n; i++)
      for (int j = 0; j < nd; j++) {
        const cdbl a = P1[(size_t)i * nd2 + 2 * j], b = P1[(size_t)i * nd2 + 2 * j + 1];
        if (ifl >= 1) P[(size_t)i * nd + j] = a.real() + I * b.real();
        if (ifl >= 2) {
          cdbl ga = G1[(size_t)i * nd2 + 2 * j], gb = G1[(size_t)i * nd2 + 2 * j + 1];
          G[((size_t)i * 2 + 0) * nd + j] = ga.real() + I * gb.real();
          G[((size_t)i * 2 + 1) * nd + j] = -ga.imag() - I * gb.imag();
        }
        if (ifl >= 3) {
          cdbl ha = H1[(size_t)i * nd2 + 2 * j], hb = H1[(size_t)i * nd2 + 2 * j + 1];
          H[((size_t)i * 3 + 0) * nd + j] = ha.real() + I * hb.real();
          H[((size_t)i * 3 + 1) * nd + j] = -ha.imag() - I * hb.imag();
          H[((size_t)i * 3 + 2) * nd + j] = -(ha.real() + I * hb.real());
        }
      }
  };
  unpack(ns, ifpgh, p1, g1, h1, pot, grad, hess);
  unpack(nt, ifpghtarg, pt1, gt1, ht1, pottarg, gradtarg, hesstarg);
}

// rfmm2d (rfmm2d.f:27-215): real densities through cfmm2d with the same nd.
void orc_rfmm2d(int nd, double eps, int ns, const double* sources, int ifcharge,
                const double* charge, int ifdipole, const double* dipstr, const double* dipvec,
                int ifpgh, double* pot, double* grad, double* hess, int nt, const double* targ,
                int ifpghtarg, double* pottarg, double* gradtarg, double* hesstarg, int ndiv,
                double* timeinfo, int* ier) {
  std::vector<cdbl> q1(ifcharge ? (size_t)nd * ns : 0), d1(ifdipole ? (size_t)nd * ns : 0);
  for (int i = 0; i < ns; i++)
    for (int j = 0; j < nd; j++) {
      if (ifcharge) q1[(size_t)i * nd + j] = charge[(size_t)i * nd + j];
      if (ifdipole) {
        cdbl v(dipvec[((size_t)i * 2 + 0) * nd + j], dipvec[((size_t)i * 2 + 1) * nd + j]);
        d1[(size_t)i * nd + j] = dipstr[(size_t)i * nd + j] * (-v);
      }
    }
  std::vector<cdbl> p1((size_t)nd * ns), g1((size_t)nd * ns), h1((size_t)nd * ns);
  std::vector<cdbl> pt1((size_t)nd * nt), gt1((size_t)nd * nt), ht1((size_t)nd * nt);
  CfmmArgs A{nd, eps, ns, sources, ifcharge, q1.data(), ifdipole, d1.data(), ifpgh, p1.data(),
             g1.data(), h1.data(), nt, targ, ifpghtarg, pt1.data(), gt1.data(), ht1.data(), ndiv,
             0, 1, timeinfo};
  *ier = run_cfmm(A, nullptr);
  auto unpack = [&](int n, int ifl, const std::vector<cdbl>& P1, const std::vector<cdbl>& G1,
                    const std::vector<cdbl>& H1, double* P, double* G, double* H) {
    for (int i = 0; i < n; i++)
      for (int j = 0; j < nd; j++) {
        size_t k = (size_t)i * nd + j;
        if (ifl >= 1) P[k] = P1[k].real();
        if (ifl >= 2) {
          G[((size_t)i * 2 + 0) * nd + j] = G1[k].real();
          G[((size_t)i * 2 + 1) * nd + j] = -G1[k].imag();
        }
        if (ifl >= 3) {
          H[((size_t)i * 3 + 0) * nd + j] = H1[k].real();
          H[((size_t)i * 3 + 1) * nd + j] = -H1[k].imag();
          H[((size_t)i * 3 + 2) * nd + j] = -H1[k].real();
        }
      }
  };
  unpack(ns, ifpgh, p1, g1, h1, pot, grad, hess);
  unpack(nt, ifpghtarg, pt1, gt1, ht1, pottarg, gradtarg, hesstarg);
}

// Direct sums (cauchykernels2d.f, lapkernels2d.f, rlapkernels2d.f).
// Outputs are overwritten (zeroed first).  OpenMP over targets.
void orc_c2ddir(int nd, const double* src, int ns, const double* charge, const double* dipstr,
                const double* trg, int nt, int ifpgh, double* pot, double* grad, double* hess,
                double thresh) {
  const cdbl* q = (const cdbl*)charge;
  const cdbl* dp = (const cdbl*)dipstr;
  cdbl* P = (cdbl*)pot;
  cdbl* G = (cdbl*)grad;
  cdbl* H = (cdbl*)hess;
  std::fill(P, P + (size_t)nd * nt, cdbl(0));
  if (ifpgh >= 2) std::fill(G, G + (size_t)nd * nt, cdbl(0));
  if (ifpgh >= 3) std::fill(H, H + (size_t)nd * nt, cdbl(0));
#pragma omp parallel for schedule(static)
  for (int j = 0; j < nt; j++)
    c2d_direct(nd, src, ns, q, dp, trg + 2 * (size_t)j, 1, ifpgh, P + (size_t)j * nd,
               ifpgh >= 2 ? G + (size_t)j * nd : nullptr, ifpgh >= 3 ? H + (size_t)j * nd : nullptr,
               thresh);
}

// Laplace form: pot += q log r - d (v.(x-y))/r^2 (lapkernels2d.f:590-689);
// grad (nd,2,nt), hess (nd,3,nt) = (xx, xy, yy).
void orc_l2ddir(int nd, const double* src, int ns, const double* charge, const double* dipstr,
                const double* dipvec, const double* trg, int nt, int ifpgh, double* pot,
                double* grad, double* hess, double thresh) {
  const cdbl* q = (const cdbl*)charge;
  const cdbl* dp = (const cdbl*)dipstr;
  cdbl* P = (cdbl*)pot;
  cdbl* G = (cdbl*)grad;
  cdbl* H = (cdbl*)hess;
  double th2 = thresh * thresh;
#pragma omp parallel for schedule(static)
  for (int j = 0; j < nt; j++) {
    std::vector<cdbl> pt(nd, 0.0), gx(nd, 0.0), gy(nd, 0.0), hxx(nd, 0.0), hxy(nd, 0.0),
        hyy(nd, 0.0);
    for (int i = 0; i < ns; i++) {
      double x = trg[2 * j] - src[2 * i], y = trg[2 * j + 1] - src[2 * i + 1];
      double rr = x * x + y * y;
      // strict comparison only for the charge variants with derivatives
      // (lapkernels2d.f:56,126,212,293,372,469,567,651,760)
      bool skip = (q && ifpgh >= 2) ? (rr < th2) : (rr <= th2);
      if (skip) continue;
      double lg = std::log(rr) / 2, r2 = rr * rr, r3 = r2 * rr;
      // first derivatives of log r
      double dx = x / rr, dy = y / rr;
      // second derivatives of log r
      double dxx = (rr - 2 * x * x) / r2, dxy = -2 * x * y / r2, dyy = (rr - 2 * y * y) / r2;
      // third derivatives of log r
      double dxxx = (-6 * x * rr + 8 * x * x * x) / r3;
      double dxxy = (-2 * y * rr + 8 * x * x * y) / r3;
      double dxyy = (-2 * x * rr + 8 * x * y * y) / r3;
      double dyyy = (-6 * y * rr + 8 * y * y * y) / r3;
      for (int d = 0; d < nd; d++) {
        if (q) {
          cdbl c = q[(size_t)i * nd + d];
          pt[d] += lg * c;
          gx[d] += dx * c;
          gy[d] += dy * c;
          hxx[d] += dxx * c;
          hxy[d] += dxy * c;
          hyy[d] += dyy * c;
        }
        if (dp) {
          cdbl d1 = dp[(size_t)i * nd + d] * dipvec[((size_t)i * 2 + 0) * nd + d];
          cdbl d2 = dp[(size_t)i * nd + d] * dipvec[((size_t)i * 2 + 1) * nd + d];
          // potential of a dipole is -v . grad_y log|x-y| = -(v . grad_x log r)
          pt[d] += -(d1 * dx + d2 * dy);
          gx[d] += -(d1 * dxx + d2 * dxy);
          gy[d] += -(d1 * dxy + d2 * dyy);
          hxx[d] += -(d1 * dxxx + d2 * dxxy);
          hxy[d] += -(d1 * dxxy + d2 * dxyy);
          hyy[d] += -(d1 * dxyy + d2 * dyyy);
        }
      }
    }
    for (int d = 0; d < nd; d++) {
      P[(size_t)j * nd + d] = pt[d];
      if (ifpgh >= 2) {
        G[((size_t)j * 2 + 0) * nd + d] = gx[d];
        G[((size_t)j * 2 + 1) * nd + d] = gy[d];
      }
      if (ifpgh >= 3) {
        H[((size_t)j * 3 + 0) * nd + d] = hxx[d];
        H[((size_t)j * 3 + 1) * nd + d] = hxy[d];
        H[((size_t)j * 3 + 2) * nd + d] = hyy[d];
      }
    }
  }
}

// Real Laplace form (rlapkernels2d.f): same formulas with real densities.
void orc_r2ddir(int nd, const double* src, int ns, const double* charge, const double* dipstr,
                const double* dipvec, const double* trg, int nt, int ifpgh, double* pot,
                double* grad, double* hess, double thresh) {
  std::vector<cdbl> qc(charge ? (size_t)nd * ns : 0), dc(dipstr ? (size_t)nd * ns : 0);
  for (size_t k = 0; k < qc.size(); k++) qc[k] = charge[k];
  for (size_t k = 0; k < dc.size(); k++) dc[k] = dipstr[k];
  std::vector<cdbl> P((size_t)nd * nt), G((size_t)nd * 2 * nt), H((size_t)nd * 3 * nt);
  orc_l2ddir(nd, src, ns, charge ? (double*)qc.data() : nullptr,
             dipstr ? (double*)dc.data() : nullptr, dipvec, trg, nt, ifpgh, (double*)P.data(),
             (double*)G.data(), (double*)H.data(), thresh);
  for (size_t k = 0; k < (size_t)nd * nt; k++) pot[k] = P[k].real();
  if (ifpgh >= 2)
    for (size_t k = 0; k < (size_t)nd * 2 * nt; k++) grad[k] = G[k].real();
  if (ifpgh >= 3)
    for (size_t k = 0; k < (size_t)nd * 3 * nt; k++) hess[k] = H[k].real();
}

// hfmm2d (src/helmholtz/hfmm2d.f:19-22); zk as (re, im).
void orc_hfmm2d(int nd, double eps, double zkr, double zki, int ns, const double* sources,
                int ifcharge, const double* charge, int ifdipole, const double* dipstr,
                const double* dipvec, int ifpgh, double* pot, double* grad, double* hess, int nt,
                const double* targ, int ifpghtarg, double* pottarg, double* gradtarg,
                double* hesstarg, int ndiv, double* timeinfo, int* ier) {
  *ier = run_hfmm(nd, eps, cdbl(zkr, zki), ns, sources, ifcharge ? (const cdbl*)charge : nullptr,
                  ifdipole ? (const cdbl*)dipstr : nullptr, ifdipole ? dipvec : nullptr, ifpgh,
                  (cdbl*)pot, (cdbl*)grad, (cdbl*)hess, nt, targ, ifpghtarg, (cdbl*)pottarg,
                  (cdbl*)gradtarg, (cdbl*)hesstarg, ndiv, timeinfo);
}

// Helmholtz direct sum (helmkernels2d.f); outputs overwritten.
void orc_h2ddir(int nd, double zkr, double zki, const double* src, int ns, const double* charge,
                const double* dipstr, const double* dipvec, const double* trg, int nt, int ifpgh,
                double* pot, double* grad, double* hess, double thresh) {
  cdbl zk(zkr, zki);
  cdbl* P = (cdbl*)pot;
  cdbl* G = (cdbl*)grad;
  cdbl* H = (cdbl*)hess;
  std::fill(P, P + (size_t)nd * nt, cdbl(0));
  if (ifpgh >= 2) std::fill(G, G + (size_t)2 * nd * nt, cdbl(0));
  if (ifpgh >= 3) std::fill(H, H + (size_t)3 * nd * nt, cdbl(0));
#pragma omp parallel for schedule(static)
  for (int j = 0; j < nt; j++)
    h2d_direct(nd, zk, src, ns, (const cdbl*)charge, (const cdbl*)dipstr, dipvec,
               trg + 2 * (size_t)j, 1, ifpgh, P + (size_t)j * nd,
               ifpgh >= 2 ? G + (size_t)j * 2 * nd : nullptr,
               ifpgh >= 3 ? H + (size_t)j * 3 * nd : nullptr, thresh);
}

// H0, H1 and the helpers' sequences for the fixture tests.
void orc_hankel01(double zr, double zi, double* h0h1) {
  cdbl a, b;
  hankel01(cdbl(zr, zi), a, b);
  h0h1[0] = a.real();
  h0h1[1] = a.imag();
  h0h1[2] = b.real();
  h0h1[3] = b.imag();
}
void orc_jbessel2d(int nterms, double zr, double zi, double rscale, double* out) {
  jbessel2d(nterms, cdbl(zr, zi), rscale, (cdbl*)out);
}
void orc_h2dall(int nterms, double zr, double zi, double rscale, double* out) {
  h2dall(nterms, cdbl(zr, zi), rscale, (cdbl*)out);
}
int orc_h2dterms(double bsize, double zkr, double zki, double eps) {
  int ier = 0;
  return h2dterms(bsize, cdbl(zkr, zki), eps, &ier);
}

// LAPACK dlaran (src/common/dlaran.f) behind hkrand (src/common/hkrand.f):
// multiplicative congruential generator mod 2^48 in four 12-bit limbs.
static int g_seed[4] = {0, 0, 0, 1};
void orc_hkrand_seed(int s) {
  g_seed[0] = g_seed[1] = g_seed[2] = 0;
  g_seed[3] = (2 * s + 1) % 4096;
}
void orc_hkrand_fill(double* out, long n) {
  const int M1 = 494, M2 = 322, M3 = 2508, M4 = 2549, IPW2 = 4096;
  const double R = 1.0 / IPW2;
  for (long k = 0; k < n; k++) {
    int it4 = g_seed[3] * M4;
    int it3 = it4 / IPW2;
    it4 -= IPW2 * it3;
    it3 += g_seed[2] * M4 + g_seed[3] * M3;
    int it2 = it3 / IPW2;
    it3 -= IPW2 * it2;
    it2 += g_seed[1] * M4 + g_seed[2] * M3 + g_seed[3] * M2;
    int it1 = it2 / IPW2;
    it2 -= IPW2 * it1;
    it1 += g_seed[0] * M4 + g_seed[1] * M3 + g_seed[2] * M2 + g_seed[3] * M1;
    it1 %= IPW2;
    g_seed[0] = it1;
    g_seed[1] = it2;
    g_seed[2] = it3;
    g_seed[3] = it4;
    out[k] = R * ((double)it1 + R * ((double)it2 + R * ((double)it3 + R * (double)it4)));
  }
}

}  // extern "C"
