// tree_oracle.cpp -- CPU restatement of TREE's force hot path (oracle).
//
// TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA path and
// the timed CPU baseline ("port" of the reference); it is never linked into
// the product library and nothing in tree_b200/ may call it.
//
// PARITY STATUS: unpinned by the reference itself.  The reference is Fortran90
// + MPI (no compiler for it exists on this image) and ships no tests, inputs or
// golden vectors.  This restatement is pinned instead by project-made known
// answers: analytic two-body forces/energies, hand-computed one-level moments of
// a small tree, and the theta->0 limit against the direct sum (tests/).
//
// What it restates (file:line are paths inside hpjeonGIT/TREE):
//   * tree build      BuildLocalTree tree.f90:39-100, Insert_Tree_e 103-274,
//                     Insert_Tree_i 277-447 (serial recursive insertion,
//                     one particle per leaf, one tree per species,
//                     anisotropic root box, children at centre +-0.25*lx).
//   * upward pass     PSeudoE tree.f90:450-553, PSeudoI 556-659 (one level
//                     deep: charge centre, dx, D, Q, QQ from child centres).
//   * walks           LocalCoulombSum tree.f90:662-717, Search_Tree_ee 721-817,
//                     _ie 820-921, _ei 925-1027, _ii 1030-1133 (recursive,
//                     children visited 1..8, OpenMP over targets).
//   * integrator      VVerletNotemp1 vverlet.f90:9-44, VVerletNotemp2 49-112.
//   * energy          TEMPORAL sample.f90:77-91.
// Every floating-point expression keeps the reference's evaluation order
// (Fortran a**2 -> a*a, a**3 -> (a*a)*a, left-to-right sums) and the file is
// compiled with -ffp-contract=off so no FMA contraction changes rounding.
//
// Documented deviations from the Fortran (each is a reference bug or an
// undefined value, not a change of method):
//   1. e-i leaf pairs at r == 0: the reference evaluates 0/0 (tree.f90:905-913,
//      1010-1018).  Here: force 0, Epot += 0.5*ff*(1/rs) (the r->0 limit of
//      (1-exp(-r/rs))/r).
//   2. Root qeff is never initialised in the reference (tree.f90:64-65 vs
//      131); here it is -Ne / +Ni (what a zeroed allocation gives).
//   3. RDF_ei: Search_Tree_ie increments the shared NS%RDF_ei inside an OpenMP
//      loop (tree.f90:918, a data race).  Here both the ie and ei passes add to
//      one reduced histogram, i.e. every e-i leaf pair is counted twice, which
//      is what the race-free reference would produce.
//   4. Identical same-species positions recurse forever in Insert_Tree_*
//      (tree.f90:128-273).  Here insertion stops at ORACLE_MAX_DEPTH and the
//      call returns ORACLE_ERR_DEPTH.
//
// Additional physics mode (no reference code; the erf-Kelbg pair law the
// device paths also carry):
//   KELBG: every leaf pair uses V = q_i q_j eps / r [1 - exp(-x^2) + sqrt(pi)
//   x erfc(x)], x = r / lambda_ij, F = q_i q_j eps (1 - exp(-x^2)) rhat / r^2;
//   self pairs are excluded by index; the far field is the reference's
//   Coulomb multipole unchanged.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>
#include <chrono>
#include <omp.h>

namespace {

constexpr double kEps = 0.0014399835661145824;  // data.f90:40, eV*um
constexpr int kNdist = 10000;                    // data.f90:38
constexpr int ORACLE_MAX_DEPTH = 200;
constexpr int ORACLE_ERR_DEPTH = -2;
constexpr int ORACLE_ERR_ARG = -1;

// TYPE BT, tree.f90:4-21.  `ox` keeps the geometric centre that PSeudo
// overwrites (tree.f90:470-471) so tree dumps can report both.
struct BT {
  int ileaf = 0;  // -1 electron leaf, 0 twig, +1 ion leaf
  int64_t pt = -1;
  int level = 0;
  double xx[3] = {0, 0, 0};
  double lx[3] = {0, 0, 0};
  double ox[3] = {0, 0, 0};
  double qeff = 0;
  double dx = 0;
  double D[3] = {0, 0, 0};
  double Q[3] = {0, 0, 0};
  double QQ[3] = {0, 0, 0};
  BT* child[8] = {nullptr, nullptr, nullptr, nullptr,
                  nullptr, nullptr, nullptr, nullptr};
};

// ijk table of Insert_Tree_e, tree.f90:116-119 (column-major RESHAPE(.,(3,8))).
const double kIJK[8][3] = {
    {-.25, -.25, -.25}, {+.25, -.25, -.25}, {-.25, +.25, -.25},
    {+.25, +.25, -.25}, {-.25, -.25, +.25}, {+.25, -.25, +.25},
    {-.25, +.25, +.25}, {+.25, +.25, +.25}};

struct Tree {
  BT* root = nullptr;
  int max_depth = 0;
  bool overflow = false;
};

// Child slot for position x in twig P: tree.f90:132-173 (z, then y, then x;
// "<" selects the low half).  Returns bias-1 (0..7).
inline int child_slot(const double* x, const BT* P) {
  int b = 0;
  if (!(x[2] < P->xx[2])) b += 4;
  if (!(x[1] < P->xx[1])) b += 2;
  if (!(x[0] < P->xx[0])) b += 1;
  return b;
}

// Insert_Tree_e / Insert_Tree_i, tree.f90:103-274 / 277-447.  `sign` is -1
// for the electron tree, +1 for the ion tree.  Written as a loop over the
// recursion's tail calls; the order of operations on each node is the
// reference's.
void insert(Tree& T, BT*& slot, BT* R, const double* x, int64_t n, int bias,
            int sign, int depth) {
  if (depth > ORACLE_MAX_DEPTH) {
    T.overflow = true;
    return;
  }
  if (slot == nullptr) {
    BT* P = new BT();  // ALLOCATE(P), tree.f90:113
    P->pt = n;
    P->ileaf = sign;
    P->qeff = (double)sign;
    P->dx = 0.0;
    P->level = depth;
    for (int k = 0; k < 3; ++k) {
      // tree.f90:123-126: P%xx = R%xx + ijk(k,bias)*R%lx ; P%lx = R%lx*0.5
      P->xx[k] = R->xx[k] + kIJK[bias][k] * R->lx[k];
      P->lx[k] = R->lx[k] * 0.5;
    }
    slot = P;
    if (depth > T.max_depth) T.max_depth = depth;
    return;
  }
  BT* P = slot;
  if (P->ileaf == 0) {
    // twig: tree.f90:128-174
    P->qeff = P->qeff + (double)sign;
    const double* xn = x + 3 * n;
    int b = child_slot(xn, P);
    insert(T, P->child[b], P, x, n, b, sign, depth + 1);
  } else {
    // occupied leaf becomes a twig: tree.f90:175-272
    P->ileaf = 0;
    int64_t m = P->pt;
    P->pt = 0;
    P->qeff = P->qeff + (double)sign;
    int bm = child_slot(x + 3 * m, P);
    insert(T, P->child[bm], P, x, m, bm, sign, depth + 1);
    int bn = child_slot(x + 3 * n, P);
    insert(T, P->child[bn], P, x, n, bn, sign, depth + 1);
  }
}

// PSeudoE / PSeudoI, tree.f90:450-553 / 556-659.
void pseudo(BT* P, const double* x) {
  if (P->ileaf != 0) {
    for (int k = 0; k < 3; ++k) {
      P->ox[k] = P->xx[k];
      P->xx[k] = x[3 * P->pt + k];
      P->D[k] = 0.0;
      P->Q[k] = 0.0;
      P->QQ[k] = 0.0;
    }
    return;
  }
  bool tag[8] = {false, false, false, false, false, false, false, false};
  double xs[8][3];
  double q[8];
  double qsum = 0.0;
  double ox[3];
  for (int k = 0; k < 3; ++k) {
    P->D[k] = 0.0;
    P->Q[k] = 0.0;
    P->QQ[k] = 0.0;
    ox[k] = P->xx[k];
    P->ox[k] = P->xx[k];
    P->xx[k] = 0.0;
  }
  for (int c = 0; c < 8; ++c) {
    BT* C = P->child[c];
    if (C == nullptr) continue;
    pseudo(C, x);
    qsum = qsum + C->qeff;
    for (int k = 0; k < 3; ++k) {
      xs[c][k] = C->xx[k];
      P->xx[k] = P->xx[k] + C->qeff * C->xx[k];
    }
    tag[c] = true;
    q[c] = C->qeff;
  }
  for (int k = 0; k < 3; ++k) P->xx[k] = P->xx[k] / qsum;
  {
    double a = P->xx[0] - ox[0];
    double b = P->xx[1] - ox[1];
    double c = P->xx[2] - ox[2];
    P->dx = std::sqrt(a * a + b * b + c * c);  // tree.f90:538
  }
  for (int c = 0; c < 8; ++c) {
    if (!tag[c]) continue;
    double d0 = xs[c][0] - P->xx[0];
    double d1 = xs[c][1] - P->xx[1];
    double d2 = xs[c][2] - P->xx[2];
    P->D[0] = P->D[0] + q[c] * d0;  // tree.f90:541-543
    P->D[1] = P->D[1] + q[c] * d1;
    P->D[2] = P->D[2] + q[c] * d2;
    P->Q[0] = P->Q[0] + q[c] * (d0 * d0) / 2.0;  // tree.f90:544-546
    P->Q[1] = P->Q[1] + q[c] * (d1 * d1) / 2.0;
    P->Q[2] = P->Q[2] + q[c] * (d2 * d2) / 2.0;
    P->QQ[0] = P->QQ[0] + q[c] * d0 * d1;  // tree.f90:547-549
    P->QQ[1] = P->QQ[1] + q[c] * d1 * d2;
    P->QQ[2] = P->QQ[2] + q[c] * d2 * d0;
  }
}

void dealloc(BT* P) {  // DEALLOC_TREE tree.f90:1136-1149
  if (!P) return;
  for (int c = 0; c < 8; ++c) dealloc(P->child[c]);
  delete P;
}

// BuildLocalTree tree.f90:39-100 for one species.
int build_tree(Tree& T, int64_t n, const double* x, int sign) {
  T.root = new BT();
  BT* R = T.root;
  if (n <= 0) {
    R->ileaf = 0;
    return 0;
  }
  double mn[3], mx[3];
  for (int k = 0; k < 3; ++k) {
    mn[k] = x[k];
    mx[k] = x[k];
  }
  for (int64_t i = 1; i < n; ++i)
    for (int k = 0; k < 3; ++k) {
      double v = x[3 * i + k];
      if (v < mn[k]) mn[k] = v;
      if (v > mx[k]) mx[k] = v;
    }
  for (int k = 0; k < 3; ++k) {
    R->xx[k] = (mx[k] + mn[k]) / 2.0;  // tree.f90:58-60
    R->lx[k] = mx[k] - mn[k];          // tree.f90:61-63
  }
  R->ileaf = 0;
  R->dx = 0.0;
  R->qeff = 0.0;  // deviation 2: reference leaves this uninitialised
  R->level = 0;
  for (int64_t i = 0; i < n; ++i) {
    // Insert_Tree_x(Root, ...) with Root associated: the twig branch.
    R->qeff = R->qeff + (double)sign;
    int b = child_slot(x + 3 * i, R);
    insert(T, R->child[b], R, x, i, b, sign, 1);
    if (T.overflow) return ORACLE_ERR_DEPTH;
  }
  pseudo(R, x);
  return 0;
}

struct Params {
  double theta, rs, dx_ei, dx_ii, lam_ee, lam_ei, lam_ii;
  int physics;  // 0 = REF (reference pair laws), 1 = KELBG (erf Kelbg)
};

struct Acc {
  double f[3];
  double epot;
  int64_t n_m2p, n_p2p;
};

// Far-field evaluation of tree.f90:744-779 (identical in all four walks).
inline void m2p(const BT* P, const double* xr, double r2, double r, double ff,
                Acc& a) {
  double R3 = r2 * r;
  double R5 = R3 * r2;
  double R7 = R5 * r2;
  double D[6], Q[10];
  D[0] = -1.0 / R3 + 3.0 * (xr[0] * xr[0]) / R5;
  D[1] = -1.0 / R3 + 3.0 * (xr[1] * xr[1]) / R5;
  D[2] = -1.0 / R3 + 3.0 * (xr[2] * xr[2]) / R5;
  D[3] = 3.0 * xr[0] * xr[1] / R5;
  D[4] = 3.0 * xr[1] * xr[2] / R5;
  D[5] = 3.0 * xr[2] * xr[0] / R5;
  Q[0] = 15.0 * ((xr[0] * xr[0]) * xr[0]) / R7 - 9.0 * xr[0] / R5;
  Q[1] = 15.0 * ((xr[1] * xr[1]) * xr[1]) / R7 - 9.0 * xr[1] / R5;
  Q[2] = 15.0 * ((xr[2] * xr[2]) * xr[2]) / R7 - 9.0 * xr[2] / R5;
  Q[3] = 15.0 * (xr[0] * xr[0]) * xr[1] / R7 - 3.0 * xr[1] / R5;
  Q[4] = 15.0 * (xr[0] * xr[0]) * xr[2] / R7 - 3.0 * xr[2] / R5;
  Q[5] = 15.0 * (xr[1] * xr[1]) * xr[0] / R7 - 3.0 * xr[0] / R5;
  Q[6] = 15.0 * (xr[1] * xr[1]) * xr[2] / R7 - 3.0 * xr[2] / R5;
  Q[7] = 15.0 * (xr[2] * xr[2]) * xr[0] / R7 - 3.0 * xr[0] / R5;
  Q[8] = 15.0 * (xr[2] * xr[2]) * xr[1] / R7 - 3.0 * xr[1] / R5;
  Q[9] = 15.0 * xr[0] * xr[1] * xr[2] / R7;
  a.epot = a.epot + 0.5 * ff *
                        (P->qeff / r +
                         (P->D[0] * xr[0] + P->D[1] * xr[1] + P->D[2] * xr[2]) / R3 +
                         P->Q[0] * D[0] + P->Q[1] * D[1] + P->Q[2] * D[2] +
                         P->QQ[0] * D[3] + P->QQ[1] * D[4] + P->QQ[2] * D[5]);
  a.f[0] = a.f[0] + ff * (P->qeff * xr[0] / R3 + D[0] * P->D[0] + D[3] * P->D[1] +
                          D[5] * P->D[2] + Q[0] * P->Q[0] + Q[5] * P->Q[1] +
                          Q[7] * P->Q[2] + Q[3] * P->QQ[0] + Q[4] * P->QQ[2] +
                          Q[9] * P->QQ[1]);
  a.f[1] = a.f[1] + ff * (P->qeff * xr[1] / R3 + D[3] * P->D[0] + D[1] * P->D[1] +
                          D[4] * P->D[2] + Q[3] * P->Q[0] + Q[1] * P->Q[1] +
                          Q[8] * P->Q[2] + Q[5] * P->QQ[0] + Q[9] * P->QQ[2] +
                          Q[6] * P->QQ[1]);
  a.f[2] = a.f[2] + ff * (P->qeff * xr[2] / R3 + D[5] * P->D[0] + D[4] * P->D[1] +
                          D[2] * P->D[2] + Q[4] * P->Q[0] + Q[6] * P->Q[1] +
                          Q[2] * P->Q[2] + Q[9] * P->QQ[0] + Q[7] * P->QQ[2] +
                          Q[8] * P->QQ[1]);
  a.n_m2p++;
}

inline void rdf_add(int64_t* hist, double r, double dxbin) {
  if (!hist) return;
  // id = INT(r/dx)+1 ; IF (id <= Ndist+1 .AND. id > 0), tree.f90:916-919
  double t = r / dxbin;
  if (!(t < (double)(kNdist + 1))) return;
  int64_t id = (int64_t)t;  // INT truncates toward zero; t >= 0
  if (id >= 0 && id <= kNdist) hist[id]++;
}

// erf-Kelbg leaf law (no reference code): adds force and 0.5*V.
inline void kelbg_pair(const double* xr, double r2, double qq, double lam,
                       Acc& a) {
  double pref = qq * kEps;
  if (r2 == 0.0) {
    // distinct particles at the same point: F = 0, V = qq*eps*sqrt(pi)/lam
    a.epot = a.epot + 0.5 * pref * std::sqrt(M_PI) / lam;
    return;
  }
  double r = std::sqrt(r2);
  double xx = r / lam;
  double g = -std::expm1(-(xx * xx));  // 1 - exp(-x^2)
  a.epot = a.epot + 0.5 * pref * (g / r + std::sqrt(M_PI) * std::erfc(xx) / lam);
  double fr = pref * g / (r2 * r);
  for (int k = 0; k < 3; ++k) a.f[k] = a.f[k] + fr * xr[k];
}

// One target against one tree; recursion order of Search_Tree_xx.
// tsign / ssign: charge signs of target and source species.
void search(const BT* P, const double* xt, int tsign, int ssign, int64_t self,
            const Params& p, Acc& a, int64_t* rdf) {
  double xr[3];
  if (P->ileaf == 0) {
    double s = P->lx[0];  // MAXVAL(P%lx(:)), tree.f90:736
    if (P->lx[1] > s) s = P->lx[1];
    if (P->lx[2] > s) s = P->lx[2];
    double r2 = 0.0;
    for (int k = 0; k < 3; ++k) {
      xr[k] = xt[k] - P->xx[k];
      r2 = r2 + xr[k] * xr[k];
    }
    double r = std::sqrt(r2);
    if ((s / p.theta + P->dx) < r) {  // tree.f90:743
      // ff = -eps for electron targets, +eps for ion targets (744, 848)
      double ff = (tsign < 0) ? -1.0 * kEps : kEps;
      m2p(P, xr, r2, r, ff, a);
    } else {
      for (int c = 0; c < 8; ++c)
        if (P->child[c]) search(P->child[c], xt, tsign, ssign, self, p, a, rdf);
    }
    return;
  }
  // leaf
  double r2 = 0.0;
  for (int k = 0; k < 3; ++k) {
    xr[k] = xt[k] - P->xx[k];
    r2 = r2 + xr[k] * xr[k];
  }
  a.n_p2p++;
  bool same = (tsign == ssign);
  if (p.physics == 1) {
    if (same && P->pt == self) {
      a.n_p2p--;
      return;
    }
    double lam = same ? (tsign < 0 ? p.lam_ee : p.lam_ii) : p.lam_ei;
    kelbg_pair(xr, r2, (double)(tsign * ssign), lam, a);
    if (!same) rdf_add(rdf, std::sqrt(r2), p.dx_ei);
    else if (tsign > 0 && r2 > 0.0) rdf_add(rdf, std::sqrt(r2), p.dx_ii);
    return;
  }
  if (same) {
    // Search_Tree_ee tree.f90:800-815 / Search_Tree_ii 1104-1131
    if (r2 > 0.01) {
      double r = std::sqrt(r2);
      double ff = kEps;
      a.epot = a.epot + 0.5 * ff / r;
      for (int k = 0; k < 3; ++k) a.f[k] = a.f[k] + ff * xr[k] / r / r2;
      if (tsign > 0) rdf_add(rdf, r, p.dx_ii);
    } else {
      a.n_p2p--;
    }
    return;
  }
  // e-i leaf, reference "Kelbg": tree.f90:897-913 / 1001-1018
  double r = std::sqrt(r2);
  double ff = -1.0 * kEps;
  if (r2 == 0.0) {
    // deviation 1: r == 0 limit instead of NaN
    a.epot = a.epot + 0.5 * ff * (1.0 / p.rs);
  } else {
    double e = std::exp(-r / p.rs);
    a.epot = a.epot + 0.5 * ff * (1. - e) / r;
    for (int k = 0; k < 3; ++k)
      a.f[k] = a.f[k] + ff * xr[k] * (1.0 / r - e * (1.0 / r + 1.0 / p.rs)) / r2;
  }
  rdf_add(rdf, r, p.dx_ei);
}

double now_s() {
  return std::chrono::duration<double>(
             std::chrono::steady_clock::now().time_since_epoch())
      .count();
}

}  // namespace

extern "C" {

typedef struct oracle_params {
  double theta;   // sd_ratio
  double rs;      // reference Kelbg screening length (um)
  double dx_ei;   // RDF bin widths (um)
  double dx_ii;
  double lam_ee;  // erf-Kelbg lengths (um), KELBG physics only
  double lam_ei;
  double lam_ii;
  int32_t physics;   // 0 REF, 1 KELBG
  int32_t nthreads;  // 0: OpenMP default
} oracle_params;

typedef struct oracle_stats {
  int64_t n_m2p;
  int64_t n_p2p;
  int32_t max_depth_e;
  int32_t max_depth_i;
  double t_build;
  double t_walk;
} oracle_stats;

// Force (main.f90:506-541, local part) in single-domain form: both trees over
// all particles, then LocalCoulombSum.  f_* are overwritten; epot[0] =
// Epot_e (ee+ie+ei), epot[1] = Epot_i (ii); rdf_* (10001 bins, may be NULL)
// are accumulated like NS%RDF_*.
int oracle_force_strided(int64_t n_el, int64_t n_ion, const double* x_el,
                         const double* x_ion, const oracle_params* prm,
                         double* f_el, double* f_ion, double* epot,
                         int64_t* rdf_ei, int64_t* rdf_ii, oracle_stats* st,
                         int64_t stride);

int oracle_force(int64_t n_el, int64_t n_ion, const double* x_el,
                 const double* x_ion, const oracle_params* prm, double* f_el,
                 double* f_ion, double* epot, int64_t* rdf_ei, int64_t* rdf_ii,
                 oracle_stats* st) {
  return oracle_force_strided(n_el, n_ion, x_el, x_ion, prm, f_el, f_ion, epot,
                              rdf_ei, rdf_ii, st, 1);
}

// Same as oracle_force, but walks only targets whose index is a multiple of
// `stride` (a bounded sample for timing; other targets' forces are left 0).
int oracle_force_strided(int64_t n_el, int64_t n_ion, const double* x_el,
                         const double* x_ion, const oracle_params* prm,
                         double* f_el, double* f_ion, double* epot,
                         int64_t* rdf_ei, int64_t* rdf_ii, oracle_stats* st,
                         int64_t stride) {
  if (stride < 1) return ORACLE_ERR_ARG;
  if (n_el < 0 || n_ion < 0 || !prm || prm->theta <= 0.0) return ORACLE_ERR_ARG;
  Params p{prm->theta, prm->rs, prm->dx_ei, prm->dx_ii,
           prm->lam_ee, prm->lam_ei, prm->lam_ii, prm->physics};
  int nth = prm->nthreads > 0 ? prm->nthreads : omp_get_max_threads();
  double t0 = now_s();
  Tree Te, Ti;
  int rc = build_tree(Te, n_el, x_el, -1);
  if (rc == 0) rc = build_tree(Ti, n_ion, x_ion, +1);
  if (rc != 0) {
    dealloc(Te.root);
    dealloc(Ti.root);
    return rc;
  }
  double t1 = now_s();
  int64_t nm2p = 0, np2p = 0;
  double ep_e = 0.0, ep_i = 0.0;
  std::vector<int64_t> hei((size_t)(kNdist + 1) * nth, 0),
      hii((size_t)(kNdist + 1) * nth, 0);
#pragma omp parallel num_threads(nth) reduction(+ : nm2p, np2p, ep_e, ep_i)
  {
    int tid = omp_get_thread_num();
    int64_t* my_ei = hei.data() + (size_t)(kNdist + 1) * tid;
    int64_t* my_ii = hii.data() + (size_t)(kNdist + 1) * tid;
    // electron targets: ee (tree.f90:682-686) then ei (697-701)
#pragma omp for schedule(static)
    for (int64_t i = 0; i < n_el; ++i) {
      if (i % stride) {
        for (int k = 0; k < 3; ++k) f_el[3 * i + k] = 0.0;
        continue;
      }
      Acc a{{0.0, 0.0, 0.0}, 0.0, 0, 0};
      const double* xt = x_el + 3 * i;
      if (n_el > 0) search(Te.root, xt, -1, -1, i, p, a, nullptr);
      double e_ee = a.epot;
      a.epot = 0.0;
      if (n_ion > 0) search(Ti.root, xt, -1, +1, -1, p, a, my_ei);
      for (int k = 0; k < 3; ++k) f_el[3 * i + k] = a.f[k];
      ep_e += e_ee + a.epot;
      nm2p += a.n_m2p;
      np2p += a.n_p2p;
    }
    // ion targets: ie (690-694) then ii (708-712)
#pragma omp for schedule(static)
    for (int64_t i = 0; i < n_ion; ++i) {
      if (i % stride) {
        for (int k = 0; k < 3; ++k) f_ion[3 * i + k] = 0.0;
        continue;
      }
      Acc a{{0.0, 0.0, 0.0}, 0.0, 0, 0};
      const double* xt = x_ion + 3 * i;
      if (n_el > 0) search(Te.root, xt, +1, -1, -1, p, a, my_ei);
      double e_ie = a.epot;
      a.epot = 0.0;
      if (n_ion > 0) search(Ti.root, xt, +1, +1, i, p, a, my_ii);
      for (int k = 0; k < 3; ++k) f_ion[3 * i + k] = a.f[k];
      ep_e += e_ie;
      ep_i += a.epot;
      nm2p += a.n_m2p;
      np2p += a.n_p2p;
    }
  }
  for (int t = 0; t < nth; ++t)
    for (int b = 0; b <= kNdist; ++b) {
      if (rdf_ei) rdf_ei[b] += hei[(size_t)(kNdist + 1) * t + b];
      if (rdf_ii) rdf_ii[b] += hii[(size_t)(kNdist + 1) * t + b];
    }
  double t2 = now_s();
  if (epot) {
    epot[0] = ep_e;
    epot[1] = ep_i;
  }
  if (st) {
    st->n_m2p = nm2p;
    st->n_p2p = np2p;
    st->max_depth_e = Te.max_depth;
    st->max_depth_i = Ti.max_depth;
    st->t_build = t1 - t0;
    st->t_walk = t2 - t1;
  }
  dealloc(Te.root);
  dealloc(Ti.root);
  return 0;
}

// One node of a pre-order (children 1..8) dump of a species tree.
typedef struct oracle_node {
  double xx[3];   // charge centre (twig) or particle position (leaf)
  double ox[3];   // geometric centre before PSeudo
  double lx[3];
  double qeff, dx;
  double D[3], Q[3], QQ[3];
  int64_t pt;     // particle index (leaf) or -1
  int32_t level;
  int32_t ileaf;
  int64_t skip;   // pre-order index just past this node's subtree
} oracle_node;

namespace {
int64_t dump_rec(const BT* P, oracle_node* out, int64_t cap, int64_t idx) {
  int64_t me = idx;
  if (idx < cap) {
    oracle_node& o = out[idx];
    for (int k = 0; k < 3; ++k) {
      o.xx[k] = P->xx[k];
      o.ox[k] = P->ox[k];
      o.lx[k] = P->lx[k];
      o.D[k] = P->D[k];
      o.Q[k] = P->Q[k];
      o.QQ[k] = P->QQ[k];
    }
    o.qeff = P->qeff;
    o.dx = P->dx;
    o.pt = P->ileaf != 0 ? P->pt : -1;
    o.level = P->level;
    o.ileaf = P->ileaf;
  }
  idx++;
  for (int c = 0; c < 8; ++c)
    if (P->child[c]) idx = dump_rec(P->child[c], out, cap, idx);
  if (me < cap) out[me].skip = idx;
  return idx;
}
}  // namespace

// Builds one species tree (sign -1 electrons, +1 ions) and dumps it in
// pre-order.  Returns the node count (or a negative error); writes at most
// `cap` nodes.
int64_t oracle_tree_dump(int64_t n, const double* x, int32_t sign,
                         oracle_node* out, int64_t cap, int32_t* max_depth) {
  Tree T;
  int rc = build_tree(T, n, x, sign < 0 ? -1 : 1);
  if (rc != 0) {
    dealloc(T.root);
    return rc;
  }
  int64_t cnt = dump_rec(T.root, out, cap, 0);
  if (max_depth) *max_depth = T.max_depth;
  dealloc(T.root);
  return cnt;
}

// FP64 O(N^2) direct sum with the same leaf laws (the theta -> 0 limit of the
// walk).  Targets are index lists into each species; outputs are per target.
// epot (may be NULL) receives the sum of 0.5*V over the listed targets.
int oracle_direct(int64_t n_el, int64_t n_ion, const double* x_el,
                  const double* x_ion, const oracle_params* prm,
                  const int64_t* t_el, int64_t nt_el, const int64_t* t_ion,
                  int64_t nt_ion, double* f_el, double* f_ion, double* epot) {
  if (!prm) return ORACLE_ERR_ARG;
  Params p{prm->theta, prm->rs, prm->dx_ei, prm->dx_ii,
           prm->lam_ee, prm->lam_ei, prm->lam_ii, prm->physics};
  int nth = prm->nthreads > 0 ? prm->nthreads : omp_get_max_threads();
  double ep = 0.0;
  int64_t total = nt_el + nt_ion;
#pragma omp parallel for num_threads(nth) schedule(dynamic, 16) reduction(+ : ep)
  for (int64_t t = 0; t < total; ++t) {
    bool is_el = t < nt_el;
    int64_t i = is_el ? t_el[t] : t_ion[t - nt_el];
    int tsign = is_el ? -1 : +1;
    const double* xt = is_el ? x_el + 3 * i : x_ion + 3 * i;
    Acc a{{0.0, 0.0, 0.0}, 0.0, 0, 0};
    for (int s = 0; s < 2; ++s) {
      int ssign = s == 0 ? -1 : +1;
      int64_t ns = s == 0 ? n_el : n_ion;
      const double* xs = s == 0 ? x_el : x_ion;
      BT leaf;
      leaf.ileaf = ssign;
      for (int64_t j = 0; j < ns; ++j) {
        leaf.pt = j;
        for (int k = 0; k < 3; ++k) leaf.xx[k] = xs[3 * j + k];
        search(&leaf, xt, tsign, ssign, (ssign == tsign) ? i : -1, p, a,
               nullptr);
      }
    }
    double* fo = is_el ? f_el + 3 * t : f_ion + 3 * (t - nt_el);
    for (int k = 0; k < 3; ++k) fo[k] = a.f[k];
    ep += a.epot;
  }
  if (epot) *epot = ep;
  return 0;
}

// VVerletNotemp1, vverlet.f90:24-30: v += 0.5*dt*f/m ; x += dt*v.
void oracle_kdk1(int64_t n, double* x, double* v, const double* f, double dt,
                 double xm) {
  for (int64_t i = 0; i < n; ++i)
    for (int k = 0; k < 3; ++k) {
      v[3 * i + k] = v[3 * i + k] + 0.5 * dt * f[3 * i + k] / xm;
      x[3 * i + k] = x[3 * i + k] + dt * v[3 * i + k];
    }
}

// VVerletNotemp2, vverlet.f90:64-76: v += 0.5*dt*f/m.
void oracle_kdk2(int64_t n, double* v, const double* f, double dt, double xm) {
  for (int64_t i = 0; i < n; ++i)
    for (int k = 0; k < 3; ++k)
      v[3 * i + k] = v[3 * i + k] + 0.5 * dt * f[3 * i + k] / xm;
}

// Sampling sums of VVerletNotemp2, vverlet.f90:86-106:
// out[0] = sum m v^2, out[1] = sum m (x.v)^2/|x|^2.
void oracle_ke(int64_t n, const double* x, const double* v, double xm,
               double* out) {
  double mv2 = 0.0, rad = 0.0;
  for (int64_t i = 0; i < n; ++i) {
    const double* xi = x + 3 * i;
    const double* vi = v + 3 * i;
    mv2 = mv2 + xm * (vi[0] * vi[0] + vi[1] * vi[1] + vi[2] * vi[2]);
    double xv = xi[0] * vi[0] + xi[1] * vi[1] + xi[2] * vi[2];
    rad = rad + xm * (xv * xv) /
                    (xi[0] * xi[0] + xi[1] * xi[1] + xi[2] * xi[2]);
  }
  out[0] = mv2;
  out[1] = rad;
}

int oracle_max_threads(void) { return omp_get_max_threads(); }

}  // extern "C"

// ===================================================================== REF8 ==
// The 8-rank form of Force (main.f90:506-701) run in one process.  The
// reference runs on exactly 8 MPI ranks (mpienv.f90:19), one per coordinate
// octant (id_FINDER, main.f90:840-862).  Each rank builds its own two species
// trees over its own particles (BuildLocalTree) and walks them for its own
// targets (LocalCoulombSum).  It then serialises each tree once per other
// rank, pruned against the plane, line or point that its octant shares with
// that rank's (CopyTree1..7, tree.f90:1204-1777, case from CriterionFind,
// main.f90:865-925): a twig is expanded when MAXVAL(lx)/theta + dx exceeds
// the distance from its charge centre to that contact set.  The receiver
// rebuilds the serialised tree (RebuildGhostTree, tree.f90:1781-1853), where
// every node sent without children -- a leaf, or a twig that was not expanded
// -- becomes a leaf, and walks it (Ghost_Tree_ee/ie/ei/ii, tree.f90:1888-2330):
// ghost twigs take the reference MAC and far field; ghost leaves are point
// charges qeff with the leaf laws and no MAC, no r^2 > 0.01 cutoff.  Per
// target the contributions arrive in the reference's order: own trees (ee or
// ie, then ei or ii), the seven electron ghost trees from ranks r-1 .. r-7,
// then the seven ion ghost trees in the same order.
//
// Particles are assigned to octants by their current positions (as right
// after a migration, data.f90:196-389).  A rank without particles of a species
// sends and walks no tree of that species (the reference would take MINVAL of
// an empty array).  The deviations of the single-domain form (r = 0 e-i
// guard, root qeff, RDF race, depth cap) apply unchanged.

namespace {

// id_FINDER: rank = 4(k-1) + 2(j-1) + (i-1), the low index for a negative
// coordinate.
inline int octant_of(const double* x) {
  const int i = x[0] < 0.0 ? 0 : 1;
  const int j = x[1] < 0.0 ? 0 : 1;
  const int k = x[2] < 0.0 ? 0 : 1;
  return 4 * k + 2 * j + i;
}

// CriterionFind: the contact case of octants a and b -- 1 y-z face, 2 x-z
// face, 3 x-y face, 4 x-axis line, 5 y-axis line, 6 z-axis line, 7 the origin.
int contact_case(int a, int b) {
  const bool sx = (a & 1) == (b & 1);
  const bool sy = ((a >> 1) & 1) == ((b >> 1) & 1);
  const bool sz = ((a >> 2) & 1) == ((b >> 2) & 1);
  if (sx) {
    if (sy) return 3;
    return sz ? 2 : 4;
  }
  if (sy) return sz ? 1 : 5;
  return sz ? 6 : 7;
}

// Distance of a charge centre from the contact set of case c (the planes,
// lines and point through the origin), in the reference's arithmetic.
double contact_distance(int c, const double* xx) {
  const double x = 0.0, y = 0.0, z = 0.0;
  switch (c) {
    case 1: return std::fabs(xx[0] - x);
    case 2: return std::fabs(xx[1] - y);
    case 3: return std::fabs(xx[2] - z);
    case 4: return std::sqrt((xx[1] - y) * (xx[1] - y) + (xx[2] - z) * (xx[2] - z));
    case 5: return std::sqrt((xx[0] - x) * (xx[0] - x) + (xx[2] - z) * (xx[2] - z));
    case 6: return std::sqrt((xx[0] - x) * (xx[0] - x) + (xx[1] - y) * (xx[1] - y));
    default:
      return std::sqrt((xx[0] - x) * (xx[0] - x) + (xx[1] - y) * (xx[1] - y) +
                       (xx[2] - z) * (xx[2] - z));
  }
}

// CopyTree<c> of P followed by RebuildGhostTree: the ghost tree as the
// receiver holds it.  Every node carries qeff, the charge centre, MAXVAL(lx)
// (in all three lx slots, so the walk's MAXVAL returns it), dx and the
// moments (zero for leaves); children keep their order and fill Child1.. in
// turn; a node without children becomes a leaf of the sign of qeff.
BT* copy_ghost(const BT* P, int c, double theta, int64_t& nodes) {
  BT* G = new BT();
  nodes++;
  double s = P->lx[0];
  if (P->lx[1] > s) s = P->lx[1];
  if (P->lx[2] > s) s = P->lx[2];
  G->qeff = P->qeff;
  G->level = P->level;
  for (int k = 0; k < 3; ++k) {
    G->xx[k] = P->xx[k];
    G->ox[k] = P->ox[k];
    G->lx[k] = s;
  }
  int nk = 0;
  if (P->ileaf == 0) {
    G->dx = P->dx;
    for (int k = 0; k < 3; ++k) {
      G->D[k] = P->D[k];
      G->Q[k] = P->Q[k];
      G->QQ[k] = P->QQ[k];
    }
    if ((s / theta + G->dx) > contact_distance(c, G->xx)) {
      for (int ch = 0; ch < 8; ++ch)
        if (P->child[ch]) G->child[nk++] = copy_ghost(P->child[ch], c, theta, nodes);
    }
  }
  G->ileaf = nk > 0 ? 0 : (G->qeff > 0.0 ? 1 : -1);
  G->pt = -1;
  return G;
}

// One target against one ghost tree (Ghost_Tree_ee/ie/ei/ii).
void ghost_search(const BT* P, const double* xt, int tsign, int ssign,
                  const Params& p, Acc& a, int64_t* rdf) {
  double xr[3];
  double r2 = 0.0;
  for (int k = 0; k < 3; ++k) {
    xr[k] = xt[k] - P->xx[k];
    r2 = r2 + xr[k] * xr[k];
  }
  if (P->ileaf == 0) {
    const double s = P->lx[0];
    const double r = std::sqrt(r2);
    if ((s / p.theta + P->dx) < r) {  // tree.f90:1910
      const double ff = (tsign < 0) ? -1.0 * kEps : kEps;
      m2p(P, xr, r2, r, ff, a);
    } else {
      for (int c = 0; c < 8; ++c)
        if (P->child[c]) ghost_search(P->child[c], xt, tsign, ssign, p, a, rdf);
    }
    return;
  }
  // ghost leaf: a point charge qeff (one particle, or a whole unexpanded twig)
  a.n_p2p++;
  const bool same = tsign == ssign;
  const double r = std::sqrt(r2);
  if (p.physics == 1) {
    const double lam = same ? (tsign < 0 ? p.lam_ee : p.lam_ii) : p.lam_ei;
    kelbg_pair(xr, r2, (double)tsign * P->qeff, lam, a);
    if (!same) rdf_add(rdf, r, p.dx_ei);
    else if (tsign > 0 && r2 > 0.0) rdf_add(rdf, r, p.dx_ii);
    return;
  }
  // ff = -eps*qeff (electron target) or +eps*qeff (ion target), tree.f90:1975,
  // 2072, 2210, 2315
  const double ff = (tsign < 0 ? -1.0 : 1.0) * kEps * P->qeff;
  if (same) {
    // Ghost_Tree_ee tree.f90:1966-1981 / Ghost_Tree_ii 2306-2326
    a.epot = a.epot + 0.5 * ff / r;
    for (int k = 0; k < 3; ++k) a.f[k] = a.f[k] + ff * xr[k] / r / r2;
    if (tsign > 0) rdf_add(rdf, r, p.dx_ii);
    return;
  }
  // Ghost_Tree_ie tree.f90:2064-2084 / Ghost_Tree_ei 2202-2222
  if (r2 == 0.0) {
    a.epot = a.epot + 0.5 * ff * (1.0 / p.rs);  // deviation 1
  } else {
    const double e = std::exp(-r / p.rs);
    a.epot = a.epot + 0.5 * ff * (1. - e) / r;
    for (int k = 0; k < 3; ++k)
      a.f[k] = a.f[k] + ff * xr[k] * (1.0 / r - e * (1.0 / r + 1.0 / p.rs)) / r2;
  }
  rdf_add(rdf, r, p.dx_ei);
}

}  // namespace

extern "C" {

typedef struct oracle_ref8_stats {
  int64_t n_el[8], n_ion[8];       // particles per rank
  int64_t ghost_nodes_e, ghost_nodes_i;  // nodes of all 56 ghost trees per species
  int64_t n_m2p_ghost, n_p2p_ghost;      // interactions with ghost trees
} oracle_ref8_stats;

// Force in the 8-rank form (see above).  Arguments and outputs as
// oracle_force; st8 (may be NULL) receives the decomposition's figures.
int oracle_force_ref8(int64_t n_el, int64_t n_ion, const double* x_el,
                      const double* x_ion, const oracle_params* prm,
                      double* f_el, double* f_ion, double* epot,
                      int64_t* rdf_ei, int64_t* rdf_ii, oracle_stats* st,
                      oracle_ref8_stats* st8) {
  if (n_el < 0 || n_ion < 0 || !prm || prm->theta <= 0.0) return ORACLE_ERR_ARG;
  Params p{prm->theta, prm->rs, prm->dx_ei, prm->dx_ii,
           prm->lam_ee, prm->lam_ei, prm->lam_ii, prm->physics};
  const int nth = prm->nthreads > 0 ? prm->nthreads : omp_get_max_threads();
  const double t0 = now_s();
  // ranks by octant, particles in input order (Init, main.f90:306-316)
  std::vector<int64_t> ie[8], ii[8];
  std::vector<double> xe[8], xi[8];
  for (int64_t i = 0; i < n_el; ++i) ie[octant_of(x_el + 3 * i)].push_back(i);
  for (int64_t i = 0; i < n_ion; ++i) ii[octant_of(x_ion + 3 * i)].push_back(i);
  Tree Te[8], Ti[8];
  int rc = 0;
  for (int r = 0; r < 8 && rc == 0; ++r) {
    for (int64_t g : ie[r]) xe[r].insert(xe[r].end(), x_el + 3 * g, x_el + 3 * g + 3);
    for (int64_t g : ii[r]) xi[r].insert(xi[r].end(), x_ion + 3 * g, x_ion + 3 * g + 3);
    if (!ie[r].empty()) rc = build_tree(Te[r], (int64_t)ie[r].size(), xe[r].data(), -1);
    if (rc == 0 && !ii[r].empty())
      rc = build_tree(Ti[r], (int64_t)ii[r].size(), xi[r].data(), +1);
  }
  // ghost trees: rank s sends to DEST(i) = (s + i) mod 8 (mpienv.f90:58-65)
  BT* Ge[8][8] = {};
  BT* Gi[8][8] = {};
  int64_t gn_e = 0, gn_i = 0;
  if (rc == 0)
    for (int s = 0; s < 8; ++s)
      for (int i = 1; i < 8; ++i) {
        const int r = (s + i) % 8;
        const int c = contact_case(r, s);
        if (Te[s].root) Ge[s][r] = copy_ghost(Te[s].root, c, p.theta, gn_e);
        if (Ti[s].root) Gi[s][r] = copy_ghost(Ti[s].root, c, p.theta, gn_i);
      }
  const double t1 = now_s();
  int64_t nm2p = 0, np2p = 0, gm2p = 0, gp2p = 0;
  double ep_e = 0.0, ep_i = 0.0;
  std::vector<int64_t> hei((size_t)(kNdist + 1) * nth, 0),
      hii((size_t)(kNdist + 1) * nth, 0);
  if (rc == 0) {
#pragma omp parallel num_threads(nth) reduction(+ : nm2p, np2p, gm2p, gp2p, ep_e, ep_i)
    {
      const int tid = omp_get_thread_num();
      int64_t* my_ei = hei.data() + (size_t)(kNdist + 1) * tid;
      int64_t* my_ii = hii.data() + (size_t)(kNdist + 1) * tid;
      for (int r = 0; r < 8; ++r) {
        const int64_t ne = (int64_t)ie[r].size(), ni = (int64_t)ii[r].size();
#pragma omp for schedule(static)
        for (int64_t k = 0; k < ne; ++k) {
          Acc a{{0.0, 0.0, 0.0}, 0.0, 0, 0};
          const double* xt = xe[r].data() + 3 * k;
          if (Te[r].root) search(Te[r].root, xt, -1, -1, k, p, a, nullptr);
          const double e_ee = a.epot;
          a.epot = 0.0;
          if (Ti[r].root) search(Ti[r].root, xt, -1, +1, -1, p, a, my_ei);
          const double e_loc = e_ee + a.epot;
          a.epot = 0.0;
          const int64_t lm = a.n_m2p, lp = a.n_p2p;
          for (int i = 1; i < 8; ++i)
            if (BT* G = Ge[(r - i + 8) % 8][r]) ghost_search(G, xt, -1, -1, p, a, nullptr);
          for (int i = 1; i < 8; ++i)
            if (BT* G = Gi[(r - i + 8) % 8][r]) ghost_search(G, xt, -1, +1, p, a, my_ei);
          const int64_t g = ie[r][k];
          for (int d = 0; d < 3; ++d) f_el[3 * g + d] = a.f[d];
          ep_e += e_loc + a.epot;
          nm2p += a.n_m2p;
          np2p += a.n_p2p;
          gm2p += a.n_m2p - lm;
          gp2p += a.n_p2p - lp;
        }
#pragma omp for schedule(static)
        for (int64_t k = 0; k < ni; ++k) {
          Acc a{{0.0, 0.0, 0.0}, 0.0, 0, 0};
          const double* xt = xi[r].data() + 3 * k;
          if (Te[r].root) search(Te[r].root, xt, +1, -1, -1, p, a, my_ei);
          const double e_ie = a.epot;
          a.epot = 0.0;
          if (Ti[r].root) search(Ti[r].root, xt, +1, +1, k, p, a, my_ii);
          double e_ii = a.epot;
          a.epot = 0.0;
          const int64_t lm = a.n_m2p, lp = a.n_p2p;
          for (int i = 1; i < 8; ++i)
            if (BT* G = Ge[(r - i + 8) % 8][r]) ghost_search(G, xt, +1, -1, p, a, my_ei);
          const double e_gie = a.epot;
          a.epot = 0.0;
          for (int i = 1; i < 8; ++i)
            if (BT* G = Gi[(r - i + 8) % 8][r]) ghost_search(G, xt, +1, +1, p, a, my_ii);
          e_ii += a.epot;
          const int64_t g = ii[r][k];
          for (int d = 0; d < 3; ++d) f_ion[3 * g + d] = a.f[d];
          ep_e += e_ie + e_gie;
          ep_i += e_ii;
          nm2p += a.n_m2p;
          np2p += a.n_p2p;
          gm2p += a.n_m2p - lm;
          gp2p += a.n_p2p - lp;
        }
      }
    }
    for (int t = 0; t < nth; ++t)
      for (int b = 0; b <= kNdist; ++b) {
        if (rdf_ei) rdf_ei[b] += hei[(size_t)(kNdist + 1) * t + b];
        if (rdf_ii) rdf_ii[b] += hii[(size_t)(kNdist + 1) * t + b];
      }
  }
  const double t2 = now_s();
  if (rc == 0 && epot) {
    epot[0] = ep_e;
    epot[1] = ep_i;
  }
  if (st) {
    st->n_m2p = nm2p;
    st->n_p2p = np2p;
    st->max_depth_e = 0;
    st->max_depth_i = 0;
    for (int r = 0; r < 8; ++r) {
      if (Te[r].max_depth > st->max_depth_e) st->max_depth_e = Te[r].max_depth;
      if (Ti[r].max_depth > st->max_depth_i) st->max_depth_i = Ti[r].max_depth;
    }
    st->t_build = t1 - t0;
    st->t_walk = t2 - t1;
  }
  if (st8) {
    for (int r = 0; r < 8; ++r) {
      st8->n_el[r] = (int64_t)ie[r].size();
      st8->n_ion[r] = (int64_t)ii[r].size();
    }
    st8->ghost_nodes_e = gn_e;
    st8->ghost_nodes_i = gn_i;
    st8->n_m2p_ghost = gm2p;
    st8->n_p2p_ghost = gp2p;
  }
  for (int s = 0; s < 8; ++s) {
    for (int r = 0; r < 8; ++r) {
      dealloc(Ge[s][r]);
      dealloc(Gi[s][r]);
    }
    dealloc(Te[s].root);
    dealloc(Ti[s].root);
  }
  return rc;
}

}  // extern "C"
