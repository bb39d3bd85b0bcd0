/*
 * mdff_oracle.c -- CPU FP64 restatement of the MDFF engforce path.
 *
 * TEST INFRASTRUCTURE ONLY (the checker, never the product): see
 * mdff_oracle.h.  Citations are file:line in the reference's src/ tree.
 *
 * Differences from the reference that are deliberate and documented:
 *  - Positions are never modified in place: the reference converts rx,ry,rz
 *    Cartesian->direct->Cartesian inside every pair routine (kardir/dirkar,
 *    lattice.f90:183-270), perturbing them at the ulp level each call; here
 *    each routine computes direct coordinates into a scratch copy with the
 *    same arithmetic.
 *  - Forces start from zero on every call (the reference keeps stale fx when
 *    no short-range potential is switched on, engforce_driver.f90:116-135).
 *  - The electric field returned is always the do_efield=.true. field.
 *  - Quadrupole tasks (task_coul(4:6)) are not built (theta is zeroed by
 *    engforce).  Of the kO dipole algorithms, scf_kO_v3 and scf_kO_v4_2 are
 *    rejected (MDFF_ERR_UNSUPPORTED).
 *  - One optional extension: a W/r^24 wall added to BMH pairs (params.wall24,
 *    zero = reference behaviour).
 */
#include "mdff_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define NT MDFF_NTYPEMAX
#define TT_MAX 8
#define KO_HIST 100 /* F_h, mu_h depth of scf_kO_v4 (moment_from_pola.f90:2050) */

/* constants.f90:65-94 */
static const double PI = 3.14159265358979323846264338327950;
#define TPI (2.0 * PI)
#define COUL_UNIT_EV 14.3996441494161
#define PRESS_UNIT_EV 0.00624150964712042

struct or_ctx {
  mdff_params p;      /* after symmetrisation / clamp / lautoES */
  int natm;
  int n_kardir;       /* in-place kardir/dirkar round trips of this engforce */
  int* itype;         /* [natm] 0-based */
  int* ipolar;        /* [natm] */
  double* qia;        /* [natm] */
  double* dipia;      /* [natm][3] */
  double* poldipia;   /* [natm][3][3]  [ia][a][b] = poldipia(a,b,ia) */
  double* invpoldipia;
  /* non_bonded derived (non_bonded.f90:455-644) */
  double rcutsq[NT][NT], sigsq[NT][NT], epsp[NT][NT], fc[NT][NT];
  double uc[NT][NT], uc1[NT][NT], uc2[NT][NT];
  double E_TT[TT_MAX + 1];
  /* cell (lattice.f90:60-180) */
  double A[3][3], B[3][3], omega, WA, WB, WC, ANORM[3];
  /* coulomb */
  int task[6];
  double coul_unit, press_unit;
  int nk;
  double *kx, *ky, *kz, *kk, *Ak, *kcoe;
  /* ASPC history dipia_ind_t(5,3,natm) -> [5][natm][3] */
  double* hist;
  /* direct coordinates at the last list build, config%xs/ys/zs
     (config.f90:66); written only by or_vnlistcheck */
  double *xs, *ys, *zs;
  int lpolar_any;
};

static int g_threads = 0;

void or_set_threads(int n) { g_threads = n; }
int or_get_threads(void) {
#ifdef _OPENMP
  return g_threads > 0 ? g_threads : omp_get_max_threads();
#else
  return 1;
#endif
}

/* ---------------------------------------------------------------------- */
/* functions.f90:28-40 -- Numerical Recipes Chebyshev erfc (NOT libm erfc)  */
double or_errfc(double x) {
  double z = fabs(x);
  double t = 1.0 / (1.0 + 0.5 * z);
  double r = t * exp(-z * z - 1.26551223 +
                     t * (1.00002368 +
                          t * (.37409196 +
                               t * (.09678418 +
                                    t * (-.18628806 +
                                         t * (.27886807 +
                                              t * (-1.13520398 +
                                                   t * (1.48851587 +
                                                        t * (-.82215223 + t * .17087277)))))))));
  if (x < 0.0) r = 2.0 - r;
  return r;
}

/* tt_damp.f90:42-58 get_TT_damp, :68-97 TT_damping_functions */
static double E_TT_tab[TT_MAX + 1];
static void tt_table(double* e) {
  e[0] = 1.0;
  for (int k = 1; k <= TT_MAX; ++k) e[k] = e[k - 1] / (double)k;
}

static void tt_damp_tab(const double* E_TT, double b, double c, double r, int order, double* f,
                        double* fd) {
  double br = b * r;
  double expbdr = exp(-br) * c;
  double ff = E_TT[order];
  for (int k = order - 1; k >= 1; --k) ff = ff * br + E_TT[k];
  ff = ff * br + E_TT[0];
  *f = 1.0 - ff * expbdr;
  /* Fortran ( br ) ** ( order ) with an integer exponent */
  double p = 1.0;
  for (int k = 0; k < order; ++k) p *= br;
  *fd = E_TT[order] * p * expbdr * b;
}

void or_tt_damp(double b, double c, double r, int order, double* f, double* fd) {
  tt_table(E_TT_tab);
  tt_damp_tab(E_TT_tab, b, c, r, order, f, fd);
}

/* Fortran NINT: round half away from zero */
static inline double fnint(double x) { return round(x); }

/* lattice.f90:60-180 (only the parts engforce needs) */
static void or_lattice(or_ctx* c, const double* Ain) {
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) c->A[a][b] = Ain[a * 3 + b];
  double(*A)[3] = c->A;
  double(*B)[3] = c->B;
  /* EXPRO (tools.f90:786-798): B(:,1) = A(:,2) x A(:,3) ... */
  int cyc[3][2] = {{1, 2}, {2, 0}, {0, 1}};
  for (int col = 0; col < 3; ++col) {
    int u = cyc[col][0], v = cyc[col][1];
    B[0][col] = A[1][u] * A[2][v] - A[2][u] * A[1][v];
    B[1][col] = A[2][u] * A[0][v] - A[0][u] * A[2][v];
    B[2][col] = A[0][u] * A[1][v] - A[1][u] * A[0][v];
  }
  double omega = B[0][0] * A[0][0] + B[1][0] * A[1][0] + B[2][0] * A[2][0];
  c->omega = omega;
  c->WA = omega / sqrt(B[0][0] * B[0][0] + B[1][0] * B[1][0] + B[2][0] * B[2][0]);
  c->WB = omega / sqrt(B[0][1] * B[0][1] + B[1][1] * B[1][1] + B[2][1] * B[2][1]);
  c->WC = omega / sqrt(B[0][2] * B[0][2] + B[1][2] * B[1][2] + B[2][2] * B[2][2]);
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) B[i][j] = B[i][j] / omega;
  for (int i = 0; i < 3; ++i)
    c->ANORM[i] = sqrt(A[0][i] * A[0][i] + A[1][i] * A[1][i] + A[2][i] * A[2][i]);
}

/* kardir (lattice.f90:183-225) into scratch arrays */
static void or_kardir(const or_ctx* c, const double* rx, const double* ry, const double* rz,
                      double* sx, double* sy, double* sz) {
  const double(*B)[3] = c->B;
  for (int n = 0; n < c->natm; ++n) {
    double vx = rx[n], vy = ry[n], vz = rz[n];
    sx[n] = vx * B[0][0] + vy * B[1][0] + vz * B[2][0];
    sy[n] = vx * B[0][1] + vy * B[1][1] + vz * B[2][1];
    sz[n] = vx * B[0][2] + vy * B[1][2] + vz * B[2][2];
  }
}

/* The reference converts the global positions to direct coordinates and
   back IN PLACE around each pass over the pairs (kardir lattice.f90:183-225,
   dirkar :232-270; e.g. ewald_dir.f90:138,739).  One round trip: V = r B
   then r = A V, each component summed left to right. */
void or_kardir_roundtrips(or_ctx* c, double* rx, double* ry, double* rz, int count) {
  const double(*A)[3] = c->A;
  const double(*B)[3] = c->B;
  for (int n = 0; n < c->natm; ++n) {
    double vx = rx[n], vy = ry[n], vz = rz[n];
    for (int k = 0; k < count; ++k) {
      double v1 = vx * B[0][0] + vy * B[1][0] + vz * B[2][0];
      double v2 = vx * B[0][1] + vy * B[1][1] + vz * B[2][1];
      double v3 = vx * B[0][2] + vy * B[1][2] + vz * B[2][2];
      vx = v1 * A[0][0] + v2 * A[0][1] + v3 * A[0][2];
      vy = v1 * A[1][0] + v2 * A[1][1] + v3 * A[1][2];
      vz = v1 * A[2][0] + v2 * A[2][1] + v3 * A[2][2];
    }
    rx[n] = vx;
    ry[n] = vy;
    rz[n] = vz;
  }
}

/* minimum image through direct coordinates (e.g. non_bonded.f90:1136-1145) */
static inline double min_image(const or_ctx* c, double dsx, double dsy, double dsz, double* rxij,
                               double* ryij, double* rzij) {
  double sxij = dsx - fnint(dsx);
  double syij = dsy - fnint(dsy);
  double szij = dsz - fnint(dsz);
  const double(*A)[3] = c->A;
  *rxij = sxij * A[0][0] + syij * A[0][1] + szij * A[0][2];
  *ryij = sxij * A[1][0] + syij * A[1][1] + szij * A[1][2];
  *rzij = sxij * A[2][0] + syij * A[2][1] + szij * A[2][2];
  return *rxij * *rxij + *ryij * *ryij + *rzij * *rzij;
}

/* 3x3 inverse by LU with partial pivoting (DGETRF/DGETRI in
   read_pos.f90:203-212); exact reciprocals for diagonal tensors. */
static int inv3(const double* m, double* out) {
  /* a diagonal tensor (the isotropic/axial polarisabilities of every deck)
     is inverted entry by entry; a zero entry stays zero (pseudo-inverse), as
     a site polarisable along x only (examples/ex04/control_twocharges_twopola.F
     pol(3,1,1)) has no defined LAPACK inverse */
  if (m[1] == 0.0 && m[2] == 0.0 && m[3] == 0.0 && m[5] == 0.0 && m[6] == 0.0 && m[7] == 0.0) {
    for (int i = 0; i < 9; ++i) out[i] = 0.0;
    for (int i = 0; i < 3; ++i) out[4 * i] = (m[4 * i] != 0.0) ? 1.0 / m[4 * i] : 0.0;
    return 0;
  }
  double a[3][3];
  int piv[3] = {0, 1, 2};
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) a[i][j] = m[i * 3 + j];
  for (int k = 0; k < 3; ++k) {
    int p = k;
    for (int i = k + 1; i < 3; ++i)
      if (fabs(a[i][k]) > fabs(a[p][k])) p = i;
    if (a[p][k] == 0.0) return -1;
    if (p != k) {
      for (int j = 0; j < 3; ++j) {
        double t = a[k][j];
        a[k][j] = a[p][j];
        a[p][j] = t;
      }
      int t = piv[k];
      piv[k] = piv[p];
      piv[p] = t;
    }
    for (int i = k + 1; i < 3; ++i) {
      a[i][k] /= a[k][k];
      for (int j = k + 1; j < 3; ++j) a[i][j] -= a[i][k] * a[k][j];
    }
  }
  /* solve for each unit vector */
  for (int col = 0; col < 3; ++col) {
    double y[3];
    for (int i = 0; i < 3; ++i) {
      double s = (piv[i] == col) ? 1.0 : 0.0;
      for (int j = 0; j < i; ++j) s -= a[i][j] * y[j];
      y[i] = s;
    }
    for (int i = 2; i >= 0; --i) {
      double s = y[i];
      for (int j = i + 1; j < 3; ++j) s -= a[i][j] * y[j];
      y[i] = s / a[i][i];
    }
    for (int i = 0; i < 3; ++i) out[i * 3 + col] = y[i];
  }
  return 0;
}

/* symmetric_pot: X(:,it) = X(it,:) for it = 1..ntype (non_bonded.f90:287-301) */
static void sym2(double X[NT][NT], int ntype) {
  for (int it = 0; it < ntype; ++it) {
    double row[NT];
    for (int k = 0; k < NT; ++k) row[k] = X[it][k];
    for (int k = 0; k < NT; ++k) X[k][it] = row[k];
  }
}
/* pim.f90:186-199: X(it2,:,it) = X(it2,it,:) */
#define SYM3(X, T)                                                  \
  do {                                                              \
    for (int it = 0; it < ntype; ++it)                              \
      for (int it2 = 0; it2 < ntype; ++it2) {                       \
        T row[NT];                                                  \
        for (int k = 0; k < NT; ++k) row[k] = (X)[it2][it][k];      \
        for (int k = 0; k < NT; ++k) (X)[it2][k][it] = row[k];      \
      }                                                             \
  } while (0)

/* kpoint_sum_init (kspace.f90:143-207) + reorder_kpt (:286-342): stable sort
   by k^2 (merge_sort, tools.f90:667-785, keeps equal keys in order). */
static void or_kmesh(or_ctx* c) {
  int kx = c->p.kES[0], ky = c->p.kES[1], kz = c->p.kES[2];
  int nk = kz + ky * (2 * kz + 1) + kx * (2 * ky + 1) * (2 * kz + 1);
  free(c->kx);
  free(c->ky);
  free(c->kz);
  free(c->kk);
  free(c->Ak);
  free(c->kcoe);
  double* tx = malloc(sizeof(double) * nk);
  double* ty = malloc(sizeof(double) * nk);
  double* tz = malloc(sizeof(double) * nk);
  double* tk = malloc(sizeof(double) * nk);
  double* ta = malloc(sizeof(double) * nk);
  double* tc = malloc(sizeof(double) * nk);
  double alpha = c->p.alphaES, alpha2 = alpha * alpha;
  const double(*B)[3] = c->B;
  int n = 0;
  for (int nx = 0; nx <= kx; ++nx) {
    int nymin = (nx == 0) ? 0 : -ky;
    for (int ny = nymin; ny <= ky; ++ny) {
      int nzmin = (nx == 0 && ny == 0) ? 1 : -kz;
      for (int nz = nzmin; nz <= kz; ++nz) {
        double X = (double)nx, Y = (double)ny, Z = (double)nz;
        double kxx = TPI * (X * B[0][0] + Y * B[0][1] + Z * B[0][2]);
        double kyy = TPI * (X * B[1][0] + Y * B[1][1] + Z * B[1][2]);
        double kzz = TPI * (X * B[2][0] + Y * B[2][1] + Z * B[2][2]);
        double kk = kxx * kxx + kyy * kyy + kzz * kzz;
        tx[n] = kxx;
        ty[n] = kyy;
        tz[n] = kzz;
        tk[n] = kk;
        ta[n] = exp(-kk * 0.25 / alpha2) / kk;
        tc[n] = 2.0 * (1.0 / kk + 1.0 / alpha2 / 4.0);
        ++n;
      }
    }
  }
  /* stable ordering by kk: insertion-merge via index sort with tie on index */
  int* idx = malloc(sizeof(int) * nk);
  for (int i = 0; i < nk; ++i) idx[i] = i;
  /* bottom-up stable merge sort on indices */
  int* tmp = malloc(sizeof(int) * nk);
  for (int w = 1; w < nk; w *= 2) {
    for (int lo = 0; lo < nk; lo += 2 * w) {
      int mid = lo + w < nk ? lo + w : nk, hi = lo + 2 * w < nk ? lo + 2 * w : nk;
      int i = lo, j = mid, o = lo;
      while (i < mid && j < hi) tmp[o++] = (tk[idx[i]] <= tk[idx[j]]) ? idx[i++] : idx[j++];
      while (i < mid) tmp[o++] = idx[i++];
      while (j < hi) tmp[o++] = idx[j++];
    }
    memcpy(idx, tmp, sizeof(int) * nk);
  }
  c->kx = malloc(sizeof(double) * nk);
  c->ky = malloc(sizeof(double) * nk);
  c->kz = malloc(sizeof(double) * nk);
  c->kk = malloc(sizeof(double) * nk);
  c->Ak = malloc(sizeof(double) * nk);
  c->kcoe = malloc(sizeof(double) * nk);
  for (int i = 0; i < nk; ++i) {
    int l = idx[i];
    c->kx[i] = tx[l];
    c->ky[i] = ty[l];
    c->kz[i] = tz[l];
    c->kk[i] = tk[l];
    c->Ak[i] = ta[l];
    c->kcoe[i] = tc[l];
  }
  c->nk = nk;
  free(idx);
  free(tmp);
  free(tx);
  free(ty);
  free(tz);
  free(tk);
  free(ta);
  free(tc);
}

/* ewald_param (coulomb.f90:363-410) */
static void or_ewald_param(or_ctx* c) {
  double rcut = 0.5 * fmin(c->WA, fmin(c->WB, c->WC));
  double cut = c->p.cutlongrange;
  c->p.cutlongrange = fmin(cut, rcut);
  cut = c->p.cutlongrange;
  double eps = fmin(fabs(c->p.epsw), 0.5);
  double tol = sqrt(fabs(log(eps * cut)));
  double alpha = sqrt(fabs(log(eps * cut * tol))) / cut;
  double tol1 = sqrt(-log(eps * cut * (2.0 * tol * alpha) * (2.0 * tol * alpha)));
  if (c->p.lautoES) {
    c->p.alphaES = alpha;
    for (int i = 0; i < 3; ++i) c->p.kES[i] = (int)fnint(0.25 + c->ANORM[i] * alpha * tol1 / PI);
  }
}

or_ctx* or_create(const mdff_params* pin, const double cell_A[9], int* status) {
  *status = MDFF_OK;
  if (!pin || pin->natm <= 0 || pin->ntype <= 0 || pin->ntype > NT) {
    *status = MDFF_ERR_BAD_ARGS;
    return NULL;
  }
  or_ctx* c = calloc(1, sizeof(or_ctx));
  c->p = *pin;
  int ntype = c->p.ntype, natm = c->p.natm;
  int tot = 0;
  for (int it = 0; it < ntype; ++it) tot += c->p.natmi[it];
  if (tot != natm) {
    *status = MDFF_ERR_BAD_ARGS;
    free(c);
    return NULL;
  }
  c->natm = natm;
  tt_table(c->E_TT);
  /* non_bonded_check_tag (non_bonded.f90:287-301) */
  if (c->p.symmetric_pot_nb) {
    sym2(c->p.epslj, ntype);
    sym2(c->p.sigmalj, ntype);
    sym2(c->p.plj, ntype);
    sym2(c->p.qlj, ntype);
    sym2(c->p.Abmhftd, ntype);
    sym2(c->p.Bbmhftd, ntype);
    sym2(c->p.Cbmhftd, ntype);
    sym2(c->p.Dbmhftd, ntype);
    sym2(c->p.BDbmhftd, ntype);
    sym2(c->p.wall24, ntype);
  }
  /* pim_check_tag (pim.f90:186-204) */
  if (c->p.symmetric_pot_pim) {
    SYM3(c->p.ldip_damping, int);
    SYM3(c->p.pol_damp_b, double);
    SYM3(c->p.pol_damp_c, double);
    SYM3(c->p.pol_damp_k, int);
  }
  for (int a = 0; a < NT; ++a)
    for (int b = 0; b < NT; ++b)
      for (int k = 0; k < NT; ++k)
        if (c->p.pol_damp_k[a][b][k] > TT_MAX || c->p.pol_damp_k[a][b][k] < 0) {
          *status = MDFF_ERR_BAD_ARGS;
          or_destroy(c);
          return NULL;
        }
  /* units (constants.f90:88-94, reduced_units :140-153) */
  c->coul_unit = c->p.lreduced ? 1.0 : COUL_UNIT_EV;
  c->press_unit = c->p.lreduced ? 1.0 : PRESS_UNIT_EV;
  /* initialize_param_non_bonded (non_bonded.f90:455-644) */
  double two16 = pow(2.0, 1.0 / 6.0);
  for (int it = 0; it < ntype; ++it)
    for (int jt = 0; jt < ntype; ++jt) {
      double rcut = c->p.cutshortrange;
      double pp = c->p.plj[it][jt], qq = c->p.qlj[it][jt];
      c->rcutsq[it][jt] = rcut * rcut;
      double ppqq = pp * qq;
      c->epsp[it][jt] = c->p.epslj[it][jt] / (qq - pp);
      c->sigsq[it][jt] = two16 * two16 * c->p.sigmalj[it][jt] * c->p.sigmalj[it][jt];
      double sr2 = c->sigsq[it][jt] / c->rcutsq[it][jt];
      double sr = sqrt(sr2);
      double srp = pow(sr, pp), srq = pow(sr, qq);
      c->uc[it][jt] = c->epsp[it][jt] * (pp * srq - qq * srp);
      c->uc1[it][jt] = c->epsp[it][jt] * ppqq / (2.0 * c->rcutsq[it][jt]) * (srq - srp);
      c->uc2[it][jt] = 0.5 * c->epsp[it][jt] *
                       ((2.0 * pp + ppqq) * srq - (2.0 * qq + ppqq) * srp);
      c->fc[it][jt] = ppqq * c->epsp[it][jt] / c->sigsq[it][jt];
    }
  /* typeinfo_init (read_pos.f90:160-237) */
  c->itype = malloc(sizeof(int) * natm);
  c->ipolar = malloc(sizeof(int) * natm);
  c->qia = malloc(sizeof(double) * natm);
  c->dipia = malloc(sizeof(double) * 3 * natm);
  c->poldipia = calloc(9 * (size_t)natm, sizeof(double));
  c->invpoldipia = calloc(9 * (size_t)natm, sizeof(double));
  c->hist = calloc((size_t)MDFF_ASPC_DEPTH * 3 * natm, sizeof(double));
  /* config.f90:268 allocates xs/ys/zs and nothing sets them before the
     first vnlistcheck; they start at zero here */
  c->xs = calloc((size_t)natm, sizeof(double));
  c->ys = calloc((size_t)natm, sizeof(double));
  c->zs = calloc((size_t)natm, sizeof(double));
  int ia = 0;
  for (int it = 0; it < ntype; ++it) {
    double inv[9];
    int ok = 0;
    if (c->p.ldip_polar[it]) {
      ok = inv3(&c->p.poldip[it][0][0], inv);
      if (ok != 0) {
        *status = MDFF_ERR_BAD_ARGS;
        or_destroy(c);
        return NULL;
      }
    }
    for (int n = 0; n < c->p.natmi[it]; ++n, ++ia) {
      c->itype[ia] = it;
      c->ipolar[ia] = c->p.ldip_polar[it] ? 1 : 0;
      c->qia[ia] = c->p.qch[it];
      for (int a = 0; a < 3; ++a) c->dipia[3 * ia + a] = c->p.dip[it][a];
      for (int a = 0; a < 9; ++a) c->poldipia[9 * ia + a] = (&c->p.poldip[it][0][0])[a];
      if (c->p.ldip_polar[it])
        for (int a = 0; a < 9; ++a) c->invpoldipia[9 * ia + a] = inv[a];
    }
  }
  /* coulomb_check_tag + pim_check_tag task selection (coulomb.f90:204-220,
     pim.f90:160-184) */
  int lqch = 0, ldip = 0, lpol = 0;
  for (int it = 0; it < NT; ++it) {
    if (c->p.qch[it] != 0.0) lqch = 1;
    for (int a = 0; a < 3; ++a)
      if (c->p.dip[it][a] != 0.0) ldip = 1;
  }
  for (int it = 0; it < ntype; ++it)
    if (c->p.ldip_polar[it]) lpol = 1;
  c->lpolar_any = lpol;
  memset(c->task, 0, sizeof(c->task));
  if (lqch) c->task[0] = 1;
  if (ldip || lpol) {
    if (lqch) c->task[1] = 1;
    c->task[2] = 1;
  }
  or_lattice(c, cell_A);
  if (c->p.lcoulomb) {
    or_ewald_param(c);
    or_kmesh(c);
  }
  return c;
}

void or_destroy(or_ctx* c) {
  if (!c) return;
  free(c->itype);
  free(c->ipolar);
  free(c->qia);
  free(c->dipia);
  free(c->poldipia);
  free(c->invpoldipia);
  free(c->hist);
  free(c->xs);
  free(c->ys);
  free(c->zs);
  free(c->kx);
  free(c->ky);
  free(c->kz);
  free(c->kk);
  free(c->Ak);
  free(c->kcoe);
  free(c);
}

int or_get_setup(or_ctx* c, or_setup_info* info) {
  info->alphaES = c->p.alphaES;
  for (int i = 0; i < 3; ++i) info->kES[i] = c->p.kES[i];
  info->nk = c->nk;
  info->cutlongrange = c->p.cutlongrange;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) info->B[i * 3 + j] = c->B[i][j];
  info->omega = c->omega;
  info->WA = c->WA;
  info->WB = c->WB;
  info->WC = c->WC;
  for (int i = 0; i < 6; ++i) info->task[i] = c->task[i];
  return MDFF_OK;
}

int or_get_kmesh(or_ctx* c, double* kx, double* ky, double* kz, double* kk, double* Ak,
                 double* kcoe) {
  size_t n = sizeof(double) * c->nk;
  memcpy(kx, c->kx, n);
  memcpy(ky, c->ky, n);
  memcpy(kz, c->kz, n);
  memcpy(kk, c->kk, n);
  memcpy(Ak, c->Ak, n);
  memcpy(kcoe, c->kcoe, n);
  return MDFF_OK;
}

int or_get_aspc(or_ctx* c, double* buf) {
  memcpy(buf, c->hist, sizeof(double) * MDFF_ASPC_DEPTH * 3 * c->natm);
  return MDFF_OK;
}
int or_set_aspc(or_ctx* c, const double* buf) {
  memcpy(c->hist, buf, sizeof(double) * MDFF_ASPC_DEPTH * 3 * c->natm);
  return MDFF_OK;
}

/* ---------------------------------------------------------------------- */
/* vnlist_pbc (tools.f90:273-368): O(N^2) half lists with the parity mask   */
static int half_mask(int ia, int ja) {
  /* 0-based indices have the same parity of ia+ja as 1-based ones */
  return (ia > ja && ((ia + ja) % 2 == 0)) || (ia < ja && ((ia + ja) % 2 != 0));
}

int or_vnlist(or_ctx* c, const double* rx, const double* ry, const double* rz, int which,
              int* point, int* list, int capacity, int* n_out) {
  int natm = c->natm;
  double cut = (which == 0) ? c->p.cutshortrange : c->p.cutlongrange;
  double rskinsq = cut + c->p.skindiff;
  rskinsq = rskinsq * rskinsq;
  double* sx = malloc(sizeof(double) * natm);
  double* sy = malloc(sizeof(double) * natm);
  double* sz = malloc(sizeof(double) * natm);
  or_kardir(c, rx, ry, rz, sx, sy, sz);
  int icount = 1, status = MDFF_OK;
  for (int ia = 0; ia < natm; ++ia) {
    int k = 0;
    for (int ja = 0; ja < natm; ++ja) {
      if (!half_mask(ia, ja)) continue;
      double rxij, ryij, rzij;
      double rijsq = min_image(c, sx[ia] - sx[ja], sy[ia] - sy[ja], sz[ia] - sz[ja], &rxij,
                               &ryij, &rzij);
      if (rijsq <= rskinsq) {
        icount++;
        k++;
        if (icount - 1 > capacity) {
          status = MDFF_ERR_LIST_OVERFLOW;
        } else {
          list[icount - 2] = ja + 1;
        }
      }
    }
    point[ia] = icount - k;
  }
  point[natm] = icount;
  *n_out = icount - 1;
  free(sx);
  free(sy);
  free(sz);
  return status;
}

/* vnlistcheck (tools.f90:444-537): the largest and second largest
   minimum-image displacement since the last build, with the reference's
   running top-2 update (:494-501); a rebuild when their sum is .gt. skindiff
   (:513), after which the direct coordinates become the new xs/ys/zs
   (:518-524).  The rebuilt lists themselves are or_vnlist's.  Positions are
   not modified (the reference converts rx in place with kardir/dirkar). */
int or_vnlistcheck(or_ctx* c, const double* rx, const double* ry, const double* rz, double* disp,
                   int* rebuilt) {
  int natm = c->natm;
  double* sx = malloc(sizeof(double) * natm);
  double* sy = malloc(sizeof(double) * natm);
  double* sz = malloc(sizeof(double) * natm);
  or_kardir(c, rx, ry, rz, sx, sy, sz);
  double drneimax = 0.0, drneimax2 = 0.0;
  for (int ia = 0; ia < natm; ++ia) {
    double x, y, z;
    double drnei = sqrt(min_image(c, sx[ia] - c->xs[ia], sy[ia] - c->ys[ia], sz[ia] - c->zs[ia],
                                  &x, &y, &z));
    if (drnei > drneimax) {
      drneimax2 = drneimax;
      drneimax = drnei;
    } else if (drnei > drneimax2) {
      drneimax2 = drnei;
    }
  }
  if (disp) *disp = drneimax + drneimax2;
  int r = (drneimax + drneimax2 > c->p.skindiff) ? 1 : 0;
  if (r) {
    memcpy(c->xs, sx, sizeof(double) * natm);
    memcpy(c->ys, sy, sizeof(double) * natm);
    memcpy(c->zs, sz, sizeof(double) * natm);
  }
  if (rebuilt) *rebuilt = r;
  free(sx);
  free(sy);
  free(sz);
  return MDFF_OK;
}

/* CSR half list, 0-based, for internal use */
typedef struct {
  int* point;
  int* list;
  int n;
} csr_t;

static void build_half(or_ctx* c, const double* sx, const double* sy, const double* sz, double cut,
                       csr_t* out) {
  int natm = c->natm;
  double rskinsq = cut + c->p.skindiff;
  rskinsq = rskinsq * rskinsq;
  int* cnt = calloc(natm + 1, sizeof(int));
  int nth = or_get_threads();
#pragma omp parallel for schedule(dynamic, 16) num_threads(nth)
  for (int ia = 0; ia < natm; ++ia) {
    int k = 0;
    for (int ja = 0; ja < natm; ++ja) {
      if (!half_mask(ia, ja)) continue;
      double x, y, z;
      if (min_image(c, sx[ia] - sx[ja], sy[ia] - sy[ja], sz[ia] - sz[ja], &x, &y, &z) <= rskinsq)
        k++;
    }
    cnt[ia] = k;
  }
  out->point = malloc(sizeof(int) * (natm + 1));
  out->point[0] = 0;
  for (int ia = 0; ia < natm; ++ia) out->point[ia + 1] = out->point[ia] + cnt[ia];
  out->n = out->point[natm];
  out->list = malloc(sizeof(int) * (out->n > 0 ? out->n : 1));
#pragma omp parallel for schedule(dynamic, 16) num_threads(nth)
  for (int ia = 0; ia < natm; ++ia) {
    int o = out->point[ia];
    for (int ja = 0; ja < natm; ++ja) {
      if (!half_mask(ia, ja)) continue;
      double x, y, z;
      if (min_image(c, sx[ia] - sx[ja], sy[ia] - sy[ja], sz[ia] - sz[ja], &x, &y, &z) <= rskinsq)
        out->list[o++] = ja;
    }
  }
  free(cnt);
}
static void free_csr(csr_t* l) {
  free(l->point);
  free(l->list);
}

/* ---------------------------------------------------------------------- */
/* engforce_bmhftd_pbc (non_bonded.f90:1076-1228) + optional r^-24 wall      */
static void or_bmhftd(or_ctx* c, const double* sx, const double* sy, const double* sz,
                      const csr_t* L, double* fx, double* fy, double* fz, double* u_out,
                      double* vir_out, double tau[3][3]) {
  int natm = c->natm;
  int lbmhftd = c->p.lbmhftd;
  double u = 0.0, vir = 0.0;
  double t[3][3] = {{0}};
  memset(fx, 0, sizeof(double) * natm);
  memset(fy, 0, sizeof(double) * natm);
  memset(fz, 0, sizeof(double) * natm);
  for (int ia = 0; ia < natm; ++ia) {
    for (int j1 = L->point[ia]; j1 < L->point[ia + 1]; ++j1) {
      int ja = L->list[j1];
      if (ja == ia) continue;
      double rxij, ryij, rzij;
      double rijsq =
          min_image(c, sx[ia] - sx[ja], sy[ia] - sy[ja], sz[ia] - sz[ja], &rxij, &ryij, &rzij);
      int p1 = c->itype[ia], p2 = c->itype[ja];
      /* the reference skips pairs with A = 0 (non_bonded.f90:1153); the
         optional wall extension acts on its own */
      double Aij = c->p.Abmhftd[p1][p2], Wij = c->p.wall24[p1][p2];
      if (Aij == 0.0 && Wij == 0.0) continue;
      if (rijsq < c->rcutsq[p1][p2]) {
        double ir2 = 1.0 / rijsq;
        double d = sqrt(rijsq);
        double u_pair = 0.0, wnum = 0.0;
        if (Aij != 0.0) {
          double erh = Aij * exp(-c->p.Bbmhftd[p1][p2] * d);
          double ir6 = ir2 * ir2 * ir2;
          double ir8 = ir6 * ir2;
          ir6 = ir6 * c->p.Cbmhftd[p1][p2];
          ir8 = ir8 * c->p.Dbmhftd[p1][p2];
          double f6, f8, fdiff6, fdiff8, ir6d, ir8d;
          if (lbmhftd) {
            tt_damp_tab(c->E_TT, c->p.BDbmhftd[p1][p2], 1.0, d, 6, &f6, &fdiff6);
            tt_damp_tab(c->E_TT, c->p.BDbmhftd[p1][p2], 1.0, d, 8, &f8, &fdiff8);
            ir6d = ir6 * f6;
            ir8d = ir8 * f8;
          } else {
            fdiff6 = 0.0;
            fdiff8 = 0.0;
            ir6d = ir6;
            ir8d = ir8;
          }
          double ir7 = 6.0 * ir6d / d;
          double ir9 = 8.0 * ir8d / d;
          u_pair = erh - ir6d - ir8d;
          wnum = c->p.Bbmhftd[p1][p2] * erh - ir7 - ir9 + ir6 * fdiff6 + ir8 * fdiff8;
        }
        if (Wij != 0.0) {
          double ir8r = (ir2 * ir2) * (ir2 * ir2);
          double uw = Wij * (ir8r * ir8r * ir8r);
          u_pair = u_pair + uw;
          wnum = wnum + 24.0 * uw / d;
        }
        u = u + u_pair;
        double wij = wnum / d;
        double fxij = wij * rxij, fyij = wij * ryij, fzij = wij * rzij;
        vir = vir + (rxij * fxij + ryij * fyij + rzij * fzij);
        fx[ia] += fxij;
        fy[ia] += fyij;
        fz[ia] += fzij;
        fx[ja] -= fxij;
        fy[ja] -= fyij;
        fz[ja] -= fzij;
        double r[3] = {rxij, ryij, rzij}, f[3] = {fxij, fyij, fzij};
        for (int a = 0; a < 3; ++a)
          for (int b = 0; b < 3; ++b) t[a][b] += (r[a] * f[b] + r[b] * f[a]);
      }
    }
  }
  vir = vir / 3.0;
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) tau[a][b] = t[a][b] / c->omega / c->press_unit * 0.5;
  *u_out = u;
  *vir_out = vir;
}

/* engforce_nmlj_pbc (non_bonded.f90:660-827) */
static void or_nmlj(or_ctx* c, const double* sx, const double* sy, const double* sz,
                    const csr_t* L, double* fx, double* fy, double* fz, double* u_out,
                    double* vir_out, double tau[3][3]) {
  int natm = c->natm, trunc = c->p.trunc;
  double u = 0.0, vir = 0.0;
  double t[3][3] = {{0}};
  memset(fx, 0, sizeof(double) * natm);
  memset(fy, 0, sizeof(double) * natm);
  memset(fz, 0, sizeof(double) * natm);
  for (int ia = 0; ia < natm; ++ia) {
    for (int j1 = L->point[ia]; j1 < L->point[ia + 1]; ++j1) {
      int ja = L->list[j1];
      if (ja == ia) continue;
      double rxij, ryij, rzij;
      double rijsq =
          min_image(c, sx[ia] - sx[ja], sy[ia] - sy[ja], sz[ia] - sz[ja], &rxij, &ryij, &rzij);
      int p1 = c->itype[ia], p2 = c->itype[ja];
      if (rijsq < c->rcutsq[p1][p2]) {
        double sr2 = c->sigsq[p1][p2] / rijsq;
        double srp = pow(sr2, c->p.plj[p1][p2] * 0.5);
        double srq = pow(sr2, c->p.qlj[p1][p2] * 0.5);
        double e = c->epsp[p1][p2] * (c->p.plj[p1][p2] * srq - c->p.qlj[p1][p2] * srp);
        if (trunc == 0) u = u + e;
        if (trunc == 1) u = u + e - c->uc[p1][p2];
        if (trunc == 2) u = u + e + c->uc1[p1][p2] * rijsq - c->uc2[p1][p2];
        double wij = c->fc[p1][p2] * (srq - srp) * sr2;
        double fxij = wij * rxij, fyij = wij * ryij, fzij = wij * rzij;
        vir = vir + wij * rijsq;
        fx[ia] += fxij;
        fy[ia] += fyij;
        fz[ia] += fzij;
        fx[ja] -= fxij;
        fy[ja] -= fyij;
        fz[ja] -= fzij;
        double r[3] = {rxij, ryij, rzij}, f[3] = {fxij, fyij, fzij};
        for (int a = 0; a < 3; ++a)
          for (int b = 0; b < 3; ++b) t[a][b] += (r[a] * f[b] + r[b] * f[a]) * 0.5;
      }
    }
  }
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) tau[a][b] = t[a][b] / c->omega / c->press_unit;
  *u_out = u;
  *vir_out = vir / 3.0;
}

/* ---------------------------------------------------------------------- */
/* Thole functions on the dd tensor of a pair of polarisable ions
 * (ewald_dir.f90:305-430): F1, F2 (Ewald radial functions) -> the damped
 * F1, F2 of T2_thole = 3 r r F2 / d^5 - F1 / d^3.  A = (alpha_i alpha_j)^(1/6)
 * with alpha = poldipia(1,1) (:164, :194); a = thole_param(ita, jta).        */
static void thole_f(int type, double a, double alpha_i, double alpha_j, double d, double* F1,
                    double* F2) {
  const double onesixth = 1.0 / 6.0, twothird = onesixth * 4.0;
  const double twopiroot = 2.0 / sqrt(PI);
  if (type == MDFF_THOLE_LINEAR) {
    /* linear (:316-347): no Ewald screening inside s = a A */
    double s = a * pow(alpha_i * alpha_j, onesixth);
    if (d < s) {
      double v = d / s;
      double v3 = v * v * v, v4 = v3 * v;
      *F2 = v4;
      *F1 = 4.0 * v3 - 3.0 * v4;
    }
  } else if (type == MDFF_THOLE_EXPON1) {
    /* expon1 (:353-373) */
    double A = pow(alpha_i * alpha_j, onesixth);
    double u = a * pow(d / A, 3.0);
    double e = exp(-u);
    *F2 = *F2 * (1.0 - (1.0 + u) * e);
    *F1 = *F1 * (1.0 - e);
  } else if (type == MDFF_THOLE_EXPON2) {
    /* expon2 (:378-399), u = a d A as written there */
    double A = pow(alpha_i * alpha_j, onesixth);
    double ar = a * d * A;
    double ar2 = ar * ar / 2.0;
    double ar3 = ar2 * ar / 3.0;
    double e = exp(-ar);
    *F2 = *F2 * (1.0 - (1.0 + ar + ar2 + ar3) * e);
    *F1 = *F1 * (1.0 - (1.0 + ar + ar2) * e);
  } else if (type == MDFF_THOLE_GAUSS) {
    /* gauss (:404-422) with the NR error function (functions.f90:44-50) */
    double ra = d / a;
    double At = twopiroot * ra;
    double e = At * exp(-ra * ra);
    double erfra = 1.0 - or_errfc(ra);
    *F2 = *F2 * (erfra - e * (1.0 + twothird * ra));
    *F1 = *F1 * (erfra - e);
  }
}

/* multipole_ES_dir (ewald_dir.f90:40-798), tasks qq / qd / dd              */
typedef struct {
  double u;
  double* ef;   /* [natm][3] */
  double* efg;  /* [natm][9] */
  double* f;    /* [natm][3] */
  double tau[3][3];
} es_acc;

static void es_dir(or_ctx* c, const double* sx, const double* sy, const double* sz,
                   const csr_t* L, const double* q, const double* mu, const int* task, int damp_ind,
                   int do_efield, int do_efg, int do_forces, int do_stress, es_acc* out) {
  int natm = c->natm;
  const mdff_params* p = &c->p;
  double alphaES = p->alphaES;
  double cutsq = p->cutlongrange * p->cutlongrange;
  double alpha2 = alphaES * alphaES, alpha3 = alpha2 * alphaES, alpha5 = alpha3 * alpha2;
  double alpha7 = alpha5 * alpha2, alpha9 = alpha7 * alpha2;
  double piroot = sqrt(PI);
  int charge_charge = task[0], charge_dipole = task[1], dipole_dipole = task[2];
  int nth = or_get_threads();
  double u_tot = 0.0;
  double tau_tot[9] = {0};
  double* ef_t = calloc((size_t)nth * natm * 3, sizeof(double));
  double* efg_t = do_efg ? calloc((size_t)nth * natm * 9, sizeof(double)) : NULL;
  double* f_t = calloc((size_t)nth * natm * 3, sizeof(double));
#pragma omp parallel num_threads(nth) reduction(+ : u_tot)
  {
    int tid = 0;
#ifdef _OPENMP
    tid = omp_get_thread_num();
#endif
    double* ef = ef_t + (size_t)tid * natm * 3;
    double* efg = efg_t ? efg_t + (size_t)tid * natm * 9 : NULL;
    double* fo = f_t + (size_t)tid * natm * 3;
    double tl[3][3] = {{0}};
    double u_dir = 0.0;
#pragma omp for schedule(dynamic, 8)
    for (int ia = 0; ia < natm; ++ia) {
      int ita = c->itype[ia];
      double qi = q[ia];
      const double* mui = mu + 3 * ia;
      int dip_i = (mui[0] != 0.0 || mui[1] != 0.0 || mui[2] != 0.0);
      for (int j1 = L->point[ia]; j1 < L->point[ia + 1]; ++j1) {
        int ja = L->list[j1];
        if (ja == ia) continue;
        double fij[3] = {0.0, 0.0, 0.0};
        int jta = c->itype[ja];
        double qj = q[ja];
        const double* muj = mu + 3 * ja;
        int dip_j = (muj[0] != 0.0 || muj[1] != 0.0 || muj[2] != 0.0);
        double qij = qi * qj;
        double r[3];
        double d2 = min_image(c, sx[ia] - sx[ja], sy[ia] - sy[ja], sz[ia] - sz[ja], &r[0], &r[1],
                              &r[2]);
        if (d2 > cutsq) continue;
        double d = sqrt(d2);
        double d3 = d2 * d, d5 = d3 * d2, d7 = d5 * d2;
        double dm1 = 1.0 / d;
        double dm3 = dm1 / d2, dm5 = dm3 / d2, dm7 = dm5 / d2;
        /* damping (ewald_dir.f90:216-228) */
        int ldamp = p->ldip_damping[ita][ita][jta] || p->ldip_damping[jta][ita][jta];
        if (!damp_ind) ldamp = 0;
        double fdamp = 1.0, fdamp2 = 1.0, fdampdiff = 0.0, fdampdiff2 = 0.0;
        if (ldamp) {
          tt_damp_tab(c->E_TT, p->pol_damp_b[ita][ita][jta], p->pol_damp_c[ita][ita][jta], d,
                      p->pol_damp_k[ita][ita][jta], &fdamp, &fdampdiff);
          tt_damp_tab(c->E_TT, p->pol_damp_b[jta][ita][jta], p->pol_damp_c[jta][ita][jta], d,
                      p->pol_damp_k[jta][ita][jta], &fdamp2, &fdampdiff2);
        }
        double expon = exp(-alpha2 * d2) / piroot;
        double F0 = or_errfc(alphaES * d);
        double F1 = F0 + 2.0 * alphaES * d * expon;
        double F2 = F1 + 4.0 * alpha3 * d3 * expon / 3.0;
        double F3 = F2 + 8.0 * alpha5 * d5 * expon / 15.0;
        (void)alpha7;
        (void)alpha9;
        double F1d = -fdamp + 1.0;
        double F2d = F1d + (d / 3.0) * fdampdiff;
        double F1d2 = -fdamp2 + 1.0;
        double F2d2 = F1d2 + (d / 3.0) * fdampdiff2;
        double T0 = dm1 * F0;
        double T1[3], T1d[3], T1d2[3];
        for (int a = 0; a < 3; ++a) {
          T1[a] = -r[a] * dm3;
          if (ldamp) {
            T1d[a] = T1[a] * F1d;
            T1d2[a] = T1[a] * F1d2;
          }
          T1[a] = T1[a] * F1;
        }
        double F2_dm5 = 3.0 * F2 * dm5, F2d_dm5 = 3.0 * F2d * dm5, F2d2_dm5 = 3.0 * F2d2 * dm5;
        double F1_dm3 = F1 * dm3, F1d_dm3 = F1d * dm3, F1d2_dm3 = F1d2 * dm3;
        double T2[3][3], T2d[3][3], T2d2[3][3];
        for (int a = 0; a < 3; ++a)
          for (int b = 0; b < 3; ++b) {
            T2[a][b] = r[a] * r[b] * F2_dm5;
            if (a == b) T2[a][a] = T2[a][a] - F1_dm3;
            if (ldamp) {
              T2d[a][b] = r[a] * r[b] * F2d_dm5;
              T2d2[a][b] = r[a] * r[b] * F2d2_dm5;
              if (a == b) {
                T2d[a][a] = T2d[a][a] - F1d_dm3;
                T2d2[a][a] = T2d2[a][a] - F1d2_dm3;
              }
            }
          }
        double F3_dm7 = F3 * dm7 * 15.0;
        double T3[3][3][3];
        for (int i = 0; i < 3; ++i)
          for (int j = 0; j < 3; ++j)
            for (int k = 0; k < 3; ++k) {
              double v = -r[i] * r[j] * r[k] * F3_dm7;
              if (i == j) v = v + r[k] * F2_dm5;
              if (i == k) v = v + r[j] * F2_dm5;
              if (j == k) v = v + r[i] * F2_dm5;
              T3[i][j][k] = v;
            }
        /* qq (ewald_dir.f90:528-553) */
        if (charge_charge) {
          u_dir = u_dir + qij * T0;
          if (do_efield) {
            for (int a = 0; a < 3; ++a) {
              ef[3 * ia + a] = ef[3 * ia + a] - qj * T1[a];
              ef[3 * ja + a] = ef[3 * ja + a] + qi * T1[a];
            }
            if (ldamp)
              for (int a = 0; a < 3; ++a) {
                ef[3 * ia + a] = ef[3 * ia + a] + qj * T1d[a];
                ef[3 * ja + a] = ef[3 * ja + a] - qi * T1d2[a];
              }
          }
          if (do_efg)
            for (int a = 0; a < 3; ++a)
              for (int b = 0; b < 3; ++b) {
                efg[9 * ia + 3 * a + b] -= qj * T2[a][b];
                efg[9 * ja + 3 * a + b] -= qi * T2[a][b];
              }
          if (do_forces)
            for (int a = 0; a < 3; ++a) fij[a] = fij[a] + qij * T1[a];
        }
        /* dd (ewald_dir.f90:557-593): energy and field with T2_thole (= T2
         * without Thole functions or unless both ions are polarisable), forces
         * with T3 */
        if (dipole_dipole && (dip_i && dip_j)) {
          double T2t[3][3];
          memcpy(T2t, T2, sizeof(T2t));
          if (p->thole_type != MDFF_THOLE_NONE && p->ldip_polar[ita] && p->ldip_polar[jta]) {
            double F1t = F1, F2t = F2;
            thole_f(p->thole_type, p->thole_param[ita][jta], p->poldip[ita][0][0],
                    p->poldip[jta][0][0], d, &F1t, &F2t);
            double F2t_dm5 = 3.0 * F2t * dm5, F1t_dm3 = F1t * dm3;
            for (int a = 0; a < 3; ++a)
              for (int b = 0; b < 3; ++b) {
                T2t[a][b] = r[a] * r[b] * F2t_dm5;
                if (a == b) T2t[a][a] = T2t[a][a] - F1t_dm3;
              }
          }
          for (int j = 0; j < 3; ++j)
            for (int k = 0; k < 3; ++k) u_dir = u_dir - mui[j] * T2t[j][k] * muj[k];
          if (do_efield)
            for (int k = 0; k < 3; ++k)
              for (int a = 0; a < 3; ++a) {
                ef[3 * ia + a] = ef[3 * ia + a] + T2t[a][k] * muj[k];
                ef[3 * ja + a] = ef[3 * ja + a] + T2t[a][k] * mui[k];
              }
          if (do_efg)
            for (int k = 0; k < 3; ++k)
              for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b) {
                  efg[9 * ia + 3 * a + b] += T3[a][b][k] * muj[k];
                  efg[9 * ja + 3 * a + b] -= T3[a][b][k] * mui[k];
                }
          if (do_forces)
            for (int j = 0; j < 3; ++j)
              for (int k = 0; k < 3; ++k)
                for (int a = 0; a < 3; ++a) fij[a] = fij[a] - mui[j] * T3[j][a][k] * muj[k];
        }
        /* qd (ewald_dir.f90:599-644) */
        if (charge_dipole && (dip_i || dip_j)) {
          for (int k = 0; k < 3; ++k) {
            u_dir = u_dir - qi * T1[k] * muj[k];
            u_dir = u_dir + qj * T1[k] * mui[k];
            if (ldamp) {
              u_dir = u_dir + qi * T1d2[k] * muj[k];
              u_dir = u_dir - qj * T1d[k] * mui[k];
            }
          }
          if (do_forces) {
            for (int j = 0; j < 3; ++j)
              for (int k = 0; k < 3; ++k) {
                fij[k] = fij[k] - qi * T2[k][j] * muj[j];
                fij[k] = fij[k] + qj * T2[k][j] * mui[j];
              }
          }
          if (ldamp && do_forces)
            for (int j = 0; j < 3; ++j)
              for (int k = 0; k < 3; ++k) {
                fij[k] = fij[k] - qj * T2d[j][k] * mui[j];
                fij[k] = fij[k] + qi * T2d2[j][k] * muj[j];
              }
        }
        if (do_forces)
          for (int a = 0; a < 3; ++a) {
            fo[3 * ia + a] -= fij[a];
            fo[3 * ja + a] += fij[a];
          }
        if (do_stress)
          for (int j = 0; j < 3; ++j)
            for (int k = 0; k < 3; ++k) tl[j][k] = tl[j][k] - (r[j] * fij[k] + r[k] * fij[j]);
      }
    }
    u_tot += u_dir;
#pragma omp critical
    {
      for (int j = 0; j < 3; ++j)
        for (int k = 0; k < 3; ++k) tau_tot[3 * j + k] += tl[j][k];
    }
  }
  /* thread reduction, fixed order */
  for (int t = 0; t < nth; ++t) {
    for (size_t i = 0; i < (size_t)natm * 3; ++i) {
      out->ef[i] += ef_t[(size_t)t * natm * 3 + i];
      out->f[i] += f_t[(size_t)t * natm * 3 + i];
    }
    if (do_efg)
      for (size_t i = 0; i < (size_t)natm * 9; ++i) out->efg[i] += efg_t[(size_t)t * natm * 9 + i];
  }
  out->u = u_tot;
  for (int j = 0; j < 3; ++j)
    for (int k = 0; k < 3; ++k)
      out->tau[j][k] = do_stress ? tau_tot[3 * j + k] / c->omega * 0.5 : 0.0;
  free(ef_t);
  free(efg_t);
  free(f_t);
}

/* multipole_ES_rec (ewald_rec.f90:38-365) */
static void es_rec(or_ctx* c, const double* rx, const double* ry, const double* rz,
                   const double* q, const double* mu, const int* task, int do_efield, int do_efg,
                   int do_forces, int do_stress, es_acc* out) {
  int natm = c->natm;
  double tpi_V = TPI / c->omega, fpi_V = tpi_V * 2.0;
  int ldip = task[1] || task[2];
  int nth = or_get_threads();
  double u_rec = 0.0;
  double tr[3][3] = {{0}};
  double* ef_t = calloc((size_t)nth * natm * 3, sizeof(double));
  double* efg_t = do_efg ? calloc((size_t)nth * natm * 9, sizeof(double)) : NULL;
  double* f_t = calloc((size_t)nth * natm * 3, sizeof(double));
  double* str_k = calloc(c->nk, sizeof(double));
#pragma omp parallel num_threads(nth)
  {
    int tid = 0;
#ifdef _OPENMP
    tid = omp_get_thread_num();
#endif
    double* ef = ef_t + (size_t)tid * natm * 3;
    double* efg = efg_t ? efg_t + (size_t)tid * natm * 9 : NULL;
    double* fo = f_t + (size_t)tid * natm * 3;
    double* ckr = malloc(sizeof(double) * natm);
    double* skr = malloc(sizeof(double) * natm);
#pragma omp for schedule(dynamic, 4)
    for (int ik = 0; ik < c->nk; ++ik) {
      if (c->kk[ik] == 0.0) continue;
      double kx = c->kx[ik], ky = c->ky[ik], kz = c->kz[ik], Ak = c->Ak[ik];
      double rhonk_R = 0.0, rhonk_I = 0.0;
      for (int ia = 0; ia < natm; ++ia) {
        double qi = q[ia];
        double k_dot_r = (kx * rx[ia] + ky * ry[ia] + kz * rz[ia]);
        ckr[ia] = cos(k_dot_r);
        skr[ia] = sin(k_dot_r);
        rhonk_R = rhonk_R + qi * ckr[ia];
        rhonk_I = rhonk_I + qi * skr[ia];
        if (!ldip) continue;
        double k_dot_mu = (mu[3 * ia] * kx + mu[3 * ia + 1] * ky + mu[3 * ia + 2] * kz);
        rhonk_R = rhonk_R - k_dot_mu * skr[ia];
        rhonk_I = rhonk_I + k_dot_mu * ckr[ia];
      }
      double str = (rhonk_R * rhonk_R + rhonk_I * rhonk_I) * Ak;
      str_k[ik] = str;
      for (int ia = 0; ia < natm; ++ia) {
        double ckria = ckr[ia], skria = skr[ia];
        double recarg2 = Ak * (rhonk_R * ckria + rhonk_I * skria);
        double recarg = Ak * (rhonk_I * ckria - rhonk_R * skria);
        double fxij = kx * recarg, fyij = ky * recarg, fzij = kz * recarg;
        if (do_efield) {
          ef[3 * ia] -= fxij;
          ef[3 * ia + 1] -= fyij;
          ef[3 * ia + 2] -= fzij;
        }
        if (do_efg) {
          /* only the upper triangle is accumulated (ewald_rec.f90:209-217) */
          efg[9 * ia + 0] += kx * kx * recarg2;
          efg[9 * ia + 4] += ky * ky * recarg2;
          efg[9 * ia + 8] += kz * kz * recarg2;
          efg[9 * ia + 1] += kx * ky * recarg2;
          efg[9 * ia + 2] += kx * kz * recarg2;
          efg[9 * ia + 5] += ky * kz * recarg2;
        }
        if (do_forces) {
          double qi = q[ia];
          fo[3 * ia] -= qi * fxij;
          fo[3 * ia + 1] -= qi * fyij;
          fo[3 * ia + 2] -= qi * fzij;
          if (!ldip) continue;
          double k_dot_mu =
              (mu[3 * ia] * kx + mu[3 * ia + 1] * ky + mu[3 * ia + 2] * kz) * recarg2;
          fo[3 * ia] += kx * k_dot_mu;
          fo[3 * ia + 1] += ky * k_dot_mu;
          fo[3 * ia + 2] += kz * k_dot_mu;
        }
      }
    }
    free(ckr);
    free(skr);
  }
  /* energy and stress in k order (ewald_rec.f90:173, 252-263) */
  for (int ik = 0; ik < c->nk; ++ik) {
    if (c->kk[ik] == 0.0) continue;
    double str = str_k[ik];
    u_rec = u_rec + str;
    if (do_stress) {
      double kv[3] = {c->kx[ik], c->ky[ik], c->kz[ik]}, kcoe = c->kcoe[ik];
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) {
          if (a == b)
            tr[a][a] = tr[a][a] + (1.0 - kcoe * kv[a] * kv[a]) * str;
          else
            tr[a][b] = tr[a][b] - kcoe * kv[a] * kv[b] * str;
        }
    }
  }
  for (int t = 0; t < nth; ++t) {
    for (size_t i = 0; i < (size_t)natm * 3; ++i) {
      out->ef[i] += ef_t[(size_t)t * natm * 3 + i] * 2.0 * fpi_V;
      out->f[i] += f_t[(size_t)t * natm * 3 + i] * 2.0 * fpi_V;
    }
    if (do_efg)
      for (size_t i = 0; i < (size_t)natm * 9; ++i)
        out->efg[i] += efg_t[(size_t)t * natm * 9 + i] * 2.0 * fpi_V;
  }
  out->u = u_rec * 2.0 * tpi_V;
  if (do_stress) {
    double tmp[3][3];
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) tmp[a][b] = tr[a][b] * 2.0;
    double s[3][3];
    for (int a = 0; a < 3; ++a) s[a][a] = tmp[a][a];
    s[0][1] = s[1][0] = (tmp[0][1] + tmp[1][0]) * 0.5;
    s[0][2] = s[2][0] = (tmp[0][2] + tmp[2][0]) * 0.5;
    s[1][2] = s[2][1] = (tmp[1][2] + tmp[2][1]) * 0.5;
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) out->tau[a][b] = s[a][b] * tpi_V / c->omega;
  } else {
    memset(out->tau, 0, sizeof(out->tau));
  }
  free(ef_t);
  free(efg_t);
  free(f_t);
  free(str_k);
}

/* multipole_ES (ewald.f90:49-314).  Adds forces into f (already scaled by
   coul_unit), returns u_coul (with u_pol), field ef (internal units), efg
   (x coul_unit), tau_coul (x coul_unit / press_unit). */
typedef struct {
  double u_coul, u_dir, u_rec, u_self, u_surf;
  double tau_coul[3][3];
  double pvirial_coul;
} es_out;

static void multipole_ES(or_ctx* c, const double* rx, const double* ry, const double* rz,
                         const double* sx, const double* sy, const double* sz, const csr_t* L,
                         const double* q, const double* mu, const int* task, int damp_ind,
                         int do_efield, int do_efg, int do_forces, int do_stress, int do_rec,
                         double u_pol, double* ef, double* efg, double* f /* [natm][3], += */,
                         es_out* o) {
  int natm = c->natm;
  double alphaES = c->p.alphaES;
  double piroot = sqrt(PI);
  double qtot[3] = {0, 0, 0}, mutot[3] = {0, 0, 0}, qsq = 0.0, musq = 0.0;
  for (int ia = 0; ia < natm; ++ia) {
    mutot[0] += mu[3 * ia];
    mutot[1] += mu[3 * ia + 1];
    mutot[2] += mu[3 * ia + 2];
    musq = musq + (mu[3 * ia] * mu[3 * ia] + mu[3 * ia + 1] * mu[3 * ia + 1] +
                   mu[3 * ia + 2] * mu[3 * ia + 2]);
    qtot[0] += q[ia] * rx[ia];
    qtot[1] += q[ia] * ry[ia];
    qtot[2] += q[ia] * rz[ia];
    qsq = qsq + q[ia] * q[ia];
  }
  double qmu_sum[3] = {qtot[0] + mutot[0], qtot[1] + mutot[1], qtot[2] + mutot[2]};
  double tpi_V = TPI / c->omega;
  double tpi_3V = tpi_V / 3.0;
  double fpi_3V = tpi_3V * 2.0;
  double alpha2 = alphaES * alphaES;
  double selfa = alphaES / piroot;
  double selfa2 = 2.0 * selfa * alpha2 / 3.0;

  es_acc dir = {0}, rec = {0};
  dir.ef = calloc((size_t)natm * 3, sizeof(double));
  dir.f = calloc((size_t)natm * 3, sizeof(double));
  dir.efg = calloc((size_t)natm * 9, sizeof(double));
  rec.ef = calloc((size_t)natm * 3, sizeof(double));
  rec.f = calloc((size_t)natm * 3, sizeof(double));
  rec.efg = calloc((size_t)natm * 9, sizeof(double));
  es_dir(c, sx, sy, sz, L, q, mu, task, damp_ind, do_efield, do_efg, do_forces, do_stress, &dir);
  c->n_kardir++; /* ewald_dir.f90:138,739 */
  if (do_rec) es_rec(c, rx, ry, rz, q, mu, task, do_efield, do_efg, do_forces, do_stress, &rec);

  double u_surf = (qtot[0] * qtot[0] + qtot[1] * qtot[1] + qtot[2] * qtot[2]) +
                  2.0 * (qtot[0] * mutot[0] + qtot[1] * mutot[1] + qtot[2] * mutot[2]) +
                  (mutot[0] * mutot[0] + mutot[1] * mutot[1] + mutot[2] * mutot[2]);
  u_surf = u_surf * tpi_3V;
  double u_self = -selfa * qsq - selfa2 * musq;
  int lsurf = c->p.lsurf;
  double cu = c->coul_unit;
  o->u_dir = dir.u;
  o->u_rec = rec.u;
  o->u_self = u_self;
  o->u_surf = lsurf ? u_surf : 0.0;
  o->u_coul = (dir.u + rec.u + (lsurf ? u_surf : 0.0) + u_self + u_pol) * cu;
  for (int ia = 0; ia < natm; ++ia)
    for (int a = 0; a < 3; ++a) {
      double e = dir.ef[3 * ia + a] + rec.ef[3 * ia + a];
      if (lsurf) e += -qmu_sum[a] * fpi_3V;
      e += 2.0 * selfa2 * mu[3 * ia + a];
      if (ef) ef[3 * ia + a] = e;
      f[3 * ia + a] += (rec.f[3 * ia + a] + dir.f[3 * ia + a]) * cu;
    }
  if (efg)
    for (int ia = 0; ia < natm; ++ia)
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) {
          double s = (a == b) ? -2.0 * selfa2 * q[ia] : 0.0;
          efg[9 * ia + 3 * a + b] = (dir.efg[9 * ia + 3 * a + b] + rec.efg[9 * ia + 3 * a + b] + s) * cu;
        }
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b)
      o->tau_coul[a][b] = (dir.tau[a][b] + rec.tau[a][b]) * cu / c->press_unit;
  o->pvirial_coul =
      1.0 / 3.0 * (o->tau_coul[0][0] + o->tau_coul[1][1] + o->tau_coul[2][2]) * c->press_unit;
  free(dir.ef);
  free(dir.f);
  free(dir.efg);
  free(rec.ef);
  free(rec.f);
  free(rec.efg);
}

/* induced_moment (moment_from_pola.f90:955-993) */
static void induced_moment(or_ctx* c, const double* E, double* mu_ind) {
  for (int ia = 0; ia < c->natm; ++ia) {
    for (int a = 0; a < 3; ++a) mu_ind[3 * ia + a] = 0.0;
    if (!c->ipolar[ia]) continue;
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b)
        mu_ind[3 * ia + a] = mu_ind[3 * ia + a] + c->poldipia[9 * ia + 3 * a + b] * E[3 * ia + b];
  }
}

/* get_rmsd_mu (moment_from_pola.f90:998-1027) */
static double get_rmsd_mu(or_ctx* c, const double* g0, const double* mu) {
  double rmsd = 0.0;
  int npol = 0;
  for (int ia = 0; ia < c->natm; ++ia) {
    if (!c->ipolar[ia]) continue;
    npol++;
    for (int a = 0; a < 3; ++a) {
      double al = c->poldipia[9 * ia + 4 * a];
      if (al == 0.0) continue;
      double d = mu[3 * ia + a] / al - g0[3 * ia + a];
      rmsd = rmsd + d * d;
    }
  }
  return sqrt(rmsd / (double)npol);
}

/* extrapolate_dipole_aspc (moment_from_pola.f90:493-598) */
static void aspc(or_ctx* c, double* mu_ind, const double* Efield, int key, int itime) {
  int natm = c->natm, eo = c->p.extrapolate_order, ext_ord;
  if (itime >= eo + 1)
    ext_ord = eo;
  else if (itime == 1 || itime == 0)
    ext_ord = 0;
  else
    ext_ord = itime - 1;
  double B[6] = {0}, W = 0.0;
  switch (ext_ord) {
    case 0: B[0] = 1.0; W = 0.0; break;
    case 1: B[0] = 2.0; B[1] = -1.0; W = 2.0 / 3.0; break;
    case 2: B[0] = 2.5; B[1] = -2.0; B[2] = 0.5; W = 0.6; break;
    case 3: B[0] = 2.8; B[1] = -2.8; B[2] = 1.2; B[3] = -0.2; W = 4.0 / 7.0; break;
    case 4:
      B[0] = 3.0; B[1] = -24.0 / 7.0; B[2] = 27.0 / 14.0; B[3] = -4.0 / 7.0; B[4] = 1.0 / 14.0;
      W = 5.0 / 9.0;
      break;
    default: break;
  }
  size_t n3 = (size_t)natm * 3;
  if (key == 1) {
    for (size_t i = 0; i < n3; ++i) {
      double s = 0.0;
      for (int k = 0; k < ext_ord + 1; ++k) s = s + B[k] * c->hist[k * n3 + i];
      mu_ind[i] = s;
    }
    for (int k = ext_ord; k >= 1; --k) memcpy(c->hist + k * n3, c->hist + (k - 1) * n3, sizeof(double) * n3);
  } else {
    double* save = malloc(sizeof(double) * n3);
    memcpy(save, mu_ind, sizeof(double) * n3);
    induced_moment(c, Efield, mu_ind);
    for (size_t i = 0; i < n3; ++i) mu_ind[i] = W * mu_ind[i] + (1.0 - W) * save[i];
    free(save);
  }
}

/* One configuration seen by the induced-dipole solvers. */
typedef struct {
  or_ctx* c;
  const double *rx, *ry, *rz, *sx, *sy, *sz;
  const csr_t* L;
  const double* qzero;  /* charges set to zero (moment_from_pola.f90:345-349) */
  double* fsink;        /* [natm][3] force sink of the field passes */
  const double* Estat;  /* damped static field of the charges (+ static dipoles) */
  int itime;
} pim_env;

static double upol_of(or_ctx* c, const double* mu) {
  double u = 0.0;
  for (int ia = 0; ia < c->natm; ++ia)
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b)
        u = u + mu[3 * ia + a] * c->invpoldipia[9 * ia + 3 * a + b] * mu[3 * ia + b];
  return u * 0.5;
}

/* Efield_ind of mu: multipole_ES with charges zeroed, the dd task, undamped,
   direct + reciprocal (moment_from_pola.f90:401-404).  do_rec = 0 with
   alphaES = 0.001 is the kO inner pass (:893-898). */
static void field_ind(pim_env* e, const double* mu, int do_rec, double u_pol, double* E) {
  int task_ind[6] = {0, 0, 1, 0, 0, 0};
  es_out o;
  memset(e->fsink, 0, sizeof(double) * 3 * e->c->natm);
  multipole_ES(e->c, e->rx, e->ry, e->rz, e->sx, e->sy, e->sz, e->L, e->qzero, mu, task_ind, 0, 1, 0, 0,
               0, do_rec, u_pol, E, NULL, e->fsink, &o);
}

/* polint (moment_from_pola.f90:2365-2412) at x = 1.  The reference's
   recurrence takes hp from xa(i+1) where Neville's scheme has xa(i+m), so
   from three points on it is not the interpolating polynomial; it is
   restated as written. */
static double polint1(const int* xa, const double* ya, int n) {
  double c[10], d[10];
  int ns = 1;
  double dif = fabs((double)(1 - xa[0]));
  for (int i = 1; i <= n; ++i) {
    double dift = fabs((double)(1 - xa[i - 1]));
    if (dift < dif) {
      ns = i;
      dif = dift;
    }
    c[i - 1] = ya[i - 1];
    d[i - 1] = ya[i - 1];
  }
  double y = ya[ns - 1], dy;
  ns = ns - 1;
  for (int m = 1; m <= n - 1; ++m) {
    for (int i = 1; i <= n - m; ++i) {
      double ho = (double)(xa[i - 1] - 1);
      double hp = (double)(xa[i] - 1);
      double w = c[i] - d[i - 1];
      double den = ho - hp;
      den = w / den;
      d[i - 1] = hp * den;
      c[i - 1] = ho * den;
    }
    if (2 * ns < n - m) {
      dy = c[ns];
    } else {
      dy = d[ns - 1];
      ns = ns - 1;
    }
    y = y + dy;
  }
  return y;
}

double or_polint(const int* xa, const double* ya, int n) { return polint1(xa, ya, n); }

/* extrapolate_dipole_poly (moment_from_pola.f90:2276-2363) */
static void poly_predict(or_ctx* c, double* mu_ind, int itime) {
  int natm = c->natm, eo = c->p.extrapolate_order;
  size_t n3 = (size_t)natm * 3;
  double* h = c->hist; /* h[k * n3 + i] = dipia_ind_t(k+1, ...) */
  int npts = 0;        /* points of a polint call */
  if (eo == 0) {
    memcpy(mu_ind, h, sizeof(double) * n3);
    return;
  }
  if (eo == 1) {
    if (itime > eo)
      for (size_t i = 0; i < n3; ++i) mu_ind[i] = 2.0 * h[i] - h[n3 + i];
    else
      memcpy(mu_ind, h, sizeof(double) * n3);
    memcpy(h + n3, h, sizeof(double) * n3);
    return;
  }
  if (itime > eo) {
    npts = eo + 1;
  } else {
    if (itime == 1) memcpy(mu_ind, h, sizeof(double) * n3);
    if (itime == 2)
      for (size_t i = 0; i < n3; ++i) mu_ind[i] = 2.0 * h[i] - h[n3 + i];
    if (itime > 2) npts = itime + 1;
  }
  if (npts > 0) {
    int xa[MDFF_ASPC_DEPTH];
    double ya[MDFF_ASPC_DEPTH];
    for (int t = 1; t <= npts; ++t) xa[t - 1] = 1 - t;
    for (size_t i = 0; i < n3; ++i) {
      for (int t = 0; t < npts; ++t) ya[t] = h[t * n3 + i];
      mu_ind[i] = polint1(xa, ya, npts);
    }
  }
  /* dipia_ind_t(ie) = dipia_ind_t(ie-1) for ie = order+1..2; the reference's
     last step (ie = 1) reads index 0, and slot 1 is overwritten by the
     converged dipoles before any read */
  for (int k = eo; k >= 1; --k) memcpy(h + k * n3, h + (k - 1) * n3, sizeof(double) * n3);
}

/* predictor of the kO algorithms (moment_from_pola.f90:1183-1184) */
static void ko_predict(or_ctx* c, double* mu_ind, const double* Efield, int itime) {
  if (c->p.algo_ext_dipole == MDFF_EXT_POLY)
    poly_predict(c, mu_ind, itime);
  else
    aspc(c, mu_ind, Efield, 1, itime);
}

/* induced_moment_inner (moment_from_pola.f90:822-942): relaxation of the
   dipole increment in the field of its near neighbours (direct space only,
   alphaES = 0.001, undamped), weight omegakO, at most 10 passes or until the
   residual falls below a tenth of the residual of f_ext. */
static void induced_moment_inner(pim_env* e, const double* f_ext, double* mu) {
  or_ctx* c = e->c;
  size_t n3 = (size_t)c->natm * 3;
  double om = c->p.omegakO;
  double* zero = calloc(n3, sizeof(double));
  double* mu_prev = malloc(sizeof(double) * n3);
  double* f_tot = malloc(sizeof(double) * n3);
  double* f = malloc(sizeof(double) * n3);
  double rmsd_ref = get_rmsd_mu(c, f_ext, zero);
  memcpy(f_tot, f_ext, sizeof(double) * n3);
  induced_moment(c, f_tot, mu);
  for (size_t i = 0; i < n3; ++i) mu[i] = om * mu[i];
  double rmsd_inner = HUGE_VAL;
  int it = 1;
  double alpha_save = c->p.alphaES;
  while (it <= 10 && rmsd_inner > 0.1 * rmsd_ref) {
    memcpy(mu_prev, mu, sizeof(double) * n3);
    c->p.alphaES = 0.001;
    field_ind(e, mu, 0, 0.0, f);
    c->p.alphaES = alpha_save;
    for (size_t i = 0; i < n3; ++i) f_tot[i] = f_ext[i] + f[i];
    rmsd_inner = get_rmsd_mu(c, f_tot, mu);
    induced_moment(c, f_tot, mu);
    for (size_t i = 0; i < n3; ++i) mu[i] = (1.0 - om) * mu_prev[i] + om * mu[i];
    it++;
  }
  free(zero);
  free(mu_prev);
  free(f_tot);
  free(f);
}

/* f = E - mu / alpha_aa on polarisable components (moment_from_pola.f90:1242-1249) */
static void ko_residual(or_ctx* c, const double* E, const double* mu, double* f) {
  for (int ia = 0; ia < c->natm; ++ia) {
    if (!c->ipolar[ia]) continue;
    for (int a = 0; a < 3; ++a)
      f[3 * ia + a] = E[3 * ia + a] - mu[3 * ia + a] / c->poldipia[9 * ia + 4 * a];
  }
}

#define SCF_CONTINUE(iscf, rmsd)                                                   \
  (((iscf) < c->p.max_scf_pol_iter && (rmsd) > c->p.conv_tol_ind) ||             \
   ((iscf) < c->p.min_scf_pol_iter))

/* moment_from_pola_scf (moment_from_pola.f90:240-485) */
static void scf_plain(pim_env* e, double* mu, double* u_pol, int* n_scf, double* rmsd_out) {
  or_ctx* c = e->c;
  size_t n3 = (size_t)c->natm * 3;
  double* Efield = malloc(sizeof(double) * n3);
  double* Eind = malloc(sizeof(double) * n3);
  memcpy(Efield, e->Estat, sizeof(double) * n3);
  int ismd = (c->p.calc == MDFF_CALC_MD), isopt = (c->p.calc == MDFF_CALC_OPT);
  int iscf = 0;
  double rmsd = HUGE_VAL;
  while (SCF_CONTINUE(iscf, rmsd)) {
    iscf++;
    if (iscf != 1 || (!ismd && !isopt))
      induced_moment(c, Efield, mu);
    else
      aspc(c, mu, Efield, 1, e->itime);
    *u_pol = upol_of(c, mu);
    field_ind(e, mu, 1, *u_pol, Eind);
    for (size_t i = 0; i < n3; ++i) Efield[i] = e->Estat[i] + Eind[i];
    if (iscf == 1 && ismd) aspc(c, mu, Efield, 2, e->itime);
    rmsd = get_rmsd_mu(c, Efield, mu);
  }
  *n_scf = iscf;
  *rmsd_out = rmsd;
  free(Efield);
  free(Eind);
}

/* moment_from_pola_scf_kO_v1 (moment_from_pola.f90:1042-1320) */
static void scf_ko_v1(pim_env* e, double* mu, double* u_pol, int* n_scf, double* rmsd_out) {
  or_ctx* c = e->c;
  size_t n3 = (size_t)c->natm * 3;
  double* Efield = malloc(sizeof(double) * n3);
  double* Eind = malloc(sizeof(double) * n3);
  double* f_ind = malloc(sizeof(double) * n3);
  double* dmu = calloc(n3, sizeof(double));
  memcpy(Efield, e->Estat, sizeof(double) * n3);
  memcpy(f_ind, Efield, sizeof(double) * n3);
  int ismd = (c->p.calc == MDFF_CALC_MD), isopt = (c->p.calc == MDFF_CALC_OPT);
  int aspc_on = c->p.algo_ext_dipole == MDFF_EXT_ASPC;
  int iscf = 0;
  double rmsd = HUGE_VAL;
  while (SCF_CONTINUE(iscf, rmsd)) {
    iscf++;
    if (iscf != 1 || (!ismd && !isopt)) {
      induced_moment_inner(e, f_ind, dmu);
      for (size_t i = 0; i < n3; ++i) mu[i] = mu[i] + dmu[i];
    } else {
      ko_predict(c, mu, Efield, e->itime);
    }
    *u_pol = upol_of(c, mu);
    field_ind(e, mu, 1, *u_pol, Eind);
    for (size_t i = 0; i < n3; ++i) Efield[i] = e->Estat[i] + Eind[i];
    if (iscf == 1 && ismd && aspc_on) aspc(c, mu, Efield, 2, e->itime);
    rmsd = get_rmsd_mu(c, Efield, mu);
    ko_residual(c, Efield, mu, f_ind);
  }
  *n_scf = iscf;
  *rmsd_out = rmsd;
  free(Efield);
  free(Eind);
  free(f_ind);
  free(dmu);
}

/* find_min (moment_from_pola.f90:2415-2455): the point of least |g| on the
   line g0 + a (g1 - g0); the step a times d1.  The 1e-10 guard is a
   single-precision literal in the reference. */
static void find_min(or_ctx* c, const double* g0, const double* g1, const double* d1, double* gmin,
                     double* dmin) {
  size_t n3 = (size_t)c->natm * 3;
  double g0sq = 0.0, g0g1mg0 = 0.0;
  for (int ia = 0; ia < c->natm; ++ia) {
    if (!c->ipolar[ia]) continue;
    for (int k = 0; k < 3; ++k) {
      double g = g0[3 * ia + k], dg = g1[3 * ia + k] - g;
      g0sq = g0sq + g * g;
      g0g1mg0 = g0g1mg0 + g * dg;
    }
  }
  double a = -g0sq / g0g1mg0;
  if (fabs(g0g1mg0) < (double)1e-10f) a = 1.0;
  for (size_t i = 0; i < n3; ++i) {
    gmin[i] = g0[i] + a * (g1[i] - g0[i]);
    dmin[i] = a * d1[i];
  }
}

/* moment_from_pola_scf_kO_v2 (moment_from_pola.f90:1335-1639) */
static void scf_ko_v2(pim_env* e, double* mu, double* u_pol, int* n_scf, double* rmsd_out) {
  or_ctx* c = e->c;
  size_t n3 = (size_t)c->natm * 3;
  double* Efield = malloc(sizeof(double) * n3);
  double* Eind = malloc(sizeof(double) * n3);
  double* f_ind = malloc(sizeof(double) * n3);
  double* f_prev = calloc(n3, sizeof(double));
  double* gmin = calloc(n3, sizeof(double));
  double* mu_prev = calloc(n3, sizeof(double));
  double* dmin = calloc(n3, sizeof(double));
  double* d1 = malloc(sizeof(double) * n3);
  double* zero = calloc(n3, sizeof(double));
  double* dmu = calloc(n3, sizeof(double));
  memcpy(Efield, e->Estat, sizeof(double) * n3);
  memcpy(f_ind, Efield, sizeof(double) * n3);
  int ismd = (c->p.calc == MDFF_CALC_MD), isopt = (c->p.calc == MDFF_CALC_OPT);
  int aspc_on = c->p.algo_ext_dipole == MDFF_EXT_ASPC;
  int iscf = 0;
  double rmsd = HUGE_VAL;
  while (SCF_CONTINUE(iscf, rmsd)) {
    iscf++;
    if (iscf != 1 || (!ismd && !isopt)) {
      induced_moment_inner(e, iscf <= 2 ? f_ind : gmin, dmu);
      for (size_t i = 0; i < n3; ++i) mu[i] = mu[i] + dmu[i];
    } else {
      ko_predict(c, mu, Efield, e->itime);
    }
    *u_pol = upol_of(c, mu);
    field_ind(e, mu, 1, *u_pol, Eind);
    for (size_t i = 0; i < n3; ++i) Efield[i] = e->Estat[i] + Eind[i];
    if (iscf == 1 && ismd && aspc_on) aspc(c, mu, Efield, 2, e->itime);
    ko_residual(c, Efield, mu, f_ind);
    if (iscf != 1) {
      for (size_t i = 0; i < n3; ++i) d1[i] = mu[i] - mu_prev[i];
      find_min(c, f_prev, f_ind, d1, gmin, dmin);
      for (size_t i = 0; i < n3; ++i) mu[i] = mu_prev[i] + dmin[i];
      rmsd = get_rmsd_mu(c, gmin, zero);
    }
    memcpy(mu_prev, mu, sizeof(double) * n3);
    memcpy(f_prev, gmin, sizeof(double) * n3);
  }
  *n_scf = iscf;
  *rmsd_out = rmsd;
  free(Efield);
  free(Eind);
  free(f_ind);
  free(f_prev);
  free(gmin);
  free(mu_prev);
  free(dmin);
  free(d1);
  free(zero);
  free(dmu);
}

/* DGESV semantics for A x = b, n <= KO_HIST: LU with partial pivoting (first
   largest |pivot|); an exactly zero pivot leaves b as given (info > 0, no
   solve). */
static void dgesv_small(int n, double* A /* [n][n] row-major */, double* b) {
  int piv[KO_HIST];
  for (int k = 0; k < n; ++k) {
    int p = k;
    double amax = fabs(A[k * n + k]);
    for (int i = k + 1; i < n; ++i)
      if (fabs(A[i * n + k]) > amax) {
        amax = fabs(A[i * n + k]);
        p = i;
      }
    piv[k] = p;
    if (A[p * n + k] == 0.0) return;
    if (p != k)
      for (int j = 0; j < n; ++j) {
        double t = A[k * n + j];
        A[k * n + j] = A[p * n + j];
        A[p * n + j] = t;
      }
    for (int i = k + 1; i < n; ++i) {
      double l = A[i * n + k] / A[k * n + k];
      A[i * n + k] = l;
      for (int j = k + 1; j < n; ++j) A[i * n + j] -= l * A[k * n + j];
    }
  }
  for (int k = 0; k < n; ++k)
    if (piv[k] != k) {
      double t = b[k];
      b[k] = b[piv[k]];
      b[piv[k]] = t;
    }
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < i; ++j) b[i] -= A[i * n + j] * b[j];
  for (int i = n - 1; i >= 0; --i) {
    for (int j = i + 1; j < n; ++j) b[i] -= A[i * n + j] * b[j];
    b[i] /= A[i * n + i];
  }
}

/* DDOTF (moment_from_pola.f90:2531-2552): dot product over polarisable ions */
static double ddotf(or_ctx* c, const double* v1, const double* v2) {
  double s = 0.0;
  for (int ia = 0; ia < c->natm; ++ia) {
    if (!c->ipolar[ia]) continue;
    for (int k = 0; k < 3; ++k) s = s + v1[3 * ia + k] * v2[3 * ia + k];
  }
  return s;
}

/* moment_from_pola_scf_kO_v4 with scf_kO_v4_1 (moment_from_pola.f90:1987-2273)
   and find_min_ex (:2457-2529): the dipoles are the combination of all
   earlier iterates whose residuals F = mu / alpha - E_ind best match E_stat
   (normal equations). */
static void scf_ko_v4_1(pim_env* e, double* mu, double* u_pol, int* n_scf, double* rmsd_out) {
  or_ctx* c = e->c;
  int natm = c->natm;
  size_t n3 = (size_t)natm * 3;
  double* Efield = malloc(sizeof(double) * n3);
  double* Eind = malloc(sizeof(double) * n3);
  double* F = calloc(n3, sizeof(double));
  double* Fh = calloc(n3 * KO_HIST, sizeof(double));
  double* muh = calloc(n3 * KO_HIST, sizeof(double));
  double* A = malloc(sizeof(double) * KO_HIST * KO_HIST);
  double b[KO_HIST];
  memcpy(Efield, e->Estat, sizeof(double) * n3);
  int ismd = (c->p.calc == MDFF_CALC_MD), isopt = (c->p.calc == MDFF_CALC_OPT);
  int aspc_on = c->p.algo_ext_dipole == MDFF_EXT_ASPC;
  int iscf = 0;
  double rmsd = HUGE_VAL;
  while (SCF_CONTINUE(iscf, rmsd)) {
    iscf++;
    if (iscf != 1 || (!ismd && !isopt)) {
      induced_moment(c, Efield, mu);
    } else {
      if (aspc_on) aspc(c, mu, Efield, 1, e->itime);
      int allzero = 1;
      for (size_t i = 0; i < n3; ++i)
        if (mu[i] != 0.0) allzero = 0;
      if (allzero) induced_moment(c, Efield, mu);
    }
    *u_pol = upol_of(c, mu);
    field_ind(e, mu, 1, *u_pol, Eind);
    for (size_t i = 0; i < n3; ++i) Efield[i] = e->Estat[i] + Eind[i];
    for (int ia = 0; ia < natm; ++ia) {
      if (!c->ipolar[ia]) continue;
      for (int a = 0; a < 3; ++a)
        F[3 * ia + a] = mu[3 * ia + a] / c->poldipia[9 * ia + 4 * a] - Eind[3 * ia + a];
    }
    /* find_min_ex */
    memcpy(Fh + (size_t)(iscf - 1) * n3, F, sizeof(double) * n3);
    memcpy(muh + (size_t)(iscf - 1) * n3, mu, sizeof(double) * n3);
    if (iscf > 1) {
      int m = iscf;
      for (int j = 0; j < m; ++j)
        for (int i = j; i < m; ++i) {
          A[i * m + j] = ddotf(c, Fh + (size_t)i * n3, Fh + (size_t)j * n3);
          A[j * m + i] = A[i * m + j];
        }
      for (int i = 0; i < m; ++i) b[i] = ddotf(c, e->Estat, Fh + (size_t)i * n3);
      dgesv_small(m, A, b);
      for (size_t k = 0; k < n3; ++k) {
        double t = 0.0, u = 0.0;
        for (int i = 0; i < m; ++i) {
          t = t + b[i] * Fh[(size_t)i * n3 + k];
          u = u + b[i] * muh[(size_t)i * n3 + k];
        }
        mu[k] = u;
        F[k] = -e->Estat[k] + t;
      }
    }
    for (int ia = 0; ia < natm; ++ia) {
      if (!c->ipolar[ia]) continue;
      for (int a = 0; a < 3; ++a)
        Efield[3 * ia + a] = -F[3 * ia + a] + mu[3 * ia + a] / c->poldipia[9 * ia + 4 * a];
    }
    if (iscf == 1 && ismd && aspc_on) aspc(c, mu, Efield, 2, e->itime);
    rmsd = get_rmsd_mu(c, Efield, mu);
  }
  *n_scf = iscf;
  *rmsd_out = rmsd;
  free(Efield);
  free(Eind);
  free(F);
  free(Fh);
  free(muh);
  free(A);
}

/* moment_from_WFc (moment_from_pola.f90:632-807): for every ion of a type
   with lwfc >= 0, mu = -2 sum (r_j - r_i) over the Wannier centres j (types
   with lwfc < 0) with |r_ij|^2 < rcut_wfc (the squared distance against
   rcut_wfc itself, :710), minimum image through direct coordinates; an ion
   of a type with lwfc > 0 must find lwfc centres (:731-737). */
static int moment_from_wfc(or_ctx* c, const double* sx, const double* sy, const double* sz, double* mu) {
  int natm = c->natm;
  const double(*A)[3] = c->A;
  for (int ia = 0; ia < natm; ++ia) {
    int it = c->itype[ia];
    if (c->p.lwfc[it] < 0) continue;
    int cnt = 0;
    double m[3] = {0.0, 0.0, 0.0};
    for (int ja = 0; ja < natm; ++ja) {
      if (c->p.lwfc[c->itype[ja]] >= 0) continue;
      double ssx = sx[ja] - sx[ia], ssy = sy[ja] - sy[ia], ssz = sz[ja] - sz[ia];
      ssx = ssx - fnint(ssx);
      ssy = ssy - fnint(ssy);
      ssz = ssz - fnint(ssz);
      double rxij = ssx * A[0][0] + ssy * A[0][1] + ssz * A[0][2];
      double ryij = ssx * A[1][0] + ssy * A[1][1] + ssz * A[1][2];
      double rzij = ssx * A[2][0] + ssy * A[2][1] + ssz * A[2][2];
      double rijsq = rxij * rxij + ryij * ryij + rzij * rzij;
      if (rijsq < c->p.rcut_wfc) {
        cnt++;
        m[0] = m[0] + rxij;
        m[1] = m[1] + ryij;
        m[2] = m[2] + rzij;
      }
    }
    if (c->p.lwfc[it] > 0 && cnt != c->p.lwfc[it]) return MDFF_ERR_BAD_ARGS;
    for (int a = 0; a < 3; ++a) mu[3 * ia + a] = -2.0 * m[a];
  }
  return MDFF_OK;
}

int or_engforce(or_ctx* c, const double* rx, const double* ry, const double* rz, int itime,
                mdff_result* out, or_extra* ex) {
  int natm = c->natm;
  if (c->p.extrapolate_order < 0 || c->p.extrapolate_order > 4) return MDFF_ERR_BAD_ARGS;
  {
    int al = c->p.algo_moment_from_pola;
    if (al < MDFF_ALGO_SCF || al > MDFF_ALGO_KO_V4_2) return MDFF_ERR_BAD_ARGS;
    if (al == MDFF_ALGO_KO_V3 || al == MDFF_ALGO_KO_V4_2) return MDFF_ERR_UNSUPPORTED;
    if (al == MDFF_ALGO_KO_V4_1 && c->p.max_scf_pol_iter > KO_HIST) return MDFF_ERR_BAD_ARGS;
  }
  double* sx = malloc(sizeof(double) * natm);
  double* sy = malloc(sizeof(double) * natm);
  double* sz = malloc(sizeof(double) * natm);
  or_kardir(c, rx, ry, rz, sx, sy, sz);
  double* f = calloc((size_t)natm * 3, sizeof(double));
  double* fx = calloc(natm, sizeof(double));
  double* fy = calloc(natm, sizeof(double));
  double* fz = calloc(natm, sizeof(double));
  int status = MDFF_OK;
  memset(out->tau, 0, sizeof(out->tau));
  memset(out->tau_nonb, 0, sizeof(out->tau_nonb));
  memset(out->tau_coul, 0, sizeof(out->tau_coul));
  out->u_lj = out->vir_lj = out->u_bmhft = out->vir_bmhft = 0.0;
  out->u_coul = out->u_pol = out->pvirial_coul = 0.0;
  c->n_kardir = 0;
  if (ex) {
    ex->n_scf = 0;
    ex->rmsd = 0.0;
  }
  /* short range (engforce_driver.f90:116-135) on the vdw half list */
  if (c->p.lnmlj || c->p.lbmhft || c->p.lbmhftd) {
    csr_t Lv;
    build_half(c, sx, sy, sz, c->p.cutshortrange, &Lv);
    if (c->p.lnmlj) {
      or_nmlj(c, sx, sy, sz, &Lv, fx, fy, fz, &out->u_lj, &out->vir_lj, out->tau_nonb);
      c->n_kardir++; /* non_bonded.f90:716,823 */
      for (int a = 0; a < 9; ++a) (&out->tau[0][0])[a] += (&out->tau_nonb[0][0])[a];
    }
    if (c->p.lbmhft || c->p.lbmhftd) {
      or_bmhftd(c, sx, sy, sz, &Lv, fx, fy, fz, &out->u_bmhft, &out->vir_bmhft, out->tau_nonb);
      c->n_kardir++; /* non_bonded.f90:1113,1221 */
      for (int a = 0; a < 9; ++a) (&out->tau[0][0])[a] += (&out->tau_nonb[0][0])[a];
    }
    free_csr(&Lv);
  }
  for (int ia = 0; ia < natm; ++ia) {
    f[3 * ia] = fx[ia];
    f[3 * ia + 1] = fy[ia];
    f[3 * ia + 2] = fz[ia];
  }
  if (c->p.lcoulomb) {
    csr_t Lc;
    build_half(c, sx, sy, sz, c->p.cutlongrange, &Lc);
    size_t n3 = (size_t)natm * 3;
    double* mu = calloc(n3, sizeof(double));
    double* ef = calloc(n3, sizeof(double));
    double* dipia_ind = calloc(n3, sizeof(double));
    double u_pol = 0.0;
    double* zero_f = calloc(n3, sizeof(double));
    /* get_dipole_moments (moment_from_pola.f90:84-224) -> moment_from_pola_scf
       (:240-485) */
    if (c->lpolar_any) {
      double* Estat = calloc(n3, sizeof(double));
      double* qzero = calloc(natm, sizeof(double));
      int ldip = 0;
      for (int it = 0; it < MDFF_NTYPEMAX; ++it)
        for (int a = 0; a < 3; ++a)
          if (c->p.dip[it][a] != 0.0) ldip = 1;
      int task_static[6] = {1, 0, 0, 0, 0, 0};
      if (ldip)
        for (int i = 0; i < 6; ++i) task_static[i] = 1;
      es_out o;
      multipole_ES(c, rx, ry, rz, sx, sy, sz, &Lc, c->qia, c->dipia, task_static, 1, 1, 0, 0, 0,
                   1, 0.0, Estat, NULL, zero_f, &o);
      pim_env env = {c, rx, ry, rz, sx, sy, sz, &Lc, qzero, zero_f, Estat, itime};
      int iscf = 0;
      double rmsd = HUGE_VAL;
      switch (c->p.algo_moment_from_pola) {
        case MDFF_ALGO_KO_V1: scf_ko_v1(&env, dipia_ind, &u_pol, &iscf, &rmsd); break;
        case MDFF_ALGO_KO_V2: scf_ko_v2(&env, dipia_ind, &u_pol, &iscf, &rmsd); break;
        case MDFF_ALGO_KO_V4_1: scf_ko_v4_1(&env, dipia_ind, &u_pol, &iscf, &rmsd); break;
        default: scf_plain(&env, dipia_ind, &u_pol, &iscf, &rmsd); break;
      }
      /* store induced dipole at t (moment_from_pola.f90:465) */
      memcpy(c->hist, dipia_ind, sizeof(double) * n3);
      if (ex) {
        ex->n_scf = iscf;
        ex->rmsd = rmsd;
      }
      free(Estat);
      free(qzero);
    }
    for (size_t i = 0; i < n3; ++i) mu[i] = c->dipia[i] + dipia_ind[i];
    /* Wannier centres (moment_from_pola.f90:130-147, moment_from_WFc :632-807) */
    if (status == MDFF_OK) {
      int lwannier = 0;
      for (int it = 0; it < c->p.ntype; ++it)
        if (c->p.lwfc[it] > 0) lwannier = 1;
      if (lwannier) {
        double* mw = calloc(n3, sizeof(double));
        status = moment_from_wfc(c, sx, sy, sz, mw);
        c->n_kardir++; /* moment_from_pola.f90:685,803 */
        if (status == MDFF_OK && c->p.ldip_wfc)
          for (size_t i = 0; i < n3; ++i) mu[i] = mu[i] + mw[i];
        free(mw);
      }
    }
    /* polarisation catastrophe (moment_from_pola.f90:176-216) */
    for (int ia = 0; ia < natm && status == MDFF_OK; ++ia)
      for (int a = 0; a < 3; ++a)
        if (mu[3 * ia + a] > 10.0) status = MDFF_ERR_CATASTROPHE;
    if (status == MDFF_OK) {
      es_out o;
      int do_efg = ex ? ex->do_efg : 0;
      multipole_ES(c, rx, ry, rz, sx, sy, sz, &Lc, c->qia, mu, c->task, 1, 1, do_efg, 1, 1, 1, u_pol,
                   ef, (ex && ex->efg) ? ex->efg : NULL, f, &o);
      out->u_coul = o.u_coul;
      out->u_pol = u_pol;
      out->pvirial_coul = o.pvirial_coul;
      memcpy(out->tau_coul, o.tau_coul, sizeof(o.tau_coul));
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) out->tau[a][b] += 2.0 * o.tau_coul[a][b];
      if (ex) {
        ex->u_dir = o.u_dir;
        ex->u_rec = o.u_rec;
        ex->u_self = o.u_self;
        ex->u_surf = o.u_surf;
      }
      if (out->mu) memcpy(out->mu, mu, sizeof(double) * n3);
      if (out->ef) memcpy(out->ef, ef, sizeof(double) * n3);
    }
    free(mu);
    free(ef);
    free(dipia_ind);
    free(zero_f);
    free_csr(&Lc);
  }
  for (int ia = 0; ia < natm; ++ia) {
    out->fx[ia] = f[3 * ia];
    out->fy[ia] = f[3 * ia + 1];
    out->fz[ia] = f[3 * ia + 2];
  }
  free(sx);
  free(sy);
  free(sz);
  free(f);
  free(fx);
  free(fy);
  free(fz);
  if (ex) ex->n_kardir = c->n_kardir;
  return status;
}
