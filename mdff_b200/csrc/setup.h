// setup.h -- host-side set-up shared by the single-configuration engine and
// the batched engine: the reference's *_init routines that turn the control
// keywords and the cell into the per-ion and per-pair tables the kernels read.
//
//  * symmetrisation of the pair / triple tables (non_bonded.f90:287-301,
//    pim.f90:189-199)
//  * lattice (lattice.f90:60-130): B = reciprocal / omega, face widths, norms
//  * tasks (coulomb.f90:204-220, pim.f90:160-184)
//  * ewald_param (coulomb.f90:363-410): real-space cutoff clamp, lautoES
//  * typeinfo_init (read_pos.f90:160-237): per-ion charge, dipole, alpha, 1/alpha
//  * initialize_param_non_bonded (non_bonded.f90:455-644): pair tables
//  * kpoint_sum_init (kspace.f90:143-207): the half-space k mesh as rows
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "../../include/mdff_gpu.h"
#include "common.cuh"
#include "realspace.cuh"

namespace mdff {

constexpr double kCoulUnit = 14.3996441494161;      // constants.f90:91
constexpr double kPressUnit = 0.00624150964712042;  // constants.f90:88
constexpr int kNT = MDFF_NTYPEMAX;

// symmetric_pot: X(:,it) = X(it,:) for it = 1..ntype (non_bonded.f90:287-301)
inline void sym2(double X[kNT][kNT], int ntype) {
  for (int it = 0; it < ntype; ++it) {
    double row[kNT];
    for (int k = 0; k < kNT; ++k) row[k] = X[it][k];
    for (int k = 0; k < kNT; ++k) X[k][it] = row[k];
  }
}
// pim.f90:189-199: X(it2,:,it) = X(it2,it,:)
template <typename T>
inline void sym3(T X[kNT][kNT][kNT], int ntype) {
  for (int it = 0; it < ntype; ++it)
    for (int it2 = 0; it2 < ntype; ++it2) {
      T row[kNT];
      for (int k = 0; k < kNT; ++k) row[k] = X[it2][it][k];
      for (int k = 0; k < kNT; ++k) X[it2][k][it] = row[k];
    }
}

// 3x3 inverse; diagonal tensors are inverted entry by entry with zero
// entries left zero (a site polarisable along one axis only).
inline bool inv3(const double* m, double* out) {
  bool diag = m[1] == 0 && m[2] == 0 && m[3] == 0 && m[5] == 0 && m[6] == 0 && m[7] == 0;
  if (diag) {
    for (int i = 0; i < 9; ++i) out[i] = 0.0;
    for (int i = 0; i < 3; ++i) out[4 * i] = m[4 * i] != 0.0 ? 1.0 / m[4 * i] : 0.0;
    return true;
  }
  double det = m[0] * (m[4] * m[8] - m[5] * m[7]) - m[1] * (m[3] * m[8] - m[5] * m[6]) +
               m[2] * (m[3] * m[7] - m[4] * m[6]);
  if (det == 0.0) return false;
  out[0] = (m[4] * m[8] - m[5] * m[7]) / det;
  out[1] = (m[2] * m[7] - m[1] * m[8]) / det;
  out[2] = (m[1] * m[5] - m[2] * m[4]) / det;
  out[3] = (m[5] * m[6] - m[3] * m[8]) / det;
  out[4] = (m[0] * m[8] - m[2] * m[6]) / det;
  out[5] = (m[2] * m[3] - m[0] * m[5]) / det;
  out[6] = (m[3] * m[7] - m[4] * m[6]) / det;
  out[7] = (m[1] * m[6] - m[0] * m[7]) / det;
  out[8] = (m[0] * m[4] - m[1] * m[3]) / det;
  return true;
}

struct Lattice {
  double A[9], B[9];  // row-major [a][b]; B = reciprocal vectors / omega
  double omega, W[3], ANORM[3];
};

// lattice (lattice.f90:60-130)
inline void lattice_of(const double* Ain, Lattice& L) {
  double A[3][3], B[3][3];
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) A[a][b] = Ain[3 * a + b];
  const int cyc[3][2] = {{1, 2}, {2, 0}, {0, 1}};
  for (int col = 0; col < 3; ++col) {
    int u = cyc[col][0], v = cyc[col][1];
    B[0][col] = A[1][u] * A[2][v] - A[2][u] * A[1][v];
    B[1][col] = A[2][u] * A[0][v] - A[0][u] * A[2][v];
    B[2][col] = A[0][u] * A[1][v] - A[1][u] * A[0][v];
  }
  double omega = B[0][0] * A[0][0] + B[1][0] * A[1][0] + B[2][0] * A[2][0];
  for (int c = 0; c < 3; ++c)
    L.W[c] = omega / std::sqrt(B[0][c] * B[0][c] + B[1][c] * B[1][c] + B[2][c] * B[2][c]);
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) B[i][j] = B[i][j] / omega;
  for (int i = 0; i < 3; ++i)
    L.ANORM[i] = std::sqrt(A[0][i] * A[0][i] + A[1][i] * A[1][i] + A[2][i] * A[2][i]);
  L.omega = omega;
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) {
      L.A[3 * a + b] = A[a][b];
      L.B[3 * a + b] = B[a][b];
    }
}

struct Setup {
  mdff_params p;  // after symmetrisation, cutoff clamp and lautoES
  Lattice L;
  double coul_unit = 0, press_unit = 0;
  int lsr = 0, task_qq = 0, task_qd = 0, task_dd = 0, lpolar = 0, ldip_static = 0, npol = 0;
  std::vector<int> itype, ipol;
  std::vector<double> q, pol, inv;  // pol / inv: [natm][9]
  std::vector<double4> dip;
  std::vector<NBPair> nb;  // [ntype][ntype]
  std::vector<ESPair> es;  // [ta][tb]
};

// Everything of the reference's set-up that needs no device.  Returns
// MDFF_OK, or MDFF_ERR_BAD_ARGS / MDFF_ERR_UNSUPPORTED with *err set.
inline int setup_system(const mdff_params* pin, const double* cellA, Setup& S, const char** err) {
  S.p = *pin;
  mdff_params& p = S.p;
  if (p.natm <= 0 || p.ntype <= 0 || p.ntype > kNT) {
    *err = "natm/ntype out of range";
    return MDFF_ERR_BAD_ARGS;
  }
  long tot = 0;
  for (int it = 0; it < p.ntype; ++it) tot += p.natmi[it];
  if (tot != p.natm) {
    *err = "sum(natmi) != natm";
    return MDFF_ERR_BAD_ARGS;
  }
  if (p.thole_type < MDFF_THOLE_NONE || p.thole_type > MDFF_THOLE_GAUSS) {
    *err = "thole_type must be one of MDFF_THOLE_* (coulomb.f90:72)";
    return MDFF_ERR_BAD_ARGS;
  }
  if (p.thole_type != MDFF_THOLE_NONE)
    for (int it = 0; it < p.ntype; ++it)
      for (int jt = 0; jt < p.ntype; ++jt)
        if (p.ldip_polar[it] && p.ldip_polar[jt] &&
            !(p.thole_param[it][jt] > 0.0 && p.poldip[it][0][0] > 0.0 && p.poldip[jt][0][0] > 0.0)) {
          *err = "Thole functions need thole_param > 0 and alpha_xx > 0 for polarisable types";
          return MDFF_ERR_BAD_ARGS;
        }
  if (p.extrapolate_order < 0 || p.extrapolate_order > 4) {
    *err = "extrapolate_order must be 0..4 (moment_from_pola.f90:524-527)";
    return MDFF_ERR_BAD_ARGS;
  }
  if (p.algo_moment_from_pola < MDFF_ALGO_SCF || p.algo_moment_from_pola > MDFF_ALGO_KO_V4_2 ||
      (p.algo_ext_dipole != MDFF_EXT_ASPC && p.algo_ext_dipole != MDFF_EXT_POLY)) {
    *err = "algo_moment_from_pola / algo_ext_dipole out of range (pim.f90:85-91)";
    return MDFF_ERR_BAD_ARGS;
  }
  if (p.algo_moment_from_pola == MDFF_ALGO_KO_V3 || p.algo_moment_from_pola == MDFF_ALGO_KO_V4_2) {
    *err = "scf_kO_v3 / scf_kO_v4_2 are not built: the reference's kO_v3 never forms a dipole "
           "increment and kO_v4_2 reads mu_h(:,:,0) (moment_from_pola.f90:1835,2186)";
    return MDFF_ERR_UNSUPPORTED;
  }
  if (p.algo_moment_from_pola != MDFF_ALGO_SCF) {
    if (p.solver != MDFF_SOLVER_SCF) {
      *err = "the kO dipole algorithms run with solver = MDFF_SOLVER_SCF";
      return MDFF_ERR_BAD_ARGS;
    }
    // f_ind = E - mu / alpha_aa on every polarisable component
    // (moment_from_pola.f90:1247, 1548, 2172)
    for (int it = 0; it < p.ntype; ++it)
      if (p.ldip_polar[it] && !(p.poldip[it][0][0] > 0.0 && p.poldip[it][1][1] > 0.0 && p.poldip[it][2][2] > 0.0)) {
        *err = "the kO dipole algorithms need alpha_xx, alpha_yy, alpha_zz > 0 on polarisable types";
        return MDFF_ERR_BAD_ARGS;
      }
    // F_h(3, natm, 100), mu_h(3, natm, 100) (moment_from_pola.f90:2050)
    if (p.algo_moment_from_pola == MDFF_ALGO_KO_V4_1 && p.max_scf_pol_iter > 100) {
      *err = "scf_kO_v4_1 keeps at most 100 iterates: max_scf_pol_iter <= 100";
      return MDFF_ERR_BAD_ARGS;
    }
  }
  // Wannier-centre types after all other types: the reference's list of
  // centres per ion (moment_from_pola.f90:718-722) assumes it
  for (int it = 1; it < p.ntype; ++it)
    if (p.lwfc[it - 1] < 0 && p.lwfc[it] >= 0) {
      *err = "Wannier-centre types (lwfc < 0) must come after all other types";
      return MDFF_ERR_BAD_ARGS;
    }
  int ntype = p.ntype, n = p.natm;
  if (p.symmetric_pot_nb) {
    sym2(p.epslj, ntype); sym2(p.sigmalj, ntype); sym2(p.plj, ntype); sym2(p.qlj, ntype);
    sym2(p.Abmhftd, ntype); sym2(p.Bbmhftd, ntype); sym2(p.Cbmhftd, ntype);
    sym2(p.Dbmhftd, ntype); sym2(p.BDbmhftd, ntype); sym2(p.wall24, ntype);
  }
  if (p.symmetric_pot_pim) {
    sym3(p.ldip_damping, ntype); sym3(p.pol_damp_b, ntype);
    sym3(p.pol_damp_c, ntype); sym3(p.pol_damp_k, ntype);
  }
  for (int a = 0; a < kNT; ++a)
    for (int b = 0; b < kNT; ++b)
      for (int c = 0; c < kNT; ++c)
        if (p.pol_damp_k[a][b][c] < 0 || p.pol_damp_k[a][b][c] > MDFF_TT_MAX) {
          *err = "pol_damp_k beyond the Tang-Toennies table (pim.f90:201-204)";
          return MDFF_ERR_BAD_ARGS;
        }
  S.coul_unit = p.lreduced ? 1.0 : kCoulUnit;
  S.press_unit = p.lreduced ? 1.0 : kPressUnit;
  S.lsr = (p.lbmhft || p.lbmhftd || p.lnmlj) ? 1 : 0;
  int lqch = 0, ldip = 0, lpol = 0;
  for (int it = 0; it < kNT; ++it) {
    if (p.qch[it] != 0.0) lqch = 1;
    for (int a = 0; a < 3; ++a)
      if (p.dip[it][a] != 0.0) ldip = 1;
  }
  for (int it = 0; it < ntype; ++it)
    if (p.ldip_polar[it]) lpol = 1;
  S.task_qq = lqch;
  S.task_qd = lqch && (ldip || lpol);
  S.task_dd = (ldip || lpol);
  S.lpolar = lpol && p.lcoulomb;
  S.ldip_static = ldip;
  lattice_of(cellA, S.L);
  if (p.lcoulomb) {
    double rcut = 0.5 * std::min(S.L.W[0], std::min(S.L.W[1], S.L.W[2]));
    p.cutlongrange = std::min(p.cutlongrange, rcut);
    double cut = p.cutlongrange;
    double eps = std::min(std::fabs(p.epsw), 0.5);
    double tol = std::sqrt(std::fabs(std::log(eps * cut)));
    double alpha = std::sqrt(std::fabs(std::log(eps * cut * tol))) / cut;
    double tol1 = std::sqrt(-std::log(eps * cut * (2.0 * tol * alpha) * (2.0 * tol * alpha)));
    if (p.lautoES) {
      p.alphaES = alpha;
      for (int i = 0; i < 3; ++i)
        p.kES[i] = (int)std::round(0.25 + S.L.ANORM[i] * alpha * tol1 / kPi);
    }
    if (p.cutlongrange <= 0.0 || p.alphaES <= 0.0) {
      *err = "cutlongrange and alphaES must be positive";
      return MDFF_ERR_BAD_ARGS;
    }
    for (int i = 0; i < 3; ++i)
      if (p.kES[i] < 0) {
        *err = "kES must be >= 0";
        return MDFF_ERR_BAD_ARGS;
      }
  }
  // per-ion tables
  S.itype.assign(n, 0);
  S.ipol.assign(n, 0);
  S.q.assign(n, 0.0);
  S.pol.assign(9 * (size_t)n, 0.0);
  S.inv.assign(9 * (size_t)n, 0.0);
  S.dip.assign(n, make_double4(0, 0, 0, 0));
  int ia = 0;
  S.npol = 0;
  for (int it = 0; it < ntype; ++it) {
    double iv[9] = {0};
    if (p.ldip_polar[it] && !inv3(&p.poldip[it][0][0], iv)) {
      *err = "singular polarisability tensor";
      return MDFF_ERR_BAD_ARGS;
    }
    for (int k = 0; k < p.natmi[it]; ++k, ++ia) {
      S.itype[ia] = it;
      S.ipol[ia] = p.ldip_polar[it] ? 1 : 0;
      S.npol += S.ipol[ia];
      S.q[ia] = p.qch[it];
      S.dip[ia] = make_double4(p.dip[it][0], p.dip[it][1], p.dip[it][2], 0.0);
      for (int a = 0; a < 9; ++a) S.pol[9 * (size_t)ia + a] = (&p.poldip[it][0][0])[a];
      if (p.ldip_polar[it])
        for (int a = 0; a < 9; ++a) S.inv[9 * (size_t)ia + a] = iv[a];
    }
  }
  // pair tables
  S.nb.assign(ntype * ntype, NBPair{});
  S.es.assign(ntype * ntype, ESPair{});
  double two16 = std::pow(2.0, 1.0 / 6.0);
  for (int it = 0; it < ntype; ++it)
    for (int jt = 0; jt < ntype; ++jt) {
      NBPair& P = S.nb[it * ntype + jt];
      P.A = p.Abmhftd[it][jt];
      P.B = p.Bbmhftd[it][jt];
      P.C = p.Cbmhftd[it][jt];
      P.D = p.Dbmhftd[it][jt];
      P.BD = p.BDbmhftd[it][jt];
      P.wall = p.wall24[it][jt];
      P.rcutsq = p.cutshortrange * p.cutshortrange;
      double pp = p.plj[it][jt], qq = p.qlj[it][jt];
      P.plj = pp;
      P.qlj = qq;
      P.epsp = p.epslj[it][jt] / (qq - pp);
      P.sigsq = two16 * two16 * p.sigmalj[it][jt] * p.sigmalj[it][jt];
      double sr = std::sqrt(P.sigsq / P.rcutsq);
      double srp = std::pow(sr, pp), srq = std::pow(sr, qq);
      P.uc = P.epsp * (pp * srq - qq * srp);
      P.uc1 = P.epsp * pp * qq / (2.0 * P.rcutsq) * (srq - srp);
      P.uc2 = 0.5 * P.epsp * ((2.0 * pp + pp * qq) * srq - (2.0 * qq + pp * qq) * srp);
      P.fc = pp * qq * P.epsp / P.sigsq;
      ESPair& E = S.es[it * ntype + jt];  // it = ta ("ia"), jt = tb ("ja")
      E.ldamp = (p.ldip_damping[it][it][jt] || p.ldip_damping[jt][it][jt]) ? 1 : 0;
      E.ka = p.pol_damp_k[it][it][jt];
      E.ba = p.pol_damp_b[it][it][jt];
      E.ca = p.pol_damp_c[it][it][jt];
      E.kb = p.pol_damp_k[jt][it][jt];
      E.bb = p.pol_damp_b[jt][it][jt];
      E.cb = p.pol_damp_c[jt][it][jt];
      // Thole functions of a pair of polarisable types (ewald_dir.f90:308-311)
      E.thole = (p.thole_type != MDFF_THOLE_NONE && p.ldip_polar[it] && p.ldip_polar[jt]) ? p.thole_type : 0;
      E.th_a = p.thole_param[it][jt];
      E.th_A = std::pow(p.poldip[it][0][0] * p.poldip[jt][0][0], 1.0 / 6.0);
    }
  return MDFF_OK;
}

// The half-space k mesh (kspace.f90:143-207) as rows (nx, ny, nz_lo, koff)
// of consecutive nz; A_k = e^{-k^2/4 alpha^2}/k^2 and (k, kcoe) per k.  The
// reference's |k|^2 order only changes the summation order.
struct KMesh {
  std::vector<int4> rows;
  std::vector<double> Ak;
  std::vector<double4> kv;
  int nk = 0;
};

inline void kmesh_of(const int kES[3], const double* B, double alphaES, KMesh& M) {
  int kx = kES[0], ky = kES[1], kz = kES[2];
  M.rows.clear();
  int koff = 0;
  for (int nx = 0; nx <= kx; ++nx) {
    int nymin = (nx == 0) ? 0 : -ky;
    for (int ny = nymin; ny <= ky; ++ny) {
      int nzlo = (nx == 0 && ny == 0) ? 1 : -kz;
      if (nzlo > kz) continue;
      M.rows.push_back(make_int4(nx, ny, nzlo, koff));
      koff += kz - nzlo + 1;
    }
  }
  M.nk = koff;
  M.Ak.assign(std::max(koff, 1), 0.0);
  M.kv.assign(std::max(koff, 1), make_double4(0, 0, 0, 0));
  double alpha2 = alphaES * alphaES;
  for (auto& r : M.rows)
    for (int nz = r.z; nz <= kz; ++nz) {
      int k = r.w + nz - r.z;
      double X = r.x, Y = r.y, Z = nz;
      double kxx = kTwoPi * (X * B[0] + Y * B[1] + Z * B[2]);
      double kyy = kTwoPi * (X * B[3] + Y * B[4] + Z * B[5]);
      double kzz = kTwoPi * (X * B[6] + Y * B[7] + Z * B[8]);
      double kk = kxx * kxx + kyy * kyy + kzz * kzz;
      M.Ak[k] = std::exp(-kk * 0.25 / alpha2) / kk;
      M.kv[k] = make_double4(kxx, kyy, kzz, 2.0 * (1.0 / kk + 1.0 / alpha2 / 4.0));
    }
}

// Scalar slots of one evaluation -> the reference's thermodynamic outputs:
// slots 0-15 short range (k_shortrange), 16-22 real-space energy and stress,
// 23-29 reciprocal, 30-37 moments [sum q r, sum mu, sum q^2, sum mu^2],
// 38 sum mu alpha^-1 mu.  Units and factors of ewald.f90:206-245,
// non_bonded.f90:1205 and engforce_driver.f90:164-177 (tau = tau_nonb + 2 tau_coul).
inline void scalars_to_result(const double* sc, const mdff_params& p, int lsr, int lpolar,
                              double omega, double coul_unit, double press_unit, mdff_result* out) {
  const int S_SR = 0, S_DIR = 16, S_REC = 23, S_MOM = 30, S_UPOL = 38;
  double inv_om = 1.0 / omega;
  out->u_lj = out->vir_lj = out->u_bmhft = out->vir_bmhft = 0.0;
  out->u_coul = out->u_pol = out->pvirial_coul = 0.0;
  double tn[3][3] = {{0}}, tc[3][3] = {{0}}, t[3][3] = {{0}};
  auto put6 = [](double m[3][3], const double* v, double f) {
    m[0][0] = v[0] * f;
    m[1][1] = v[1] * f;
    m[2][2] = v[2] * f;
    m[0][1] = m[1][0] = v[3] * f;
    m[0][2] = m[2][0] = v[4] * f;
    m[1][2] = m[2][1] = v[5] * f;
  };
  if (lsr) {
    double f = inv_om / press_unit * 0.5;
    if (p.lnmlj) {
      out->u_lj = sc[S_SR + 2];
      out->vir_lj = sc[S_SR + 3] / 3.0;
      put6(tn, sc + S_SR + 10, f);
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) t[a][b] += tn[a][b];
    }
    if (p.lbmhft || p.lbmhftd) {
      out->u_bmhft = sc[S_SR + 0];
      out->vir_bmhft = sc[S_SR + 1] / 3.0;
      put6(tn, sc + S_SR + 4, f);
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) t[a][b] += tn[a][b];
    }
  }
  if (p.lcoulomb) {
    double cu = coul_unit;
    double a = p.alphaES;
    double selfa = a / std::sqrt(kPi);
    double selfa2 = 2.0 * selfa * a * a / 3.0;
    const double* m = sc + S_MOM;
    double u_self = -selfa * m[6] - selfa2 * m[7];
    double tpi_3V = kTwoPi / omega / 3.0;
    double u_surf = (m[0] * m[0] + m[1] * m[1] + m[2] * m[2]) +
                    2.0 * (m[0] * m[3] + m[1] * m[4] + m[2] * m[5]) +
                    (m[3] * m[3] + m[4] * m[4] + m[5] * m[5]);
    u_surf *= tpi_3V;
    double u_pol = lpolar ? sc[S_UPOL] * 0.5 : 0.0;
    double u_dir = sc[S_DIR], u_rec = sc[S_REC];
    out->u_pol = u_pol;
    out->u_coul = (u_dir + u_rec + (p.lsurf ? u_surf : 0.0) + u_self + u_pol) * cu;
    double td[3][3], tr[3][3];
    put6(td, sc + S_DIR + 1, inv_om * 0.5);
    put6(tr, sc + S_REC + 1, 1.0);
    for (int x = 0; x < 3; ++x)
      for (int y = 0; y < 3; ++y) tc[x][y] = (td[x][y] + tr[x][y]) * cu / press_unit;
    out->pvirial_coul = 1.0 / 3.0 * (tc[0][0] + tc[1][1] + tc[2][2]) * press_unit;
    for (int x = 0; x < 3; ++x)
      for (int y = 0; y < 3; ++y) t[x][y] += 2.0 * tc[x][y];
  }
  memcpy(out->tau_nonb, tn, sizeof(tn));
  memcpy(out->tau_coul, tc, sizeof(tc));
  memcpy(out->tau, t, sizeof(t));
}

}  // namespace mdff
