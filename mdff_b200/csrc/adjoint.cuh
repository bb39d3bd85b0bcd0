// adjoint.cuh -- gradients of a batched evaluation with respect to
// force-field parameters (the differentiable fitting path).  No counterpart
// in the reference, which has no derivatives with respect to its potential
// parameters.
//
// For one configuration let J = g_U U + u_F . F + u_mu . mu (the upstream
// gradients of the total energy, the forces and the induced dipoles).  The
// dipoles solve R(mu, theta) = alpha^-1 mu - E(mu, theta) = 0 with H = dR/dmu
// = alpha^-1 - T symmetric, so
//     dJ/dtheta = dJ/dtheta|_mu - lambda . dR/dtheta,   H lambda = dJ/dmu,
// one adjoint solve with the forward's own PCG operator.  Every term
// differentiates the expressions the forward evaluates (es_force_ipair, the
// short-range pair, the reciprocal sums), not an idealised energy, so the
// gradient is that of the computed forces to the solver tolerance.
//
//   dJ/dmu_j = g_U cu R_j + d(u_F . F)/dmu_j + u_mu_j, with
//     real space  -cu d(Du . f_ab)/dm   per pair (Du = u_a - u_b)
//     reciprocal  cu (8 pi/V) sum_k A_k k [ (k.u_j) Re(rho P_j*) - Re(sigma P_j*) ],
//                 sigma(k) = sum_i (k.u_i)(q_i + i k.mu_i) P_i, P_i = e^{i k.r_i}
//   parameters: Buckingham A, rho, C per type pair (short-range forces and
//   energy); isotropic polarisability per type (u_pol and alpha^-1 in R);
//   Tang-Toennies b, c of the charge field on a dipole type (damped qd
//   forces / energy and the damped static field); one charge scale s on all
//   charges (qq terms scale with s^2, qd terms and the charge field with s).
#pragma once
#include "batch.cuh"

namespace mdff {

enum { FIT_A = 0, FIT_RHO = 1, FIT_C = 2, FIT_POL = 3, FIT_TTB = 4, FIT_TTC = 5, FIT_QSCALE = 6 };
constexpr int kFitMax = 16;

struct FitParam {
  int kind, t1, t2, pad;
};

struct AdjArgs {
  const double* gE;    // [nconf] dJ/dU (U = u_lj + u_bmhft + u_coul, eV)
  const double* gF;    // [3][ntot] dJ/dF
  const double* gmu;   // [ntot][3] dJ/dmu or null
  double4* w;          // [ntot] u_F as 4-vectors
  double4* rhs;        // [ntot]
  double4* lam;        // [ntot]
  double2 *rq, *rm, *sq, *sm, *rl;  // [sum nk] structure-factor channels
  double* grad;        // [nconf][kFitMax]
  double* info;        // [nconf][4]: adjoint iterations, rmsd, tolerance
  double qscale;       // current charge scale (s in the s-derivatives)
  double tol_rel;      // adjoint solve tolerance relative to rms(rhs)
  int nparam;
  FitParam prm[kFitMax];
};

// d f / d b and d f / d c of tt_damp (f = 1 - c e^{-x} sum_k x^k/k!, fd = c b
// e^{-x} x^n/n!, x = b r):
//   df/dc = (f - 1)/c ... evaluated without dividing by c:  -e^{-x} S(x)
//   dfd/dc = b e^{-x} x^n/n!
//   df/db = r c e^{-x} x^n/n! = (r/b) fd
//   dfd/db = c e^{-x} x^n/n! (1 + n - x)
__device__ __forceinline__ void tt_damp_grad(double b, double c, double r, int n, double& dfdb,
                                             double& dfddb, double& dfdc, double& dfddc) {
  double f1, fd1;
  tt_damp<double>(b, 1.0, r, n, f1, fd1);  // c = 1: f1 = 1 - e^{-x}S, fd1 = b e^{-x} x^n/n!
  double x = b * r;
  double en = (b != 0.0) ? fd1 / b : 0.0;  // e^{-x} x^n / n!
  if (b == 0.0) {
    // x = 0: e^{-x} x^n/n! = 1 for n = 0, else 0
    en = (n == 0) ? 1.0 : 0.0;
  }
  dfdc = f1 - 1.0;
  dfddc = fd1;
  // order 0 keeps the reference's f = 1 - c (1 + x) e^{-x} (tt_damp.f90:85-93)
  dfdb = (n == 0) ? c * r * x * en : c * r * en;
  dfddb = c * en * (1.0 + (double)n - x);
}

// gradient of one canonical real-space pair (a = "ia", r = r_a - r_b) from
// the visit of ion `own_a ? a : b`: accumulates this ion's share into g[],
// and returns d(u_F . F)/d m_own in dm.
struct PairAdj {
  const FitParam* prm;
  int nparam;
  double qscale, gU, cu;
};

__device__ __forceinline__ void es_pair_adjoint(const PairAdj& J, const ESPair& P, int ta, int tb,
                                                double d2, double alpha, const double (&r)[3],
                                                double qa, double qb, const double (&ma)[3],
                                                const double (&mb)[3], bool dip_a, bool dip_b,
                                                int task_qq, int task_qd, int task_dd,
                                                const double (&wa)[3], const double (&wb)[3],
                                                const double (&lown)[3], bool own_a,
                                                double (&dm)[3], double* g) {
  Radial<double> rd;
  radial<double, true>(d2, alpha, rd);
  const bool ldamp = P.ldamp != 0;
  double fa = 1.0, fda = 0.0, fb = 1.0, fdb = 0.0;
  if (ldamp) {
    tt_damp<double>(P.ba, P.ca, rd.d, P.ka, fa, fda);
    tt_damp<double>(P.bb, P.cb, rd.d, P.kb, fb, fdb);
  }
  double F1d = ldamp ? 1.0 - fa : 0.0, F2d = ldamp ? F1d + (rd.d / 3.0) * fda : 0.0;
  double F1d2 = ldamp ? 1.0 - fb : 0.0, F2d2 = ldamp ? F1d2 + (rd.d / 3.0) * fdb : 0.0;
  double B0 = rd.dm1 * rd.F0, B1 = rd.F1 * rd.dm3, B2 = 3.0 * rd.F2 * rd.dm5, B3 = 15.0 * rd.F3 * rd.dm7;
  double B1d = F1d * rd.dm3, B2d = 3.0 * F2d * rd.dm5, B1d2 = F1d2 * rd.dm3, B2d2 = 3.0 * F2d2 * rd.dm5;
  double rma = r[0] * ma[0] + r[1] * ma[1] + r[2] * ma[2];
  double rmb = r[0] * mb[0] + r[1] * mb[1] + r[2] * mb[2];
  double D[3] = {wa[0] - wb[0], wa[1] - wb[1], wa[2] - wb[2]};
  double Dr = D[0] * r[0] + D[1] * r[1] + D[2] * r[2];
  double Dma = D[0] * ma[0] + D[1] * ma[1] + D[2] * ma[2];
  double Dmb = D[0] * mb[0] + D[1] * mb[1] + D[2] * mb[2];
  const bool dd = task_dd && dip_a && dip_b;
  const bool qd = task_qd && (dip_a || dip_b);
  // d(D . f_ab)/dm_own
  for (int c = 0; c < 3; ++c) dm[c] = 0.0;
  if (own_a) {
    if (dd)
      for (int c = 0; c < 3; ++c)
        dm[c] += B3 * rmb * Dr * r[c] - B2 * (Dr * mb[c] + rmb * D[c] + Dmb * r[c]);
    if (qd)
      for (int c = 0; c < 3; ++c) {
        dm[c] += qb * (B2 * Dr * r[c] - B1 * D[c]);
        if (ldamp) dm[c] -= qb * (B2d * Dr * r[c] - B1d * D[c]);
      }
  } else {
    if (dd)
      for (int c = 0; c < 3; ++c)
        dm[c] += B3 * rma * Dr * r[c] - B2 * (Dr * ma[c] + Dma * r[c] + rma * D[c]);
    if (qd)
      for (int c = 0; c < 3; ++c) {
        dm[c] -= qa * (B2 * Dr * r[c] - B1 * D[c]);
        if (ldamp) dm[c] += qa * (B2d2 * Dr * r[c] - B1d2 * D[c]);
      }
  }
  for (int c = 0; c < 3; ++c) dm[c] *= -J.cu;  // u_F . F = -cu D . f_ab
  if (!g) return;
  // this visit's share: force on own = sgn cu f_ab, energy halved (both visits)
  const double sgn = own_a ? -1.0 : 1.0;
  const double* wo = own_a ? wa : wb;
  double wr = wo[0] * r[0] + wo[1] * r[1] + wo[2] * r[2];
  double wma = wo[0] * ma[0] + wo[1] * ma[1] + wo[2] * ma[2];
  double wmb = wo[0] * mb[0] + wo[1] * mb[1] + wo[2] * mb[2];
  double lr = lown[0] * r[0] + lown[1] * r[1] + lown[2] * r[2];
  for (int p = 0; p < J.nparam; ++p) {
    const FitParam& fp = J.prm[p];
    if (fp.kind == FIT_QSCALE) {
      double s = J.qscale;
      double val = 0.0;
      if (task_qq) {
        // w.f_qq, u_qq scale with s^2; the charge field on own with s
        double wf_qq = -qa * qb * B1 * wr;
        val += J.cu * sgn * 2.0 * wf_qq + 0.5 * J.gU * J.cu * 2.0 * qa * qb * B0;
        double Eown_r = own_a ? qb * (B1 - (ldamp ? B1d : 0.0)) * lr
                              : -qa * (B1 - (ldamp ? B1d2 : 0.0)) * lr;
        val += Eown_r;
      }
      if (qd) {
        double wf_qd = -qa * (B2 * wr * rmb - B1 * wmb) + qb * (B2 * wr * rma - B1 * wma);
        double u_qd = qa * B1 * rmb - qb * B1 * rma;
        if (ldamp) {
          wf_qd += -qb * (B2d * wr * rma - B1d * wma) + qa * (B2d2 * wr * rmb - B1d2 * wmb);
          u_qd += -qa * B1d2 * rmb + qb * B1d * rma;
        }
        val += J.cu * sgn * wf_qd + 0.5 * J.gU * J.cu * u_qd;
      }
      g[p] += val / s;
    } else if ((fp.kind == FIT_TTB || fp.kind == FIT_TTC) && ldamp) {
      // parameter (X = dipole type, Y = charge type): role a if (ta, tb) =
      // (X, Y) [table (X, X, Y)], role b if (tb, ta) = (X, Y) [table (X, Y, X)]
      for (int role = 0; role < 2; ++role) {
        bool hit = role == 0 ? (ta == fp.t1 && tb == fp.t2) : (tb == fp.t1 && ta == fp.t2);
        if (!hit) continue;
        double bb = role == 0 ? P.ba : P.bb, cc = role == 0 ? P.ca : P.cb;
        int kk = role == 0 ? P.ka : P.kb;
        double dfdb, dfddb, dfdc, dfddc;
        tt_damp_grad(bb, cc, rd.d, kk, dfdb, dfddb, dfdc, dfddc);
        double df = fp.kind == FIT_TTB ? dfdb : dfdc;
        double dfd = fp.kind == FIT_TTB ? dfddb : dfddc;
        double dB1 = -df * rd.dm3;                              // d(B1d)/dtheta
        double dB2 = 3.0 * (-df + (rd.d / 3.0) * dfd) * rd.dm5;  // d(B2d)/dtheta
        double val = 0.0;
        if (role == 0) {
          // f_ab += -qb (B2d r rma - B1d ma); u += qb B1d rma; Ea -= qb B1d r
          if (qd) {
            double wdf = -qb * (dB2 * wr * rma - dB1 * wma);
            val += J.cu * sgn * wdf + 0.5 * J.gU * J.cu * qb * dB1 * rma;
          }
          if (task_qq && own_a) val += -qb * dB1 * lr;
        } else {
          // f_ab += qa (B2d2 r rmb - B1d2 mb); u += -qa B1d2 rmb; Eb += qa B1d2 r
          if (qd) {
            double wdf = qa * (dB2 * wr * rmb - dB1 * wmb);
            val += J.cu * sgn * wdf - 0.5 * J.gU * J.cu * qa * dB1 * rmb;
          }
          if (task_qq && !own_a) val += qa * dB1 * lr;
        }
        g[p] += val;
      }
    }
  }
}

// Buckingham / BMH pair parameters from the visit of ion i (r = r_i - r_j):
// w_i . r dwij/dtheta + 1/2 g_U du/dtheta
__device__ __forceinline__ void sr_pair_adjoint(const PairAdj& J, const NBPair& P, int lbmhftd,
                                                int ti, int tj, double rijsq,
                                                const double (&r)[3], const double (&wi)[3],
                                                double* g) {
  if (P.A == 0.0) return;  // the reference skips the pair (non_bonded.f90:1153)
  double d = sqrt(rijsq);
  double wr = wi[0] * r[0] + wi[1] * r[1] + wi[2] * r[2];
  double e = exp(-P.B * d);
  double ir6 = 1.0 / (rijsq * rijsq * rijsq);
  double f6 = 1.0, fd6 = 0.0;
  if (lbmhftd) tt_damp<double>(P.BD, 1.0, d, 6, f6, fd6);
  for (int p = 0; p < J.nparam; ++p) {
    const FitParam& fp = J.prm[p];
    if (fp.kind > FIT_C) continue;
    bool hit = (ti == fp.t1 && tj == fp.t2) || (ti == fp.t2 && tj == fp.t1);
    if (!hit) continue;
    double du, dw;
    if (fp.kind == FIT_A) {
      du = e;
      dw = P.B * e / d;
    } else if (fp.kind == FIT_RHO) {
      // B = 1/rho: d/drho = -B^2 d/dB
      double duB = -P.A * d * e, dwB = P.A * e * (1.0 - P.B * d) / d;
      du = -P.B * P.B * duB;
      dw = -P.B * P.B * dwB;
    } else {
      du = -f6 * ir6;
      dw = (-6.0 * f6 * ir6 / d + fd6 * ir6) / d;
    }
    g[p] += wr * dw + 0.5 * J.gU * du;
  }
}

// ---------------------------------------------------------------------------
// one structure-factor channel over this CTA's k rows (FP64 tables):
//   W_i(k) = [ (hasq ? q_i : 0) + i (hasv ? k.v_i : 0) ] * (hasw ? k.w_i : 1)
// v from S.v, w from S.w; out[k] = sum_i W_i(k) e^{i k.r_i} (not A-scaled).
__device__ void bsf(cgx::cluster_group& cl, const BatchArgs& a, BCtx& X, const BShared& S,
                    const double4* __restrict__ Sw, bool hasq, bool hasv, bool hasw,
                    double2* __restrict__ out) {
  const BConf& c = *X.c;
  if (c.nk == 0) return;
  const int4* rows = a.rows + c.row_off;
  const int kz = c.kz;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  cl.sync();
  int r0 = (int)((long long)c.nrows * X.rank / X.C), r1 = (int)((long long)c.nrows * (X.rank + 1) / X.C);
  const int ntile = (2 * kz + 1 + kBNZ - 1) / kBNZ;
  int nitems = (r1 - r0) * ntile;
  for (int it = warp; it < nitems; it += nwarp) {
    int row = r0 + it / ntile, tile = it % ntile;
    int4 ri = rows[row];
    int nx = ri.x, ny = ri.y;
    int nz0 = ri.z + tile * kBNZ;
    if (nz0 > kz) continue;
    int nzn = min(kBNZ, kz - nz0 + 1);
    double accR[kBNZ], accI[kBNZ];
#pragma unroll
    for (int t = 0; t < kBNZ; ++t) accR[t] = accI[t] = 0.0;
    for (int i = lane; i < X.n; i += 32) {
      double2 XY = bphase<double>(a, c, i, nx, ny, 0);
      double2 Z1 = btab<double>(a, c, c.kx + 1 + c.ky + 1 + 1, i);
      double2 P = bphase_z<double>(a, c, i, XY, nz0);
      double qv = hasq ? S.s[i].w : 0.0;
      double kv = 0.0, v3 = 0.0, kw = 1.0, w3 = 0.0;
      if (hasv) {
        double4 u = S.v[i];
        double3 m = bmvec(c, u.x, u.y, u.z);
        kv = nx * m.x + ny * m.y + nz0 * m.z;
        v3 = m.z;
      }
      if (hasw) {
        double4 u = Sw[i];
        double3 m = bmvec(c, u.x, u.y, u.z);
        kw = nx * m.x + ny * m.y + nz0 * m.z;
        w3 = m.z;
      }
#pragma unroll
      for (int t = 0; t < kBNZ; ++t) {
        double wr = qv * kw, wi = kv * kw;
        accR[t] += wr * P.x - wi * P.y;
        accI[t] += wr * P.y + wi * P.x;
        kv += v3;
        kw += w3;
        P = cmul(P, Z1);
      }
    }
#pragma unroll
    for (int t = 0; t < kBNZ; ++t) {
      double vr = warp_sum(accR[t]);
      double vi = warp_sum(accI[t]);
      if (lane == 0 && t < nzn) {
        int kl = ri.w + (nz0 - ri.z) + t;
        out[c.k_off + kl] = make_double2(vr, vi);
      }
    }
  }
  cl.sync();
}

// per own ion: out_i = 2 pi B [ sum_k A_k n (k.w_i) Re(X1 P_i*) - sum_k A_k n Re(X2 P_i*) ]
// (channels X1, X2 not A-scaled; w from Sw)
__device__ void brecsum(const BatchArgs& a, const BCtx& X, const BShared& S,
                        const double4* __restrict__ Sw, const double2* __restrict__ X1,
                        const double2* __restrict__ X2, double4* __restrict__ outv) {
  const BConf& c = *X.c;
  const int4* rows = a.rows + c.row_off;
  const int kz = c.kz;
  int mown = X.i1 - X.i0;
  int sub = 1;
  while (sub < 32 && mown * sub * 2 <= (int)blockDim.x) sub *= 2;
  int slots = blockDim.x / sub;
  int iters = (mown + slots - 1) / slots;
  const int half = kBKChunk / 2;  // rho' chunk holds X1 in [0, half), X2 in [half, 2 half)
  for (int itn = 0; itn < iters; ++itn) {
    int slot = itn * slots + (int)threadIdx.x / sub;
    int me = threadIdx.x % sub;
    bool act = slot < mown;
    int i = X.i0 + (act ? slot : 0);
    double H[3] = {0, 0, 0}, K[3] = {0, 0, 0};
    double4 u = Sw[i];
    double3 m = bmvec(c, u.x, u.y, u.z);
    double2 Z1 = btab<double>(a, c, c.kx + 1 + c.ky + 1 + 1, i);
    int ra = 0;
    while (ra < c.nrows) {
      int kbase = rows[ra].w;
      int rb = ra;
      while (rb < c.nrows) {
        int4 rr = rows[rb];
        if (rr.w + (kz - rr.z + 1) - kbase > half) break;
        ++rb;
      }
      int kend = (rb < c.nrows) ? rows[rb].w : c.nk;
      __syncthreads();
      for (int k = threadIdx.x; k < kend - kbase; k += blockDim.x) {
        size_t gk = (size_t)c.k_off + kbase + k;
        double A = a.Ak[gk];
        double2 p1 = __ldcg(X1 + gk), p2 = __ldcg(X2 + gk);
        S.rho[k] = make_double2(A * p1.x, A * p1.y);
        S.rho[half + k] = make_double2(A * p2.x, A * p2.y);
      }
      __syncthreads();
      if (act) {
        for (int r = ra + me; r < rb; r += sub) {
          int4 ri = rows[r];
          int nx = ri.x, ny = ri.y, nz_lo = ri.z;
          double2 XY = bphase<double>(a, c, i, nx, ny, 0);
          double2 P = bphase_z<double>(a, c, i, XY, nz_lo);
          double kw = nx * m.x + ny * m.y + nz_lo * m.z;
          double T0 = 0, Tz = 0, U0 = 0, Uz = 0;
          int nn = kz - nz_lo + 1;
          const double2* x1 = S.rho + (ri.w - kbase);
          const double2* x2 = S.rho + half + (ri.w - kbase);
          for (int t = 0; t < nn; ++t) {
            double2 v1 = x1[t], v2 = x2[t];
            double re1 = v1.x * P.x + v1.y * P.y;  // Re(X1 P*)
            double re2 = v2.x * P.x + v2.y * P.y;
            double tt = kw * re1;
            T0 += tt;
            Tz += t * tt;
            U0 += re2;
            Uz += t * re2;
            kw += m.z;
            P = cmul(P, Z1);
          }
          H[0] += nx * T0;
          H[1] += ny * T0;
          H[2] += nz_lo * T0 + Tz;
          K[0] += nx * U0;
          K[1] += ny * U0;
          K[2] += nz_lo * U0 + Uz;
        }
      }
      ra = rb;
    }
    for (int o = 1; o < sub; o <<= 1)
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        H[d] += __shfl_xor_sync(FULL_MASK, H[d], o);
        K[d] += __shfl_xor_sync(FULL_MASK, K[d], o);
      }
    if (act && me == 0) {
      double o3[3];
      for (int d = 0; d < 3; ++d)
        o3[d] = kTwoPi * (c.B[3 * d] * (H[0] - K[0]) + c.B[3 * d + 1] * (H[1] - K[1]) +
                          c.B[3 * d + 2] * (H[2] - K[2]));
      outv[X.off + i] = make_double4(o3[0], o3[1], o3[2], 0.0);
    }
  }
}

// ---------------------------------------------------------------------------
// adjoint of one configuration (the forward of the same positions has run:
// a.s, a.tab64, a.x (induced dipoles), a.mu (total), a.E (field) are valid)
__device__ void bconfig_adjoint(cgx::cluster_group& cl, const BatchArgs& a, const AdjArgs& J, BCtx& X,
                                const BShared& S, double4* Sw) {
  const BConf& c = *X.c;
  const bool coul = (c.flags & BF_COUL) != 0, polar = (c.flags & BF_POLAR) != 0;
  const int task_qq = (c.flags & BF_QQ) ? 1 : 0, task_qd = (c.flags & BF_QD) ? 1 : 0;
  const int task_dd = (c.flags & BF_DD) ? 1 : 0;
  const double cu = c.coul_unit;
  const double gU = J.gE[X.cfg];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  PairAdj PJ;
  PJ.prm = J.prm;
  PJ.nparam = J.nparam;
  PJ.qscale = J.qscale;
  PJ.gU = gU;
  PJ.cu = cu;
  // ---- load -------------------------------------------------------------
  for (int i = X.i0 + threadIdx.x; i < X.i1; i += blockDim.x) {
    int gi = X.off + i;
    J.w[gi] = make_double4(J.gF[gi], J.gF[a.ntot + gi], J.gF[2 * (size_t)a.ntot + gi], 0.0);
  }
  for (int k = threadIdx.x; k < c.ntype * c.ntype; k += blockDim.x) {
    S.nb[k] = a.nbtab[c.nb_off + k];
    S.es[k] = a.estab[c.es_off + k];
  }
  cl.sync();
  for (int i = threadIdx.x; i < X.n; i += blockDim.x) {
    S.s[i] = ldcg4(a.s + X.off + i);
    S.t[i] = a.typ[X.off + i];
    S.v[i] = ldcg4(a.mu + X.off + i);
    Sw[i] = ldcg4(J.w + X.off + i);
  }
  __syncthreads();
  double g[kFitMax];
  for (int p = 0; p < kFitMax; ++p) g[p] = 0.0;
  int iters = 0;
  double rmsd = 0.0, tol = 0.0;
  if (coul && polar) {
    // ---- right-hand side: g_U cu R + d(u_F.F)/dmu + u_mu ---------------------
    for (int i = X.i0 + warp; i < X.i1; i += nwarp) {
      int gi = X.off + i;
      double dm[3] = {0, 0, 0};
      if (a.ipol[gi]) {
        double4 si = S.s[i];
        int ti = S.t[i];
        double4 mui = S.v[i], wi4 = Sw[i];
        for (int j = lane; j < X.n; j += 32) {
          if (j == i) continue;
          double4 sj = S.s[j];
          double rxd, ryd, rzd;
          double r2d = min_image_exact(c.A, xsub(si.x, sj.x), xsub(si.y, sj.y), xsub(si.z, sj.z),
                                       rxd, ryd, rzd);
          if (r2d > c.rc2) continue;
          int tj = S.t[j];
          double4 muj = S.v[j], wj4 = Sw[j];
          bool ia = half_mask(i, j);
          double sg = ia ? 1.0 : -1.0;
          double r[3] = {sg * rxd, sg * ryd, sg * rzd};
          double4 ma4 = ia ? mui : muj, mb4 = ia ? muj : mui, wa4 = ia ? wi4 : wj4, wb4 = ia ? wj4 : wi4;
          double ma[3] = {ma4.x, ma4.y, ma4.z}, mb[3] = {mb4.x, mb4.y, mb4.z};
          double wa[3] = {wa4.x, wa4.y, wa4.z}, wb[3] = {wb4.x, wb4.y, wb4.z};
          double zero[3] = {0, 0, 0}, d3[3];
          int ta = ia ? ti : tj, tb = ia ? tj : ti;
          es_pair_adjoint(PJ, S.es[ta * c.ntype + tb], ta, tb, r2d, c.alpha, r, ia ? si.w : sj.w,
                          ia ? sj.w : si.w, ma, mb, ma4.x != 0.0 || ma4.y != 0.0 || ma4.z != 0.0,
                          mb4.x != 0.0 || mb4.y != 0.0 || mb4.z != 0.0, task_qq, task_qd, task_dd,
                          wa, wb, zero, ia, d3, nullptr);
          for (int d = 0; d < 3; ++d) dm[d] += d3[d];
        }
      }
      for (int d = 0; d < 3; ++d) dm[d] = warp_sum(dm[d]);
      if (lane == 0) J.rhs[gi] = make_double4(dm[0], dm[1], dm[2], 0.0);
    }
    // reciprocal: rho = sum (q + i k.mu) P and sigma = sum (k.u)(q + i k.mu) P
    bsf(cl, a, X, S, Sw, task_qq != 0, true, false, J.rq);
    bsf(cl, a, X, S, Sw, task_qq != 0, true, true, J.sq);
    __syncthreads();
    brecsum(a, X, S, Sw, J.rq, J.sq, J.lam);  // lam as scratch
    __syncthreads();
    const double scale8 = 2.0 * (2.0 * (kTwoPi / c.omega));
    double v1[1] = {0.0};
    for (int i = X.i0 + threadIdx.x; i < X.i1; i += blockDim.x) {
      int gi = X.off + i;
      double4 o = make_double4(0, 0, 0, 0);
      if (a.ipol[gi]) {
        double4 rr = J.rhs[gi], rc = J.lam[gi];
        double4 ax = bmat3(a.inv + 9 * (size_t)gi, a.x[gi]);
        double4 E = a.E[gi];
        double R[3] = {ax.x - E.x, ax.y - E.y, ax.z - E.z};
        double gm[3] = {0, 0, 0};
        if (J.gmu) {
          gm[0] = J.gmu[3 * (size_t)gi];
          gm[1] = J.gmu[3 * (size_t)gi + 1];
          gm[2] = J.gmu[3 * (size_t)gi + 2];
        }
        o.x = rr.x + cu * scale8 * rc.x + gU * cu * R[0] + gm[0];
        o.y = rr.y + cu * scale8 * rc.y + gU * cu * R[1] + gm[1];
        o.z = rr.z + cu * scale8 * rc.z + gU * cu * R[2] + gm[2];
        v1[0] += o.x * o.x + o.y * o.y + o.z * o.z;
      }
      J.rhs[gi] = o;
    }
    cluster_sum<1>(cl, X, S, v1);
    double rms = sqrt(v1[0] / (3.0 * max(c.npol, 1)));
    tol = fmax(J.tol_rel * rms, 1e-300);
    // ---- adjoint solve H lambda = rhs, lambda0 = alpha rhs -------------------
    for (int i = X.i0 + threadIdx.x; i < X.i1; i += blockDim.x) {
      int gi = X.off + i;
      J.lam[gi] = a.ipol[gi] ? bmat3(a.pol + 9 * (size_t)gi, J.rhs[gi]) : make_double4(0, 0, 0, 0);
    }
    if (rms > 0.0) bsolve<false>(cl, a, X, S, J.rhs, J.lam, tol, 4 * c.maxit, iters, rmsd);
    cl.sync();
    for (int i = threadIdx.x; i < X.n; i += blockDim.x) S.v[i] = ldcg4(a.mu + X.off + i);
    __syncthreads();
  } else {
    for (int i = X.i0 + threadIdx.x; i < X.i1; i += blockDim.x) J.lam[X.off + i] = make_double4(0, 0, 0, 0);
  }
  // ---- parameter gradient ----------------------------------------------------
  bool any_sr = false, any_es = false;
  for (int p = 0; p < J.nparam; ++p) {
    if (J.prm[p].kind <= FIT_C) any_sr = true;
    if (J.prm[p].kind >= FIT_TTB) any_es = true;
  }
  any_sr = any_sr && (c.flags & BF_SR) && (c.flags & BF_BMH);
  any_es = any_es && coul;
  const int lbmhftd = (c.flags & BF_BMHFTD) ? 1 : 0;
  for (int i = X.i0 + warp; i < X.i1; i += nwarp) {
    int gi = X.off + i;
    double4 si = S.s[i];
    int ti = S.t[i];
    double4 mui = S.v[i], wi4 = Sw[i];
    double4 li4 = J.lam[gi];
    double wi[3] = {wi4.x, wi4.y, wi4.z}, li[3] = {li4.x, li4.y, li4.z};
    for (int j = lane; j < X.n; j += 32) {
      if (j == i) continue;
      double4 sj = S.s[j];
      double rxd, ryd, rzd;
      double r2d = min_image_exact(c.A, xsub(si.x, sj.x), xsub(si.y, sj.y), xsub(si.z, sj.z), rxd,
                                   ryd, rzd);
      int tj = S.t[j];
      if (any_sr) {
        const NBPair& P = S.nb[ti * c.ntype + tj];
        if (r2d < P.rcutsq) {
          double r[3] = {rxd, ryd, rzd};
          sr_pair_adjoint(PJ, P, lbmhftd, ti, tj, r2d, r, wi, g);
        }
      }
      if (any_es && r2d <= c.rc2) {
        double4 muj = S.v[j], wj4 = Sw[j];
        bool ia = half_mask(i, j);
        double sg = ia ? 1.0 : -1.0;
        double r[3] = {sg * rxd, sg * ryd, sg * rzd};
        double4 ma4 = ia ? mui : muj, mb4 = ia ? muj : mui, wa4 = ia ? wi4 : wj4, wb4 = ia ? wj4 : wi4;
        double ma[3] = {ma4.x, ma4.y, ma4.z}, mb[3] = {mb4.x, mb4.y, mb4.z};
        double wa[3] = {wa4.x, wa4.y, wa4.z}, wb[3] = {wb4.x, wb4.y, wb4.z};
        double d3[3];
        int ta = ia ? ti : tj, tb = ia ? tj : ti;
        es_pair_adjoint(PJ, S.es[ta * c.ntype + tb], ta, tb, r2d, c.alpha, r, ia ? si.w : sj.w,
                        ia ? sj.w : si.w, ma, mb, ma4.x != 0.0 || ma4.y != 0.0 || ma4.z != 0.0,
                        mb4.x != 0.0 || mb4.y != 0.0 || mb4.z != 0.0, task_qq, task_qd, task_dd,
                        wa, wb, li, ia, d3, g);
      }
    }
  }
  // per-ion terms: polarisability, self energy of the charges
  const double selfa = c.alpha / sqrt(kPi);
  for (int i = X.i0 + threadIdx.x; i < X.i1; i += blockDim.x) {
    int gi = X.off + i;
    int ti = S.t[i];
    for (int p = 0; p < J.nparam; ++p) {
      const FitParam& fp = J.prm[p];
      if (fp.kind == FIT_POL && ti == fp.t1 && a.ipol[gi]) {
        double al = a.pol[9 * (size_t)gi];
        double4 m = a.x[gi], l = J.lam[gi];
        double mm = m.x * m.x + m.y * m.y + m.z * m.z, lm = l.x * m.x + l.y * m.y + l.z * m.z;
        g[p] += lm / (al * al) - 0.5 * gU * cu * mm / (al * al);
      }
      if (fp.kind == FIT_QSCALE && coul && task_qq) {
        double q = S.s[i].w;
        g[p] += gU * cu * (-2.0 * selfa * q * q) / J.qscale;
      }
    }
  }
  // reciprocal charge-scale terms: rho_lambda, then per k over this CTA's rows
  bool has_s = false;
  for (int p = 0; p < J.nparam; ++p) has_s = has_s || J.prm[p].kind == FIT_QSCALE;
  if (has_s && coul && task_qq && c.nk > 0) {
    // channels: rq = rho_q, rm = rho_mu, sq = sigma_q, sm = sigma_mu, rl = rho_lambda
    bsf(cl, a, X, S, Sw, true, false, false, J.rq);
    bsf(cl, a, X, S, Sw, false, true, false, J.rm);
    bsf(cl, a, X, S, Sw, true, false, true, J.sq);
    bsf(cl, a, X, S, Sw, false, true, true, J.sm);
    cl.sync();
    for (int i = threadIdx.x; i < X.n; i += blockDim.x) S.v[i] = ldcg4(J.lam + X.off + i);
    __syncthreads();
    bsf(cl, a, X, S, Sw, false, true, false, J.rl);
    const double fpi_V = 2.0 * (kTwoPi / c.omega), epi_V = 2.0 * fpi_V;
    double acc = 0.0;
    int r0 = (int)((long long)c.nrows * X.rank / X.C), r1 = (int)((long long)c.nrows * (X.rank + 1) / X.C);
    int k0 = a.rows[c.row_off + r0].w;
    int k1 = (r1 < c.nrows) ? a.rows[c.row_off + r1].w : c.nk;
    if (r0 >= r1) k1 = k0;
    for (int k = k0 + threadIdx.x; k < k1; k += blockDim.x) {
      size_t gk = (size_t)c.k_off + k;
      double A = a.Ak[gk];
      double2 q = __ldcg(J.rq + gk), m = __ldcg(J.rm + gk), sq = __ldcg(J.sq + gk);
      double2 sm = __ldcg(J.sm + gk), l = __ldcg(J.rl + gk);
      double qq = q.x * q.x + q.y * q.y, qm = q.x * m.x + q.y * m.y;  // Re(conj(q) m)
      // Im(conj(x) y) = x.re y.im - x.im y.re
      double iqsq = q.x * sq.y - q.y * sq.x, iqsm = q.x * sm.y - q.y * sm.x;
      double imsq = m.x * sq.y - m.y * sq.x;
      double rql = q.x * l.x + q.y * l.y;
      acc += A * (gU * cu * fpi_V * (2.0 * qq + 2.0 * qm) +
                  cu * epi_V * (2.0 * iqsq + iqsm + imsq) - epi_V * rql);
    }
    for (int p = 0; p < J.nparam; ++p)
      if (J.prm[p].kind == FIT_QSCALE) g[p] += acc / J.qscale;
  }
  cluster_sum<kFitMax>(cl, X, S, g);
  if (X.rank == 0 && threadIdx.x == 0) {
    for (int p = 0; p < kFitMax; ++p) J.grad[(size_t)X.cfg * kFitMax + p] = g[p];
    J.info[4 * (size_t)X.cfg] = iters;
    J.info[4 * (size_t)X.cfg + 1] = rmsd;
    J.info[4 * (size_t)X.cfg + 2] = tol;
  }
}

__global__ void __launch_bounds__(512) k_batch_adjoint(BatchArgs a, AdjArgs J, int nmax) {
  extern __shared__ __align__(16) unsigned char bsm[];
  BShared S = batch_smem(bsm, nmax);
  double4* Sw = reinterpret_cast<double4*>(bsm + batch_smem_extra_offset(nmax));
  cgx::cluster_group cl = cgx::this_cluster();
  BCtx X;
  X.rank = (int)cl.block_rank();
  X.C = (int)cl.num_blocks();
  while (true) {
    if (X.rank == 0 && threadIdx.x == 0) *S.cfg = atomicAdd(a.queue, 1);
    cl.sync();
    int qpos = *cl.map_shared_rank(S.cfg, 0);
    cl.sync();
    if (qpos >= a.nconf) break;
    int cfg = a.order[qpos];
    const BConf* c = a.conf + cfg;
    X.c = c;
    X.cfg = cfg;
    X.n = c->n;
    X.off = c->off;
    X.i0 = (int)((long long)X.n * X.rank / X.C);
    X.i1 = (int)((long long)X.n * (X.rank + 1) / X.C);
    X.part = a.part + (size_t)cfg * kBMaxC * 2 * kBPart;
    X.parity = 0;
    bconfig_adjoint(cl, a, J, X, S, Sw);
    __syncthreads();
  }
}

}  // namespace mdff
