// realspace.cuh -- real-space pair kernels over the full Verlet list.
//
//  * k_shortrange: engforce_bmhftd_pbc (non_bonded.f90:1076-1228) and
//    engforce_nmlj_pbc (non_bonded.f90:660-827).
//  * k_es_field:   the field-only Ewald real-space passes of the PIM solve
//    (multipole_ES_dir with do_forces=.false., ewald_dir.f90:40-798): the
//    damped charge field (static pass, moment_from_pola.f90:327-330) and the
//    undamped dipole T2 field (induced pass, moment_from_pola.f90:401-404).
//  * k_es_force:   the final multipole_ES_dir with qq + qd + dd tasks, damping,
//    energy, field, forces and stress (engforce_driver.f90:164-166).
//
// Warp per atom i; lanes stride i's row.  Each pair is visited from both
// sides; the reference's role of the pair (which ion is "ia") is recovered
// from the parity mask, so asymmetric damping tables behave as in the
// reference.  Where every damped pair uses one Tang-Toennies order the
// kernels are instantiated for it (compile-time Horner, tt_damp_k).  Per-atom sums are formed in registers with no atomics; pair
// energies/stresses are halved and reduced per block in a fixed order.
#pragma once
#include "common.cuh"

namespace mdff {

struct NBPair {        // per ordered type pair (ti,tj), after symmetrisation
  double A, B, C, D, BD, wall;
  double rcutsq;
  double epsp, plj, qlj, sigsq, fc, uc, uc1, uc2;
};

struct ESPair {        // per ordered role pair (ta = type of "ia", tb = type of "ja")
  int ldamp;           // ldip_damping(ta,ta,tb) .or. ldip_damping(tb,ta,tb)
  int ka, kb;          // TT orders for the field on a / on b
  int thole;           // MDFF_THOLE_* when both types are polarisable, else 0
  double ba, ca, bb, cb;  // TT b, c for the field on a: (ta,ta,tb); on b: (tb,ta,tb)
  double th_a, th_A;   // thole_param(ta,tb), (alpha_xx(ta) alpha_xx(tb))^(1/6)
};

// FP32 copy of an ESPair for the FP32 passes: the damping and Thole
// parameters converted once per block instead of once per pair visit
struct ESPairF {
  int ldamp, ka, kb, thole;
  float ba, ca, bb, cb;
  float th_a, th_A;
};
__device__ __forceinline__ ESPairF espair_f(const ESPair& P) {
  return ESPairF{P.ldamp, P.ka, P.kb, P.thole, (float)P.ba, (float)P.ca, (float)P.bb,
                 (float)P.cb, (float)P.th_a, (float)P.th_A};
}
// the table a pass of precision R keeps in shared memory
template <typename R>
struct espair_t {
  typedef ESPair T;
};
template <>
struct espair_t<float> {
  typedef ESPairF T;
};
template <typename PT>
__device__ __forceinline__ PT espair_as(const ESPair& P);
template <>
__device__ __forceinline__ ESPair espair_as<ESPair>(const ESPair& P) { return P; }
template <>
__device__ __forceinline__ ESPairF espair_as<ESPairF>(const ESPair& P) { return espair_f(P); }

// Thole functions on the dipole-dipole tensor (ewald_dir.f90:305-430): the
// radial functions F1, F2 of T2 = 3 r r F2 / d^5 - F1 / d^3 for the field and
// energy of a pair of polarisable ions (the force keeps the plain tensor)
template <typename R, typename PT = ESPair>
__device__ __forceinline__ void thole_radial(const PT& P, R d, R& F1, R& F2) {
  switch (P.thole) {
    case 1: {  // linear: no Ewald screening inside s = a A (:316-347)
      R sth = (R)(P.th_a * P.th_A);
      if (d < sth) {
        R v = d / sth;
        R v3 = v * v * v, v4 = v3 * v;
        F2 = v4;
        F1 = R(4) * v3 - R(3) * v4;
      }
    } break;
    case 2: {  // expon1 (:353-373)
      R x = d / (R)P.th_A;
      R u = (R)P.th_a * (x * x * x);
      R e = rexp<R>(-u);
      F2 = F2 * (R(1) - (R(1) + u) * e);
      F1 = F1 * (R(1) - e);
    } break;
    case 3: {  // expon2 (:378-399): u = a d A as written there
      R ar = (R)P.th_a * d * (R)P.th_A;
      R ar2 = ar * ar / R(2);
      R ar3 = ar2 * ar / R(3);
      R e = rexp<R>(-ar);
      F2 = F2 * (R(1) - (R(1) + ar + ar2 + ar3) * e);
      F1 = F1 * (R(1) - (R(1) + ar + ar2) * e);
    } break;
    case 4: {  // gauss (:404-422), NR error function
      R ra = d / (R)P.th_a;
      R e = (R)1.1283791670955125739 * ra * rexp<R>(-ra * ra);
      R erfra = R(1) - nr_erfc<R>(ra);
      F2 = F2 * (erfra - e * (R(1) + (R(2) / R(3)) * ra));
      F1 = F1 * (erfra - e);
    } break;
    default: break;
  }
}

// --------------------------------------------------------------------------
// short range.  Partials per block: [u_bmh, vir_bmh, u_lj, vir_lj,
// tau_bmh(6: xx yy zz xy xz yz), tau_lj(6)] -> 16 doubles.
constexpr int kSRPart = 16;

// one BMH / BMHFTD (+ r^-24 wall) pair at r^2 = rijsq: energy u and the force
// scalar wij (F_i = wij r_ij) of engforce_bmhftd_pbc (non_bonded.f90:1153-1200).
// The reference skips pairs with A = 0 (:1153); the optional wall acts on its own.
template <typename R>
__device__ __forceinline__ void sr_pair_bmh(const NBPair& P, int lbmhftd, R rijsq, R& u, R& wij) {
  // 1/d from one reciprocal square root; d, 1/r^2 and the divisions by d of
  // non_bonded.f90:1180-1200 become products (a few ulp from the reference's
  // square root and quotients)
  R dinv = rinv_sqrt<R>(rijsq);
  R d = rijsq * dinv;
  R ir2 = dinv * dinv;
  R wnum = R(0);
  u = R(0);
  if (P.A != 0.0) {
    R erh = (R)P.A * rexp<R>(-(R)P.B * d);
    R ir6 = ir2 * ir2 * ir2;
    R ir8 = ir6 * ir2;
    ir6 = ir6 * (R)P.C;
    ir8 = ir8 * (R)P.D;
    R f6 = R(1), f8 = R(1), fd6 = R(0), fd8 = R(0);
    if (lbmhftd) {
      tt_damp_k<R, 6>((R)P.BD, R(1), d, 6, f6, fd6);
      tt_damp_k<R, 8>((R)P.BD, R(1), d, 8, f8, fd8);
    }
    R ir6d = ir6 * f6, ir8d = ir8 * f8;
    R ir7 = R(6) * ir6d * dinv;
    R ir9 = R(8) * ir8d * dinv;
    u = erh - ir6d - ir8d;
    wnum = (R)P.B * erh - ir7 - ir9 + ir6 * fd6 + ir8 * fd8;
  }
  if (P.wall != 0.0) {
    R ir8r = (ir2 * ir2) * (ir2 * ir2);
    R uw = (R)P.wall * (ir8r * ir8r * ir8r);
    u += uw;
    wnum += R(24) * uw * dinv;
  }
  wij = wnum * dinv;
}

// one n-m LJ pair (engforce_nmlj_pbc, non_bonded.f90:740-790): energy with the
// trunc shift, force scalar wij (F_i = wij r_ij)
template <typename R>
__device__ __forceinline__ void sr_pair_lj(const NBPair& P, int trunc, R rijsq, R& e, R& wij) {
  R sr2 = (R)P.sigsq / rijsq;
  R srp, srq;
  if (sizeof(R) == 8) {
    srp = (R)pow((double)sr2, 0.5 * P.plj);
    srq = (R)pow((double)sr2, 0.5 * P.qlj);
  } else {
    srp = powf((float)sr2, 0.5f * (float)P.plj);
    srq = powf((float)sr2, 0.5f * (float)P.qlj);
  }
  e = (R)P.epsp * ((R)P.plj * srq - (R)P.qlj * srp);
  if (trunc == 1) e = e - (R)P.uc;
  if (trunc == 2) e = e + (R)P.uc1 * rijsq - (R)P.uc2;
  wij = (R)P.fc * (srq - srp) * sr2;
}

// MODE bit 0: BMH / BMHFTD (+ wall), bit 1: n-m LJ.  One instantiation per
// mode keeps the accumulators of the absent potential out of the registers.
template <typename R, int MODE>
static __global__ void __launch_bounds__(256, MODE == 3 ? 2 : 4) k_shortrange(
    const double4* __restrict__ s, const int* __restrict__ itype, const int* __restrict__ nbr,
    const int* __restrict__ nnb, int cap, int natm, const CellC* __restrict__ cell,
    const NBPair* __restrict__ tab, int ntype, int lbmhftd, int trunc,
    double* __restrict__ force /* SoA [3][natm] */, double* __restrict__ part) {
  constexpr bool do_bmh = (MODE & 1) != 0, do_lj = (MODE & 2) != 0;
  __shared__ NBPair stab[MDFF_NT * MDFF_NT];
  __shared__ double red[kSRPart * 8];
  for (int k = threadIdx.x; k < ntype * ntype; k += blockDim.x) stab[k] = tab[k];
  __syncthreads();
  int lane = threadIdx.x & 31;
  int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  double acc[kSRPart];
#pragma unroll
  for (int k = 0; k < kSRPart; ++k) acc[k] = 0.0;
  double fb[3] = {0, 0, 0}, fl[3] = {0, 0, 0};
  if (i < natm) {
    double4 si = s[i];
    int ti = itype[i];
    int n = nnb[i];
    const int* row = nbr + (size_t)i * cap;
    for (int k = lane; k < n; k += 32) {
      int j = row[k];
      double4 sj = s[j];
      int tj = tag_type(sj.w);
      double rxd, ryd, rzd;
      double r2d = min_image_exact(cell->A, xsub(si.x, sj.x), xsub(si.y, sj.y), xsub(si.z, sj.z),
                                   rxd, ryd, rzd);
      const NBPair& P = stab[ti * ntype + tj];
      if (r2d >= P.rcutsq) continue;  // non_bonded.f90:1154 strict <
      R rx = (R)rxd, ry = (R)ryd, rz = (R)rzd, rijsq = (R)r2d;
      // the reference skips pairs with A = 0 (non_bonded.f90:1153); the
      // optional r^-24 wall extension acts on its own
      if (do_bmh && (P.A != 0.0 || P.wall != 0.0)) {
        R u, wij;
        sr_pair_bmh<R>(P, lbmhftd, rijsq, u, wij);
        R fx = wij * rx, fy = wij * ry, fz = wij * rz;
        fb[0] += (double)fx;
        fb[1] += (double)fy;
        fb[2] += (double)fz;
        acc[0] += 0.5 * (double)u;
        acc[1] += 0.5 * (double)(rx * fx + ry * fy + rz * fz);
        acc[4] += (double)(rx * fx);  // 0.5*(r_a f_b + r_b f_a) on the diagonal = r_a f_a
        acc[5] += (double)(ry * fy);
        acc[6] += (double)(rz * fz);
        acc[7] += 0.5 * (double)(rx * fy + ry * fx);
        acc[8] += 0.5 * (double)(rx * fz + rz * fx);
        acc[9] += 0.5 * (double)(ry * fz + rz * fy);
      }
      if (do_lj) {
        R e, wij;
        sr_pair_lj<R>(P, trunc, rijsq, e, wij);
        R fx = wij * rx, fy = wij * ry, fz = wij * rz;
        fl[0] += (double)fx;
        fl[1] += (double)fy;
        fl[2] += (double)fz;
        acc[2] += 0.5 * (double)e;
        acc[3] += 0.5 * (double)(wij * rijsq);
        acc[10] += (double)(rx * fx);
        acc[11] += (double)(ry * fy);
        acc[12] += (double)(rz * fz);
        acc[13] += 0.5 * (double)(rx * fy + ry * fx);
        acc[14] += 0.5 * (double)(rx * fz + rz * fx);
        acc[15] += 0.5 * (double)(ry * fz + rz * fy);
      }
    }
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      fb[a] = warp_sum(fb[a]);
      fl[a] = warp_sum(fl[a]);
    }
    if (lane == 0) {
      // the reference zeroes fx in each short-range routine, so with both
      // on only the BMH forces survive (non_bonded.f90:699-701, 1104-1106)
      const double* f = do_bmh ? fb : fl;
      force[i] = f[0];
      force[natm + i] = f[1];
      force[2 * natm + i] = f[2];
    }
  }
  block_sum<kSRPart>(acc, red);
  if (threadIdx.x == 0)
    for (int k = 0; k < kSRPart; ++k) part[(size_t)blockIdx.x * kSRPart + k] = acc[k];
}

// --------------------------------------------------------------------------
// Ewald real-space radial functions F0..F3 (ewald_dir.f90:230-236).
template <typename R>
struct Radial {
  R d, dm1, dm3, dm5, dm7, F0, F1, F2, F3;
};

// (FP64: the reference's divisions by d, d^2, sqrt(pi), 3 and 15 are products
// with reciprocals, ~1 ulp from its quotients)
template <typename R, bool NEED_F3>
__device__ __forceinline__ void radial(R d2, R alpha, Radial<R>& o) {
  const R rpiroot = (R)0.56418958354775628695;  // 1/sqrt(pi)
  R rinv = rinv_sqrt<R>(d2);
  R dm2 = rinv * rinv;
  R d = d2 * rinv;
  o.d = d;
  o.dm1 = rinv;
  o.dm3 = rinv * dm2;
  o.dm5 = o.dm3 * dm2;
  o.dm7 = o.dm5 * dm2;
  R a2 = alpha * alpha, a3 = a2 * alpha;
  R expon = rexp<R>(-a2 * d2) * rpiroot;
  o.F0 = nr_erfc<R>(alpha * d);
  o.F1 = o.F0 + R(2) * alpha * d * expon;
  R d3 = d2 * d;
  o.F2 = o.F1 + (R(4) / R(3)) * a3 * d3 * expon;
  if (NEED_F3) {
    R a5 = a3 * a2, d5 = d3 * d2;
    o.F3 = o.F2 + (R(8) / R(15)) * a5 * d5 * expon;
  } else {
    o.F3 = R(0);
  }
}

// FP32: no IEEE divisions (each is a multi-instruction sequence): 1/d from
// rsqrtf, powers by multiplication, constants folded
template <>
__device__ __forceinline__ void radial<float, false>(float d2, float alpha, Radial<float>& o) {
  float rinv = rsqrtf(d2);
  float dm2 = rinv * rinv;
  o.d = d2 * rinv;
  o.dm1 = rinv;
  o.dm3 = rinv * dm2;
  o.dm5 = o.dm3 * dm2;
  o.dm7 = o.dm5 * dm2;
  float a2 = alpha * alpha;
  float expon = expf(-a2 * d2) * 0.56418958354775628695f;  // 1/sqrt(pi)
  float z = alpha * o.d;
  float t = __frcp_rn(1.0f + 0.5f * z);
  float p = -.82215223f + t * .17087277f;
  p = 1.48851587f + t * p;
  p = -1.13520398f + t * p;
  p = .27886807f + t * p;
  p = -.18628806f + t * p;
  p = .09678418f + t * p;
  p = .37409196f + t * p;
  p = 1.00002368f + t * p;
  o.F0 = t * expf(-z * z - 1.26551223f + t * p);
  float ade = alpha * o.d * expon;
  o.F1 = o.F0 + 2.0f * ade;
  o.F2 = o.F1 + (4.0f / 3.0f) * a2 * d2 * ade;
  o.F3 = 0.0f;
}
template <>
__device__ __forceinline__ void radial<float, true>(float d2, float alpha, Radial<float>& o) {
  float rinv = rsqrtf(d2);
  float dm2 = rinv * rinv;
  o.d = d2 * rinv;
  o.dm1 = rinv;
  o.dm3 = rinv * dm2;
  o.dm5 = o.dm3 * dm2;
  o.dm7 = o.dm5 * dm2;
  float a2 = alpha * alpha;
  float expon = expf(-a2 * d2) * 0.56418958354775628695f;  // 1/sqrt(pi)
  float z = alpha * o.d;
  float t = __frcp_rn(1.0f + 0.5f * z);
  float p = -.82215223f + t * .17087277f;
  p = 1.48851587f + t * p;
  p = -1.13520398f + t * p;
  p = .27886807f + t * p;
  p = -.18628806f + t * p;
  p = .09678418f + t * p;
  p = .37409196f + t * p;
  p = 1.00002368f + t * p;
  o.F0 = t * expf(-z * z - 1.26551223f + t * p);
  float ade = z * expon;
  float a2d2 = a2 * d2;
  o.F1 = o.F0 + 2.0f * ade;
  o.F2 = o.F1 + (4.0f / 3.0f) * a2d2 * ade;
  o.F3 = o.F2 + (8.0f / 15.0f) * a2d2 * a2d2 * ade;
}

// --------------------------------------------------------------------------
// field-only pass.  Adds into E (AoS double4 [natm]):
//   QQ : E_i += q_j r_ij dm3 (F1 - F1d_i)       (qq block, ewald_dir.f90:533-541)
//   DD : E_i += T2(r_ij) . mu_j                  (dd block, ewald_dir.f90:566-571)
// dd_mask: 0 -> the reference's condition any(mu_i /= 0) .and. any(mu_j /= 0)
//          1 -> both ions polarisable (the linear operator of the CG solve)
template <typename R>
struct vec4t;
template <>
struct vec4t<double> {
  typedef double4 T;
};
template <>
struct vec4t<float> {
  typedef float4 T;
};

// minimum-image vector of the pair (i, j) and its square.  FP64: the
// reference's exact arithmetic.  FP32: the direct-coordinate difference and
// its image shift in FP64 (positions of a 50 A box need it), A.s in FP32.
template <typename R>
__device__ __forceinline__ R pair_vec(const double* A, double4 si, double4 sj, R& rx, R& ry, R& rz);
template <>
__device__ __forceinline__ double pair_vec<double>(const double* A, double4 si, double4 sj,
                                                   double& rx, double& ry, double& rz) {
  return min_image_exact(A, xsub(si.x, sj.x), xsub(si.y, sj.y), xsub(si.z, sj.z), rx, ry, rz);
}
template <>
__device__ __forceinline__ float pair_vec<float>(const double* A, double4 si, double4 sj,
                                                 float& rx, float& ry, float& rz) {
  // the image shift in FP64 too, so that a pair across the boundary keeps
  // FP32's relative precision in its (small) direct-coordinate difference
  double ddx = si.x - sj.x, ddy = si.y - sj.y, ddz = si.z - sj.z;
  float dx = (float)(ddx - rint(ddx)), dy = (float)(ddy - rint(ddy)), dz = (float)(ddz - rint(ddz));
  rx = dx * (float)A[0] + dy * (float)A[1] + dz * (float)A[2];
  ry = dx * (float)A[3] + dy * (float)A[4] + dz * (float)A[5];
  rz = dx * (float)A[6] + dy * (float)A[7] + dz * (float)A[8];
  return rx * rx + ry * ry + rz * rz;
}

// the same FP32 pair vector with the cell matrix already in FP32 registers
__device__ __forceinline__ float pair_vec_f(const float (&A)[9], double4 si, double4 sj, float& rx,
                                            float& ry, float& rz) {
  double ddx = si.x - sj.x, ddy = si.y - sj.y, ddz = si.z - sj.z;
  float dx = (float)(ddx - rint(ddx)), dy = (float)(ddy - rint(ddy)), dz = (float)(ddz - rint(ddz));
  rx = dx * A[0] + dy * A[1] + dz * A[2];
  ry = dx * A[3] + dy * A[4] + dz * A[5];
  rz = dx * A[6] + dy * A[7] + dz * A[8];
  return rx * rx + ry * ry + rz * rz;
}

// field at i from j of the field-only passes (k_es_field): the charge field
// q_j r dm3 (F1 - F1d) with the pair's damping roles, and the dipole field
// T2 . mu_j (ewald_dir.f90:533-541, 566-571); added into (ex, ey, ez).
template <typename R, bool QQ, bool DD, int K = 0>
__device__ __forceinline__ void es_field_pair(const ESPair* stab, int ntype, int i, int j, int ti,
                                              int tj, R rx, R ry, R rz, R r2, R alpha, int damp,
                                              double qj, bool dd, R mx, R my, R mz, R& ex, R& ey,
                                              R& ez, int thole = 0) {
  Radial<R> g;
  radial<R, false>(r2, alpha, g);
  if (QQ && qj != 0.0) {
    R F1d = R(0);
    if (damp) {
      bool i_is_a = half_mask(i, j);
      int ta = i_is_a ? ti : tj, tb = i_is_a ? tj : ti;
      const ESPair& P = stab[ta * ntype + tb];
      if (P.ldamp && (i_is_a ? P.ca : P.cb) != 0.0) {  // c = 0 damps nothing
        R fdm, fdd;
        if (i_is_a)
          tt_damp_k<R, K>((R)P.ba, (R)P.ca, g.d, P.ka, fdm, fdd);
        else
          tt_damp_k<R, K>((R)P.bb, (R)P.cb, g.d, P.kb, fdm, fdd);
        F1d = R(1) - fdm;
      }
    }
    R c = (R)qj * g.dm3 * (g.F1 - F1d);
    ex += c * rx;
    ey += c * ry;
    ez += c * rz;
  }
  if (DD && dd) {
    R F1 = g.F1, F2 = g.F2;
    if (thole) {
      bool i_is_a = half_mask(i, j);
      const ESPair& P = stab[(i_is_a ? ti : tj) * ntype + (i_is_a ? tj : ti)];
      if (P.thole) thole_radial<R>(P, g.d, F1, F2);
    }
    R B1 = F1 * g.dm3, B2 = R(3) * F2 * g.dm5;
    R rm = rx * mx + ry * my + rz * mz;
    ex += B2 * rx * rm - B1 * mx;
    ey += B2 * ry * rm - B1 * my;
    ez += B2 * rz * rm - B1 * mz;
  }
}

// dipoles converted for the FP32 passes
static __global__ void k_to_float4(const double4* __restrict__ in, int n, float4* __restrict__ out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double4 v = in[i];
  out[i] = make_float4((float)v.x, (float)v.y, (float)v.z, 0.f);
}

// field-only pass.  Adds into E (AoS double4 [natm]):
//   QQ : E_i += q_j r_ij dm3 (F1 - F1d_i)       (qq block, ewald_dir.f90:533-541)
//   DD : E_i += T2(r_ij) . mu_j                  (dd block, ewald_dir.f90:566-571)
// dd_mask: 0 -> the reference's condition any(mu_i /= 0) .and. any(mu_j /= 0)
//          1 -> both ions polarisable (the linear operator of the CG solve)
// mu is double4 for FP64 and float4 for FP32 (k_to_float4).  K: compile-time
// Tang-Toennies order of the damped charge field (0 = per pair).
template <typename R, bool QQ, bool DD, int K = 0>
static __global__ void __launch_bounds__(256) k_es_field(
    const double4* __restrict__ s, const double* __restrict__ q, const int* __restrict__ itype,
    const int* __restrict__ ipolar, const typename vec4t<R>::T* __restrict__ mu,
    const int* __restrict__ nbr, const int* __restrict__ nnb, int cap, int natm,
    const CellC* __restrict__ cell, const ESPair* __restrict__ tab, int ntype, double alpha,
    double cutsq, int damp, int dd_mask, double4* __restrict__ E, int thole = 0) {
  typedef typename vec4t<R>::T M4;
  __shared__ ESPair stab[MDFF_NT * MDFF_NT];
  __shared__ double cA[9];
  for (int k = threadIdx.x; k < ntype * ntype; k += blockDim.x) stab[k] = tab[k];
  if (threadIdx.x < 9) cA[threadIdx.x] = cell->A[threadIdx.x];
  __syncthreads();
  int lane = threadIdx.x & 31;
  int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (i >= natm) return;
  double4 si = s[i];
  int ti = itype[i];
  M4 mui;
  if (DD) mui = mu[i];
  bool dip_i = DD && (dd_mask ? (ipolar[i] != 0) : (mui.x != 0 || mui.y != 0 || mui.z != 0));
  int n = nnb[i];
  const int* row = nbr + (size_t)i * cap;
  R ex = R(0), ey = R(0), ez = R(0);
  const R rc2 = (R)cutsq;
  if (QQ || dip_i) {
    for (int k = lane; k < n; k += 32) {
      int j = row[k];
      // the partner's charge and dipole first: a pair with neither term
      // skips the minimum image (the non-polarisable partners of a dipole
      // field of the solver)
      M4 muj{};
      bool dd = false;
      if (DD && dip_i) {
        muj = mu[j];
        dd = dd_mask ? (ipolar[j] != 0) : (muj.x != 0 || muj.y != 0 || muj.z != 0);
      }
      double qj = QQ ? q[j] : 0.0;
      if (!dd && (!QQ || qj == 0.0)) continue;
      double4 sj = s[j];
      R rx, ry, rz;
      R r2 = pair_vec<R>(cA, si, sj, rx, ry, rz);
      if (r2 > rc2) continue;  // ewald_dir.f90:202 ( d2 .gt. cutsq ) cycle
      int tj = ((QQ && damp) || (DD && thole)) ? itype[j] : 0;
      es_field_pair<R, QQ, DD, K>(stab, ntype, i, j, ti, tj, rx, ry, rz, r2, (R)alpha, damp, qj, dd,
                               DD ? (R)muj.x : R(0), DD ? (R)muj.y : R(0), DD ? (R)muj.z : R(0),
                               ex, ey, ez, thole);
    }
  }
  double dx = warp_sum((double)ex), dy = warp_sum((double)ey), dz = warp_sum((double)ez);
  if (lane == 0) {
    double4 o = E[i];
    E[i] = make_double4(o.x + dx, o.y + dy, o.z + dz, 0.0);
  }
}

// --------------------------------------------------------------------------
// FP32 static pass with a pair cache.  Same damped charge field as
// k_es_field<float, true, false>, at the polarisable ions only (the dipole
// solvers read the static field there; other rows are left at zero), and in
// the same sweep the rows of the
// polarisable ions keep, for every polarisable partner within rc, the FP32
// terms of the undamped dipole field T2(r) mu = B2 r (r.mu) - B1 mu:
//   cr[i][m] = (rx, ry, rz, B2), cb1[i][m] = B1, cj[i][m] = j,  cn[i] = count
// (compacted with a warp ballot, row order kept).  The FP32 iterations of the
// dipole solve then read these instead of recomputing erfc / exp per pair
// (positions are fixed within a call).  K: compile-time Tang-Toennies order
// (0 = per pair).
//
// RES: the same pass merged with the dipole solve's first residual, for a
// first guess x0 that does not depend on the static field (the ASPC
// predictor): E also gets the undamped dipole field T2(r) x0_j of every
// polarisable partner (the induced field of x0, moment_from_pola.f90:401-404;
// ewald_dir.f90:566-571) from the cached FP32 terms, with FP64 products and
// sums, so that the residual sees the same pair tensor as the FP32 operator
// (k_dd_cached_rec) and the FP64 residuals after it (k_dd_cached64).  The
// charge field is the same code and order as without RES.
template <int K, bool RES = false>
static __global__ void __launch_bounds__(256) k_static_cache(
    const double4* __restrict__ s, const double* __restrict__ q, const int* __restrict__ itype,
    const int* __restrict__ ipolar, const int* __restrict__ nbr, const int* __restrict__ nnb,
    int cap, int natm, const CellC* __restrict__ cell, const ESPair* __restrict__ tab, int ntype,
    double alpha, double cutsq, int has_q, double4* __restrict__ E, float4* __restrict__ cr,
    float* __restrict__ cb1, int* __restrict__ cj, int* __restrict__ cn, int thole = 0,
    const double4* __restrict__ x0 = nullptr) {
  __shared__ ESPairF stab[MDFF_NT * MDFF_NT];
  __shared__ double cA[9];
  for (int k = threadIdx.x; k < ntype * ntype; k += blockDim.x) stab[k] = espair_f(tab[k]);
  if (threadIdx.x < 9) cA[threadIdx.x] = cell->A[threadIdx.x];
  __syncthreads();
  float A32[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) A32[k] = (float)cA[k];
  int lane = threadIdx.x & 31;
  int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (i >= natm) return;
  bool pol_i = ipolar[i] != 0;
  // the static field is wanted at the polarisable ions only (the dipole
  // solvers read it there); other rows keep E = 0 and an empty cache row
  if (!pol_i) {
    if (lane == 0) cn[i] = 0;
    return;
  }
  double4 si = s[i];
  int ti = itype[i];
  int n = nnb[i];
  const int* row = nbr + (size_t)i * cap;
  size_t cbase = (size_t)i * cap;
  float ex = 0.f, ey = 0.f, ez = 0.f;
  double tx = 0.0, ty = 0.0, tz = 0.0;  // RES: T2 x0
  const float rc2 = (float)cutsq;
  int m = 0;
  for (int k0 = 0; k0 < n; k0 += 32) {
    int k = k0 + lane;
    bool keep = false;
    float rx = 0.f, ry = 0.f, rz = 0.f, B1 = 0.f, B2 = 0.f;
    int j = 0;
    if (k < n) {
      j = row[k];
      double4 sj = s[j];
      float r2 = pair_vec_f(A32, si, sj, rx, ry, rz);
      if (r2 <= rc2) {  // ewald_dir.f90:202
        const float qj = has_q ? tag_q(sj.w) : 0.f;
        const bool pp = pol_i && tag_pol(sj.w);
        if (pp || qj != 0.f) {
          Radial<float> g;
          radial<float, false>(r2, (float)alpha, g);
          if (qj != 0.f) {
            float F1d = 0.f;
            const int tj = tag_type(sj.w);
            bool i_is_a = half_mask(i, j);
            int ta = i_is_a ? ti : tj, tb = i_is_a ? tj : ti;
            const ESPairF& P = stab[ta * ntype + tb];
            if (P.ldamp && (i_is_a ? P.ca : P.cb) != 0.f) {  // c = 0 damps nothing
              float fdm, fdd;
              if (i_is_a)
                tt_damp_k<float, K>(P.ba, P.ca, g.d, P.ka, fdm, fdd);
              else
                tt_damp_k<float, K>(P.bb, P.cb, g.d, P.kb, fdm, fdd);
              F1d = 1.f - fdm;
            }
            float c = qj * g.dm3 * (g.F1 - F1d);
            ex += c * rx;
            ey += c * ry;
            ez += c * rz;
          }
          if (pp) {
            keep = true;
            float F1 = g.F1, F2 = g.F2;
            if (thole) {
              const int tj = tag_type(sj.w);
              bool i_is_a = half_mask(i, j);
              const ESPairF& P = stab[(i_is_a ? ti : tj) * ntype + (i_is_a ? tj : ti)];
              if (P.thole) thole_radial<float, ESPairF>(P, g.d, F1, F2);
            }
            B1 = F1 * g.dm3;
            B2 = 3.f * F2 * g.dm5;
            if (RES) {
              const double4 xj = x0[j];
              const double drx = rx, dry = ry, drz = rz, dB1 = B1, dB2 = B2;
              const double rm = drx * xj.x + dry * xj.y + drz * xj.z;
              tx += dB2 * drx * rm - dB1 * xj.x;
              ty += dB2 * dry * rm - dB1 * xj.y;
              tz += dB2 * drz * rm - dB1 * xj.z;
            }
          }
        }
      }
    }
    unsigned bal = __ballot_sync(FULL_MASK, keep);
    if (keep) {
      int pos = m + __popc(bal & ((1u << lane) - 1u));
      cr[cbase + pos] = make_float4(rx, ry, rz, B2);
      cb1[cbase + pos] = B1;
      cj[cbase + pos] = j;
    }
    m += __popc(bal);
  }
  double dx = warp_sum((double)ex), dy = warp_sum((double)ey), dz = warp_sum((double)ez);
  if (RES) {
    dx += warp_sum(tx);
    dy += warp_sum(ty);
    dz += warp_sum(tz);
  }
  if (lane == 0) {
    double4 o = E[i];
    E[i] = make_double4(o.x + dx, o.y + dy, o.z + dz, 0.0);
    cn[i] = m;
  }
}

// this lane's part of the cached dipole field of row i: entries lane, lane +
// 32, ... in that order.  Four entries per lane are in flight at once (their
// cache words first, then the four dipole gathers), so the row costs a
// quarter of the dependent load round trips of a one-entry loop.
// (R = float: FP32 dipoles and sums; R = double: FP64 dipoles, the cached
// terms widened, FP64 products and sums)
template <typename R>
__device__ __forceinline__ void dd_cached_row(const typename vec4t<R>::T* __restrict__ mu,
                                              const float4* __restrict__ cr,
                                              const float* __restrict__ cb1,
                                              const int* __restrict__ cj, size_t base, int n,
                                              int lane, R& ex, R& ey, R& ez) {
  typedef typename vec4t<R>::T M4;
  constexpr int U = 4;
  for (int k0 = lane; k0 < n; k0 += 32 * U) {
    float4 r[U];
    float b1[U];
    int j[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int k = k0 + 32 * u;
      const bool ok = k < n;
      j[u] = ok ? cj[base + k] : 0;
      r[u] = ok ? cr[base + k] : make_float4(0.f, 0.f, 0.f, 0.f);
      b1[u] = ok ? cb1[base + k] : 0.f;
    }
    M4 m[U];
#pragma unroll
    for (int u = 0; u < U; ++u) m[u] = (k0 + 32 * u < n) ? mu[j[u]] : M4{};
#pragma unroll
    for (int u = 0; u < U; ++u) {
      if (k0 + 32 * u >= n) break;
      const R x = r[u].x, y = r[u].y, z = r[u].z, w = r[u].w, b = b1[u];
      R rm = x * m[u].x + y * m[u].y + z * m[u].z;
      ex += w * x * rm - b * m[u].x;
      ey += w * y * rm - b * m[u].y;
      ez += w * z * rm - b * m[u].z;
    }
  }
}

// the cached dipole field of every row as a warp-summed double4 (0 for rows
// without partners), for the CG operator to add in its final kernel: it runs
// on a side stream beside the reciprocal pass of the same operator
static __global__ void __launch_bounds__(256) k_dd_cached_part(
    const float4* __restrict__ mu, const float4* __restrict__ cr, const float* __restrict__ cb1,
    const int* __restrict__ cj, const int* __restrict__ cn, int cap, int natm,
    double4* __restrict__ Edd) {
  int lane = threadIdx.x & 31;
  int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (i >= natm) return;
  int n = cn[i];
  float ex = 0.f, ey = 0.f, ez = 0.f;
  dd_cached_row<float>(mu, cr, cb1, cj, (size_t)i * cap, n, lane, ex, ey, ez);
  double dx = warp_sum((double)ex), dy = warp_sum((double)ey), dz = warp_sum((double)ez);
  if (lane == 0) Edd[i] = make_double4(dx, dy, dz, 0.0);
}

// FP32 dipole field of mu (float4) from the pair cache of k_static_cache:
// E_i += sum_m T2(r_im) mu_j over the polarisable partners (k_es_field<float,
// false, true> with dd_mask = 1, without the per-pair radial functions)
static __global__ void __launch_bounds__(256) k_dd_cached(
    const float4* __restrict__ mu, const float4* __restrict__ cr, const float* __restrict__ cb1,
    const int* __restrict__ cj, const int* __restrict__ cn, int cap, int natm,
    double4* __restrict__ E) {
  int lane = threadIdx.x & 31;
  int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (i >= natm) return;
  int n = cn[i];
  if (n == 0) return;
  size_t base = (size_t)i * cap;
  float ex = 0.f, ey = 0.f, ez = 0.f;
  dd_cached_row<float>(mu, cr, cb1, cj, base, n, lane, ex, ey, ez);
  double dx = warp_sum((double)ex), dy = warp_sum((double)ey), dz = warp_sum((double)ez);
  if (lane == 0) {
    double4 o = E[i];
    E[i] = make_double4(o.x + dx, o.y + dy, o.z + dz, 0.0);
  }
}

// FP64 dipole field of mu (double4) from the same pair cache, FP64 products
// and sums: the real-space half of the mixed solver's FP64 residuals, which
// thus see the pair tensor of its FP32 operator
static __global__ void __launch_bounds__(256) k_dd_cached64(
    const double4* __restrict__ mu, const float4* __restrict__ cr, const float* __restrict__ cb1,
    const int* __restrict__ cj, const int* __restrict__ cn, int cap, int natm,
    double4* __restrict__ E) {
  int lane = threadIdx.x & 31;
  int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (i >= natm) return;
  int n = cn[i];
  if (n == 0) return;
  double ex = 0.0, ey = 0.0, ez = 0.0;
  dd_cached_row<double>(mu, cr, cb1, cj, (size_t)i * cap, n, lane, ex, ey, ez);
  ex = warp_sum(ex);
  ey = warp_sum(ey);
  ez = warp_sum(ez);
  if (lane == 0) {
    double4 o = E[i];
    E[i] = make_double4(o.x + ex, o.y + ey, o.z + ez, 0.0);
  }
}

// --------------------------------------------------------------------------
// final real-space pass: qq + qd + dd with damping; energy, field, force,
// (FP32: three blocks per SM, 80 registers, measured 14% faster than two)
// stress.  Partials per block: [u, tau xx yy zz xy xz yz] -> 7 doubles
// (tau is the reference's  - sum (r_j f_k + r_k f_j)  before *0.5/omega).
constexpr int kESPart = 7;

// one pair of the final real-space pass seen from ion i, r = r_i - r_j: the
// qq, qd and dd blocks of multipole_ES_dir (ewald_dir.f90:528-644) written in
// i's frame.  The reference's formulas are role-symmetric once the damping of
// the field on i (Di) and on j (Dj) are picked from its (ta,ta,tb) /
// (tb,ta,tb) tables by i's role (ewald_dir.f90:218-222):
//   f_i = q_i q_j B1 r + dd: -B3 (r.m_i)(r.m_j) r + B2 [(m_i.m_j) r + m_i (r.m_j) + m_j (r.m_i)]
//         + qd: q_i (T2 - T2d_j) m_j - q_j (T2 - T2d_i) m_i
//   E_i = q_j (B1 - B1d_i) r + dd: T2 m_j
//   u   = q_i q_j B0 + dd: -(m_i.T2.m_j) + qd: q_i (B1 - B1d_j)(r.m_j) - q_j (B1 - B1d_i)(r.m_i)
// (f_i = the reference's -f_ij when i is "ia", +f_ij when i is "ja").  Only
// i's field is formed.  K: compile-time Tang-Toennies order (0 = per pair).
template <typename R, int K, bool THOLE, typename PT = ESPair>
__device__ __forceinline__ void es_force_ipair(const PT& P, bool i_is_a, bool ldamp, R d2,
                                               R alpha, const R (&r)[3], R qi, R qj,
                                               const R (&mi)[3], const R (&mj)[3], bool dip_i,
                                               bool dip_j, int task_qq, int task_qd, int task_dd,
                                               R& u, R (&fi)[3], R (&Ei)[3]) {
  Radial<R> g;
  radial<R, true>(d2, alpha, g);
  const R B0 = g.dm1 * g.F0, B1 = g.F1 * g.dm3, B2 = R(3) * g.F2 * g.dm5;
  R C1i = B1, C2i = B2, C1j = B1, C2j = B2;  // B - B_damped for the field on i / on j
  if (ldamp) {
    // a role with c = 0 damps nothing (f = 1, fd = 0 at any order): skipped
    // (the field on a non-polarisable ion, warp-uniform for its rows)
    const R ci = (R)(i_is_a ? P.ca : P.cb), cj = (R)(i_is_a ? P.cb : P.ca);
    R fdm, fdd;
    if (ci != R(0)) {
      tt_damp_k<R, K>((R)(i_is_a ? P.ba : P.bb), ci, g.d, i_is_a ? P.ka : P.kb, fdm, fdd);
      const R F1d = R(1) - fdm;
      C1i = B1 - F1d * g.dm3;
      C2i = B2 - R(3) * (F1d + (g.d / R(3)) * fdd) * g.dm5;
    }
    if (cj != R(0)) {
      tt_damp_k<R, K>((R)(i_is_a ? P.bb : P.ba), cj, g.d, i_is_a ? P.kb : P.ka, fdm, fdd);
      const R F1d = R(1) - fdm;
      C1j = B1 - F1d * g.dm3;
      C2j = B2 - R(3) * (F1d + (g.d / R(3)) * fdd) * g.dm5;
    }
  }
  const R rmi = r[0] * mi[0] + r[1] * mi[1] + r[2] * mi[2];
  const R rmj = r[0] * mj[0] + r[1] * mj[1] + r[2] * mj[2];
  u = R(0);
  R fr = R(0);  // coefficient of r in f_i
  R fmi = R(0), fmj = R(0);  // coefficients of m_i and m_j in f_i
  R er = R(0), emj = R(0);   // E_i = er r + emj m_j
  if (task_qq) {
    u += qi * qj * B0;
    fr += qi * qj * B1;
    er += qj * C1i;
  }
  if (task_dd && dip_i && dip_j) {
    R B1t = B1, B2t = B2;
    if (THOLE && P.thole) {
      R F1t = g.F1, F2t = g.F2;
      thole_radial<R, PT>(P, g.d, F1t, F2t);
      B1t = F1t * g.dm3;
      B2t = R(3) * F2t * g.dm5;
    }
    const R B3 = R(15) * g.F3 * g.dm7;
    const R mij = mi[0] * mj[0] + mi[1] * mj[1] + mi[2] * mj[2];
    u -= B2t * rmi * rmj - B1t * mij;
    er += B2t * rmj;
    emj -= B1t;
    fr += B2 * mij - B3 * rmi * rmj;
    fmi += B2 * rmj;
    fmj += B2 * rmi;
  }
  if (task_qd && (dip_i || dip_j)) {
    u += qi * C1j * rmj - qj * C1i * rmi;
    fr += qi * C2j * rmj - qj * C2i * rmi;
    fmj -= qi * C1j;
    fmi += qj * C1i;
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    fi[c] = fr * r[c] + fmi * mi[c] + fmj * mj[c];
    Ei[c] = er * r[c] + emj * mj[c];
  }
}

// per-ion charge and dipole of the final pass: FP64 from q[] and the double4
// dipoles, FP32 from one float4 (mu_x, mu_y, mu_z, q) written by k_mu_total
template <typename R>
__device__ __forceinline__ void load_qm(const double* q, const double4* mu, const float4* qm32,
                                        int j, R& qj, R (&mj)[3]);
template <>
__device__ __forceinline__ void load_qm<double>(const double* q, const double4* mu, const float4*,
                                                int j, double& qj, double (&mj)[3]) {
  double4 m = mu[j];
  qj = q[j];
  mj[0] = m.x;
  mj[1] = m.y;
  mj[2] = m.z;
}
template <>
__device__ __forceinline__ void load_qm<float>(const double*, const double4*, const float4* qm32,
                                               int j, float& qj, float (&mj)[3]) {
  float4 m = qm32[j];
  qj = m.w;
  mj[0] = m.x;
  mj[1] = m.y;
  mj[2] = m.z;
}

// final real-space pass, warp per ion over the full list; each visit of a
// pair adds i's force and field and half the pair's energy and stress.
// A lane sums its visits in R (FP32 in the mixed engine: about nine visits
// per lane on the 12k glass, so no FP64 conversion and add per visit) and the
// lanes' sums are widened to FP64 for the warp and block reductions.
template <typename R>
__device__ __forceinline__ R pvec(const double* A, const float (&A32)[9], double4 si, double4 sj,
                                  R (&r)[3]);
template <>
__device__ __forceinline__ double pvec<double>(const double* A, const float (&)[9], double4 si,
                                               double4 sj, double (&r)[3]) {
  return pair_vec<double>(A, si, sj, r[0], r[1], r[2]);
}
template <>
__device__ __forceinline__ float pvec<float>(const double*, const float (&A32)[9], double4 si,
                                             double4 sj, float (&r)[3]) {
  return pair_vec_f(A32, si, sj, r[0], r[1], r[2]);
}

template <typename R, int K, bool THOLE>
static __global__ void __launch_bounds__(256, sizeof(R) == 4 ? 4 : 2) k_es_force(
    const double4* __restrict__ s, const double* __restrict__ q, const int* __restrict__ itype,
    const double4* __restrict__ mu, const float4* __restrict__ qm32, const int* __restrict__ nbr,
    const int* __restrict__ nnb, int cap, int natm, const CellC* __restrict__ cell,
    const ESPair* __restrict__ tab, int ntype, double alpha, double cutsq, int task_qq,
    int task_qd, int task_dd, int damp_ind, double fscale, double4* __restrict__ E,
    double* __restrict__ force /* SoA [3][natm], += */, double* __restrict__ part) {
  typedef typename espair_t<R>::T PT;
  __shared__ PT stab[MDFF_NT * MDFF_NT];
  __shared__ double cA[9];
  __shared__ double red[kESPart * 8];
  for (int k = threadIdx.x; k < ntype * ntype; k += blockDim.x) stab[k] = espair_as<PT>(tab[k]);
  if (threadIdx.x < 9) cA[threadIdx.x] = cell->A[threadIdx.x];
  __syncthreads();
  float A32[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) A32[k] = (float)cA[k];
  int lane = threadIdx.x & 31;
  int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  double acc[kESPart];
#pragma unroll
  for (int k = 0; k < kESPart; ++k) acc[k] = 0.0;
  if (i < natm) {
    const double4 si = s[i];
    const int ti = itype[i];
    R qi, mi[3];
    load_qm<R>(q, mu, qm32, i, qi, mi);
    const bool dip_i = mi[0] != R(0) || mi[1] != R(0) || mi[2] != R(0);
    const int n = nnb[i];
    const int* row = nbr + (size_t)i * cap;
    const R rc2 = (R)cutsq, ra = (R)alpha;
    R e[3] = {0, 0, 0}, f[3] = {0, 0, 0};
    R la[kESPart];
#pragma unroll
    for (int k = 0; k < kESPart; ++k) la[k] = R(0);
    for (int k = lane; k < n; k += 32) {
      const int j = row[k];
      const double4 sj = s[j];
      R r[3];
      const R r2 = pvec<R>(cA, A32, si, sj, r);
      if (r2 > rc2) continue;  // ewald_dir.f90:202 ( d2 .gt. cutsq ) cycle
      R qj, mj[3];
      load_qm<R>(q, mu, qm32, j, qj, mj);
      const bool dip_j = mj[0] != R(0) || mj[1] != R(0) || mj[2] != R(0);
      const int tj = tag_type(sj.w);
      const bool i_is_a = half_mask(i, j);
      const PT& P = stab[(i_is_a ? ti : tj) * ntype + (i_is_a ? tj : ti)];
      R u, fi[3], Ei[3];
      es_force_ipair<R, K, THOLE, PT>(P, i_is_a, damp_ind && P.ldamp, r2, ra, r, qi, qj, mi, mj,
                                      dip_i, dip_j, task_qq, task_qd, task_dd, u, fi, Ei);
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        f[c] += fi[c];
        e[c] += Ei[c];
      }
      la[0] += u;
      la[1] += r[0] * fi[0];
      la[2] += r[1] * fi[1];
      la[3] += r[2] * fi[2];
      la[4] += r[0] * fi[1] + r[1] * fi[0];
      la[5] += r[0] * fi[2] + r[2] * fi[0];
      la[6] += r[1] * fi[2] + r[2] * fi[1];
    }
    // halves of the pair energy and of the off-diagonal stress sums
    acc[0] = 0.5 * (double)la[0];
#pragma unroll
    for (int k = 1; k < 4; ++k) acc[k] = (double)la[k];
#pragma unroll
    for (int k = 4; k < kESPart; ++k) acc[k] = 0.5 * (double)la[k];
    double ed[3], fd[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      ed[c] = warp_sum((double)e[c]);
      fd[c] = warp_sum((double)f[c]);
    }
    if (lane == 0) {
      double4 o = E[i];
      E[i] = make_double4(o.x + ed[0], o.y + ed[1], o.z + ed[2], 0.0);
      force[i] += fd[0] * fscale;
      force[natm + i] += fd[1] * fscale;
      force[2 * natm + i] += fd[2] * fscale;
    }
  }
  block_sum<kESPart>(acc, red);
  if (threadIdx.x == 0)
    for (int k = 0; k < kESPart; ++k) part[(size_t)blockIdx.x * kESPart + k] = acc[k];
}

// --------------------------------------------------------------------------
// real-space electric field gradient (multipole_ES_dir with do_efg,
// ewald_dir.f90:543-545, 577-582), FP64, full list, warp per ion:
//   efg_i -= q_j T2(r_ij)            (charges; undamped)
//   efg_i += T3(r_ij) . mu_j         (both dipoles non-zero)
// T2 and T3 are even / odd in r, so the reference's ia / ja updates are the
// same expression from either side.  Out: efg[i][9] (overwritten).
static __global__ void __launch_bounds__(256) k_es_efg(
    const double4* __restrict__ s, const double* __restrict__ q, const double4* __restrict__ mu,
    const int* __restrict__ nbr, const int* __restrict__ nnb, int cap, int natm,
    const CellC* __restrict__ cell, double alpha, double cutsq, int task_qq, int task_dd,
    double* __restrict__ efg) {
  int lane = threadIdx.x & 31;
  int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (i >= natm) return;
  double4 si = s[i];
  double4 mi = mu[i];
  bool dip_i = mi.x != 0.0 || mi.y != 0.0 || mi.z != 0.0;
  int n = nnb[i];
  const int* row = nbr + (size_t)i * cap;
  double e[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) e[k] = 0.0;
  for (int k = lane; k < n; k += 32) {
    int j = row[k];
    double4 sj = s[j];
    double r[3];
    double r2 = min_image_exact(cell->A, xsub(si.x, sj.x), xsub(si.y, sj.y), xsub(si.z, sj.z),
                                r[0], r[1], r[2]);
    if (r2 > cutsq) continue;
    Radial<double> g;
    radial<double, true>(r2, alpha, g);
    double F2 = 3.0 * g.F2 * g.dm5, F1 = g.F1 * g.dm3, F3 = 15.0 * g.F3 * g.dm7;
    if (task_qq) {
      double qj = q[j];
#pragma unroll
      for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b) e[3 * a + b] -= qj * (r[a] * r[b] * F2 - (a == b ? F1 : 0.0));
    }
    double4 mj = mu[j];
    if (task_dd && dip_i && (mj.x != 0.0 || mj.y != 0.0 || mj.z != 0.0)) {
      double m[3] = {mj.x, mj.y, mj.z};
      double rm = r[0] * m[0] + r[1] * m[1] + r[2] * m[2];
#pragma unroll
      for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b)
          e[3 * a + b] += -r[a] * r[b] * rm * F3 +
                          F2 * ((a == b ? rm : 0.0) + r[b] * m[a] + r[a] * m[b]);
    }
  }
#pragma unroll
  for (int k = 0; k < 9; ++k) e[k] = warp_sum(e[k]);
  if (lane == 0)
    for (int k = 0; k < 9; ++k) efg[9 * (size_t)i + k] = e[k];
}

// fixed-order reduction of per-block partials: out[v] = sum_b part[b*nv+v];
// one block per value (grid = nv), the same order for every launch
static __global__ void k_reduce_partials(const double* __restrict__ part, int nblk, int nv,
                                         double* __restrict__ out) {
  pdl_wait();
  pdl_trigger();
  __shared__ double sh[256];
  const int v = blockIdx.x;
  double acc = 0.0;
  for (int b = threadIdx.x; b < nblk; b += blockDim.x) acc += part[(size_t)b * nv + v];
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int w = blockDim.x >> 1; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[v] = sh[0];
}

}  // namespace mdff
