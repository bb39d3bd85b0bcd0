// pim.cuh -- induced-dipole (PIM) solve and the self / surface terms.
//
//  * SCF: moment_from_pola_scf (moment_from_pola.f90:240-485) step by step:
//    induced_moment (:955-993), ASPC predictor/corrector (:493-598),
//    u_pol (:387-395), get_rmsd_mu (:998-1027).
//  * CG:  preconditioned conjugate gradients on (alpha^-1 - T) mu = E_stat,
//    the linear system whose fixed point the SCF iterates to; preconditioner
//    alpha; stop on the reference's rmsd measure (for diagonal alpha the CG
//    residual E - alpha^-1 mu is exactly (mu/alpha_aa - E) up to sign).
//  * self and surface field terms of multipole_ES (ewald.f90:182-213).
// Vectors are double4 [natm] (xyz + pad).  Reductions are per-block partials
// summed in a fixed order (deterministic).
#pragma once
#include "common.cuh"

namespace mdff {

struct PolDev {
  const double* pol;     // [natm][9] poldipia (row-major a,b)
  const double* invpol;  // [natm][9]
  const int* ipolar;     // [natm]
};

__device__ __forceinline__ double4 matvec3(const double* m, double4 v) {
  return make_double4(m[0] * v.x + m[1] * v.y + m[2] * v.z, m[3] * v.x + m[4] * v.y + m[5] * v.z,
                      m[6] * v.x + m[7] * v.y + m[8] * v.z, 0.0);
}

// mu_i = alpha_i E_i on polarisable ions, 0 elsewhere (induced_moment)
__global__ void k_induce(const double4* __restrict__ E, PolDev P, int natm, double4* __restrict__ mu) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= natm) return;
  const double* a = P.pol + 9 * (size_t)i;
  mu[i] = P.ipolar[i] ? make_double4(((a[0] * E[i].x) + a[1] * E[i].y) + a[2] * E[i].z,
                                     ((a[3] * E[i].x) + a[4] * E[i].y) + a[5] * E[i].z,
                                     ((a[6] * E[i].x) + a[7] * E[i].y) + a[8] * E[i].z, 0.0)
                      : make_double4(0, 0, 0, 0);
}

// ASPC predictor: mu = sum_k B_k hist[k]; hist[k] = hist[k-1] for k = ord..1
__global__ void k_aspc_predict(double4* __restrict__ hist, int natm, int ord, double b0, double b1,
                               double b2, double b3, double b4, double4* __restrict__ mu) {
  pdl_wait();
  pdl_trigger();
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= natm) return;
  double B[5] = {b0, b1, b2, b3, b4};
  double4 s = make_double4(0, 0, 0, 0);
  for (int k = 0; k <= ord; ++k) {
    double4 h = hist[(size_t)k * natm + i];
    s.x = s.x + B[k] * h.x;
    s.y = s.y + B[k] * h.y;
    s.z = s.z + B[k] * h.z;
  }
  mu[i] = s;
  for (int k = ord; k >= 1; --k) hist[(size_t)k * natm + i] = hist[(size_t)(k - 1) * natm + i];
}

// ASPC corrector: mu = w alpha E + (1 - w) mu
__global__ void k_aspc_correct(const double4* __restrict__ E, PolDev P, int natm, double wgt,
                               double4* __restrict__ mu) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= natm) return;
  double4 m = make_double4(0, 0, 0, 0);
  if (P.ipolar[i]) m = matvec3(P.pol + 9 * (size_t)i, E[i]);
  double4 o = mu[i];
  mu[i] = make_double4(wgt * m.x + (1.0 - wgt) * o.x, wgt * m.y + (1.0 - wgt) * o.y,
                       wgt * m.z + (1.0 - wgt) * o.z, 0.0);
}

// partials of u_pol = 1/2 sum mu alpha^-1 mu  (slot 0)
__global__ void k_upol_part(const double4* __restrict__ mu, PolDev P, int natm,
                            double* __restrict__ part) {
  pdl_wait();
  pdl_trigger();
  __shared__ double red[32];
  double v[1] = {0.0};
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < natm && P.ipolar[i]) {
    const double* a = P.invpol + 9 * (size_t)i;
    double m[3] = {mu[i].x, mu[i].y, mu[i].z};
    for (int x = 0; x < 3; ++x)
      for (int y = 0; y < 3; ++y) v[0] += m[x] * a[3 * x + y] * m[y];
  }
  block_sum<1>(v, red);
  if (threadIdx.x == 0) part[blockIdx.x] = v[0];
}

// partials of get_rmsd_mu: sum over polarisable ions, components with
// alpha_aa /= 0, of (mu_a/alpha_aa - E_a)^2.  Slot 0 of each block.
__global__ void k_rmsd_part(const double4* __restrict__ mu, const double4* __restrict__ E, PolDev P,
                            int natm, double* __restrict__ part) {
  __shared__ double red[32];
  double v[1] = {0.0};
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < natm && P.ipolar[i]) {
    const double* a = P.pol + 9 * (size_t)i;
    double m[3] = {mu[i].x, mu[i].y, mu[i].z}, e[3] = {E[i].x, E[i].y, E[i].z};
    for (int x = 0; x < 3; ++x) {
      double al = a[4 * x];
      if (al == 0.0) continue;
      double d = m[x] / al - e[x];
      v[0] += d * d;
    }
  }
  block_sum<1>(v, red);
  if (threadIdx.x == 0) part[blockIdx.x] = v[0];
}

// out = a + b
__global__ void k_add4(const double4* __restrict__ a, const double4* __restrict__ b, int n,
                       double4* __restrict__ out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  out[i] = make_double4(a[i].x + b[i].x, a[i].y + b[i].y, a[i].z + b[i].z, 0.0);
}

// moments for self / surface terms: partial sums of
// [qtot(3) = sum q r, mutot(3), qsq, musq]
__global__ void k_moments_part(const double* __restrict__ pos, const double* __restrict__ q,
                               const double4* __restrict__ mu, int natm, int has_q,
                               double* __restrict__ part) {
  pdl_wait();
  pdl_trigger();
  __shared__ double red[8 * 32];
  double v[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < natm) {
    double qi = has_q ? q[i] : 0.0;
    double4 m = mu ? mu[i] : make_double4(0, 0, 0, 0);
    v[0] = qi * pos[i];
    v[1] = qi * pos[natm + i];
    v[2] = qi * pos[2 * natm + i];
    v[3] = m.x;
    v[4] = m.y;
    v[5] = m.z;
    v[6] = qi * qi;
    v[7] = m.x * m.x + m.y * m.y + m.z * m.z;
  }
  block_sum<8>(v, red);
  if (threadIdx.x == 0)
    for (int k = 0; k < 8; ++k) part[(size_t)blockIdx.x * 8 + k] = v[k];
}

// E += 2 selfa2 mu  (+ surface  -fpi_3V (qtot + mutot)  when lsurf);
// mom = reduced [qtot(3), mutot(3), qsq, musq]
__global__ void k_self_surf_field(const double4* __restrict__ mu, int natm, double selfa2,
                                  int lsurf, double fpi_3V, const double* __restrict__ mom,
                                  double4* __restrict__ E) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= natm) return;
  double4 m = mu ? mu[i] : make_double4(0, 0, 0, 0);
  double4 o = E[i];
  double s0 = 0.0, s1 = 0.0, s2 = 0.0;
  if (lsurf) {
    s0 = -(mom[0] + mom[3]) * fpi_3V;
    s1 = -(mom[1] + mom[4]) * fpi_3V;
    s2 = -(mom[2] + mom[5]) * fpi_3V;
  }
  E[i] = make_double4(o.x + s0 + 2.0 * selfa2 * m.x, o.y + s1 + 2.0 * selfa2 * m.y,
                      o.z + s2 + 2.0 * selfa2 * m.z, 0.0);
}

// ---- conjugate gradients ----------------------------------------------------
// A x = alpha^-1 x - T x on polarisable ions (T x = field of x).  The step
// scalars (r.z, p.q) stay on the device; only the rmsd goes to the host.

// r = b + Tx - alpha^-1 x ; z = alpha r ; p = z ; partial r.z and rmsd
// FP32 operands of the next operator application of the direction p (when w32
// is given): w32 = (0, m), m = 2 pi B^T p, mu32 = p, as k_rec_weights writes them
// (and w32 again at the ion's slot in w32s, when the ion has one)
__device__ __forceinline__ void cg_dir_weights(const CellC* __restrict__ cell, double4 u, int i,
                                               float4* __restrict__ w32, float4* __restrict__ mu32,
                                               const SlotW& sw) {
  const double* B = cell->B;
  double m1 = kTwoPi * (B[0] * u.x + B[3] * u.y + B[6] * u.z);
  double m2 = kTwoPi * (B[1] * u.x + B[4] * u.y + B[7] * u.z);
  double m3 = kTwoPi * (B[2] * u.x + B[5] * u.y + B[8] * u.z);
  const float4 wv = make_float4(0.f, (float)m1, (float)m2, (float)m3);
  w32[i] = wv;
  mu32[i] = make_float4((float)u.x, (float)u.y, (float)u.z, 0.f);
  sw.put(i, wv);
}

__global__ void k_cg_init(const double4* __restrict__ b, const double4* __restrict__ Tx,
                          const double4* __restrict__ x, PolDev P, int natm, double4* __restrict__ r,
                          double4* __restrict__ z, double4* __restrict__ p, double* __restrict__ part,
                          const CellC* __restrict__ cell, float4* __restrict__ w32,
                          float4* __restrict__ mu32, SlotW sw) {
  pdl_wait();
  pdl_trigger();
  __shared__ double red[2 * 32];
  double v[2] = {0.0, 0.0};
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < natm) {
    double4 ri = make_double4(0, 0, 0, 0), zi = make_double4(0, 0, 0, 0);
    if (P.ipolar[i]) {
      double4 ax = matvec3(P.invpol + 9 * (size_t)i, x[i]);
      // b = nullptr: Tx already holds b + T x (the merged static pass)
      const double4 bi = b ? b[i] : make_double4(0.0, 0.0, 0.0, 0.0);
      ri = make_double4(bi.x + Tx[i].x - ax.x, bi.y + Tx[i].y - ax.y, bi.z + Tx[i].z - ax.z, 0);
      zi = matvec3(P.pol + 9 * (size_t)i, ri);
      const double* a = P.pol + 9 * (size_t)i;
      double rr[3] = {ri.x, ri.y, ri.z};
      for (int c = 0; c < 3; ++c)
        if (a[4 * c] != 0.0) v[1] += rr[c] * rr[c];
    }
    r[i] = ri;
    z[i] = zi;
    p[i] = zi;
    if (w32) cg_dir_weights(cell, zi, i, w32, mu32, sw);
    v[0] = ri.x * zi.x + ri.y * zi.y + ri.z * zi.z;
  }
  block_sum<2>(v, red);
  if (threadIdx.x == 0) {
    part[(size_t)blockIdx.x * 2] = v[0];
    part[(size_t)blockIdx.x * 2 + 1] = v[1];
  }
}

// q = alpha^-1 p - Tp (polarisable ions); partial p.q
__global__ void k_cg_Ap(const double4* __restrict__ p, const double4* __restrict__ Tp, PolDev P,
                        int natm, double4* __restrict__ qv, double* __restrict__ part) {
  pdl_wait();
  pdl_trigger();
  __shared__ double red[32];
  double v[1] = {0.0};
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < natm) {
    double4 qi = make_double4(0, 0, 0, 0);
    if (P.ipolar[i]) {
      double4 ap = matvec3(P.invpol + 9 * (size_t)i, p[i]);
      qi = make_double4(ap.x - Tp[i].x, ap.y - Tp[i].y, ap.z - Tp[i].z, 0);
    }
    qv[i] = qi;
    v[0] = p[i].x * qi.x + p[i].y * qi.y + p[i].z * qi.z;
  }
  block_sum<1>(v, red);
  if (threadIdx.x == 0) part[blockIdx.x] = v[0];
}

// al = rz / pq ; x += al p ; r -= al q ; z = alpha_pol r ;
// partial r.z (new) and rmsd^2
// (acc: the structure factor is linear in the dipoles, so acc += al rho'(p)
// with rho'(p) = rhoA of this step's operator keeps acc = rho' of the charges
// and the current x; nk k vectors, grid-stride)
__global__ void k_cg_update(const double* __restrict__ rz_p, const double* __restrict__ pq_p,
                            PolDev P, int natm, const double4* __restrict__ p,
                            const double4* __restrict__ qv, double4* __restrict__ x,
                            double4* __restrict__ r, double4* __restrict__ z,
                            double* __restrict__ part, double2* __restrict__ acc = nullptr,
                            const double2* __restrict__ rhoA = nullptr, int nk = 0) {
  pdl_wait();
  pdl_trigger();
  __shared__ double red[2 * 32];
  double v[2] = {0.0, 0.0};
  double rz = *rz_p, pq = *pq_p;
  double al = (pq != 0.0) ? rz / pq : 0.0;
  if (acc)
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nk; k += gridDim.x * blockDim.x) {
      const double2 a = acc[k], d = rhoA[k];
      acc[k] = make_double2(a.x + al * d.x, a.y + al * d.y);
    }
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < natm && P.ipolar[i]) {
    double4 xi = x[i], ri = r[i], pi = p[i], qi = qv[i];
    xi.x += al * pi.x;
    xi.y += al * pi.y;
    xi.z += al * pi.z;
    ri.x -= al * qi.x;
    ri.y -= al * qi.y;
    ri.z -= al * qi.z;
    double4 zi = matvec3(P.pol + 9 * (size_t)i, ri);
    x[i] = xi;
    r[i] = ri;
    z[i] = zi;
    v[0] = ri.x * zi.x + ri.y * zi.y + ri.z * zi.z;
    const double* a = P.pol + 9 * (size_t)i;
    double rr[3] = {ri.x, ri.y, ri.z};
    for (int c = 0; c < 3; ++c)
      if (a[4 * c] != 0.0) v[1] += rr[c] * rr[c];
  }
  block_sum<2>(v, red);
  if (threadIdx.x == 0) {
    part[(size_t)blockIdx.x * 2] = v[0];
    part[(size_t)blockIdx.x * 2 + 1] = v[1];
  }
}

// p = z + beta p with beta = rz_new / rz
__global__ void k_cg_dir(const double* __restrict__ rz_p, const double* __restrict__ rzn_p,
                         int natm, const double4* __restrict__ z, double4* __restrict__ p,
                         const CellC* __restrict__ cell, float4* __restrict__ w32,
                         float4* __restrict__ mu32, SlotW sw) {
  pdl_wait();
  pdl_trigger();
  double rz = *rz_p, rzn = *rzn_p;
  double be = (rz != 0.0) ? rzn / rz : 0.0;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < natm) {
    double4 pi = p[i], zi = z[i];
    double4 pn = make_double4(zi.x + be * pi.x, zi.y + be * pi.y, zi.z + be * pi.z, 0.0);
    p[i] = pn;
    if (w32) cg_dir_weights(cell, pn, i, w32, mu32, sw);
  }
}

__global__ void k_copy1(double* __restrict__ dst, const double* __restrict__ src) {
  if (threadIdx.x == 0 && blockIdx.x == 0) *dst = *src;
}

// moment_from_WFc (moment_from_pola.f90:632-807), warp per ion over its
// (full, ascending) neighbour row: every ion of a type with lwfc >= 0 sums
// r_j - r_i (minimum image, the reference's two-rounding arithmetic) over
// the Wannier centres j (lwfc < 0) with |r_ij|^2 < rcut_wfc, in ascending j as
// the reference does; mu_wfc = -2 sum.  An ion of a type with lwfc > 0 that
// finds a different number of centres sets *bad (the reference STOPs).
__global__ void k_wfc_dipoles(const double4* __restrict__ s, const int* __restrict__ itype,
                              const int* __restrict__ lwfc, const int* __restrict__ nbr,
                              const int* __restrict__ nnb, int cap, int natm,
                              const CellC* __restrict__ cell, double rcut_wfc,
                              double4* __restrict__ mu_wfc, int* __restrict__ bad) {
  int lane = threadIdx.x & 31;
  int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (i >= natm) return;
  const int lw = lwfc[itype[i]];
  if (lw < 0) {
    if (lane == 0) mu_wfc[i] = make_double4(0, 0, 0, 0);
    return;
  }
  const double4 si = s[i];
  const int n = nnb[i];
  double ax = 0.0, ay = 0.0, az = 0.0;
  int cnt = 0;
  for (int k0 = 0; k0 < n; k0 += 32) {
    int k = k0 + lane;
    bool hit = false;
    double rx = 0.0, ry = 0.0, rz = 0.0;
    if (k < n) {
      int j = nbr[(size_t)i * cap + k];
      if (lwfc[itype[j]] < 0) {
        double4 sj = s[j];
        double r2 = min_image_exact(cell->A, xsub(sj.x, si.x), xsub(sj.y, si.y), xsub(sj.z, si.z), rx, ry, rz);
        hit = r2 < rcut_wfc;
      }
    }
    unsigned m = __ballot_sync(FULL_MASK, hit);
    while (m) {  // in ascending neighbour order
      int l = __ffs(m) - 1;
      m &= m - 1;
      double x = __shfl_sync(FULL_MASK, rx, l), y = __shfl_sync(FULL_MASK, ry, l),
             z = __shfl_sync(FULL_MASK, rz, l);
      ax = ax + x;
      ay = ay + y;
      az = az + z;
      cnt++;
    }
  }
  if (lane == 0) {
    mu_wfc[i] = make_double4(-2.0 * ax, -2.0 * ay, -2.0 * az, 0.0);
    if (lw > 0 && cnt != lw) atomicExch(bad, 1);
  }
}

// mu_tot = (dipia + mu_ind) [+ mu_wfc] ; catastrophe flag if any component > 10
// (moment_from_pola.f90:136-147, 176-178: positive components only)
// qm32 (optional): (mu_x, mu_y, mu_z, q) in FP32 for the mixed final pass
__global__ void k_mu_total(const double4* __restrict__ dip, const double4* __restrict__ mu_ind,
                           const double4* __restrict__ mu_wfc, int natm, double4* __restrict__ mu_tot,
                           int* __restrict__ flag, const double* __restrict__ q = nullptr,
                           float4* __restrict__ qm32 = nullptr) {
  pdl_wait();
  pdl_trigger();
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= natm) return;
  double4 a = dip[i], b = mu_ind[i];
  double4 m = make_double4(a.x + b.x, a.y + b.y, a.z + b.z, 0.0);
  if (mu_wfc) {
    double4 w = mu_wfc[i];
    m = make_double4(m.x + w.x, m.y + w.y, m.z + w.z, 0.0);
  }
  mu_tot[i] = m;
  if (qm32) qm32[i] = make_float4((float)m.x, (float)m.y, (float)m.z, (float)q[i]);
  if (m.x > 10.0 || m.y > 10.0 || m.z > 10.0) atomicExch(flag, 1);
}

}  // namespace mdff
