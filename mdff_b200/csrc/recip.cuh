// recip.cuh -- Ewald reciprocal-space sum (multipole_ES_rec, ewald_rec.f90:38-365).
//
// The reference evaluates COS/SIN(k.r) afresh for every (k, ion) pair of the
// half-space mesh (kspace.f90:143-207).  Here k = 2 pi B n, so
//   e^{i k.r} = X_nx(s_x) Y_ny(s_y) Z_nz(s_z),  X_n = e^{2 pi i n s_x}, ...
// with s the direct coordinates.  Per-ion tables of X, Y, Z (one sincospi
// each, FP64) are built once per pass; the mesh is walked as rows (nx, ny)
// of consecutive nz, where the phase advances by one complex multiply.
// Likewise k.mu = n . m with m = 2 pi B^T mu, and sum_k k f(k) = 2 pi B sum_k n f(k).
//
//   k_rec_rho   : rho(k) = sum_i (q_i + i k.mu_i) e^{i k.r_i}   (ewald_rec.f90:118-148)
//                 block = (row, nz tile) x ion chunk; fixed-order partials.
//   k_rec_sum   : rho over chunks; rho' = A_k rho; str = A_k |rho|^2 (:173)
//   k_rec_energy: u_rec and the stress (:255-263, 300-358), one block, fixed order
//   k_rec_field : per ion sum over k of recarg / recarg2 (:181-250), ion-major,
//                 rho' of the block's k chunk staged in shared memory
//   k_rec_field_sum : chunk sum, E = -2 pi B G, F = q E + 2 pi B H, scaled
#pragma once
#include "common.cuh"
#include "realspace.cuh"

namespace mdff {

template <typename R>
struct cplx;
template <>
struct cplx<double> {
  typedef double2 T;
};
template <>
struct cplx<float> {
  typedef float2 T;
};

// self field 2 selfa2 mu_i (+ the surface field -fpi_3V (qtot + mutot) of the
// reduced moments mom[0..5] when lsurf), added to E by k_rec_field_sum when on;
// the same sums as k_self_surf_field
struct SelfField {
  int on, lsurf;
  const double4* mu;
  double selfa2, fpi_3V;
  const double* mom;
};

struct RecMesh {
  int kmax[3];
  int nrows;
  const int4* rows;      // (nx, ny, nz_lo, koff)
  int nk;
  const double* Ak;      // [nk] in row order
  const double4* kvec;   // [nk] (kx, ky, kz, kcoe)
};

// per-ion phase tables: [n][natm], X: n = 0..kx, Y: 0..ky, Z: 0..max(kz, 4).
// s is wrapped to [-0.5, 0.5) first: e^{2 pi i n s} is periodic in s.
template <typename R>
static __global__ void k_rec_tables(const double4* __restrict__ s, int natm, int kx, int ky, int kz,
                             typename cplx<R>::T* __restrict__ tab) {
  pdl_wait();
  pdl_trigger();
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= natm) return;
  double sv[3] = {s[i].x, s[i].y, s[i].z};
  int km[3] = {kx, ky, kz};
  int off = 0;
  for (int a = 0; a < 3; ++a) {
    double w = sv[a] - rint(sv[a]);
    for (int n = 0; n <= km[a]; ++n) {
      double sn, cs;
      sincospi(2.0 * (double)n * w, &sn, &cs);
      typename cplx<R>::T v;
      v.x = (R)cs;
      v.y = (R)sn;
      tab[(size_t)(off + n) * natm + i] = v;
    }
    off += km[a] + 1;
  }
}

// per-ion weights (q, m1, m2, m3), m = 2 pi B^T mu  (k.mu = n.m)
static __global__ void k_rec_weights(const double* __restrict__ q, const double4* __restrict__ mu,
                              int natm, const CellC* __restrict__ cell, int has_q, int has_mu,
                              double4* __restrict__ w, float4* __restrict__ w32,
                              float4* __restrict__ mu32, SlotW sw = SlotW()) {
  pdl_wait();
  pdl_trigger();
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= natm) return;
  const double* B = cell->B;
  double qi = has_q ? q[i] : 0.0;
  double m1 = 0.0, m2 = 0.0, m3 = 0.0;
  if (has_mu) {
    double4 u = mu[i];
    m1 = kTwoPi * (B[0] * u.x + B[3] * u.y + B[6] * u.z);
    m2 = kTwoPi * (B[1] * u.x + B[4] * u.y + B[7] * u.z);
    m3 = kTwoPi * (B[2] * u.x + B[5] * u.y + B[8] * u.z);
  }
  w[i] = make_double4(qi, m1, m2, m3);
  if (w32) {
    const float4 wv = make_float4((float)qi, (float)m1, (float)m2, (float)m3);
    w32[i] = wv;
    sw.put(i, wv);
  }
  if (mu32) {
    double4 u = mu[i];
    mu32[i] = make_float4((float)u.x, (float)u.y, (float)u.z, 0.f);
  }
}

template <typename C>
__device__ __forceinline__ C cmul(C a, C b) {
  C r;
  r.x = a.x * b.x - a.y * b.y;
  r.y = a.x * b.y + a.y * b.x;
  return r;
}
template <typename C>
__device__ __forceinline__ C cconj(C a) {
  a.y = -a.y;
  return a;
}

// phase of (nx, ny, nz) for ion i from the tables
template <typename R>
__device__ __forceinline__ typename cplx<R>::T phase_xyz(const typename cplx<R>::T* __restrict__ tab,
                                                         int natm, int i, int nx, int ny, int nz,
                                                         int kx, int ky) {
  typedef typename cplx<R>::T C;
  C X = tab[(size_t)nx * natm + i];
  int ay = ny < 0 ? -ny : ny;
  C Y = tab[(size_t)(kx + 1 + ay) * natm + i];
  if (ny < 0) Y = cconj(Y);
  int az = nz < 0 ? -nz : nz;
  C Z = tab[(size_t)(kx + 1 + ky + 1 + az) * natm + i];
  if (nz < 0) Z = cconj(Z);
  return cmul(cmul(X, Y), Z);
}

// XY * Z_nz for ion i (Z_{-n} = conj Z_n); |nz| must not exceed the table's kz
template <typename R>
__device__ __forceinline__ typename cplx<R>::T phase_z(const typename cplx<R>::T* __restrict__ tab,
                                                       int natm, int i, typename cplx<R>::T XY,
                                                       int nz, int kx, int ky) {
  typedef typename cplx<R>::T C;
  int az = nz < 0 ? -nz : nz;
  C Z = tab[(size_t)(kx + 1 + ky + 1 + az) * natm + i];
  if (nz < 0) Z = cconj(Z);
  return cmul(XY, Z);
}

// rho partials.  grid.x = nrows * ntiles, grid.y = ion chunks; block 128.
// part[chunk][k] (double2).  Each thread keeps NZT accumulators (one per nz
// of the tile) over its ions; the phase advances by one complex multiply per
// nz and is re-anchored on the exact table every 4 nz (FP32 drift bound).
// Warp partial sums in R, block and chunk sums in FP64, fixed order.
template <typename R, bool HAS_Q, bool HAS_MU, int NZT>
static __global__ void __launch_bounds__(128) k_rec_rho(const typename cplx<R>::T* __restrict__ tab,
                                                 const double4* __restrict__ w, int natm,
                                                 int chunk, RecMesh M, int ntiles,
                                                 double2* __restrict__ part) {
  pdl_wait();
  pdl_trigger();
  typedef typename cplx<R>::T C;
  __shared__ double red[2 * NZT][4];
  int row = blockIdx.x / ntiles, tile = blockIdx.x % ntiles;
  int4 ri = M.rows[row];
  int nx = ri.x, ny = ri.y, nz_lo = ri.z, koff = ri.w;
  int kz = M.kmax[2];
  int nz0 = nz_lo + tile * NZT;
  if (nz0 > kz) return;
  int nzn = kz - nz0 + 1;
  if (nzn > NZT) nzn = NZT;
  int a0 = blockIdx.y * chunk, a1 = a0 + chunk;
  if (a1 > natm) a1 = natm;
  R accR[NZT], accI[NZT];
#pragma unroll
  for (int t = 0; t < NZT; ++t) accR[t] = accI[t] = R(0);
  const int kx = M.kmax[0], ky = M.kmax[1];
  const size_t zoff = (size_t)(kx + 1 + ky + 1);
  for (int i = a0 + threadIdx.x; i < a1; i += blockDim.x) {
    C XY = phase_xyz<R>(tab, natm, i, nx, ny, 0, kx, ky);
    C Z1 = tab[(zoff + 1) * natm + i];
    double4 wi = w[i];
    R q = (R)wi.x;
    R m3 = (R)wi.w;
    R km = (R)(nx * wi.y + ny * wi.z + nz0 * wi.w);
    C P;
#pragma unroll
    for (int t = 0; t < NZT; ++t) {
      if ((t & 3) == 0 && (t == 0 || sizeof(R) == 4)) {
        // anchor on the table; slots beyond the row's end only compute
        // values that are never stored, so clamp their index into the table
        int nz = nz0 + t;
        nz = nz > kz ? kz : nz;
        P = phase_z<R>(tab, natm, i, XY, nz, kx, ky);
      }
      if (HAS_Q) {
        accR[t] += q * P.x;
        accI[t] += q * P.y;
      }
      if (HAS_MU) {
        accR[t] -= km * P.y;
        accI[t] += km * P.x;
        km += m3;
      }
      if (t + 1 < NZT && ((t + 1) & 3) != 0) P = cmul(P, Z1);
      else if (t + 1 < NZT && sizeof(R) == 8) P = cmul(P, Z1);
    }
  }
  int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
#pragma unroll
  for (int t = 0; t < NZT; ++t) {
    R vr = warp_sum(accR[t]);
    R vi = warp_sum(accI[t]);
    if (lane == 0) {
      red[2 * t][wp] = (double)vr;
      red[2 * t + 1][wp] = (double)vi;
    }
  }
  __syncthreads();
  if ((int)threadIdx.x < nzn) {
    int t = threadIdx.x;
    double vr = red[2 * t][0] + red[2 * t][1] + red[2 * t][2] + red[2 * t][3];
    double vi = red[2 * t + 1][0] + red[2 * t + 1][1] + red[2 * t + 1][2] + red[2 * t + 1][3];
    int k = koff + (nz0 - nz_lo) + t;
    part[(size_t)blockIdx.y * M.nk + k] = make_double2(vr, vi);
  }
}

// rho' (k) = A_k sum over ion chunks of the structure-factor partials, the
// chunks in order (k_rec_sum and the field kernels' staging give the same bits)
static __device__ __forceinline__ double2 rho_prime(const double2* __restrict__ part, int nchunk,
                                                    const double* __restrict__ Ak, int nk, int k) {
  double r = 0.0, im = 0.0;
  for (int c = 0; c < nchunk; ++c) {
    double2 v = part[(size_t)c * nk + k];
    r += v.x;
    im += v.y;
  }
  double A = Ak[k];
  return make_double2(A * r, A * im);
}

// rho = sum over chunks; rhoA = A_k rho; str = A_k |rho|^2 (acc: also a
// copy of rhoA, the start of the dipole solve's accumulated rho')
static __global__ void k_rec_sum(const double2* __restrict__ part, int nchunk, RecMesh M,
                          double2* __restrict__ rhoA, double* __restrict__ str,
                          double2* __restrict__ acc = nullptr) {
  pdl_wait();
  pdl_trigger();
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= M.nk) return;
  double r = 0.0, im = 0.0;
  for (int c = 0; c < nchunk; ++c) {
    double2 v = part[(size_t)c * M.nk + k];
    r += v.x;
    im += v.y;
  }
  double A = M.Ak[k];
  rhoA[k] = make_double2(A * r, A * im);
  str[k] = (r * r + im * im) * A;
  if (acc) acc[k] = make_double2(A * r, A * im);
}

// rhoA and str of the force pass from the dipole solve's accumulated rho'
// (rho' of the charges and the first guess, plus alpha_k rho'(p_k) of every
// CG step: the structure factor is linear in the dipoles); str = |rho'|^2 / A_k
static __global__ void k_rec_acc_finish(const double2* __restrict__ acc, RecMesh M,
                                        double2* __restrict__ rhoA, double* __restrict__ str) {
  pdl_wait();
  pdl_trigger();
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= M.nk) return;
  const double2 a = acc[k];
  rhoA[k] = a;
  str[k] = (a.x * a.x + a.y * a.y) / M.Ak[k];
}

// u_rec (x2 x tpi_V) and tau_rec (x2, symmetric, x tpi_V/omega): out[0..6] =
// u, tau xx yy zz xy xz yz.  One block.
static __global__ void k_rec_energy(const double* __restrict__ str, RecMesh M, double tpi_V,
                             double omega, int do_stress, double* __restrict__ out) {
  pdl_wait();
  pdl_trigger();
  __shared__ double red[7 * 32];
  double v[7] = {0, 0, 0, 0, 0, 0, 0};
  for (int k = threadIdx.x; k < M.nk; k += blockDim.x) {
    double s = str[k];
    double4 kv = M.kvec[k];
    v[0] += s;
    if (do_stress) {
      v[1] += (1.0 - kv.w * kv.x * kv.x) * s;
      v[2] += (1.0 - kv.w * kv.y * kv.y) * s;
      v[3] += (1.0 - kv.w * kv.z * kv.z) * s;
      v[4] -= kv.w * kv.x * kv.y * s;
      v[5] -= kv.w * kv.x * kv.z * s;
      v[6] -= kv.w * kv.y * kv.z * s;
    }
  }
  block_sum<7>(v, red);
  if (threadIdx.x == 0) {
    out[0] = v[0] * 2.0 * tpi_V;
    for (int a = 1; a < 7; ++a) out[a] = v[a] * 2.0 * tpi_V / omega;
  }
}

// field / force partials.  grid.x = ion blocks (128), grid.y = k chunks
// (row ranges rc[c]..rc[c+1]); dynamic smem = rho' of the chunk.
// G accumulates sum_k n recarg, H accumulates sum_k n (k.mu) recarg2.
template <typename R, bool HAS_MU_FORCE>
static __global__ void __launch_bounds__(128) k_rec_field(const typename cplx<R>::T* __restrict__ tab,
                                                   const double4* __restrict__ w, int natm,
                                                   const int* __restrict__ imap, int nion,
                                                   RecMesh M, const int* __restrict__ rchunk,
                                                   const double2* __restrict__ rhoA,
                                                   const double2* __restrict__ part, int npart,
                                                   double4* __restrict__ Gpart,
                                                   double4* __restrict__ Hpart) {
  pdl_wait();
  pdl_trigger();
  typedef typename cplx<R>::T C;
  extern __shared__ unsigned char shraw[];
  C* sh = reinterpret_cast<C*>(shraw);
  int r0 = rchunk[blockIdx.y], r1 = rchunk[blockIdx.y + 1];
  int k0 = M.rows[r0].w;
  int k1 = (r1 < M.nrows) ? M.rows[r1].w : M.nk;
  for (int k = k0 + threadIdx.x; k < k1; k += blockDim.x) {
    double2 v = npart ? rho_prime(part, npart, M.Ak, M.nk, k) : rhoA[k];
    C c;
    c.x = (R)v.x;
    c.y = (R)v.y;
    sh[k - k0] = c;
  }
  __syncthreads();
  // thread slot -> ion (imap: the ions whose field is wanted, else all)
  const int sl = blockIdx.x * blockDim.x + threadIdx.x;
  if (sl >= nion) return;
  const int i = imap ? imap[sl] : sl;
  const int kx = M.kmax[0], ky = M.kmax[1], kz = M.kmax[2];
  double4 wi = w[i];
  R m3 = (R)wi.w;
  C Z1 = tab[(size_t)(kx + 1 + ky + 1 + 1) * natm + i];
  double G[3] = {0, 0, 0}, H[3] = {0, 0, 0};
  for (int r = r0; r < r1; ++r) {
    int4 ri = M.rows[r];
    int nx = ri.x, ny = ri.y, nz_lo = ri.z;
    C XY = phase_xyz<R>(tab, natm, i, nx, ny, 0, kx, ky);
    // sums over the row, nz measured from the row start: Sz = sum t recarg
    R S0 = R(0), Sz = R(0), T0 = R(0), Tz = R(0);
    R km = (R)(nx * wi.y + ny * wi.z + nz_lo * wi.w);
    const C* rr = sh + (ri.w - k0);
    int nn = kz - nz_lo + 1;
    C P = phase_z<R>(tab, natm, i, XY, nz_lo, kx, ky);
    int t0 = 0;
    R tf = R(0);  // t0 as R, advanced by 4 (no int->float conversion per term)
    for (; t0 + 4 <= nn; t0 += 4, tf += R(4)) {
      if (sizeof(R) == 4 && t0 > 0) P = phase_z<R>(tab, natm, i, XY, nz_lo + t0, kx, ky);
      R a[4], b[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        C rho = rr[t0 + u];
        a[u] = rho.y * P.x - rho.x * P.y;
        if (HAS_MU_FORCE) b[u] = (km + R(u) * m3) * (rho.x * P.x + rho.y * P.y);
        if (u < 3 || sizeof(R) == 8) P = cmul(P, Z1);
      }
      // sum_u a_u and sum_u u a_u of the group (u = 0..3)
      R sa = (a[0] + a[1]) + (a[2] + a[3]);
      R sb = a[1] + R(2) * a[2] + R(3) * a[3];
      S0 += sa;
      Sz += tf * sa + sb;
      if (HAS_MU_FORCE) {
        R ta = (b[0] + b[1]) + (b[2] + b[3]);
        R tb = b[1] + R(2) * b[2] + R(3) * b[3];
        T0 += ta;
        Tz += tf * ta + tb;
        km += R(4) * m3;
      }
    }
    if (t0 < nn) {
      if (sizeof(R) == 4 && t0 > 0) P = phase_z<R>(tab, natm, i, XY, nz_lo + t0, kx, ky);
      for (int t = t0; t < nn; ++t) {
        C rho = rr[t];
        R recarg = rho.y * P.x - rho.x * P.y;
        R tt_ = (R)t;
        S0 += recarg;
        Sz += tt_ * recarg;
        if (HAS_MU_FORCE) {
          R recarg2 = rho.x * P.x + rho.y * P.y;
          R tt = km * recarg2;
          T0 += tt;
          Tz += tt_ * tt;
          km += m3;
        }
        P = cmul(P, Z1);
      }
    }
    G[0] += (double)nx * (double)S0;
    G[1] += (double)ny * (double)S0;
    G[2] += (double)nz_lo * (double)S0 + (double)Sz;
    if (HAS_MU_FORCE) {
      H[0] += (double)nx * (double)T0;
      H[1] += (double)ny * (double)T0;
      H[2] += (double)nz_lo * (double)T0 + (double)Tz;
    }
  }
  Gpart[(size_t)blockIdx.y * natm + i] = make_double4(G[0], G[1], G[2], 0.0);
  if (HAS_MU_FORCE) Hpart[(size_t)blockIdx.y * natm + i] = make_double4(H[0], H[1], H[2], 0.0);
}

// reciprocal electric field gradient (ewald_rec.f90:209-217): per ion
// sum_k k_a k_b recarg2 on the upper triangle only (the reference never
// fills the lower one), scaled by 2 fpi_V and added into efg[i][9].  FP64,
// ion-major over all k rows; rho' = A_k rho of the final pass.
// N_pq = sum_k n_p n_q recarg2 per row from sums over nz, k_a k_b =
// 4 pi^2 sum_pq B_ap B_bq n_p n_q.
static __global__ void __launch_bounds__(128) k_rec_efg(const double2* __restrict__ tab, int natm,
                                                      RecMesh M, const double2* __restrict__ rhoA,
                                                      const CellC* __restrict__ cell, double scale,
                                                      double* __restrict__ efg) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= natm) return;
  const int kx = M.kmax[0], ky = M.kmax[1], kz = M.kmax[2];
  double2 Z1 = tab[(size_t)(kx + 1 + ky + 1 + 1) * natm + i];
  double N[6] = {0, 0, 0, 0, 0, 0};  // xx yy zz xy xz yz
  for (int r = 0; r < M.nrows; ++r) {
    int4 ri = M.rows[r];
    int nx = ri.x, ny = ri.y, nz_lo = ri.z;
    double2 XY = phase_xyz<double>(tab, natm, i, nx, ny, 0, kx, ky);
    double2 P = phase_z<double>(tab, natm, i, XY, nz_lo, kx, ky);
    double S0 = 0.0, S1 = 0.0, S2 = 0.0;
    int nn = kz - nz_lo + 1;
    const double2* rr = rhoA + ri.w;
    for (int t = 0; t < nn; ++t) {
      double2 rho = rr[t];
      double v = rho.x * P.x + rho.y * P.y;  // recarg2
      double nz = (double)(nz_lo + t);
      S0 += v;
      S1 += nz * v;
      S2 += nz * nz * v;
      P = cmul(P, Z1);
    }
    N[0] += (double)nx * nx * S0;
    N[1] += (double)ny * ny * S0;
    N[2] += S2;
    N[3] += (double)nx * ny * S0;
    N[4] += (double)nx * S1;
    N[5] += (double)ny * S1;
  }
  const double* B = cell->B;
  double Nm[3][3] = {{N[0], N[3], N[4]}, {N[3], N[1], N[5]}, {N[4], N[5], N[2]}};
  for (int a = 0; a < 3; ++a)
    for (int b = a; b < 3; ++b) {
      double v = 0.0;
      for (int p = 0; p < 3; ++p)
        for (int qq = 0; qq < 3; ++qq) v += B[3 * a + p] * B[3 * b + qq] * Nm[p][qq];
      efg[9 * (size_t)i + 3 * a + b] += kTwoPi * kTwoPi * v * scale;
    }
}

// chunk sum and scaling.  E += -(2 pi B G) * 2 fpi_V (ewald_rec.f90:193-198,
// 300-352); with do_forces, F += [q (-2 pi B G) + 2 pi B H] * 2 fpi_V * coul_unit.
// Four threads per ion split the chunk partials (fixed order, shuffle sum).
static __global__ void k_rec_field_sum(const double4* __restrict__ Gpart, const double4* __restrict__ Hpart,
                                int nchunk, int natm, const CellC* __restrict__ cell,
                                const double* __restrict__ q, double scale /* 2 fpi_V */,
                                int has_mu_force, int do_forces, double coul_unit,
                                double4* __restrict__ E, double* __restrict__ force,
                                SelfField sf, const int* __restrict__ ipolar) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  int i = t >> 2, sub = t & 3;
  double g[3] = {0, 0, 0}, h[3] = {0, 0, 0};
  if (i < natm) {
    for (int c = sub; c < nchunk; c += 4) {
      double4 v = Gpart[(size_t)c * natm + i];
      g[0] += v.x;
      g[1] += v.y;
      g[2] += v.z;
      if (has_mu_force) {
        double4 u = Hpart[(size_t)c * natm + i];
        h[0] += u.x;
        h[1] += u.y;
        h[2] += u.z;
      }
    }
  }
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    g[a] += __shfl_xor_sync(FULL_MASK, g[a], 1);
    g[a] += __shfl_xor_sync(FULL_MASK, g[a], 2);
    h[a] += __shfl_xor_sync(FULL_MASK, h[a], 1);
    h[a] += __shfl_xor_sync(FULL_MASK, h[a], 2);
  }
  if (i >= natm || sub != 0) return;
  // (ipolar: the partials cover the polarisable ions only, the field is
  // wanted there; other ions keep their real-space part)
  if (ipolar && !ipolar[i]) return;
  const double* B = cell->B;
  double e[3], fm[3];
  for (int a = 0; a < 3; ++a) {
    e[a] = -kTwoPi * (B[3 * a + 0] * g[0] + B[3 * a + 1] * g[1] + B[3 * a + 2] * g[2]) * scale;
    fm[a] = kTwoPi * (B[3 * a + 0] * h[0] + B[3 * a + 1] * h[1] + B[3 * a + 2] * h[2]) * scale;
  }
  // self (+ surface) field of the same moments, field only (no force)
  double s[3] = {0.0, 0.0, 0.0};
  if (sf.on) {
    double4 m = sf.mu ? sf.mu[i] : make_double4(0, 0, 0, 0);
    if (sf.lsurf) {
      s[0] = -(sf.mom[0] + sf.mom[3]) * sf.fpi_3V;
      s[1] = -(sf.mom[1] + sf.mom[4]) * sf.fpi_3V;
      s[2] = -(sf.mom[2] + sf.mom[5]) * sf.fpi_3V;
    }
    s[0] += 2.0 * sf.selfa2 * m.x;
    s[1] += 2.0 * sf.selfa2 * m.y;
    s[2] += 2.0 * sf.selfa2 * m.z;
  }
  double4 o = E[i];
  E[i] = make_double4(o.x + e[0] + s[0], o.y + e[1] + s[1], o.z + e[2] + s[2], 0.0);
  if (do_forces) {
    double qi = q[i];
    force[i] += (qi * e[0] + (has_mu_force ? fm[0] : 0.0)) * coul_unit;
    force[natm + i] += (qi * e[1] + (has_mu_force ? fm[1] : 0.0)) * coul_unit;
    force[2 * natm + i] += (qi * e[2] + (has_mu_force ? fm[2] : 0.0)) * coul_unit;
  }
}

// The CG operator's last step, fused: E_i = (reciprocal field from the chunk
// partials G + self / surface field) + real-space dipole field from the FP32
// pair cache of k_static_cache, written (not added).  The same operations, in
// the same order, as k_rec_field_sum (no forces) into a zeroed E followed by
// k_dd_cached, so the results are identical; one launch and no memset instead.
static __global__ void __launch_bounds__(256) k_dd_cached_rec(
    const float4* __restrict__ mu, const float4* __restrict__ cr, const float* __restrict__ cb1,
    const int* __restrict__ cj, const int* __restrict__ cn, int cap, int natm,
    const double4* __restrict__ Gpart, int nchunk, const CellC* __restrict__ cell, double scale,
    SelfField sf, double4* __restrict__ E, const double4* __restrict__ Edd,
    const int* __restrict__ ipolar) {
  pdl_wait();
  pdl_trigger();
  int lane = threadIdx.x & 31;
  int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (i >= natm) return;
  // (ipolar: the operator is wanted at the polarisable ions only; its
  // reciprocal partials may cover only those)
  if (ipolar && !ipolar[i]) {
    if (lane == 0) E[i] = make_double4(0.0, 0.0, 0.0, 0.0);
    return;
  }
  // lanes 0-3: strided chunk sums of the reciprocal partials, as the four
  // threads of an ion in k_rec_field_sum (loads issued before the pair loop)
  double g[3] = {0.0, 0.0, 0.0};
  if (lane < 4)
    for (int c = lane; c < nchunk; c += 4) {
      double4 v = Gpart[(size_t)c * natm + i];
      g[0] += v.x;
      g[1] += v.y;
      g[2] += v.z;
    }
  double4 mi = (lane == 0 && sf.on && sf.mu) ? sf.mu[i] : make_double4(0, 0, 0, 0);
  // the cached dipole field: already summed by k_dd_cached_part (Edd), else here
  double dx, dy, dz;
  if (Edd) {
    double4 v = Edd[i];
    dx = v.x;
    dy = v.y;
    dz = v.z;
  } else {
    float ex = 0.f, ey = 0.f, ez = 0.f;
    dd_cached_row<float>(mu, cr, cb1, cj, (size_t)i * cap, cn[i], lane, ex, ey, ez);
    dx = warp_sum((double)ex);
    dy = warp_sum((double)ey);
    dz = warp_sum((double)ez);
  }
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    g[a] += __shfl_xor_sync(FULL_MASK, g[a], 1);
    g[a] += __shfl_xor_sync(FULL_MASK, g[a], 2);
  }
  if (lane != 0) return;
  const double* B = cell->B;
  double e[3];
  for (int a = 0; a < 3; ++a)
    e[a] = -kTwoPi * (B[3 * a + 0] * g[0] + B[3 * a + 1] * g[1] + B[3 * a + 2] * g[2]) * scale;
  double s3[3] = {0.0, 0.0, 0.0};
  if (sf.on) {
    if (sf.lsurf) {
      s3[0] = -(sf.mom[0] + sf.mom[3]) * sf.fpi_3V;
      s3[1] = -(sf.mom[1] + sf.mom[4]) * sf.fpi_3V;
      s3[2] = -(sf.mom[2] + sf.mom[5]) * sf.fpi_3V;
    }
    s3[0] += 2.0 * sf.selfa2 * mi.x;
    s3[1] += 2.0 * sf.selfa2 * mi.y;
    s3[2] += 2.0 * sf.selfa2 * mi.z;
  }
  E[i] = make_double4((0.0 + e[0] + s3[0]) + dx, (0.0 + e[1] + s3[1]) + dy,
                      (0.0 + e[2] + s3[2]) + dz, 0.0);
}


}  // namespace mdff

namespace mdff {

// ===========================================================================
// FP32 reciprocal kernels with Blackwell packed FP32x2 arithmetic.  Each
// thread carries two ions in the two lanes of float2 values (lane x = ion a,
// lane y = ion b), so one packed FFMA2 advances both ions' phases, one shared
// rho' load serves both, and the per-term instruction count halves.  Same
// operations and roundings per ion as the scalar FP32 kernels above.

__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ float2 f2s(float a) { return make_float2(a, a); }

// packed complex multiply of (re, im) lane pairs by (zr, zi) lane pairs
__device__ __forceinline__ void cmul2(float2& re, float2& im, float2 zr, float2 zi) {
  float2 nre = __ffma2_rn(re, zr, __fmul2_rn(im, f2(-zi.x, -zi.y)));
  float2 nim = __ffma2_rn(re, zi, __fmul2_rn(im, zr));
  re = nre;
  im = nim;
}

// table phase X_nx Y_ny Z_nz of one ion (float)
__device__ __forceinline__ float2 phase1(const float2* __restrict__ tab, int natm, int i, int nx,
                                         int ny, int nz, int kx, int ky) {
  return phase_xyz<float>(tab, natm, i, nx, ny, nz, kx, ky);
}

// structure factor, FP32x2.  Thread t of the block handles ions a = i, b = i + 128
// of each 256-ion step of its chunk (b absent -> weight 0).
template <bool HAS_Q, bool HAS_MU, int NZT>
static __global__ void __launch_bounds__(128) k_rec_rho_x2(const float2* __restrict__ tab,
                                                    const float4* __restrict__ w, int natm,
                                                    int chunk, RecMesh M, int ntiles,
                                                    double2* __restrict__ part) {
  pdl_wait();
  pdl_trigger();
  __shared__ double red[2 * NZT][4];
  int row = blockIdx.x / ntiles, tile = blockIdx.x % ntiles;
  int4 ri = M.rows[row];
  int nx = ri.x, ny = ri.y, nz_lo = ri.z, koff = ri.w;
  int kz = M.kmax[2];
  int nz0 = nz_lo + tile * NZT;
  if (nz0 > kz) return;
  int nzn = kz - nz0 + 1;
  if (nzn > NZT) nzn = NZT;
  int a0 = blockIdx.y * chunk, a1 = a0 + chunk;
  if (a1 > natm) a1 = natm;
  float2 accR[NZT], accI[NZT];
#pragma unroll
  for (int t = 0; t < NZT; ++t) accR[t] = accI[t] = f2s(0.f);
  const int kx = M.kmax[0], ky = M.kmax[1];
  const size_t zoff = (size_t)(kx + 1 + ky + 1);
  const float fnx = (float)nx, fny = (float)ny, fnz0 = (float)nz0;
  for (int base = a0; base < a1; base += 256) {
    int ia = base + threadIdx.x, ib = ia + 128;
    if (ia >= a1) break;
    bool vb = ib < a1;
    int ibb = vb ? ib : ia;
    float2 XYa = phase1(tab, natm, ia, nx, ny, 0, kx, ky);
    float2 XYb = phase1(tab, natm, ibb, nx, ny, 0, kx, ky);
    float2 Pa = phase_z<float>(tab, natm, ia, XYa, nz0, kx, ky);
    float2 Pb = phase_z<float>(tab, natm, ibb, XYb, nz0, kx, ky);
    float2 Z1a = tab[(zoff + 1) * natm + ia], Z1b = tab[(zoff + 1) * natm + ibb];
    float2 Z4a = tab[(zoff + 4) * natm + ia], Z4b = tab[(zoff + 4) * natm + ibb];
    float2 zr = f2(Z1a.x, Z1b.x), zi = f2(Z1a.y, Z1b.y);
    float2 z4r = f2(Z4a.x, Z4b.x), z4i = f2(Z4a.y, Z4b.y);
    float4 wa = w[ia], wb = w[ibb];
    float2 q = f2(wa.x, vb ? wb.x : 0.f);
    float2 m3 = f2(wa.w, vb ? wb.w : 0.f);
    float2 km = f2(fnx * wa.y + fny * wa.z + fnz0 * wa.w,
                   vb ? fnx * wb.y + fny * wb.z + fnz0 * wb.w : 0.f);
    // phase at t = 4g + u: (P0 Z4^g) Z1^u
    float2 gre = f2(Pa.x, Pb.x), gim = f2(Pa.y, Pb.y);
    float2 pre = gre, pim = gim;
#pragma unroll
    for (int t = 0; t < NZT; ++t) {
      if (t > 0) {
        if ((t & 3) == 0) {
          cmul2(gre, gim, z4r, z4i);
          pre = gre;
          pim = gim;
        } else {
          cmul2(pre, pim, zr, zi);
        }
      }
      if (HAS_Q) {
        accR[t] = __ffma2_rn(q, pre, accR[t]);
        accI[t] = __ffma2_rn(q, pim, accI[t]);
      }
      if (HAS_MU) {
        accR[t] = __ffma2_rn(f2(-km.x, -km.y), pim, accR[t]);
        accI[t] = __ffma2_rn(km, pre, accI[t]);
        km = __fadd2_rn(km, m3);
      }
    }
  }
  int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
#pragma unroll
  for (int t = 0; t < NZT; ++t) {
    float vr = warp_sum(accR[t].x + accR[t].y);
    float vi = warp_sum(accI[t].x + accI[t].y);
    if (lane == 0) {
      red[2 * t][wp] = (double)vr;
      red[2 * t + 1][wp] = (double)vi;
    }
  }
  __syncthreads();
  if ((int)threadIdx.x < nzn) {
    int t = threadIdx.x;
    double vr = red[2 * t][0] + red[2 * t][1] + red[2 * t][2] + red[2 * t][3];
    double vi = red[2 * t + 1][0] + red[2 * t + 1][1] + red[2 * t + 1][2] + red[2 * t + 1][3];
    int k = koff + (nz0 - nz_lo) + t;
    part[(size_t)blockIdx.y * M.nk + k] = make_double2(vr, vi);
  }
}

// field / force partials, FP32x2: ions a = blockIdx.x*256 + tid, b = a + 128.
template <bool HAS_MU_FORCE>
static __global__ void __launch_bounds__(128) k_rec_field_x2(const float2* __restrict__ tab,
                                                      const float4* __restrict__ w, int natm,
                                                      RecMesh M, const int* __restrict__ rchunk,
                                                      const double2* __restrict__ rhoA,
                                                      const double2* __restrict__ part, int npart,
                                                      double4* __restrict__ Gpart,
                                                      double4* __restrict__ Hpart) {
  pdl_wait();
  pdl_trigger();
  extern __shared__ unsigned char shraw[];
  float2* sh = reinterpret_cast<float2*>(shraw);
  int r0 = rchunk[blockIdx.y], r1 = rchunk[blockIdx.y + 1];
  int k0 = M.rows[r0].w;
  int k1 = (r1 < M.nrows) ? M.rows[r1].w : M.nk;
  for (int k = k0 + threadIdx.x; k < k1; k += blockDim.x) {
    double2 v = npart ? rho_prime(part, npart, M.Ak, M.nk, k) : rhoA[k];
    sh[k - k0] = make_float2((float)v.x, (float)v.y);
  }
  __syncthreads();
  int ia = blockIdx.x * 256 + threadIdx.x, ib = ia + 128;
  if (ia >= natm) return;
  bool vb = ib < natm;
  int ibb = vb ? ib : ia;
  const int kx = M.kmax[0], ky = M.kmax[1], kz = M.kmax[2];
  const size_t zoff = (size_t)(kx + 1 + ky + 1);
  float4 wa = w[ia], wb = w[ibb];
  float2 m3 = f2(wa.w, wb.w);
  float2 Z1a = tab[(zoff + 1) * natm + ia], Z1b = tab[(zoff + 1) * natm + ibb];
  float2 Z4a = tab[(zoff + 4) * natm + ia], Z4b = tab[(zoff + 4) * natm + ibb];
  float2 zr = f2(Z1a.x, Z1b.x), zi = f2(Z1a.y, Z1b.y);
  float2 z4r = f2(Z4a.x, Z4b.x), z4i = f2(Z4a.y, Z4b.y);
  double Ga[3] = {0, 0, 0}, Gb[3] = {0, 0, 0}, Ha[3] = {0, 0, 0}, Hb[3] = {0, 0, 0};
  for (int r = r0; r < r1; ++r) {
    int4 ri = M.rows[r];
    int nx = ri.x, ny = ri.y, nz_lo = ri.z;
    float2 XYa = phase1(tab, natm, ia, nx, ny, 0, kx, ky);
    float2 XYb = phase1(tab, natm, ibb, nx, ny, 0, kx, ky);
    float2 Pa = phase_z<float>(tab, natm, ia, XYa, nz_lo, kx, ky);
    float2 Pb = phase_z<float>(tab, natm, ibb, XYb, nz_lo, kx, ky);
    float2 gre = f2(Pa.x, Pb.x), gim = f2(Pa.y, Pb.y);
    float2 S0 = f2s(0.f), Sz = f2s(0.f), T0 = f2s(0.f), Tz = f2s(0.f);
    float fnx = (float)nx, fny = (float)ny, fnz = (float)nz_lo;
    float2 km = f2(fnx * wa.y + fny * wa.z + fnz * wa.w, fnx * wb.y + fny * wb.z + fnz * wb.w);
    const float2* rr = sh + (ri.w - k0);
    int nn = kz - nz_lo + 1;
    int t0 = 0;
    float tf = 0.f;
    for (; t0 + 4 <= nn; t0 += 4, tf += 4.f) {
      if (t0 > 0) cmul2(gre, gim, z4r, z4i);
      float2 pre = gre, pim = gim;
      float2 a[4], b[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        float2 rho = rr[t0 + u];
        // recarg = rho_I cos - rho_R sin ; recarg2 = rho_R cos + rho_I sin
        a[u] = __ffma2_rn(f2s(rho.y), pre, __fmul2_rn(f2s(-rho.x), pim));
        if (HAS_MU_FORCE) {
          float2 r2 = __ffma2_rn(f2s(rho.x), pre, __fmul2_rn(f2s(rho.y), pim));
          float2 kmu = __ffma2_rn(f2s((float)u), m3, km);
          b[u] = __fmul2_rn(kmu, r2);
        }
        if (u < 3) cmul2(pre, pim, zr, zi);
      }
      float2 sa = __fadd2_rn(__fadd2_rn(a[0], a[1]), __fadd2_rn(a[2], a[3]));
      float2 sb = __ffma2_rn(f2s(3.f), a[3], __ffma2_rn(f2s(2.f), a[2], a[1]));
      S0 = __fadd2_rn(S0, sa);
      Sz = __fadd2_rn(Sz, __ffma2_rn(f2s(tf), sa, sb));
      if (HAS_MU_FORCE) {
        float2 ta = __fadd2_rn(__fadd2_rn(b[0], b[1]), __fadd2_rn(b[2], b[3]));
        float2 tb = __ffma2_rn(f2s(3.f), b[3], __ffma2_rn(f2s(2.f), b[2], b[1]));
        T0 = __fadd2_rn(T0, ta);
        Tz = __fadd2_rn(Tz, __ffma2_rn(f2s(tf), ta, tb));
        km = __ffma2_rn(f2s(4.f), m3, km);
      }
    }
    if (t0 < nn) {
      if (t0 > 0) cmul2(gre, gim, z4r, z4i);
      float2 pre = gre, pim = gim;
      for (int t = t0; t < nn; ++t) {
        float2 rho = rr[t];
        float2 a = __ffma2_rn(f2s(rho.y), pre, __fmul2_rn(f2s(-rho.x), pim));
        float2 tt_ = f2s((float)t);
        S0 = __fadd2_rn(S0, a);
        Sz = __ffma2_rn(tt_, a, Sz);
        if (HAS_MU_FORCE) {
          float2 r2 = __ffma2_rn(f2s(rho.x), pre, __fmul2_rn(f2s(rho.y), pim));
          float2 b = __fmul2_rn(km, r2);
          T0 = __fadd2_rn(T0, b);
          Tz = __ffma2_rn(tt_, b, Tz);
          km = __fadd2_rn(km, m3);
        }
        cmul2(pre, pim, zr, zi);
      }
    }
    Ga[0] += (double)nx * (double)S0.x;
    Ga[1] += (double)ny * (double)S0.x;
    Ga[2] += (double)nz_lo * (double)S0.x + (double)Sz.x;
    Gb[0] += (double)nx * (double)S0.y;
    Gb[1] += (double)ny * (double)S0.y;
    Gb[2] += (double)nz_lo * (double)S0.y + (double)Sz.y;
    if (HAS_MU_FORCE) {
      Ha[0] += (double)nx * (double)T0.x;
      Ha[1] += (double)ny * (double)T0.x;
      Ha[2] += (double)nz_lo * (double)T0.x + (double)Tz.x;
      Hb[0] += (double)nx * (double)T0.y;
      Hb[1] += (double)ny * (double)T0.y;
      Hb[2] += (double)nz_lo * (double)T0.y + (double)Tz.y;
    }
  }
  Gpart[(size_t)blockIdx.y * natm + ia] = make_double4(Ga[0], Ga[1], Ga[2], 0.0);
  if (HAS_MU_FORCE) Hpart[(size_t)blockIdx.y * natm + ia] = make_double4(Ha[0], Ha[1], Ha[2], 0.0);
  if (vb) {
    Gpart[(size_t)blockIdx.y * natm + ib] = make_double4(Gb[0], Gb[1], Gb[2], 0.0);
    if (HAS_MU_FORCE) Hpart[(size_t)blockIdx.y * natm + ib] = make_double4(Hb[0], Hb[1], Hb[2], 0.0);
  }
}

}  // namespace mdff
