// batch.cuh -- batched engforce: many independent configurations of uneven
// ion counts in one persistent kernel.
//
// The reference evaluates one configuration per engforce call
// (engforce_driver.f90:102-190); a batch of small boxes would leave a B200
// mostly idle, one launch sequence per box.  Here one thread-block cluster of
// C CTAs owns one configuration at a time and takes the next one from a
// device work queue (configurations are queued in descending cost order, so
// the tail is short).  Inside a cluster each CTA owns a slice of the ions
// (pair sums, fields, forces, solver vectors) and a slice of the k-mesh rows
// (structure factor); the CTAs exchange vectors through L2 and meet at
// hardware cluster barriers.  Boxes are small (the real-space cutoff is
// clamped to half the box, coulomb.f90:377-383), so each ion loops over all
// ions of its box with the minimum image instead of a Verlet list: the pair
// set and each pair's arithmetic are those of the list-based engine.
//
// Per configuration, in order:
//   load      direct coordinates (kardir, lattice.f90:183-225), phase tables
//   short     engforce_bmhftd_pbc / engforce_nmlj_pbc (FP64)
//   static    damped charge (+ static dipole) field (moment_from_pola.f90:327-330)
//   solve     PCG on (alpha^-1 - T) mu = E_stat with FP64 residual refinement
//             (calc = 'other': the first guess is alpha E_stat)
//   force     multipole_ES with forces, energy, stress (ewald.f90:49-314)
// Scalars land in the single-configuration engine's slot layout.
#pragma once
#include <cooperative_groups.h>

#include "common.cuh"
#include "realspace.cuh"
#include "recip.cuh"

namespace mdff {

namespace cgx = cooperative_groups;

constexpr int kBMaxT = 4;          // types of a batched configuration
constexpr int kBPart = 16;         // values per CTA partial slot
constexpr int kBKChunk = 1024;     // k of rho' staged per shared-memory chunk
constexpr int kBNZ = 8;            // nz per structure-factor work item
constexpr int kBMaxC = 8;          // largest cluster
constexpr int kBSlots = 48;        // per-configuration scalar slots

// scalar slots of a configuration (same offsets as the single engine)
enum {
  BS_SR = 0,     // 16
  BS_DIR = 16,   // 7
  BS_REC = 23,   // 7
  BS_MOM = 30,   // 8
  BS_UPOL = 38,
  BS_ITER = 39,
  BS_CONV = 40,
  BS_RMSD = 41,
  BS_CATA = 42,
  BS_STAT = 43   // 0 = ok, else an MDFF_ERR_* code
};

enum {
  BF_COUL = 1, BF_SR = 2, BF_BMH = 4, BF_BMHFTD = 8, BF_LJ = 16, BF_POLAR = 32,
  BF_QQ = 64, BF_QD = 128, BF_DD = 256, BF_SURF = 512, BF_DIPST = 1024, BF_THOLE = 2048,
  BF_WFC = 4096
};

struct BConf {
  int off, n, ntype, flags;
  int nk, nrows, row_off, k_off;
  int kx, ky, kz, ntab;
  long long tab_off;
  int tab_ld;            // leading dimension of the tables (= n)
  int trunc, maxit, npol;
  int nb_off, es_off, pad0, pad1;
  double A[9], B[9], omega;
  double alpha, rc2, coul_unit, tol;
  int lwfc[kBMaxT];      // Wannier centres per type (BF_WFC): < 0 centre type
  int ldip_wfc, pad2;
  double rcut_wfc;
};

struct BatchArgs {
  int nconf, ntot;
  const BConf* conf;
  const int* order;      // queue position -> configuration (descending cost)
  int* queue;            // zeroed before every launch
  const double* pos;     // [3][ntot] Cartesian
  const int* typ;        // [ntot] type within its configuration
  const double* q;       // [ntot]
  const int* ipol;       // [ntot] polarisable flag (ldip_polar of the type)
  const double* pol;     // [ntot][9]
  const double* inv;     // [ntot][9]
  const double4* dip;    // [ntot] static dipoles
  const NBPair* nbtab;   // per configuration, [ntype][ntype] at nb_off
  const ESPair* estab;
  const int4* rows;      // per configuration at row_off: (nx, ny, nz_lo, k)
  const double* Ak;      // per configuration at k_off
  const double4* kvec;
  double4* s;            // [ntot] direct coordinates, w = q
  double2* tab64;        // phase tables, [entry][ion] per configuration
  float2* tab32;
  double2* rho;          // [sum nk] rho' = A_k rho
  double4 *Estat, *x, *r, *z, *p, *mu;  // [ntot]
  double4* E;            // [ntot] final field
  double* force;         // [3][ntot]
  double* part;          // [nconf][kBMaxC][2][kBPart]
  double* out;           // [nconf][kBSlots]
};

// shared-memory layout of one CTA for configurations of up to nmax ions
struct BShared {
  double4* s;      // [nmax]
  double4* v;      // [nmax] vector operand (FP64)
  float4* v32;     // [nmax] vector operand (FP32)
  int* t;          // [nmax]
  double2* rho;    // [kBKChunk]
  NBPair* nb;      // [kBMaxT^2]
  ESPair* es;      // [kBMaxT^2]
  double* red;     // [kBPart * 32]
  double* res;     // [kBPart]
  int* cfg;        // [1]
};

__host__ __device__ inline size_t batch_smem_bytes(int nmax) {
  size_t b = 0;
  b += sizeof(double4) * nmax * 2;
  b += sizeof(double2) * kBKChunk;
  b += sizeof(float4) * nmax;
  b += sizeof(NBPair) * kBMaxT * kBMaxT;
  b += sizeof(ESPair) * kBMaxT * kBMaxT;
  b += sizeof(double) * kBPart * 33;
  b += sizeof(int) * nmax + 16;
  return b;
}

// offset of the adjoint's extra [nmax] double4 array after the layout
// (rounded up to 16 bytes: vector loads need the alignment)
__host__ __device__ inline size_t batch_smem_extra_offset(int nmax) {
  return (batch_smem_bytes(nmax) + 15) & ~(size_t)15;
}

__device__ inline BShared batch_smem(unsigned char* base, int nmax) {
  BShared S;
  size_t o = 0;
  S.s = reinterpret_cast<double4*>(base + o); o += sizeof(double4) * nmax;
  S.v = reinterpret_cast<double4*>(base + o); o += sizeof(double4) * nmax;
  S.rho = reinterpret_cast<double2*>(base + o); o += sizeof(double2) * kBKChunk;
  S.v32 = reinterpret_cast<float4*>(base + o); o += sizeof(float4) * nmax;
  S.nb = reinterpret_cast<NBPair*>(base + o); o += sizeof(NBPair) * kBMaxT * kBMaxT;
  S.es = reinterpret_cast<ESPair*>(base + o); o += sizeof(ESPair) * kBMaxT * kBMaxT;
  S.red = reinterpret_cast<double*>(base + o); o += sizeof(double) * kBPart * 32;
  S.res = reinterpret_cast<double*>(base + o); o += sizeof(double) * kBPart;
  S.t = reinterpret_cast<int*>(base + o); o += sizeof(int) * nmax;
  S.cfg = reinterpret_cast<int*>(base + o);
  return S;
}

// what one CTA knows about the configuration it works on
struct BCtx {
  const BConf* c;
  int cfg, rank, C, i0, i1, n, off;
  double* part;   // this configuration's partial slots
  int parity;
};

// Sum NV values over the cluster; every thread of every CTA receives the
// same result (partials are summed in rank order).  Slots are double-buffered
// by parity: a slot is rewritten two reductions later, after a barrier that
// every reader has passed.
template <int NV>
__device__ void cluster_sum(cgx::cluster_group& cl, BCtx& X, const BShared& S, double (&v)[NV]) {
  block_sum<NV>(v, S.red);
  double* mine = X.part + ((size_t)X.rank * 2 + X.parity) * kBPart;
  if (threadIdx.x == 0)
#pragma unroll
    for (int k = 0; k < NV; ++k) mine[k] = v[k];
  cl.sync();
  if ((int)threadIdx.x < NV) {
    double acc = 0.0;
    for (int c = 0; c < X.C; ++c)
      acc += __ldcg(X.part + ((size_t)c * 2 + X.parity) * kBPart + threadIdx.x);
    S.res[threadIdx.x] = acc;
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < NV; ++k) v[k] = S.res[k];
  __syncthreads();
  X.parity ^= 1;
}

// L2 load of a 4-vector written by another CTA of the cluster
__device__ __forceinline__ double4 ldcg4(const double4* p) {
  const double2* q = reinterpret_cast<const double2*>(p);
  double2 a = __ldcg(q), b = __ldcg(q + 1);
  return make_double4(a.x, a.y, b.x, b.y);
}

// all ions' 4-vectors of the configuration from global memory into shared
__device__ inline void gather_vec(const BCtx& X, const double4* __restrict__ g, double4* sh) {
  for (int i = threadIdx.x; i < X.n; i += blockDim.x) sh[i] = ldcg4(g + X.off + i);
}
__device__ inline void gather_vec32(const BCtx& X, const double4* __restrict__ g, float4* sh) {
  for (int i = threadIdx.x; i < X.n; i += blockDim.x) {
    double4 v = ldcg4(g + X.off + i);
    sh[i] = make_float4((float)v.x, (float)v.y, (float)v.z, 0.f);
  }
}

template <typename R>
__device__ __forceinline__ typename cplx<R>::T btab(const BatchArgs& a, const BConf& c, int e, int i);
template <>
__device__ __forceinline__ double2 btab<double>(const BatchArgs& a, const BConf& c, int e, int i) {
  return a.tab64[c.tab_off + (long long)e * c.tab_ld + i];
}
template <>
__device__ __forceinline__ float2 btab<float>(const BatchArgs& a, const BConf& c, int e, int i) {
  return a.tab32[c.tab_off + (long long)e * c.tab_ld + i];
}

// X_nx Y_ny Z_nz of ion i (negative indices by conjugation)
template <typename R>
__device__ __forceinline__ typename cplx<R>::T bphase(const BatchArgs& a, const BConf& c, int i,
                                                      int nx, int ny, int nz) {
  typedef typename cplx<R>::T Cx;
  Cx X = btab<R>(a, c, nx, i);
  int ay = ny < 0 ? -ny : ny;
  Cx Y = btab<R>(a, c, c.kx + 1 + ay, i);
  if (ny < 0) Y = cconj(Y);
  int az = nz < 0 ? -nz : nz;
  Cx Z = btab<R>(a, c, c.kx + 1 + c.ky + 1 + az, i);
  if (nz < 0) Z = cconj(Z);
  return cmul(cmul(X, Y), Z);
}
template <typename R>
__device__ __forceinline__ typename cplx<R>::T bphase_z(const BatchArgs& a, const BConf& c, int i,
                                                        typename cplx<R>::T XY, int nz) {
  typedef typename cplx<R>::T Cx;
  int az = nz < 0 ? -nz : nz;
  Cx Z = btab<R>(a, c, c.kx + 1 + c.ky + 1 + az, i);
  if (nz < 0) Z = cconj(Z);
  return cmul(XY, Z);
}

// m = 2 pi B^T mu (so that k.mu = n.m)
__device__ __forceinline__ double3 bmvec(const BConf& c, double mx, double my, double mz) {
  return make_double3(kTwoPi * (c.B[0] * mx + c.B[3] * my + c.B[6] * mz),
                      kTwoPi * (c.B[1] * mx + c.B[4] * my + c.B[7] * mz),
                      kTwoPi * (c.B[2] * mx + c.B[5] * my + c.B[8] * mz));
}

// ---------------------------------------------------------------------------
// reciprocal space (multipole_ES_rec, ewald_rec.f90:38-365) of one
// configuration.  Weights: q from S.s[].w (has_q), mu from S.v (FP64) or
// S.v32 (FP32).  Adds the field into E[own] and, with forces, q E + F_mu into
// force[own] * coul_unit.  With do_str, es[0..6] receives this CTA's share of
// (u_rec, tau_rec) already scaled as k_rec_energy.
template <typename R>
__device__ void brec(cgx::cluster_group& cl, const BatchArgs& a, BCtx& X, const BShared& S,
                     bool has_q, bool has_mu, bool forces, bool do_str, double4* __restrict__ Eown,
                     double* __restrict__ force, double (&es)[7]) {
  typedef typename cplx<R>::T Cx;
  const BConf& c = *X.c;
  for (int k = 0; k < 7; ++k) es[k] = 0.0;
  if (c.nk == 0) return;
  const int4* rows = a.rows + c.row_off;
  const int kz = c.kz;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  // readers of the previous rho' are done before it is overwritten
  cl.sync();
  // ---- rho over this CTA's rows, all ions; lanes split the ions -----------
  int r0 = (int)((long long)c.nrows * X.rank / X.C), r1 = (int)((long long)c.nrows * (X.rank + 1) / X.C);
  const int ntile = (2 * kz + 1 + kBNZ - 1) / kBNZ;
  int nitems = (r1 - r0) * ntile;
  for (int it = warp; it < nitems; it += nwarp) {
    int row = r0 + it / ntile, tile = it % ntile;
    int4 ri = rows[row];
    int nx = ri.x, ny = ri.y;
    int nz0 = ri.z + tile * kBNZ;
    if (nz0 > kz) continue;  // warp-uniform
    int nzn = min(kBNZ, kz - nz0 + 1);
    R accR[kBNZ], accI[kBNZ];
#pragma unroll
    for (int t = 0; t < kBNZ; ++t) accR[t] = accI[t] = R(0);
    for (int i = lane; i < X.n; i += 32) {
      Cx XY = bphase<R>(a, c, i, nx, ny, 0);
      Cx Z1 = btab<R>(a, c, c.kx + 1 + c.ky + 1 + 1, i);
      R qv = has_q ? (R)S.s[i].w : R(0);
      R km = R(0), m3 = R(0);
      if (has_mu) {
        double4 mu = S.v[i];
        double3 m = bmvec(c, mu.x, mu.y, mu.z);
        km = (R)(nx * m.x + ny * m.y + nz0 * m.z);
        m3 = (R)m.z;
      }
      Cx P;
#pragma unroll
      for (int t = 0; t < kBNZ; ++t) {
        if ((t & 3) == 0 && (t == 0 || sizeof(R) == 4)) {
          int nz = min(nz0 + t, kz);
          P = bphase_z<R>(a, c, i, XY, nz);
        }
        accR[t] += qv * P.x - km * P.y;
        accI[t] += qv * P.y + km * P.x;
        km += m3;
        if (t + 1 < kBNZ && (((t + 1) & 3) != 0 || sizeof(R) == 8)) P = cmul(P, Z1);
      }
    }
#pragma unroll
    for (int t = 0; t < kBNZ; ++t) {
      R vr = warp_sum(accR[t]);
      R vi = warp_sum(accI[t]);
      if (lane == 0 && t < nzn) {
        int kl = ri.w + (nz0 - ri.z) + t;
        double A = a.Ak[c.k_off + kl];
        double rr = (double)vr, ii = (double)vi;
        a.rho[c.k_off + kl] = make_double2(A * rr, A * ii);
        if (do_str) {
          double st = (rr * rr + ii * ii) * A;
          double4 kv = a.kvec[c.k_off + kl];
          es[0] += st;
          es[1] += (1.0 - kv.w * kv.x * kv.x) * st;
          es[2] += (1.0 - kv.w * kv.y * kv.y) * st;
          es[3] += (1.0 - kv.w * kv.z * kv.z) * st;
          es[4] -= kv.w * kv.x * kv.y * st;
          es[5] -= kv.w * kv.x * kv.z * st;
          es[6] -= kv.w * kv.y * kv.z * st;
        }
      }
    }
  }
  if (do_str) {
    double tpi_V = kTwoPi / c.omega;
    es[0] *= 2.0 * tpi_V;
    for (int k = 1; k < 7; ++k) es[k] *= 2.0 * tpi_V / c.omega;
  }
  cl.sync();
  // ---- field / force of this CTA's ions over all k -----------------------
  const bool muf = forces && has_mu;
  int mown = X.i1 - X.i0;
  int sub = 1;
  while (sub < 32 && mown * sub * 2 <= (int)blockDim.x) sub *= 2;
  int slots = blockDim.x / sub;
  int iters = (mown + slots - 1) / slots;
  const double scale = 2.0 * (2.0 * (kTwoPi / c.omega));
  for (int itn = 0; itn < iters; ++itn) {
    int slot = itn * slots + (int)threadIdx.x / sub;
    int me = threadIdx.x % sub;
    bool act = slot < mown;
    int i = X.i0 + (act ? slot : 0);
    double G[3] = {0, 0, 0}, H[3] = {0, 0, 0};
    R m1 = R(0), m2 = R(0), m3 = R(0);
    if (muf) {
      double4 mu = S.v[i];
      double3 m = bmvec(c, mu.x, mu.y, mu.z);
      m1 = (R)m.x;
      m2 = (R)m.y;
      m3 = (R)m.z;
    }
    Cx Z1 = btab<R>(a, c, c.kx + 1 + c.ky + 1 + 1, i);
    int ra = 0;
    while (ra < c.nrows) {
      int kbase = rows[ra].w;
      int rb = ra;
      while (rb < c.nrows) {
        int4 rr = rows[rb];
        if (rr.w + (kz - rr.z + 1) - kbase > kBKChunk) break;
        ++rb;
      }
      int kend = (rb < c.nrows) ? rows[rb].w : c.nk;
      __syncthreads();
      for (int k = threadIdx.x; k < kend - kbase; k += blockDim.x)
        S.rho[k] = __ldcg(a.rho + c.k_off + kbase + k);
      __syncthreads();
      if (act) {
        for (int r = ra + me; r < rb; r += sub) {
          int4 ri = rows[r];
          int nx = ri.x, ny = ri.y, nz_lo = ri.z;
          Cx XY = bphase<R>(a, c, i, nx, ny, 0);
          Cx P = bphase_z<R>(a, c, i, XY, nz_lo);
          R S0 = R(0), Sz = R(0), T0 = R(0), Tz = R(0);
          R km = muf ? (R)nx * m1 + (R)ny * m2 + (R)nz_lo * m3 : R(0);
          int nn = kz - nz_lo + 1;
          const double2* rr = S.rho + (ri.w - kbase);
          R tf = R(0);
          for (int t = 0; t < nn; ++t, tf += R(1)) {
            if (sizeof(R) == 4 && t > 0 && (t & 3) == 0) P = bphase_z<R>(a, c, i, XY, nz_lo + t);
            double2 rv = rr[t];
            R rhoR = (R)rv.x, rhoI = (R)rv.y;
            R recarg = rhoI * P.x - rhoR * P.y;
            S0 += recarg;
            Sz += tf * recarg;
            if (muf) {
              R tt = km * (rhoR * P.x + rhoI * P.y);
              T0 += tt;
              Tz += tf * tt;
              km += m3;
            }
            P = cmul(P, Z1);
          }
          G[0] += (double)nx * (double)S0;
          G[1] += (double)ny * (double)S0;
          G[2] += (double)nz_lo * (double)S0 + (double)Sz;
          if (muf) {
            H[0] += (double)nx * (double)T0;
            H[1] += (double)ny * (double)T0;
            H[2] += (double)nz_lo * (double)T0 + (double)Tz;
          }
        }
      }
      ra = rb;
    }
    // sum the sub-threads of the ion (consecutive lanes)
    for (int o = 1; o < sub; o <<= 1)
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        G[d] += __shfl_xor_sync(FULL_MASK, G[d], o);
        H[d] += __shfl_xor_sync(FULL_MASK, H[d], o);
      }
    if (act && me == 0) {
      double e[3], fm[3];
      for (int d = 0; d < 3; ++d) {
        e[d] = -kTwoPi * (c.B[3 * d] * G[0] + c.B[3 * d + 1] * G[1] + c.B[3 * d + 2] * G[2]) * scale;
        fm[d] = kTwoPi * (c.B[3 * d] * H[0] + c.B[3 * d + 1] * H[1] + c.B[3 * d + 2] * H[2]) * scale;
      }
      int gi = X.off + i;
      double4 o = Eown[gi];
      Eown[gi] = make_double4(o.x + e[0], o.y + e[1], o.z + e[2], 0.0);
      if (forces) {
        double qi = S.s[i].w;
        force[gi] += (qi * e[0] + (muf ? fm[0] : 0.0)) * c.coul_unit;
        force[a.ntot + gi] += (qi * e[1] + (muf ? fm[1] : 0.0)) * c.coul_unit;
        force[2 * (size_t)a.ntot + gi] += (qi * e[2] + (muf ? fm[2] : 0.0)) * c.coul_unit;
      }
    }
  }
}

// ---------------------------------------------------------------------------
// real-space field of the vector in S.v / S.v32 on this CTA's ions (warp per
// ion, lanes over all ions of the box).  QQ: damped charge field; DD: dipole
// field with dd_mask as k_es_field.  Result added into E[own].
template <typename R, bool QQ, bool DD>
__device__ void bfield(const BatchArgs& a, const BCtx& X, const BShared& S, int damp, int dd_mask,
                       double4* __restrict__ E) {
  const BConf& c = *X.c;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  const R rc2 = (R)c.rc2;
  for (int i = X.i0 + warp; i < X.i1; i += nwarp) {
    double4 si = S.s[i];
    int ti = S.t[i];
    bool dip_i = false;
    if (DD) {
      if (dd_mask) dip_i = a.ipol[X.off + i] != 0;
      else {
        double4 m = S.v[i];
        dip_i = m.x != 0 || m.y != 0 || m.z != 0;
      }
    }
    R ex = R(0), ey = R(0), ez = R(0);
    if (QQ || dip_i) {
      for (int j = lane; j < X.n; j += 32) {
        if (j == i) continue;
        double4 sj = S.s[j];
        R rx, ry, rz;
        R r2 = pair_vec<R>(c.A, si, sj, rx, ry, rz);
        if (r2 > rc2) continue;  // ewald_dir.f90:202
        R mx = R(0), my = R(0), mz = R(0);
        bool dd = false;
        if (DD && dip_i) {
          if (sizeof(R) == 4) {
            float4 m = S.v32[j];
            mx = (R)m.x; my = (R)m.y; mz = (R)m.z;
          } else {
            double4 m = S.v[j];
            mx = (R)m.x; my = (R)m.y; mz = (R)m.z;
          }
          if (dd_mask) {
            dd = a.ipol[X.off + j] != 0;
          } else {
            double4 m = S.v[j];
            dd = m.x != 0 || m.y != 0 || m.z != 0;
          }
        }
        double qj = QQ ? sj.w : 0.0;
        if (!dd && (!QQ || qj == 0.0)) continue;
        es_field_pair<R, QQ, DD>(S.es, c.ntype, i, j, ti, S.t[j], rx, ry, rz, r2, (R)c.alpha, damp,
                                 qj, dd, mx, my, mz, ex, ey, ez, (c.flags & BF_THOLE) ? 1 : 0);
      }
    }
    double dx = warp_sum((double)ex), dy = warp_sum((double)ey), dz = warp_sum((double)ez);
    if (lane == 0) {
      int gi = X.off + i;
      double4 o = E[gi];
      E[gi] = make_double4(o.x + dx, o.y + dy, o.z + dz, 0.0);
    }
  }
}

// ---------------------------------------------------------------------------
// short range (FP64) on this CTA's ions: forces overwrite force[own];
// acc[16] as k_shortrange.
__device__ void bshort(const BatchArgs& a, const BCtx& X, const BShared& S, double (&acc)[kSRPart]) {
  const BConf& c = *X.c;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  const int do_bmh = (c.flags & BF_BMH) ? 1 : 0, do_lj = (c.flags & BF_LJ) ? 1 : 0;
  const int lbmhftd = (c.flags & BF_BMHFTD) ? 1 : 0;
  for (int k = 0; k < kSRPart; ++k) acc[k] = 0.0;
  for (int i = X.i0 + warp; i < X.i1; i += nwarp) {
    double4 si = S.s[i];
    int ti = S.t[i];
    double fb[3] = {0, 0, 0}, fl[3] = {0, 0, 0};
    for (int j = lane; j < X.n; j += 32) {
      if (j == i) continue;
      double4 sj = S.s[j];
      double rx, ry, rz;
      double r2 = min_image_exact(c.A, xsub(si.x, sj.x), xsub(si.y, sj.y), xsub(si.z, sj.z), rx,
                                  ry, rz);
      const NBPair& P = S.nb[ti * c.ntype + S.t[j]];
      if (r2 >= P.rcutsq) continue;  // non_bonded.f90:1154 strict <
      if (do_bmh && (P.A != 0.0 || P.wall != 0.0)) {
        double u, wij;
        sr_pair_bmh<double>(P, lbmhftd, r2, u, wij);
        double fx = wij * rx, fy = wij * ry, fz = wij * rz;
        fb[0] += fx;
        fb[1] += fy;
        fb[2] += fz;
        acc[0] += 0.5 * u;
        acc[1] += 0.5 * (rx * fx + ry * fy + rz * fz);
        acc[4] += rx * fx;
        acc[5] += ry * fy;
        acc[6] += rz * fz;
        acc[7] += 0.5 * (rx * fy + ry * fx);
        acc[8] += 0.5 * (rx * fz + rz * fx);
        acc[9] += 0.5 * (ry * fz + rz * fy);
      }
      if (do_lj) {
        double e, wij;
        sr_pair_lj<double>(P, c.trunc, r2, e, wij);
        double fx = wij * rx, fy = wij * ry, fz = wij * rz;
        fl[0] += fx;
        fl[1] += fy;
        fl[2] += fz;
        acc[2] += 0.5 * e;
        acc[3] += 0.5 * (wij * r2);
        acc[10] += rx * fx;
        acc[11] += ry * fy;
        acc[12] += rz * fz;
        acc[13] += 0.5 * (rx * fy + ry * fx);
        acc[14] += 0.5 * (rx * fz + rz * fx);
        acc[15] += 0.5 * (ry * fz + rz * fy);
      }
    }
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      fb[d] = warp_sum(fb[d]);
      fl[d] = warp_sum(fl[d]);
    }
    if (lane == 0) {
      const double* f = do_bmh ? fb : fl;  // non_bonded.f90:699-701, 1104-1106
      int gi = X.off + i;
      a.force[gi] = f[0];
      a.force[a.ntot + gi] = f[1];
      a.force[2 * (size_t)a.ntot + gi] = f[2];
    }
  }
}

// final real-space pass (k_es_force) on this CTA's ions; mu in S.v (FP64).
template <typename R>
__device__ void bforce(const BatchArgs& a, const BCtx& X, const BShared& S, double (&acc)[kESPart]) {
  const BConf& c = *X.c;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  const int task_qq = (c.flags & BF_QQ) ? 1 : 0, task_qd = (c.flags & BF_QD) ? 1 : 0;
  const int task_dd = (c.flags & BF_DD) ? 1 : 0;
  for (int k = 0; k < kESPart; ++k) acc[k] = 0.0;
  for (int i = X.i0 + warp; i < X.i1; i += nwarp) {
    double4 si = S.s[i];
    int ti = S.t[i];
    double qi = si.w;
    double4 mui = S.v[i];
    double e[3] = {0, 0, 0}, f[3] = {0, 0, 0};
    for (int j = lane; j < X.n; j += 32) {
      if (j == i) continue;
      double4 sj = S.s[j];
      double rxd, ryd, rzd;
      double r2d = min_image_exact(c.A, xsub(si.x, sj.x), xsub(si.y, sj.y), xsub(si.z, sj.z), rxd,
                                   ryd, rzd);
      if (r2d > c.rc2) continue;
      int tj = S.t[j];
      double qj = sj.w;
      double4 muj = S.v[j];
      bool i_is_a = half_mask(i, j);
      const ESPair& P = S.es[(i_is_a ? ti : tj) * c.ntype + (i_is_a ? tj : ti)];
      R r[3] = {(R)rxd, (R)ryd, (R)rzd};
      R mi[3] = {(R)mui.x, (R)mui.y, (R)mui.z}, mj[3] = {(R)muj.x, (R)muj.y, (R)muj.z};
      bool dip_i = (mui.x != 0.0 || mui.y != 0.0 || mui.z != 0.0);
      bool dip_j = (muj.x != 0.0 || muj.y != 0.0 || muj.z != 0.0);
      R u, fi[3], Ei[3];
      // the single engine's pair (i's frame; Thole on the dd field and energy
      // where the pair's table entry has it)
      es_force_ipair<R, 0, true>(P, i_is_a, P.ldamp != 0, (R)r2d, (R)c.alpha, r, (R)qi, (R)qj, mi,
                                 mj, dip_i, dip_j, task_qq, task_qd, task_dd, u, fi, Ei);
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        f[d] += (double)fi[d];
        e[d] += (double)Ei[d];
      }
      acc[0] += 0.5 * (double)u;
      acc[1] += (double)(r[0] * fi[0]);
      acc[2] += (double)(r[1] * fi[1]);
      acc[3] += (double)(r[2] * fi[2]);
      acc[4] += 0.5 * (double)(r[0] * fi[1] + r[1] * fi[0]);
      acc[5] += 0.5 * (double)(r[0] * fi[2] + r[2] * fi[0]);
      acc[6] += 0.5 * (double)(r[1] * fi[2] + r[2] * fi[1]);
    }
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      e[d] = warp_sum(e[d]);
      f[d] = warp_sum(f[d]);
    }
    if (lane == 0) {
      int gi = X.off + i;
      a.E[gi] = make_double4(e[0], e[1], e[2], 0.0);
      a.force[gi] += f[0] * c.coul_unit;
      a.force[a.ntot + gi] += f[1] * c.coul_unit;
      a.force[2 * (size_t)a.ntot + gi] += f[2] * c.coul_unit;
    }
  }
}

__device__ __forceinline__ double4 bmat3(const double* m, double4 v) {
  return make_double4(m[0] * v.x + m[1] * v.y + m[2] * v.z, m[3] * v.x + m[4] * v.y + m[5] * v.z,
                      m[6] * v.x + m[7] * v.y + m[8] * v.z, 0.0);
}

// self (+ surface) field of the vector v on own ions: E += 2 selfa2 v_i
// (- fpi_3V (qtot + vtot) with lsurf), ewald.f90:182-213
__device__ void bself(const BatchArgs& a, const BCtx& X, const double4* __restrict__ v, double selfa2,
                      bool lsurf, double fpi_3V, const double* tot, double4* __restrict__ E) {
  for (int i = X.i0 + threadIdx.x; i < X.i1; i += blockDim.x) {
    int gi = X.off + i;
    double4 m = v[gi];
    double s0 = 0.0, s1 = 0.0, s2 = 0.0;
    if (lsurf) {
      s0 = -(tot[0] + tot[3]) * fpi_3V;
      s1 = -(tot[1] + tot[4]) * fpi_3V;
      s2 = -(tot[2] + tot[5]) * fpi_3V;
    }
    double4 o = E[gi];
    E[gi] = make_double4(o.x + s0 + 2.0 * selfa2 * m.x, o.y + s1 + 2.0 * selfa2 * m.y,
                         o.z + s2 + 2.0 * selfa2 * m.z, 0.0);
  }
}

// moments [sum q r (3), sum v (3), sum q^2, sum v^2] over the cluster
__device__ void bmoments(cgx::cluster_group& cl, const BatchArgs& a, BCtx& X, const BShared& S,
                         const double4* __restrict__ v, bool has_q, double (&m)[8]) {
  for (int k = 0; k < 8; ++k) m[k] = 0.0;
  for (int i = X.i0 + threadIdx.x; i < X.i1; i += blockDim.x) {
    int gi = X.off + i;
    double qi = has_q ? S.s[i].w : 0.0;
    double4 u = v ? v[gi] : make_double4(0, 0, 0, 0);
    m[0] += qi * a.pos[gi];
    m[1] += qi * a.pos[a.ntot + gi];
    m[2] += qi * a.pos[2 * (size_t)a.ntot + gi];
    m[3] += u.x;
    m[4] += u.y;
    m[5] += u.z;
    m[6] += qi * qi;
    m[7] += u.x * u.x + u.y * u.y + u.z * u.z;
  }
  cluster_sum<8>(cl, X, S, m);
}

// T v (field of a dipole set alone: dd undamped between polarisable ions,
// reciprocal dipole part, self / surface) on own ions into Tv.  The vector
// must be in global memory (vg) for all ions of the box; it is gathered here.
template <typename R>
__device__ void bmatvec(cgx::cluster_group& cl, const BatchArgs& a, BCtx& X, const BShared& S,
                        const double4* __restrict__ vg, double4* __restrict__ Tv) {
  const BConf& c = *X.c;
  cl.sync();  // every CTA's slice of vg is written
  gather_vec(X, vg, S.v);
  if (sizeof(R) == 4) gather_vec32(X, vg, S.v32);
  for (int i = X.i0 + threadIdx.x; i < X.i1; i += blockDim.x) Tv[X.off + i] = make_double4(0, 0, 0, 0);
  __syncthreads();
  double es[7];
  brec<R>(cl, a, X, S, false, true, false, false, Tv, nullptr, es);
  __syncthreads();
  bfield<R, false, true>(a, X, S, 0, 1, Tv);
  double tot[6] = {0, 0, 0, 0, 0, 0};
  if (c.flags & BF_SURF) {
    double m[8];
    bmoments(cl, a, X, S, vg, false, m);
    for (int k = 0; k < 6; ++k) tot[k] = m[k];
  }
  __syncthreads();
  double al = c.alpha;
  double selfa2 = 2.0 * (al / sqrt(kPi)) * al * al / 3.0;
  bself(a, X, vg, selfa2, (c.flags & BF_SURF) != 0, 2.0 * (kTwoPi / c.omega / 3.0), tot, Tv);
  __syncthreads();
}

// PCG on (alpha^-1 - T) x = b over the polarisable ions of the configuration,
// x holding the first guess.  The true residual is formed with the FP64
// operator; with MIXED the inner iterations use the FP32 operator and stop
// at 1e-4 of that residual (iterative refinement), else they run to tol.
// Stops on the reference's rmsd measure (get_rmsd_mu, moment_from_pola.f90:
// 998-1027) <= tol, or after maxit inner iterations / 8 refinements.
template <bool MIXED>
__device__ void bsolve(cgx::cluster_group& cl, const BatchArgs& a, BCtx& X, const BShared& S,
                       const double4* __restrict__ b, double4* __restrict__ x, double tol,
                       int maxit, int& iters, double& rmsd) {
  typedef typename std::conditional<MIXED, float, double>::type RM;
  const BConf& c = *X.c;
  const double npol = (double)max(c.npol, 1);
  int outer = 0;
  iters = 0;
  while (true) {
    // true residual with the FP64 operator
    bmatvec<double>(cl, a, X, S, x, a.p);
    double v2[2] = {0.0, 0.0};
    for (int i = X.i0 + threadIdx.x; i < X.i1; i += blockDim.x) {
      int gi = X.off + i;
      double4 ri = make_double4(0, 0, 0, 0), zi = make_double4(0, 0, 0, 0);
      if (a.ipol[gi]) {
        double4 ax = bmat3(a.inv + 9 * (size_t)gi, x[gi]);
        double4 bi = b[gi], tx = a.p[gi];
        ri = make_double4(bi.x + tx.x - ax.x, bi.y + tx.y - ax.y, bi.z + tx.z - ax.z, 0.0);
        zi = bmat3(a.pol + 9 * (size_t)gi, ri);
        const double* pl = a.pol + 9 * (size_t)gi;
        double rr[3] = {ri.x, ri.y, ri.z};
        for (int d = 0; d < 3; ++d)
          if (pl[4 * d] != 0.0) v2[1] += rr[d] * rr[d];
      }
      a.r[gi] = ri;
      a.z[gi] = zi;
      a.p[gi] = zi;
      v2[0] += ri.x * zi.x + ri.y * zi.y + ri.z * zi.z;
    }
    cluster_sum<2>(cl, X, S, v2);
    double rz = v2[0];
    rmsd = sqrt(v2[1] / npol);
    if (rmsd <= tol || iters >= maxit || outer >= 8) break;
    ++outer;
    // FP64 operator: the recurrence residual is final.  FP32 operator: trusted
    // to half the tolerance when the starting residual is small (the drift from
    // the true residual is ~ the FP32 matvec error times that start), else a
    // 1e-4 reduction and a new FP64 residual (iterative refinement).
    const double kGap = 3e-6;
    const bool trust = !MIXED || kGap * rmsd <= 0.5 * tol;
    const double tol_in = !MIXED ? tol : (trust ? 0.5 * tol : fmax(tol, 1e-4 * rmsd));
    double rms_last = rmsd;
    while (true) {
      // Tp into Estat-free scratch: a.E (own rows) holds T p
      bmatvec<RM>(cl, a, X, S, a.p, a.E);
      double pq[1] = {0.0};
      for (int i = X.i0 + threadIdx.x; i < X.i1; i += blockDim.x) {
        int gi = X.off + i;
        double4 qi = make_double4(0, 0, 0, 0);
        if (a.ipol[gi]) {
          double4 ap = bmat3(a.inv + 9 * (size_t)gi, a.p[gi]);
          double4 tp = a.E[gi];
          qi = make_double4(ap.x - tp.x, ap.y - tp.y, ap.z - tp.z, 0.0);
        }
        a.E[gi] = qi;  // q = A p
        double4 pi = a.p[gi];
        pq[0] += pi.x * qi.x + pi.y * qi.y + pi.z * qi.z;
      }
      cluster_sum<1>(cl, X, S, pq);
      double alp = (pq[0] != 0.0) ? rz / pq[0] : 0.0;
      double u2[2] = {0.0, 0.0};
      for (int i = X.i0 + threadIdx.x; i < X.i1; i += blockDim.x) {
        int gi = X.off + i;
        if (!a.ipol[gi]) continue;
        double4 xi = x[gi], ri = a.r[gi], pi = a.p[gi], qi = a.E[gi];
        xi.x += alp * pi.x;
        xi.y += alp * pi.y;
        xi.z += alp * pi.z;
        ri.x -= alp * qi.x;
        ri.y -= alp * qi.y;
        ri.z -= alp * qi.z;
        double4 zi = bmat3(a.pol + 9 * (size_t)gi, ri);
        x[gi] = xi;
        a.r[gi] = ri;
        a.z[gi] = zi;
        u2[0] += ri.x * zi.x + ri.y * zi.y + ri.z * zi.z;
        const double* pl = a.pol + 9 * (size_t)gi;
        double rr[3] = {ri.x, ri.y, ri.z};
        for (int d = 0; d < 3; ++d)
          if (pl[4 * d] != 0.0) u2[1] += rr[d] * rr[d];
      }
      cluster_sum<2>(cl, X, S, u2);
      ++iters;
      double rms_in = sqrt(u2[1] / npol);
      rms_last = rms_in;
      if (!(rms_in > tol_in && iters < maxit)) break;
      double be = (rz != 0.0) ? u2[0] / rz : 0.0;
      rz = u2[0];
      for (int i = X.i0 + threadIdx.x; i < X.i1; i += blockDim.x) {
        int gi = X.off + i;
        double4 pi = a.p[gi], zi = a.z[gi];
        a.p[gi] = make_double4(zi.x + be * pi.x, zi.y + be * pi.y, zi.z + be * pi.z, 0.0);
      }
    }
    if (trust && (rms_last <= tol_in || iters >= maxit)) {
      rmsd = rms_last;
      break;
    }
  }
}

// ---------------------------------------------------------------------------
// one configuration, whole cluster
template <bool MIXED>
__device__ void bconfig(cgx::cluster_group& cl, const BatchArgs& a, BCtx& X, const BShared& S) {
  typedef typename std::conditional<MIXED, float, double>::type RM;
  const BConf& c = *X.c;
  double* out = a.out + (size_t)X.cfg * kBSlots;
  const bool coul = (c.flags & BF_COUL) != 0;
  // ---- load --------------------------------------------------------------
  for (int i = X.i0 + threadIdx.x; i < X.i1; i += blockDim.x) {
    int gi = X.off + i;
    double sx, sy, sz;
    kardir_exact(c.B, a.pos[gi], a.pos[a.ntot + gi], a.pos[2 * (size_t)a.ntot + gi], sx, sy, sz);
    a.s[gi] = make_double4(sx, sy, sz, a.q[gi]);
    if (coul && c.nk > 0) {
      // e^{2 pi i n s}, s wrapped to [-0.5, 0.5) (k_rec_tables)
      double sv[3] = {sx, sy, sz};
      int km[3] = {c.kx, c.ky, c.ntab - (c.kx + 1) - (c.ky + 1) - 1};
      int e0 = 0;
      for (int d = 0; d < 3; ++d) {
        double w = sv[d] - rint(sv[d]);
        for (int m = 0; m <= km[d]; ++m) {
          double sn, cs;
          sincospi(2.0 * (double)m * w, &sn, &cs);
          long long o = c.tab_off + (long long)(e0 + m) * c.tab_ld + i;
          a.tab64[o] = make_double2(cs, sn);
          if (MIXED) a.tab32[o] = make_float2((float)cs, (float)sn);
        }
        e0 += km[d] + 1;
      }
    }
  }
  for (int k = threadIdx.x; k < c.ntype * c.ntype; k += blockDim.x) {
    S.nb[k] = a.nbtab[c.nb_off + k];
    S.es[k] = a.estab[c.es_off + k];
  }
  cl.sync();
  for (int i = threadIdx.x; i < X.n; i += blockDim.x) {
    S.s[i] = ldcg4(a.s + X.off + i);
    S.t[i] = a.typ[X.off + i];
  }
  __syncthreads();
  // ---- short range -------------------------------------------------------
  {
    double acc[kSRPart];
    if (c.flags & BF_SR) {
      bshort(a, X, S, acc);
    } else {
      for (int k = 0; k < kSRPart; ++k) acc[k] = 0.0;
      for (int i = X.i0 + threadIdx.x; i < X.i1; i += blockDim.x) {
        int gi = X.off + i;
        a.force[gi] = a.force[a.ntot + gi] = a.force[2 * (size_t)a.ntot + gi] = 0.0;
      }
    }
    cluster_sum<kSRPart>(cl, X, S, acc);
    if (X.rank == 0 && threadIdx.x == 0)
      for (int k = 0; k < kSRPart; ++k) out[BS_SR + k] = acc[k];
  }
  if (!coul) {
    for (int i = X.i0 + threadIdx.x; i < X.i1; i += blockDim.x) {
      a.mu[X.off + i] = make_double4(0, 0, 0, 0);
      a.E[X.off + i] = make_double4(0, 0, 0, 0);
    }
    return;
  }
  const double al = c.alpha;
  const double selfa2 = 2.0 * (al / sqrt(kPi)) * al * al / 3.0;
  const double fpi_3V = 2.0 * (kTwoPi / c.omega / 3.0);
  const bool lsurf = (c.flags & BF_SURF) != 0;
  const bool dipst = (c.flags & BF_DIPST) != 0;
  const bool task_qq = (c.flags & BF_QQ) != 0;
  int iters = 0, conv = 1;
  double rmsd = 0.0;
  for (int i = X.i0 + threadIdx.x; i < X.i1; i += blockDim.x) a.x[X.off + i] = make_double4(0, 0, 0, 0);
  if (c.flags & BF_POLAR) {
    // ---- static field: damped charges + static dipoles --------------------
    for (int i = X.i0 + threadIdx.x; i < X.i1; i += blockDim.x)
      a.Estat[X.off + i] = make_double4(0, 0, 0, 0);
    gather_vec(X, a.dip, S.v);
    if (MIXED) gather_vec32(X, a.dip, S.v32);
    __syncthreads();
    if (task_qq && dipst) bfield<RM, true, true>(a, X, S, 1, 0, a.Estat);
    else if (task_qq) bfield<RM, true, false>(a, X, S, 1, 0, a.Estat);
    else if (dipst) bfield<RM, false, true>(a, X, S, 1, 0, a.Estat);
    __syncthreads();
    double es[7];
    brec<RM>(cl, a, X, S, task_qq, dipst, false, false, a.Estat, nullptr, es);
    double tot[6] = {0, 0, 0, 0, 0, 0};
    if (lsurf) {
      double m[8];
      bmoments(cl, a, X, S, a.dip, true, m);
      for (int k = 0; k < 6; ++k) tot[k] = m[k];
    }
    __syncthreads();
    bself(a, X, a.dip, selfa2, lsurf, fpi_3V, tot, a.Estat);
    __syncthreads();
    // ---- PCG: (alpha^-1 - T) x = E_stat, x0 = alpha E_stat ----------------
    for (int i = X.i0 + threadIdx.x; i < X.i1; i += blockDim.x) {
      int gi = X.off + i;
      a.x[gi] = a.ipol[gi] ? bmat3(a.pol + 9 * (size_t)gi, a.Estat[gi]) : make_double4(0, 0, 0, 0);
    }
    const double tol = c.tol;
    bsolve<MIXED>(cl, a, X, S, a.Estat, a.x, tol, c.maxit, iters, rmsd);
    conv = rmsd <= tol ? 1 : 0;
  }
  // ---- u_pol, total dipoles (+ Wannier centres), catastrophe -------------
  {
    const bool wfc = (c.flags & BF_WFC) != 0;
    double v[3] = {0.0, 0.0, 0.0};
    for (int i = X.i0 + threadIdx.x; i < X.i1; i += blockDim.x) {
      int gi = X.off + i;
      double4 m = a.x[gi];
      if (a.ipol[gi]) {
        const double* iv = a.inv + 9 * (size_t)gi;
        double mm[3] = {m.x, m.y, m.z};
        for (int p = 0; p < 3; ++p)
          for (int q2 = 0; q2 < 3; ++q2) v[0] += mm[p] * iv[3 * p + q2] * mm[q2];
      }
      double4 d = a.dip[gi];
      double4 t = make_double4(d.x + m.x, d.y + m.y, d.z + m.z, 0.0);
      if (wfc && c.lwfc[S.t[i]] >= 0) {
        // moment_from_WFc (moment_from_pola.f90:686-738): -2 sum (r_c - r_i)
        // over the centres c with |r|^2 < rcut_wfc, in ascending centre order
        const double4 si = S.s[i];
        double w[3] = {0.0, 0.0, 0.0};
        int cnt = 0;
        for (int j = 0; j < X.n; ++j) {
          if (c.lwfc[S.t[j]] >= 0) continue;
          const double4 sj = S.s[j];
          double rx, ry, rz;
          const double r2 = min_image_exact(c.A, xsub(sj.x, si.x), xsub(sj.y, si.y), xsub(sj.z, si.z),
                                            rx, ry, rz);
          if (r2 < c.rcut_wfc) {
            ++cnt;
            w[0] += rx;
            w[1] += ry;
            w[2] += rz;
          }
        }
        if (c.lwfc[S.t[i]] > 0 && cnt != c.lwfc[S.t[i]]) v[2] = 1.0;  // :731-737
        if (c.ldip_wfc) {
          t.x = t.x + -2.0 * w[0];
          t.y = t.y + -2.0 * w[1];
          t.z = t.z + -2.0 * w[2];
        }
      }
      a.mu[gi] = t;
      if (t.x > 10.0 || t.y > 10.0 || t.z > 10.0) v[1] = 1.0;  // moment_from_pola.f90:176-178
    }
    cluster_sum<3>(cl, X, S, v);
    if (X.rank == 0 && threadIdx.x == 0) {
      out[BS_UPOL] = v[0];
      out[BS_ITER] = iters;
      out[BS_CONV] = conv;
      out[BS_RMSD] = rmsd;
      out[BS_CATA] = v[1] > 0.0 ? 1.0 : 0.0;
      out[BS_STAT] = v[2] > 0.0 ? (double)MDFF_ERR_BAD_ARGS : 0.0;
    }
  }
  // ---- final pass: forces, energy, field, stress --------------------------
  cl.sync();
  gather_vec(X, a.mu, S.v);
  __syncthreads();
  {
    double acc[kESPart];
    bforce<RM>(a, X, S, acc);
    cluster_sum<kESPart>(cl, X, S, acc);
    if (X.rank == 0 && threadIdx.x == 0)
      for (int k = 0; k < kESPart; ++k) out[BS_DIR + k] = acc[k];
  }
  __syncthreads();
  {
    bool has_mu = (c.flags & (BF_QD | BF_DD)) != 0;
    double es[7];
    brec<RM>(cl, a, X, S, task_qq, has_mu, true, true, a.E, a.force, es);
    cluster_sum<7>(cl, X, S, es);
    if (X.rank == 0 && threadIdx.x == 0)
      for (int k = 0; k < 7; ++k) out[BS_REC + k] = es[k];
  }
  double m[8];
  bmoments(cl, a, X, S, a.mu, true, m);
  if (X.rank == 0 && threadIdx.x == 0)
    for (int k = 0; k < 8; ++k) out[BS_MOM + k] = m[k];
  __syncthreads();
  bself(a, X, a.mu, selfa2, lsurf, fpi_3V, m, a.E);
}

// Persistent kernel: one cluster per configuration at a time, configurations
// taken from the queue in descending cost order.
template <bool MIXED>
__global__ void __launch_bounds__(512) k_batch(BatchArgs a, int nmax) {
  extern __shared__ __align__(16) unsigned char bsm[];
  BShared S = batch_smem(bsm, nmax);
  cgx::cluster_group cl = cgx::this_cluster();
  BCtx X;
  X.rank = (int)cl.block_rank();
  X.C = (int)cl.num_blocks();
  X.parity = 0;
  while (true) {
    if (X.rank == 0 && threadIdx.x == 0) *S.cfg = atomicAdd(a.queue, 1);
    cl.sync();
    int qpos = *cl.map_shared_rank(S.cfg, 0);
    cl.sync();  // rank 0 may overwrite its slot only after every CTA read it
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
    bconfig<MIXED>(cl, a, X, S);
    __syncthreads();
  }
}

}  // namespace mdff
