// ko.cuh -- the kO induced-dipole algorithms of the SCF solver
// (moment_from_pola.f90:822-942, 1042-1639, 1987-2273, 2276-2529) as
// device kernels; the host side (mdff_gpu.cu) runs their loops.
//
//  * kO_v1: mu += the relaxed increment of induced_moment_inner, whose field
//    is the direct-space dipole field at alphaES = 0.001 (near neighbours
//    only), weight omegakO.
//  * kO_v2: kO_v1 followed by the line minimisation find_min along the last
//    step.
//  * kO_v4_1: the dipoles are the combination of all earlier iterates whose
//    residuals F = mu / alpha - E_ind best match E_stat (normal equations,
//    find_min_ex).
//  * extrapolate_dipole_poly: the predictor of kO_v1 / kO_v2 for
//    algo_ext_dipole = 'poly' (coefficients formed on the host).
// Vectors are double4 [natm] (xyz + pad); partial sums per 256-thread block,
// summed in a fixed order by k_reduce_partials.
#pragma once
#include "common.cuh"
#include "pim.cuh"

namespace mdff {

// mu = sum_{k < npts} c_k hist[k] (npts = 0 leaves mu as it is), then
// hist[k] = hist[k-1] for k = nshift..1 (moment_from_pola.f90:2294-2360)
__global__ void k_poly_predict(double4* __restrict__ hist, int natm, int npts, double c0, double c1,
                               double c2, double c3, double c4, int nshift,
                               double4* __restrict__ mu) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= natm) return;
  const double C[5] = {c0, c1, c2, c3, c4};
  if (npts > 0) {
    double4 s = make_double4(0, 0, 0, 0);
    for (int k = 0; k < npts; ++k) {
      double4 h = hist[(size_t)k * natm + i];
      s.x = s.x + C[k] * h.x;
      s.y = s.y + C[k] * h.y;
      s.z = s.z + C[k] * h.z;
    }
    mu[i] = s;
  }
  for (int k = nshift; k >= 1; --k) hist[(size_t)k * natm + i] = hist[(size_t)(k - 1) * natm + i];
}

// Start of induced_moment_inner (moment_from_pola.f90:858-883):
// mu = omegakO alpha f_ext on polarisable ions; partial of sum f_ext^2 over
// polarisable components (get_rmsd_mu against zero dipoles).
__global__ void k_ko_start(const double4* __restrict__ f_ext, PolDev P, int natm, double omega,
                           double4* __restrict__ mu, double* __restrict__ part) {
  __shared__ double red[32];
  double v[1] = {0.0};
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < natm) {
    double4 m = make_double4(0, 0, 0, 0);
    if (P.ipolar[i]) {
      double4 f = f_ext[i];
      m = matvec3(P.pol + 9 * (size_t)i, f);
      m = make_double4(omega * m.x, omega * m.y, omega * m.z, 0.0);
      v[0] = f.x * f.x + f.y * f.y + f.z * f.z;
    }
    mu[i] = m;
  }
  block_sum<1>(v, red);
  if (threadIdx.x == 0) part[blockIdx.x] = v[0];
}

// One pass of the inner loop (moment_from_pola.f90:890-932):
// f_tot = f_ext + (direct field of mu at alphaES = 0.001) + its self field
// 2 selfa2 mu (+ surface field -fpi_3V sum mu with lsurf, ewald.f90:182-213);
// partial of sum (mu / alpha_aa - f_tot)^2; mu <- (1 - w) mu + w alpha f_tot.
__global__ void k_ko_relax(const double4* __restrict__ f_ext, const double4* __restrict__ f_dir,
                           PolDev P, int natm, double omega, double self2, int lsurf,
                           double fpi_3V, const double* __restrict__ mom, double4* __restrict__ mu,
                           double* __restrict__ part) {
  __shared__ double red[32];
  double v[1] = {0.0};
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < natm) {
    double4 m = mu[i], fe = f_ext[i], fd = f_dir[i];
    double sx = self2 * m.x, sy = self2 * m.y, sz = self2 * m.z;
    if (lsurf) {
      sx = sx - mom[3] * fpi_3V;
      sy = sy - mom[4] * fpi_3V;
      sz = sz - mom[5] * fpi_3V;
    }
    double4 ft = make_double4(fe.x + (fd.x + sx), fe.y + (fd.y + sy), fe.z + (fd.z + sz), 0.0);
    double4 o = make_double4(0, 0, 0, 0);
    if (P.ipolar[i]) {
      const double* a = P.pol + 9 * (size_t)i;
      double mm[3] = {m.x, m.y, m.z}, ff[3] = {ft.x, ft.y, ft.z};
      for (int x = 0; x < 3; ++x) {
        double al = a[4 * x];
        if (al == 0.0) continue;
        double d = mm[x] / al - ff[x];
        v[0] += d * d;
      }
      double4 t = matvec3(a, ft);
      o = make_double4((1.0 - omega) * m.x + omega * t.x, (1.0 - omega) * m.y + omega * t.y,
                       (1.0 - omega) * m.z + omega * t.z, 0.0);
    }
    mu[i] = o;
  }
  block_sum<1>(v, red);
  if (threadIdx.x == 0) part[blockIdx.x] = v[0];
}

// f = E - mu / alpha_aa on polarisable components, other ions keep f
// (moment_from_pola.f90:1242-1249); partial of sum f^2 = get_rmsd_mu(E, mu)
__global__ void k_ko_residual(const double4* __restrict__ E, const double4* __restrict__ mu, PolDev P,
                              int natm, double4* __restrict__ f, double* __restrict__ part) {
  __shared__ double red[32];
  double v[1] = {0.0};
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < natm && P.ipolar[i]) {
    const double* a = P.pol + 9 * (size_t)i;
    double4 e = E[i], m = mu[i];
    double4 r = make_double4(e.x - m.x / a[0], e.y - m.y / a[4], e.z - m.z / a[8], 0.0);
    f[i] = r;
    v[0] = r.x * r.x + r.y * r.y + r.z * r.z;
  }
  block_sum<1>(v, red);
  if (threadIdx.x == 0) part[blockIdx.x] = v[0];
}

// find_min (moment_from_pola.f90:2415-2455), dot products over polarisable
// ions: [sum g0.g0, sum g0.(g1 - g0)]
__global__ void k_findmin_dots(const double4* __restrict__ g0, const double4* __restrict__ g1, PolDev P,
                               int natm, double* __restrict__ part) {
  __shared__ double red[2 * 32];
  double v[2] = {0.0, 0.0};
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < natm && P.ipolar[i]) {
    double4 a = g0[i], b = g1[i];
    v[0] = a.x * a.x + a.y * a.y + a.z * a.z;
    v[1] = a.x * (b.x - a.x) + a.y * (b.y - a.y) + a.z * (b.z - a.z);
  }
  block_sum<2>(v, red);
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = v[0];
    part[2 * blockIdx.x + 1] = v[1];
  }
}

// gmin = g0 + a (g1 - g0) (in place over g0), mu = mu_prev + a (mu -
// mu_prev); partial of sum gmin^2 over polarisable ions
// (moment_from_pola.f90:1553-1562)
__global__ void k_findmin_apply(double4* __restrict__ g, const double4* __restrict__ g1, double a,
                                const double4* __restrict__ mu_prev, PolDev P, int natm,
                                double4* __restrict__ mu, double* __restrict__ part) {
  __shared__ double red[32];
  double v[1] = {0.0};
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < natm) {
    double4 g0 = g[i], gg = g1[i], mp = mu_prev[i], m = mu[i];
    double4 r = make_double4(g0.x + a * (gg.x - g0.x), g0.y + a * (gg.y - g0.y), g0.z + a * (gg.z - g0.z), 0.0);
    g[i] = r;
    mu[i] = make_double4(mp.x + a * (m.x - mp.x), mp.y + a * (m.y - mp.y), mp.z + a * (m.z - mp.z), 0.0);
    if (P.ipolar[i]) v[0] = r.x * r.x + r.y * r.y + r.z * r.z;
  }
  block_sum<1>(v, red);
  if (threadIdx.x == 0) part[blockIdx.x] = v[0];
}

// partial count of nonzero dipole components (all(mu == 0), moment_from_pola.f90:2128)
__global__ void k_count_nonzero(const double4* __restrict__ mu, int natm, double* __restrict__ part) {
  __shared__ double red[32];
  double v[1] = {0.0};
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < natm) {
    double4 m = mu[i];
    v[0] = (double)((m.x != 0.0) + (m.y != 0.0) + (m.z != 0.0));
  }
  block_sum<1>(v, red);
  if (threadIdx.x == 0) part[blockIdx.x] = v[0];
}

// kO_v4_1 iterate m (0-based): F_h[m] = mu / alpha_aa - E_ind on polarisable
// ions (0 elsewhere), mu_h[m] = mu (moment_from_pola.f90:2165-2173, 2476-2477)
__global__ void k_diis_store(const double4* __restrict__ mu, const double4* __restrict__ Eind, PolDev P,
                             int natm, double4* __restrict__ Fm, double4* __restrict__ mum) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= natm) return;
  double4 m = mu[i], r = make_double4(0, 0, 0, 0);
  if (P.ipolar[i]) {
    const double* a = P.pol + 9 * (size_t)i;
    double4 e = Eind[i];
    r = make_double4(m.x / a[0] - e.x, m.y / a[4] - e.y, m.z / a[8] - e.z, 0.0);
  }
  Fm[i] = r;
  mum[i] = m;
}

// DDOTF (moment_from_pola.f90:2531-2552) of F_h[m] with F_h[j] (blockIdx.y
// = j <= m) and with E_stat (blockIdx.y = m + 1); partials [block][m + 2]
__global__ void k_diis_dots(const double4* __restrict__ Fh, int m, int natm, const int* __restrict__ ipolar,
                            const double4* __restrict__ Estat, double* __restrict__ part) {
  __shared__ double red[32];
  double v[1] = {0.0};
  int j = blockIdx.y;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < natm && ipolar[i]) {
    double4 a = Fh[(size_t)m * natm + i];
    double4 b = (j <= m) ? Fh[(size_t)j * natm + i] : Estat[i];
    v[0] = a.x * b.x + a.y * b.y + a.z * b.z;
  }
  block_sum<1>(v, red);
  if (threadIdx.x == 0) part[(size_t)blockIdx.x * (m + 2) + j] = v[0];
}

// find_min_ex combination (moment_from_pola.f90:2505-2521) and the field of
// kO_v4 (:2188-2195): mu = sum x_i mu_h[i]; F = -E_stat + sum x_i F_h[i]
// (first iterate: F = F_h[0], mu = mu_h[0]); E = -F + mu / alpha_aa on
// polarisable components (other ions keep E).
__global__ void k_diis_combine(const double4* __restrict__ Fh, const double4* __restrict__ muh,
                               const double* __restrict__ x, int m, int first, int natm,
                               const double4* __restrict__ Estat, PolDev P, double4* __restrict__ mu,
                               double4* __restrict__ E) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= natm) return;
  double4 F, u;
  if (first) {
    F = Fh[i];
    u = muh[i];
  } else {
    double t[3] = {0, 0, 0}, s[3] = {0, 0, 0};
    for (int k = 0; k < m; ++k) {
      double xk = x[k];
      double4 f = Fh[(size_t)k * natm + i], g = muh[(size_t)k * natm + i];
      t[0] = t[0] + xk * f.x;
      t[1] = t[1] + xk * f.y;
      t[2] = t[2] + xk * f.z;
      s[0] = s[0] + xk * g.x;
      s[1] = s[1] + xk * g.y;
      s[2] = s[2] + xk * g.z;
    }
    double4 es = Estat[i];
    F = make_double4(-es.x + t[0], -es.y + t[1], -es.z + t[2], 0.0);
    u = make_double4(s[0], s[1], s[2], 0.0);
  }
  mu[i] = u;
  if (P.ipolar[i]) {
    const double* a = P.pol + 9 * (size_t)i;
    E[i] = make_double4(-F.x + u.x / a[0], -F.y + u.y / a[4], -F.z + u.z / a[8], 0.0);
  }
}

}  // namespace mdff
