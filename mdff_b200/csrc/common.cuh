// common.cuh -- device helpers shared by the engine's kernels (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define MDFF_NT 16
#define MDFF_TT_MAX 8
#define WARP 32
#define FULL_MASK 0xffffffffu

namespace mdff {

constexpr double kPi = 3.14159265358979323846264338327950;
constexpr double kTwoPi = 2.0 * kPi;

// Cell matrices in constant memory: A (direct), B (reciprocal / omega) as in
// lattice.f90:60-180, row-major [a][b] = simu_cell%A(a+1,b+1).
struct CellC {
  double A[9];
  double B[9];
  double omega;
};

// ---------------------------------------------------------------------------
// Exact (non-contracted) FP64 arithmetic for everything that decides list
// membership or cutoffs, so the GPU makes the same inclusion decisions as the
// reference's Fortran arithmetic (two roundings per multiply-add).
__device__ __forceinline__ double xmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double xadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double xsub(double a, double b) { return __dsub_rn(a, b); }

// kardir (lattice.f90:183-225): s = (x*B11 + y*B21) + z*B31, ...
__device__ __forceinline__ void kardir_exact(const double* B, double x, double y, double z,
                                             double& sx, double& sy, double& sz) {
  sx = xadd(xadd(xmul(x, B[0]), xmul(y, B[3])), xmul(z, B[6]));
  sy = xadd(xadd(xmul(x, B[1]), xmul(y, B[4])), xmul(z, B[7]));
  sz = xadd(xadd(xmul(x, B[2]), xmul(y, B[5])), xmul(z, B[8]));
}

// The fourth word of an ion's direct coordinates (s[i].w) carries its FP32
// charge (bits 0-31), type (bits 32-47) and polarisable flag (bit 48), so that
// a pair kernel's gather of a neighbour's coordinates brings them along in the
// same 32-byte sector instead of three more gathers.  Bit patterns only: no
// arithmetic is ever done on the word.
__device__ __forceinline__ double ion_tag(float q, int type, int pol) {
  unsigned long long b = (unsigned long long)(unsigned)__float_as_int(q) |
                         ((unsigned long long)(type & 0xffff) << 32) |
                         ((unsigned long long)(pol != 0) << 48);
  return __longlong_as_double((long long)b);
}
__device__ __forceinline__ int tag_type(double w) {
  return (int)((__double_as_longlong(w) >> 32) & 0xffff);
}
__device__ __forceinline__ bool tag_pol(double w) {
  return ((__double_as_longlong(w) >> 48) & 1) != 0;
}
__device__ __forceinline__ float tag_q(double w) {
  return __int_as_float((int)(__double_as_longlong(w) & 0xffffffffll));
}

// dirkar (lattice.f90:232-270): x = (s1*A11 + s2*A12) + s3*A13, ...
__device__ __forceinline__ void dirkar_exact(const double* A, double sx, double sy, double sz,
                                             double& x, double& y, double& z) {
  x = xadd(xadd(xmul(sx, A[0]), xmul(sy, A[1])), xmul(sz, A[2]));
  y = xadd(xadd(xmul(sx, A[3]), xmul(sy, A[4])), xmul(sz, A[5]));
  z = xadd(xadd(xmul(sx, A[6]), xmul(sy, A[7])), xmul(sz, A[8]));
}

// Fortran NINT: round half away from zero (C round()).
__device__ __forceinline__ double fnint(double x) { return round(x); }

// minimum image through direct coordinates (e.g. non_bonded.f90:1136-1145):
// s = ds - nint(ds); r = A s; returns r^2, all with two-rounding arithmetic.
__device__ __forceinline__ double min_image_exact(const double* A, double dsx, double dsy,
                                                  double dsz, double& rx, double& ry,
                                                  double& rz) {
  double sx = xsub(dsx, fnint(dsx));
  double sy = xsub(dsy, fnint(dsy));
  double sz = xsub(dsz, fnint(dsz));
  rx = xadd(xadd(xmul(sx, A[0]), xmul(sy, A[1])), xmul(sz, A[2]));
  ry = xadd(xadd(xmul(sx, A[3]), xmul(sy, A[4])), xmul(sz, A[5]));
  rz = xadd(xadd(xmul(sx, A[6]), xmul(sy, A[7])), xmul(sz, A[8]));
  return xadd(xadd(xmul(rx, rx), xmul(ry, ry)), xmul(rz, rz));
}

// the reference's half-list parity mask (tools.f90:318-319): the pair (i,j)
// is stored in row i (i is the "ia" role of every pair loop) iff this holds.
__device__ __forceinline__ bool half_mask(int i, int j) {
  return (i > j && (((i + j) & 1) == 0)) || (i < j && (((i + j) & 1) != 0));
}

// ---------------------------------------------------------------------------
// Numerical Recipes erfc (functions.f90:28-40); the FP64 parity path must use
// this polynomial, not the library erfc (which differs by up to ~1e-7).
template <typename R>
__device__ __forceinline__ R nr_erfc(R x);

template <>
__device__ __forceinline__ double nr_erfc<double>(double x) {
  double z = fabs(x);
  double t = 1.0 / (1.0 + 0.5 * z);
  double p = -.82215223 + t * .17087277;
  p = 1.48851587 + t * p;
  p = -1.13520398 + t * p;
  p = .27886807 + t * p;
  p = -.18628806 + t * p;
  p = .09678418 + t * p;
  p = .37409196 + t * p;
  p = 1.00002368 + t * p;
  double r = t * exp(-z * z - 1.26551223 + t * p);
  return (x < 0.0) ? 2.0 - r : r;
}

template <>
__device__ __forceinline__ float nr_erfc<float>(float x) {
  float z = fabsf(x);
  float t = 1.0f / (1.0f + 0.5f * z);
  float p = -.82215223f + t * .17087277f;
  p = 1.48851587f + t * p;
  p = -1.13520398f + t * p;
  p = .27886807f + t * p;
  p = -.18628806f + t * p;
  p = .09678418f + t * p;
  p = .37409196f + t * p;
  p = 1.00002368f + t * p;
  float r = t * expf(-z * z - 1.26551223f + t * p);
  return (x < 0.0f) ? 2.0f - r : r;
}

template <typename R>
__device__ __forceinline__ R rexp(R x);
template <>
__device__ __forceinline__ double rexp<double>(double x) { return exp(x); }
template <>
__device__ __forceinline__ float rexp<float>(float x) { return expf(x); }

template <typename R>
__device__ __forceinline__ R rsqrt_(R x);
template <>
__device__ __forceinline__ double rsqrt_<double>(double x) { return sqrt(x); }
template <>
__device__ __forceinline__ float rsqrt_<float>(float x) { return sqrtf(x); }

// 1/sqrt(x)
template <typename R>
__device__ __forceinline__ R rinv_sqrt(R x);
template <>
__device__ __forceinline__ double rinv_sqrt<double>(double x) { return rsqrt(x); }
template <>
__device__ __forceinline__ float rinv_sqrt<float>(float x) { return rsqrtf(x); }

// Tang-Toennies damping (tt_damp.f90:68-97):
//   f  = 1 - c e^{-br} sum_{k=0}^{n} (br)^k / k!
//   fd = c b e^{-br} (br)^n / n!
// with the reference's Horner order (order 0 keeps its f = 1 - c(1+br)e^{-br}).
template <typename R>
__device__ __forceinline__ void tt_damp(R b, R c, R r, int order, R& f, R& fd) {
  R br = b * r;
  R expbdr = rexp<R>(-br) * c;
  // E_TT(k) = 1/k! built as E_TT(k-1)/k (tt_damp.f90:50-53)
  R e[MDFF_TT_MAX + 1];
  e[0] = R(1);
#pragma unroll
  for (int k = 1; k <= MDFF_TT_MAX; ++k) e[k] = e[k - 1] / R(k);
  R ff = e[0];
  R pw = R(1);
  // f = E(order); for k = order-1..1: f = f*br + E(k); f = f*br + E(0)
  R acc = R(0);
#pragma unroll
  for (int k = MDFF_TT_MAX; k >= 1; --k) {
    if (k == order) acc = e[k];
    else if (k < order) acc = acc * br + e[k];
  }
  ff = (order >= 1) ? acc * br + e[0] : e[0] * br + e[0];
#pragma unroll
  for (int k = 1; k <= MDFF_TT_MAX; ++k)
    if (k <= order) pw = pw * br;
  f = R(1) - ff * expbdr;
  R eo = e[0];
#pragma unroll
  for (int k = 1; k <= MDFF_TT_MAX; ++k)
    if (k == order) eo = e[k];
  fd = eo * pw * expbdr * b;
}

// 1/k! built as the reference's E_TT table, E(k) = E(k-1) / k (tt_damp.f90:50-53)
template <typename R, int k>
__host__ __device__ constexpr R inv_fact() {
  if constexpr (k == 0)
    return R(1);
  else
    return inv_fact<R, k - 1>() / R(k);
}

// Horner sum of tt_damp.f90:80-84 for a compile-time order: acc = E(K), then
// acc = acc*br + E(k) for k = K-1 .. 1, then acc*br + E(0)
template <typename R, int K, int k>
__device__ __forceinline__ R tt_horner(R acc, R br) {
  if constexpr (k < 1) {
    return acc * br + R(1);
  } else {
    constexpr R ek = inv_fact<R, k>();
    return tt_horner<R, K, k - 1>(acc * br + ek, br);
  }
}

// Tang-Toennies damping with a compile-time order K in 1..8 (the same
// operations as tt_damp for that order, without the runtime-order selects);
// K = 0 falls back to tt_damp with the runtime order.
template <typename R, int K>
__device__ __forceinline__ void tt_damp_k(R b, R c, R r, int order, R& f, R& fd) {
  if constexpr (K == 0) {
    tt_damp<R>(b, c, r, order, f, fd);
  } else {
    static_assert(K >= 1 && K <= MDFF_TT_MAX, "TT order");
    R br = b * r;
    R expbdr = rexp<R>(-br) * c;
    constexpr R eK = inv_fact<R, K>();
    R ff = tt_horner<R, K, K - 1>(eK, br);
    R pw = br;
#pragma unroll
    for (int k = 2; k <= K; ++k) pw = pw * br;
    f = R(1) - ff * expbdr;
    fd = eK * pw * expbdr * b;
  }
}

// ---------------------------------------------------------------------------
// Programmatic dependent launch.  A kernel launched with the PDL attribute
// (pdl_launch on the host) may be scheduled while its predecessor on the
// stream is still finishing: pdl_wait(), the first statement of such a
// kernel, returns once the predecessor grid has completed and its writes are
// visible; pdl_trigger() lets this kernel's own successor be scheduled.  Both
// are no-ops in a kernel launched without the attribute.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// ---------------------------------------------------------------------------
// warp / block reductions (fixed order -> deterministic)
template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL_MASK, v, o);
  return v;
}

// Sum NV values over the block; result valid in thread 0.  smem: NV*nwarps.
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double* smem) {
  int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int k = 0; k < NV; ++k) v[k] = warp_sum(v[k]);
  __syncthreads();
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < NV; ++k) smem[k * nw + w] = v[k];
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) {
      double s = 0.0;
      for (int i = 0; i < nw; ++i) s += smem[k * nw + i];
      v[k] = s;
    }
  }
  __syncthreads();
}

// FP32 weights at the ion slots of the tensor-core structure factor: w32s[slot[i]]
// for the ions with a slot (slot[i] >= 0); inactive without w32s
struct SlotW {
  float4* w32s = nullptr;
  const int* slot = nullptr;
  __device__ __forceinline__ void put(int i, float4 v) const {
    if (w32s) {
      const int sl = slot[i];
      if (sl >= 0) w32s[sl] = v;
    }
  }
};

}  // namespace mdff
