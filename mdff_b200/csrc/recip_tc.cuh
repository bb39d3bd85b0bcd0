// recip_tc.cuh -- the FP32 structure factor of the Ewald sum on the 5th-generation
// tensor cores (tcgen05, kind::tf32, accumulator in tensor memory).
//
// rho(k) = sum_i (q_i + i k.mu_i) e^{i k.r_i}   (ewald_rec.f90:118-148)
// With e^{i k.r} = X_nx Y_ny Z_nz (per-ion phase tables) and k.mu = nx m1 + ny m2
// + nz m3 (m = 2 pi B^T mu), each mesh row (nx, ny) and each nz:
//   rho(nx, ny, nz) = sum_i U_i Z_nz(i) + nz sum_i V_i Z_nz(i),
//   U_i = (q_i + i (nx m1_i + ny m2_i)) X_nx Y_ny,   V_i = i m3_i X_nx Y_ny.
// For a tile of mesh rows this is a real GEMM over the ions:
//   D[m][c] = sum_i A[m][i] B[c][i],
//   A rows m = (component, row), components Re U, Im U, Re V, Im V,
//   B rows c = Re Z_0..Re Z_kz, Im Z_0..Im Z_kz (zero-padded to N),
// and Z_{-n} = conj Z_n gives both signs of nz from the same D.
//
// Each CTA (256 threads) owns 32 mesh rows (64 without dipoles: U only) and one
// ion chunk.  Per block of 32 ions the threads generate A and B in shared memory
// in the canonical no-swizzle K-major layout (8-row x 16-byte core matrices),
// split into TF32 high and low parts (round-to-nearest), and one thread issues
// A_hi [B_hi | B_lo] (N = 2 x 32) and A_lo B_hi per k-step of 8 (the three
// products of split TF32); D stays in tensor memory across the whole chunk.  Two stages: the
// threads fill one while the tensor core reads the other, released by
// tcgen05.commit on an mbarrier.  The epilogue reads D (tcgen05.ld), combines
// the components in FP64 and writes per-chunk partials rho(k) in the same layout
// as the CUDA-core kernels (k_rec_sum adds the chunks in order).
//
// Every wait is bounded: a wait that gives up sets err[0] = 1, the CTA stops
// issuing, waits (bounded) for what it issued, frees its tensor memory and
// returns; the host reports MDFF_ERR_TIMEOUT.
#pragma once
#include "recip.cuh"

namespace mdff {
namespace tc {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// FP32 -> TF32 bit pattern, round to nearest (ties away), low 13 bits zero
__device__ __forceinline__ uint32_t tf32_rna(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}

// x = hi + lo with hi, lo TF32 (|x - hi - lo| <= 2^-22 |x|)
__device__ __forceinline__ uint32_t tf32_round(uint32_t b) { return (b + 0x1000u) & 0xFFFFE000u; }
__device__ __forceinline__ void tf32_split(float x, uint32_t& hi, uint32_t& lo) {
  hi = tf32_round(__float_as_uint(x));
  lo = tf32_round(__float_as_uint(x - __uint_as_float(hi)));
}

// shared-memory matrix descriptor: no swizzle, K-major; lbo = byte distance of
// adjacent 16-byte K chunks, sbo = byte distance of adjacent 8-row groups
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// byte offset of element (r, k) of an R-row x 32-column K-major tile
__device__ __forceinline__ uint32_t canon(int r, int k, int R) {
  return (uint32_t)((((k >> 2) * (R >> 3) + (r >> 3)) << 7) + ((r & 7) << 4) + ((k & 3) << 2));
}

// instruction descriptor: D f32, A and B tf32, both K-major, M x N
__host__ __device__ constexpr uint32_t idesc_tf32(int M, int N) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) |
         ((uint32_t)(M >> 4) << 24);
}

// bounded wait on an mbarrier phase: each try_wait may suspend the thread for
// up to kSuspendNs before it reports, so a pending phase costs few issue slots;
// the whole wait gives up after limit tries (about limit x kSuspendNs at most)
constexpr uint32_t kSuspendNs = 1000;
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, long limit) {
  for (long it = 0; it < limit; ++it) {
    uint32_t ok;
    asm volatile(
        "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3; "
        "selp.b32 %0, 1, 0, p; }"
        : "=r"(ok)
        : "r"(bar), "r"(parity), "r"(kSuspendNs)
        : "memory");
    if (ok) return true;
  }
  return false;
}

__device__ __forceinline__ void mbar_init(uint32_t bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar));
}

__device__ __forceinline__ void mma_tf32(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc,
                                         uint32_t accumulate) {
  uint32_t z = 0;
  asm volatile(
      "{ .reg .pred p; setp.ne.b32 p, %4, 0; "
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %5, %5, %5}, p; }" ::"r"(d),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate), "r"(z));
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
               : "memory");
}

__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// 32 consecutive 32-bit columns of this warp's 32 tensor-memory lanes
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float* v) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,"
      "%15,%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]),
        "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]),
        "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int c = 0; c < 32; ++c) v[c] = __uint_as_float(r[c]);
}

constexpr int KB = 32;                 // ions per K block
constexpr long kWaitLimit = 1L << 22;  // try_wait polls before a wait gives up

// bytes of one pipeline stage: A hi + lo (128 x KB), B hi + lo (N x KB)
__host__ __device__ constexpr int stage_bytes(int N) { return 2 * 128 * KB * 4 + 2 * N * KB * 4; }

}  // namespace tc

// B rows of the structure-factor GEMM for kz: 2 (kz + 1) rounded up to 16
__host__ __device__ constexpr int rho_tc_n(int kz) { return ((2 * (kz + 1) + 15) / 16) * 16; }

// table staging of one K block: rows X_0..X_kx, Y_0..Y_ky, Z_0..Z_kz of the
// phase tables (32 ions each, row stride 272 bytes so that lanes on different
// rows hit different banks) and the 32 weights
constexpr int kStageRow = 32 * 8 + 16;
__host__ __device__ constexpr int rho_tc_staging(int kx, int ky, int kz) {
  return (kx + ky + kz + 3) * kStageRow + 32 * 16;
}

// B rows of the kernel instantiation that serves kz (32 or 64; 0: none)
__host__ __device__ constexpr int rho_tc_nb(int kz) {
  return rho_tc_n(kz) <= 32 ? 32 : (rho_tc_n(kz) <= 64 ? 64 : 0);
}

// dynamic shared memory of k_rec_rho_tc<., ., N>: two operand stages, two
// table stagings, alignment slack
__host__ __device__ constexpr size_t rho_tc_smem_n(int N, int kx, int ky, int kz) {
  return 2 * (size_t)tc::stage_bytes(N) + 2 * (size_t)rho_tc_staging(kx, ky, kz) + 1024;
}
inline size_t rho_tc_smem(int kx, int ky, int kz) { return rho_tc_smem_n(rho_tc_nb(kz), kx, ky, kz); }

// structure factor on the tensor cores.  grid = (row tiles, ion chunks),
// kRhoTcThreads threads; part[chunk][k] = this chunk's rho(k).  Requires
// N = rho_tc_n(kz) <= 64.  The table rows and weights of K block kb + 1 are
// copied to shared memory (cp.async, coalesced) while the threads generate
// block kb from the staged copy and the tensor core multiplies block kb - 1.
constexpr int kRhoTcThreads = 256;

__device__ __forceinline__ void cp_async8(uint32_t dst, const void* src, int bytes) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(dst), "l"(src), "r"(bytes) : "memory");
}
__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src, int bytes) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(bytes) : "memory");
}

template <bool HAS_Q, bool HAS_MU, int N>
static __global__ void __launch_bounds__(kRhoTcThreads) k_rec_rho_tc(
    const float2* __restrict__ tab, const float4* __restrict__ w, int natm, int chunk, RecMesh M,
    double2* __restrict__ part, int* __restrict__ err, const int* __restrict__ wait_cfg) {
  pdl_wait();
  pdl_trigger();
  constexpr int NT = kRhoTcThreads;
  constexpr int RPT = HAS_MU ? 32 : 64;         // mesh rows per tile
  constexpr int KB = tc::KB;
  constexpr int AJ = RPT * (KB / 4) / NT;       // A items (row, 4 ions) per thread
  extern __shared__ unsigned char smraw[];
  unsigned char* sm = (unsigned char*)(((uintptr_t)smraw + 1023) & ~(uintptr_t)1023);
  __shared__ __align__(8) uint64_t mbar[2];
  __shared__ uint32_t tslot;
  __shared__ int abort_flag;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int kx = M.kmax[0], ky = M.kmax[1], kz = M.kmax[2];
  const int nzc = kz + 1;
  static_assert(N == 32 || N == 64, "B rows: 32 or 64");
  // tensor memory: columns [0, N) A_hi B_hi + A_lo B_hi, [N, 2N) A_hi B_lo
  constexpr int ncols = 2 * N;
  const int stage = tc::stage_bytes(N);
  {
    // the launch must provide this instantiation's shared memory
    uint32_t dyn;
    asm("mov.u32 %0, %%dynamic_smem_size;" : "=r"(dyn));
    if (dyn < rho_tc_smem_n(N, kx, ky, kz) || rho_tc_nb(kz) != N) {
      if (threadIdx.x == 0) atomicExch(err, 2);
      return;
    }
  }
  // B is one tile of 2N rows: B_hi rows [0, N), B_lo rows [N, 2N)
  const int offAL = 128 * KB * 4, offB = 2 * 128 * KB * 4;
  const int TR = kx + ky + kz + 3;  // staged table rows
  const int sbytes = rho_tc_staging(kx, ky, kz);
  unsigned char* stg0 = sm + 2 * stage;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     tc::smem_u32(&tslot)),
                 "r"(ncols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    abort_flag = 0;
    tc::mbar_init(tc::smem_u32(&mbar[0]));
    tc::mbar_init(tc::smem_u32(&mbar[1]));
    asm volatile("fence.mbarrier_init.release.cluster;");
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = tslot;

  const int r0 = blockIdx.x * RPT;
  const int a0 = blockIdx.y * chunk;
  const int a1 = min(a0 + chunk, natm);
  // this thread's mesh row (fixed: NT is a multiple of RPT)
  const int rl = tid % RPT;
  const bool row_ok = r0 + rl < M.nrows;
  int nx = 0, ny = 0;
  if (row_ok) {
    int4 ri = M.rows[r0 + rl];
    nx = ri.x;
    ny = ri.y;
  }
  const int ay = ny < 0 ? -ny : ny;
  const float sy = ny < 0 ? -1.f : 1.f;
  const float fnx = (float)nx, fny = (float)ny;
  const float rowf = row_ok ? 1.f : 0.f;  // rows past the mesh generate zeros
  const uint32_t idesc1 = tc::idesc_tf32(128, 2 * N), idesc2 = tc::idesc_tf32(128, N);
  const uint32_t lboA = (128 / 8) * 128, lboB = (uint32_t)(2 * N / 8) * 128;

  // copy table rows t (global row t of the [X | Y | Z] tables) and weights of
  // K block kb into staging buffer kb & 1; ions past a1 are zero-filled
  // element e = tid + NT q of a block is table row t = tid / 32 + 8 q, ion
  // j = lane: the same ion for all of this thread's copies
  const size_t row_step = (size_t)(NT / 32) * natm;
  auto stage_tables = [&](int kb) {
    const int i = a0 + kb * KB + lane;
    const bool ok = i < a1;
    const int nb = ok ? 8 : 0;
    uint32_t dst = tc::smem_u32(stg0 + (kb & 1) * sbytes) + (uint32_t)(warp * kStageRow + lane * 8);
    const float2* src = tab + (size_t)warp * natm + (ok ? i : a0);
    for (int t = warp; t < TR; t += NT / 32) {
      cp_async8(dst, src, nb);
      dst += (NT / 32) * kStageRow;
      src += row_step;
    }
    if (tid < 32)
      cp_async16(tc::smem_u32(stg0 + (kb & 1) * sbytes + TR * kStageRow + lane * 16), w + (ok ? i : a0),
                 ok ? 16 : 0);
    asm volatile("cp.async.commit_group;" ::: "memory");
  };

  const int nkb = (a1 - a0 + KB - 1) / KB;
  // polls of the wait for a free operand stage: tc::kWaitLimit unless the
  // host set a limit (a test hook; the drain wait below keeps kWaitLimit)
  const long opwait = *wait_cfg >= 0 ? (long)*wait_cfg : tc::kWaitLimit;
  if (nkb > 0) stage_tables(0);
  int issued = 0;  // K blocks committed by thread 0
  for (int kb = 0; kb < nkb; ++kb) {
    const int st = kb & 1;
    unsigned char* S = sm + st * stage;
    const unsigned char* T = stg0 + st * sbytes;
    if (kb + 1 < nkb) {
      stage_tables(kb + 1);
      asm volatile("cp.async.wait_group 1;" ::: "memory");
    } else {
      asm volatile("cp.async.wait_group 0;" ::: "memory");
    }
    // one thread waits for the tensor core to release stage st; the barrier
    // holds the others
    if (kb >= 2 && tid == 0 &&
        !tc::mbar_wait(tc::smem_u32(&mbar[st]), ((kb - 2) >> 1) & 1, opwait))
      abort_flag = 1;
    __syncthreads();
    if (abort_flag) break;
    const float4* Tw = reinterpret_cast<const float4*>(T + TR * kStageRow);
#pragma unroll
    for (int j = 0; j < AJ; ++j) {
      int kc = tid / RPT + j * (NT / RPT);
      const float4* Xr = reinterpret_cast<const float4*>(T + nx * kStageRow + kc * 32);
      const float4* Yr = reinterpret_cast<const float4*>(T + (kx + 1 + ay) * kStageRow + kc * 32);
      float4 x01 = Xr[0], x23 = Xr[1], y01 = Yr[0], y23 = Yr[1];
      float2 X[4] = {make_float2(x01.x, x01.y), make_float2(x01.z, x01.w), make_float2(x23.x, x23.y),
                     make_float2(x23.z, x23.w)};
      float2 Y[4] = {make_float2(y01.x, y01.y), make_float2(y01.z, y01.w), make_float2(y23.x, y23.y),
                     make_float2(y23.z, y23.w)};
      float v[4][4];  // [component][ion]
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        float4 wi = Tw[kc * 4 + u];
        float Pr = X[u].x * Y[u].x - X[u].y * (sy * Y[u].y);
        float Pi = X[u].x * (sy * Y[u].y) + X[u].y * Y[u].x;
        float q = HAS_Q ? rowf * wi.x : 0.f;
        float km = HAS_MU ? rowf * (fnx * wi.y + fny * wi.z) : 0.f;
        float m3 = HAS_MU ? rowf * wi.w : 0.f;
        v[0][u] = q * Pr - km * Pi;
        v[1][u] = q * Pi + km * Pr;
        v[2][u] = -m3 * Pi;
        v[3][u] = m3 * Pr;
      }
#pragma unroll
      for (int c = 0; c < (HAS_MU ? 4 : 2); ++c) {
        uint32_t hi[4], lo[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) tc::tf32_split(v[c][u], hi[u], lo[u]);
        uint32_t o = tc::canon(c * RPT + rl, kc * 4, 128);
        *reinterpret_cast<uint4*>(S + o) = make_uint4(hi[0], hi[1], hi[2], hi[3]);
        *reinterpret_cast<uint4*>(S + offAL + o) = make_uint4(lo[0], lo[1], lo[2], lo[3]);
      }
    }
    // B: rows c = Re Z_c | Im Z_(c - nzc) | 0, high parts then low parts
    for (int it = tid; it < N * (KB / 4); it += NT) {
      int c = it % N, kc = it / N;
      bool im = c >= nzc;
      int n = im ? c - nzc : c;
      float z[4] = {0.f, 0.f, 0.f, 0.f};
      if (c < 2 * nzc) {
        const float4* Zr = reinterpret_cast<const float4*>(T + (kx + 1 + ky + 1 + n) * kStageRow + kc * 32);
        float4 z01 = Zr[0], z23 = Zr[1];
        z[0] = im ? z01.y : z01.x;
        z[1] = im ? z01.w : z01.z;
        z[2] = im ? z23.y : z23.x;
        z[3] = im ? z23.w : z23.z;
      }
      uint32_t hi[4], lo[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) tc::tf32_split(z[u], hi[u], lo[u]);
      *reinterpret_cast<uint4*>(S + offB + tc::canon(c, kc * 4, 2 * N)) = make_uint4(hi[0], hi[1], hi[2], hi[3]);
      *reinterpret_cast<uint4*>(S + offB + tc::canon(N + c, kc * 4, 2 * N)) = make_uint4(lo[0], lo[1], lo[2], lo[3]);
    }
    tc::fence_async_smem();
    __syncthreads();
    if (tid == 0) {
      tc::fence_after_sync();
      const uint32_t base = tc::smem_u32(S);
#pragma unroll
      for (int s = 0; s < KB / 8; ++s) {
        uint32_t oa = (uint32_t)s * 2 * lboA, ob = (uint32_t)s * 2 * lboB;
        uint64_t aH = tc::smem_desc(base + oa, lboA, 128), aL = tc::smem_desc(base + offAL + oa, lboA, 128);
        // the first N rows of the B tile are B_hi: the same descriptor with N rows
        uint64_t bB = tc::smem_desc(base + offB + ob, lboB, 128);
        tc::mma_tf32(tmem, aH, bB, idesc1, (kb > 0 || s > 0) ? 1u : 0u);
        tc::mma_tf32(tmem, aL, bB, idesc2, 1u);
      }
      tc::mma_commit(tc::smem_u32(&mbar[st]));
    }
    issued = kb + 1;
  }
  asm volatile("cp.async.wait_group 0;" ::: "memory");
  if (issued > 0 && tid == 0) {
    // the last commit covers every MMA issued before it
    int last = issued - 1;
    if (!tc::mbar_wait(tc::smem_u32(&mbar[last & 1]), (last >> 1) & 1, tc::kWaitLimit))
      abort_flag = 1;
  }
  __syncthreads();
  const bool all_ok = abort_flag == 0 && issued == nkb;
  if (!all_ok && tid == 0) atomicExch(err, 1);
  // epilogue: D (128 lanes x N columns) -> shared (row stride N + 1) -> rho.
  // Warps 0-3 read the four 32-lane quarters of tensor memory.
  float* Dsm = reinterpret_cast<float*>(sm);
  if (all_ok && nkb > 0 && warp < 4) {
    tc::fence_after_sync();
    for (int c0 = 0; c0 < N; c0 += 32) {
      float v[32], vl[32];
      tc::tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
      tc::tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(N + c0), vl);
      int m = warp * 32 + lane;
#pragma unroll
      for (int c = 0; c < 32; ++c)
        if (c0 + c < N) Dsm[m * (N + 1) + c0 + c] = v[c] + vl[c];
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    tc::fence_after_sync();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols));
  }
  if (!all_ok) return;
  const int nzs = 2 * kz + 1;
  for (int idx = tid; idx < RPT * nzs; idx += NT) {
    int lr = idx / nzs, t = idx % nzs;
    int r = r0 + lr;
    if (r >= M.nrows) continue;
    int4 ri = M.rows[r];
    int nz = ri.z + t;
    if (nz > kz) continue;
    int n = nz < 0 ? -nz : nz;
    double s = nz < 0 ? -1.0 : 1.0;
    double re = 0.0, imv = 0.0;
    if (nkb > 0) {
      const float* Ur = Dsm + (size_t)(0 * RPT + lr) * (N + 1);
      const float* Ui = Dsm + (size_t)(1 * RPT + lr) * (N + 1);
      re = (double)Ur[n] - s * (double)Ui[nzc + n];
      imv = s * (double)Ur[nzc + n] + (double)Ui[n];
      if (HAS_MU) {
        const float* Vr = Dsm + (size_t)(2 * RPT + lr) * (N + 1);
        const float* Vi = Dsm + (size_t)(3 * RPT + lr) * (N + 1);
        re += (double)nz * ((double)Vr[n] - s * (double)Vi[nzc + n]);
        imv += (double)nz * (s * (double)Vr[nzc + n] + (double)Vi[n]);
      }
    }
    part[(size_t)blockIdx.y * M.nk + ri.w + t] = make_double2(re, imv);
  }
}

}  // namespace mdff

namespace mdff {

// ===========================================================================
// Field / force partials of the FP32 reciprocal pass on the tensor cores.
//
// For ion i and mesh row (nx, ny) with P = X_nx Y_ny (ewald_rec.f90:181-250):
//   a(k) = Im(rho'_k conj(e^{i k.r_i})),  G_i = sum_k n_k a(k),
//   H_i  = sum_k n_k (k.mu_i) Re(rho'_k conj(e^{i k.r_i})).
// Over the nz of a row, with conj(Z_-n) = Z_n:
//   T  = sum_nz rho'(nz) conj(Z_nz),  T1 = sum_nz nz rho'(nz) conj(Z_nz),
//   T2 = sum_nz nz^2 rho'(nz) conj(Z_nz),
// linear in the ion features f = (Re Z_0..Re Z_kz, Im Z_0..Im Z_kz): a GEMM
//   D[i][c] = sum_f A[i][f] B[c][f]
// with A = ion features (M = 128 ions per tile, K = KF), B = per-row
// coefficients of Re T, Im T, Re T1, Im T1 (+ Re T2, Im T2 for the dipole
// force) from rho'(+n), rho'(-n).  Then per (ion, row), in FP32 from D and P:
//   S0 = Im(conj(P) T), Sz = Im(conj(P) T1)  ->  G += (nx S0, ny S0, Sz) in FP64
// and for H, with km = nx m1 + ny m2:
//   T0 = km Re(conj(P) T) + m3 Re(conj(P) T1),  Tz = km Re(conj(P) T1) + m3 Re(conj(P) T2)
//   -> H += (nx T0, ny T0, Tz).
// K is only 2 (kz + 1) features, so the FP32 accumulation in the tensor core
// is short; operands are split TF32 (A_hi B_hi + A_hi B_lo + A_lo B_hi).
//
// B tiles are built once per pass (k_rec_field_btiles, which also sums the
// structure-factor chunks when no energy is needed).  CTA = 128 ions x a
// group of row tiles (128 columns each), 256 threads: the next B tile is copied
// in (cp.async) while the tensor core multiplies the current one into one half
// of a double-buffered tensor-memory accumulator and the threads reduce the
// previous one from the other half.
constexpr int kFieldTcThreads = 256;

// features per ion (K), 32 or 64 (0: kz too large for this kernel)
__host__ __device__ constexpr int field_tc_kf(int kz) {
  return 2 * (kz + 1) <= 32 ? 32 : (2 * (kz + 1) <= 64 ? 64 : 0);
}
// rows per 128-column tile
__host__ __device__ constexpr int field_tc_rpt(bool has_h) { return has_h ? 16 : 32; }
// A hi + lo and two B buffers (hi + lo), each 128 x KF TF32, + alignment slack
__host__ __device__ constexpr size_t field_tc_smem(int KF) { return (size_t)6 * 128 * KF * 4 + 1024; }

// B tiles of the field GEMM, once per pass: tile t = [hi | lo], each 128
// columns x KF features in the canonical K-major layout (the shared-memory
// image the field kernel copies).  grid = (tiles, RPT / kBtRows): each CTA
// builds the columns of kBtRows mesh rows.  rho'(row, nz) is staged in shared
// memory, zero outside the row's nz range: from rhoA, or (npart > 0) summed
// from the structure-factor chunk partials in chunk order (rho_prime, the same
// sums as k_rec_sum), which saves that pass when no energy is needed.
constexpr int kBtRows = 4;

template <bool HAS_H, int KF>
static __global__ void __launch_bounds__(128) k_rec_field_btiles(RecMesh M, const double2* __restrict__ rhoA,
                                                                 const double2* __restrict__ part, int npart,
                                                                 uint32_t* __restrict__ fb) {
  pdl_wait();
  pdl_trigger();
  constexpr int CPR = HAS_H ? 8 : 4, RPT = 128 / CPR;
  constexpr int TILE = 128 * KF * 4;
  const int kz = M.kmax[2], nzc = kz + 1, nzs = 2 * kz + 1;
  extern __shared__ double2 rs[];  // [kBtRows][nzs]
  const int t = blockIdx.x, lr0 = blockIdx.y * kBtRows;
  for (int e = threadIdx.x; e < kBtRows * nzs; e += blockDim.x) {
    int lr = e / nzs, nz = e % nzs - kz;
    int row = t * RPT + lr0 + lr;
    double2 v = make_double2(0.0, 0.0);
    if (row < M.nrows) {
      int4 ri = M.rows[row];
      if (nz >= ri.z) {
        int k = ri.w + nz - ri.z;
        v = npart ? rho_prime(part, npart, M.Ak, M.nk, k) : rhoA[k];
      }
    }
    rs[e] = v;
  }
  __syncthreads();
  unsigned char* Bh = reinterpret_cast<unsigned char*>(fb) + (size_t)t * 2 * TILE;
  unsigned char* Bl = Bh + TILE;
  for (int it = threadIdx.x; it < kBtRows * CPR * (KF / 4); it += blockDim.x) {
    int cl = it % (kBtRows * CPR), fc = it / (kBtRows * CPR);
    int lr = cl / CPR, type = cl % CPR;
    int c = lr0 * CPR + cl;  // column in the tile
    bool ok = t * RPT + lr0 + lr < M.nrows && type < 6;
    uint32_t hi[4], lo[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      int f = fc * 4 + u;
      float x = 0.f;
      if (ok && f < 2 * nzc) {
        bool zi = f >= nzc;
        int n = zi ? f - nzc : f;
        double2 rp = rs[lr * nzs + kz + n];
        double2 rm = n > 0 ? rs[lr * nzs + kz - n] : make_double2(0.0, 0.0);
        double sr = rp.x + rm.x, si = rp.y + rm.y, dr = rp.x - rm.x, di = rp.y - rm.y;
        double fn = (double)n, c0;
        switch (type) {
          case 0: c0 = zi ? di : sr; break;
          case 1: c0 = zi ? -dr : si; break;
          case 2: c0 = fn * (zi ? si : dr); break;
          case 3: c0 = fn * (zi ? -sr : di); break;
          case 4: c0 = fn * fn * (zi ? di : sr); break;
          default: c0 = fn * fn * (zi ? -dr : si); break;
        }
        x = (float)c0;
      }
      tc::tf32_split(x, hi[u], lo[u]);
    }
    uint32_t o = tc::canon(c, fc * 4, 128);
    *reinterpret_cast<uint4*>(Bh + o) = make_uint4(hi[0], hi[1], hi[2], hi[3]);
    *reinterpret_cast<uint4*>(Bl + o) = make_uint4(lo[0], lo[1], lo[2], lo[3]);
  }
}

template <bool HAS_H, int KF>
static __global__ void __launch_bounds__(kFieldTcThreads) k_rec_field_tc(
    const float2* __restrict__ tab, const float4* __restrict__ w, int natm, RecMesh M,
    const uint32_t* __restrict__ fb, int tiles_per_group, double4* __restrict__ Gpart,
    double4* __restrict__ Hpart, int* __restrict__ err) {
  pdl_wait();
  pdl_trigger();
  constexpr int NT = kFieldTcThreads;
  constexpr int CPR = HAS_H ? 8 : 4;     // columns per mesh row (6 used with H)
  constexpr int RPT = 128 / CPR;         // mesh rows per tile
  constexpr int RPC = 32 / CPR;          // mesh rows per 32-column chunk
  constexpr int TILE = 128 * KF * 4;     // bytes of one 128-row operand
  constexpr uint32_t LBO = (128 / 8) * 128, SBO = 128;
  extern __shared__ unsigned char smraw[];
  unsigned char* sm = (unsigned char*)(((uintptr_t)smraw + 1023) & ~(uintptr_t)1023);
  __shared__ __align__(8) uint64_t mbar[2];
  __shared__ uint32_t tslot;
  __shared__ int abort_flag;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int kx = M.kmax[0], ky = M.kmax[1], kz = M.kmax[2];
  const int nzc = kz + 1;
  const size_t zoff = (size_t)(kx + 1 + ky + 1);
  {
    uint32_t dyn;
    asm("mov.u32 %0, %%dynamic_smem_size;" : "=r"(dyn));
    if (dyn < field_tc_smem(KF) || field_tc_kf(kz) != KF) {
      if (tid == 0) atomicExch(err, 2);
      return;
    }
  }
  const int ntile = (M.nrows + RPT - 1) / RPT;
  const int tbeg = blockIdx.y * tiles_per_group;
  const int tend = min(tbeg + tiles_per_group, ntile);
  const int i0 = blockIdx.x * 128;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     tc::smem_u32(&tslot)),
                 "r"(256));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    abort_flag = 0;
    tc::mbar_init(tc::smem_u32(&mbar[0]));
    tc::mbar_init(tc::smem_u32(&mbar[1]));
    asm volatile("fence.mbarrier_init.release.cluster;");
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = tslot;
  unsigned char* Ahi = sm;
  unsigned char* Alo = sm + TILE;
  auto Bbuf = [&](int b) { return sm + 2 * TILE + b * 2 * TILE; };
  const int T = tend - tbeg;
  // B tile t (hi | lo, 2 TILE bytes) -> buffer b, 16-byte copies
  auto load_b = [&](int t, int b) {
    const uint4* src = reinterpret_cast<const uint4*>(fb) + (size_t)t * (2 * TILE / 16);
    uint32_t dst = tc::smem_u32(Bbuf(b));
    for (int e = tid; e < 2 * TILE / 16; e += NT) cp_async16(dst + e * 16, src + e, 16);
    asm volatile("cp.async.commit_group;" ::: "memory");
  };
  if (T > 0) load_b(tbeg, 0);

  // A: ion features, items (ion m, 4 features) with m = it % 128
  for (int it = tid; it < 128 * (KF / 4); it += NT) {
    int m = it & 127, fc = it >> 7;
    int i = i0 + m;
    uint32_t hi[4], lo[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      int f = fc * 4 + u;
      float x = 0.f;
      if (i < natm && f < 2 * nzc) {
        float2 Z = tab[(zoff + (f < nzc ? f : f - nzc)) * natm + i];
        x = f < nzc ? Z.x : Z.y;
      }
      tc::tf32_split(x, hi[u], lo[u]);
    }
    uint32_t o = tc::canon(m, fc * 4, 128);
    *reinterpret_cast<uint4*>(Ahi + o) = make_uint4(hi[0], hi[1], hi[2], hi[3]);
    *reinterpret_cast<uint4*>(Alo + o) = make_uint4(lo[0], lo[1], lo[2], lo[3]);
  }
  // per-thread sums: ion m = 32 (warp & 3) + lane, column chunks (warp >> 2) and +2
  const int q = warp & 3, hh = warp >> 2;
  const int m = q * 32 + lane, ion = i0 + m;
  const bool ion_ok = ion < natm;
  const int ionc = ion_ok ? ion : 0;
  float4 wi = ion_ok ? w[ion] : make_float4(0.f, 0.f, 0.f, 0.f);
  double G[3] = {0.0, 0.0, 0.0}, H[3] = {0.0, 0.0, 0.0};
  auto epilogue = [&](int t, int b) {
#pragma unroll
    for (int cc = 0; cc < 2; ++cc) {
      int ch = hh + 2 * cc;
      // the chunk's rows and this ion's phases X_nx Y_ny first (loads in flight together)
      int nxr[RPC], nyr[RPC];
      float okr[RPC];
      float2 X[RPC], Y[RPC];
#pragma unroll
      for (int jj = 0; jj < RPC; ++jj) {
        int row = t * RPT + ch * RPC + jj;
        bool ok = row < M.nrows;
        int4 ri = M.rows[ok ? row : 0];
        nxr[jj] = ri.x;
        nyr[jj] = ri.y;
        okr[jj] = (ok && ion_ok) ? 1.f : 0.f;
        int ay = ri.y < 0 ? -ri.y : ri.y;
        X[jj] = tab[(size_t)ri.x * natm + ionc];
        Y[jj] = tab[(size_t)(kx + 1 + ay) * natm + ionc];
      }
      float v[32];
      tc::tmem_ld32(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(b * 128 + ch * 32), v);
#pragma unroll
      for (int jj = 0; jj < RPC; ++jj) {
        int nx = nxr[jj], ny = nyr[jj];
        float Yi = ny < 0 ? -Y[jj].y : Y[jj].y;
        float Pr = okr[jj] * (X[jj].x * Y[jj].x - X[jj].y * Yi);
        float Pi = okr[jj] * (X[jj].x * Yi + X[jj].y * Y[jj].x);
        const float* d = v + jj * CPR;
        float s0 = Pr * d[1] - Pi * d[0];
        float sz = Pr * d[3] - Pi * d[2];
        G[0] += (double)nx * (double)s0;
        G[1] += (double)ny * (double)s0;
        G[2] += (double)sz;
        if (HAS_H) {
          float reA = Pr * d[0] + Pi * d[1], reB = Pr * d[2] + Pi * d[3], reC = Pr * d[4] + Pi * d[5];
          float km = (float)nx * wi.y + (float)ny * wi.z;
          float t0 = km * reA + wi.w * reB, tz = km * reB + wi.w * reC;
          H[0] += (double)nx * (double)t0;
          H[1] += (double)ny * (double)t0;
          H[2] += (double)tz;
        }
      }
    }
  };

  const uint32_t idesc = tc::idesc_tf32(128, 128);
  int issued = 0, done = 0;  // tiles multiplied / tiles whose MMA completion was seen
  for (int k = 0; k < T; ++k) {
    const int b = k & 1;
    if (k >= 1) {
      // tile k - 1 multiplied: B buffer (k + 1) & 1 is free, its D is ready
      if (tid == 0 && !tc::mbar_wait(tc::smem_u32(&mbar[(k - 1) & 1]), ((k - 1) >> 1) & 1, tc::kWaitLimit))
        abort_flag = 1;
      __syncthreads();
      if (abort_flag) break;
      done = k;
    }
    if (k + 1 < T) {
      load_b(tbeg + k + 1, (k + 1) & 1);
      asm volatile("cp.async.wait_group 1;" ::: "memory");
    } else {
      asm volatile("cp.async.wait_group 0;" ::: "memory");
    }
    tc::fence_async_smem();
    __syncthreads();
    if (tid == 0) {
      tc::fence_after_sync();
      const uint32_t aH = tc::smem_u32(Ahi), aL = tc::smem_u32(Alo);
      const uint32_t bH = tc::smem_u32(Bbuf(b)), bL = bH + TILE;
      const uint32_t d = tmem + (uint32_t)(b * 128);
#pragma unroll
      for (int s = 0; s < KF / 8; ++s) {
        uint32_t o = (uint32_t)s * 2 * LBO;
        uint64_t dAH = tc::smem_desc(aH + o, LBO, SBO), dAL = tc::smem_desc(aL + o, LBO, SBO);
        uint64_t dBH = tc::smem_desc(bH + o, LBO, SBO), dBL = tc::smem_desc(bL + o, LBO, SBO);
        tc::mma_tf32(d, dAH, dBH, idesc, s > 0 ? 1u : 0u);
        tc::mma_tf32(d, dAH, dBL, idesc, 1u);
        tc::mma_tf32(d, dAL, dBH, idesc, 1u);
      }
      tc::mma_commit(tc::smem_u32(&mbar[b]));
    }
    issued = k + 1;
    if (k >= 1) {
      tc::fence_after_sync();
      epilogue(tbeg + k - 1, (k - 1) & 1);
    }
    tc::fence_before_sync();
  }
  asm volatile("cp.async.wait_group 0;" ::: "memory");
  if (!abort_flag && issued > done) {
    if (tid == 0 && !tc::mbar_wait(tc::smem_u32(&mbar[(issued - 1) & 1]), ((issued - 1) >> 1) & 1, tc::kWaitLimit))
      abort_flag = 1;
    __syncthreads();
    if (!abort_flag) {
      tc::fence_after_sync();
      epilogue(tbeg + issued - 1, (issued - 1) & 1);
      done = issued;
    }
  } else if (abort_flag && issued > done && tid == 0) {
    // stopped early: let the last issued MMA finish before freeing its memory
    tc::mbar_wait(tc::smem_u32(&mbar[(issued - 1) & 1]), ((issued - 1) >> 1) & 1, tc::kWaitLimit);
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    tc::fence_after_sync();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(256));
  }
  if (abort_flag) {
    if (tid == 0) atomicExch(err, 1);
    return;
  }
  // combine the two column halves of each ion (A is free: every MMA is done)
  double* red = reinterpret_cast<double*>(sm);
  if (hh == 1) {
    red[m * 6 + 0] = G[0];
    red[m * 6 + 1] = G[1];
    red[m * 6 + 2] = G[2];
    red[m * 6 + 3] = H[0];
    red[m * 6 + 4] = H[1];
    red[m * 6 + 5] = H[2];
  }
  __syncthreads();
  if (hh == 0 && ion_ok) {
    Gpart[(size_t)blockIdx.y * natm + ion] =
        make_double4(G[0] + red[m * 6 + 0], G[1] + red[m * 6 + 1], G[2] + red[m * 6 + 2], 0.0);
    if (HAS_H)
      Hpart[(size_t)blockIdx.y * natm + ion] =
          make_double4(H[0] + red[m * 6 + 3], H[1] + red[m * 6 + 4], H[2] + red[m * 6 + 5], 0.0);
  }
}

}  // namespace mdff
