// recip_tc.cuh -- the FP32 structure factor of the Ewald sum on the 5th-generation
// tensor cores (tcgen05, kind::tf32, accumulator in tensor memory).
//
// rho(k) = sum_i (q_i + i k.mu_i) e^{i k.r_i}   (ewald_rec.f90:118-148)
// The tensor cores serve the FP32 CG operator, where only dipoles contribute.
// With e^{i k.r} = X_nx Y_ny Z_nz (per-ion phase tables), P = X_nx Y_ny and
// k.mu = nx m1 + ny m2 + nz m3 (m = 2 pi B^T mu), each mesh row (nx, ny) and nz:
//   rho(nx, ny, nz) = i (nx S_1 + ny S_2 + nz S_3),   S_a = sum_i P_i m_a,i Z_nz(i).
// For a tile of 64 mesh rows this is a real GEMM over the ions:
//   D[m][c] = sum_i A[m][i] B[c][i],
//   A rows m = Re P of the 64 rows, then Im P of the 64 rows (M = 128),
//   B rows c = m_a Re Z_n, m_a Im Z_n for a = 1..3, n = 0..kz (6 (kz + 1)
//   rows, zero-padded),
// and Z_{-n} = conj Z_n gives both signs of nz from the same D.
//
// Each CTA (one per SM) owns 64 mesh rows and one ion chunk.  Per block of 32
// ions, 16 warps generate A and B in shared memory in the canonical no-swizzle
// K-major layout (8-row x 16-byte core matrices), split into TF32 high and low
// parts (round-to-nearest), and one thread of a 17th warp issues the three
// products of split TF32 per k-step of 8, A_hi [B_hi | B_lo] as one product
// where N allows and A_lo B_hi; D stays in tensor memory across the whole
// chunk.  Two operand stages and three table stagings, handed over by
// mbarriers only (no CTA-wide barrier in the K loop).  The epilogue reads D (tcgen05.ld), combines
// the products in FP64 and writes per-chunk partials rho(k) in the same layout
// as the CUDA-core kernels (the consumers add the chunks in order).
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

constexpr long kWaitLimit = 1L << 22;  // try_wait polls before a wait gives up

}  // namespace tc

// B rows of one split part of the structure-factor GEMM for kz: 6 (kz + 1)
// rounded up to 32 when the high and low parts fit one MMA (2 Nr <= 256: B_hi
// and B_lo in one N = 2 Nr product, the low part's accumulator columns start
// 32-aligned), else rounded up to 16 (three products of N = Nr)
__host__ __device__ constexpr int rho_tc_nr(int kz) {
  return 2 * (((6 * (kz + 1) + 31) / 32) * 32) <= 256 ? ((6 * (kz + 1) + 31) / 32) * 32
                                                      : ((6 * (kz + 1) + 15) / 16) * 16;
}
__host__ __device__ constexpr bool rho_tc_fused(int kz) { return 2 * rho_tc_nr(kz) <= 256; }
// tensor-memory columns allocated for the accumulator (a power of two >= 32)
__host__ __device__ constexpr int rho_tc_cols(int kz) {
  return (rho_tc_fused(kz) ? 2 : 1) * rho_tc_nr(kz) <= 32    ? 32
         : (rho_tc_fused(kz) ? 2 : 1) * rho_tc_nr(kz) <= 64  ? 64
         : (rho_tc_fused(kz) ? 2 : 1) * rho_tc_nr(kz) <= 128 ? 128
                                                              : 256;
}

constexpr int kRhoTcRows = 64;                        // mesh rows per tile (A rows: Re P, Im P)
constexpr int kRhoTcKB = 32;                          // ions per K block
constexpr int kRhoTcGen = kRhoTcRows * kRhoTcKB / 4;  // operand-generating threads: one A item each
constexpr int kRhoTcThreads = kRhoTcGen + 64;         // + the MMA warp and the copy warp; one CTA per SM
constexpr int kRhoTcStg = 3;                          // table staging buffers

// bytes of one operand stage: A hi + lo (128 x KB), B hi then lo (2 Nr x KB)
__host__ __device__ constexpr int rho_tc_stage(int Nr) {
  return 2 * 128 * kRhoTcKB * 4 + 2 * Nr * kRhoTcKB * 4;
}

// table staging of one K block: rows X_0..X_kx, Y_0..Y_ky, Z_0..Z_kz of the
// phase tables (KB ions each, row stride KB x 8 + 16 bytes so that lanes on
// different rows hit different banks) and the KB weights
constexpr int kStageRow = kRhoTcKB * 8 + 16;
__host__ __device__ constexpr int rho_tc_staging(int kx, int ky, int kz) {
  return (kx + ky + kz + 3) * kStageRow + kRhoTcKB * 16;
}

// dynamic shared memory of k_rec_rho_tc: two operand stages and the table
// stagings (the epilogue's accumulator copy, 128 x (Nr + 1) floats, reuses
// them), alignment slack
__host__ __device__ constexpr size_t rho_tc_pipe_bytes(int kx, int ky, int kz) {
  return 2 * (size_t)rho_tc_stage(rho_tc_nr(kz)) + kRhoTcStg * (size_t)rho_tc_staging(kx, ky, kz);
}
__host__ __device__ constexpr size_t rho_tc_smem(int kx, int ky, int kz) {
  return (rho_tc_pipe_bytes(kx, ky, kz) > (size_t)128 * (rho_tc_nr(kz) + 1) * 4
              ? rho_tc_pipe_bytes(kx, ky, kz)
              : (size_t)128 * (rho_tc_nr(kz) + 1) * 4) +
         1024;
}
// the mesh fits one MMA's N and one CTA's shared memory
inline bool rho_tc_fits(int kx, int ky, int kz) {
  return rho_tc_nr(kz) <= 256 && rho_tc_smem(kx, ky, kz) <= 227 * 1024;
}

__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src, int bytes) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(bytes) : "memory");
}

namespace tc {
// bounded wait on an mbarrier phase that also gives up once another thread of
// the CTA has set the abort flag
__device__ __forceinline__ bool mbar_wait_ab(uint32_t bar, uint32_t parity, long limit,
                                             const volatile int* abort) {
  for (long it = 0; it < limit; ++it) {
    uint32_t ok;
    asm volatile(
        "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3; "
        "selp.b32 %0, 1, 0, p; }"
        : "=r"(ok)
        : "r"(bar), "r"(parity), "r"(kSuspendNs)
        : "memory");
    if (ok) return true;
    if (*abort) return false;
  }
  return false;
}
__device__ __forceinline__ void mbar_init_n(uint32_t bar, int count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count));
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("{ .reg .b64 st; mbarrier.arrive.shared::cta.b64 st, [%0]; }" ::"r"(bar) : "memory");
}
// the phase also waits for tx_bytes of asynchronous copies
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t tx_bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(tx_bytes) : "memory");
}
// bulk copy global -> this CTA's shared memory (no multicast), completion
// counted in bytes on the mbarrier; 16-byte aligned, size a multiple of 16
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}
}  // namespace tc

// The phase tables of the structure factor blocked by K block, once per call
// (positions fixed): block kb holds the rows X_0..X_kx, Y_0..Y_ky, Z_0..Z_kz
// of ion slots 32 kb .. 32 kb + 31 (slot s is ion imap[s], or s without a
// map; zero past nion slots), each row 32 complex values
// and 16 bytes of padding (kStageRow bytes: the bank-spread row stride of the
// staging buffers), so that one bulk copy stages a K block.
// grid = K blocks, 256 threads.
static __global__ void __launch_bounds__(256) k_rec_rho_timg(const float2* __restrict__ tab, int natm,
                                                             const int* __restrict__ imap, int nion, int kx,
                                                             int ky, int kz, float2* __restrict__ img) {
  pdl_wait();
  pdl_trigger();
  constexpr int RW = kStageRow / (int)sizeof(float2);  // row width in float2 (32 ions + padding)
  const int TR = kx + ky + kz + 3;
  float2* blk = img + (size_t)blockIdx.x * TR * RW;
  for (int e = threadIdx.x; e < TR * RW; e += blockDim.x) {
    const int t = e / RW, j = e % RW;
    const int sl = blockIdx.x * kRhoTcKB + j;
    const int i = (j < kRhoTcKB && sl < nion) ? (imap ? imap[sl] : sl) : -1;
    blk[e] = i >= 0 ? tab[(size_t)t * natm + i] : make_float2(0.f, 0.f);
  }
}

// structure factor of the dipoles on the tensor cores.  grid = (row tiles of
// 64 mesh rows, ion chunks of a multiple of 32 ions), one CTA per SM;
// part[chunk][k] = this chunk's rho(k).  The K dimension runs over ion slots
// (the polarisable ions, where the induced dipoles live; the weights ws and
// the blocked tables are in slot order).  Warps 0-15 generate the operands
// from staged tables; one thread of warp 16 issues the MMAs; one thread of
// warp 17 stages each K block's table block and weights with two bulk copies.  No CTA-wide barrier inside the K loop:
// mbarriers carry each dependency, with one arrival per generating warp,
//   tfull[b]  the tables and weights of a K block landed in staging buffer b
//             (bytes of the bulk copies),
//   sfree[b]  every warp has generated the block staged in buffer b,
//   full[s]   operand stage s written (after each lane's fence.proxy.async),
//   empty[s]  the MMAs that read stage s are complete (tcgen05.commit),
// so the copies run up to three K blocks ahead of the generation, which runs
// up to two ahead of the products.
static __global__ void __launch_bounds__(kRhoTcThreads, 1) k_rec_rho_tc(
    const float2* __restrict__ timg, const float4* __restrict__ ws, int nion, int chunk, RecMesh M,
    double2* __restrict__ part, int* __restrict__ err, const int* __restrict__ wait_cfg) {
  pdl_wait();
  pdl_trigger();
  constexpr int NG = kRhoTcGen, RPT = kRhoTcRows, KB = kRhoTcKB, KC = KB / 4, NS = kRhoTcStg;
  static_assert(RPT * KC == NG, "A items: one (row, 4 ions) per generating thread");
  extern __shared__ unsigned char smraw[];
  unsigned char* sm = (unsigned char*)(((uintptr_t)smraw + 1023) & ~(uintptr_t)1023);
  __shared__ __align__(8) uint64_t full[2], empty[2], tfull[NS], sfree[NS];
  __shared__ uint32_t tslot;
  __shared__ int abort_flag, issued_sh;
  const volatile int* abort_v = &abort_flag;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int kx = M.kmax[0], ky = M.kmax[1], kz = M.kmax[2];
  const int nzc = kz + 1;
  const int Nr = rho_tc_nr(kz);
  const bool fused = rho_tc_fused(kz);
  const int ncols = rho_tc_cols(kz);
  const int stage = rho_tc_stage(Nr);
  {
    // the launch must provide the mesh's shared memory
    uint32_t dyn;
    asm("mov.u32 %0, %%dynamic_smem_size;" : "=r"(dyn));
    if (dyn < rho_tc_smem(kx, ky, kz) || Nr > 256) {
      if (tid == 0) atomicExch(err, 2);
      return;
    }
  }
  // stage layout: A_hi (128 x KB), A_lo, then one B tile of 2 Nr rows: B_hi
  // rows [0, Nr), B_lo rows [Nr, 2 Nr) ((Nr / 8) 8-row groups of 128 bytes on)
  const int offAL = 128 * KB * 4, offB = 2 * 128 * KB * 4;
  const int NB2 = 2 * Nr;
  const uint32_t offLo = (uint32_t)(Nr / 8) * 128;
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
    issued_sh = 0;
    for (int s = 0; s < 2; ++s) {
      tc::mbar_init_n(tc::smem_u32(&full[s]), NG / 32);
      tc::mbar_init_n(tc::smem_u32(&empty[s]), 1);
    }
    for (int b = 0; b < NS; ++b) {
      tc::mbar_init_n(tc::smem_u32(&tfull[b]), 1);
      tc::mbar_init_n(tc::smem_u32(&sfree[b]), NG / 32);
    }
    asm volatile("fence.mbarrier_init.release.cluster;");
  }
  {
    // B padding rows [6 nzc, Nr) of both parts are zero in both stages
    const int padr = Nr - 6 * nzc;
    for (int e = tid; e < 4 * padr * KC; e += blockDim.x) {
      const int kc = e % KC, rest = e / KC;
      const int c = 6 * nzc + rest % padr, sp = rest / padr;
      unsigned char* S = sm + (sp >> 1) * stage + offB;
      *reinterpret_cast<uint4*>(S + tc::canon((sp & 1) * Nr + c, kc * 4, NB2)) = make_uint4(0u, 0u, 0u, 0u);
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = tslot;

  const int r0 = blockIdx.x * RPT;
  const int a0 = blockIdx.y * chunk;
  const int a1 = min(a0 + chunk, nion);
  const int kb0 = a0 / KB;
  const int nkb = (a1 - a0 + KB - 1) / KB;
  const uint32_t lboA = (128 / 8) * 128, lboB = (uint32_t)(NB2 / 8) * 128;

  if (warp < NG / 32) {
    // ---- operand generation ------------------------------------------------
    // A item of this thread: mesh row rl (fixed), ions 4 kcA .. 4 kcA + 3;
    // rows past the mesh take row (0, 0) and their products are never read
    const int rl = tid % RPT, kcA = tid / RPT;
    int nx = 0, ny = 0;
    if (r0 + rl < M.nrows) {
      int4 ri = M.rows[r0 + rl];
      nx = ri.x;
      ny = ri.y;
    }
    const int ay = ny < 0 ? -ny : ny;
    const float sy = ny < 0 ? -1.f : 1.f;  // Y_{-n} = conj Y_n
    const int xoff = nx * kStageRow + kcA * 32, yoff = (kx + 1 + ay) * kStageRow + kcA * 32;
    const uint32_t oA = tc::canon(rl, kcA * 4, 128), oAi = tc::canon(RPT + rl, kcA * 4, 128);
    // B items (at most two per thread: 3 nzc KC <= 2 NG for Nr <= 256): rows
    // (2a) nzc + n = m_a Re Z_n and (2a + 1) nzc + n = m_a Im Z_n, ions 4 kc ..;
    // consecutive threads take consecutive n (rows 16 bytes apart)
    const int nB = 3 * nzc * KC;
    int zoff[2], woff[2];
    uint32_t oB[2], oBi[2];
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      const int it = tid + q * NG;
      const int n = it % nzc, rest = it / nzc;
      const int kc = rest % KC, a = rest / KC;
      zoff[q] = (kx + 1 + ky + 1 + n) * kStageRow + kc * 32;
      woff[q] = TR * kStageRow + kc * 64 + (a + 1) * 4;  // weight component m_a of ion 4 kc
      oB[q] = tc::canon(2 * a * nzc + n, kc * 4, NB2);
      oBi[q] = tc::canon((2 * a + 1) * nzc + n, kc * 4, NB2);
    }
    // polls of the wait for a free operand stage: tc::kWaitLimit unless the
    // host set a limit (a test hook)
    const long opwait = *wait_cfg >= 0 ? (long)*wait_cfg : tc::kWaitLimit;
    // the warp leaves the loop together: a wait counts when every lane's did
    auto warp_ok = [](bool ok) { return __all_sync(0xffffffffu, ok) != 0; };
    for (int kb = 0; kb < nkb; ++kb) {
      const int st = kb & 1, b = kb % NS;
      if (!warp_ok(tc::mbar_wait_ab(tc::smem_u32(&tfull[b]), (kb / NS) & 1, tc::kWaitLimit, abort_v))) {
        abort_flag = 1;
        break;
      }
      // operand stage st is free once the MMAs of block kb - 2 completed
      if (kb >= 2 && !warp_ok(tc::mbar_wait_ab(tc::smem_u32(&empty[st]), ((kb - 2) >> 1) & 1, opwait, abort_v))) {
        abort_flag = 1;
        break;
      }
      unsigned char* S = sm + st * stage;
      const unsigned char* T = stg0 + b * sbytes;
      {
        const float4* Xr = reinterpret_cast<const float4*>(T + xoff);
        const float4* Yr = reinterpret_cast<const float4*>(T + yoff);
        const float4 x01 = Xr[0], x23 = Xr[1], y01 = Yr[0], y23 = Yr[1];
        const float xr[4] = {x01.x, x01.z, x23.x, x23.z}, xi[4] = {x01.y, x01.w, x23.y, x23.w};
        const float yr[4] = {y01.x, y01.z, y23.x, y23.z};
        const float yi[4] = {sy * y01.y, sy * y01.w, sy * y23.y, sy * y23.w};
        uint32_t ph[4], pl[4], qh[4], ql[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          tc::tf32_split(xr[u] * yr[u] - xi[u] * yi[u], ph[u], pl[u]);
          tc::tf32_split(xr[u] * yi[u] + xi[u] * yr[u], qh[u], ql[u]);
        }
        *reinterpret_cast<uint4*>(S + oA) = make_uint4(ph[0], ph[1], ph[2], ph[3]);
        *reinterpret_cast<uint4*>(S + offAL + oA) = make_uint4(pl[0], pl[1], pl[2], pl[3]);
        *reinterpret_cast<uint4*>(S + oAi) = make_uint4(qh[0], qh[1], qh[2], qh[3]);
        *reinterpret_cast<uint4*>(S + offAL + oAi) = make_uint4(ql[0], ql[1], ql[2], ql[3]);
      }
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        if (tid + q * NG >= nB) break;
        const float4* Zr = reinterpret_cast<const float4*>(T + zoff[q]);
        const float4 z01 = Zr[0], z23 = Zr[1];
        const float zr[4] = {z01.x, z01.z, z23.x, z23.z}, zi[4] = {z01.y, z01.w, z23.y, z23.w};
        const float* wm = reinterpret_cast<const float*>(T + woff[q]);
        uint32_t rh[4], rlo[4], ih[4], ilo[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const float m = wm[4 * u];
          tc::tf32_split(m * zr[u], rh[u], rlo[u]);
          tc::tf32_split(m * zi[u], ih[u], ilo[u]);
        }
        *reinterpret_cast<uint4*>(S + offB + oB[q]) = make_uint4(rh[0], rh[1], rh[2], rh[3]);
        *reinterpret_cast<uint4*>(S + offB + offLo + oB[q]) = make_uint4(rlo[0], rlo[1], rlo[2], rlo[3]);
        *reinterpret_cast<uint4*>(S + offB + oBi[q]) = make_uint4(ih[0], ih[1], ih[2], ih[3]);
        *reinterpret_cast<uint4*>(S + offB + offLo + oBi[q]) = make_uint4(ilo[0], ilo[1], ilo[2], ilo[3]);
      }
      // every lane's writes visible to the tensor core, then one arrival per
      // warp: operand stage st written, staging buffer b read
      tc::fence_async_smem();
      __syncwarp();
      if (lane == 0) {
        tc::mbar_arrive(tc::smem_u32(&full[st]));
        tc::mbar_arrive(tc::smem_u32(&sfree[b]));
      }
    }
  } else if (warp == NG / 32 + 1) {
    // ---- copies: the table block and the weights of K block kb (both in slot
    // order) into staging buffer kb % NS once every warp has generated block
    // kb - NS from it, two bulk copies
    if (lane == 0) {
      const size_t tblk = (size_t)TR * kStageRow / sizeof(float2);  // table image block, float2
      const uint32_t tbytes = (uint32_t)(TR * kStageRow), wbytes = 16u * KB;
      int copied = 0;
      for (int kb = 0; kb < nkb; ++kb) {
        const int b = kb % NS;
        if (kb >= NS && !tc::mbar_wait_ab(tc::smem_u32(&sfree[b]), (kb / NS - 1) & 1, tc::kWaitLimit, abort_v)) {
          abort_flag = 1;
          break;
        }
        const uint32_t dst = tc::smem_u32(stg0 + b * sbytes), fb = tc::smem_u32(&tfull[b]);
        tc::mbar_expect_tx(fb, tbytes + wbytes);
        tc::bulk_g2s(dst, timg + (size_t)(kb0 + kb) * tblk, tbytes, fb);
        tc::bulk_g2s(dst + tbytes, ws + (size_t)(kb0 + kb) * KB, wbytes, fb);
        copied = kb + 1;
      }
      // no copy may still be landing when the CTA leaves (after an abort):
      // wait (bounded) for the last block copied into each buffer
      for (int b = 0; b < NS && b < copied; ++b) {
        const int last = b + NS * ((copied - 1 - b) / NS);
        if (!tc::mbar_wait(tc::smem_u32(&tfull[b]), (last / NS) & 1, tc::kWaitLimit)) abort_flag = 1;
      }
    }
  } else if (lane == 0) {
    // ---- MMA issue: the three products of split TF32.  Fused: A_hi [B_hi |
    // B_lo] (N = 2 Nr: columns [0, Nr) and [Nr, 2 Nr)) and A_lo B_hi into
    // columns [0, Nr); else all three into columns [0, Nr).
    const uint32_t idesc = tc::idesc_tf32(128, Nr), idesc2 = tc::idesc_tf32(128, NB2);
    int issued = 0;
    for (int kb = 0; kb < nkb; ++kb) {
      const int st = kb & 1;
      if (!tc::mbar_wait_ab(tc::smem_u32(&full[st]), (kb >> 1) & 1, tc::kWaitLimit, abort_v)) {
        abort_flag = 1;
        break;
      }
      tc::fence_after_sync();
      const uint32_t base = tc::smem_u32(sm + st * stage);
#pragma unroll
      for (int s = 0; s < KB / 8; ++s) {
        const uint32_t oa = (uint32_t)s * 2 * lboA, ob = (uint32_t)s * 2 * lboB;
        const uint64_t aH = tc::smem_desc(base + oa, lboA, 128), aL = tc::smem_desc(base + offAL + oa, lboA, 128);
        const uint64_t bH = tc::smem_desc(base + offB + ob, lboB, 128);
        const uint32_t acc = (kb > 0 || s > 0) ? 1u : 0u;
        if (fused) {
          tc::mma_tf32(tmem, aH, bH, idesc2, acc);
        } else {
          tc::mma_tf32(tmem, aH, bH, idesc, acc);
          tc::mma_tf32(tmem, aH, tc::smem_desc(base + offB + offLo + ob, lboB, 128), idesc, 1u);
        }
        tc::mma_tf32(tmem, aL, bH, idesc, 1u);
      }
      tc::mma_commit(tc::smem_u32(&empty[st]));
      issued = kb + 1;
    }
    // the last commit covers every MMA issued before it (waited for even
    // after an abort: tensor memory is freed only once they are done)
    if (issued > 0) {
      const int last = issued - 1;
      if (!tc::mbar_wait(tc::smem_u32(&empty[last & 1]), (last >> 1) & 1, tc::kWaitLimit)) abort_flag = 1;
    }
    issued_sh = issued;
  }
  __syncthreads();
  const bool all_ok = abort_flag == 0 && issued_sh == nkb;
  if (!all_ok && tid == 0) atomicExch(err, 1);
  // epilogue: D (128 lanes x Nr columns, plus the low part's Nr when fused)
  // -> shared (row stride Nr + 1).  A generating warp w reads lane quarter
  // w % 4, column blocks w / 4, w / 4 + NG / 128, ...
  float* Dsm = reinterpret_cast<float*>(sm);
  const int ldd = Nr + 1;
  if (all_ok && nkb > 0 && warp < NG / 32) {
    tc::fence_after_sync();
    const int q = warp & 3;
    for (int cb = warp >> 2; cb * 32 < Nr; cb += NG / 128) {
      float v[32];
      const uint32_t ta = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(cb * 32);
      tc::tmem_ld32(ta, v);
      if (fused) {
        float v2[32];
        tc::tmem_ld32(ta + (uint32_t)Nr, v2);
#pragma unroll
        for (int c = 0; c < 32; ++c) v[c] += v2[c];
      }
      const int m = q * 32 + lane;
#pragma unroll
      for (int c = 0; c < 32; ++c)
        if (cb * 32 + c < Nr) Dsm[m * ldd + cb * 32 + c] = v[c];
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    tc::fence_after_sync();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols));
  }
  if (!all_ok) return;
  // rho(nz) = i (nx S1 + ny S2 + nz S3), S_a(+-n) from the four real products
  // of (Re P, Im P) with (m_a Re Z_n, m_a Im Z_n), combined in FP64
  const int nzs = 2 * kz + 1;
  for (int idx = tid; idx < RPT * nzs; idx += blockDim.x) {
    const int lr = idx / nzs, t = idx % nzs;
    const int r = r0 + lr;
    if (r >= M.nrows) continue;
    const int4 ri = M.rows[r];
    const int nz = ri.z + t;
    if (nz > kz) continue;
    const int n = nz < 0 ? -nz : nz;
    const double s = nz < 0 ? -1.0 : 1.0;
    double re = 0.0, imv = 0.0;
    if (nkb > 0) {
      const float* Dr = Dsm + (size_t)lr * ldd;
      const float* Di = Dsm + (size_t)(RPT + lr) * ldd;
      const double coef[3] = {(double)ri.x, (double)ri.y, (double)nz};
      double Tr = 0.0, Ti = 0.0;
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        const int cr = 2 * a * nzc + n, ci = (2 * a + 1) * nzc + n;
        const double Sr = (double)Dr[cr] - s * (double)Di[ci];
        const double Si = (double)Di[cr] + s * (double)Dr[ci];
        Tr += coef[a] * Sr;
        Ti += coef[a] * Si;
      }
      re = -Ti;
      imv = Tr;
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
// structure-factor chunks when no energy is needed).  The ions are all of them
// or the subset imap (the polarisable ions, where the dipole solve's operator
// needs its field).  CTA = 128 ions x a
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
// A hi + lo and two B buffers (hi + lo), each 128 x KF TF32, the Y_0..Y_ky
// phases of the CTA's 128 ions (the epilogue's), + alignment slack
__host__ __device__ constexpr size_t field_tc_smem(int KF, int ky) {
  return (size_t)6 * 128 * KF * 4 + (size_t)(ky + 1) * 128 * 8 + 1024;
}

// B tiles of the field GEMM, once per pass: tile t = [hi | lo], each 128
// columns x KF features in the canonical K-major layout (the shared-memory
// image the field kernel copies).  grid = (tiles, RPT / kBtRows): each CTA
// builds the columns of kBtRows mesh rows.  rho'(row, nz) is staged in shared
// memory, zero outside the row's nz range: from rhoA, or (npart > 0) summed
// from the structure-factor chunk partials in chunk order (rho_prime, the same
// sums as k_rec_sum), which saves that pass when no energy is needed; rho_out
// (optional) receives those rho' values.
constexpr int kBtRows = 4;

template <bool HAS_H, int KF>
static __global__ void __launch_bounds__(128) k_rec_field_btiles(RecMesh M, const double2* __restrict__ rhoA,
                                                                 const double2* __restrict__ part, int npart,
                                                                 uint32_t* __restrict__ fb,
                                                                 double2* __restrict__ rho_out) {
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
        if (rho_out) rho_out[k] = v;  // each k is staged by one CTA
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
    const float2* __restrict__ tab, const float4* __restrict__ w, int natm, const int* __restrict__ imap,
    int nion, RecMesh M,
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
    if (dyn < field_tc_smem(KF, ky) || field_tc_kf(kz) != KF) {
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
  float2* Ys = reinterpret_cast<float2*>(sm + 6 * TILE);  // [ky + 1][128]
  const int T = tend - tbeg;
  // B tile t (hi | lo, 2 TILE bytes) -> buffer b, 16-byte copies
  auto load_b = [&](int t, int b) {
    const uint4* src = reinterpret_cast<const uint4*>(fb) + (size_t)t * (2 * TILE / 16);
    uint32_t dst = tc::smem_u32(Bbuf(b));
    for (int e = tid; e < 2 * TILE / 16; e += NT) cp_async16(dst + e * 16, src + e, 16);
    asm volatile("cp.async.commit_group;" ::: "memory");
  };
  if (T > 0) load_b(tbeg, 0);
  // the ion of tile slot s (imap: a subset of the ions), -1 past the ions
  auto ion_of = [&](int s) { return s < nion ? (imap ? imap[s] : s) : -1; };

  // A: ion features, items (ion m, 4 features) with m = it % 128
  for (int it = tid; it < 128 * (KF / 4); it += NT) {
    int m = it & 127, fc = it >> 7;
    int i = ion_of(i0 + m);
    uint32_t hi[4], lo[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      int f = fc * 4 + u;
      float x = 0.f;
      if (i >= 0 && f < 2 * nzc) {
        float2 Z = tab[(zoff + (f < nzc ? f : f - nzc)) * natm + i];
        x = f < nzc ? Z.x : Z.y;
      }
      tc::tf32_split(x, hi[u], lo[u]);
    }
    uint32_t o = tc::canon(m, fc * 4, 128);
    *reinterpret_cast<uint4*>(Ahi + o) = make_uint4(hi[0], hi[1], hi[2], hi[3]);
    *reinterpret_cast<uint4*>(Alo + o) = make_uint4(lo[0], lo[1], lo[2], lo[3]);
  }
  // the epilogue's Y_ny phases of the CTA's ions (zero past the ions); made
  // visible by the barrier before the first products
  for (int e = tid; e < (ky + 1) * 128; e += NT) {
    const int a = e >> 7, i = ion_of(i0 + (e & 127));
    Ys[e] = i >= 0 ? tab[(size_t)(kx + 1 + a) * natm + i] : make_float2(0.f, 0.f);
  }
  // per-thread sums: ion m = 32 (warp & 3) + lane, column chunks (warp >> 2) and +2
  const int q = warp & 3, hh = warp >> 2;
  const int m = q * 32 + lane, ion = ion_of(i0 + m);
  const bool ion_ok = ion >= 0;
  const int ionc = ion_ok ? ion : 0;
  const float4 wi = ion_ok ? w[ion] : make_float4(0.f, 0.f, 0.f, 0.f);
  double G[3] = {0.0, 0.0, 0.0}, H[3] = {0.0, 0.0, 0.0};
  // The rows a thread visits come in non-decreasing nx.  With conj(P) =
  // conj(X_nx) conj(Y'_ny) (Y' = Y, conjugated for ny < 0) and Q = conj(Y') T,
  // the rows of one nx are accumulated in FP32,
  //   W0 = sum Q, W1 = sum ny Q, V0 = sum conj(Y') T1
  //   (+ W2 = sum ny^2 Q, V1 = sum ny conj(Y') T1, U0 = sum conj(Y') T2 with H),
  // and conj(X_nx) and the FP64 sums are applied once per nx (flush):
  //   G += (nx Im(cX W0), Im(cX W1), Im(cX V0)),
  //   H += (nx (m1 nx Re(cX W0) + m2 Re(cX W1) + m3 Re(cX V0)),
  //         m1 nx Re(cX W1) + m2 Re(cX W2) + m3 Re(cX V1),
  //         m1 nx Re(cX V0) + m2 Re(cX V1) + m3 Re(cX U0)).
  int gnx = -1;
  float2 xval = make_float2(0.f, 0.f);
  float2 W0{}, W1{}, V0{}, W2{}, V1{}, U0{};
  auto flush = [&]() {
    if (gnx >= 0) {
      const float xr = xval.x, xi = xval.y;
      auto cre = [&](float2 a) { return xr * a.x + xi * a.y; };
      auto cim = [&](float2 a) { return xr * a.y - xi * a.x; };
      const double dnx = (double)gnx;
      G[0] += dnx * (double)cim(W0);
      G[1] += (double)cim(W1);
      G[2] += (double)cim(V0);
      if (HAS_H) {
        const float fx = (float)gnx, rW0 = cre(W0), rW1 = cre(W1), rV0 = cre(V0), rV1 = cre(V1);
        H[0] += dnx * (double)(wi.y * fx * rW0 + wi.z * rW1 + wi.w * rV0);
        H[1] += (double)(wi.y * fx * rW1 + wi.z * cre(W2) + wi.w * rV1);
        H[2] += (double)(wi.y * fx * rV0 + wi.z * rV1 + wi.w * cre(U0));
      }
    }
    W0 = W1 = V0 = W2 = V1 = U0 = make_float2(0.f, 0.f);
  };
  auto epilogue = [&](int t, int b) {
#pragma unroll
    for (int cc = 0; cc < 2; ++cc) {
      int ch = hh + 2 * cc;
      // the chunk's rows and this ion's Y_ny (shared) first
      int nxr[RPC], nyr[RPC];
      float okr[RPC];
      bool rok[RPC];
      float2 Y[RPC];
#pragma unroll
      for (int jj = 0; jj < RPC; ++jj) {
        int row = t * RPT + ch * RPC + jj;
        bool ok = row < M.nrows;
        int4 ri = M.rows[ok ? row : 0];
        nxr[jj] = ri.x;
        nyr[jj] = ri.y;
        rok[jj] = ok;
        okr[jj] = (ok && ion_ok) ? 1.f : 0.f;
        int ay = ri.y < 0 ? -ri.y : ri.y;
        Y[jj] = Ys[ay * 128 + m];
      }
      float v[32];
      tc::tmem_ld32(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(b * 128 + ch * 32), v);
#pragma unroll
      for (int jj = 0; jj < RPC; ++jj) {
        if (rok[jj] && nxr[jj] != gnx) {
          flush();
          gnx = nxr[jj];
          xval = tab[(size_t)gnx * natm + ionc];
        }
        const int ny = nyr[jj];
        const float fy = (float)ny;
        const float yr = okr[jj] * Y[jj].x, yi = okr[jj] * (ny < 0 ? -Y[jj].y : Y[jj].y);
        const float* d = v + jj * CPR;
        const float qr = yr * d[0] + yi * d[1], qi = yr * d[1] - yi * d[0];
        const float vr = yr * d[2] + yi * d[3], vi = yr * d[3] - yi * d[2];
        W0.x += qr;
        W0.y += qi;
        W1.x += fy * qr;
        W1.y += fy * qi;
        V0.x += vr;
        V0.y += vi;
        if (HAS_H) {
          W2.x += fy * fy * qr;
          W2.y += fy * fy * qi;
          V1.x += fy * vr;
          V1.y += fy * vi;
          U0.x += yr * d[4] + yi * d[5];
          U0.y += yr * d[5] - yi * d[4];
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
  flush();
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
