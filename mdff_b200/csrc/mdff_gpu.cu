// mdff_gpu.cu -- the C ABI of include/mdff_gpu.h and the host-side driver of
// one engforce call (engforce_driver.f90:102-190) on a B200.
//
// One handle = one device, one stream, buffers sized at creation for 180 GB
// HBM (everything stays resident between calls: positions, the Verlet list,
// per-ion tables, ASPC history).  The only host<->device traffic of a call is
// the positions in, the forces / dipoles / fields out, and a few scalars.
#include <cuda_runtime.h>

#include <algorithm>
#include <type_traits>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/mdff_gpu.h"
#include "common.cuh"
#include "recip_tc.cuh"
#include "nlist.cuh"
#include "pim.cuh"
#include "ko.cuh"
#include "realspace.cuh"
#include "recip.cuh"
#include "setup.h"

using namespace mdff;

namespace {

constexpr int NT = MDFF_NTYPEMAX;
constexpr int kRhoThreads = 128;
constexpr int kRhoChunk = 3072;    // ions per structure-factor block (4 chunks at 12k ions: fuller waves)
constexpr int kFieldThreads = 128;
constexpr int kKoHist = 100;       // F_h, mu_h depth of scf_kO_v4 (moment_from_pola.f90:2050)

// scalar slots (device doubles, copied to the host at the end of a call)
enum {
  S_SR = 0,      // 16: short range
  S_DIR = 16,    // 7: es dir u, tau
  S_REC = 23,    // 7: rec u, tau
  S_MOM = 30,    // 8: moments of the final pass
  S_UPOL = 38,   // u_pol
  S_RMS = 39,    // SCF rmsd^2 sum
  S_CG = 40,     // 40 rz, 41 rmsd^2 (init), 42 pq, 43 rzn, 44 rmsd^2 (update),
                 // 45 inner tolerance, 46 iterations, 47 iteration cap, 48 rmsd
  S_KO = 49,     // 2: kO algorithms (inner residual, find_min dot products)
  S_MOM2 = 52,   // 8: moments of field passes
  S_DISP = 60,
  S_CGP = 64,    // CG plan of the graph: 64 rmsd of the FP64 residual, 65 stop,
                 // 66 outer iterations, 67 recurrence trusted
  S_NSCAL = 72
};

// FP32 CG: the recurrence residual drifts from the true one by about the FP32
// matvec error, a few 1e-6 of the residual it started from (see solve_cg)
constexpr double kCgGap = 3e-6;
// what a reciprocal pass does with the CG solve's accumulated rho' (rec_mode)
enum { REC_PLAIN = 0, REC_SAVE_ACC = 1, REC_NEED_RHOA = 2, REC_FROM_ACC = 3 };

thread_local std::string g_err;

}  // namespace

struct mdff_ctx {
  mdff_params p;
  int natm = 0, ntype = 0, device = 0;
  cudaStream_t st = nullptr;
  // side streams: st_sr runs the short-range pass beside the whole Coulomb
  // chain; st_rs runs the real-space half of a field or force pass beside
  // its reciprocal half.  Each is joined into st before the first kernel that
  // writes the same outputs.  Used when overlap is on (MDFF_OVERLAP unset or
  // not 0) and per-class profiling is off.
  cudaStream_t st_sr = nullptr, st_rs = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join_sr = nullptr, ev_join_rs = nullptr;
  bool overlap = true, call_overlap = false, sr_open = false, rs_open = false;
  std::string err;
  // cell / units / tasks
  double A[9], B[9], omega = 0, W[3], ANORM[3];
  double coul_unit = kCoulUnit, press_unit = kPressUnit;
  int task_qq = 0, task_qd = 0, task_dd = 0;
  int lpolar = 0, ldip_static = 0, lsr = 0, npol = 0;
  // mesh
  std::vector<int4> rows;
  int nk = 0;
  std::vector<int> rchunk;
  int max_chunk_k = 0;
  // device
  CellC* d_cell = nullptr;
  double* d_pos = nullptr;       // [3][natm]
  double4* d_s = nullptr;
  int* d_itype = nullptr;
  int* d_ipolar = nullptr;
  // the polarisable ions (ascending index): the ions where the dipole
  // solve's fields are needed
  std::vector<int> polidx;
  int* d_polidx = nullptr;
  double* d_q = nullptr;
  double* d_qzero = nullptr;
  double4* d_dipia = nullptr;
  double* d_pol = nullptr;
  double* d_invpol = nullptr;
  NBPair* d_nbtab = nullptr;
  ESPair* d_estab = nullptr;
  // list
  ListDev L{};
  int ncell = 0;
  double rskin_build = 0;
  bool have_list = false;
  double2* d_disp_part = nullptr;
  int* h_flags = nullptr;        // pinned copy of L.flags
  // recip
  int4* d_rows = nullptr;
  double* d_Ak = nullptr;
  double4* d_kvec = nullptr;
  int* d_rchunk = nullptr;
  double2* d_tab64 = nullptr;
  float2* d_tab32 = nullptr;
  double4* d_w = nullptr;
  float4* d_w32 = nullptr;
  double2* d_rho_part = nullptr;
  double2* d_rhoA = nullptr;
  // rho' of the charges and the dipoles of the CG solve, accumulated over
  // its steps (the structure factor is linear in the dipoles) for the force
  // pass; rho_acc_ok once this call's merged first residual seeded it.
  // rec_mode selects what the next reciprocal pass does with it.
  double2* d_rho_acc = nullptr;
  bool rho_acc_ok = false;
  int rec_mode = 0;
  double* d_str = nullptr;
  int n_rho_chunks = 0;
  int nsm = 0;  // SMs of the device
  // FP32 structure factor of the CG operator on the tensor cores
  // (k_rec_rho_tc): ion chunk size and count; off when the mesh does not
  // fit (6 (kz + 1) > 256 B rows, or more shared memory than one CTA has) or
  // MDFF_REC_TC=0 in the environment
  bool rho_tc = false;
  int tc_chunk = 0, n_tc_chunks = 0;
  // its phase tables blocked by K block of kRhoTcKB ions (tc_nkb blocks),
  // built per call with the FP32 tables
  float2* d_rho_timg = nullptr;
  int tc_nkb = 0;
  // its FP32 weights in slot order (written beside d_w32 by the weight and CG
  // direction kernels), and the slot of each ion (-1: none)
  float4* d_w32s = nullptr;
  int* d_polslot = nullptr;
  // FP32 reciprocal field / force partials on the tensor cores
  // (k_rec_field_tc, B tiles in d_fb); off when kz > 31 or MDFF_FIELD_TC=0
  // in the environment
  bool field_tc = false;
  uint32_t* d_fb = nullptr;
  double4* d_G = nullptr;
  double4* d_H = nullptr;
  // pim
  double4 *d_Estat = nullptr, *d_Eind = nullptr, *d_Efield = nullptr, *d_mu_ind = nullptr;
  double4 *d_mu_tot = nullptr, *d_hist = nullptr, *d_E = nullptr;
  double4 *d_r = nullptr, *d_z = nullptr, *d_pv = nullptr, *d_qv = nullptr, *d_Tp = nullptr;
  float4* d_mu32 = nullptr;      // FP32 copy of the dipoles of an FP32 pass
  float4* d_qm32 = nullptr;      // (mu_tot, q) in FP32 for the mixed final pass
  double* d_rtpos = nullptr;     // [3][natm] positions of mdff_gpu_kardir_roundtrips
  double4* d_Edd = nullptr;      // cached real-space dipole field of a CG operator (side stream)
  double* d_fsr = nullptr;       // short-range forces SoA [3][natm] (copied into d_force by ef_back)
  double4* d_hist_save = nullptr;  // ASPC history at the start of a call ([5][natm])
  // whole-step graph (run_engforce_graph)
  cudaGraph_t step_graph = nullptr;
  cudaGraphExec_t step_exec = nullptr;
  int step_gen = -1;
  int step_fp32 = -1, step_launches = 0;
  // Tang-Toennies order shared by every damped ion pair (both field roles), the
  // compile-time order of the damped real-space kernels; 0 = orders differ
  int tt_k = 0;
  // FP32 dipole-field pair cache of the mixed mode (k_static_cache), ELL [natm][cap]
  float4* d_ddr = nullptr;
  float* d_ddb1 = nullptr;
  int *d_ddj = nullptr, *d_ddn = nullptr;
  bool dd_cache_ok = false;
  double* d_efg = nullptr;       // [natm][9] electric field gradient (mdff_gpu_efg)
  // kO dipole algorithms (ko.cuh): residual f_ind, increment, find_min
  // point / previous residual (in place), previous dipoles, inner field;
  // kO_v4_1 iterates F_h, mu_h [kKoHist][natm] and their weights
  double4 *d_ko_f = nullptr, *d_ko_dmu = nullptr, *d_ko_g = nullptr, *d_ko_muprev = nullptr;
  double4 *d_ko_fdir = nullptr, *d_Fh = nullptr, *d_muh = nullptr;
  double* d_ko_x = nullptr;
  double* h_ko = nullptr;        // pinned [kKoHist + 2]
  bool have_state = false;       // an engforce has run: positions, list, dipoles valid
  // outputs / reductions
  double* d_force = nullptr;     // [3][natm]
  double* d_part = nullptr;
  double* d_part2 = nullptr;     // partial sums of the side-stream passes
  size_t part_cap = 0;
  double* d_scal = nullptr;
  double* h_scal = nullptr;      // pinned
  int* d_cata = nullptr;         // [0] catastrophe, [1] tensor-core wait gave up, [2] Wannier count,
                                 // [3] operand-wait polls of k_rec_rho_tc (-1 = default; kept across calls)
  int* h_cata = nullptr;
  // Wannier centres: per-type lwfc, the centres' dipoles of the last call
  bool lwannier = false;
  int* d_lwfc = nullptr;
  double4* d_mu_wfc = nullptr;
  double* d_pack = nullptr;      // [natm][3] staging for mu/ef output
  double* d_ekin_part = nullptr;
  // stats
  mdff_stats stats{};
  int launches = 0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  int launches_call = 0;         // kernels launched by the current API call
  // CUDA graph of one inner CG iteration inside a device-side while loop
  cudaGraph_t cg_graph = nullptr;
  cudaGraphExec_t cg_exec = nullptr;
  int cg_gen = -1;              // buffer generation the graph was built for
  int cg_fp32 = -1;
  int cg_body_launches = 0;
  int gen = 0;                  // bumped whenever device buffers are reallocated
  // MD driver state: forces in d_force belong to the positions of md_pos
  bool md_valid = false;
  const double* md_pos = nullptr;
  // per-kernel-class timing (mdff_gpu_profile)
  struct KRec {
    int cls;
    cudaEvent_t a, b;
    double work;
  };
  bool prof = false;
  std::vector<KRec> pool;
  size_t pool_used = 0;
  double kms[MDFF_NKCLASS] = {0};
  long long kl[MDFF_NKCLASS] = {0};
  double kwork[MDFF_NKCLASS] = {0};
};

enum { KC_LIST = 0, KC_SR = 1, KC_ESFIELD = 2, KC_ESFORCE = 3, KC_RHO = 4, KC_RECF = 5, KC_OTHER = 6 };

// open a timed region of class cls on the handle's stream (no-op unless profiling)
static int prof_begin(mdff_ctx* h, int cls, double work) {
  if (!h->prof) return -1;
  if (h->pool_used == h->pool.size()) {
    mdff_ctx::KRec r;
    r.cls = 0;
    r.work = 0;
    cudaEventCreate(&r.a);
    cudaEventCreate(&r.b);
    h->pool.push_back(r);
  }
  mdff_ctx::KRec& r = h->pool[h->pool_used];
  r.cls = cls;
  r.work = work;
  cudaEventRecord(r.a, h->st);
  return (int)h->pool_used++;
}
static void prof_end(mdff_ctx* h, int idx) {
  if (idx < 0) return;
  cudaEventRecord(h->pool[idx].b, h->st);
}
// after the stream is idle: fold the recorded regions into the totals
static void prof_collect(mdff_ctx* h) {
  for (size_t i = 0; i < h->pool_used; ++i) {
    float ms = 0.f;
    mdff_ctx::KRec& r = h->pool[i];
    if (cudaEventElapsedTime(&ms, r.a, r.b) == cudaSuccess) {
      h->kms[r.cls] += ms;
      h->kl[r.cls] += 1;
      h->kwork[r.cls] += r.work;
    }
  }
  h->pool_used = 0;
}

// ---------------------------------------------------------------------------
#define CK(call)                                                                       \
  do {                                                                                 \
    cudaError_t e_ = (call);                                                           \
    if (e_ != cudaSuccess) {                                                           \
      h->err = std::string(#call) + ": " + cudaGetErrorString(e_);                     \
      return MDFF_ERR_CUDA;                                                            \
    }                                                                                  \
  } while (0)

#define LAUNCH_CHECK()                                                                 \
  do {                                                                                 \
    h->launches++;                                                                     \
    cudaError_t e_ = cudaGetLastError();                                               \
    if (e_ != cudaSuccess) {                                                           \
      h->err = std::string("kernel launch: ") + cudaGetErrorString(e_);                \
      return MDFF_ERR_CUDA;                                                            \
    }                                                                                  \
  } while (0)

static inline int cdiv(long a, long b) { return (int)((a + b - 1) / b); }

template <typename T>
static int dalloc(mdff_ctx* h, T** p, size_t n) {
  if (n == 0) n = 1;
  cudaError_t e = cudaMalloc((void**)p, n * sizeof(T));
  if (e != cudaSuccess) {
    h->err = std::string("cudaMalloc: ") + cudaGetErrorString(e);
    return MDFF_ERR_NOMEM;
  }
  cudaMemsetAsync(*p, 0, n * sizeof(T), h->st);
  return MDFF_OK;
}
#define DALLOC(ptr, n)                          \
  do {                                          \
    int s_ = dalloc(h, &(ptr), (n));            \
    if (s_) return s_;                          \
  } while (0)

// launch with programmatic stream serialization (kernels that start with
// pdl_wait): the kernel may be scheduled while its predecessor on the stream
// finishes, which hides the launch latency between short dependent kernels
template <typename... KP, typename... A>
static cudaError_t pdl_launch(void (*k)(KP...), dim3 g, dim3 b, size_t smem, cudaStream_t st, A... args) {
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = g;
  cfg.blockDim = b;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, k, args...);
}

#define PDL_CHECK(call)                                                                  \
  do {                                                                                   \
    h->launches++;                                                                       \
    cudaError_t e_ = (call);                                                             \
    if (e_ != cudaSuccess) {                                                             \
      h->err = std::string("kernel launch: ") + cudaGetErrorString(e_);                  \
      return MDFF_ERR_CUDA;                                                              \
    }                                                                                    \
  } while (0)

__global__ void k_seti(int* p, int v) {
  if (threadIdx.x == 0) *p = v;
}

// AoS [natm][3] from double4
__global__ void k_pack3(const double4* __restrict__ v, int natm, double* __restrict__ out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= natm) return;
  out[3 * i] = v[i].x;
  out[3 * i + 1] = v[i].y;
  out[3 * i + 2] = v[i].z;
}
__global__ void k_unpack3(const double* __restrict__ in, int natm, double4* __restrict__ v) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= natm) return;
  v[i] = make_double4(in[3 * i], in[3 * i + 1], in[3 * i + 2], 0.0);
}

// velocity Verlet halves (prop_velocity_verlet, integration.f90:132-194)
// an engforce makes a few more round trips than SCF iterations; a count far
// above that is a caller's mistake, refused before a long launch
constexpr int kMaxRoundTrips = 1 << 20;

// count in-place kardir/dirkar round trips (lattice.f90:183-270) of SoA
// positions [3][natm], in the reference's two-rounding arithmetic
__global__ void k_kardir_roundtrips(double* __restrict__ pos, int natm,
                                    const CellC* __restrict__ cell, int count) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= natm) return;
  double x = pos[i], y = pos[natm + i], z = pos[2 * natm + i];
  for (int k = 0; k < count; ++k) {
    double sx, sy, sz;
    kardir_exact(cell->B, x, y, z, sx, sy, sz);
    dirkar_exact(cell->A, sx, sy, sz, x, y, z);
  }
  pos[i] = x;
  pos[natm + i] = y;
  pos[2 * natm + i] = z;
}

__global__ void k_vv_kick_drift(double* __restrict__ pos, double* __restrict__ vel,
                                const double* __restrict__ f, const double* __restrict__ invm,
                                int natm, double dt) {
  pdl_wait();
  pdl_trigger();
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= natm) return;
  for (int a = 0; a < 3; ++a) {
    size_t k = (size_t)a * natm + i;
    double v = vel[k] + 0.5 * dt * f[k] * invm[i];
    vel[k] = v;
    pos[k] += dt * v;
  }
}
__global__ void k_vv_kick(double* __restrict__ vel, const double* __restrict__ f,
                          const double* __restrict__ invm, int natm, double dt,
                          double* __restrict__ part) {
  pdl_wait();
  pdl_trigger();
  __shared__ double red[32];
  double e[1] = {0.0};
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < natm) {
    for (int a = 0; a < 3; ++a) {
      size_t k = (size_t)a * natm + i;
      double v = vel[k] + 0.5 * dt * f[k] * invm[i];
      vel[k] = v;
      e[0] += 0.5 * v * v / invm[i];
    }
  }
  block_sum<1>(e, red);
  if (threadIdx.x == 0) part[blockIdx.x] = e[0];
}

// ---------------------------------------------------------------------------
// set-up (host): the reference's *_init routines

// lattice (lattice.f90:60-130): B = reciprocal / omega, face widths, norms
static void lattice(mdff_ctx* h, const double* Ain) {
  Lattice L;
  lattice_of(Ain, L);
  memcpy(h->A, L.A, sizeof(L.A));
  memcpy(h->B, L.B, sizeof(L.B));
  memcpy(h->W, L.W, sizeof(L.W));
  memcpy(h->ANORM, L.ANORM, sizeof(L.ANORM));
  h->omega = L.omega;
}

// k mesh as rows (nx, ny) of consecutive nz (kspace.f90:143-207, same
// half-space; the reference's |k|^2 order only changes summation order)
static int build_mesh(mdff_ctx* h) {
  h->gen++;
  KMesh KM;
  kmesh_of(h->p.kES, h->B, h->p.alphaES, KM);
  h->rows = KM.rows;
  h->nk = KM.nk;
  int nk = h->nk;
  const std::vector<double>& Ak = KM.Ak;
  const std::vector<double4>& kv = KM.kv;
  // k chunks of the field pass: enough blocks to fill 148 SMs several times,
  // at most 2048 k (32 KB of rho') per chunk
  int nrows = (int)h->rows.size();
  int atom_blocks = cdiv(h->natm, 2 * kFieldThreads);
  int nch = std::max(1, std::min(nrows, cdiv(4 * 148 * 2, atom_blocks)));
  nch = std::max(nch, std::min(nrows, cdiv(nk, 2048)));
  h->rchunk.assign(1, 0);
  double per = (double)nk / nch;
  int r = 0;
  for (int c = 1; c < nch; ++c) {
    double target = per * c;
    while (r < nrows && h->rows[r].w < target) ++r;
    if (r > h->rchunk.back() && r < nrows) h->rchunk.push_back(r);
  }
  h->rchunk.push_back(nrows);
  h->max_chunk_k = 0;
  for (size_t c = 0; c + 1 < h->rchunk.size(); ++c) {
    int a = h->rows[h->rchunk[c]].w;
    int b = (h->rchunk[c + 1] < nrows) ? h->rows[h->rchunk[c + 1]].w : nk;
    h->max_chunk_k = std::max(h->max_chunk_k, b - a);
  }
  cudaFree(h->d_rows);
  cudaFree(h->d_Ak);
  cudaFree(h->d_kvec);
  cudaFree(h->d_rchunk);
  cudaFree(h->d_rho_part);
  cudaFree(h->d_rhoA);
  cudaFree(h->d_str);
  cudaFree(h->d_G);
  cudaFree(h->d_H);
  h->d_rows = nullptr;
  DALLOC(h->d_rows, std::max(nrows, 1));
  DALLOC(h->d_Ak, std::max(nk, 1));
  DALLOC(h->d_kvec, std::max(nk, 1));
  DALLOC(h->d_rchunk, h->rchunk.size());
  h->n_rho_chunks = cdiv(h->natm, kRhoChunk);
  {
    // tensor-core structure factor: one CTA per SM over (row tiles x ion chunks)
    const char* env = std::getenv("MDFF_REC_TC");
    h->rho_tc = rho_tc_fits(h->p.kES[0], h->p.kES[1], h->p.kES[2]) && nrows > 0 && !(env && env[0] == '0');
    // its K dimension: the polarisable ions (where induced dipoles live)
    int nion = h->polidx.empty() ? h->natm : (int)h->polidx.size();
    int tiles = cdiv(nrows, kRhoTcRows);
    int nchunk = std::max(1, (h->nsm > 0 ? h->nsm : 148) / std::max(tiles, 1));
    h->tc_chunk = std::max(kRhoTcKB, cdiv(cdiv(nion, nchunk), kRhoTcKB) * kRhoTcKB);
    h->n_tc_chunks = cdiv(nion, h->tc_chunk);
    h->tc_nkb = cdiv(nion, kRhoTcKB);
    cudaFree(h->d_rho_timg);
    cudaFree(h->d_w32s);
    cudaFree(h->d_polslot);
    h->d_rho_timg = nullptr;
    h->d_w32s = nullptr;
    h->d_polslot = nullptr;
    if (h->rho_tc) {
      DALLOC(h->d_rho_timg, (size_t)h->tc_nkb * rho_tc_staging(h->p.kES[0], h->p.kES[1], h->p.kES[2]) / sizeof(float2));
      DALLOC(h->d_w32s, (size_t)h->tc_nkb * kRhoTcKB);  // zero past the slots
      std::vector<int> slot(h->natm, -1);
      if (h->polidx.empty())
        for (int i = 0; i < h->natm; ++i) slot[i] = i;
      else
        for (size_t k = 0; k < h->polidx.size(); ++k) slot[h->polidx[k]] = (int)k;
      DALLOC(h->d_polslot, h->natm);
      CK(cudaMemcpy(h->d_polslot, slot.data(), sizeof(int) * h->natm, cudaMemcpyHostToDevice));
    }
  }
  DALLOC(h->d_rho_part, (size_t)std::max(h->n_rho_chunks, h->n_tc_chunks) * std::max(nk, 1));
  if (h->rho_tc)
    CK(cudaFuncSetAttribute(k_rec_rho_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            (int)rho_tc_smem(h->p.kES[0], h->p.kES[1], h->p.kES[2])));
  {
    const char* env = std::getenv("MDFF_FIELD_TC");
    int kf = field_tc_kf(h->p.kES[2]);
    h->field_tc = kf > 0 && nrows > 0 && !(env && env[0] == '0') &&
                  field_tc_smem(kf, h->p.kES[1]) <= 227 * 1024;
    cudaFree(h->d_fb);
    h->d_fb = nullptr;
    if (h->field_tc) {
      // B tiles for the smaller row tile (with dipole forces): hi + lo per tile
      DALLOC(h->d_fb, (size_t)cdiv(nrows, field_tc_rpt(true)) * 2 * 128 * kf);
      int smem = (int)field_tc_smem(kf, h->p.kES[1]);
      if (kf == 32) {
        CK(cudaFuncSetAttribute(k_rec_field_tc<true, 32>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        CK(cudaFuncSetAttribute(k_rec_field_tc<false, 32>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
      } else {
        CK(cudaFuncSetAttribute(k_rec_field_tc<true, 64>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        CK(cudaFuncSetAttribute(k_rec_field_tc<false, 64>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
      }
    }
  }
  DALLOC(h->d_rhoA, std::max(nk, 1));
  cudaFree(h->d_rho_acc);
  h->d_rho_acc = nullptr;
  DALLOC(h->d_rho_acc, std::max(nk, 1));
  DALLOC(h->d_str, std::max(nk, 1));
  DALLOC(h->d_G, (size_t)(h->rchunk.size() - 1) * h->natm);
  DALLOC(h->d_H, (size_t)(h->rchunk.size() - 1) * h->natm);
  CK(cudaMemcpyAsync(h->d_rows, h->rows.data(), sizeof(int4) * nrows, cudaMemcpyHostToDevice, h->st));
  CK(cudaMemcpyAsync(h->d_Ak, Ak.data(), sizeof(double) * nk, cudaMemcpyHostToDevice, h->st));
  CK(cudaMemcpyAsync(h->d_kvec, kv.data(), sizeof(double4) * nk, cudaMemcpyHostToDevice, h->st));
  CK(cudaMemcpyAsync(h->d_rchunk, h->rchunk.data(), sizeof(int) * h->rchunk.size(),
                     cudaMemcpyHostToDevice, h->st));
  CK(cudaStreamSynchronize(h->st));
  h->stats.nk = nk;
  return MDFF_OK;
}

// list geometry for the current cell: cells per axis wide enough for the
// build cutoff (fractional width >= rskin / face width)
static int setup_list_cells(mdff_ctx* h) {
  int nc[3];
  for (int a = 0; a < 3; ++a) {
    int n = (int)std::floor(h->W[a] / (h->rskin_build * (1.0 + 1e-9) + 1e-9));
    nc[a] = std::max(1, std::min(n, 1024));
    h->L.nc[a] = nc[a];
  }
  int ncell = nc[0] * nc[1] * nc[2];
  h->gen++;  // the list geometry is captured in the graphs
  if (ncell != h->ncell) {
    cudaFree(h->L.cell_count);
    cudaFree(h->L.cell_start);
    cudaFree(h->L.cell_fill);
    DALLOC(h->L.cell_count, ncell);
    DALLOC(h->L.cell_start, ncell + 1);
    DALLOC(h->L.cell_fill, ncell);
    h->ncell = ncell;
  }
  return MDFF_OK;
}

static int alloc_list(mdff_ctx* h, int cap) {
  cap = ((cap + 31) / 32) * 32;
  h->gen++;
  cudaFree(h->L.nbr);
  h->L.nbr = nullptr;
  DALLOC(h->L.nbr, (size_t)h->natm * cap);
  h->L.cap = cap;
  h->dd_cache_ok = false;
  if (h->p.precision == MDFF_PREC_MIXED && h->lpolar) {
    cudaFree(h->d_ddr);
    cudaFree(h->d_ddb1);
    cudaFree(h->d_ddj);
    h->d_ddr = nullptr;
    h->d_ddb1 = nullptr;
    h->d_ddj = nullptr;
    DALLOC(h->d_ddr, (size_t)h->natm * cap);
    DALLOC(h->d_ddb1, (size_t)h->natm * cap);
    DALLOC(h->d_ddj, (size_t)h->natm * cap);
    if (!h->d_ddn) DALLOC(h->d_ddn, h->natm);
    if (!h->d_Edd) DALLOC(h->d_Edd, h->natm);
  }
  h->stats.list_capacity = cap * h->natm;
  return MDFF_OK;
}

static int upload_cell(mdff_ctx* h) {
  CellC c;
  memcpy(c.A, h->A, sizeof(c.A));
  memcpy(c.B, h->B, sizeof(c.B));
  c.omega = h->omega;
  CK(cudaMemcpyAsync(h->d_cell, &c, sizeof(CellC), cudaMemcpyHostToDevice, h->st));
  CK(cudaStreamSynchronize(h->st));
  return MDFF_OK;
}

// ---------------------------------------------------------------------------
// device passes

static int list_update(mdff_ctx* h) {
  int n = h->natm;
  int pr = prof_begin(h, KC_LIST, 0);
  if (!h->have_list) {
    k_seti<<<1, 32, 0, h->st>>>(&h->L.flags[0], 1);
    LAUNCH_CHECK();
  } else {
    int nb = cdiv(n, 256);
    PDL_CHECK(pdl_launch(k_disp_partial, dim3(nb), dim3(256), 0, h->st, h->d_s, h->L.sref, n, h->d_cell, h->d_disp_part));
    PDL_CHECK(pdl_launch(k_disp_final, dim3(1), dim3(32), 0, h->st, h->d_disp_part, nb, h->L.skindiff, h->L.flags,
                                      h->d_scal + S_DISP));
  }
  PDL_CHECK(pdl_launch(k_cell_count, dim3(cdiv(n, 256)), dim3(256), 0, h->st, h->d_s, n, h->L));
  PDL_CHECK(pdl_launch(k_cell_scan, dim3(1), dim3(1024), 0, h->st, h->L, h->ncell));
  PDL_CHECK(pdl_launch(k_cell_scatter, dim3(cdiv(n, 256)), dim3(256), 0, h->st, n, h->L));
  // grid-stride build and sort: a step without a rebuild launches a few
  // blocks per SM that read the flag and leave
  int nsm = h->nsm > 0 ? h->nsm : 148;
  PDL_CHECK(pdl_launch(k_build_rows, dim3(std::min(cdiv((long)n * 32, 256), 8 * nsm)), dim3(256), 0, h->st, h->d_s, n, h->d_cell, h->L));
  int P = 1;
  while (P < h->L.cap) P <<= 1;
  PDL_CHECK(pdl_launch(k_sort_rows, dim3(std::min(n, 8 * nsm)), dim3(256), P * sizeof(int), h->st, h->L, n));
  PDL_CHECK(pdl_launch(k_build_done, dim3(cdiv(n, 256)), dim3(256), 0, h->st, h->d_s, n, h->L));
  PDL_CHECK(pdl_launch(k_build_clear, dim3(1), dim3(256), 0, h->st, h->L, h->ncell));
  prof_end(h, pr);
  h->have_list = true;
  return MDFF_OK;
}

static int reduce_into(mdff_ctx* h, int nblk, int nv, double* out) {
  PDL_CHECK(pdl_launch(k_reduce_partials, dim3(nv), dim3(256), 0, h->st, (const double*)h->d_part, nblk,
                       nv, out));
  return MDFF_OK;
}

// ---- side streams ---------------------------------------------------------
// side stream s waits for everything issued on st so far
static int fork_to(mdff_ctx* h, cudaStream_t s) {
  CK(cudaEventRecord(h->ev_fork, h->st));
  CK(cudaStreamWaitEvent(s, h->ev_fork, 0));
  return MDFF_OK;
}
// stream of the short-range pass (st when overlap is off for this call)
static int sr_fork(mdff_ctx* h, cudaStream_t* s) {
  *s = h->st;
  if (!h->call_overlap) return MDFF_OK;
  int e = fork_to(h, h->st_sr);
  if (e) return e;
  h->sr_open = true;
  *s = h->st_sr;
  return MDFF_OK;
}
static int sr_join(mdff_ctx* h) {
  if (!h->sr_open) return MDFF_OK;
  h->sr_open = false;
  CK(cudaEventRecord(h->ev_join_sr, h->st_sr));
  CK(cudaStreamWaitEvent(h->st, h->ev_join_sr, 0));
  return MDFF_OK;
}
// stream of the real-space half of a pass; rec_pass_t joins it before its
// final sum into the same field / forces
static int rs_fork(mdff_ctx* h, cudaStream_t* s) {
  *s = h->st;
  if (!h->call_overlap) return MDFF_OK;
  int e = fork_to(h, h->st_rs);
  if (e) return e;
  h->rs_open = true;
  *s = h->st_rs;
  return MDFF_OK;
}
static int rs_join(mdff_ctx* h) {
  if (!h->rs_open) return MDFF_OK;
  h->rs_open = false;
  CK(cudaEventRecord(h->ev_join_rs, h->st_rs));
  CK(cudaStreamWaitEvent(h->st, h->ev_join_rs, 0));
  return MDFF_OK;
}

// moments [qtot(3), mutot(3), qsq, musq] of (q?, mu) into out (device)
static int moments(mdff_ctx* h, const double4* mu, int has_q, double* out) {
  int n = h->natm, nb = cdiv(n, 256);
  PDL_CHECK(pdl_launch(k_moments_part, dim3(nb), dim3(256), 0, h->st, h->d_pos, h->d_q, mu, n, has_q, h->d_part));
  return reduce_into(h, nb, 8, out);
}

static PolDev poldev(mdff_ctx* h) { return PolDev{h->d_pol, h->d_invpol, h->d_ipolar}; }
// the slot-ordered FP32 weights of the tensor-core structure factor (inactive without it)
static SlotW slotw(const mdff_ctx* h) {
  SlotW sw;
  if (h->d_w32s) {
    sw.w32s = h->d_w32s;
    sw.slot = h->d_polslot;
  }
  return sw;
}

// nz tile of the structure factor: the width (8, 11, 13 or 16) that wastes
// the fewest accumulator slots on rows of nzmax consecutive nz
static int pick_nzt(int nzmax) {
  // a whole row in one tile when it fits in 25 accumulators (per-ion set-up
  // of the phases is then shared by all nz of the row)
  if (nzmax == 25) return 25;
  if (nzmax == 21) return 21;
  const int cand[4] = {16, 13, 11, 8};
  int best = 16, waste = 1 << 30;
  for (int c : cand) {
    int w = cdiv(nzmax, c) * c - nzmax;
    if (w < waste) {
      waste = w;
      best = c;
    }
  }
  return best;
}

template <typename R, int NZT>
static void launch_rho(mdff_ctx* h, dim3 g, const typename cplx<R>::T* tab, int n, int chunk,
                       const RecMesh& M, int ntiles, int has_q, int has_mu) {
  if constexpr (std::is_same<R, float>::value) {
    // FP32: two ions per thread in packed FP32x2 lanes
    if (has_q && has_mu)
      (void)pdl_launch(k_rec_rho_x2<true, true, NZT>, dim3(g), dim3(kRhoThreads), 0, h->st, tab, h->d_w32, n, chunk, M, ntiles, h->d_rho_part);
    else if (has_q)
      (void)pdl_launch(k_rec_rho_x2<true, false, NZT>, dim3(g), dim3(kRhoThreads), 0, h->st, tab, h->d_w32, n, chunk, M, ntiles, h->d_rho_part);
    else
      (void)pdl_launch(k_rec_rho_x2<false, true, NZT>, dim3(g), dim3(kRhoThreads), 0, h->st, tab, h->d_w32, n, chunk, M, ntiles, h->d_rho_part);
    return;
  }
  if (has_q && has_mu)
    (void)pdl_launch(k_rec_rho<R, true, true, NZT>, dim3(g), dim3(kRhoThreads), 0, h->st, tab, h->d_w, n, chunk, M, ntiles, h->d_rho_part);
  else if (has_q)
    (void)pdl_launch(k_rec_rho<R, true, false, NZT>, dim3(g), dim3(kRhoThreads), 0, h->st, tab, h->d_w, n, chunk, M, ntiles, h->d_rho_part);
  else
    (void)pdl_launch(k_rec_rho<R, false, true, NZT>, dim3(g), dim3(kRhoThreads), 0, h->st, tab, h->d_w, n, chunk, M, ntiles, h->d_rho_part);
}

// ion slots of the tensor-core structure factor: the polarisable ions
static int rho_tc_nion(const mdff_ctx* h) { return h->polidx.empty() ? h->natm : (int)h->polidx.size(); }

// FP32 structure factor of the dipoles on the tensor cores into d_rho_part
// (n_tc_chunks chunks); a launch error surfaces at the caller's LAUNCH_CHECK
static void launch_rho_tc(mdff_ctx* h, const RecMesh& M, int n) {
  size_t smem = rho_tc_smem(M.kmax[0], M.kmax[1], M.kmax[2]);
  dim3 g((unsigned)cdiv(M.nrows, kRhoTcRows), (unsigned)h->n_tc_chunks);
  (void)n;
  (void)pdl_launch(k_rec_rho_tc, g, dim3(kRhoTcThreads), smem, h->st, (const float2*)h->d_rho_timg,
                   (const float4*)h->d_w32s, rho_tc_nion(h), h->tc_chunk, M,
                   h->d_rho_part, h->d_cata + 1, (const int*)(h->d_cata + 3));
}

// FP32 field / force partials on the tensor cores into d_G / d_H (B tiles
// built first into d_fb); returns the number of partial chunks written.
// imap (nion entries): the ions whose partials are wanted (nullptr: all n)
template <int KF>
static int launch_field_tc_k(mdff_ctx* h, const RecMesh& M, int n, bool muf, int npart, const int* imap,
                             int nion, double2* rho_out) {
  int rpt = field_tc_rpt(muf);
  int ntile = cdiv(M.nrows, rpt);
  int ion_tiles = cdiv(nion, 128);
  int nalloc = (int)h->rchunk.size() - 1;
  int ng = std::max(1, std::min({(2 * (h->nsm > 0 ? h->nsm : 148)) / std::max(ion_tiles, 1), ntile, nalloc}));
  int tpg = cdiv(ntile, ng);
  ng = cdiv(ntile, tpg);
  dim3 g((unsigned)ion_tiles, (unsigned)ng);
  size_t smem = field_tc_smem(KF, M.kmax[1]);
  size_t bsmem = (size_t)kBtRows * (2 * M.kmax[2] + 1) * sizeof(double2);
  dim3 gb((unsigned)ntile, (unsigned)(rpt / kBtRows));
  int* err = h->d_cata + 1;
  const double2* rhoA = h->d_rhoA;
  const double2* rpart = h->d_rho_part;
  const float2* tab = h->d_tab32;
  const float4* w = h->d_w32;
  const uint32_t* fb = h->d_fb;
  h->launches++;  // two launches here; the caller's LAUNCH_CHECK counts one
  if (muf) {
    (void)pdl_launch(k_rec_field_btiles<true, KF>, gb, dim3(128), bsmem, h->st, M, rhoA, rpart, npart, h->d_fb, rho_out);
    (void)pdl_launch(k_rec_field_tc<true, KF>, g, dim3(kFieldTcThreads), smem, h->st, tab, w, n, imap, nion,
                     M, fb, tpg, h->d_G, h->d_H, err);
  } else {
    (void)pdl_launch(k_rec_field_btiles<false, KF>, gb, dim3(128), bsmem, h->st, M, rhoA, rpart, npart, h->d_fb, rho_out);
    (void)pdl_launch(k_rec_field_tc<false, KF>, g, dim3(kFieldTcThreads), smem, h->st, tab, w, n, imap, nion,
                     M, fb, tpg, h->d_G, h->d_H, err);
  }
  return ng;
}

static int launch_field_tc(mdff_ctx* h, const RecMesh& M, int n, bool muf, int npart, const int* imap,
                           int nion, double2* rho_out) {
  if (field_tc_kf(M.kmax[2]) == 32) return launch_field_tc_k<32>(h, M, n, muf, npart, imap, nion, rho_out);
  return launch_field_tc_k<64>(h, M, n, muf, npart, imap, nion, rho_out);
}

// reciprocal pass: E += rec field (+ the self / surface field sf, when on);
// force += rec force * coul_unit (if forces); energy (7 doubles) into e_out
// (if non-null)
template <typename R>
static int rec_pass_t(mdff_ctx* h, const typename cplx<R>::T* tab, const double4* mu, int has_q,
                      int has_mu, int forces, double4* E, double* e_out, float4* mu32,
                      SelfField sf, int* defer_nch, bool weights_ready, bool pol_dipoles) {
  int n = h->natm;
  if (h->nk == 0) {
    int e = rs_join(h);
    if (e) return e;
    if (sf.on) {
      k_self_surf_field<<<cdiv(n, 256), 256, 0, h->st>>>(sf.mu, n, sf.selfa2, sf.lsurf, sf.fpi_3V, sf.mom, E);
      LAUNCH_CHECK();
    }
    return MDFF_OK;
  }
  RecMesh M;
  M.kmax[0] = h->p.kES[0];
  M.kmax[1] = h->p.kES[1];
  M.kmax[2] = h->p.kES[2];
  M.nrows = (int)h->rows.size();
  M.rows = h->d_rows;
  M.nk = h->nk;
  M.Ak = h->d_Ak;
  M.kvec = h->d_kvec;
  constexpr bool F32 = std::is_same<R, float>::value;
  // (the FP32 CG direction kernels write the FP32 weights themselves)
  if (!(F32 && weights_ready)) {
    PDL_CHECK(pdl_launch(k_rec_weights, dim3(cdiv(n, 256)), dim3(256), 0, h->st, h->d_q, mu, n, h->d_cell, has_q, has_mu, h->d_w,
                         F32 ? h->d_w32 : nullptr, mu32, slotw(h)));
  }
  int nzt = pick_nzt(2 * M.kmax[2] + 1);
  int ntiles = cdiv(2 * M.kmax[2] + 1, nzt);
  dim3 g((unsigned)(M.nrows * ntiles), (unsigned)h->n_rho_chunks);
  int chunk = kRhoChunk;
  // algorithmic op counts per (k, ion) term (add = mul = 1, FMA = 2,
  // sin/cos/exp/sqrt = 1): structure factor k.r 5 + sin,cos 2 + q part 4 +
  // k.mu 5 + mu part 4; field/force pass: recarg/recarg2 8 + field 6 + F_q 6 + F_mu 12
  double ops_rho = (has_q && has_mu) ? 20.0 : (has_mu ? 16.0 : 11.0);
  double ops_fld = (forces && has_mu) ? 32.0 : (forces ? 17.0 : 20.0);
  int pr = prof_begin(h, KC_RHO, (double)h->nk * n * ops_rho);
  int nparts = h->n_rho_chunks;
  const int mode = h->rec_mode;
  // the tensor-core structure factor serves the FP32 CG operator (dipoles
  // alone, no forces), whose error the FP64 residual refinement removes; the
  // static field and the force pass keep the CUDA-core kernels (FP32 sums
  // with round-to-nearest).  The force pass after a CG solve takes the
  // solve's accumulated rho' instead (REC_FROM_ACC).
  if (mode == REC_FROM_ACC) {
    nparts = 0;
    PDL_CHECK(pdl_launch(k_rec_acc_finish, dim3(cdiv(h->nk, 256)), dim3(256), 0, h->st,
                         (const double2*)h->d_rho_acc, M, h->d_rhoA, h->d_str));
  } else if (F32 && h->rho_tc && pol_dipoles && !has_q && has_mu && !forces) {
    nparts = h->n_tc_chunks;
    launch_rho_tc(h, M, n);
  } else {
    switch (nzt) {
      case 8: launch_rho<R, 8>(h, g, tab, n, chunk, M, ntiles, has_q, has_mu); break;
      case 11: launch_rho<R, 11>(h, g, tab, n, chunk, M, ntiles, has_q, has_mu); break;
      case 13: launch_rho<R, 13>(h, g, tab, n, chunk, M, ntiles, has_q, has_mu); break;
      case 21: launch_rho<R, 21>(h, g, tab, n, chunk, M, ntiles, has_q, has_mu); break;
      case 25: launch_rho<R, 25>(h, g, tab, n, chunk, M, ntiles, has_q, has_mu); break;
      default: launch_rho<R, 16>(h, g, tab, n, chunk, M, ntiles, has_q, has_mu); break;
    }
  }
  LAUNCH_CHECK();
  prof_end(h, pr);
  double tpi_V = kTwoPi / h->omega;
  // without energy the field pass sums the chunk partials while staging rho'
  // (the CUDA-core field kernels when there are few chunks; the tensor-core
  // B-tile builder always)
  int npart = 0;
  const bool field_tc = F32 && h->field_tc;
  if (mode == REC_FROM_ACC) {
    // rhoA and str are in place
  } else if (e_out || (nparts > 4 && !field_tc) || mode == REC_SAVE_ACC || (mode == REC_NEED_RHOA && !field_tc)) {
    // (REC_SAVE_ACC: this rho' starts the solve's accumulation; REC_NEED_RHOA:
    // the CG step after this operator adds it, which the tensor-core B-tile
    // builder writes while it sums the partials)
    PDL_CHECK(pdl_launch(k_rec_sum, dim3(cdiv(h->nk, 256)), dim3(256), 0, h->st, (const double2*)h->d_rho_part, nparts,
                         M, h->d_rhoA, h->d_str, mode == REC_SAVE_ACC ? h->d_rho_acc : (double2*)nullptr));
  } else {
    npart = nparts;
  }
  if (e_out) {
    PDL_CHECK(pdl_launch(k_rec_energy, dim3(1), dim3(1024), 0, h->st, h->d_str, M, tpi_V, h->omega, 1, e_out));
  }
  int nch = (int)h->rchunk.size() - 1;
  // a pass without forces feeds the dipole solvers, which read its field at
  // the polarisable ions only: the field kernels run over those (ion map)
  // and the final sum leaves the other ions' reciprocal part out
  const bool field_pol = !forces && h->d_polidx;
  const int* imap = field_pol ? h->d_polidx : nullptr;
  const int nion = field_pol ? (int)h->polidx.size() : n;
  dim3 gf((unsigned)cdiv(nion, kFieldThreads), (unsigned)nch);
  size_t smem = (size_t)h->max_chunk_k * sizeof(typename cplx<R>::T);
  bool muf = forces && has_mu;
  pr = prof_begin(h, KC_RECF, (double)h->nk * n * ops_fld);
  if (field_tc) {
    nch = launch_field_tc(h, M, n, muf, npart, imap, nion,
                          (mode == REC_NEED_RHOA && npart) ? h->d_rhoA : (double2*)nullptr);
  } else if constexpr (std::is_same<R, float>::value) {
    dim3 gx((unsigned)cdiv(n, 2 * kFieldThreads), (unsigned)nch);
    if (muf)
      (void)pdl_launch(k_rec_field_x2<true>, dim3(gx), dim3(kFieldThreads), smem, h->st, tab, h->d_w32, n, M, h->d_rchunk, h->d_rhoA, h->d_rho_part, npart, h->d_G, h->d_H);
    else
      (void)pdl_launch(k_rec_field_x2<false>, dim3(gx), dim3(kFieldThreads), smem, h->st, tab, h->d_w32, n, M, h->d_rchunk, h->d_rhoA, h->d_rho_part, npart, h->d_G, h->d_H);
  } else if (muf)
    (void)pdl_launch(k_rec_field<R, true>, dim3(gf), dim3(kFieldThreads), smem, h->st, tab, h->d_w, n, imap, nion, M, h->d_rchunk, h->d_rhoA, h->d_rho_part, npart, h->d_G, h->d_H);
  else
    PDL_CHECK(pdl_launch(k_rec_field<R, false>, dim3(gf), dim3(kFieldThreads), smem, h->st, tab, h->d_w, n, imap, nion, M, h->d_rchunk, h->d_rhoA, h->d_rho_part, npart, h->d_G, h->d_H));
  prof_end(h, pr);
  double fpi_V = 2.0 * tpi_V;
  // the real-space half of this pass (side stream) adds into the same E / forces
  int e = rs_join(h);
  if (e) return e;
  if (defer_nch) {
    // the caller's kernel sums the field partials (k_dd_cached_rec)
    *defer_nch = nch;
    return MDFF_OK;
  }
  k_rec_field_sum<<<cdiv((long)n * 4, 256), 256, 0, h->st>>>(h->d_G, h->d_H, nch, n, h->d_cell, h->d_q,
                                                   2.0 * fpi_V, muf ? 1 : 0, forces, h->coul_unit, E,
                                                   h->d_force, sf, field_pol ? h->d_ipolar : nullptr);
  LAUNCH_CHECK();
  return MDFF_OK;
}

// pol_dipoles: the dipoles mu are nonzero at the polarisable ions only (the
// induced dipoles and the solver's directions)
static int rec_pass(mdff_ctx* h, bool fp32, const double4* mu, int has_q, int has_mu, int forces,
                    double4* E, double* e_out, SelfField sf, float4* mu32 = nullptr,
                    int* defer_nch = nullptr, bool weights_ready = false, bool pol_dipoles = false) {
  if (fp32)
    return rec_pass_t<float>(h, h->d_tab32, mu, has_q, has_mu, forces, E, e_out, mu32, sf, defer_nch, weights_ready,
                             pol_dipoles);
  return rec_pass_t<double>(h, h->d_tab64, mu, has_q, has_mu, forces, E, e_out, mu32, sf, defer_nch, false, false);
}

// the self field 2 selfa2 mu (+ surface field of the reduced moments in mom
// when lsurf) of one moment set (field_dipole_ES_self / surface, coulomb.f90)
static SelfField self_field(mdff_ctx* h, const double4* mu, const double* mom) {
  double a = h->p.alphaES;
  SelfField sf;
  sf.on = 1;
  sf.lsurf = h->p.lsurf;
  sf.mu = mu;
  sf.selfa2 = 2.0 * (a / std::sqrt(kPi)) * a * a / 3.0;
  sf.fpi_3V = 2.0 * (kTwoPi / h->omega / 3.0);
  sf.mom = mom;
  return sf;
}

static int build_tables(mdff_ctx* h) {
  if (h->nk == 0) return MDFF_OK;
  int n = h->natm;
  int kzt = std::max(h->p.kES[2], 4);
  PDL_CHECK(pdl_launch(k_rec_tables<double>, dim3(cdiv(n, 128)), dim3(128), 0, h->st, h->d_s, n, h->p.kES[0], h->p.kES[1], kzt, h->d_tab64));
  if (h->p.precision == MDFF_PREC_MIXED) {
    PDL_CHECK(pdl_launch(k_rec_tables<float>, dim3(cdiv(n, 128)), dim3(128), 0, h->st, h->d_s, n, h->p.kES[0], h->p.kES[1], kzt, h->d_tab32));
    // the same tables blocked by K block for the tensor-core structure
    // factor of the dipole solve
    if (h->rho_tc && h->lpolar)
      PDL_CHECK(pdl_launch(k_rec_rho_timg, dim3((unsigned)h->tc_nkb), dim3(256), 0, h->st, (const float2*)h->d_tab32, n,
                           (const int*)h->d_polidx, rho_tc_nion(h), h->p.kES[0], h->p.kES[1], h->p.kES[2],
                           h->d_rho_timg));
  }
  return MDFF_OK;
}

// field of a dipole set alone (charges zeroed, dd task, undamped): the SCF
// induced pass / the CG operator.  E = T mu.
// weights_ready: d_w32 / d_mu32 already hold the FP32 operands of mu (written
// by the CG direction kernels)
static int field_of_mu(mdff_ctx* h, const double4* mu, int dd_mask, bool fp32, double4* E,
                       bool weights_ready = false, bool cached64 = false) {
  int n = h->natm;
  // FP32 CG operator with the pair cache: one kernel writes E (reciprocal +
  // self + cached real-space dipole field)
  const bool fused = fp32 && dd_mask == 1 && h->dd_cache_ok && h->nk > 0;
  if (!fused) CK(cudaMemsetAsync(E, 0, sizeof(double4) * n, h->st));
  double cutsq = h->p.cutlongrange * h->p.cutlongrange;
  int nb = cdiv((long)n * 32, 256);
  int s;
  if (h->p.lsurf) {
    s = moments(h, mu, 0, h->d_scal + S_MOM2);
    if (s) return s;
  }
  // reciprocal first: its weights kernel also writes the FP32 dipoles; its
  // final kernel adds the self / surface field
  int nch = 0;
  SelfField sf = self_field(h, mu, h->d_scal + S_MOM2);
  if (!fp32) {
    // FP64: the real-space dipole field beside the reciprocal pass (cached64:
    // the FP32 operator's cached pair tensor, FP64 products and sums)
    cudaStream_t rs;
    if ((s = rs_fork(h, &rs))) return s;
    int pr = prof_begin(h, KC_ESFIELD, 0);
    if (cached64 && dd_mask == 1 && h->dd_cache_ok)
      k_dd_cached64<<<nb, 256, 0, rs>>>(mu, h->d_ddr, h->d_ddb1, h->d_ddj, h->d_ddn, h->L.cap, n, E);
    else
      k_es_field<double, false, true><<<nb, 256, 0, rs>>>(h->d_s, h->d_q, h->d_itype, h->d_ipolar, mu, h->L.nbr, h->L.nnb, h->L.cap, n, h->d_cell, h->d_estab, h->ntype, h->p.alphaES, cutsq, 0, dd_mask, E, h->p.thole_type);
    LAUNCH_CHECK();
    prof_end(h, pr);
    return rec_pass(h, false, mu, 0, 1, 0, E, nullptr, sf);
  }
  // the CG operator with its FP32 operands ready (inside the CG graph too):
  // the cached real-space dipole field on the side stream beside the
  // reciprocal pass, whose rs_join joins it before the final kernel adds it
  const bool dd_side = fused && weights_ready && h->overlap && !h->prof && h->d_Edd;
  if (dd_side) {
    if ((s = fork_to(h, h->st_rs))) return s;
    h->rs_open = true;
    k_dd_cached_part<<<nb, 256, 0, h->st_rs>>>(h->d_mu32, h->d_ddr, h->d_ddb1, h->d_ddj, h->d_ddn,
                                                h->L.cap, n, h->d_Edd);
    LAUNCH_CHECK();
  }
  s = rec_pass(h, fp32, mu, 0, 1, 0, E, nullptr, sf, h->d_mu32, fused ? &nch : nullptr, weights_ready, true);
  if (s) return s;
  int pr = prof_begin(h, KC_ESFIELD, 0);
  if (fused)
    k_dd_cached_rec<<<nb, 256, 0, h->st>>>(h->d_mu32, h->d_ddr, h->d_ddb1, h->d_ddj, h->d_ddn, h->L.cap, n,
                                           h->d_G, nch, h->d_cell, 2.0 * (2.0 * (kTwoPi / h->omega)), sf, E,
                                           dd_side ? h->d_Edd : nullptr, h->d_ipolar);
  else if (fp32 && dd_mask == 1 && h->dd_cache_ok)
    k_dd_cached<<<nb, 256, 0, h->st>>>(h->d_mu32, h->d_ddr, h->d_ddb1, h->d_ddj, h->d_ddn, h->L.cap, n, E);
  else
    k_es_field<float, false, true><<<nb, 256, 0, h->st>>>(h->d_s, h->d_q, h->d_itype, h->d_ipolar, h->d_mu32, h->L.nbr, h->L.nnb, h->L.cap, n, h->d_cell, h->d_estab, h->ntype, h->p.alphaES, cutsq, 0, dd_mask, E, h->p.thole_type);
  LAUNCH_CHECK();
  prof_end(h, pr);
  return MDFF_OK;
}

// static field of the charges (+ static dipoles), damped (moment_from_pola.f90:327-330)
static int static_field(mdff_ctx* h, bool fp32) {
  int n = h->natm;
  double4* E = h->d_Estat;
  CK(cudaMemsetAsync(E, 0, sizeof(double4) * n, h->st));
  double cutsq = h->p.cutlongrange * h->p.cutlongrange;
  int nb = cdiv((long)n * 32, 256);
  bool qq = h->task_qq != 0, dd = h->ldip_static != 0;
#define ESFK(R, Q, D, MU, K)                                                                        \
  k_es_field<R, Q, D, K><<<nb, 256, 0, rs>>>(h->d_s, h->d_q, h->d_itype, h->d_ipolar, MU, h->L.nbr, \
                                             h->L.nnb, h->L.cap, n, h->d_cell, h->d_estab, h->ntype, \
                                             h->p.alphaES, cutsq, 1, 0, E, h->p.thole_type)
  // the damped charge field with the compile-time Tang-Toennies order when it applies
#define ESF(R, Q, D, MU)                    \
  do {                                      \
    if (h->tt_k == 4) ESFK(R, Q, D, MU, 4); \
    else ESFK(R, Q, D, MU, 0);              \
  } while (0)
  if (fp32 && dd) {
    k_to_float4<<<cdiv(n, 256), 256, 0, h->st>>>(h->d_dipia, n, h->d_mu32);
    LAUNCH_CHECK();
  }
  h->dd_cache_ok = false;
  // the real-space half beside the reciprocal pass (joined before its final sum)
  cudaStream_t rs;
  int s;
  if ((s = rs_fork(h, &rs))) return s;
  if (fp32 && !dd && h->lpolar && h->d_ddr) {
    // damped charge field + the pair cache of the FP32 solver iterations
    int pr = prof_begin(h, KC_ESFIELD, 0);
#define STC(K)                                                                                      \
  k_static_cache<K><<<nb, 256, 0, rs>>>(h->d_s, h->d_q, h->d_itype, h->d_ipolar, h->L.nbr, h->L.nnb, \
                                        h->L.cap, n, h->d_cell, h->d_estab, h->ntype, h->p.alphaES,   \
                                        cutsq, qq ? 1 : 0, E, h->d_ddr, h->d_ddb1, h->d_ddj, h->d_ddn, \
                                        h->p.thole_type)
    if (h->tt_k == 4) STC(4);
    else STC(0);
#undef STC
    LAUNCH_CHECK();
    prof_end(h, pr);
    h->dd_cache_ok = true;
  } else if (qq || dd) {
    int pr = prof_begin(h, KC_ESFIELD, 0);
    if (fp32) {
      if (qq && dd) ESF(float, true, true, h->d_mu32);
      else if (qq) ESF(float, true, false, h->d_mu32);
      else ESFK(float, false, true, h->d_mu32, 0);
    } else {
      if (qq && dd) ESF(double, true, true, h->d_dipia);
      else if (qq) ESF(double, true, false, h->d_dipia);
      else ESFK(double, false, true, h->d_dipia, 0);
    }
    LAUNCH_CHECK();
    prof_end(h, pr);
  }
#undef ESF
#undef ESFK
  if (h->p.lsurf) {
    s = moments(h, h->d_dipia, 1, h->d_scal + S_MOM2);
    if (s) return s;
  }
  s = rec_pass(h, fp32, h->d_dipia, h->task_qq ? 1 : 0, dd ? 1 : 0, 0, E, nullptr,
               self_field(h, h->d_dipia, h->d_scal + S_MOM2));
  if (s) return s;
  return MDFF_OK;
}

static int read_scal(mdff_ctx* h, int slot, double* v) {
  CK(cudaMemcpyAsync(h->h_scal + slot, h->d_scal + slot, sizeof(double), cudaMemcpyDeviceToHost, h->st));
  CK(cudaStreamSynchronize(h->st));
  *v = h->h_scal[slot];
  return MDFF_OK;
}

// ASPC order and coefficients (moment_from_pola.f90:514-563)
static void aspc_coef(int itime, int order, int* ord, double B[5], double* w) {
  int e;
  if (itime >= order + 1) e = order;
  else if (itime == 1 || itime == 0) e = 0;
  else e = itime - 1;
  for (int k = 0; k < 5; ++k) B[k] = 0.0;
  switch (e) {
    case 0: B[0] = 1.0; *w = 0.0; break;
    case 1: B[0] = 2.0; B[1] = -1.0; *w = 2.0 / 3.0; break;
    case 2: B[0] = 2.5; B[1] = -2.0; B[2] = 0.5; *w = 0.6; break;
    case 3: B[0] = 2.8; B[1] = -2.8; B[2] = 1.2; B[3] = -0.2; *w = 4.0 / 7.0; break;
    default:
      e = 4;
      B[0] = 3.0; B[1] = -24.0 / 7.0; B[2] = 27.0 / 14.0; B[3] = -4.0 / 7.0; B[4] = 1.0 / 14.0;
      *w = 5.0 / 9.0;
      break;
  }
  *ord = e;
}

static int aspc_predict(mdff_ctx* h, int itime) {
  int ord;
  double B[5], w;
  aspc_coef(itime, h->p.extrapolate_order, &ord, B, &w);
  PDL_CHECK(pdl_launch(k_aspc_predict, dim3(cdiv(h->natm, 256)), dim3(256), 0, h->st, h->d_hist, h->natm, ord, B[0], B[1], B[2], B[3], B[4], h->d_mu_ind));
  return MDFF_OK;
}

// moment_from_pola_scf (moment_from_pola.f90:240-485)
static int solve_scf(mdff_ctx* h, int itime, bool fp32) {
  int n = h->natm, nb = cdiv(n, 256), s;
  PolDev P = poldev(h);
  CK(cudaMemcpyAsync(h->d_Efield, h->d_Estat, sizeof(double4) * n, cudaMemcpyDeviceToDevice, h->st));
  bool ismd = h->p.calc == MDFF_CALC_MD, isopt = h->p.calc == MDFF_CALC_OPT;
  int iscf = 0;
  double rmsd = HUGE_VAL;
  while (((iscf < h->p.max_scf_pol_iter) && (rmsd > h->p.conv_tol_ind)) ||
         (iscf < h->p.min_scf_pol_iter)) {
    iscf++;
    if (iscf != 1 || (!ismd && !isopt)) {
      k_induce<<<nb, 256, 0, h->st>>>(h->d_Efield, P, n, h->d_mu_ind);
      LAUNCH_CHECK();
    } else {
      s = aspc_predict(h, itime);
      if (s) return s;
    }
    k_upol_part<<<nb, 256, 0, h->st>>>(h->d_mu_ind, P, n, h->d_part);
    LAUNCH_CHECK();
    if ((s = reduce_into(h, nb, 1, h->d_scal + S_UPOL))) return s;
    if ((s = field_of_mu(h, h->d_mu_ind, 0, fp32, h->d_Eind))) return s;
    k_add4<<<nb, 256, 0, h->st>>>(h->d_Estat, h->d_Eind, n, h->d_Efield);
    LAUNCH_CHECK();
    if (iscf == 1 && ismd) {
      int ord;
      double B[5], w;
      aspc_coef(itime, h->p.extrapolate_order, &ord, B, &w);
      k_aspc_correct<<<nb, 256, 0, h->st>>>(h->d_Efield, P, n, w, h->d_mu_ind);
      LAUNCH_CHECK();
    }
    k_rmsd_part<<<nb, 256, 0, h->st>>>(h->d_mu_ind, h->d_Efield, P, n, h->d_part);
    LAUNCH_CHECK();
    if ((s = reduce_into(h, nb, 1, h->d_scal + S_RMS))) return s;
    double r2;
    if ((s = read_scal(h, S_RMS, &r2))) return s;
    rmsd = std::sqrt(r2 / (double)h->npol);
  }
  h->stats.n_pol_iter = iscf;
  h->stats.rmsd = rmsd;
  h->stats.converged = rmsd <= h->p.conv_tol_ind;
  CK(cudaMemcpyAsync(h->d_hist, h->d_mu_ind, sizeof(double4) * n, cudaMemcpyDeviceToDevice, h->st));
  return MDFF_OK;
}

// ---------------------------------------------------------------------------
// kO dipole algorithms of the SCF solver (moment_from_pola.f90:822-942,
// 1042-1639, 1987-2529); kernels in ko.cuh

static int read_scals(mdff_ctx* h, int slot, int nv, double* v) {
  CK(cudaMemcpyAsync(h->h_scal + slot, h->d_scal + slot, sizeof(double) * nv, cudaMemcpyDeviceToHost, h->st));
  CK(cudaStreamSynchronize(h->st));
  for (int k = 0; k < nv; ++k) v[k] = h->h_scal[slot + k];
  return MDFF_OK;
}

// polint (moment_from_pola.f90:2365-2412) at x = 1 on the abscissae
// xa(t) = 1 - t, t = 1..n, is linear in the ordinates: w[k] is its value for
// the k-th unit ordinate vector.  The recurrence is the reference's, whose hp
// is taken at xa(i+1) where Neville's scheme has xa(i+m) (from three points
// on the result is not the interpolating polynomial).
static void polint_weights(int n, double w[MDFF_ASPC_DEPTH]) {
  int xa[MDFF_ASPC_DEPTH];
  for (int t = 1; t <= n; ++t) xa[t - 1] = 1 - t;
  int ns = 1;
  double dif = std::fabs((double)(1 - xa[0]));
  for (int i = 1; i <= n; ++i) {
    double dift = std::fabs((double)(1 - xa[i - 1]));
    if (dift < dif) {
      ns = i;
      dif = dift;
    }
  }
  // c[i][k], d[i][k]: the tableaux of unit ordinate k
  double c[MDFF_ASPC_DEPTH][MDFF_ASPC_DEPTH], d[MDFF_ASPC_DEPTH][MDFF_ASPC_DEPTH];
  for (int i = 0; i < n; ++i)
    for (int k = 0; k < n; ++k) c[i][k] = d[i][k] = (i == k) ? 1.0 : 0.0;
  for (int k = 0; k < n; ++k) w[k] = (k == ns - 1) ? 1.0 : 0.0;
  ns = ns - 1;
  for (int m = 1; m <= n - 1; ++m) {
    for (int i = 1; i <= n - m; ++i) {
      double ho = (double)(xa[i - 1] - 1), hp = (double)(xa[i] - 1);
      for (int k = 0; k < n; ++k) {
        double den = (c[i][k] - d[i - 1][k]) / (ho - hp);
        d[i - 1][k] = hp * den;
        c[i - 1][k] = ho * den;
      }
    }
    if (2 * ns < n - m) {
      for (int k = 0; k < n; ++k) w[k] += c[ns][k];
    } else {
      for (int k = 0; k < n; ++k) w[k] += d[ns - 1][k];
      ns = ns - 1;
    }
  }
}

// extrapolate_dipole_poly (moment_from_pola.f90:2276-2363): order 0 repeats
// the last dipoles; order 1 extrapolates linearly from the second call on;
// higher orders use polint over order + 1 stored dipoles (itime + 1 while
// itime <= order), then shift the history.  The reference's last shift step
// reads dipia_ind_t(0); slot 1 is overwritten by the converged dipoles
// before any read, so the shift stops at slot 2.
static int poly_predict(mdff_ctx* h, int itime) {
  int eo = h->p.extrapolate_order, npts = 0, nshift = 0;
  double w[MDFF_ASPC_DEPTH] = {0, 0, 0, 0, 0};
  if (eo == 0) {
    npts = 1;
    w[0] = 1.0;
  } else if (eo == 1) {
    nshift = 1;
    if (itime > eo) {
      npts = 2;
      w[0] = 2.0;
      w[1] = -1.0;
    } else {
      npts = 1;
      w[0] = 1.0;
    }
  } else {
    nshift = eo;
    if (itime > eo) {
      npts = eo + 1;
      polint_weights(npts, w);
    } else if (itime == 1) {
      npts = 1;
      w[0] = 1.0;
    } else if (itime == 2) {
      npts = 2;
      w[0] = 2.0;
      w[1] = -1.0;
    } else if (itime > 2) {
      npts = itime + 1;
      polint_weights(npts, w);
    }
  }
  k_poly_predict<<<cdiv(h->natm, 256), 256, 0, h->st>>>(h->d_hist, h->natm, npts, w[0], w[1], w[2], w[3],
                                                       w[4], nshift, h->d_mu_ind);
  LAUNCH_CHECK();
  return MDFF_OK;
}

// induced_moment_inner (moment_from_pola.f90:822-942): the dipole increment
// dmu relaxed in the direct-space dipole field at alphaES = 0.001 (undamped,
// near neighbours only), weight omegakO, at most 10 passes or until its
// residual is a tenth of the residual of f_ext.
static int ko_inner(mdff_ctx* h, const double4* f_ext, double4* dmu) {
  int n = h->natm, nb = cdiv(n, 256), nbw = cdiv((long)n * 32, 256), s;
  PolDev P = poldev(h);
  const double om = h->p.omegakO;
  k_ko_start<<<nb, 256, 0, h->st>>>(f_ext, P, n, om, dmu, h->d_part);
  LAUNCH_CHECK();
  if ((s = reduce_into(h, nb, 1, h->d_scal + S_KO))) return s;
  double r2;
  if ((s = read_scal(h, S_KO, &r2))) return s;
  const double rmsd_ref = std::sqrt(r2 / (double)h->npol);
  const double a = 0.001;  // moment_from_pola.f90:893
  const double selfa2 = 2.0 * (a / std::sqrt(kPi)) * (a * a) / 3.0;
  const double fpi_3V = 2.0 * (kTwoPi / h->omega / 3.0);
  const double cutsq = h->p.cutlongrange * h->p.cutlongrange;
  double rmsd_inner = HUGE_VAL;
  for (int it = 1; it <= 10 && rmsd_inner > 0.1 * rmsd_ref; ++it) {
    CK(cudaMemsetAsync(h->d_ko_fdir, 0, sizeof(double4) * n, h->st));
    if (h->p.lsurf && (s = moments(h, dmu, 0, h->d_scal + S_MOM2))) return s;
    int pr = prof_begin(h, KC_ESFIELD, 0);
    k_es_field<double, false, true><<<nbw, 256, 0, h->st>>>(
        h->d_s, h->d_q, h->d_itype, h->d_ipolar, dmu, h->L.nbr, h->L.nnb, h->L.cap, n, h->d_cell, h->d_estab,
        h->ntype, a, cutsq, 0, 0, h->d_ko_fdir, h->p.thole_type);
    LAUNCH_CHECK();
    prof_end(h, pr);
    k_ko_relax<<<nb, 256, 0, h->st>>>(f_ext, h->d_ko_fdir, P, n, om, 2.0 * selfa2, h->p.lsurf, fpi_3V,
                                      h->d_scal + S_MOM2, dmu, h->d_part);
    LAUNCH_CHECK();
    if ((s = reduce_into(h, nb, 1, h->d_scal + S_KO))) return s;
    if ((s = read_scal(h, S_KO, &r2))) return s;
    rmsd_inner = std::sqrt(r2 / (double)h->npol);
  }
  return MDFF_OK;
}

// u_pol of the current dipoles into S_UPOL (moment_from_pola.f90:387-395)
static int upol_pass(mdff_ctx* h) {
  int nb = cdiv(h->natm, 256);
  k_upol_part<<<nb, 256, 0, h->st>>>(h->d_mu_ind, poldev(h), h->natm, h->d_part);
  LAUNCH_CHECK();
  return reduce_into(h, nb, 1, h->d_scal + S_UPOL);
}

static int aspc_correct(mdff_ctx* h, int itime) {
  int ord;
  double B[5], w;
  aspc_coef(itime, h->p.extrapolate_order, &ord, B, &w);
  k_aspc_correct<<<cdiv(h->natm, 256), 256, 0, h->st>>>(h->d_Efield, poldev(h), h->natm, w, h->d_mu_ind);
  LAUNCH_CHECK();
  return MDFF_OK;
}

// moment_from_pola_scf_kO_v1 (moment_from_pola.f90:1042-1320) and, with
// find_min along the last step, moment_from_pola_scf_kO_v2 (:1335-1639)
static int solve_ko_v12(mdff_ctx* h, int itime, bool fp32, bool v2) {
  int n = h->natm, nb = cdiv(n, 256), s;
  PolDev P = poldev(h);
  CK(cudaMemcpyAsync(h->d_Efield, h->d_Estat, sizeof(double4) * n, cudaMemcpyDeviceToDevice, h->st));
  CK(cudaMemcpyAsync(h->d_ko_f, h->d_Estat, sizeof(double4) * n, cudaMemcpyDeviceToDevice, h->st));
  CK(cudaMemsetAsync(h->d_ko_g, 0, sizeof(double4) * n, h->st));
  CK(cudaMemsetAsync(h->d_ko_muprev, 0, sizeof(double4) * n, h->st));
  const bool ismd = h->p.calc == MDFF_CALC_MD, isopt = h->p.calc == MDFF_CALC_OPT;
  const bool aspc_on = h->p.algo_ext_dipole == MDFF_EXT_ASPC;
  int iscf = 0;
  double rmsd = HUGE_VAL;
  while (((iscf < h->p.max_scf_pol_iter) && (rmsd > h->p.conv_tol_ind)) ||
         (iscf < h->p.min_scf_pol_iter)) {
    iscf++;
    if (iscf != 1 || (!ismd && !isopt)) {
      // kO_v2 relaxes along the line-minimised residual from its third pass
      const double4* fx = (v2 && iscf > 2) ? h->d_ko_g : h->d_ko_f;
      if ((s = ko_inner(h, fx, h->d_ko_dmu))) return s;
      k_add4<<<nb, 256, 0, h->st>>>(h->d_mu_ind, h->d_ko_dmu, n, h->d_mu_ind);
      LAUNCH_CHECK();
    } else {
      s = aspc_on ? aspc_predict(h, itime) : poly_predict(h, itime);
      if (s) return s;
    }
    if ((s = upol_pass(h))) return s;
    if ((s = field_of_mu(h, h->d_mu_ind, 0, fp32, h->d_Eind))) return s;
    k_add4<<<nb, 256, 0, h->st>>>(h->d_Estat, h->d_Eind, n, h->d_Efield);
    LAUNCH_CHECK();
    if (iscf == 1 && ismd && aspc_on && (s = aspc_correct(h, itime))) return s;
    k_ko_residual<<<nb, 256, 0, h->st>>>(h->d_Efield, h->d_mu_ind, P, n, h->d_ko_f, h->d_part);
    LAUNCH_CHECK();
    if (!v2) {
      if ((s = reduce_into(h, nb, 1, h->d_scal + S_RMS))) return s;
      double r2;
      if ((s = read_scal(h, S_RMS, &r2))) return s;
      rmsd = std::sqrt(r2 / (double)h->npol);
      continue;
    }
    if (iscf != 1) {
      // find_min (moment_from_pola.f90:2415-2455); its 1e-10 guard is a
      // single-precision literal
      k_findmin_dots<<<nb, 256, 0, h->st>>>(h->d_ko_g, h->d_ko_f, P, n, h->d_part);
      LAUNCH_CHECK();
      if ((s = reduce_into(h, nb, 2, h->d_scal + S_KO))) return s;
      double dots[2];
      if ((s = read_scals(h, S_KO, 2, dots))) return s;
      double alpha = -dots[0] / dots[1];
      if (std::fabs(dots[1]) < (double)1e-10f) alpha = 1.0;
      k_findmin_apply<<<nb, 256, 0, h->st>>>(h->d_ko_g, h->d_ko_f, alpha, h->d_ko_muprev, P, n, h->d_mu_ind,
                                             h->d_part);
      LAUNCH_CHECK();
      if ((s = reduce_into(h, nb, 1, h->d_scal + S_RMS))) return s;
      double r2;
      if ((s = read_scal(h, S_RMS, &r2))) return s;
      rmsd = std::sqrt(r2 / (double)h->npol);
    }
    CK(cudaMemcpyAsync(h->d_ko_muprev, h->d_mu_ind, sizeof(double4) * n, cudaMemcpyDeviceToDevice, h->st));
  }
  h->stats.n_pol_iter = iscf;
  h->stats.rmsd = rmsd;
  h->stats.converged = rmsd <= h->p.conv_tol_ind;
  CK(cudaMemcpyAsync(h->d_hist, h->d_mu_ind, sizeof(double4) * n, cudaMemcpyDeviceToDevice, h->st));
  return MDFF_OK;
}

// A x = b for the kO_v4_1 weights with DGESV's semantics
// (moment_from_pola.f90:2500): LU with partial pivoting (first largest
// |pivot|); an exactly zero pivot leaves b as given (INFO > 0, no solve).
static void lu_solve(int n, std::vector<double>& A, double* b) {
  std::vector<int> piv(n);
  for (int k = 0; k < n; ++k) {
    int p = k;
    for (int i = k + 1; i < n; ++i)
      if (std::fabs(A[(size_t)i * n + k]) > std::fabs(A[(size_t)p * n + k])) p = i;
    piv[k] = p;
    if (A[(size_t)p * n + k] == 0.0) return;
    if (p != k)
      for (int j = 0; j < n; ++j) std::swap(A[(size_t)k * n + j], A[(size_t)p * n + j]);
    for (int i = k + 1; i < n; ++i) {
      double l = A[(size_t)i * n + k] / A[(size_t)k * n + k];
      A[(size_t)i * n + k] = l;
      for (int j = k + 1; j < n; ++j) A[(size_t)i * n + j] -= l * A[(size_t)k * n + j];
    }
  }
  for (int k = 0; k < n; ++k) std::swap(b[k], b[piv[k]]);
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < i; ++j) b[i] -= A[(size_t)i * n + j] * b[j];
  for (int i = n - 1; i >= 0; --i) {
    for (int j = i + 1; j < n; ++j) b[i] -= A[(size_t)i * n + j] * b[j];
    b[i] /= A[(size_t)i * n + i];
  }
}

// moment_from_pola_scf_kO_v4 with scf_kO_v4_1 (moment_from_pola.f90:1987-2273)
// and find_min_ex (:2457-2529).  The Gram matrix of the residuals F_h is
// grown by one row per iteration (earlier iterates do not change).
static int solve_ko_v4(mdff_ctx* h, int itime, bool fp32) {
  int n = h->natm, nb = cdiv(n, 256), s;
  PolDev P = poldev(h);
  CK(cudaMemcpyAsync(h->d_Efield, h->d_Estat, sizeof(double4) * n, cudaMemcpyDeviceToDevice, h->st));
  const bool ismd = h->p.calc == MDFF_CALC_MD, isopt = h->p.calc == MDFF_CALC_OPT;
  const bool aspc_on = h->p.algo_ext_dipole == MDFF_EXT_ASPC;
  std::vector<double> G((size_t)kKoHist * kKoHist), Aw;
  double b[kKoHist];
  int iscf = 0;
  double rmsd = HUGE_VAL;
  while (((iscf < h->p.max_scf_pol_iter) && (rmsd > h->p.conv_tol_ind)) ||
         (iscf < h->p.min_scf_pol_iter)) {
    iscf++;
    if (iscf > kKoHist) {
      h->err = "scf_kO_v4_1 ran past its 100 stored iterates";
      return MDFF_ERR_BAD_ARGS;
    }
    bool induce = iscf != 1 || (!ismd && !isopt);
    if (!induce) {
      if (aspc_on && (s = aspc_predict(h, itime))) return s;
      k_count_nonzero<<<nb, 256, 0, h->st>>>(h->d_mu_ind, n, h->d_part);
      LAUNCH_CHECK();
      if ((s = reduce_into(h, nb, 1, h->d_scal + S_KO))) return s;
      double nz;
      if ((s = read_scal(h, S_KO, &nz))) return s;
      induce = nz == 0.0;
    }
    if (induce) {
      k_induce<<<nb, 256, 0, h->st>>>(h->d_Efield, P, n, h->d_mu_ind);
      LAUNCH_CHECK();
    }
    if ((s = upol_pass(h))) return s;
    if ((s = field_of_mu(h, h->d_mu_ind, 0, fp32, h->d_Eind))) return s;
    k_add4<<<nb, 256, 0, h->st>>>(h->d_Estat, h->d_Eind, n, h->d_Efield);
    LAUNCH_CHECK();
    const int m = iscf - 1;
    k_diis_store<<<nb, 256, 0, h->st>>>(h->d_mu_ind, h->d_Eind, P, n, h->d_Fh + (size_t)m * n,
                                        h->d_muh + (size_t)m * n);
    LAUNCH_CHECK();
    k_diis_dots<<<dim3(nb, m + 2), 256, 0, h->st>>>(h->d_Fh, m, n, h->d_ipolar, h->d_Estat, h->d_part);
    LAUNCH_CHECK();
    if ((s = reduce_into(h, nb, m + 2, h->d_ko_x))) return s;
    CK(cudaMemcpyAsync(h->h_ko, h->d_ko_x, sizeof(double) * (m + 2), cudaMemcpyDeviceToHost, h->st));
    CK(cudaStreamSynchronize(h->st));
    for (int j = 0; j <= m; ++j) G[(size_t)m * kKoHist + j] = G[(size_t)j * kKoHist + m] = h->h_ko[j];
    b[m] = h->h_ko[m + 1];
    if (iscf > 1) {
      const int k = m + 1;
      Aw.assign((size_t)k * k, 0.0);
      for (int i = 0; i < k; ++i)
        for (int j = 0; j < k; ++j) Aw[(size_t)i * k + j] = G[(size_t)i * kKoHist + j];
      for (int i = 0; i < k; ++i) h->h_ko[i] = b[i];
      lu_solve(k, Aw, h->h_ko);
      CK(cudaMemcpyAsync(h->d_ko_x, h->h_ko, sizeof(double) * k, cudaMemcpyHostToDevice, h->st));
    }
    k_diis_combine<<<nb, 256, 0, h->st>>>(h->d_Fh, h->d_muh, h->d_ko_x, m + 1, iscf == 1 ? 1 : 0, n, h->d_Estat,
                                          P, h->d_mu_ind, h->d_Efield);
    LAUNCH_CHECK();
    if (iscf == 1 && ismd && aspc_on && (s = aspc_correct(h, itime))) return s;
    k_rmsd_part<<<nb, 256, 0, h->st>>>(h->d_mu_ind, h->d_Efield, P, n, h->d_part);
    LAUNCH_CHECK();
    if ((s = reduce_into(h, nb, 1, h->d_scal + S_RMS))) return s;
    double r2;
    if ((s = read_scal(h, S_RMS, &r2))) return s;
    rmsd = std::sqrt(r2 / (double)h->npol);
  }
  h->stats.n_pol_iter = iscf;
  h->stats.rmsd = rmsd;
  h->stats.converged = rmsd <= h->p.conv_tol_ind;
  CK(cudaMemcpyAsync(h->d_hist, h->d_mu_ind, sizeof(double4) * n, cudaMemcpyDeviceToDevice, h->st));
  return MDFF_OK;
}

// the step scalars after an inner CG iteration: rz <- rz_new, count, rmsd of
// the recurrence residual, and (inside the graph) the while-loop condition
__global__ void k_cg_inner_check(double* __restrict__ sc, int npol, int in_graph,
                                 cudaGraphConditionalHandle hc) {
  pdl_wait();
  pdl_trigger();
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  sc[0] = sc[3];
  double it = sc[6] + 1.0;
  sc[6] = it;
  double rm = sqrt(sc[4] / (double)npol);
  sc[8] = rm;
  if (in_graph) cudaGraphSetConditional(hc, (rm > sc[5] && it < sc[7]) ? 1u : 0u);
}

// head of the CG graph: the decision solve_cg's host loop takes after a FP64
// residual (stop, or the inner tolerance and whether the recurrence is
// trusted), taken on the device so that the graph follows the residual
// without a host round trip; sets the WHILE condition of the inner loop
__global__ void k_cg_plan(double* __restrict__ sc, double* __restrict__ plan, int npol, double tol,
                          double maxit, int fp32, cudaGraphConditionalHandle hc) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const double rmsd = sqrt(sc[1] / (double)npol);
  const double outer = plan[2];
  plan[0] = rmsd;
  const bool stop = rmsd <= tol || sc[6] >= maxit || outer >= 8.0;
  plan[1] = stop ? 1.0 : 0.0;
  if (!stop) {
    const bool trust = !fp32 || kCgGap * rmsd <= 0.5 * tol;
    sc[5] = !fp32 ? tol : (trust ? tol - kCgGap * rmsd : fmax(tol, 1e-4 * rmsd));
    sc[7] = maxit;
    plan[2] = outer + 1.0;
    plan[3] = trust ? 1.0 : 0.0;
  }
  cudaGraphSetConditional(hc, stop ? 0u : 1u);
}

__global__ void k_setd2(double* __restrict__ a, double va, double* __restrict__ b, double vb) {
  pdl_wait();
  pdl_trigger();
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    *a = va;
    *b = vb;
  }
}

// one inner CG iteration: p -> T p -> q = A p; x, r, z updated; p <- z + beta p
static bool rho_acc_enabled(const mdff_ctx* h);

static int cg_iteration(mdff_ctx* h, bool fp32, int in_graph, cudaGraphConditionalHandle hc) {
  int n = h->natm, nb = cdiv(n, 256), s;
  PolDev P = poldev(h);
  double* sc = h->d_scal + S_CG;
  // with the accumulated structure factor the operator's rho'(p) stays in
  // rhoA for the update, which adds al rho'(p)
  const bool acc = rho_acc_enabled(h);
  h->rec_mode = acc ? REC_NEED_RHOA : REC_PLAIN;
  s = field_of_mu(h, h->d_pv, 1, fp32, h->d_Tp, fp32);
  h->rec_mode = REC_PLAIN;
  if (s) return s;
  PDL_CHECK(pdl_launch(k_cg_Ap, dim3(nb), dim3(256), 0, h->st, (const double4*)h->d_pv,
                       (const double4*)h->d_Tp, P, n, h->d_qv, h->d_part));
  if ((s = reduce_into(h, nb, 1, sc + 2))) return s;
  PDL_CHECK(pdl_launch(k_cg_update, dim3(nb), dim3(256), 0, h->st, (const double*)(sc + 0),
                       (const double*)(sc + 2), P, n, h->d_pv, (const double4*)h->d_qv, h->d_mu_ind, h->d_r,
                       h->d_z, h->d_part, acc ? h->d_rho_acc : (double2*)nullptr, (const double2*)h->d_rhoA,
                       h->nk));
  if ((s = reduce_into(h, nb, 2, sc + 3))) return s;
  PDL_CHECK(pdl_launch(k_cg_dir, dim3(nb), dim3(256), 0, h->st, (const double*)(sc + 0),
                       (const double*)(sc + 3), n, (const double4*)h->d_z, h->d_pv,
                       (const CellC*)h->d_cell, fp32 ? h->d_w32 : (float4*)nullptr, h->d_mu32, slotw(h)));
  PDL_CHECK(pdl_launch(k_cg_inner_check, dim3(1), dim3(32), 0, h->st, sc, h->npol, in_graph, hc));
  return MDFF_OK;
}

// graph: while (cond) { cg_iteration }  -- built once per buffer generation
static int build_cg_graph(mdff_ctx* h, bool fp32) {
  if (h->cg_exec) cudaGraphExecDestroy(h->cg_exec);
  if (h->cg_graph) cudaGraphDestroy(h->cg_graph);
  h->cg_exec = nullptr;
  h->cg_graph = nullptr;
  cudaGraph_t g;
  CK(cudaGraphCreate(&g, 0));
  h->cg_graph = g;
  cudaGraphConditionalHandle hc;
  CK(cudaGraphConditionalHandleCreate(&hc, g, 1, cudaGraphCondAssignDefault));
  // head: k_cg_plan decides from the FP64 residual and sets the condition
  double* sc = h->d_scal + S_CG;
  double* plan = h->d_scal + S_CGP;
  int npol = h->npol;
  double tol = h->p.cg_tol > 0 ? h->p.cg_tol : h->p.conv_tol_ind;
  double maxit = (double)(h->p.cg_max_iter > 0 ? h->p.cg_max_iter : 200);
  int f32 = fp32 ? 1 : 0;
  void* kargs[] = {&sc, &plan, &npol, &tol, &maxit, &f32, &hc};
  cudaKernelNodeParams kp = {};
  kp.func = (void*)k_cg_plan;
  kp.gridDim = dim3(1);
  kp.blockDim = dim3(32);
  kp.sharedMemBytes = 0;
  kp.kernelParams = kargs;
  cudaGraphNode_t head;
  CK(cudaGraphAddKernelNode(&head, g, nullptr, 0, &kp));
  cudaGraphNodeParams cp = {};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = hc;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaGraphNode_t node;
  CK(cudaGraphAddNode(&node, g, &head, 1, &cp));
  cudaGraph_t body = cp.conditional.phGraph_out[0];
  bool prof = h->prof, ovl = h->call_overlap;
  h->prof = false;
  h->call_overlap = false;
  int launches0 = h->launches;
  CK(cudaStreamBeginCaptureToGraph(h->st, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
  int s = cg_iteration(h, fp32, 1, hc);
  cudaGraph_t captured;
  cudaError_t e = cudaStreamEndCapture(h->st, &captured);
  h->prof = prof;
  h->call_overlap = ovl;
  h->cg_body_launches = h->launches - launches0;
  h->launches = launches0;
  if (s) return s;
  if (e != cudaSuccess) {
    h->err = std::string("cudaStreamEndCapture: ") + cudaGetErrorString(e);
    return MDFF_ERR_CUDA;
  }
  CK(cudaGraphInstantiate(&h->cg_exec, g, 0));
  h->cg_gen = h->gen;
  h->cg_fp32 = fp32 ? 1 : 0;
  return MDFF_OK;
}

// preconditioned CG on (alpha^-1 - T) mu = E_stat.  fp32: matvecs in FP32,
// residual refreshed with an FP64 matvec (iterative refinement).  The inner
// iterations run as one CUDA-graph launch (device-side while loop, headed by
// the device-side stop / tolerance decision); the host reads the outcome
// once per outer (FP64 residual) iteration.  Without the graph (per-kernel
// profiling) the host loop below takes the same decisions itself.  The pieces
// (prologue, FP64 residual, the outcome of a graph launch, epilogue) are also
// the parts of the whole-step graph (run_engforce_graph).

static double cg_tol_of(const mdff_ctx* h) { return h->p.cg_tol > 0 ? h->p.cg_tol : h->p.conv_tol_ind; }
static int cg_maxit_of(const mdff_ctx* h) { return h->p.cg_max_iter > 0 ? h->p.cg_max_iter : 200; }

// first guess (ASPC predictor for calc md / opt, else alpha E_stat) and the
// loop counters
static int cg_prologue(mdff_ctx* h, int itime) {
  int n = h->natm, nb = cdiv(n, 256), s;
  PolDev P = poldev(h);
  if (h->p.calc == MDFF_CALC_MD || h->p.calc == MDFF_CALC_OPT) {
    if ((s = aspc_predict(h, itime))) return s;
  } else {
    k_induce<<<nb, 256, 0, h->st>>>(h->d_Estat, P, n, h->d_mu_ind);
    LAUNCH_CHECK();
  }
  double* sc = h->d_scal + S_CG;
  double* plan = h->d_scal + S_CGP;
  PDL_CHECK(pdl_launch(k_setd2, dim3(1), dim3(32), 0, h->st, sc + 6, 0.0, sc + 7, (double)cg_maxit_of(h)));
  PDL_CHECK(pdl_launch(k_setd2, dim3(1), dim3(32), 0, h->st, plan + 1, 0.0, plan + 2, 0.0));
  return MDFF_OK;
}

// true residual of the current dipoles (FP64 matvec), the CG start vectors
// and their norms (sc[0], sc[1]).  With the FP32 operator's pair cache the
// real-space half applies the cached pair tensor (FP64 products and sums):
// the refinement then converges on the system its operator approximates.
static int cg_residual(mdff_ctx* h, bool fp32) {
  int n = h->natm, nb = cdiv(n, 256), s;
  PolDev P = poldev(h);
  if ((s = field_of_mu(h, h->d_mu_ind, 1, false, h->d_Tp, false, fp32))) return s;
  PDL_CHECK(pdl_launch(k_cg_init, dim3(nb), dim3(256), 0, h->st, h->d_Estat, h->d_Tp, h->d_mu_ind, P, n, h->d_r, h->d_z, h->d_pv, h->d_part,
                                   h->d_cell, fp32 ? h->d_w32 : nullptr, h->d_mu32, slotw(h)));
  return reduce_into(h, nb, 2, h->d_scal + S_CG);
}

// The static pass can merge with the first FP64 residual when the first
// guess does not need the static field: the ASPC predictor (calc md / opt)
// of the CG solver, without static dipoles (whose field the static pass adds)
static bool cg_merged(const mdff_ctx* h) {
  return h->p.lcoulomb && h->lpolar && h->p.solver == MDFF_SOLVER_CG && !h->ldip_static &&
         (h->p.calc == MDFF_CALC_MD || h->p.calc == MDFF_CALC_OPT);
}

// The force pass takes its structure factor from the solve's accumulation:
// after the merged first residual (rho' of the charges and x0) every CG step
// adds al rho'(p), so the accumulation is rho' of the charges and the final
// dipoles, which are the total dipoles here (no static dipoles, no Wannier
// centres)
static bool rho_acc_enabled(const mdff_ctx* h) { return cg_merged(h) && !h->lwannier && h->nk > 0; }

// the static field plus the field of the first guess x0 (real space on the
// side stream: FP64, or in the mixed engine the FP32 static pass that writes
// the pair cache of its CG operator and applies the cached pair tensor to x0
// with FP64 products and sums; reciprocal space in FP64 with the charges and
// x0 together), then the CG start vectors from b + T x0 as one vector: one
// pass over pairs and k vectors instead of the static pass and a residual pass
static int merged_residual(mdff_ctx* h, bool fp32) {
  int n = h->natm, nb = cdiv(n, 256), s;
  PolDev P = poldev(h);
  double4* E = h->d_Tp;
  CK(cudaMemsetAsync(E, 0, sizeof(double4) * n, h->st));
  double cutsq = h->p.cutlongrange * h->p.cutlongrange;
  int nbw = cdiv((long)n * 32, 256);
  if (h->p.lsurf && (s = moments(h, h->d_mu_ind, 1, h->d_scal + S_MOM2))) return s;
  cudaStream_t rs;
  if ((s = rs_fork(h, &rs))) return s;
  int pr = prof_begin(h, KC_ESFIELD, 0);
  if (fp32 && h->d_ddr) {
#define SRC(K)                                                                                    \
  k_static_cache<K, true><<<nbw, 256, 0, rs>>>(h->d_s, h->d_q, h->d_itype, h->d_ipolar, h->L.nbr,  \
                                               h->L.nnb, h->L.cap, n, h->d_cell, h->d_estab,       \
                                               h->ntype, h->p.alphaES, cutsq, h->task_qq ? 1 : 0,  \
                                               E, h->d_ddr, h->d_ddb1, h->d_ddj, h->d_ddn,         \
                                               h->p.thole_type, h->d_mu_ind)
    if (h->tt_k == 4) SRC(4);
    else SRC(0);
#undef SRC
    h->dd_cache_ok = true;
  } else {
#define ESF2(K)                                                                                    \
  k_es_field<double, true, true, K><<<nbw, 256, 0, rs>>>(h->d_s, h->d_q, h->d_itype, h->d_ipolar,  \
                                                         h->d_mu_ind, h->L.nbr, h->L.nnb, h->L.cap, \
                                                         n, h->d_cell, h->d_estab, h->ntype,       \
                                                         h->p.alphaES, cutsq, 1, 1, E, h->p.thole_type)
    if (h->tt_k == 4) ESF2(4);
    else ESF2(0);
#undef ESF2
  }
  LAUNCH_CHECK();
  prof_end(h, pr);
  // (its rho' of the charges and x0 also starts the solve's accumulation)
  const bool acc = rho_acc_enabled(h);
  h->rec_mode = acc ? REC_SAVE_ACC : REC_PLAIN;
  s = rec_pass(h, false, h->d_mu_ind, h->task_qq ? 1 : 0, 1, 0, E, nullptr,
               self_field(h, h->d_mu_ind, h->d_scal + S_MOM2));
  h->rec_mode = REC_PLAIN;
  if (s) return s;
  h->rho_acc_ok = acc;
  PDL_CHECK(pdl_launch(k_cg_init, dim3(nb), dim3(256), 0, h->st, (const double4*)nullptr, (const double4*)E,
                       (const double4*)h->d_mu_ind, P, n, h->d_r, h->d_z, h->d_pv, h->d_part,
                       (const CellC*)h->d_cell, fp32 ? h->d_w32 : (float4*)nullptr, h->d_mu32, slotw(h)));
  return reduce_into(h, nb, 2, h->d_scal + S_CG);
}

// the solve's first FP64 residual: merged with the static pass when it can be
static int cg_first_residual(mdff_ctx* h, bool fp32) {
  return cg_merged(h) ? merged_residual(h, fp32) : cg_residual(h, fp32);
}

// outcome of one launch of the CG graph from the host copies of the scalars:
// true when the solve is finished; *rmsd, *it as the loop leaves them
static bool cg_graph_outcome(const mdff_ctx* h, double* rmsd, int* it) {
  const double* hs = h->h_scal;
  const double* hp = hs + S_CGP;
  *rmsd = hp[0];
  *it = (int)hs[S_CG + 6];
  if (hp[1] != 0.0) return true;  // converged (or a limit) at the FP64 residual
  if (hp[3] != 0.0) {             // trusted recurrence: its residual is final
    double rin = hs[S_CG + 8];
    if (rin <= hs[S_CG + 5]) {
      *rmsd = rin;
      return true;
    }
    if (*it >= cg_maxit_of(h)) return true;
  }
  return false;
}

// u_pol of the converged dipoles, which become the newest ASPC history entry
static int cg_epilogue(mdff_ctx* h) {
  int n = h->natm, nb = cdiv(n, 256), s;
  PolDev P = poldev(h);
  PDL_CHECK(pdl_launch(k_upol_part, dim3(nb), dim3(256), 0, h->st, h->d_mu_ind, P, n, h->d_part));
  if ((s = reduce_into(h, nb, 1, h->d_scal + S_UPOL))) return s;
  CK(cudaMemcpyAsync(h->d_hist, h->d_mu_ind, sizeof(double4) * n, cudaMemcpyDeviceToDevice, h->st));
  return MDFF_OK;
}

static void cg_stats(mdff_ctx* h, double rmsd0, double rmsd, int it, int nres) {
  h->stats.rmsd_initial = rmsd0;
  h->stats.n_fp64_residuals = nres;
  h->stats.n_pol_iter = it;
  h->stats.rmsd = rmsd;
  h->stats.converged = rmsd <= cg_tol_of(h);
}

// further outer iterations after a first graph launch that did not finish
// the solve (the FP64 residual of the dipoles it left, then the CG graph)
// (*first: the rmsd of the first FP64 residual of the solve, when it is this
// call's; estat_missing: the static field was merged into the first
// residual and is formed alone before the next one)
static int cg_continue(mdff_ctx* h, bool fp32, double* rmsd, int* it, int* nres, double* first,
                       bool estat_missing) {
  int s;
  while (true) {
    if (estat_missing) {
      if ((s = static_field(h, fp32))) return s;
      estat_missing = false;
    }
    if ((s = cg_residual(h, fp32))) return s;
    ++*nres;
    CK(cudaGraphLaunch(h->cg_exec, h->st));
    CK(cudaMemcpyAsync(h->h_scal + S_CG, h->d_scal + S_CG, sizeof(double) * (S_CGP + 4 - S_CG),
                       cudaMemcpyDeviceToHost, h->st));
    CK(cudaStreamSynchronize(h->st));
    if (*nres == 1 && first) *first = h->h_scal[S_CGP];
    if (cg_graph_outcome(h, rmsd, it)) return MDFF_OK;
  }
}

static int solve_cg(mdff_ctx* h, int itime, bool fp32) {
  int s;
  double tol = cg_tol_of(h);
  int maxit = cg_maxit_of(h);
  double* sc = h->d_scal + S_CG;
  bool use_graph = !h->prof;
  if ((s = cg_prologue(h, itime))) return s;
  double rmsd = HUGE_VAL, rmsd0 = HUGE_VAL;
  int outer = 0, it = 0, nres = 0;
  const bool merged = cg_merged(h);
  if (use_graph) {
    if ((s = cg_first_residual(h, fp32))) return s;
    nres = 1;
    // (built after the first residual, which decides whether the FP32 pair
    // cache serves the operator)
    if (h->cg_exec == nullptr || h->cg_gen != h->gen || h->cg_fp32 != (fp32 ? 1 : 0))
      if ((s = build_cg_graph(h, fp32))) return s;
    CK(cudaGraphLaunch(h->cg_exec, h->st));
    CK(cudaMemcpyAsync(h->h_scal + S_CG, h->d_scal + S_CG, sizeof(double) * (S_CGP + 4 - S_CG),
                       cudaMemcpyDeviceToHost, h->st));
    CK(cudaStreamSynchronize(h->st));
    rmsd0 = h->h_scal[S_CGP];
    if (!cg_graph_outcome(h, &rmsd, &it) &&
        (s = cg_continue(h, fp32, &rmsd, &it, &nres, nullptr, merged)))
      return s;
    h->launches += h->cg_body_launches * it + nres;  // + one k_cg_plan per graph launch
    cg_stats(h, rmsd0, rmsd, it, nres);
    return cg_epilogue(h);
  }
  bool need_residual = true, estat_missing = merged;
  while (true) {
    if (need_residual) {
      if (nres == 0) {
        if ((s = cg_first_residual(h, fp32))) return s;
      } else {
        if (estat_missing) {
          if ((s = static_field(h, fp32))) return s;
          estat_missing = false;
        }
        if ((s = cg_residual(h, fp32))) return s;
      }
      CK(cudaMemcpyAsync(h->h_scal + S_CG, sc, sizeof(double) * 9, cudaMemcpyDeviceToHost, h->st));
      CK(cudaStreamSynchronize(h->st));
      ++nres;
      rmsd = std::sqrt(h->h_scal[S_CG + 1] / (double)h->npol);
      if (nres == 1) rmsd0 = rmsd;
      it = (int)h->h_scal[S_CG + 6];
      if (rmsd <= tol || it >= maxit || outer >= 8) break;
    }
    outer++;
    // Inner CG on the residual.  FP64: the recurrence residual is exact to
    // rounding, so its convergence is final.  FP32 operator: the recurrence
    // drifts from the true residual by about the FP32 matvec error (~1e-6
    // relative) summed over the corrections, at most kCgGap = 3e-6 of the
    // residual it started from (measured); when that bound is at most half
    // the tolerance the recurrence is trusted down to the tolerance less the
    // bound and no second FP64 residual is formed, else it reduces the
    // residual by 1e-4 and a new FP64 residual restarts it (iterative
    // refinement).
    bool trust = !fp32 || kCgGap * rmsd <= 0.5 * tol;
    double tol_in = !fp32 ? tol : (trust ? tol - kCgGap * rmsd : std::max(tol, 1e-4 * rmsd));
    k_setd2<<<1, 32, 0, h->st>>>(sc + 5, tol_in, sc + 7, (double)maxit);
    LAUNCH_CHECK();
    while (true) {
      if ((s = cg_iteration(h, fp32, 0, 0))) return s;
      CK(cudaMemcpyAsync(h->h_scal + S_CG, sc, sizeof(double) * 9, cudaMemcpyDeviceToHost, h->st));
      CK(cudaStreamSynchronize(h->st));
      if (!(h->h_scal[S_CG + 8] > tol_in && h->h_scal[S_CG + 6] < maxit)) break;
    }
    need_residual = true;
    if (trust) {
      double rin = h->h_scal[S_CG + 8];
      it = (int)h->h_scal[S_CG + 6];
      if (rin <= tol_in) {
        rmsd = rin;
        break;
      }
      if (it >= maxit) break;
    }
  }
  cg_stats(h, rmsd0, rmsd, it, nres);
  return cg_epilogue(h);
}

// One engforce on the positions in h->d_pos; results stay on the device,
// scalars land in h->h_scal.  It is three parts: ef_front (list, short
// range on its side stream, phase tables, static field), the dipole solve,
// ef_back (the converged dipoles' force pass, the joins and the copies of the
// scalars and flags to the host), and ef_status on the host after the sync.
// ef_back can run again on the same front: the short-range pass writes its
// own buffer, which ef_back copies into the forces before adding the rest.

static int ef_front(mdff_ctx* h, bool fp32) {
  int n = h->natm, s;
  h->rho_acc_ok = false;
  PDL_CHECK(pdl_launch(k_kardir, dim3(cdiv(n, 256)), dim3(256), 0, h->st, h->d_pos, n, h->d_cell, h->d_itype,
                       h->d_ipolar, h->d_q, h->d_s));
  if ((s = list_update(h))) return s;
  CK(cudaMemsetAsync(h->d_scal, 0, sizeof(double) * S_NSCAL, h->st));
  int nbw = cdiv((long)n * 32, 256);
  if (h->lsr) {
    int do_bmh = (h->p.lbmhft || h->p.lbmhftd) ? 1 : 0;
    // beside the Coulomb chain; joined before the force pass
    cudaStream_t ss;
    if ((s = sr_fork(h, &ss))) return s;
    int pr = prof_begin(h, KC_SR, 0);
    // short range stays FP64 in the mixed mode too: BKS-type pair forces of
    // tens of eV/A cancel to net forces of a few eV/A, and FP32 rounding of the
    // pair terms alone gives ~1e-5 relative force error
#define SRK(MODE)                                                                              \
  k_shortrange<double, MODE><<<nbw, 256, 0, ss>>>(h->d_s, h->d_itype, h->L.nbr, h->L.nnb,        \
                                                  h->L.cap, n, h->d_cell, h->d_nbtab, h->ntype,    \
                                                  h->p.lbmhftd, h->p.trunc, h->d_fsr, h->d_part2)
    if (do_bmh && h->p.lnmlj) SRK(3);
    else if (do_bmh) SRK(1);
    else SRK(2);
#undef SRK
    LAUNCH_CHECK();
    prof_end(h, pr);
    k_reduce_partials<<<kSRPart, 256, 0, ss>>>(h->d_part2, nbw, kSRPart, h->d_scal + S_SR);
    LAUNCH_CHECK();
  }
  // per-call flags: [0] catastrophe, [1] a tensor-core wait gave up, [2] Wannier count
  CK(cudaMemsetAsync(h->d_cata, 0, 3 * sizeof(int), h->st));
  if (h->p.lcoulomb) {
    if ((s = build_tables(h))) return s;
    CK(cudaMemsetAsync(h->d_mu_ind, 0, sizeof(double4) * n, h->st));
    h->stats.n_pol_iter = 0;
    if (h->lpolar) {
      // the ASPC history as the call found it (a redo after a list overflow
      // restores it: the predictors shift it in place)
      if (h->d_hist_save)
        CK(cudaMemcpyAsync(h->d_hist_save, h->d_hist, sizeof(double4) * MDFF_ASPC_DEPTH * n,
                           cudaMemcpyDeviceToDevice, h->st));
      // (merged into the solve's first residual when it can be)
      if (!cg_merged(h) && (s = static_field(h, fp32))) return s;
    }
  }
  return MDFF_OK;
}

static int ef_solve(mdff_ctx* h, int itime, bool fp32) {
  if (!h->p.lcoulomb || !h->lpolar) return MDFF_OK;
  const int algo = h->p.algo_moment_from_pola;
  if (h->p.solver == MDFF_SOLVER_CG) return solve_cg(h, itime, fp32);
  if (algo == MDFF_ALGO_KO_V1 || algo == MDFF_ALGO_KO_V2) return solve_ko_v12(h, itime, fp32, algo == MDFF_ALGO_KO_V2);
  if (algo == MDFF_ALGO_KO_V4_1) return solve_ko_v4(h, itime, fp32);
  return solve_scf(h, itime, fp32);
}

static int ef_back(mdff_ctx* h, bool fp32) {
  int n = h->natm, s;
  int nbw = cdiv((long)n * 32, 256);
  if (h->p.lcoulomb) {
    // dipoles of the Wannier centres (moment_from_pola.f90:136-147)
    if (h->lwannier) {
      k_wfc_dipoles<<<nbw, 256, 0, h->st>>>(h->d_s, h->d_itype, h->d_lwfc, h->L.nbr, h->L.nnb, h->L.cap, n,
                                            h->d_cell, h->p.rcut_wfc, h->d_mu_wfc, h->d_cata + 2);
      LAUNCH_CHECK();
    }
    PDL_CHECK(pdl_launch(k_mu_total, dim3(cdiv(n, 256)), dim3(256), 0, h->st, h->d_dipia, h->d_mu_ind,
                                                (h->lwannier && h->p.ldip_wfc) ? h->d_mu_wfc : nullptr, n,
                                                h->d_mu_tot, h->d_cata, h->d_q, fp32 ? h->d_qm32 : nullptr));
    CK(cudaMemsetAsync(h->d_E, 0, sizeof(double4) * n, h->st));
  }
  // the forces start from the short-range pass's (zero without one)
  if ((s = sr_join(h))) return s;
  if (h->lsr)
    CK(cudaMemcpyAsync(h->d_force, h->d_fsr, sizeof(double) * 3 * n, cudaMemcpyDeviceToDevice, h->st));
  else
    CK(cudaMemsetAsync(h->d_force, 0, sizeof(double) * 3 * n, h->st));
  if (h->p.lcoulomb) {
    double cutsq = h->p.cutlongrange * h->p.cutlongrange;
    // the real-space force pass runs beside the reciprocal one, which joins
    // it before its final sum
    cudaStream_t rs;
    if ((s = rs_fork(h, &rs))) return s;
    int prf = prof_begin(h, KC_ESFORCE, 0);
#define ESFORCE(R, K, TH)                                                                        \
  k_es_force<R, K, TH><<<nbw, 256, 0, rs>>>(h->d_s, h->d_q, h->d_itype, h->d_mu_tot, h->d_qm32,  \
                                            h->L.nbr, h->L.nnb, h->L.cap, n, h->d_cell,          \
                                            h->d_estab, h->ntype, h->p.alphaES, cutsq,           \
                                            h->task_qq, h->task_qd, h->task_dd, 1, h->coul_unit, \
                                            h->d_E, h->d_force, h->d_part2)
    const bool thole = h->p.thole_type != MDFF_THOLE_NONE;
    if (fp32 && thole) ESFORCE(float, 0, true);
    else if (fp32 && h->tt_k == 4) ESFORCE(float, 4, false);
    else if (fp32) ESFORCE(float, 0, false);
    else if (thole) ESFORCE(double, 0, true);
    else if (h->tt_k == 4) ESFORCE(double, 4, false);
    else ESFORCE(double, 0, false);
#undef ESFORCE
    LAUNCH_CHECK();
    prof_end(h, prf);
    k_reduce_partials<<<kESPart, 256, 0, rs>>>(h->d_part2, nbw, kESPart, h->d_scal + S_DIR);
    LAUNCH_CHECK();
    int has_mu = (h->task_qd || h->task_dd) ? 1 : 0;
    if ((s = moments(h, h->d_mu_tot, 1, h->d_scal + S_MOM))) return s;
    h->rec_mode = (h->rho_acc_ok && rho_acc_enabled(h)) ? REC_FROM_ACC : REC_PLAIN;
    s = rec_pass(h, fp32, h->d_mu_tot, h->task_qq ? 1 : 0, has_mu, 1, h->d_E, h->d_scal + S_REC,
                 self_field(h, h->d_mu_tot, h->d_scal + S_MOM));
    h->rec_mode = REC_PLAIN;
    if (s) return s;
  }
  if ((s = rs_join(h))) return s;
  CK(cudaMemcpyAsync(h->h_scal, h->d_scal, sizeof(double) * S_NSCAL, cudaMemcpyDeviceToHost, h->st));
  CK(cudaMemcpyAsync(h->h_flags, h->L.flags, sizeof(int) * 4, cudaMemcpyDeviceToHost, h->st));
  CK(cudaMemcpyAsync(h->h_cata, h->d_cata, 3 * sizeof(int), cudaMemcpyDeviceToHost, h->st));
  return MDFF_OK;
}

// in-place kardir/dirkar round trips of the global positions that the
// reference's engforce makes for this call: one per short-range routine
// (non_bonded.f90:716,823 and :1113,1221), one per multipole_ES_dir
// (ewald_dir.f90:138,739: the static field, one per SCF iteration, the final
// pass) and one for the Wannier centres (moment_from_pola.f90:685,803).
// Defined for the reference's own solver (SCF, algorithm 'scf'); -1 otherwise.
static int kardir_count(const mdff_ctx* h) {
  if (h->p.lcoulomb && h->lpolar &&
      (h->p.solver != MDFF_SOLVER_SCF || h->p.algo_moment_from_pola != MDFF_ALGO_SCF))
    return -1;
  int n = (h->p.lnmlj ? 1 : 0) + ((h->p.lbmhft || h->p.lbmhftd) ? 1 : 0);
  if (h->p.lcoulomb) n += 1 + (h->lpolar ? 1 + h->stats.n_pol_iter : 0) + (h->lwannier ? 1 : 0);
  return n;
}

// status of a call from the host copies of its flags (after the sync)
static int ef_status(mdff_ctx* h) {
  h->stats.n_kardir = kardir_count(h);
  h->stats.list_rebuilds = h->h_flags[3];
  h->stats.list_needed = h->h_flags[2] * h->natm;
  if (h->h_flags[1]) return MDFF_ERR_LIST_OVERFLOW;
  if (h->h_cata[1]) {
    h->err = h->h_cata[1] == 2 ? "tensor-core reciprocal kernel launched with too little shared memory"
                               : "a tensor-core reciprocal-kernel wait gave up";
    return MDFF_ERR_TIMEOUT;
  }
  if (h->h_cata[2]) {
    h->err = "a Wannier centre is missing for an ion of a type with lwfc > 0 (moment_from_pola.f90:731-737)";
    return MDFF_ERR_BAD_ARGS;
  }
  if (h->h_cata[0]) return MDFF_ERR_CATASTROPHE;
  if (h->lpolar && !h->stats.converged && h->p.fail_on_nonconvergence) return MDFF_ERR_NOT_CONVERGED;
  return MDFF_OK;
}

static int run_engforce(mdff_ctx* h, int itime) {
  bool fp32 = h->p.precision == MDFF_PREC_MIXED;
  int s;
  h->launches = 0;
  // side work of an earlier call that ended early is joined first
  if ((s = sr_join(h)) || (s = rs_join(h))) return s;
  h->call_overlap = h->overlap && !h->prof;
  if ((s = ef_front(h, fp32))) return s;
  if ((s = ef_solve(h, itime, fp32))) return s;
  if ((s = ef_back(h, fp32))) return s;
  CK(cudaStreamSynchronize(h->st));
  prof_collect(h);
  return ef_status(h);
}

// ---------------------------------------------------------------------------
// Whole-step graph.  In the steady state of an MD run with the CG solver (the
// list built, the ASPC order ramp past, no per-kernel profiling) one
// engforce is the same ~130 launches every step; they are replayed as one
// CUDA graph: ef_front + the CG prologue and first FP64 residual (captured),
// k_cg_plan, the CG inner WHILE node, the CG epilogue + ef_back (captured).
// The host then reads the scalars once.  A solve that needs another outer
// iteration (rare: the trusted-recurrence test failed) continues with the CG
// graph and repeats ef_back; a list overflow redoes the call without the
// graph after growing the list.

static bool step_graph_usable(const mdff_ctx* h, int itime) {
  if (h->prof || !h->have_list || h->lwannier) return false;
  if (!h->lpolar || !h->p.lcoulomb) return true;
  if (h->p.solver != MDFF_SOLVER_CG) return false;
  if (h->p.calc == MDFF_CALC_MD || h->p.calc == MDFF_CALC_OPT)
    return itime >= h->p.extrapolate_order + 1;  // constant ASPC coefficients
  return true;
}

static int capture_begin(mdff_ctx* h) {
  CK(cudaStreamBeginCapture(h->st, cudaStreamCaptureModeThreadLocal));
  return MDFF_OK;
}
static int capture_end(mdff_ctx* h, int s, cudaGraph_t* g) {
  cudaError_t e = cudaStreamEndCapture(h->st, g);
  if (s) {
    if (e == cudaSuccess && *g) cudaGraphDestroy(*g);
    *g = nullptr;
    return s;
  }
  if (e != cudaSuccess) {
    h->err = std::string("cudaStreamEndCapture: ") + cudaGetErrorString(e);
    return MDFF_ERR_CUDA;
  }
  return MDFF_OK;
}

static void step_graph_free(mdff_ctx* h) {
  if (h->step_exec) cudaGraphExecDestroy(h->step_exec);
  if (h->step_graph) cudaGraphDestroy(h->step_graph);
  h->step_exec = nullptr;
  h->step_graph = nullptr;
}

static int build_step_graph(mdff_ctx* h, int itime, bool fp32) {
  step_graph_free(h);
  const bool cg = h->p.lcoulomb && h->lpolar;
  int s;
  // the operator reads the FP32 pair cache when the front fills it
  if (cg && fp32 && h->d_ddr) h->dd_cache_ok = true;
  if (cg && (h->cg_exec == nullptr || h->cg_gen != h->gen || h->cg_fp32 != (fp32 ? 1 : 0)))
    if ((s = build_cg_graph(h, fp32))) return s;
  bool prof = h->prof;
  h->prof = false;
  h->call_overlap = h->overlap;
  int launches0 = h->launches;
  h->launches = 0;
  // front: list, short range, tables, static field, CG prologue + FP64 residual
  cudaGraph_t gA = nullptr, gB = nullptr;
  if ((s = capture_begin(h))) return s;
  s = ef_front(h, fp32);
  if (!s && cg) s = cg_prologue(h, itime);
  if (!s && cg) s = cg_first_residual(h, fp32);
  // a capture ends joined: the short-range pass (~100 us) joins at the end of
  // the front, which takes longer (static field + FP64 residual)
  if (!s) s = sr_join(h);
  if ((s = capture_end(h, s, &gA))) return s;
  // back: CG epilogue, force pass, copies to the host
  if ((s = capture_begin(h))) {
    cudaGraphDestroy(gA);
    return s;
  }
  s = cg ? cg_epilogue(h) : MDFF_OK;
  if (!s) s = ef_back(h, fp32);
  if ((s = capture_end(h, s, &gB))) {
    cudaGraphDestroy(gA);
    return s;
  }
  h->step_launches = h->launches;
  h->launches = launches0;
  h->prof = prof;
  cudaGraph_t g;
  CK(cudaGraphCreate(&g, 0));
  h->step_graph = g;
  cudaGraphNode_t nA, nB, last;
  CK(cudaGraphAddChildGraphNode(&nA, g, nullptr, 0, gA));
  last = nA;
  if (cg) {
    // k_cg_plan + the inner WHILE node, as in the CG graph
    cudaGraphConditionalHandle hc;
    CK(cudaGraphConditionalHandleCreate(&hc, g, 1, cudaGraphCondAssignDefault));
    double* sc = h->d_scal + S_CG;
    double* plan = h->d_scal + S_CGP;
    int npol = h->npol;
    double tol = cg_tol_of(h);
    double maxit = (double)cg_maxit_of(h);
    int f32 = fp32 ? 1 : 0;
    void* kargs[] = {&sc, &plan, &npol, &tol, &maxit, &f32, &hc};
    cudaKernelNodeParams kp = {};
    kp.func = (void*)k_cg_plan;
    kp.gridDim = dim3(1);
    kp.blockDim = dim3(32);
    kp.kernelParams = kargs;
    cudaGraphNode_t head;
    CK(cudaGraphAddKernelNode(&head, g, &last, 1, &kp));
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = hc;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t wnode;
    CK(cudaGraphAddNode(&wnode, g, &head, 1, &cp));
    bool ovl = h->call_overlap;
    h->call_overlap = false;
    int l0 = h->launches;
    CK(cudaStreamBeginCaptureToGraph(h->st, cp.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                     cudaStreamCaptureModeThreadLocal));
    s = cg_iteration(h, fp32, 1, hc);
    cudaGraph_t captured;
    cudaError_t e = cudaStreamEndCapture(h->st, &captured);
    h->call_overlap = ovl;
    h->launches = l0;
    if (s) return s;
    if (e != cudaSuccess) {
      h->err = std::string("cudaStreamEndCapture: ") + cudaGetErrorString(e);
      return MDFF_ERR_CUDA;
    }
    last = wnode;
  }
  CK(cudaGraphAddChildGraphNode(&nB, g, &last, 1, gB));
  cudaGraphDestroy(gA);
  cudaGraphDestroy(gB);
  CK(cudaGraphInstantiate(&h->step_exec, g, 0));
  h->step_gen = h->gen;
  h->step_fp32 = fp32 ? 1 : 0;
  return MDFF_OK;
}

// one engforce through the whole-step graph; *used = false when the call
// is not in the graph's steady state (the caller runs run_engforce instead)
static int run_engforce_graph(mdff_ctx* h, int itime, bool* used) {
  *used = false;
  if (!step_graph_usable(h, itime)) return MDFF_OK;
  bool fp32 = h->p.precision == MDFF_PREC_MIXED;
  int s;
  if ((s = sr_join(h)) || (s = rs_join(h))) return s;
  if (!h->step_exec || h->step_gen != h->gen || h->step_fp32 != (fp32 ? 1 : 0))
    if ((s = build_step_graph(h, itime, fp32))) return s;
  *used = true;
  h->launches = 0;
  CK(cudaGraphLaunch(h->step_exec, h->st));
  CK(cudaStreamSynchronize(h->st));
  h->launches = h->step_launches;
  if (h->p.lcoulomb && h->lpolar) {
    double rmsd, rmsd0 = h->h_scal[S_CGP];
    int it, nres = 1;
    if (!cg_graph_outcome(h, &rmsd, &it)) {
      // another outer iteration: from the dipoles the graph left, then the
      // back part again on the converged dipoles
      h->call_overlap = h->overlap;
      if ((s = cg_continue(h, fp32, &rmsd, &it, &nres, nullptr, cg_merged(h)))) return s;
      if ((s = cg_epilogue(h)) || (s = ef_back(h, fp32))) return s;
      CK(cudaStreamSynchronize(h->st));
    }
    h->launches += h->cg_body_launches * it + nres;
    cg_stats(h, rmsd0, rmsd, it, nres);
  }
  return ef_status(h);
}

// overflow -> grow the rows and redo the call (the reference STOPs instead,
// tools.f90:337-350)
static int engforce_retry(mdff_ctx* h, int itime) {
  bool used = false;
  int s = run_engforce_graph(h, itime, &used);
  if (!used && !s) s = run_engforce(h, itime);
  h->launches_call += h->launches;
  for (int tries = 0; s == MDFF_ERR_LIST_OVERFLOW && tries < 3; ++tries) {
    int need = h->h_flags[2];
    int cap = (int)(need * 1.25) + 32;
    int e = alloc_list(h, cap);
    if (e) return e;
    k_seti<<<1, 32, 0, h->st>>>(&h->L.flags[1], 0);
    h->have_list = false;
    // the predictors of the failed attempt shifted the ASPC history
    if (h->d_hist_save)
      CK(cudaMemcpyAsync(h->d_hist, h->d_hist_save, sizeof(double4) * MDFF_ASPC_DEPTH * h->natm,
                         cudaMemcpyDeviceToDevice, h->st));
    s = run_engforce(h, itime);
    h->launches_call += h->launches;
  }
  h->have_state = (s == MDFF_OK || s == MDFF_ERR_NOT_CONVERGED);
  return s;
}

// device-timeline span of one API call (events on the handle's stream)
static void call_begin(mdff_ctx* h) {
  h->launches_call = 0;
  cudaEventRecord(h->ev0, h->st);
}
static void call_end(mdff_ctx* h) {
  cudaEventRecord(h->ev1, h->st);
  cudaEventSynchronize(h->ev1);
  float ms = 0;
  cudaEventElapsedTime(&ms, h->ev0, h->ev1);
  h->stats.ms_last = ms;
  h->stats.n_launches = h->launches_call;
}

// host scalars of the last call into *out (ewald.f90:228-246,
// engforce_driver.f90:116-177, non_bonded.f90:1201-1205)
static void fill_scalars(mdff_ctx* h, mdff_result* out) {
  scalars_to_result(h->h_scal, h->p, h->lsr, h->lpolar, h->omega, h->coul_unit, h->press_unit, out);
}

// ---------------------------------------------------------------------------
// saturating FMA loop: 8 independent chains per thread, register resident
template <typename T>
__global__ void k_fma_peak(T* out, int iters, T a, T b) {
  T x0 = (T)threadIdx.x, x1 = x0 + (T)1, x2 = x0 + (T)2, x3 = x0 + (T)3;
  T x4 = x0 + (T)4, x5 = x0 + (T)5, x6 = x0 + (T)6, x7 = x0 + (T)7;
  for (int i = 0; i < iters; ++i) {
    x0 = x0 * a + b; x1 = x1 * a + b; x2 = x2 * a + b; x3 = x3 * a + b;
    x4 = x4 * a + b; x5 = x5 * a + b; x6 = x6 * a + b; x7 = x7 * a + b;
  }
  T s = ((x0 + x1) + (x2 + x3)) + ((x4 + x5) + (x6 + x7));
  if (s == (T)-12345.678) out[blockIdx.x] = s;  // keeps the loop live
}

// ---------------------------------------------------------------------------
// C ABI

extern "C" {

int mdff_gpu_abi_version(void) { return MDFF_ABI_VERSION; }

int mdff_gpu_struct_size(int which) {
  switch (which) {
    case 0: return (int)sizeof(mdff_params);
    case 1: return (int)sizeof(mdff_result);
    case 2: return (int)sizeof(mdff_stats);
    case 3: return (int)sizeof(mdff_batch_desc);
    case 4: return (int)sizeof(mdff_batch_conf);
    default: return -1;
  }
}

const char* mdff_gpu_strerror(int s) {
  switch (s) {
    case MDFF_OK: return "ok";
    case MDFF_ERR_BAD_ARGS: return "invalid argument";
    case MDFF_ERR_CUDA: return "CUDA error";
    case MDFF_ERR_CATASTROPHE: return "polarization catastrophe: a dipole component > 10 eA";
    case MDFF_ERR_LIST_OVERFLOW: return "Verlet list overflow";
    case MDFF_ERR_NOT_CONVERGED: return "induced-dipole solve did not converge";
    case MDFF_ERR_TIMEOUT: return "device wait timed out";
    case MDFF_ERR_NO_DEVICE: return "no usable CUDA device";
    case MDFF_ERR_UNSUPPORTED: return "feature not supported";
    case MDFF_ERR_NOMEM: return "device allocation failed";
    default: return "unknown status";
  }
}

const char* mdff_gpu_last_error(mdff_handle h) { return h ? h->err.c_str() : g_err.c_str(); }

static int create_impl(mdff_ctx* h, const mdff_params* pin, const double* cellA) {
  Setup S;
  const char* serr = nullptr;
  int s0 = setup_system(pin, cellA, S, &serr);
  if (s0) {
    h->err = serr;
    return s0;
  }
  h->p = S.p;
  mdff_params& p = h->p;
  h->natm = p.natm;
  h->ntype = p.ntype;
  int n = p.natm;
  h->coul_unit = S.coul_unit;
  h->press_unit = S.press_unit;
  h->lsr = S.lsr;
  h->task_qq = S.task_qq;
  h->task_qd = S.task_qd;
  h->task_dd = S.task_dd;
  h->lpolar = S.lpolar;
  h->ldip_static = S.ldip_static;
  lattice(h, cellA);
  h->stats.alphaES = p.alphaES;
  for (int i = 0; i < 3; ++i) h->stats.kES[i] = p.kES[i];
  h->stats.cutlongrange = p.cutlongrange;
  // device
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= p.device) {
    h->err = "no CUDA device";
    return MDFF_ERR_NO_DEVICE;
  }
  h->device = p.device;
  CK(cudaSetDevice(h->device));
  CK(cudaDeviceGetAttribute(&h->nsm, cudaDevAttrMultiProcessorCount, h->device));
  // the main chain and the real-space halves at the highest priority; the
  // short-range pass fills the SMs they leave idle
  int prio_lo = 0, prio_hi = 0;
  CK(cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi));
  CK(cudaStreamCreateWithPriority(&h->st, cudaStreamNonBlocking, prio_hi));
  CK(cudaStreamCreateWithPriority(&h->st_rs, cudaStreamNonBlocking, prio_hi));
  CK(cudaStreamCreateWithPriority(&h->st_sr, cudaStreamNonBlocking, prio_lo));
  CK(cudaEventCreateWithFlags(&h->ev_fork, cudaEventDisableTiming));
  CK(cudaEventCreateWithFlags(&h->ev_join_sr, cudaEventDisableTiming));
  CK(cudaEventCreateWithFlags(&h->ev_join_rs, cudaEventDisableTiming));
  {
    const char* ov = std::getenv("MDFF_OVERLAP");
    h->overlap = !(ov && ov[0] == '0');
  }
  CK(cudaEventCreate(&h->ev0));
  CK(cudaEventCreate(&h->ev1));
  h->npol = S.npol;
  DALLOC(h->d_cell, 1);
  DALLOC(h->d_pos, 3 * (size_t)n);
  DALLOC(h->d_s, n);
  DALLOC(h->d_itype, n);
  DALLOC(h->d_ipolar, n);
  DALLOC(h->d_q, n);
  DALLOC(h->d_qzero, n);
  DALLOC(h->d_dipia, n);
  DALLOC(h->d_pol, 9 * (size_t)n);
  DALLOC(h->d_invpol, 9 * (size_t)n);
  CK(cudaMemcpyAsync(h->d_itype, S.itype.data(), sizeof(int) * n, cudaMemcpyHostToDevice, h->st));
  CK(cudaMemcpyAsync(h->d_ipolar, S.ipol.data(), sizeof(int) * n, cudaMemcpyHostToDevice, h->st));
  for (int i = 0; i < n; ++i)
    if (S.ipol[i]) h->polidx.push_back(i);
  if (!h->polidx.empty()) {
    DALLOC(h->d_polidx, h->polidx.size());
    CK(cudaMemcpyAsync(h->d_polidx, h->polidx.data(), sizeof(int) * h->polidx.size(), cudaMemcpyHostToDevice,
                       h->st));
  }
  CK(cudaMemcpyAsync(h->d_q, S.q.data(), sizeof(double) * n, cudaMemcpyHostToDevice, h->st));
  CK(cudaMemcpyAsync(h->d_dipia, S.dip.data(), sizeof(double4) * n, cudaMemcpyHostToDevice, h->st));
  CK(cudaMemcpyAsync(h->d_pol, S.pol.data(), sizeof(double) * 9 * n, cudaMemcpyHostToDevice, h->st));
  CK(cudaMemcpyAsync(h->d_invpol, S.inv.data(), sizeof(double) * 9 * n, cudaMemcpyHostToDevice, h->st));
  const std::vector<NBPair>& nb = S.nb;
  const std::vector<ESPair>& es = S.es;
  DALLOC(h->d_nbtab, nb.size());
  DALLOC(h->d_estab, es.size());
  CK(cudaMemcpyAsync(h->d_nbtab, nb.data(), sizeof(NBPair) * nb.size(), cudaMemcpyHostToDevice, h->st));
  CK(cudaMemcpyAsync(h->d_estab, es.data(), sizeof(ESPair) * es.size(), cudaMemcpyHostToDevice, h->st));
  {
    // a role with c = 0 damps nothing at any order (f = 1, fd = 0 exactly),
    // so only the roles with c != 0 have to share the order
    int k = -1;
    bool same = true;
    for (const ESPair& e : es) {
      if (!e.ldamp) continue;
      const int ord[2] = {e.ka, e.kb};
      const double c[2] = {e.ca, e.cb};
      for (int r = 0; r < 2; ++r) {
        if (c[r] == 0.0) continue;
        if (k < 0) k = ord[r];
        same = same && ord[r] == k;
      }
    }
    h->tt_k = (same && k == 4) ? 4 : 0;  // the instantiated order (examples use 4)
  }
  // list
  double cut = 0.0;
  if (h->lsr) cut = std::max(cut, p.cutshortrange);
  if (p.lcoulomb) cut = std::max(cut, p.cutlongrange);
  h->rskin_build = cut + p.skindiff;
  h->L.rskinsq = h->rskin_build * h->rskin_build;
  h->L.skindiff = p.skindiff;
  DALLOC(h->L.nnb, n);
  DALLOC(h->L.flags, 4);
  DALLOC(h->L.sref, n);
  DALLOC(h->L.cell_of, n);
  DALLOC(h->L.cell_atoms, n);
  DALLOC(h->d_disp_part, cdiv(n, 256));
  CK(cudaMallocHost((void**)&h->h_flags, sizeof(int) * 4));
  lattice(h, cellA);
  double dens = n / h->omega;
  double est = 4.0 / 3.0 * kPi * h->rskin_build * h->rskin_build * h->rskin_build * dens * 1.4 + 64;
  int cap = (int)std::min<double>(est, (double)n + 32);
  int s;
  if ((s = alloc_list(h, std::max(cap, 32)))) return s;
  if ((s = setup_list_cells(h))) return s;
  if ((s = upload_cell(h))) return s;
  // reciprocal mesh and tables
  if (p.lcoulomb) {
    if ((s = build_mesh(h))) return s;
    int ntab = p.kES[0] + 1 + p.kES[1] + 1 + std::max(p.kES[2], 4) + 1;
    DALLOC(h->d_tab64, (size_t)ntab * n);
    if (p.precision == MDFF_PREC_MIXED) DALLOC(h->d_tab32, (size_t)ntab * n);
    DALLOC(h->d_w, n);
    DALLOC(h->d_w32, (size_t)cdiv(n, kRhoTcKB) * kRhoTcKB);  // whole K blocks, zero past the ions
  }
  // pim and outputs
  DALLOC(h->d_Estat, n);
  DALLOC(h->d_Eind, n);
  DALLOC(h->d_Efield, n);
  DALLOC(h->d_mu_ind, n);
  DALLOC(h->d_mu_tot, n);
  DALLOC(h->d_hist, (size_t)MDFF_ASPC_DEPTH * n);
  if (h->lpolar) DALLOC(h->d_hist_save, (size_t)MDFF_ASPC_DEPTH * n);
  DALLOC(h->d_E, n);
  DALLOC(h->d_r, n);
  DALLOC(h->d_z, n);
  DALLOC(h->d_pv, n);
  DALLOC(h->d_qv, n);
  DALLOC(h->d_Tp, n);
  DALLOC(h->d_mu32, n);
  if (p.precision == MDFF_PREC_MIXED && p.lcoulomb) DALLOC(h->d_qm32, n);
  if (p.algo_moment_from_pola != MDFF_ALGO_SCF) {
    DALLOC(h->d_ko_f, n);
    DALLOC(h->d_ko_dmu, n);
    DALLOC(h->d_ko_g, n);
    DALLOC(h->d_ko_muprev, n);
    DALLOC(h->d_ko_fdir, n);
    DALLOC(h->d_ko_x, kKoHist + 2);
    CK(cudaMallocHost((void**)&h->h_ko, sizeof(double) * (kKoHist + 2)));
    if (p.algo_moment_from_pola == MDFF_ALGO_KO_V4_1) {
      DALLOC(h->d_Fh, (size_t)kKoHist * n);
      DALLOC(h->d_muh, (size_t)kKoHist * n);
    }
  }
  DALLOC(h->d_force, 3 * (size_t)n);
  if (h->lsr) DALLOC(h->d_fsr, 3 * (size_t)n);
  DALLOC(h->d_pack, 3 * (size_t)n);
  h->part_cap = (size_t)std::max(cdiv((long)n * 32, 256), cdiv(n, 256)) * 16 + 64;
  // kO_v4_1 Gram row: kKoHist + 2 dot products per block
  h->part_cap = std::max(h->part_cap, (size_t)cdiv(n, 256) * (kKoHist + 2));
  DALLOC(h->d_part, h->part_cap);
  DALLOC(h->d_part2, h->part_cap);
  DALLOC(h->d_scal, S_NSCAL);
  DALLOC(h->d_cata, 4);  // [0] catastrophe, [1] a tensor-core wait gave up, [2] Wannier count
  k_seti<<<1, 32, 0, h->st>>>(h->d_cata + 3, -1);  // [3] default operand-wait limit
  LAUNCH_CHECK();
  for (int it = 0; it < p.ntype; ++it)
    if (p.lwfc[it] > 0) h->lwannier = true;
  if (h->lwannier) {
    DALLOC(h->d_lwfc, NT);
    DALLOC(h->d_mu_wfc, n);
    CK(cudaMemcpyAsync(h->d_lwfc, p.lwfc, sizeof(int) * NT, cudaMemcpyHostToDevice, h->st));
    if (p.rcut_wfc >= h->L.rskinsq) {
      h->err = "rcut_wfc (a squared distance) must be below the squared list cutoff";
      return MDFF_ERR_BAD_ARGS;
    }
  }
  DALLOC(h->d_ekin_part, cdiv(n, 256));
  CK(cudaMallocHost((void**)&h->h_scal, sizeof(double) * S_NSCAL));
  CK(cudaMallocHost((void**)&h->h_cata, 3 * sizeof(int)));
  CK(cudaStreamSynchronize(h->st));
  return MDFF_OK;
}

int mdff_gpu_create(const mdff_params* p, const double cell_A[9], mdff_handle* out) {
  if (!p || !cell_A || !out) return MDFF_ERR_BAD_ARGS;
  *out = nullptr;
  mdff_ctx* h = new mdff_ctx();
  int s = create_impl(h, p, cell_A);
  if (s != MDFF_OK) {
    g_err = h->err;
    mdff_gpu_destroy(h);
    return s;
  }
  *out = h;
  return MDFF_OK;
}

int mdff_gpu_set_cell(mdff_handle h, const double cell_A[9]) {
  if (!h || !cell_A) return MDFF_ERR_BAD_ARGS;
  CK(cudaSetDevice(h->device));
  lattice(h, cell_A);
  int s;
  if ((s = setup_list_cells(h))) return s;
  if ((s = upload_cell(h))) return s;
  if (h->p.lcoulomb && (s = build_mesh(h))) return s;
  h->have_list = false;
  h->md_valid = false;
  return MDFF_OK;
}

static int outputs_to_host(mdff_ctx* h, mdff_result* out) {
  int n = h->natm;
  CK(cudaMemcpyAsync(out->fx, h->d_force, sizeof(double) * n, cudaMemcpyDeviceToHost, h->st));
  CK(cudaMemcpyAsync(out->fy, h->d_force + n, sizeof(double) * n, cudaMemcpyDeviceToHost, h->st));
  CK(cudaMemcpyAsync(out->fz, h->d_force + 2 * (size_t)n, sizeof(double) * n, cudaMemcpyDeviceToHost, h->st));
  if (out->mu) {
    k_pack3<<<cdiv(n, 256), 256, 0, h->st>>>(h->d_mu_tot, n, h->d_pack);
    LAUNCH_CHECK();
    CK(cudaMemcpyAsync(out->mu, h->d_pack, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, h->st));
  }
  if (out->ef) {
    // the pack buffer is reused: wait for the dipole copy
    CK(cudaStreamSynchronize(h->st));
    k_pack3<<<cdiv(n, 256), 256, 0, h->st>>>(h->d_E, n, h->d_pack);
    LAUNCH_CHECK();
    CK(cudaMemcpyAsync(out->ef, h->d_pack, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, h->st));
  }
  CK(cudaStreamSynchronize(h->st));
  return MDFF_OK;
}

int mdff_gpu_engforce(mdff_handle h, const double* rx, const double* ry, const double* rz,
                      int itime, mdff_result* out) {
  if (!h || !rx || !ry || !rz || !out || !out->fx || !out->fy || !out->fz) return MDFF_ERR_BAD_ARGS;
  CK(cudaSetDevice(h->device));
  int n = h->natm;
  h->md_valid = false;
  call_begin(h);
  CK(cudaMemcpyAsync(h->d_pos, rx, sizeof(double) * n, cudaMemcpyHostToDevice, h->st));
  CK(cudaMemcpyAsync(h->d_pos + n, ry, sizeof(double) * n, cudaMemcpyHostToDevice, h->st));
  CK(cudaMemcpyAsync(h->d_pos + 2 * (size_t)n, rz, sizeof(double) * n, cudaMemcpyHostToDevice, h->st));
  int s = engforce_retry(h, itime);
  if (s != MDFF_OK && s != MDFF_ERR_CATASTROPHE && s != MDFF_ERR_NOT_CONVERGED) return s;
  fill_scalars(h, out);
  int s2 = outputs_to_host(h, out);
  call_end(h);
  return s2 ? s2 : s;
}

int mdff_gpu_engforce_device(mdff_handle h, const double* d_pos, int itime, double* d_force,
                             double* d_mu, double* d_ef, mdff_result* out) {
  if (!h || !d_pos || !d_force || !out) return MDFF_ERR_BAD_ARGS;
  CK(cudaSetDevice(h->device));
  int n = h->natm;
  h->md_valid = false;
  call_begin(h);
  if (d_pos != h->d_pos)
    CK(cudaMemcpyAsync(h->d_pos, d_pos, sizeof(double) * 3 * n, cudaMemcpyDeviceToDevice, h->st));
  int s = engforce_retry(h, itime);
  if (s != MDFF_OK && s != MDFF_ERR_CATASTROPHE && s != MDFF_ERR_NOT_CONVERGED) return s;
  fill_scalars(h, out);
  if (d_force != h->d_force)
    CK(cudaMemcpyAsync(d_force, h->d_force, sizeof(double) * 3 * n, cudaMemcpyDeviceToDevice, h->st));
  if (d_mu) {
    k_pack3<<<cdiv(n, 256), 256, 0, h->st>>>(h->d_mu_tot, n, d_mu);
    LAUNCH_CHECK();
  }
  if (d_ef) {
    k_pack3<<<cdiv(n, 256), 256, 0, h->st>>>(h->d_E, n, d_ef);
    LAUNCH_CHECK();
  }
  call_end(h);
  return s;
}

int mdff_gpu_get_aspc_history(mdff_handle h, double* buf) {
  if (!h || !buf) return MDFF_ERR_BAD_ARGS;
  CK(cudaSetDevice(h->device));
  int n = h->natm;
  for (int k = 0; k < MDFF_ASPC_DEPTH; ++k) {
    k_pack3<<<cdiv(n, 256), 256, 0, h->st>>>(h->d_hist + (size_t)k * n, n, h->d_pack);
    LAUNCH_CHECK();
    CK(cudaMemcpyAsync(buf + (size_t)k * 3 * n, h->d_pack, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, h->st));
    CK(cudaStreamSynchronize(h->st));
  }
  return MDFF_OK;
}

int mdff_gpu_set_aspc_history(mdff_handle h, const double* buf) {
  if (!h || !buf) return MDFF_ERR_BAD_ARGS;
  CK(cudaSetDevice(h->device));
  h->md_valid = false;
  int n = h->natm;
  for (int k = 0; k < MDFF_ASPC_DEPTH; ++k) {
    CK(cudaMemcpyAsync(h->d_pack, buf + (size_t)k * 3 * n, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, h->st));
    k_unpack3<<<cdiv(n, 256), 256, 0, h->st>>>(h->d_pack, n, h->d_hist + (size_t)k * n);
    LAUNCH_CHECK();
    CK(cudaStreamSynchronize(h->st));
  }
  return MDFF_OK;
}

int mdff_gpu_kardir_roundtrips(mdff_handle h, double* rx, double* ry, double* rz, int count) {
  if (!h || !rx || !ry || !rz || count < 0) return MDFF_ERR_BAD_ARGS;
  if (count > kMaxRoundTrips) {
    h->err = "mdff_gpu_kardir_roundtrips: count above " + std::to_string(kMaxRoundTrips);
    return MDFF_ERR_BAD_ARGS;
  }
  CK(cudaSetDevice(h->device));
  const int n = h->natm;
  if (n == 0 || count == 0) return MDFF_OK;
  if (!h->d_rtpos) DALLOC(h->d_rtpos, 3 * (size_t)n);
  double* host[3] = {rx, ry, rz};
  for (int a = 0; a < 3; ++a)
    CK(cudaMemcpyAsync(h->d_rtpos + (size_t)a * n, host[a], sizeof(double) * n,
                       cudaMemcpyHostToDevice, h->st));
  k_kardir_roundtrips<<<cdiv(n, 256), 256, 0, h->st>>>(h->d_rtpos, n, h->d_cell, count);
  LAUNCH_CHECK();
  for (int a = 0; a < 3; ++a)
    CK(cudaMemcpyAsync(host[a], h->d_rtpos + (size_t)a * n, sizeof(double) * n,
                       cudaMemcpyDeviceToHost, h->st));
  CK(cudaStreamSynchronize(h->st));
  return MDFF_OK;
}

int mdff_gpu_get_stats(mdff_handle h, mdff_stats* s) {
  if (!h || !s) return MDFF_ERR_BAD_ARGS;
  *s = h->stats;
  return MDFF_OK;
}

int mdff_gpu_verlet_half_list(mdff_handle h, int which, const double* rx, const double* ry,
                              const double* rz, int* point, int* list, int capacity, int* n_out) {
  if (!h || !rx || !ry || !rz || !point || !n_out || (which != 0 && which != 1)) return MDFF_ERR_BAD_ARGS;
  CK(cudaSetDevice(h->device));
  int n = h->natm, s;
  h->md_valid = false;
  double cut = which == 0 ? h->p.cutshortrange : h->p.cutlongrange;
  if (cut + h->p.skindiff > h->rskin_build + 1e-12) return MDFF_ERR_UNSUPPORTED;
  CK(cudaMemcpyAsync(h->d_pos, rx, sizeof(double) * n, cudaMemcpyHostToDevice, h->st));
  CK(cudaMemcpyAsync(h->d_pos + n, ry, sizeof(double) * n, cudaMemcpyHostToDevice, h->st));
  CK(cudaMemcpyAsync(h->d_pos + 2 * (size_t)n, rz, sizeof(double) * n, cudaMemcpyHostToDevice, h->st));
  for (int tries = 0; tries < 4; ++tries) {
    h->launches = 0;
    k_kardir<<<cdiv(n, 256), 256, 0, h->st>>>(h->d_pos, n, h->d_cell, h->d_itype, h->d_ipolar, h->d_q,
                                                h->d_s);
    LAUNCH_CHECK();
    h->have_list = false;
    if ((s = list_update(h))) return s;
    CK(cudaMemcpyAsync(h->h_flags, h->L.flags, sizeof(int) * 4, cudaMemcpyDeviceToHost, h->st));
    CK(cudaStreamSynchronize(h->st));
    if (!h->h_flags[1]) break;
    if ((s = alloc_list(h, (int)(h->h_flags[2] * 1.25) + 32))) return s;
    k_seti<<<1, 32, 0, h->st>>>(&h->L.flags[1], 0);
  }
  if (h->h_flags[1]) return MDFF_ERR_LIST_OVERFLOW;
  int* d_out = nullptr;
  int* d_cnt = nullptr;
  DALLOC(d_out, (size_t)n * h->L.cap);
  DALLOC(d_cnt, n);
  double rs = cut + h->p.skindiff;
  k_export_half<<<cdiv((long)n * 32, 256), 256, 0, h->st>>>(h->d_s, n, h->d_cell, h->L, rs * rs, d_out, d_cnt);
  LAUNCH_CHECK();
  std::vector<int> cnt(n), rows((size_t)n * h->L.cap);
  CK(cudaMemcpyAsync(cnt.data(), d_cnt, sizeof(int) * n, cudaMemcpyDeviceToHost, h->st));
  CK(cudaMemcpyAsync(rows.data(), d_out, sizeof(int) * (size_t)n * h->L.cap, cudaMemcpyDeviceToHost, h->st));
  CK(cudaStreamSynchronize(h->st));
  cudaFree(d_out);
  cudaFree(d_cnt);
  int icount = 1, status = MDFF_OK;
  for (int i = 0; i < n; ++i) {
    point[i] = icount;
    for (int k = 0; k < cnt[i]; ++k) {
      if (icount - 1 < capacity && list) list[icount - 1] = rows[(size_t)i * h->L.cap + k] + 1;
      else status = MDFF_ERR_LIST_OVERFLOW;
      icount++;
    }
  }
  point[n] = icount;
  *n_out = icount - 1;
  return status;
}

int mdff_gpu_md_nve(mdff_handle h, double* d_pos, double* d_vel, const double* d_invmass, double dt,
                    int nsteps, int itime0, double* ekin_pot) {
  if (!h || !d_pos || !d_vel || !d_invmass || nsteps < 0) return MDFF_ERR_BAD_ARGS;
  CK(cudaSetDevice(h->device));
  int n = h->natm, s;
  mdff_result r{};
  call_begin(h);
  CK(cudaMemcpyAsync(h->d_pos, d_pos, sizeof(double) * 3 * n, cudaMemcpyDeviceToDevice, h->st));
  // forces at t0, unless the last call of this driver left them for d_pos
  if (!(h->md_valid && h->md_pos == d_pos)) {
    s = engforce_retry(h, itime0);
    if (s) return s;
  }
  h->md_valid = false;
  for (int step = 0; step < nsteps; ++step) {
    PDL_CHECK(pdl_launch(k_vv_kick_drift, dim3(cdiv(n, 256)), dim3(256), 0, h->st, h->d_pos, d_vel, h->d_force, d_invmass, n, dt));
    s = engforce_retry(h, itime0 + step + 1);
    if (s) return s;
    int nb = cdiv(n, 256);
    PDL_CHECK(pdl_launch(k_vv_kick, dim3(nb), dim3(256), 0, h->st, d_vel, h->d_force, d_invmass, n, dt, h->d_ekin_part));
    k_reduce_partials<<<1, 256, 0, h->st>>>(h->d_ekin_part, nb, 1, h->d_scal + S_NSCAL - 1);
    LAUNCH_CHECK();
    h->launches_call += 3;
    if (ekin_pot) {
      fill_scalars(h, &r);
      double ek;
      if ((s = read_scal(h, S_NSCAL - 1, &ek))) return s;
      ekin_pot[2 * step] = ek;
      ekin_pot[2 * step + 1] = r.u_lj + r.u_bmhft + r.u_coul;
    }
  }
  CK(cudaMemcpyAsync(d_pos, h->d_pos, sizeof(double) * 3 * n, cudaMemcpyDeviceToDevice, h->st));
  call_end(h);
  h->md_valid = true;
  h->md_pos = d_pos;
  return MDFF_OK;
}

// efg = (efg + diag(-2 selfa2 q_i)) * coul_unit  (ewald.f90 self term of the gradient)
__global__ void k_efg_finish(const double* __restrict__ q, int natm, double selfa2, double cu,
                             double* __restrict__ efg) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= natm) return;
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) {
      double s = (a == b) ? -2.0 * selfa2 * q[i] : 0.0;
      efg[9 * (size_t)i + 3 * a + b] = (efg[9 * (size_t)i + 3 * a + b] + s) * cu;
    }
}

int mdff_gpu_efg(mdff_handle h, double* efg) {
  if (!h || !efg) return MDFF_ERR_BAD_ARGS;
  if (!h->p.lcoulomb || !h->have_state) {
    h->err = "efg needs lcoulomb and a completed engforce call";
    return MDFF_ERR_BAD_ARGS;
  }
  CK(cudaSetDevice(h->device));
  int n = h->natm;
  if (!h->d_efg) DALLOC(h->d_efg, 9 * (size_t)n);
  double cutsq = h->p.cutlongrange * h->p.cutlongrange;
  k_es_efg<<<cdiv((long)n * 32, 256), 256, 0, h->st>>>(h->d_s, h->d_q, h->d_mu_tot, h->L.nbr, h->L.nnb, h->L.cap, n, h->d_cell, h->p.alphaES, cutsq, h->task_qq, h->task_dd, h->d_efg);
  LAUNCH_CHECK();
  if (h->nk > 0) {
    // FP64 structure factor of the final charges and dipoles
    RecMesh M;
    M.kmax[0] = h->p.kES[0];
    M.kmax[1] = h->p.kES[1];
    M.kmax[2] = h->p.kES[2];
    M.nrows = (int)h->rows.size();
    M.rows = h->d_rows;
    M.nk = h->nk;
    M.Ak = h->d_Ak;
    M.kvec = h->d_kvec;
    int has_q = h->task_qq ? 1 : 0, has_mu = (h->task_qd || h->task_dd) ? 1 : 0;
    k_rec_weights<<<cdiv(n, 256), 256, 0, h->st>>>(h->d_q, h->d_mu_tot, n, h->d_cell, has_q, has_mu, h->d_w, nullptr, nullptr);
    LAUNCH_CHECK();
    int nzt = pick_nzt(2 * M.kmax[2] + 1);
    int ntiles = cdiv(2 * M.kmax[2] + 1, nzt);
    dim3 gr((unsigned)(M.nrows * ntiles), (unsigned)h->n_rho_chunks);
    switch (nzt) {
      case 8: launch_rho<double, 8>(h, gr, h->d_tab64, n, kRhoChunk, M, ntiles, has_q, has_mu); break;
      case 11: launch_rho<double, 11>(h, gr, h->d_tab64, n, kRhoChunk, M, ntiles, has_q, has_mu); break;
      case 13: launch_rho<double, 13>(h, gr, h->d_tab64, n, kRhoChunk, M, ntiles, has_q, has_mu); break;
      case 21: launch_rho<double, 21>(h, gr, h->d_tab64, n, kRhoChunk, M, ntiles, has_q, has_mu); break;
      case 25: launch_rho<double, 25>(h, gr, h->d_tab64, n, kRhoChunk, M, ntiles, has_q, has_mu); break;
      default: launch_rho<double, 16>(h, gr, h->d_tab64, n, kRhoChunk, M, ntiles, has_q, has_mu); break;
    }
    LAUNCH_CHECK();
    k_rec_sum<<<cdiv(h->nk, 256), 256, 0, h->st>>>(h->d_rho_part, h->n_rho_chunks, M, h->d_rhoA, h->d_str);
    LAUNCH_CHECK();
    double fpi_V = 2.0 * (kTwoPi / h->omega);
    k_rec_efg<<<cdiv(n, 128), 128, 0, h->st>>>(h->d_tab64, n, M, h->d_rhoA, h->d_cell, 2.0 * fpi_V, h->d_efg);
    LAUNCH_CHECK();
  }
  double a = h->p.alphaES;
  double selfa2 = 2.0 * (a / std::sqrt(kPi)) * a * a / 3.0;
  k_efg_finish<<<cdiv(n, 256), 256, 0, h->st>>>(h->d_q, n, selfa2, h->coul_unit, h->d_efg);
  LAUNCH_CHECK();
  CK(cudaMemcpyAsync(efg, h->d_efg, sizeof(double) * 9 * n, cudaMemcpyDeviceToHost, h->st));
  CK(cudaStreamSynchronize(h->st));
  return MDFF_OK;
}

int mdff_gpu_profile(mdff_handle h, int enable) {
  if (!h) return MDFF_ERR_BAD_ARGS;
  h->prof = enable != 0;
  h->pool_used = 0;
  for (int c = 0; c < MDFF_NKCLASS; ++c) {
    h->kms[c] = 0;
    h->kl[c] = 0;
    h->kwork[c] = 0;
  }
  return MDFF_OK;
}

int mdff_gpu_set_tc_wait_limit(mdff_handle h, int polls) {
  if (!h) return MDFF_ERR_BAD_ARGS;
  CK(cudaSetDevice(h->device));
  k_seti<<<1, 32, 0, h->st>>>(h->d_cata + 3, polls < 0 ? -1 : polls);
  LAUNCH_CHECK();
  CK(cudaStreamSynchronize(h->st));
  return MDFF_OK;
}

int mdff_gpu_kernel_times(mdff_handle h, double* ms, long long* launches, double* work) {
  if (!h) return MDFF_ERR_BAD_ARGS;
  for (int c = 0; c < MDFF_NKCLASS; ++c) {
    if (ms) ms[c] = h->kms[c];
    if (launches) launches[c] = h->kl[c];
    if (work) work[c] = h->kwork[c];
  }
  return MDFF_OK;
}

int mdff_gpu_peak_flops(int device, int fp64, double* tflops) {
  if (!tflops) return MDFF_ERR_BAD_ARGS;
  if (cudaSetDevice(device) != cudaSuccess) return MDFF_ERR_NO_DEVICE;
  int nsm = 0;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
  int blocks = nsm * 8, threads = 256, iters = 1 << 14;
  void* out = nullptr;
  if (cudaMalloc(&out, sizeof(double) * blocks) != cudaSuccess) return MDFF_ERR_NOMEM;
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  float best = 1e30f;
  for (int rep = 0; rep < 4; ++rep) {
    cudaEventRecord(a);
    if (fp64)
      k_fma_peak<double><<<blocks, threads>>>((double*)out, iters, 0.999999, 1e-7);
    else
      k_fma_peak<float><<<blocks, threads>>>((float*)out, iters, 0.999999f, 1e-7f);
    cudaEventRecord(b);
    cudaEventSynchronize(b);
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    if (rep > 0) best = std::min(best, ms);
  }
  cudaError_t e = cudaGetLastError();
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaFree(out);
  if (e != cudaSuccess) return MDFF_ERR_CUDA;
  double flops = 2.0 * 8.0 * iters * (double)blocks * threads;
  *tflops = flops / (best * 1e-3) / 1e12;
  return MDFF_OK;
}

void mdff_gpu_destroy(mdff_handle h) {
  if (!h) return;
  for (auto& r : h->pool) {
    cudaEventDestroy(r.a);
    cudaEventDestroy(r.b);
  }
  cudaSetDevice(h->device);
  // side-stream work of a call that returned early may still run
  if (h->st_sr) cudaStreamSynchronize(h->st_sr);
  if (h->st_rs) cudaStreamSynchronize(h->st_rs);
  if (h->st) cudaStreamSynchronize(h->st);
  void* ptrs[] = {h->d_cell, h->d_pos, h->d_s, h->d_itype, h->d_ipolar, h->d_q, h->d_qzero,
                  h->d_dipia, h->d_pol, h->d_invpol, h->d_nbtab, h->d_estab, h->L.nbr, h->L.nnb,
                  h->L.flags, h->L.sref, h->L.cell_of, h->L.cell_count, h->L.cell_start,
                  h->L.cell_fill, h->L.cell_atoms, h->d_disp_part, h->d_rows, h->d_Ak, h->d_kvec,
                  h->d_rchunk, h->d_tab64, h->d_tab32, h->d_w, h->d_w32, h->d_rho_part, h->d_rhoA, h->d_str,
                  h->d_G, h->d_H, h->d_Estat, h->d_Eind, h->d_Efield, h->d_mu_ind, h->d_mu_tot,
                  h->d_hist, h->d_E, h->d_r, h->d_z, h->d_pv, h->d_qv, h->d_Tp, h->d_mu32, h->d_force,
                  h->d_part, h->d_scal, h->d_cata, h->d_pack, h->d_ekin_part, h->d_ddr,
                  h->d_ddb1, h->d_ddj, h->d_ddn, h->d_efg, h->d_fb, h->d_ko_f, h->d_ko_dmu,
                  h->d_ko_g, h->d_ko_muprev, h->d_ko_fdir, h->d_Fh, h->d_muh, h->d_ko_x, h->d_part2,
                  h->d_lwfc, h->d_mu_wfc, h->d_qm32, h->d_Edd, h->d_fsr, h->d_hist_save,
                  h->d_rho_timg, h->d_polidx, h->d_rho_acc, h->d_w32s, h->d_polslot,
                  h->d_rtpos};
  for (void* q : ptrs)
    if (q) cudaFree(q);
  step_graph_free(h);
  if (h->cg_exec) cudaGraphExecDestroy(h->cg_exec);
  if (h->cg_graph) cudaGraphDestroy(h->cg_graph);
  if (h->h_scal) cudaFreeHost(h->h_scal);
  if (h->h_flags) cudaFreeHost(h->h_flags);
  if (h->h_cata) cudaFreeHost(h->h_cata);
  if (h->h_ko) cudaFreeHost(h->h_ko);
  if (h->ev_fork) cudaEventDestroy(h->ev_fork);
  if (h->ev_join_sr) cudaEventDestroy(h->ev_join_sr);
  if (h->ev_join_rs) cudaEventDestroy(h->ev_join_rs);
  if (h->st_sr) cudaStreamDestroy(h->st_sr);
  if (h->st_rs) cudaStreamDestroy(h->st_rs);
  if (h->ev0) cudaEventDestroy(h->ev0);
  if (h->ev1) cudaEventDestroy(h->ev1);
  if (h->st) cudaStreamDestroy(h->st);
  delete h;
}

}  // extern "C"
