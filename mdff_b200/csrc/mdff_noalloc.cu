// mdff_noalloc.cu -- the reference's half Verlet list, computed without any
// device allocation.
//
// Some callers of this library cannot allocate device memory: a host program
// whose device memory is owned by another runtime's caching pool (a PyTorch
// process, a Fortran code whose GPU memory is reserved up front) may see a
// cudaMalloc fail or fragment that pool, and analysis / restart utilities that
// only need the neighbour list should not create a full engine (which sizes
// every per-step buffer).  For them mdff_gpu_verlet_half_list_noalloc builds
// the same list as mdff_gpu_verlet_half_list with all its scratch memory in one
// file-scope static __device__ array of fixed size (every GPU that loads this
// library holds it until the process exits).  The caller passes host inputs
// and host outputs, exactly as for the existing entry point.
//
// Limits: natm <= kNAMaxAtoms (32768), list entries <= kNAMaxEntries
// (4,194,304), row length <= kNAMaxRow (4096); larger inputs are rejected
// with MDFF_ERR_BAD_ARGS and a message on stderr (MDFF_ERR_LIST_OVERFLOW is
// kept for a caller capacity below the list size, as the existing entry
// point returns it).  All calls share the one array, and each call
// clears what must start at zero; two calls that overlap on the same GPU
// (from two host threads) race on it.  The first call on a device looks up
// the array's device address (cudaGetSymbolAddress, with that device
// current) and caches it.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <vector>

#include "../../include/mdff_gpu.h"
#include "common.cuh"

using namespace mdff;

namespace {

constexpr int kNAMaxAtoms = 32768;
constexpr int kNAMaxCells = 32768;
constexpr int kNAMaxEntries = 4 * 1024 * 1024;
constexpr int kNAMaxRow = 4096;
constexpr int kNAMaxDevices = 64;

constexpr size_t al256(size_t x) { return (x + 255) & ~size_t(255); }
// byte offsets of the regions of the scratch array
constexpr size_t O_POS = 0;
constexpr size_t O_S = al256(O_POS + sizeof(double) * 3 * kNAMaxAtoms);
constexpr size_t O_CELLOF = al256(O_S + sizeof(double4) * kNAMaxAtoms);
constexpr size_t O_CATOMS = al256(O_CELLOF + sizeof(int) * kNAMaxAtoms);
constexpr size_t O_ROWOFF = al256(O_CATOMS + sizeof(int) * kNAMaxAtoms);
constexpr size_t O_CCOUNT = al256(O_ROWOFF + sizeof(int) * (kNAMaxAtoms + 1));
constexpr size_t O_CSTART = al256(O_CCOUNT + sizeof(int) * kNAMaxCells);
constexpr size_t O_CFILL = al256(O_CSTART + sizeof(int) * (kNAMaxCells + 1));
constexpr size_t O_FLAGS = al256(O_CFILL + sizeof(int) * kNAMaxCells);
constexpr size_t O_CELLC = al256(O_FLAGS + sizeof(int) * 4);
constexpr size_t O_LIST = al256(O_CELLC + sizeof(CellC));
constexpr size_t kNAScratchBytes = al256(O_LIST + sizeof(int) * (size_t)kNAMaxEntries);

}  // namespace

// the only device memory this entry point uses (~18.4 MB)
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNAScratchBytes];

namespace {

std::mutex g_na_mutex;
unsigned char* g_na_addr[kNAMaxDevices] = {nullptr};

// device address of g_noalloc_scratch on `dev` (which must be current);
// looked up once per device and cached.
int na_scratch(int dev, unsigned char** out) {
  if (dev < 0 || dev >= kNAMaxDevices) return MDFF_ERR_BAD_ARGS;
  std::lock_guard<std::mutex> lock(g_na_mutex);
  if (!g_na_addr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr) {
      fprintf(stderr, "mdff_gpu_verlet_half_list_noalloc: cudaGetSymbolAddress: %s\n",
              cudaGetErrorString(e));
      return MDFF_ERR_CUDA;
    }
    g_na_addr[dev] = static_cast<unsigned char*>(p);
  }
  *out = g_na_addr[dev];
  return MDFF_OK;
}

__global__ void k_na_zero(int* p, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) p[i] = 0;
}

__global__ void k_na_kardir(const double* __restrict__ pos, int n, const CellC* __restrict__ c,
                            double4* __restrict__ s) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double sx, sy, sz;
  kardir_exact(c->B, pos[i], pos[n + i], pos[2 * n + i], sx, sy, sz);
  s[i] = make_double4(sx, sy, sz, 0.0);
}

__device__ __forceinline__ int na_cell(double s, int n) {
  double w = s - floor(s);
  int c = (int)(w * (double)n);
  return c < 0 ? 0 : (c >= n ? n - 1 : c);
}

__global__ void k_na_cell_count(const double4* __restrict__ s, int n, int nc0, int nc1, int nc2,
                                int* __restrict__ cell_of, int* __restrict__ count) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int c = (na_cell(s[i].x, nc0) * nc1 + na_cell(s[i].y, nc1)) * nc2 + na_cell(s[i].z, nc2);
  cell_of[i] = c;
  atomicAdd(&count[c], 1);
}

// single-block exclusive scan: out[k] = sum_{m<k} in[m], out[n] = total
// (in and out may alias)
__global__ void k_na_scan(const int* in, int n, int* out) {
  __shared__ int warp_tot[32];
  __shared__ int carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int base = 0; base < n; base += blockDim.x) {
    int i = base + threadIdx.x;
    int v = (i < n) ? in[i] : 0;
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int x = v;
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(FULL_MASK, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) warp_tot[w] = x;
    __syncthreads();
    if (w == 0) {
      int t = (lane < (int)(blockDim.x >> 5)) ? warp_tot[lane] : 0;
      for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(FULL_MASK, t, o);
        if (lane >= o) t += y;
      }
      warp_tot[lane] = t;
    }
    __syncthreads();
    int off = carry + (w > 0 ? warp_tot[w - 1] : 0) + x - v;
    __syncthreads();
    if (i < n) out[i] = off;
    if (threadIdx.x == blockDim.x - 1) carry = off + v;
    __syncthreads();
  }
  if (threadIdx.x == 0) out[n] = carry;
}

__global__ void k_na_cell_scatter(int n, const int* __restrict__ cell_of,
                                  const int* __restrict__ start, int* __restrict__ fill,
                                  int* __restrict__ atoms) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int c = cell_of[i];
  atoms[start[c] + atomicAdd(&fill[c], 1)] = i;
}

// neighbour cells of atom i along each axis (all cells when an axis has < 3)
__device__ __forceinline__ void na_axes(int ci, int nc0, int nc1, int nc2, int ox[3][3], int no[3]) {
  int c0[3] = {ci / (nc2 * nc1), (ci / nc2) % nc1, ci % nc2};
  int nc[3] = {nc0, nc1, nc2};
  for (int a = 0; a < 3; ++a) {
    if (nc[a] >= 3) {
      no[a] = 3;
      ox[a][0] = (c0[a] + nc[a] - 1) % nc[a];
      ox[a][1] = c0[a];
      ox[a][2] = (c0[a] + 1) % nc[a];
    } else {
      no[a] = nc[a];
      for (int k = 0; k < nc[a]; ++k) ox[a][k] = k;
    }
  }
}

// warp per atom: number of half-list entries of row i (parity mask of
// tools.f90:318-319, r^2 <= rs2 with the reference's arithmetic)
__global__ void k_na_count_rows(const double4* __restrict__ s, int n, const CellC* __restrict__ c,
                                int nc0, int nc1, int nc2, const int* __restrict__ cell_of,
                                const int* __restrict__ start, const int* __restrict__ atoms,
                                double rs2, int* __restrict__ rowcnt, int* __restrict__ flags) {
  int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  int lane = threadIdx.x & 31;
  if (i >= n) return;
  int ox[3][3], no[3];
  na_axes(cell_of[i], nc0, nc1, nc2, ox, no);
  double4 si = s[i];
  int count = 0;
  for (int a = 0; a < no[0]; ++a)
    for (int b = 0; b < no[1]; ++b)
      for (int d = 0; d < no[2]; ++d) {
        int cc = (ox[0][a] * nc1 + ox[1][b]) * nc2 + ox[2][d];
        for (int k = start[cc] + lane; k < start[cc + 1]; k += 32) {
          int j = atoms[k];
          if (!half_mask(i, j)) continue;
          double4 sj = s[j];
          double rx, ry, rz;
          if (min_image_exact(c->A, xsub(si.x, sj.x), xsub(si.y, sj.y), xsub(si.z, sj.z), rx, ry,
                              rz) <= rs2)
            ++count;
        }
      }
  count = warp_sum(count);
  if (lane == 0) {
    rowcnt[i] = count;
    atomicMax(&flags[0], count);
  }
}

// block per row: gather the row, bitonic sort ascending, write 1-based
__global__ void k_na_fill_rows(const double4* __restrict__ s, int n, const CellC* __restrict__ c,
                               int nc0, int nc1, int nc2, const int* __restrict__ cell_of,
                               const int* __restrict__ start, const int* __restrict__ atoms,
                               double rs2, const int* __restrict__ rowoff, int P,
                               int* __restrict__ list) {
  extern __shared__ int sh[];
  __shared__ int cnt;
  int i = blockIdx.x;
  if (i >= n) return;
  for (int k = threadIdx.x; k < P; k += blockDim.x) sh[k] = 0x7fffffff;
  if (threadIdx.x == 0) cnt = 0;
  __syncthreads();
  int ox[3][3], no[3];
  na_axes(cell_of[i], nc0, nc1, nc2, ox, no);
  double4 si = s[i];
  for (int a = 0; a < no[0]; ++a)
    for (int b = 0; b < no[1]; ++b)
      for (int d = 0; d < no[2]; ++d) {
        int cc = (ox[0][a] * nc1 + ox[1][b]) * nc2 + ox[2][d];
        for (int k = start[cc] + threadIdx.x; k < start[cc + 1]; k += blockDim.x) {
          int j = atoms[k];
          if (!half_mask(i, j)) continue;
          double4 sj = s[j];
          double rx, ry, rz;
          if (min_image_exact(c->A, xsub(si.x, sj.x), xsub(si.y, sj.y), xsub(si.z, sj.z), rx, ry,
                              rz) <= rs2) {
            int slot = atomicAdd(&cnt, 1);
            if (slot < P) sh[slot] = j;
          }
        }
      }
  __syncthreads();
  for (int size = 2; size <= P; size <<= 1)
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      for (int t = threadIdx.x; t < (P >> 1); t += blockDim.x) {
        int lo = 2 * stride * (t / stride) + (t % stride), hi = lo + stride;
        bool up = ((lo & size) == 0);
        int x = sh[lo], y = sh[hi];
        if ((x > y) == up) {
          sh[lo] = y;
          sh[hi] = x;
        }
      }
      __syncthreads();
    }
  int o = rowoff[i], m = rowoff[i + 1] - o;
  for (int k = threadIdx.x; k < m; k += blockDim.x) list[o + k] = sh[k] + 1;
}

// lattice (lattice.f90:60-130): B = reciprocal / omega, face widths
void na_lattice(const double* Ain, CellC* c, double W[3]) {
  double A[3][3], B[3][3];
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) A[a][b] = Ain[3 * a + b];
  const int cyc[3][2] = {{1, 2}, {2, 0}, {0, 1}};
  for (int col = 0; col < 3; ++col) {
    int u = cyc[col][0], v = cyc[col][1];
    B[0][col] = A[1][u] * A[2][v] - A[2][u] * A[1][v];
    B[1][col] = A[2][u] * A[0][v] - A[0][u] * A[2][v];
    B[2][col] = A[0][u] * A[1][v] - A[1][u] * A[0][v];
  }
  double omega = B[0][0] * A[0][0] + B[1][0] * A[1][0] + B[2][0] * A[2][0];
  for (int k = 0; k < 3; ++k)
    W[k] = omega / std::sqrt(B[0][k] * B[0][k] + B[1][k] * B[1][k] + B[2][k] * B[2][k]);
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) {
      c->A[3 * a + b] = A[a][b];
      c->B[3 * a + b] = B[a][b] / omega;
    }
  c->omega = omega;
}

int na_fail(const char* what) {
  fprintf(stderr, "mdff_gpu_verlet_half_list_noalloc: %s\n", what);
  return MDFF_ERR_BAD_ARGS;
}

#define NA_CK(call)                                                                       \
  do {                                                                                    \
    cudaError_t e_ = (call);                                                              \
    if (e_ != cudaSuccess) {                                                              \
      fprintf(stderr, "mdff_gpu_verlet_half_list_noalloc: %s: %s\n", #call,               \
              cudaGetErrorString(e_));                                                    \
      return MDFF_ERR_CUDA;                                                               \
    }                                                                                     \
  } while (0)

}  // namespace

extern "C" int mdff_gpu_verlet_half_list_noalloc(const mdff_params* p, const double cell_A[9],
                                                 int which, const double* rx, const double* ry,
                                                 const double* rz, int* point, int* list,
                                                 int capacity, int* n_out) {
  if (!p || !cell_A || !rx || !ry || !rz || !point || !n_out || (which != 0 && which != 1))
    return MDFF_ERR_BAD_ARGS;
  int n = p->natm;
  if (n <= 0) return na_fail("natm must be positive");
  if (n > kNAMaxAtoms) return na_fail("natm exceeds the static scratch limit of 32768 ions");
  CellC cc;
  double W[3];
  na_lattice(cell_A, &cc, W);
  // the cutoffs of verlet_vdw / verlet_coul (config.f90:129-130), with the
  // half-cell clamp of cutlongrange that coulomb_init applies (coulomb.f90:377-383)
  double cut = p->cutshortrange;
  if (which == 1) {
    cut = p->cutlongrange;
    if (p->lcoulomb) cut = std::min(cut, 0.5 * std::min(W[0], std::min(W[1], W[2])));
  }
  double rs = cut + p->skindiff;
  if (!(rs > 0.0)) return na_fail("cutoff + skindiff must be positive");
  int nc[3];
  for (int a = 0; a < 3; ++a)
    nc[a] = std::max(1, std::min((int)std::floor(W[a] / (rs * (1.0 + 1e-9) + 1e-9)), 1024));
  while ((long)nc[0] * nc[1] * nc[2] > kNAMaxCells) {  // coarser cells stay a superset
    int a = (nc[0] >= nc[1] && nc[0] >= nc[2]) ? 0 : (nc[1] >= nc[2] ? 1 : 2);
    nc[a] = std::max(1, nc[a] - 1);
  }
  int ncell = nc[0] * nc[1] * nc[2];

  NA_CK(cudaSetDevice(p->device));
  unsigned char* base = nullptr;
  int st = na_scratch(p->device, &base);
  if (st) return st;
  double* d_pos = reinterpret_cast<double*>(base + O_POS);
  double4* d_s = reinterpret_cast<double4*>(base + O_S);
  int* d_cell_of = reinterpret_cast<int*>(base + O_CELLOF);
  int* d_atoms = reinterpret_cast<int*>(base + O_CATOMS);
  int* d_rowoff = reinterpret_cast<int*>(base + O_ROWOFF);
  int* d_ccount = reinterpret_cast<int*>(base + O_CCOUNT);
  int* d_cstart = reinterpret_cast<int*>(base + O_CSTART);
  int* d_cfill = reinterpret_cast<int*>(base + O_CFILL);
  int* d_flags = reinterpret_cast<int*>(base + O_FLAGS);
  CellC* d_cell = reinterpret_cast<CellC*>(base + O_CELLC);
  int* d_list = reinterpret_cast<int*>(base + O_LIST);

  NA_CK(cudaMemcpy(d_pos, rx, sizeof(double) * n, cudaMemcpyHostToDevice));
  NA_CK(cudaMemcpy(d_pos + n, ry, sizeof(double) * n, cudaMemcpyHostToDevice));
  NA_CK(cudaMemcpy(d_pos + 2 * (size_t)n, rz, sizeof(double) * n, cudaMemcpyHostToDevice));
  NA_CK(cudaMemcpy(d_cell, &cc, sizeof(CellC), cudaMemcpyHostToDevice));
  // the array keeps the previous call's contents: clear the counters
  k_na_zero<<<64, 256>>>(d_ccount, ncell);
  k_na_zero<<<64, 256>>>(d_cfill, ncell);
  k_na_zero<<<1, 32>>>(d_flags, 4);
  k_na_kardir<<<(n + 255) / 256, 256>>>(d_pos, n, d_cell, d_s);
  k_na_cell_count<<<(n + 255) / 256, 256>>>(d_s, n, nc[0], nc[1], nc[2], d_cell_of, d_ccount);
  k_na_scan<<<1, 1024>>>(d_ccount, ncell, d_cstart);
  k_na_cell_scatter<<<(n + 255) / 256, 256>>>(n, d_cell_of, d_cstart, d_cfill, d_atoms);
  double rs2 = rs * rs;
  k_na_count_rows<<<(int)(((long)n * 32 + 255) / 256), 256>>>(
      d_s, n, d_cell, nc[0], nc[1], nc[2], d_cell_of, d_cstart, d_atoms, rs2, d_rowoff, d_flags);
  k_na_scan<<<1, 1024>>>(d_rowoff, n, d_rowoff);
  NA_CK(cudaGetLastError());
  int total = 0, maxrow = 0;
  NA_CK(cudaMemcpy(&total, d_rowoff + n, sizeof(int), cudaMemcpyDeviceToHost));
  NA_CK(cudaMemcpy(&maxrow, d_flags, sizeof(int), cudaMemcpyDeviceToHost));
  *n_out = total;
  // a list larger than the static array is a hard limit of this entry point,
  // not a short caller capacity: a different status, so that a caller that
  // grows its buffer on MDFF_ERR_LIST_OVERFLOW does not retry for ever
  if (total > kNAMaxEntries) {
    fprintf(stderr,
            "mdff_gpu_verlet_half_list_noalloc: %d list entries exceed the static scratch limit "
            "of %d\n", total, kNAMaxEntries);
    return MDFF_ERR_BAD_ARGS;
  }
  if (maxrow > kNAMaxRow) return na_fail("a row longer than 4096 entries exceeds the sort buffer");
  int P = 1;
  while (P < std::max(maxrow, 1)) P <<= 1;
  k_na_fill_rows<<<n, 128, P * sizeof(int)>>>(d_s, n, d_cell, nc[0], nc[1], nc[2], d_cell_of,
                                              d_cstart, d_atoms, rs2, d_rowoff, P, d_list);
  NA_CK(cudaGetLastError());
  std::vector<int> off(n + 1);
  NA_CK(cudaMemcpy(off.data(), d_rowoff, sizeof(int) * (n + 1), cudaMemcpyDeviceToHost));
  for (int i = 0; i <= n; ++i) point[i] = off[i] + 1;
  int ncopy = std::min(total, capacity);
  if (ncopy > 0 && list)
    NA_CK(cudaMemcpy(list, d_list, sizeof(int) * ncopy, cudaMemcpyDeviceToHost));
  return total > capacity ? MDFF_ERR_LIST_OVERFLOW : MDFF_OK;
}
