// nlist.cuh -- Verlet neighbour list on the device.
//
// Replaces vnlist_pbc (tools.f90:273-368) and vnlistcheck (tools.f90:444-537).
// The reference builds two half lists by an O(N^2) scan with a parity mask;
// here a cell list in direct (fractional) coordinates enumerates candidates,
// every candidate is tested with the reference's exact two-rounding
// arithmetic (r^2 <= (cut+skin)^2), and each row is sorted ascending.  The
// result is the FULL list (both (i,j) and (j,i)); the reference's half list
// is exactly its subset selected by the parity mask (the distance test is
// symmetric bit for bit: s_i - s_j = -(s_j - s_i), nint(-x) = -nint(x)).
#pragma once
#include "common.cuh"

namespace mdff {

struct ListDev {
  int* nbr;        // [natm][cap] sorted ascending per row
  int* nnb;        // [natm] entries per row
  int cap;         // row capacity
  int* flags;      // [0] rebuild requested, [1] overflow, [2] max row length, [3] rebuild count
  double4* sref;   // direct coordinates at the last build
  int* cell_of;    // [natm]
  int* cell_count; // [ncell]
  int* cell_start; // [ncell+1]
  int* cell_fill;  // [ncell]
  int* cell_atoms; // [natm]
  int nc[3];       // cells per axis
  double rskinsq;  // build cutoff^2
  double skindiff;
};

// direct coordinates (kardir) of the Cartesian SoA positions
// with the ion's tag (charge, type, polarisable flag) in the fourth word
__global__ void k_kardir(const double* __restrict__ pos, int natm, const CellC* __restrict__ cell,
                         const int* __restrict__ itype, const int* __restrict__ ipolar,
                         const double* __restrict__ q, double4* __restrict__ s) {
  pdl_wait();
  pdl_trigger();
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= natm) return;
  double sx, sy, sz;
  kardir_exact(cell->B, pos[i], pos[natm + i], pos[2 * natm + i], sx, sy, sz);
  s[i] = make_double4(sx, sy, sz, ion_tag((float)q[i], itype[i], ipolar[i]));
}

// vnlistcheck: largest and second largest displacement since the last build
// (minimum image); one partial (max1, max2) per block.
__global__ void k_disp_partial(const double4* __restrict__ s, const double4* __restrict__ sref,
                               int natm, const CellC* __restrict__ cell, double2* __restrict__ part) {
  pdl_wait();
  pdl_trigger();
  __shared__ double m1s[32], m2s[32];
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  double m1 = 0.0, m2 = 0.0;
  if (i < natm) {
    double rx, ry, rz;
    double d2 = min_image_exact(cell->A, xsub(s[i].x, sref[i].x), xsub(s[i].y, sref[i].y),
                                xsub(s[i].z, sref[i].z), rx, ry, rz);
    m1 = sqrt(d2);
  }
  // warp top-2 merge
  for (int o = 16; o > 0; o >>= 1) {
    double a1 = __shfl_xor_sync(FULL_MASK, m1, o), a2 = __shfl_xor_sync(FULL_MASK, m2, o);
    double n1 = fmax(m1, a1);
    double n2 = fmax(fmin(m1, a1), fmax(m2, a2));
    m1 = n1;
    m2 = n2;
  }
  int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) {
    m1s[w] = m1;
    m2s[w] = m2;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0, b = 0.0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) {
      double n1 = fmax(a, m1s[k]);
      double n2 = fmax(fmin(a, m1s[k]), fmax(b, m2s[k]));
      a = n1;
      b = n2;
    }
    part[blockIdx.x] = make_double2(a, b);
  }
}

// one warp: lanes merge strided block partials, then the warp's top-2 merge
// (the top two of a multiset do not depend on the order of the merges)
__global__ void k_disp_final(const double2* __restrict__ part, int nb, double skindiff,
                             int* __restrict__ flags, double* __restrict__ disp_out) {
  pdl_wait();
  pdl_trigger();
  double a = 0.0, b = 0.0;
  for (int k = threadIdx.x; k < nb; k += 32) {
    double n1 = fmax(a, part[k].x);
    double n2 = fmax(fmin(a, part[k].x), fmax(b, part[k].y));
    a = n1;
    b = n2;
  }
  for (int o = 16; o > 0; o >>= 1) {
    double a1 = __shfl_xor_sync(FULL_MASK, a, o), b1 = __shfl_xor_sync(FULL_MASK, b, o);
    double n1 = fmax(a, a1);
    double n2 = fmax(fmin(a, a1), fmax(b, b1));
    a = n1;
    b = n2;
  }
  if (threadIdx.x != 0) return;
  if (disp_out) disp_out[0] = a + b;
  // tools.f90:513: if ( drneimax + drneimax2 .gt. skindiff ) rebuild
  if (a + b > skindiff) flags[0] = 1;
}

// ---- cell list --------------------------------------------------------------
__device__ __forceinline__ int cell_index(double s, int n) {
  double w = s - floor(s);  // wrap into [0,1)
  int c = (int)(w * (double)n);
  return c < 0 ? 0 : (c >= n ? n - 1 : c);
}

__global__ void k_cell_count(const double4* __restrict__ s, int natm, ListDev L) {
  pdl_wait();
  pdl_trigger();
  if (L.flags[0] == 0) return;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= natm) return;
  int cx = cell_index(s[i].x, L.nc[0]), cy = cell_index(s[i].y, L.nc[1]),
      cz = cell_index(s[i].z, L.nc[2]);
  int c = (cx * L.nc[1] + cy) * L.nc[2] + cz;
  L.cell_of[i] = c;
  atomicAdd(&L.cell_count[c], 1);
}

// single-block exclusive scan of the cell counts
__global__ void k_cell_scan(ListDev L, int ncell) {
  pdl_wait();
  pdl_trigger();
  if (L.flags[0] == 0) return;
  __shared__ int warp_tot[32];
  __shared__ int carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int base = 0; base < ncell; base += blockDim.x) {
    int i = base + threadIdx.x;
    int v = (i < ncell) ? L.cell_count[i] : 0;
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
    if (i < ncell) {
      L.cell_start[i] = off;
      L.cell_fill[i] = 0;
    }
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) carry = off + v;
    __syncthreads();
  }
  if (threadIdx.x == 0) L.cell_start[ncell] = carry;
}

__global__ void k_cell_scatter(int natm, ListDev L) {
  pdl_wait();
  pdl_trigger();
  if (L.flags[0] == 0) return;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= natm) return;
  int c = L.cell_of[i];
  int slot = atomicAdd(&L.cell_fill[c], 1);
  L.cell_atoms[L.cell_start[c] + slot] = i;
}

// one row of the list: warp-cooperative over the 27 (or fewer) neighbour cells
__device__ __forceinline__ void build_row(const double4* __restrict__ s, int i, int lane,
                                          const CellC* __restrict__ cell, ListDev L) {
  double4 si = s[i];
  int ci = L.cell_of[i];
  int cz0 = ci % L.nc[2], cy0 = (ci / L.nc[2]) % L.nc[1], cx0 = ci / (L.nc[2] * L.nc[1]);
  // neighbour-cell offsets per axis: {-1,0,1} when the axis has >= 3 cells,
  // otherwise every cell of that axis once
  int ox[3][3], no[3];
  for (int a = 0; a < 3; ++a) {
    int n = L.nc[a];
    int c0 = a == 0 ? cx0 : (a == 1 ? cy0 : cz0);
    if (n >= 3) {
      no[a] = 3;
      ox[a][0] = (c0 + n - 1) % n;
      ox[a][1] = c0;
      ox[a][2] = (c0 + 1) % n;
    } else {
      no[a] = n;
      for (int k = 0; k < n; ++k) ox[a][k] = k;
    }
  }
  int count = 0;
  int* row = L.nbr + (size_t)i * L.cap;
  for (int a = 0; a < no[0]; ++a)
    for (int b = 0; b < no[1]; ++b)
      for (int c = 0; c < no[2]; ++c) {
        int cc = (ox[0][a] * L.nc[1] + ox[1][b]) * L.nc[2] + ox[2][c];
        int beg = L.cell_start[cc], end = L.cell_start[cc + 1];
        for (int base = beg; base < end; base += 32) {
          int k = base + lane;
          bool take = false;
          int j = -1;
          if (k < end) {
            j = L.cell_atoms[k];
            if (j != i) {
              double4 sj = s[j];
              double rx, ry, rz;
              double r2 = min_image_exact(cell->A, xsub(si.x, sj.x), xsub(si.y, sj.y),
                                          xsub(si.z, sj.z), rx, ry, rz);
              take = (r2 <= L.rskinsq);
            }
          }
          unsigned m = __ballot_sync(FULL_MASK, take);
          if (take) {
            int pos = count + __popc(m & ((1u << lane) - 1u));
            if (pos < L.cap) row[pos] = j;
          }
          count += __popc(m);
        }
      }
  if (lane == 0) {
    L.nnb[i] = count < L.cap ? count : L.cap;
    atomicMax(&L.flags[2], count);
    if (count > L.cap) L.flags[1] = 1;
  }
}

// warp per atom (grid-stride over atoms, so that a launch without a rebuild
// costs a few blocks): enumerate neighbour cells, exact distance test, append.
__global__ void k_build_rows(const double4* __restrict__ s, int natm, const CellC* __restrict__ cell,
                             ListDev L) {
  pdl_wait();
  pdl_trigger();
  if (L.flags[0] == 0) return;
  int lane = threadIdx.x & 31;
  int nwarp = (gridDim.x * blockDim.x) >> 5;
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < natm; i += nwarp)
    build_row(s, i, lane, cell, L);
}

// block per row (grid-stride over rows): bitonic sort of the row into
// ascending j (the reference's row order); P = power of two >= cap, smem P ints.
__global__ void k_sort_rows(ListDev L, int natm) {
  pdl_wait();
  pdl_trigger();
  if (L.flags[0] == 0) return;
  extern __shared__ int sh[];
  for (int i = blockIdx.x; i < natm; i += gridDim.x) {
    int n = L.nnb[i];
    int P = 1;
    while (P < n) P <<= 1;
    int* row = L.nbr + (size_t)i * L.cap;
    for (int k = threadIdx.x; k < P; k += blockDim.x) sh[k] = (k < n) ? row[k] : 0x7fffffff;
    __syncthreads();
    for (int size = 2; size <= P; size <<= 1) {
      for (int stride = size >> 1; stride > 0; stride >>= 1) {
        for (int t = threadIdx.x; t < (P >> 1); t += blockDim.x) {
          int lo = 2 * stride * (t / stride) + (t % stride);
          int hi = lo + stride;
          bool up = ((lo & size) == 0);
          int a = sh[lo], b = sh[hi];
          if ((a > b) == up) {
            sh[lo] = b;
            sh[hi] = a;
          }
        }
        __syncthreads();
      }
    }
    for (int k = threadIdx.x; k < n; k += blockDim.x) row[k] = sh[k];
    __syncthreads();  // sh is reused by the next row
  }
}

// after a build: remember positions for the next check, clear the request
__global__ void k_build_done(const double4* __restrict__ s, int natm, ListDev L) {
  pdl_wait();
  pdl_trigger();
  if (L.flags[0] == 0) return;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < natm) L.sref[i] = s[i];
}

__global__ void k_build_clear(ListDev L, int ncell) {
  pdl_wait();
  pdl_trigger();
  // runs as one block after k_build_done; resets the cell counters
  if (L.flags[0] == 0) return;
  for (int c = threadIdx.x; c < ncell; c += blockDim.x) L.cell_count[c] = 0;
  __syncthreads();
  if (threadIdx.x == 0) {
    L.flags[3] += 1;
    L.flags[0] = 0;
  }
}

// export of the reference's half list at cutoff^2 rs2: warp per row, keeps
// the masked entries with r^2 <= rs2 in ascending order.
__global__ void k_export_half(const double4* __restrict__ s, int natm, const CellC* __restrict__ cell,
                              ListDev L, double rs2, int* __restrict__ out, int* __restrict__ cnt) {
  int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  int lane = threadIdx.x & 31;
  if (warp >= natm) return;
  int i = warp;
  const int* row = L.nbr + (size_t)i * L.cap;
  int* o = out + (size_t)i * L.cap;
  int n = L.nnb[i], count = 0;
  double4 si = s[i];
  for (int base = 0; base < n; base += 32) {
    int k = base + lane;
    bool take = false;
    int j = -1;
    if (k < n) {
      j = row[k];
      if (half_mask(i, j)) {
        double4 sj = s[j];
        double rx, ry, rz;
        double r2 = min_image_exact(cell->A, xsub(si.x, sj.x), xsub(si.y, sj.y), xsub(si.z, sj.z),
                                    rx, ry, rz);
        take = (r2 <= rs2);
      }
    }
    unsigned m = __ballot_sync(FULL_MASK, take);
    if (take) o[count + __popc(m & ((1u << lane) - 1u))] = j;
    count += __popc(m);
  }
  if (lane == 0) cnt[i] = count;
}

}  // namespace mdff
