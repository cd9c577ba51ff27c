// mv_grid.cu -- uniform grid (neighbour search), prefix sums, face ordering and the
// cell -> face CSR.
//
// Replaces RTree::bulk_load (rtree_nn.rs:6-8) with a device counting sort of the
// generators into a row-major uniform grid (SoA positions, coalesced for the shell
// gather of the cell kernel), and the serial flatten + Voronoi::finalize
// (voronoi.rs:226, 241-263) with scans and scatters.
#include <algorithm>
#include <cstdint>

#include <cub/device/device_radix_sort.cuh>

#include "mv_internal.h"

namespace mv {

// ------------------------------------------------------------ preparation --
// Generator::new (generator.rs:13-24): zero the unused coordinates.  Also records the
// extent of the generators and flags non-finite coordinates.
__device__ __forceinline__ unsigned long long ord_key(double v) {
  unsigned long long b = (unsigned long long)__double_as_longlong(v);
  return (b & 0x8000000000000000ull) ? ~b : (b | 0x8000000000000000ull);
}
__device__ __forceinline__ double ord_val(unsigned long long k) {
  unsigned long long b = (k & 0x8000000000000000ull) ? (k & 0x7fffffffffffffffull) : ~k;
  return __longlong_as_double((long long)b);
}

__global__ void prep_kernel(const double* __restrict__ xyz, int n, int dim, double* __restrict__ gen,
                            unsigned long long* ext_keys /* [6]: min x,y,z, -max x,y,z */,
                            int* bad) {
  __shared__ unsigned long long smin[3], smax[3];
  if (threadIdx.x < 3) {
    smin[threadIdx.x] = ~0ull;
    smax[threadIdx.x] = 0ull;
  }
  __syncthreads();
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) {
    double c[3] = {xyz[3 * (int64_t)k], xyz[3 * (int64_t)k + 1], xyz[3 * (int64_t)k + 2]};
    if (dim == 1) c[1] = 0.0, c[2] = 0.0;
    if (dim == 2) c[2] = 0.0;
    bool fin = true;
    for (int i = 0; i < 3; i++) {
      gen[3 * (int64_t)k + i] = c[i];
      fin &= isfinite(c[i]);
    }
    if (!fin) atomicExch(bad, 1);
    for (int i = 0; i < 3; i++) {
      atomicMin(&smin[i], ord_key(c[i]));
      atomicMax(&smax[i], ord_key(c[i]));
    }
  }
  __syncthreads();
  if (threadIdx.x < 3) {
    atomicMin(&ext_keys[threadIdx.x], smin[threadIdx.x]);
    atomicMax(&ext_keys[3 + threadIdx.x], smax[threadIdx.x]);
  }
}

__global__ void ext_finish_kernel(const unsigned long long* ext_keys, double* ext) {
  int i = threadIdx.x;
  if (i < 6) ext[i] = ord_val(ext_keys[i]);
}

struct GridParams {
  int G[3];
  double a[3], inv[3];
  int dim;
};

__global__ void cell_index_kernel(const double* __restrict__ gen, int n, GridParams gp,
                                  int32_t* __restrict__ cid, int32_t* __restrict__ count) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  int c[3];
  for (int i = 0; i < 3; i++) {
    double f = floor((gen[3 * (int64_t)k + i] - gp.a[i]) * gp.inv[i]);
    if (!(f >= 0.0)) f = 0.0;
    if (f > gp.G[i] - 1) f = gp.G[i] - 1;
    c[i] = (int)f;
  }
  int id = c[0] + gp.G[0] * (c[1] + gp.G[1] * c[2]);
  cid[k] = id;
  atomicAdd(count + id, 1);
}

__global__ void scatter_kernel(const double* __restrict__ gen, int n, const int32_t* __restrict__ cid,
                               const int32_t* __restrict__ start, int32_t* __restrict__ fill,
                               double* __restrict__ sx, double* __restrict__ sy,
                               double* __restrict__ sz, int32_t* __restrict__ sid) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  int c = cid[k];
  int pos = start[c] + atomicAdd(fill + c, 1);
  sx[pos] = gen[3 * (int64_t)k];
  sy[pos] = gen[3 * (int64_t)k + 1];
  sz[pos] = gen[3 * (int64_t)k + 2];
  sid[pos] = k;
}

// --------------------------------------------------- dense cells (2nd level) --
// A coarse cell holding more than DENSE_MIN generators is dense: its generators are
// stored sorted by the Morton key of their position inside the cell (fkey_bits(dim) bits
// per active axis).  The cells of every level of the cell's implicit octree are then
// contiguous ranges of sorted positions, found by binary search on the keys, so a
// query scans the cells of the level that matches its radius, whatever the local
// density (Gaussian clumps span many orders of magnitude inside one coarse cell).
// Sparse cells keep key 0 and their generators in input order.
constexpr int DENSE_MIN = 32;

__global__ void dense_flag_kernel(const int32_t* __restrict__ count, int64_t ncell,
                                  int32_t* __restrict__ dflag) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncell) return;
  dflag[c] = count[c] > DENSE_MIN;
}

// sort key of generator k: coarse cell << FKEY_BITS | Morton key inside a dense cell
__global__ void dense_key_kernel(const double* __restrict__ gen, int n, GridParams gp,
                                 const int32_t* __restrict__ cid, const int32_t* __restrict__ dflag,
                                 unsigned long long* __restrict__ key, int32_t* __restrict__ val) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const int c = cid[k];
  uint32_t m = 0;
  if (dflag[c]) {
    const int bits = fkey_bits(gp.dim);
    const int cc[3] = {c % gp.G[0], (c / gp.G[0]) % gp.G[1], c / (gp.G[0] * gp.G[1])};
    uint32_t q[3] = {0u, 0u, 0u};
    for (int i = 0; i < gp.dim; i++) q[i] = fine_q(gen[3 * (int64_t)k + i], gp.a[i], gp.inv[i], cc[i], bits);
    m = morton(gp.dim, q[0], q[1], q[2]);
  }
  key[k] = ((unsigned long long)c << FKEY_BITS) | m;
  val[k] = k;
}

// sorted position s <- generator val[s]; fkey = the Morton part of its sort key
__global__ void dense_gather_kernel(const double* __restrict__ gen, int n,
                                    const unsigned long long* __restrict__ key,
                                    const int32_t* __restrict__ val, double* __restrict__ sx,
                                    double* __restrict__ sy, double* __restrict__ sz,
                                    int32_t* __restrict__ sid, uint32_t* __restrict__ fkey) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const int k = val[s];
  sx[s] = gen[3 * (int64_t)k];
  sy[s] = gen[3 * (int64_t)k + 1];
  sz[s] = gen[3 * (int64_t)k + 2];
  sid[s] = k;
  fkey[s] = (uint32_t)(key[s] & ((1ull << FKEY_BITS) - 1ull));
}

// ------------------------------------------------------------------- scans --
// Exclusive scan of int32 counts into int64 offsets, out[n] = total.
constexpr int SCAN_THREADS = 256;
constexpr int SCAN_ITEMS = 16;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;

__device__ __forceinline__ long long block_excl_scan(long long v, long long* total) {
  __shared__ long long wsum[SCAN_THREADS / 32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  long long x = v;
  for (int o = 1; o < 32; o <<= 1) {
    long long y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) wsum[w] = x;
  __syncthreads();
  if (w == 0) {
    long long s = lane < SCAN_THREADS / 32 ? wsum[lane] : 0;
    for (int o = 1; o < 32; o <<= 1) {
      long long y = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += y;
    }
    if (lane < SCAN_THREADS / 32) wsum[lane] = s;
  }
  __syncthreads();
  long long wpre = w > 0 ? wsum[w - 1] : 0;
  *total = wsum[SCAN_THREADS / 32 - 1];
  __syncthreads();
  return wpre + x - v;
}

template <class In>
__global__ void scan_reduce_kernel(const In* __restrict__ in, int64_t n, long long* __restrict__ sums) {
  int64_t base = (int64_t)blockIdx.x * SCAN_TILE;
  long long s = 0;
  for (int i = 0; i < SCAN_ITEMS; i++) {
    int64_t k = base + (int64_t)i * SCAN_THREADS + threadIdx.x;
    if (k < n) s += (long long)in[k];
  }
  long long tot;
  block_excl_scan(s, &tot);
  if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}

__global__ void scan_sums_kernel(long long* sums, int nb) {
  long long carry = 0;
  for (int base = 0; base < nb; base += SCAN_THREADS) {
    int k = base + threadIdx.x;
    long long v = k < nb ? sums[k] : 0;
    long long tot;
    long long ex = block_excl_scan(v, &tot);
    if (k < nb) sums[k] = carry + ex;
    carry += tot;
  }
}

template <class In, class Out>
__global__ void scan_final_kernel(const In* __restrict__ in, int64_t n, const long long* __restrict__ sums,
                                  Out* __restrict__ out) {
  int64_t base = (int64_t)blockIdx.x * SCAN_TILE;
  // each thread owns SCAN_ITEMS consecutive items
  long long v[SCAN_ITEMS];
  long long s = 0;
  for (int i = 0; i < SCAN_ITEMS; i++) {
    int64_t k = base + (int64_t)threadIdx.x * SCAN_ITEMS + i;
    v[i] = k < n ? (long long)in[k] : 0;
    s += v[i];
  }
  long long tot;
  long long ex = block_excl_scan(s, &tot) + sums[blockIdx.x];
  for (int i = 0; i < SCAN_ITEMS; i++) {
    int64_t k = base + (int64_t)threadIdx.x * SCAN_ITEMS + i;
    if (k < n) out[k] = (Out)ex;
    if (k == n - 1) out[n] = (Out)(ex + v[i]);
    ex += v[i];
  }
}

// --------------------------------------------------------------- faces/CSR --

// staging slot -> final position: faces grouped by left cell in cell order, inside a
// cell in clipping-plane order (flatten!, voronoi.rs:226)
__global__ void reorder_faces_kernel(FaceArrays st, int64_t F, const int64_t* __restrict__ stage_off,
                                     const int64_t* __restrict__ face_off, FaceArrays out) {
  int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= F) return;
  int left = st.left[q];
  int64_t f = face_off[left] + (q - stage_off[left]);
  out.left[f] = left;
  out.right[f] = st.right[q];
  out.area[f] = st.area[q];
  for (int i = 0; i < 3; i++) {
    out.centroid[3 * f + i] = st.centroid[3 * q + i];
    out.normal[3 * f + i] = st.normal[3 * q + i];
  }
  out.code[f] = st.code[q];
}

// faces linked to their right cell (voronoi.rs:248-250: internal, unshifted faces)
__global__ void in_count_kernel(const int32_t* __restrict__ right, const uint8_t* __restrict__ code,
                                int64_t F, int32_t* __restrict__ in_count) {
  int64_t f = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= F) return;
  int r = right[f];
  if (r >= 0 && code[f] == 13) atomicAdd(in_count + r, 1);
}

__global__ void conn_count_kernel(const int32_t* __restrict__ face_count,
                                  const int32_t* __restrict__ in_count, int n,
                                  int32_t* __restrict__ conn_count) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) conn_count[k] = face_count[k] + in_count[k];
}

// A cell's connections are its incoming faces (all from lower-indexed cells, so with
// smaller face indices) followed by its own faces in order.
__global__ void conn_fill_kernel(const int32_t* __restrict__ left, const int32_t* __restrict__ right,
                                 const uint8_t* __restrict__ code, int64_t F,
                                 const int64_t* __restrict__ face_off,
                                 const int64_t* __restrict__ conn_off,
                                 const int32_t* __restrict__ in_count, int32_t* __restrict__ cursor,
                                 int32_t* __restrict__ conn) {
  int64_t f = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= F) return;
  int l = left[f];
  conn[conn_off[l] + in_count[l] + (f - face_off[l])] = (int32_t)f;
  int r = right[f];
  if (r >= 0 && code[f] == 13) {
    int slot = atomicAdd(cursor + r, 1);
    conn[conn_off[r] + slot] = (int32_t)f;
  }
}

__global__ void conn_sort_kernel(const int64_t* __restrict__ conn_off,
                                 const int32_t* __restrict__ in_count, int n,
                                 int32_t* __restrict__ conn) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  int32_t* a = conn + conn_off[k];
  int m = in_count[k];
  for (int i = 1; i < m; i++) {
    int32_t v = a[i];
    int j = i - 1;
    while (j >= 0 && a[j] > v) {
      a[j + 1] = a[j];
      j--;
    }
    a[j + 1] = v;
  }
}

// ------------------------------------------------------------------ batches --
// A batch concatenates its tessellations: tessellation j owns the input indices and
// sorted positions [pos[j], pos[j + 1]) and the grid cells [cbase[j], cbase[j + 1])
// (its own grid plus one empty end cell, so that its cell_start slice ends with its
// own end).  The kernels below find a point's, cell's or face's tessellation by binary
// search over these bases.
__device__ __forceinline__ int batch_find(const int32_t* __restrict__ base, int nj, int64_t v) {
  int a = 0, b = nj - 1;
  while (a < b) {
    const int m = (a + b + 1) >> 1;
    if (base[m] <= v)
      a = m;
    else
      b = m - 1;
  }
  return a;
}

__global__ void batch_ext_init_kernel(unsigned long long* ext_keys, int nj) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < 6 * nj) ext_keys[i] = (i % 6) < 3 ? ~0ull : 0ull;
}

// Generator::new per tessellation (its dimensionality) and each tessellation's extent;
// a warp whose points all belong to one tessellation reduces before its atomics.
__global__ void batch_prep_kernel(const double* __restrict__ xyz, int n, const int32_t* __restrict__ pos,
                                  int nj, const BatchGrid* __restrict__ bg, double* __restrict__ gen,
                                  unsigned long long* ext_keys, int* bad) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int lane = threadIdx.x & 31;
  int j = -1;
  unsigned long long kmin[3] = {~0ull, ~0ull, ~0ull}, kmax[3] = {0ull, 0ull, 0ull};
  if (k < n) {
    j = batch_find(pos, nj, k);
    const int dim = bg[j].dim;
    double c[3] = {xyz[3 * (int64_t)k], xyz[3 * (int64_t)k + 1], xyz[3 * (int64_t)k + 2]};
    if (dim == 1) c[1] = 0.0, c[2] = 0.0;
    if (dim == 2) c[2] = 0.0;
    bool fin = true;
    for (int i = 0; i < 3; i++) {
      gen[3 * (int64_t)k + i] = c[i];
      fin &= isfinite(c[i]);
      kmin[i] = kmax[i] = ord_key(c[i]);
    }
    if (!fin) atomicExch(bad, 1);
  }
  const int j0 = __shfl_sync(0xffffffffu, j, 0);
  if (__all_sync(0xffffffffu, j == j0) && j0 >= 0) {
    for (int o = 16; o > 0; o >>= 1)
      for (int i = 0; i < 3; i++) {
        kmin[i] = min(kmin[i], __shfl_xor_sync(0xffffffffu, kmin[i], o));
        kmax[i] = max(kmax[i], __shfl_xor_sync(0xffffffffu, kmax[i], o));
      }
    if (lane == 0)
      for (int i = 0; i < 3; i++) {
        atomicMin(&ext_keys[6 * j0 + i], kmin[i]);
        atomicMax(&ext_keys[6 * j0 + 3 + i], kmax[i]);
      }
  } else if (j >= 0) {
    for (int i = 0; i < 3; i++) {
      atomicMin(&ext_keys[6 * j + i], kmin[i]);
      atomicMax(&ext_keys[6 * j + 3 + i], kmax[i]);
    }
  }
}

__global__ void batch_ext_finish_kernel(const unsigned long long* ext_keys, double* ext, int nj) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < 6 * nj) ext[i] = ord_val(ext_keys[i]);
}

// grid cell (batch-wide index) of each generator, and the cell counts
__global__ void batch_cell_index_kernel(const double* __restrict__ gen, int n,
                                        const int32_t* __restrict__ pos, int nj,
                                        const BatchGrid* __restrict__ bg, int32_t* __restrict__ cid,
                                        int32_t* __restrict__ count) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const BatchGrid& g = bg[batch_find(pos, nj, k)];
  int c[3];
  for (int i = 0; i < 3; i++) {
    double f = floor((gen[3 * (int64_t)k + i] - g.a[i]) * g.inv[i]);
    if (!(f >= 0.0)) f = 0.0;
    if (f > g.G[i] - 1) f = g.G[i] - 1;
    c[i] = (int)f;
  }
  const int id = g.cbase + c[0] + g.G[0] * (c[1] + g.G[1] * c[2]);
  cid[k] = id;
  atomicAdd(count + id, 1);
}

// sort key: batch cell << FKEY_BITS | Morton key inside a dense cell
__global__ void batch_key_kernel(const double* __restrict__ gen, int n, const int32_t* __restrict__ pos,
                                 int nj, const BatchGrid* __restrict__ bg, const int32_t* __restrict__ cid,
                                 const int32_t* __restrict__ dflag, unsigned long long* __restrict__ key,
                                 int32_t* __restrict__ val) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const int c = cid[k];
  uint32_t m = 0;
  if (dflag[c]) {
    const BatchGrid& g = bg[batch_find(pos, nj, k)];
    const int bits = fkey_bits(g.dim);
    const int lc = c - g.cbase;
    const int cc[3] = {lc % g.G[0], (lc / g.G[0]) % g.G[1], lc / (g.G[0] * g.G[1])};
    uint32_t q[3] = {0u, 0u, 0u};
    for (int i = 0; i < g.dim; i++) q[i] = fine_q(gen[3 * (int64_t)k + i], g.a[i], g.inv[i], cc[i], bits);
    m = morton(g.dim, q[0], q[1], q[2]);
  }
  key[k] = ((unsigned long long)c << FKEY_BITS) | m;
  val[k] = k;
}

// sorted position s <- generator val[s]; sid holds the tessellation-local index
__global__ void batch_gather_kernel(const double* __restrict__ gen, int n,
                                    const unsigned long long* __restrict__ key,
                                    const int32_t* __restrict__ val, const int32_t* __restrict__ pos,
                                    int nj, double* __restrict__ sx, double* __restrict__ sy,
                                    double* __restrict__ sz, int32_t* __restrict__ sid,
                                    uint32_t* __restrict__ fkey) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const int k = val[s];
  sx[s] = gen[3 * (int64_t)k];
  sy[s] = gen[3 * (int64_t)k + 1];
  sz[s] = gen[3 * (int64_t)k + 2];
  sid[s] = k - pos[batch_find(pos, nj, k)];
  fkey[s] = (uint32_t)(key[s] & ((1ull << FKEY_BITS) - 1ull));
}

// cell_start entries of tessellation j's cells (and end cell) become local positions
__global__ void batch_local_starts_kernel(int32_t* __restrict__ start, int64_t ncell,
                                          const int32_t* __restrict__ cbase, const int32_t* __restrict__ pos,
                                          int nj) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncell) return;
  start[c] -= pos[batch_find(cbase, nj, c)];
}

// Voronoi::finalize over a batch: faces carry the batch position of their left cell
// until the CSR is built; right indices are local to the tessellation
__global__ void batch_in_count_kernel(const int32_t* __restrict__ left, const int32_t* __restrict__ right,
                                      const uint8_t* __restrict__ code, int64_t F,
                                      const int32_t* __restrict__ pos, int nj,
                                      int32_t* __restrict__ in_count) {
  const int64_t f = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= F) return;
  const int r = right[f];
  if (r >= 0 && code[f] == 13) atomicAdd(in_count + r + pos[batch_find(pos, nj, left[f])], 1);
}

__global__ void batch_conn_fill_kernel(const int32_t* __restrict__ left, const int32_t* __restrict__ right,
                                       const uint8_t* __restrict__ code, const int64_t* __restrict__ face_off,
                                       const int64_t* __restrict__ conn_off,
                                       const int32_t* __restrict__ in_count, int32_t* __restrict__ cursor,
                                       int64_t F, const int32_t* __restrict__ pos, int nj,
                                       int32_t* __restrict__ conn) {
  const int64_t f = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= F) return;
  const int l = left[f];
  conn[conn_off[l] + in_count[l] + (f - face_off[l])] = (int32_t)f;
  const int r = right[f];
  if (r >= 0 && code[f] == 13) {
    const int rg = r + pos[batch_find(pos, nj, l)];
    const int slot = atomicAdd(cursor + rg, 1);
    conn[conn_off[rg] + slot] = (int32_t)f;
  }
}

// first face and first connection of each tessellation (j = nj: the totals)
__global__ void batch_bases_kernel(const int64_t* __restrict__ face_off, const int64_t* __restrict__ conn_off,
                                   const int32_t* __restrict__ pos, int nj, int64_t* __restrict__ fbase,
                                   int64_t* __restrict__ cbase_conn) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j > nj) return;
  fbase[j] = face_off[pos[j]];
  if (conn_off != nullptr) cbase_conn[j] = conn_off[pos[j]];
}

// faces: left becomes local; CSR: offsets and face indices become local
__global__ void batch_local_faces_kernel(int32_t* __restrict__ left, int64_t F,
                                         const int32_t* __restrict__ pos, int nj) {
  const int64_t f = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= F) return;
  left[f] -= pos[batch_find(pos, nj, left[f])];
}

__global__ void batch_local_conn_kernel(int64_t* __restrict__ conn_off,
                                        const int32_t* __restrict__ conn_count,
                                        int32_t* __restrict__ conn, int n, const int32_t* __restrict__ pos,
                                        int nj, const int64_t* __restrict__ fbase,
                                        const int64_t* __restrict__ cbase_conn) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n) return;
  const int j = batch_find(pos, nj, c);
  const int64_t o = conn_off[c];
  const int32_t fb = (int32_t)fbase[j];
  for (int i = 0; i < conn_count[c]; i++) conn[o + i] -= fb;
  conn_off[c] = o - cbase_conn[j];
}

// ---------------------------------------------------------------- launchers --
static inline int nblk(int64_t n, int t) { return (int)((n + t - 1) / t); }

void launch_prep(const double* xyz, int n, int dim, double* gen, unsigned long long* ext_keys,
                 double* ext, int* bad, cudaStream_t st) {
  if (n > 0) prep_kernel<<<nblk(n, 256), 256, 0, st>>>(xyz, n, dim, gen, ext_keys, bad);
  ext_finish_kernel<<<1, 32, 0, st>>>(ext_keys, ext);
}

void launch_grid(const double* gen, int n, const int G[3], const double a[3], const double inv[3],
                 int32_t* cid, int32_t* count, int32_t* start, int32_t* fill, double* sx, double* sy,
                 double* sz, int32_t* sid, long long* scan_tmp, cudaStream_t st);

template <class In, class Out>
static void scan_impl(const In* in, int64_t n, Out* out, long long* tmp, cudaStream_t st) {
  if (n <= 0) {
    cudaMemsetAsync(out, 0, sizeof(Out), st);
    return;
  }
  int nb = (int)((n + SCAN_TILE - 1) / SCAN_TILE);
  scan_reduce_kernel<In><<<nb, SCAN_THREADS, 0, st>>>(in, n, tmp);
  scan_sums_kernel<<<1, SCAN_THREADS, 0, st>>>(tmp, nb);
  scan_final_kernel<In, Out><<<nb, SCAN_THREADS, 0, st>>>(in, n, tmp, out);
}

size_t scan_tmp_elems(int64_t n) { return (size_t)((n + SCAN_TILE - 1) / SCAN_TILE) + 1; }

void scan_i32_to_i32(const int32_t* in, int64_t n, int32_t* out, long long* tmp, cudaStream_t st) {
  scan_impl<int32_t, int32_t>(in, n, out, tmp, st);
}
void scan_i32_to_i64(const int32_t* in, int64_t n, int64_t* out, long long* tmp, cudaStream_t st) {
  scan_impl<int32_t, int64_t>(in, n, out, tmp, st);
}

void launch_grid(const double* gen, int n, const int G[3], const double a[3], const double inv[3],
                 int32_t* cid, int32_t* count, int32_t* start, int32_t* fill, double* sx, double* sy,
                 double* sz, int32_t* sid, long long* scan_tmp, cudaStream_t st) {
  GridParams gp;
  for (int i = 0; i < 3; i++) gp.G[i] = G[i], gp.a[i] = a[i], gp.inv[i] = inv[i];
  gp.dim = 3;
  int64_t ncell = (int64_t)G[0] * G[1] * G[2];
  if (n > 0) cell_index_kernel<<<nblk(n, 256), 256, 0, st>>>(gen, n, gp, cid, count);
  scan_i32_to_i32(count, ncell, start, scan_tmp, st);
  if (n > 0) scatter_kernel<<<nblk(n, 256), 256, 0, st>>>(gen, n, cid, start, fill, sx, sy, sz, sid);
}

// First half of the two-level grid: coarse cell index, counts, starts and the dense
// cells (flags and their running count).  The host reads the number of dense cells,
// then calls launch_grid_dense (or scatters coarse-only).
void launch_grid_coarse(const double* gen, int n, const int G[3], const double a[3],
                        const double inv[3], int32_t* cid, int32_t* count, int32_t* start,
                        int32_t* dflag, int32_t* dprefix, int dim, long long* scan_tmp, cudaStream_t st) {
  GridParams gp;
  for (int i = 0; i < 3; i++) gp.G[i] = G[i], gp.a[i] = a[i], gp.inv[i] = inv[i];
  gp.dim = dim;
  const int64_t ncell = (int64_t)G[0] * G[1] * G[2];
  if (n > 0) cell_index_kernel<<<nblk(n, 256), 256, 0, st>>>(gen, n, gp, cid, count);
  scan_i32_to_i32(count, ncell, start, scan_tmp, st);
  dense_flag_kernel<<<nblk(ncell, 256), 256, 0, st>>>(count, ncell, dflag);
  scan_i32_to_i32(dflag, ncell, dprefix, scan_tmp, st);
}

// Scratch bytes of launch_grid_dense's radix sort.
size_t grid_dense_sort_bytes(int n, int64_t ncell) {
  size_t bytes = 0;
  int end_bit = FKEY_BITS;
  while ((1ll << (end_bit - FKEY_BITS)) < ncell) end_bit++;
  cub::DeviceRadixSort::SortPairs(nullptr, bytes, (const unsigned long long*)nullptr,
                                  (unsigned long long*)nullptr, (const int32_t*)nullptr,
                                  (int32_t*)nullptr, n, 0, end_bit);
  return bytes;
}

// Second half when some cells are dense: one stable radix sort of (cell, Morton key)
// pairs orders the generators by coarse cell and, inside dense cells, by key.
cudaError_t launch_grid_dense(const double* gen, int n, const int G[3], const double a[3],
                              const double inv[3], int dim, const int32_t* cid, const int32_t* dflag,
                              unsigned long long* key_a, unsigned long long* key_b, int32_t* val_a,
                              int32_t* val_b, void* sort_tmp, size_t sort_bytes, double* sx,
                              double* sy, double* sz, int32_t* sid, uint32_t* fkey, cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  GridParams gp;
  for (int i = 0; i < 3; i++) gp.G[i] = G[i], gp.a[i] = a[i], gp.inv[i] = inv[i];
  gp.dim = dim;
  const int64_t ncell = (int64_t)G[0] * G[1] * G[2];
  int end_bit = FKEY_BITS;
  while ((1ll << (end_bit - FKEY_BITS)) < ncell) end_bit++;
  dense_key_kernel<<<nblk(n, 256), 256, 0, st>>>(gen, n, gp, cid, dflag, key_a, val_a);
  cudaError_t e = cub::DeviceRadixSort::SortPairs(sort_tmp, sort_bytes, key_a, key_b, val_a, val_b,
                                                  n, 0, end_bit, st);
  if (e != cudaSuccess) return e;
  dense_gather_kernel<<<nblk(n, 256), 256, 0, st>>>(gen, n, key_b, val_b, sx, sy, sz, sid, fkey);
  return cudaGetLastError();
}

void launch_scatter(const double* gen, int n, const int32_t* cid, const int32_t* start,
                    int32_t* fill, double* sx, double* sy, double* sz, int32_t* sid, cudaStream_t st) {
  if (n > 0) scatter_kernel<<<nblk(n, 256), 256, 0, st>>>(gen, n, cid, start, fill, sx, sy, sz, sid);
}

void launch_reorder(const FaceArrays& stage, int64_t F, const int64_t* stage_off,
                    const int64_t* face_off, const FaceArrays& out, cudaStream_t st) {
  if (F > 0) reorder_faces_kernel<<<nblk(F, 256), 256, 0, st>>>(stage, F, stage_off, face_off, out);
}

void launch_csr_counts(const FaceArrays& f, int64_t F, const int32_t* face_count, int n,
                       int32_t* in_count, int32_t* conn_count, cudaStream_t st) {
  if (F > 0) in_count_kernel<<<nblk(F, 256), 256, 0, st>>>(f.right, f.code, F, in_count);
  if (n > 0) conn_count_kernel<<<nblk(n, 256), 256, 0, st>>>(face_count, in_count, n, conn_count);
}

void launch_csr_fill(const FaceArrays& f, int64_t F, const int64_t* face_off, const int64_t* conn_off,
                     const int32_t* in_count, int32_t* cursor, int n, int32_t* conn, cudaStream_t st) {
  if (F > 0)
    conn_fill_kernel<<<nblk(F, 256), 256, 0, st>>>(f.left, f.right, f.code, F, face_off, conn_off,
                                                   in_count, cursor, conn);
  if (n > 0) conn_sort_kernel<<<nblk(n, 256), 256, 0, st>>>(conn_off, in_count, n, conn);
}

// ------------------------------------------------------------ batch launchers --
void launch_batch_grid(const double* xyz, int n, const int32_t* pos, const int32_t* cbase, int nj,
                       const BatchGrid* bg, int64_t ncell, double* gen, unsigned long long* ext_keys,
                       double* ext, int* bad, int32_t* cid, int32_t* count, int32_t* start,
                       int32_t* dflag, int32_t* dprefix, long long* scan_tmp, cudaStream_t st) {
  batch_ext_init_kernel<<<nblk(6 * (int64_t)nj, 256), 256, 0, st>>>(ext_keys, nj);
  if (n > 0) batch_prep_kernel<<<nblk(n, 256), 256, 0, st>>>(xyz, n, pos, nj, bg, gen, ext_keys, bad);
  batch_ext_finish_kernel<<<nblk(6 * (int64_t)nj, 256), 256, 0, st>>>(ext_keys, ext, nj);
  if (n > 0) batch_cell_index_kernel<<<nblk(n, 256), 256, 0, st>>>(gen, n, pos, nj, bg, cid, count);
  scan_i32_to_i32(count, ncell, start, scan_tmp, st);
  dense_flag_kernel<<<nblk(ncell, 256), 256, 0, st>>>(count, ncell, dflag);
  scan_i32_to_i32(dflag, ncell, dprefix, scan_tmp, st);
}

size_t batch_sort_bytes(int n, int64_t ncell) { return grid_dense_sort_bytes(n, ncell); }

cudaError_t launch_batch_sort(const double* gen, int n, const int32_t* pos, const int32_t* cbase, int nj,
                              const BatchGrid* bg, int64_t ncell, const int32_t* cid, const int32_t* dflag,
                              unsigned long long* key_a, unsigned long long* key_b, int32_t* val_a,
                              int32_t* val_b, void* sort_tmp, size_t sort_bytes, double* sx, double* sy,
                              double* sz, int32_t* sid, uint32_t* fkey, int32_t* start, cudaStream_t st) {
  if (n > 0) {
    int end_bit = FKEY_BITS;
    while ((1ll << (end_bit - FKEY_BITS)) < ncell) end_bit++;
    batch_key_kernel<<<nblk(n, 256), 256, 0, st>>>(gen, n, pos, nj, bg, cid, dflag, key_a, val_a);
    cudaError_t e = cub::DeviceRadixSort::SortPairs(sort_tmp, sort_bytes, key_a, key_b, val_a, val_b, n, 0,
                                                    end_bit, st);
    if (e != cudaSuccess) return e;
    batch_gather_kernel<<<nblk(n, 256), 256, 0, st>>>(gen, n, key_b, val_b, pos, nj, sx, sy, sz, sid, fkey);
  }
  batch_local_starts_kernel<<<nblk(ncell, 256), 256, 0, st>>>(start, ncell, cbase, pos, nj);
  return cudaGetLastError();
}

void launch_batch_csr(const FaceArrays& f, int64_t F, const int64_t* face_off, const int32_t* face_count,
                      int n, const int32_t* pos, int nj, int32_t* in_count, int32_t* conn_count,
                      cudaStream_t st) {
  if (F > 0)
    batch_in_count_kernel<<<nblk(F, 256), 256, 0, st>>>(f.left, f.right, f.code, F, pos, nj, in_count);
  if (n > 0) conn_count_kernel<<<nblk(n, 256), 256, 0, st>>>(face_count, in_count, n, conn_count);
}

void launch_batch_csr_fill(const FaceArrays& f, int64_t F, const int64_t* face_off, const int64_t* conn_off,
                           const int32_t* in_count, int32_t* cursor, int n, const int32_t* pos, int nj,
                           int32_t* conn, cudaStream_t st) {
  if (F > 0)
    batch_conn_fill_kernel<<<nblk(F, 256), 256, 0, st>>>(f.left, f.right, f.code, face_off, conn_off,
                                                         in_count, cursor, F, pos, nj, conn);
  if (n > 0) conn_sort_kernel<<<nblk(n, 256), 256, 0, st>>>(conn_off, in_count, n, conn);
}

void launch_batch_localize(FaceArrays& f, int64_t F, const int64_t* face_off, int64_t* conn_off,
                           const int32_t* conn_count, int32_t* conn, int n, const int32_t* pos, int nj,
                           int64_t* fbase, int64_t* cbase_conn, cudaStream_t st) {
  batch_bases_kernel<<<nblk(nj + 1, 256), 256, 0, st>>>(face_off, conn_off, pos, nj, fbase, cbase_conn);
  if (F > 0) batch_local_faces_kernel<<<nblk(F, 256), 256, 0, st>>>(f.left, F, pos, nj);
  if (conn_off != nullptr && n > 0)
    batch_local_conn_kernel<<<nblk(n, 256), 256, 0, st>>>(conn_off, conn_count, conn, n, pos, nj, fbase,
                                                          cbase_conn);
}

}  // namespace mv
