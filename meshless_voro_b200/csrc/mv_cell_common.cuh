// mv_cell_common.cuh -- device building blocks shared by the cell kernels.
//
// The fused cell kernel (mv_cells.cu) and the staged shell / clip / integral kernels
// (mv_staged.cu) are built from these pieces:
//   * the nearest-first neighbour shell (rtree_nn.rs:10-240) gathered from the
//     uniform grid and sorted by (f64 squared distance, original index, shift code);
//   * the exact clip decision (half_space.rs:40-47, boundary.rs:49-64,
//     geometry.rs:271-314), Vertex::from_dual (convex_cell.rs:28-48) and the ring of a
//     clip (compute_boundary + SimpleCycle, convex_cell.rs:421-441, simple_cycle.rs);
//   * the cell and face integrals (convex_cell.rs:131-187, voronoi_cell.rs:40-100,
//     integrals.rs) over a read-only view of a finished cell.
// Cell-state functions are templates over the shared-memory layout `SM`, which
// provides the plane arrays pnx/pny/pnz/pd/pright/pcode/rptr, the vertex arrays
// vx/vy/vz/vr2/f4/vd0/vd1/vd2/ord/ea/eb under those names (f4 holds the f32 offset
// v - x of the filter; ord is 4-byte aligned) and plane_point(J, k), the point p of
// boundary plane k.
#pragma once
#include <cstdint>

#include "../../include/mvgpu.h"
#include "mv_exact.cuh"
#include "mv_geom.cuh"
#include "mv_internal.h"

namespace mv {

constexpr unsigned FULL = 0xffffffffu;

template <int VMAX_, int PMAX_, int CMAX_, int KMAX_, typename PIdx_, int MINB_>
struct Tier {
  static constexpr int MINB = MINB_;  // min resident blocks per SM (register budget)
  static constexpr int VMAX = VMAX_;  // vertices
  static constexpr int PMAX = PMAX_;  // clipping planes
  static constexpr int CMAX = CMAX_;  // neighbour-shell entries
  static constexpr int KMAX = KMAX_;  // neighbours set up per batch
  static constexpr int NW = VMAX / 32;
  using PIdx = PIdx_;
  static constexpr unsigned NONE = (unsigned)(PIdx)(~0u);
  static_assert(VMAX % 32 == 0 && PMAX % 32 == 0 && CMAX % 32 == 0, "tier sizes");
  static_assert(PMAX < (int)NONE && VMAX < (int)NONE, "index type too small");
  static_assert(KMAX <= 32, "batch is set up by one lane per neighbour");
};

// ------------------------------------------------------------ small helpers --
__device__ __forceinline__ unsigned lanemask_lt() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

__device__ __forceinline__ int warp_excl_scan(int v, int lane, int* total) {
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(FULL, x, o);
    if (lane >= o) x += y;
  }
  *total = __shfl_sync(FULL, x, 31);
  return x - v;
}

__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(FULL, v, o));
  return v;
}

// Largest non-negative double over the warp: non-negative binary64 values order like
// their bit patterns, so two 32-bit warp reductions give the exact maximum.
__device__ __forceinline__ double warp_max_nonneg(double v) {
  const unsigned long long b = (unsigned long long)__double_as_longlong(v);
  const unsigned hi = (unsigned)(b >> 32), lo = (unsigned)b;
  const unsigned mhi = __reduce_max_sync(FULL, hi);
  const unsigned mlo = __reduce_max_sync(FULL, hi == mhi ? lo : 0u);
  return __longlong_as_double((long long)(((unsigned long long)mhi << 32) | mlo));
}

__device__ __forceinline__ D3 shfl_d3(D3 v, int src) {
  return {__shfl_sync(FULL, v.x, src), __shfl_sync(FULL, v.y, src), __shfl_sync(FULL, v.z, src)};
}

template <int NW>
__device__ __forceinline__ int rank_below(const unsigned (&m)[NW], int p) {
  int r = 0;
#pragma unroll
  for (int w = 0; w < NW; w++) {
    if (w < (p >> 5))
      r += __popc(m[w]);
    else if (w == (p >> 5))
      r += __popc(m[w] & ((1u << (p & 31)) - 1u));
  }
  return r;
}

// position of the s-th (1-based) set bit
template <int NW>
__device__ __forceinline__ int select_bit(const unsigned (&m)[NW], int s) {
#pragma unroll
  for (int w = 0; w < NW; w++) {
    int c = __popc(m[w]);
    if (s <= c) return 32 * w + (int)__fns(m[w], 0, s);
    s -= c;
  }
  return -1;
}

// position of the s-th (1-based) set bit of a 64-bit mask
__device__ __forceinline__ int select64(unsigned long long m, int s) {
  const unsigned lo = (unsigned)m;
  const int c = __popc(lo);
  return s <= c ? (int)__fns(lo, 0, s) : 32 + (int)__fns((unsigned)(m >> 32), 0, s - c);
}

__device__ __forceinline__ unsigned valid_bits(int nv, int w) {
  const int lim = nv - 32 * w;
  return lim >= 32 ? FULL : (lim <= 0 ? 0u : ((1u << lim) - 1u));
}

__device__ __forceinline__ void iloc(const Job& J, D3 l, int64_t out[3]) {
  const uint64_t mask = 0xFFFFFFFFFFFFFull;
  double c0 = 1.0 + (l.x - J.iloc_a[0]) * J.iloc_inv[0];
  double c1 = 1.0 + (l.y - J.iloc_a[1]) * J.iloc_inv[1];
  double c2 = 1.0 + (l.z - J.iloc_a[2]) * J.iloc_inv[2];
  out[0] = (int64_t)((uint64_t)__double_as_longlong(c0) & mask);
  out[1] = (int64_t)((uint64_t)__double_as_longlong(c1) & mask);
  out[2] = (int64_t)((uint64_t)__double_as_longlong(c2) & mask);
}

__device__ __forceinline__ D3 load_gen(const Job& J, int orig) {
  const double* g = J.gen + 3 * (int64_t)orig;
  return {__ldg(g), __ldg(g + 1), __ldg(g + 2)};
}

// HalfSpace::right_loc (half_space.rs:53-65)
template <class SM>
__device__ __forceinline__ D3 right_loc(const Job& J, const SM& S, int k, D3 x) {
  int r = S.pright[k];
  if (r >= 0) {
    D3 l = load_gen(J, r);
    int code = S.pcode[k];
    if (code != 13) l = add(l, D3{J.shift[code][0], J.shift[code][1], J.shift[code][2]});
    return l;
  }
  D3 pr = plane_project({S.pnx[k], S.pny[k], S.pnz[k]}, S.plane_point(J, k), x);
  return sub(scale(2.0, pr), x);
}

// Exact decision of clip_by_plane for an undecided vertex in slot `s`
// (convex_cell.rs:370-382).
template <class SM>
__device__ __noinline__ int exact_clip(const Job& J, const SM& S, int s, D3 x, D3 ngb) {
  int64_t A[3], B[3], C[3], Dd[3], W[3];
  iloc(J, x, A);
  iloc(J, right_loc(J, S, S.vd0[s], x), B);
  iloc(J, right_loc(J, S, S.vd1[s], x), C);
  iloc(J, right_loc(J, S, S.vd2[s], x), Dd);
  iloc(J, ngb, W);
  return in_sphere_exact_sign(A, B, C, Dd, W);
}

// Whether the exact decision of exact_clip is the zero determinant of five corners of
// one axis-aligned box (box_corners), found without multi-limb arithmetic: the vertex
// is then kept.
template <class SM>
__device__ __noinline__ bool exact_clip_box_zero(const Job& J, const SM& S, int s, D3 x, D3 ngb) {
  int64_t A[3], B[3], C[3], Dd[3], W[3];
  iloc(J, x, A);
  iloc(J, right_loc(J, S, S.vd0[s], x), B);
  iloc(J, right_loc(J, S, S.vd1[s], x), C);
  iloc(J, right_loc(J, S, S.vd2[s], x), Dd);
  iloc(J, ngb, W);
  return box_corners(A, B, C, Dd, W);
}

// Vertex::from_dual (convex_cell.rs:28-48) into slot `slot`; *r2 receives the
// vertex's squared distance to the generator (kept in S.vr2 when STORE_R2; otherwise
// vertex_r2 recomputes it).
template <class PIdx, bool STORE_R2 = true, class SM>
__device__ __forceinline__ bool make_vertex(SM& S, int slot, int i, int j, int k, D3 x, int dim,
                                            double* r2) {
  D3 loc;
  bool ok = intersect3({S.pnx[i], S.pny[i], S.pnz[i]}, S.pd[i], {S.pnx[j], S.pny[j], S.pnz[j]},
                       S.pd[j], {S.pnx[k], S.pny[k], S.pnz[k]}, S.pd[k], &loc);
  if (!ok) return false;
  D3 dl = loc;
  if (dim == 1) dl = {loc.x, 0.0, 0.0};
  if (dim == 2) dl = {loc.x, loc.y, 0.0};
  D3 r = sub(x, dl);
  const double rr = dot(r, r);
  S.vx[slot] = loc.x;
  S.vy[slot] = loc.y;
  S.vz[slot] = loc.z;
  if constexpr (STORE_R2) S.vr2[slot] = rr;
  S.f4[slot] = make_float4(__double2float_rn(loc.x - x.x), __double2float_rn(loc.y - x.y),
                           __double2float_rn(loc.z - x.z), 0.f);
  S.vd0[slot] = (PIdx)i;
  S.vd1[slot] = (PIdx)j;
  S.vd2[slot] = (PIdx)k;
  *r2 = rr;
  return true;
}

// The squared distance of the vertex in slot `slot` to the generator, as make_vertex
// computes it (Vertex::from_dual, convex_cell.rs:38-42).
template <class SM>
__device__ __forceinline__ double vertex_r2(const SM& S, int slot, D3 x, int dim) {
  D3 dl = {S.vx[slot], S.vy[slot], S.vz[slot]};
  if (dim == 1) dl = {dl.x, 0.0, 0.0};
  if (dim == 2) dl = {dl.x, dl.y, 0.0};
  const D3 r = sub(x, dl);
  return dot(r, r);
}

// Vertex duals of the initial cuboid (convex_cell.rs:298-307), one vertex per lane.
__device__ __forceinline__ void cuboid_duals(int lane, int* i0, int* i1, int* i2) {
  switch (lane) {
    case 0: *i0 = 2, *i1 = 5, *i2 = 0; break;
    case 1: *i0 = 5, *i1 = 3, *i2 = 0; break;
    case 2: *i0 = 1, *i1 = 5, *i2 = 2; break;
    case 3: *i0 = 5, *i1 = 1, *i2 = 3; break;
    case 4: *i0 = 4, *i1 = 2, *i2 = 0; break;
    case 5: *i0 = 4, *i1 = 0, *i2 = 3; break;
    case 6: *i0 = 2, *i1 = 4, *i2 = 1; break;
    default: *i0 = 4, *i1 = 3, *i2 = 1; break;
  }
}

// Bound on |v - x| over the cell's vertices for the f32 filter: r2 omits the
// extruded dimensions, whose vertex coordinates are +-0.5.
__device__ __forceinline__ double amax_of(double max_r2, int dim) {
  return sqrt((max_r2 + 0.26 * (3 - dim)) * (1.0 + 1e-9)) * (1.0 + 1e-9);
}

// The same bound in f32, rounded up, from the safety radius sr = 2 sqrt(max_r2):
// sqrt(max_r2) <= sr / 2 (1 + 2^-52), |v - x| exceeds the rounded sqrt(max_r2) by a
// few ulps at most, and sqrt(a + b) <= sqrt(a) + sqrt(b) covers the extruded
// dimensions (sqrt(0.26) < 0.51, sqrt(0.52) < 0.7212).
__device__ __forceinline__ float amax32_of_sr(double sr, int dim) {
  const float h = __fmul_ru(__double2float_ru(sr), 0.50000006f);
  return dim == 3 ? h : __fadd_ru(h, dim == 2 ? 0.51f : 0.7212f);
}

enum CellResult {
  CELL_DONE = 0,
  CELL_OVERFLOW = 1,
  CELL_ERROR = 2,
  CELL_FACE_OVERFLOW = 3,
  CELL_RETRY = 4,  // staged path: the cell needs the fused kernel (more neighbours)
  CELL_REC_OVERFLOW = 5,  // export build: no room for the cell's record
  CELL_EXACT = 6  // staged path: a vertex needs the exact predicate; the fused kernel builds the cell
};

// Event counts of one cell, kept in warp-uniform registers (a lane-0 branch inside
// the clip loop would split the warp) and flushed once per cell.
struct CellCount {
  unsigned c[ST_COUNT];
};
#define WCNT(CC, slot, v) ((CC).c[slot] += (unsigned)(v))

// ------------------------------------------------------------- neighbour shell --
// First position in [a, b) whose dense-cell key is >= k (the keys of a dense cell are
// sorted).
__device__ __forceinline__ int32_t fkey_lower_bound(const Job& J, int32_t a, int32_t b, uint32_t k) {
  while (a < b) {
    const int32_t m = (a + b) >> 1;
    if (__ldg(J.fkey + m) < k)
      a = m + 1;
    else
      b = m;
  }
  return a;
}

// Radius of a cell's first shell: R0, scaled down in dense cells by the local density,
// taken from the finest octree cell around the generator that still holds 8 generators
// (lane l counts level l), so that the first shell holds about as many candidates as in
// a uniform region.  Shells are prefixes of the same nearest-first stream, so the
// radius only moves work between shells, never the result.
__device__ __forceinline__ double first_radius(const Job& J, D3 x, int lane) {
  if (J.fkey == nullptr) return J.R0;
  const double xa[3] = {x.x, x.y, x.z};
  int c[3];
#pragma unroll
  for (int i = 0; i < 3; i++) {
    double f = floor((xa[i] - J.ga[i]) * J.ginv[i]);
    if (!(f >= 0.0)) f = 0.0;
    if (f > J.G[i] - 1) f = J.G[i] - 1;
    c[i] = (int)f;
  }
  const int64_t cc = (int64_t)c[0] + (int64_t)J.G[0] * (c[1] + (int64_t)J.G[1] * c[2]);
  if (!__ldg(J.cell_dense + cc)) return J.R0;
  const int32_t cs = __ldg(J.cell_start + cc), ce = __ldg(J.cell_start + cc + 1);
  const int B = J.fbits, dim = J.dim;
  uint32_t q[3] = {0u, 0u, 0u};
  for (int i = 0; i < dim; i++) q[i] = fine_q(xa[i], J.ga[i], J.ginv[i], c[i], B);
  const uint32_t key = morton(dim, q[0], q[1], q[2]);
  int cl = 0;
  if (lane <= B) {
    const int sh = dim * (B - lane);
    const uint32_t klo = (key >> sh) << sh;
    const int32_t a = fkey_lower_bound(J, cs, ce, klo);
    cl = fkey_lower_bound(J, a, ce, klo + (1u << sh)) - a;
  }
  const unsigned bal = __ballot_sync(FULL, lane <= B && cl >= 8);
  if (bal == 0u) return J.R0;
  const int L = 31 - __clz(bal);
  const int cnt = __shfl_sync(FULL, cl, L);
  const double ratio = (double)cnt * exp2((double)(dim * L)) / J.ppc_mean;
  if (!(ratio > 1.0)) return J.R0;
  return J.R0 * pow(ratio, -1.0 / dim);
}

template <int CMAX>
struct ShellBuf {
  unsigned long long key[CMAX];  // f64 squared distance bits
  uint32_t tie[CMAX];            // original index * 27 + shift code
  int32_t cpos[CMAX];            // grid-sorted position of the generator
  int32_t sstart[96];
  int32_t spref[97];
  int32_t gbin;                  // next bin of a staged shell (big shells), -1: none
  int32_t total;                 // elements of the current shell (all its groups)
  uint8_t scode[96];
};

// ------------------------------------------------------------------ big shells --
// A shell of the fused kernel that holds more than the shared-memory buffer (up to
// BIG_CAP elements) is staged in the warp's slot of a global buffer, bucketed by d2 into
// BIG_BINS bins and consumed group by group, each group (whole bins, at most CMAX
// elements) sorted in shared memory.  Bins are monotone in d2, so the groups come in
// stream order and each group sorted by (d2, tie) continues the nearest-first stream
// exactly.  Dense clumps make such shells common: the safety radius of a cell on the
// surface of a compact clump takes in the whole clump.
constexpr int BIG_CAP = 32768;
constexpr int BIG_BINS = 2048;
constexpr size_t BIG_SLOT_BYTES = (size_t)BIG_CAP * 32 + (size_t)BIG_BINS * 8;

struct BigView {
  unsigned long long* keyA;  // the gathered shell (elements >= CMAX; the rest in shared)
  unsigned long long* keyB;  // the shell bucketed by bin
  uint32_t* tieA;
  uint32_t* tieB;
  int32_t* cposA;
  int32_t* cposB;
  int32_t* pinc;             // [BIG_BINS] inclusive prefix of the bin counts
  int32_t* hist;             // [BIG_BINS] bin counts, then the bucketing cursors
};

__device__ __forceinline__ BigView big_view(char* slot) {
  BigView V;
  V.keyA = reinterpret_cast<unsigned long long*>(slot);
  V.keyB = V.keyA + BIG_CAP;
  V.tieA = reinterpret_cast<uint32_t*>(V.keyB + BIG_CAP);
  V.tieB = V.tieA + BIG_CAP;
  V.cposA = reinterpret_cast<int32_t*>(V.tieB + BIG_CAP);
  V.cposB = V.cposA + BIG_CAP;
  V.pinc = V.cposB + BIG_CAP;
  V.hist = V.pinc + BIG_BINS;
  return V;
}

__device__ __forceinline__ int big_bin(unsigned long long key, double lo2, double scale) {
  const double t = (__longlong_as_double((long long)key) - lo2) * scale;
  return t >= (double)(BIG_BINS - 1) ? BIG_BINS - 1 : (t > 0.0 ? (int)t : 0);
}

// Buckets the cnt (CMAX < cnt <= BIG_CAP) elements of a gathered shell [lo2, R2) into
// the slot's B arrays by bin and returns the largest bin count; when that exceeds CMAX
// nothing is bucketed and the caller narrows the shell instead.  The counters live in
// the slot (global memory, private to the warp).
template <int CMAX>
__device__ __noinline__ int big_bucket(ShellBuf<CMAX>& B, char* slot, int lane, int cnt, double lo2,
                                       double R2) {
  const BigView V = big_view(slot);
  for (int i = lane; i < CMAX; i += 32) {
    V.keyA[i] = B.key[i];
    V.tieA[i] = B.tie[i];
    V.cposA[i] = B.cpos[i];
  }
  for (int i = lane; i < BIG_BINS; i += 32) V.hist[i] = 0;
  __syncwarp();
  const double scale = (double)BIG_BINS / (R2 - lo2);
  for (int i = lane; i < cnt; i += 32) atomicAdd(&V.hist[big_bin(V.keyA[i], lo2, scale)], 1);
  __syncwarp();
  // lane l owns bins [PER l, PER (l + 1))
  constexpr int PER = BIG_BINS / 32;
  int sum = 0, mx = 0;
  for (int k = 0; k < PER; k++) {
    const int c = V.hist[PER * lane + k];
    sum += c;
    mx = max(mx, c);
  }
  mx = (int)__reduce_max_sync(FULL, (unsigned)mx);
  if (mx > CMAX) return mx;
  int tot;
  int ex = warp_excl_scan(sum, lane, &tot);
  for (int k = 0; k < PER; k++) {
    const int c = V.hist[PER * lane + k];
    V.hist[PER * lane + k] = ex;
    ex += c;
    V.pinc[PER * lane + k] = ex;
  }
  __syncwarp();
  for (int i = lane; i < cnt; i += 32) {
    const unsigned long long key = V.keyA[i];
    const int pos = atomicAdd(&V.hist[big_bin(key, lo2, scale)], 1);
    V.keyB[pos] = key;
    V.tieB[pos] = V.tieA[i];
    V.cposB[pos] = V.cposA[i];
  }
  __syncwarp();
  return mx;
}

// Loads the next group of whole bins, starting at bin B.gbin, that holds at most CMAX
// elements into B (unsorted) and returns its size; B.gbin moves past the group (-1
// after the last bin).
template <int CMAX>
__device__ __noinline__ int big_group(ShellBuf<CMAX>& B, char* slot, int lane) {
  const BigView V = big_view(slot);
  const int b = B.gbin;
  const int base = b > 0 ? V.pinc[b - 1] : 0;
  // the last bin e >= b with pinc[e] <= base + CMAX (bin b alone holds <= CMAX)
  int lo = b, hi = BIG_BINS - 1;
  while (lo < hi) {
    const int m = (lo + hi + 1) >> 1;
    if (V.pinc[m] <= base + CMAX)
      lo = m;
    else
      hi = m - 1;
  }
  const int end = V.pinc[lo];
  for (int i = lane; i < end - base; i += 32) {
    B.key[i] = V.keyB[base + i];
    B.tie[i] = V.tieB[base + i];
    B.cpos[i] = V.cposB[base + i];
  }
  if (lane == 0) B.gbin = lo + 1 < BIG_BINS ? lo + 1 : -1;
  __syncwarp();
  return end - base;
}

// The warp's staging slot (global warp index).
__device__ __forceinline__ char* big_slot(const Job& J) {
  if (J.big == nullptr) return nullptr;
  const size_t w = (size_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  return J.big + w * BIG_SLOT_BYTES;
}
// Elements a shell of the fused kernel may hold: a staging slot, or without slots the
// count at which the gather stops (the shared buffer then takes CMAX of them).
template <int CMAX>
__device__ __forceinline__ int big_fits(const Job& J) {
  return J.big != nullptr ? BIG_CAP : 32 * CMAX;
}

// Tessellation of batch position pos (the last j with pos_base[j] <= pos).
__device__ __forceinline__ int job_of(const JobTable& T, int pos) {
  int a = 0, b = T.njobs - 1;
  while (a < b) {
    const int m = (a + b + 1) >> 1;
    if (__ldg(T.pos_base + m) <= pos)
      a = m;
    else
      b = m - 1;
  }
  return a;
}

// Gathers every stream element (generator, periodic image) with lo2 <= d2 < R*R into
// B (unsorted) and returns how many there are (may exceed CMAX; once the count passes
// stop the gather ends early and returns a count above stop).  With BIG and a slot,
// elements CMAX .. BIG_CAP - 1 go to the slot's A arrays.  *exhausted is set
// when the enumerated cells cover every image and none lies beyond R, i.e. the stream
// ends with this shell.  d2 is the reference's squared distance:
// (g - q).length_squared() for nn_iter (rstar) and |(q + s) - g|^2 for
// wrapping_nn_iter (rtree_nn.rs:138-146).
//
// Grid rows (y, z) go to lanes; a lane turns the cells of its row that the ball
// reaches into contiguous segments of sorted positions (one per periodic image).  A
// segment that contains a dense cell (J.dprefix) is deferred: its cells are then
// visited one by one, and a dense cell contributes the octree cells that the shell
// reaches.  Without the ball test (all images enumerated) every cell counts whole.
template <int CMAX, bool BIG, bool DENSE, bool CODE_ONLY>
__device__ __noinline__ int gather_shell_impl(const Job& J, ShellBuf<CMAX>& B, int lane, D3 x, double R,
                                              double lo2, const double* ext, bool* exhausted,
                                              int stop, char* big) {
  const double xa[3] = {x.x, x.y, x.z};
  int lo[3], hi[3];
  bool all = true;
#pragma unroll
  for (int i = 0; i < 3; i++) {
    int G = J.G[i];
    bool wrap = J.periodic && i < J.dim;
    int umin = wrap ? -G : 0, umax = wrap ? 2 * G - 1 : G - 1;
    double fl = floor((xa[i] - R - J.ga[i]) * J.ginv[i]) - 1.0;
    double fh = floor((xa[i] + R - J.ga[i]) * J.ginv[i]) + 1.0;
    lo[i] = fl < (double)umin ? umin : (int)fl;
    hi[i] = fh > (double)umax ? umax : (int)fh;
    if (lo[i] > umin || hi[i] < umax) all = false;
  }
  const double R2 = R * R;
  const double R2v = R2 * (1.0 + 1e-9);
  int beyond = 0;
  const int ny = hi[1] - lo[1] + 1, nz = hi[2] - lo[2] + 1;
  const int nrows = ny * nz;
  int count = 0;

  // bounds of coarse cell c (image m) along axis i, inflated against rounding; the
  // edge cells reach the generators' extent (periodic) or infinity (rectangular)
  auto cell_lo = [&](int i, int c, int m) -> double {
    const bool wrap = J.periodic && i < J.dim;
    double blo = J.ga[i] + c * J.gh[i];
    if (c == 0) blo = wrap ? fmin(blo, ext[i]) : -__longlong_as_double(0x7ff0000000000000ll);
    return blo + m * J.gw[i] - J.geps[i];
  };
  auto cell_hi = [&](int i, int c, int m) -> double {
    const bool wrap = J.periodic && i < J.dim;
    double bhi = J.ga[i] + (c + 1) * J.gh[i];
    if (c == J.G[i] - 1) bhi = wrap ? fmax(bhi, ext[3 + i]) : __longlong_as_double(0x7ff0000000000000ll);
    return bhi + m * J.gw[i] + J.geps[i];
  };
  auto dist1 = [&](int i, double blo, double bhi) -> double {
    return xa[i] < blo ? blo - xa[i] : (xa[i] > bhi ? xa[i] - bhi : 0.0);
  };
  // box-distance of unwrapped grid coordinate u along axis i
  auto box_d = [&](int i, int u) -> double {
    const int G = J.G[i];
    const int m = u < 0 ? -1 : (u >= G ? 1 : 0);
    const int c = u - m * G;
    return dist1(i, cell_lo(i, c, m), cell_hi(i, c, m));
  };

  // the elements of the segments [0, nsegs) of B (spref: running element counts)
  auto flush = [&](int nsegs_total, int total) {
    for (int t0 = 0; t0 < total && count <= stop; t0 += 32) {
      const int t = t0 + lane;
      bool keep = false;
      double d2 = 0.0;
      uint32_t tie = 0;
      int s = 0;
      if (t < total) {
        int a = 0, b = nsegs_total - 1;
        while (a < b) {
          int mid = (a + b + 1) >> 1;
          if (B.spref[mid] <= t)
            a = mid;
          else
            b = mid - 1;
        }
        s = B.sstart[a] + (t - B.spref[a]);
        const int code = B.scode[a];
        const double px = __ldg(J.sx + s), py = __ldg(J.sy + s), pz = __ldg(J.sz + s);
        const int orig = CODE_ONLY ? 0 : __ldg(J.sid + s);
        if (J.periodic) {
          const double ddx = (x.x + J.qshift[code][0]) - px;
          const double ddy = (x.y + J.qshift[code][1]) - py;
          const double ddz = (x.z + J.qshift[code][2]) - pz;
          d2 = ddx * ddx + ddy * ddy + ddz * ddz;
        } else {
          D3 dd = sub(D3{px, py, pz}, x);
          d2 = dot(dd, dd);
        }
        keep = (d2 >= lo2) && (d2 < R2);
        beyond += (d2 >= R2);
        tie = CODE_ONLY ? (uint32_t)code : (uint32_t)orig * 27u + (uint32_t)code;
      }
      const unsigned bal = __ballot_sync(FULL, keep);
      const int pos = count + __popc(bal & lanemask_lt());
      if (keep && pos < CMAX) {
        B.key[pos] = (unsigned long long)__double_as_longlong(d2);
        B.tie[pos] = tie;
        B.cpos[pos] = s;
      } else if (BIG && keep && big != nullptr && pos < BIG_CAP) {
        const BigView V = big_view(big);
        V.keyA[pos] = (unsigned long long)__double_as_longlong(d2);
        V.tieA[pos] = tie;
        V.cposA[pos] = s;
      }
      count += __popc(bal);
    }
    __syncwarp();
  };
  // segments of one per lane (len 0: none) into B, then their elements
  auto emit1 = [&](int32_t st0, int32_t len, int code) {
    const bool has = len > 0;
    const unsigned bal = __ballot_sync(FULL, has);
    const int at = __popc(bal & lanemask_lt());
    int tot;
    const int off = warp_excl_scan(len, lane, &tot);
    if (has) B.sstart[at] = st0, B.spref[at] = off, B.scode[at] = (uint8_t)code;
    __syncwarp();
    if (bal) flush(__popc(bal), tot);
  };
  // the octree cells of dense cell (cx, cy, cz), image (mx, my, mz), that the shell
  // [lo, R) reaches, at the level whose cells are at least half the shell's thickness
  // wide (at most five per axis for a first shell, 33 for the thinnest); a cell that
  // lies inside the inner radius holds no element of the shell
  auto dense_cell = [&](int cx, int cy, int cz, int mx, int my, int mz, int code) {
    const int64_t cc = (int64_t)cx + (int64_t)J.G[0] * (cy + (int64_t)J.G[1] * cz);
    const int32_t cs = __ldg(J.cell_start + cc), ce = __ldg(J.cell_start + cc + 1);
    if (all) {
      emit1(cs, lane == 0 ? ce - cs : 0, code);
      return;
    }
    const int B = J.fbits, dim = J.dim;
    double hmin = J.gh[0];
    for (int i = 1; i < dim; i++) hmin = fmin(hmin, J.gh[i]);
    // the level: cells at least half as wide as the shell is thick (R / 8 at the
    // thinnest), so that a thin shell's octree cells inside the inner radius drop out
    const double span = fmax(R - sqrt(lo2), 0.125 * R);
    const double r = 2.0 * hmin / span;
    const int L = r >= 2.0 ? min(B, ilogb(r)) : 0;
    const int nL = 1 << L;
    const int c3[3] = {cx, cy, cz}, m3[3] = {mx, my, mz};
    int ja[3], jn[3];
    double base[3], w[3], clo[3], chi[3];
#pragma unroll
    for (int i = 0; i < 3; i++) {
      clo[i] = cell_lo(i, c3[i], m3[i]);
      chi[i] = cell_hi(i, c3[i], m3[i]);
      base[i] = J.ga[i] + c3[i] * J.gh[i] + m3[i] * J.gw[i];
      w[i] = J.gh[i] / nL;
      ja[i] = 0, jn[i] = 1;
      if (i < dim) {
        const double fa = floor((xa[i] - R - base[i] - J.geps[i]) / w[i]);
        const double fb = floor((xa[i] + R - base[i] + J.geps[i]) / w[i]);
        const int lo_j = fa < 0.0 ? 0 : (fa > nL - 1 ? nL - 1 : (int)fa);
        const int hi_j = fb > nL - 1 ? nL - 1 : (fb < 0.0 ? 0 : (int)fb);
        ja[i] = lo_j, jn[i] = hi_j - lo_j + 1;
      }
    }
    const int sh = dim * (B - L);
    const int ncl = jn[0] * jn[1] * jn[2];
    const double lo2p = lo2 * (1.0 - 1e-9);
    for (int r0 = 0; r0 < ncl && count <= stop; r0 += 32) {
      const int t = r0 + lane;
      int32_t st0 = 0, len = 0;
      if (t < ncl) {
        const int j[3] = {ja[0] + t % jn[0], ja[1] + (t / jn[0]) % jn[1], ja[2] + t / (jn[0] * jn[1])};
        double dmin2 = 0.0, dmax2 = 0.0;
#pragma unroll
        for (int i = 0; i < 3; i++) {
          double blo = clo[i], bhi = chi[i];
          if (i < dim) {
            if (j[i] > 0) blo = base[i] + j[i] * w[i] - J.geps[i];
            if (j[i] < nL - 1) bhi = base[i] + (j[i] + 1) * w[i] + J.geps[i];
          }
          const double dn = dist1(i, blo, bhi);
          const double df = fmax(fabs(xa[i] - blo), fabs(bhi - xa[i]));
          dmin2 += dn * dn;
          dmax2 += df * df;
        }
        if (dmin2 < R2v && !(dmax2 < lo2p)) {
          const uint32_t klo = morton(dim, (uint32_t)j[0], (uint32_t)j[1], (uint32_t)j[2]) << sh;
          st0 = fkey_lower_bound(J, cs, ce, klo);
          len = fkey_lower_bound(J, st0, ce, klo + (1u << sh)) - st0;
        }
      }
      emit1(st0, len, code);
    }
  };

  // the x-distances of the cells lo[0] .. hi[0] are the same for every row: with at
  // most 32 of them, lane j holds cell lo[0] + j's and the rows read them by shuffle
  const int nx = hi[0] - lo[0] + 1;
  const bool xlanes = nx <= 32;
  double dx2l = 0.0;
  if (xlanes && lane < nx) {
    const double dx = box_d(0, lo[0] + lane);
    dx2l = dx * dx;
  }
  for (int row0 = 0; row0 < nrows && count <= stop; row0 += 32) {
    const int row = row0 + lane;
    int nseg = 0;
    int32_t s0a = 0, s0b = 0, s0c = 0, sla = 0, slb = 0, slc = 0;
    int sca = 0, scb = 0, scc = 0;
    // cell ranges holding a dense cell, deferred (one per image): c0 | c1 << 16, 0: none
    int dfr[3] = {-1, -1, -1};
    int my = 0, mz = 0, cy = 0, cz = 0;
    int uy = 0, uz = 0;
    double byz2 = 0.0;
    bool rowin = false;
    if (row < nrows) {
      uy = lo[1] + row % ny, uz = lo[2] + row / ny;
      const double dy = box_d(1, uy), dz = box_d(2, uz);
      byz2 = dy * dy + dz * dz;
      rowin = all || byz2 < R2v;
    }
    // the row's cells within the ball: the first and last x cell that pass
    int first = 1 << 30, last = -(1 << 30);
    if (xlanes) {
      for (int j = 0; j < nx; j++) {
        const double dx2 = __shfl_sync(FULL, dx2l, j);
        if (rowin && (all || dx2 + byz2 < R2v)) {
          first = min(first, lo[0] + j);
          last = max(last, lo[0] + j);
        }
      }
    } else if (rowin) {
      for (int ux = lo[0]; ux <= hi[0]; ux++) {
        double dx = box_d(0, ux);
        if (all || dx * dx + byz2 < R2v) {
          first = min(first, ux);
          last = max(last, ux);
        }
      }
    }
    if (row < nrows) {
      if (rowin) {
        const int Gx = J.G[0], Gy = J.G[1], Gz = J.G[2];
        my = uy < 0 ? -1 : (uy >= Gy ? 1 : 0);
        mz = uz < 0 ? -1 : (uz >= Gz ? 1 : 0);
        cy = uy - my * Gy, cz = uz - mz * Gz;
        const int64_t rowbase = (int64_t)Gx * (cy + (int64_t)Gy * cz);
        for (int mx = -1; mx <= 1; mx++) {
          int a = max(first, mx * Gx), b = min(last, mx * Gx + Gx - 1);
          if (a > b) continue;
          int c0 = a - mx * Gx, c1 = b - mx * Gx;
          if (DENSE && __ldg(J.dprefix + rowbase + c1 + 1) > __ldg(J.dprefix + rowbase + c0)) {
            dfr[mx + 1] = c0 | (c1 << 16);
            continue;
          }
          int32_t ps = __ldg(J.cell_start + rowbase + c0);
          int32_t pe = __ldg(J.cell_start + rowbase + c1 + 1);
          if (pe > ps) {
            const int code = (mx + 1) + 3 * (my + 1) + 9 * (mz + 1);
            if (nseg == 0) {
              s0a = ps, sla = pe - ps, sca = code;
            } else if (nseg == 1) {
              s0b = ps, slb = pe - ps, scb = code;
            } else {
              s0c = ps, slc = pe - ps, scc = code;
            }
            nseg++;
          }
        }
      }
    }
    int nsegs_total;
    const int segoff = warp_excl_scan(nseg, lane, &nsegs_total);
    const int mylen = sla + slb + slc;
    int total;
    const int lenoff = warp_excl_scan(mylen, lane, &total);
    if (nseg > 0) {
      B.sstart[segoff] = s0a, B.spref[segoff] = lenoff, B.scode[segoff] = (uint8_t)sca;
    }
    if (nseg > 1) {
      B.sstart[segoff + 1] = s0b, B.spref[segoff + 1] = lenoff + sla;
      B.scode[segoff + 1] = (uint8_t)scb;
    }
    if (nseg > 2) {
      B.sstart[segoff + 2] = s0c, B.spref[segoff + 2] = lenoff + sla + slb;
      B.scode[segoff + 2] = (uint8_t)scc;
    }
    __syncwarp();
    flush(nsegs_total, total);
    // the deferred ranges, cell by cell (a sparse cell is one segment)
    for (int im = 0; im < (DENSE ? 3 : 0); im++) {
      unsigned pend = __ballot_sync(FULL, dfr[im] >= 0);
      while (pend) {
        const int src = __ffs(pend) - 1;
        pend &= pend - 1;
        const int rg = __shfl_sync(FULL, dfr[im], src);
        const int ry = __shfl_sync(FULL, cy, src), rz = __shfl_sync(FULL, cz, src);
        const int rmy = __shfl_sync(FULL, my, src), rmz = __shfl_sync(FULL, mz, src);
        const int mx = im - 1;
        const int code = (mx + 1) + 3 * (rmy + 1) + 9 * (rmz + 1);
        const int64_t rowbase = (int64_t)J.G[0] * (ry + (int64_t)J.G[1] * rz);
        for (int c = rg & 0xffff; c <= (rg >> 16) && count <= stop; c++) {
          if (__ldg(J.cell_dense + rowbase + c)) {
            dense_cell(c, ry, rz, mx, rmy, rmz, code);
          } else {
            const int32_t ps = __ldg(J.cell_start + rowbase + c);
            const int32_t pe = __ldg(J.cell_start + rowbase + c + 1);
            emit1(ps, lane == 0 ? pe - ps : 0, code);
          }
        }
      }
    }
  }
  *exhausted = all && count <= stop && !__any_sync(FULL, beyond > 0);
  return count;
}

// gather_shell_impl without the dense-cell code when the build has no dense cell (the
// uniform-density case keeps its registers), with it otherwise.
// With CODE_ONLY, B.tie holds the shift code alone (no load of the original index per
// element); the caller completes it where the full order is needed.
template <int CMAX, bool BIG = false, bool CODE_ONLY = false>
__device__ __forceinline__ int gather_shell(const Job& J, ShellBuf<CMAX>& B, int lane, D3 x, double R,
                                            double lo2, const double* ext, bool* exhausted, int stop,
                                            char* big = nullptr) {
  return J.dprefix != nullptr
             ? gather_shell_impl<CMAX, BIG, true, CODE_ONLY>(J, B, lane, x, R, lo2, ext, exhausted, stop, big)
             : gather_shell_impl<CMAX, BIG, false, CODE_ONLY>(J, B, lane, x, R, lo2, ext, exhausted, stop, big);
}

// Bitonic sort of the shell [0, n) by (key, tie) ascending, carrying cpos; n <= CMAX.
template <int CMAX>
__device__ __noinline__ void sort_shell(ShellBuf<CMAX>& B, int lane, int n) {
  int np2 = 32;
  while (np2 < n) np2 <<= 1;
  for (int i = n + lane; i < np2; i += 32) {
    B.key[i] = ~0ull;
    B.tie[i] = ~0u;
    B.cpos[i] = 0;
  }
  __syncwarp();
  for (int k = 2; k <= np2; k <<= 1) {
    for (int jl = __ffs(k) - 2; jl >= 0; jl--) {
      const int j = 1 << jl;
      for (int i = lane; i < (np2 >> 1); i += 32) {
        const int lo = ((i >> jl) << (jl + 1)) | (i & (j - 1));
        const int hi = lo + j;
        const bool asc = (lo & k) == 0;
        const unsigned long long ka = B.key[lo], kb = B.key[hi];
        const uint32_t ta = B.tie[lo], tb = B.tie[hi];
        const bool gt = (ka > kb) || (ka == kb && ta > tb);
        if (gt == asc) {
          const int32_t pa = B.cpos[lo], pb = B.cpos[hi];
          B.key[lo] = kb;
          B.key[hi] = ka;
          B.tie[lo] = tb;
          B.tie[hi] = ta;
          B.cpos[lo] = pb;
          B.cpos[hi] = pa;
        }
      }
      __syncwarp();
    }
  }
}

// Bitonic sort of 32 * EPL shell entries held in registers, element i = lane + 32 e
// in slot e of every lane: exchanges across lanes (stride < 32) go through warp
// shuffles, exchanges inside a lane (stride >= 32) through registers, so the sort
// touches no shared memory.  Entries order by (key, tie); (key, tie) pairs are
// distinct except for the padding entries, which are identical.
template <int EPL>
__device__ __forceinline__ void sort_regs(unsigned long long (&key)[EPL], uint32_t (&tie)[EPL],
                                          int32_t (&pos)[EPL], int lane) {
#pragma unroll
  for (int k = 2; k <= 32 * EPL; k <<= 1) {
#pragma unroll
    for (int j = k >> 1; j > 0; j >>= 1) {
      if (j >= 32) {
#pragma unroll
        for (int e = 0; e < EPL; e++) {
          const int pe = e ^ (j >> 5);
          if (pe > e) {
            const bool asc = ((32 * e) & k) == 0;
            const bool gt = key[e] > key[pe] || (key[e] == key[pe] && tie[e] > tie[pe]);
            if (gt == asc) {
              const unsigned long long tk = key[e];
              const uint32_t tt = tie[e];
              const int32_t tp = pos[e];
              key[e] = key[pe], tie[e] = tie[pe], pos[e] = pos[pe];
              key[pe] = tk, tie[pe] = tt, pos[pe] = tp;
            }
          }
        }
      } else {
#pragma unroll
        for (int e = 0; e < EPL; e++) {
          const unsigned long long ok = __shfl_xor_sync(FULL, key[e], j);
          const uint32_t ot = __shfl_xor_sync(FULL, tie[e], j);
          const int32_t op = __shfl_xor_sync(FULL, pos[e], j);
          const bool asc = (((lane + 32 * e) & k) == 0);
          const bool lower = (lane & j) == 0;
          const bool gt = key[e] > ok || (key[e] == ok && tie[e] > ot);  // mine > other
          // the lower index of the pair keeps the smaller entry when ascending
          if (gt == (lower == asc)) key[e] = ok, tie[e] = ot, pos[e] = op;
        }
      }
    }
  }
}

// -------------------------------------------------------------------- ring --
// Replay of compute_boundary (convex_cell.rs:421-441) + SimpleCycle
// (simple_cycle.rs:17-78) for the removed vertices at positions [nvf, nv), with the
// whole warp: step i of the reference's loop takes the first removed vertex at or after
// position i whose dual triangle extends the cycle (failed try_extend calls change
// nothing), so one ballot over the candidates, 32 at a time, finds it; the rotation /
// case order of try_extend is kept per candidate.  The cycle's successor pointers end in S.rptr and its
// iteration order in (S.ea, S.eb); returns the edge count, -1 on failure, -2 when the
// ring exceeds the tier's vertex capacity.
template <class T, class SM>
__device__ __noinline__ int ring_replay_warp(SM& S, int lane, int nvf, int nv, int np) {
  using PIdx = typename T::PIdx;
  for (int i = lane; i < np; i += 32) S.rptr[i] = (PIdx)i;
  __syncwarp();
  const int s0 = S.ord[nvf];
  int start = S.vd0[s0];
  int len = 3;
  if (lane == 0) {
    const int a = S.vd0[s0], b = S.vd1[s0], c = S.vd2[s0];
    S.rptr[a] = (PIdx)b;
    S.rptr[b] = (PIdx)c;
    S.rptr[c] = (PIdx)a;
  }
  __syncwarp();
  const int n = nv - nvf;
  for (int i = 1; i < n; i++) {
    int found = -1, how = 0;
    for (int base = i; base < n && found < 0; base += 32) {
      const int idx = base + lane;
      int code = 0;  // 1 + 2 * rotation + case (0: grow the cycle, 1: absorb a node)
      if (idx < n) {
        const int sl = S.ord[nvf + idx];
        const int t[3] = {S.vd0[sl], S.vd1[sl], S.vd2[sl]};
        const bool in[3] = {S.rptr[t[0]] != (PIdx)t[0], S.rptr[t[1]] != (PIdx)t[1],
                            S.rptr[t[2]] != (PIdx)t[2]};
#pragma unroll
        for (int a = 0; a < 3; a++) {
          const int j = a == 2 ? 0 : a + 1, k = a == 0 ? 2 : a - 1;
          if (code == 0) {
            if (!in[a] && in[j] && in[k] && S.rptr[t[k]] == (PIdx)t[j])
              code = 1 + 2 * a;
            else if (in[a] && in[j] && in[k] && S.rptr[t[k]] == (PIdx)t[j] &&
                     S.rptr[t[j]] == (PIdx)t[a])
              code = 2 + 2 * a;
          }
        }
      }
      const unsigned bal = __ballot_sync(FULL, code != 0);
      if (bal) {
        const int src = __ffs(bal) - 1;
        found = base + src;
        how = __shfl_sync(FULL, code, src);
      }
    }
    if (found < 0) return -1;
    const int sl = S.ord[nvf + found];
    const int t[3] = {S.vd0[sl], S.vd1[sl], S.vd2[sl]};
    const int a = (how - 1) >> 1;
    const int ta = t[a], tb = t[a == 2 ? 0 : a + 1], tc = t[a == 0 ? 2 : a - 1];
    const bool grow = ((how - 1) & 1) == 0;
    __syncwarp();
    if (lane == 0) {
      S.rptr[tc] = (PIdx)ta;
      S.rptr[grow ? ta : tb] = (PIdx)tb;
      if (found > i) {
        const PIdx tmp = S.ord[nvf + i];
        S.ord[nvf + i] = S.ord[nvf + found];
        S.ord[nvf + found] = tmp;
      }
    }
    if (grow) {
      len += 1;
    } else {
      if (start == tb) start = ta;
      len -= 1;
    }
    __syncwarp();
  }
  if (len > T::VMAX) return -2;
  if (lane == 0) {
    int cur = start;
    for (int e = 0; e < len; e++) {
      const int nxt = S.rptr[cur];
      S.ea[e] = (PIdx)cur;
      S.eb[e] = (PIdx)nxt;
      cur = nxt;
    }
  }
  __syncwarp();
  return len;
}

// ring_replay_warp for at most 32 removed vertices with each triangle held by its lane:
// lane j starts with the triangle at position nvf + j and tracks the position the
// reference's swaps give it (the triangle at position i moves to the winner's position
// when step i takes a later one), so a step is a reduction of the positions of the
// triangles that extend the cycle rather than a scan of shared memory.  The removed
// vertices' order in `ord` is left as it was: only their slots are reused, and the
// vertices that replace them take ring order.  Returns as ring_replay_warp.
template <class T, class SM>
__device__ __noinline__ int ring_replay_lanes(SM& S, int lane, int nvf, int nv, int np) {
  using PIdx = typename T::PIdx;
  const int n = nv - nvf;
  if (n > 32) return ring_replay_warp<T>(S, lane, nvf, nv, np);
  for (int i = lane; i < np; i += 32) S.rptr[i] = (PIdx)i;
  int t[3] = {0, 0, 0};
  if (lane < n) {
    const int sl = S.ord[nvf + lane];
    t[0] = S.vd0[sl], t[1] = S.vd1[sl], t[2] = S.vd2[sl];
  }
  int pos = lane;
  bool open = lane > 0 && lane < n;  // not yet part of the cycle
  int start = __shfl_sync(FULL, t[0], 0);
  __syncwarp();
  if (lane == 0) {
    S.rptr[t[0]] = (PIdx)t[1];
    S.rptr[t[1]] = (PIdx)t[2];
    S.rptr[t[2]] = (PIdx)t[0];
  }
  __syncwarp();
  int len = 3;
  for (int i = 1; i < n; i++) {
    int code = 0;  // 1 + 2 * rotation + case (0: grow the cycle, 1: absorb a node)
    if (open) {
      const bool in[3] = {S.rptr[t[0]] != (PIdx)t[0], S.rptr[t[1]] != (PIdx)t[1],
                          S.rptr[t[2]] != (PIdx)t[2]};
#pragma unroll
      for (int a = 0; a < 3; a++) {
        const int j = a == 2 ? 0 : a + 1, k = a == 0 ? 2 : a - 1;
        if (code == 0) {
          if (!in[a] && in[j] && in[k] && S.rptr[t[k]] == (PIdx)t[j])
            code = 1 + 2 * a;
          else if (in[a] && in[j] && in[k] && S.rptr[t[k]] == (PIdx)t[j] && S.rptr[t[j]] == (PIdx)t[a])
            code = 2 + 2 * a;
        }
      }
    }
    const unsigned key = code ? (unsigned)pos : 64u;
    const unsigned m = __reduce_min_sync(FULL, key);
    if (m == 64u) return -1;
    const int w = __ffs(__ballot_sync(FULL, key == m)) - 1;
    const int how = __shfl_sync(FULL, code, w);
    const int a = (how - 1) >> 1;
    const int w0 = __shfl_sync(FULL, t[0], w), w1 = __shfl_sync(FULL, t[1], w),
              w2 = __shfl_sync(FULL, t[2], w);
    const int ta = a == 0 ? w0 : (a == 1 ? w1 : w2);
    const int tb = a == 0 ? w1 : (a == 1 ? w2 : w0);
    const int tc = a == 0 ? w2 : (a == 1 ? w0 : w1);
    const bool grow = ((how - 1) & 1) == 0;
    __syncwarp();
    if (lane == 0) {
      S.rptr[tc] = (PIdx)ta;
      S.rptr[grow ? ta : tb] = (PIdx)tb;
    }
    if (lane == w) open = false;
    else if (open && pos == i) pos = (int)m;  // swap(i, m) of compute_boundary
    if (grow) {
      len += 1;
    } else {
      if (start == tb) start = ta;
      len -= 1;
    }
    __syncwarp();
  }
  if (len > T::VMAX) return -2;
  if (lane == 0) {
    int cur = start;
    for (int e = 0; e < len; e++) {
      const int nxt = S.rptr[cur];
      S.ea[e] = (PIdx)cur;
      S.eb[e] = (PIdx)nxt;
      cur = nxt;
    }
  }
  __syncwarp();
  return len;
}

// Parallel ring: the boundary edges of the union of the removed dual triangles form
// the same cycle the serial algorithm builds; it starts at the first removed
// vertex's dual[0] whenever that node is still on the boundary.  Returns the edge
// count, or -1 when the serial replay must decide.
template <class T, class SM>
__device__ __forceinline__ int ring_parallel(SM& S, int lane, int nvf, int nv) {
  using PIdx = typename T::PIdx;
  const int r = nv - nvf;
  if (r > 32) return -1;  // large removal sets: the serial replay decides
  int t0 = 0, t1 = 0, t2 = 0;
  if (lane < r) {
    const int sl = S.ord[nvf + lane];
    t0 = S.vd0[sl], t1 = S.vd1[sl], t2 = S.vd2[sl];
    S.rptr[t0] = (PIdx)T::NONE;
    S.rptr[t1] = (PIdx)T::NONE;
    S.rptr[t2] = (PIdx)T::NONE;
  }
  __syncwarp();
  // an edge u->w of a removed triangle is on the boundary iff no other removed
  // triangle holds w->u
  bool b01 = lane < r, b12 = lane < r, b20 = lane < r;
  for (int k = 0; k < r; k++) {
    const int a = __shfl_sync(FULL, t0, k), b = __shfl_sync(FULL, t1, k),
              c = __shfl_sync(FULL, t2, k);
    if (k == lane) continue;
    b01 = b01 && !((a == t1 && b == t0) || (b == t1 && c == t0) || (c == t1 && a == t0));
    b12 = b12 && !((a == t2 && b == t1) || (b == t2 && c == t1) || (c == t2 && a == t1));
    b20 = b20 && !((a == t0 && b == t2) || (b == t0 && c == t2) || (c == t0 && a == t2));
  }
  if (b01) S.rptr[t0] = (PIdx)t1;
  if (b12) S.rptr[t1] = (PIdx)t2;
  if (b20) S.rptr[t2] = (PIdx)t0;
  __syncwarp();
  bool conflict = (b01 && S.rptr[t0] != (PIdx)t1) || (b12 && S.rptr[t1] != (PIdx)t2) ||
                  (b20 && S.rptr[t2] != (PIdx)t0);
  if (__any_sync(FULL, conflict)) return -1;
  const int E = __popc(__ballot_sync(FULL, b01)) + __popc(__ballot_sync(FULL, b12)) +
                __popc(__ballot_sync(FULL, b20));
  const int start = S.vd0[S.ord[nvf]];
  if (S.rptr[start] == (PIdx)T::NONE) return -1;
  if (E > T::VMAX) return -1;
  int ok = 1;
  if (lane == 0) {
    int cur = start;
    for (int e = 0; e < E; e++) {
      const int nxt = S.rptr[cur];
      if (nxt == (int)T::NONE || (e < E - 1 && nxt == start)) {
        ok = 0;
        break;
      }
      S.ea[e] = (PIdx)cur;
      S.eb[e] = (PIdx)nxt;
      cur = nxt;
    }
    if (ok && cur != start) ok = 0;
  }
  ok = __shfl_sync(FULL, ok, 0);
  __syncwarp();
  return ok ? E : -1;
}

// Parallel ring with ranked edges: as ring_parallel, but each boundary edge goes to
// its own lane, and its position in the SimpleCycle iteration order (starting at the
// first removed vertex's dual[0]) comes from pointer jumping over warp shuffles
// instead of a walk.  Lane e < E receives edge (*eu -> *ew) at ring position *erank.
// Returns E, or -1 when the serial replay must decide (the start node is interior,
// the edges do not form one cycle through it, or more than 32 edges).
//
// The boundary test uses S.plm, one 32-bit lane mask per plane (zero between calls):
// removed triangle `lane` sets its bit on its three planes.  The dual of a convex cell
// is a triangulated sphere, so an edge {u, w} belongs to exactly two triangles, with
// opposite orientations; edge u->w of a removed triangle is therefore interior (the
// other triangle, holding w->u, is removed as well) exactly when another removed
// triangle holds both u and w.
template <class T, class SM>
__device__ __forceinline__ int ring_ranked(SM& S, int lane, int nvf, int nv, int* eu, int* ew,
                                           int* erank) {
  using PIdx = typename T::PIdx;
  const int r = nv - nvf;
  if (r > 32) return -1;
  int t0 = 0, t1 = 0, t2 = 0;
  const unsigned me = 1u << lane;
  if (lane < r) {
    const int sl = S.ord[nvf + lane];
    t0 = S.vd0[sl], t1 = S.vd1[sl], t2 = S.vd2[sl];
    S.rptr[t0] = (PIdx)T::NONE;
    S.rptr[t1] = (PIdx)T::NONE;
    S.rptr[t2] = (PIdx)T::NONE;
    atomicOr(&S.plm[t0], me);
    atomicOr(&S.plm[t1], me);
    atomicOr(&S.plm[t2], me);
  }
  const int start = S.vd0[S.ord[nvf]];
  __syncwarp();
  bool b01 = false, b12 = false, b20 = false;
  if (lane < r) {
    const unsigned m0 = S.plm[t0] & ~me, m1 = S.plm[t1] & ~me, m2 = S.plm[t2] & ~me;
    b01 = (m0 & m1) == 0u;
    b12 = (m1 & m2) == 0u;
    b20 = (m2 & m0) == 0u;
  }
  __syncwarp();
  if (lane < r) S.plm[t0] = 0u, S.plm[t1] = 0u, S.plm[t2] = 0u;
  const unsigned m01 = __ballot_sync(FULL, b01), m12 = __ballot_sync(FULL, b12),
                 m20 = __ballot_sync(FULL, b20);
  const int n01 = __popc(m01), n12 = __popc(m12);
  const int E = n01 + n12 + __popc(m20);
  if (E > 32) return -1;
  // compact the edges: edge index by ballot rank; rptr maps a node to the edge leaving it
  const unsigned lt = lanemask_lt();
  const int p01 = __popc(m01 & lt), p12 = n01 + __popc(m12 & lt), p20 = n01 + n12 + __popc(m20 & lt);
  if (b01) S.ea[p01] = (PIdx)t0, S.eb[p01] = (PIdx)t1, S.rptr[t0] = (PIdx)p01;
  if (b12) S.ea[p12] = (PIdx)t1, S.eb[p12] = (PIdx)t2, S.rptr[t1] = (PIdx)p12;
  if (b20) S.ea[p20] = (PIdx)t2, S.eb[p20] = (PIdx)t0, S.rptr[t2] = (PIdx)p20;
  __syncwarp();
  int u = 0, w = 0, nx = lane, d = 0;
  bool broken = false;
  if (lane < E) {
    u = S.ea[lane], w = S.eb[lane];
    nx = S.rptr[w];
    d = 1;
    // two boundary edges leave u, or none leaves w
    broken = S.rptr[u] != (PIdx)lane || nx == (int)T::NONE;
  }
  const int se = S.rptr[start];
  __syncwarp();
  if (__any_sync(FULL, broken) || se == (int)T::NONE) return -1;
  // distance from each edge to the start edge along the cycle
  if (lane == se) nx = lane, d = 0;
  for (int span = 1; span < E; span <<= 1) {
    const int dn = __shfl_sync(FULL, d, nx);
    const int nn = __shfl_sync(FULL, nx, nx);
    d += dn;
    nx = nn;
  }
  if (__any_sync(FULL, lane < E && nx != se)) return -1;  // not one cycle through the start
  *eu = u;
  *ew = w;
  *erank = d == 0 ? 0 : E - d;
  return E;
}

// ------------------------------------------------------------ cell records --
// A finished cell as the staged integral kernel and the cell export read it, in words:
// header (np as int32; nv | flags as int32), safety radius, then for the stored planes
// pl in [pb, np): normals / offsets / generator projections (7 (np - pb) f64); the
// vertex locations in the reference's order (3 nv f64); the stored planes' right
// generators (int32); their shift codes and the vertex duals (bytes, the duals as
// plane indices).
//
// A compact record (the plain builds) leaves out the six boundary planes when no
// vertex lies on one of them (pb = 6): the integral step reads a plane only through a
// vertex dual.  A full record (export builds: the cell export reads every plane) keeps
// them (pb = 0).  Recomputing the vertex locations from their dual planes instead of
// storing them was measured slower (the integral kernel's three IEEE divisions per
// vertex cost more than the loads they save).
constexpr int REC_PB6 = 1 << 16;  // nv word flag: planes start at 6

__host__ __device__ __forceinline__ int64_t rec_words(int np, int nv, int pb = 0) {
  const int ps = np - pb;
  return 2 + 7 * (int64_t)ps + 3 * (int64_t)nv + (ps + 1) / 2 + (ps + 3 * nv + 7) / 8;
}

// Writes the cell held in shared memory (SM layout, see the top of this file, plus
// bisector_point(J, k, x), the HalfSpace point p of plane k) as a record (full or
// compact) at words allocated from *counter in rec[0, cap), and its offset to
// *off_slot.  Returns false when the buffer is full or a plane index does not fit the
// record's bytes.
template <class SM>
__device__ bool write_record(const Job& J, double* rec, int64_t cap, unsigned long long* counter,
                             int64_t* off_slot, const SM& S, int lane, D3 x, int np, int nv,
                             double sr, bool full) {
  if (np > 255) return false;
  int pb = 0;
  if (!full) {
    bool onb = false;
    for (int q = lane; q < nv; q += 32) {
      const int sl = S.ord[q];
      onb |= S.vd0[sl] < 6 || S.vd1[sl] < 6 || S.vd2[sl] < 6;
    }
    pb = __any_sync(FULL, onb) ? 0 : 6;
  }
  const int ps = np - pb;
  const int64_t words = rec_words(np, nv, pb);
  unsigned long long off = 0;
  if (lane == 0) off = atomicAdd(counter, (unsigned long long)words);
  off = __shfl_sync(FULL, off, 0);
  if ((int64_t)off + words > cap) return false;
  double* R = rec + off;
  if (lane == 0) {
    reinterpret_cast<int32_t*>(R)[0] = np;
    reinterpret_cast<int32_t*>(R)[1] = nv | (pb ? REC_PB6 : 0);
    R[1] = sr;
  }
  double* nx = R + 2;
  double *ny = nx + ps, *nz = ny + ps, *dd = nz + ps, *qx = dd + ps, *qy = qx + ps, *qz = qy + ps;
  double *vxo = qz + ps, *vyo = vxo + nv, *vzo = vyo + nv;
  int32_t* rt = reinterpret_cast<int32_t*>(vzo + nv);
  uint8_t* pc = reinterpret_cast<uint8_t*>(vzo + nv + (ps + 1) / 2);
  uint8_t *d0 = pc + ps, *d1 = d0 + nv, *d2 = d1 + nv;
  for (int k = lane; k < ps; k += 32) {
    const int pl = k + pb;
    const D3 nn = {S.pnx[pl], S.pny[pl], S.pnz[pl]};
    const D3 pr = plane_project(nn, S.bisector_point(J, pl, x), x);  // Plane::project_onto
    nx[k] = nn.x, ny[k] = nn.y, nz[k] = nn.z, dd[k] = S.pd[pl];
    qx[k] = pr.x, qy[k] = pr.y, qz[k] = pr.z;
    rt[k] = S.pright[pl];
    pc[k] = S.pcode[pl];
  }
  for (int q = lane; q < nv; q += 32) {
    const int sl = S.ord[q];
    vxo[q] = S.vx[sl], vyo[q] = S.vy[sl], vzo[q] = S.vz[sl];
    d0[q] = (uint8_t)S.vd0[sl], d1[q] = (uint8_t)S.vd1[sl], d2[q] = (uint8_t)S.vd2[sl];
  }
  if (lane == 0) *off_slot = (int64_t)off;
  __syncwarp();
  return true;
}

// The record at R as the integral step and the cell export read it.  Plane accessors
// take the plane index pl (>= pb).
struct RecordView {
  const double *nx, *ny, *nz, *dd, *qx, *qy, *qz, *vx, *vy, *vz;
  const int32_t* rt;
  const uint8_t *pc, *d0, *d1, *d2;
  int np, nv, pb;
  double sr;
  __device__ explicit RecordView(const double* R) {
    np = __ldg(reinterpret_cast<const int32_t*>(R));
    const int w = __ldg(reinterpret_cast<const int32_t*>(R) + 1);
    nv = w & 0xffff;
    pb = (w & REC_PB6) ? 6 : 0;
    sr = __ldg(R + 1);
    const int ps = np - pb;
    // plane arrays indexed by pl - pb
    nx = R + 2, ny = nx + ps, nz = ny + ps, dd = nz + ps;
    qx = dd + ps, qy = qx + ps, qz = qy + ps;
    vx = qz + ps, vy = vx + nv, vz = vy + nv;
    rt = reinterpret_cast<const int32_t*>(vz + nv);
    pc = reinterpret_cast<const uint8_t*>(vz + nv + (ps + 1) / 2);
    d0 = pc + ps, d1 = d0 + nv, d2 = d1 + nv;
  }
  __device__ D3 normal(int pl) const {
    const int k = pl - pb;
    return {__ldg(nx + k), __ldg(ny + k), __ldg(nz + k)};
  }
  __device__ double d(int pl) const { return __ldg(dd + pl - pb); }
  __device__ D3 proj(int pl) const {
    const int k = pl - pb;
    return {__ldg(qx + k), __ldg(qy + k), __ldg(qz + k)};
  }
  __device__ int right(int pl) const { return __ldg(rt + pl - pb); }
  __device__ int code(int pl) const { return __ldg(pc + pl - pb); }
  __device__ int dual(int q, int i) const {
    return i == 0 ? __ldg(d0 + q) : (i == 1 ? __ldg(d1 + q) : __ldg(d2 + q));
  }
  __device__ D3 loc(int q) const { return {__ldg(vx + q), __ldg(vy + q), __ldg(vz + q)}; }
};

// Projection of x on the line of planes dual[i] & dual[i+1] of vertex q:
// project_onto_intersection (geometry.rs:41-47) of plane dual[(i+1)%3] with dual[i].
template <class View>
__device__ __forceinline__ bool line_projection(const View& V, int q, int i, D3 x, D3* out) {
  const int cur = V.dual(q, i);
  const int nx = V.dual(q, i == 2 ? 0 : i + 1);
  const D3 cn = V.normal(cur);
  const D3 nn = V.normal(nx);
  const D3 perp = cross(nn, cn);
  return intersect3(nn, V.d(nx), cn, V.d(cur), perp, dot(x, perp), out);
}

// --------------------------------------------------------------- integrals --
// Scratch of the integral step: projections on the plane-pair lines of STEP vertices
// and their 6 STEP tets' values (rows 16-byte aligned, read two tets at a time, and
// padded by 6 values so that lanes reading different rows at the same column hit
// different banks).
// With PM > 0, pm[pl] collects per step the (vertex, dual slot) pairs of plane pl as
// bits 3 vl + i (zero between steps), so that a face sums only its own tets.
template <int STEP = 5, int PM = 0>
struct TetScratch {
  static constexpr int NT = 6 * STEP;
  double ix[3 * STEP], iy[3 * STEP], iz[3 * STEP];
  alignas(16) double val[8][NT + 6];
  uint32_t pm[PM > 0 ? PM : 1];
};

// Integrals and face emission of a finished cell (convex_cell.rs:131-187,
// voronoi_cell.rs:40-100) over a view V of the cell: V.normal(pl), V.d(pl),
// V.proj(pl) (the generator projected on plane pl), V.right(pl), V.code(pl),
// V.dual(q, i) and V.loc(q) for vertex position q in the reference's order.  Each
// step of STEP vertices (STEP <= 10) projects on their 3 STEP plane-pair lines (one
// per lane), builds their 6 STEP tets and accumulates them in the reference's tet
// order: lanes 0-3 the cell integrals, lane p (and p + 32k) the integrals of face p.
template <class T, int STEP, int PM, class View>
__device__ __forceinline__ int integrate_view(const Job& J, const View& V, TetScratch<STEP, PM>& Sc,
                                              int lane, int self, D3 x, int nv, int np, double sr,
                                              int* err_code) {
  static_assert(3 * STEP <= 32, "one projection per lane");
  const int dim = J.dim;
  double cacc = 0.0;  // lanes 0..3: volume, centroid x, y, z
  double fa[T::PMAX / 32], fcx[T::PMAX / 32], fcy[T::PMAX / 32], fcz[T::PMAX / 32];
  unsigned ftouched = 0;
#pragma unroll
  for (int k = 0; k < T::PMAX / 32; k++) fa[k] = 0.0, fcx[k] = 0.0, fcy[k] = 0.0, fcz[k] = 0.0;
  for (int base = 0; base < nv; base += STEP) {
    const int nstep = min(STEP, nv - base);
    // projections on the lines dual[i] & dual[i+1]: project_onto_intersection
    // (geometry.rs:41-47) of plane dual[(i+1)%3] with dual[i]
    bool ok = true;
    if (lane < 3 * nstep) {
      const int vl = lane / 3, i = lane - 3 * vl;
      D3 pr = {0.0, 0.0, 0.0};
      ok = line_projection(V, base + vl, i, x, &pr);
      Sc.ix[lane] = pr.x;
      Sc.iy[lane] = pr.y;
      Sc.iz[lane] = pr.z;
    }
    if (__any_sync(FULL, !ok)) {
      *err_code = MV_ERR_DET;
      return CELL_ERROR;
    }
    if constexpr (PM >= T::PMAX) {
      if (lane < nstep) {
        const int q = base + lane;
        atomicOr(&Sc.pm[V.dual(q, 0)], 1u << (3 * lane));
        atomicOr(&Sc.pm[V.dual(q, 1)], 1u << (3 * lane + 1));
        atomicOr(&Sc.pm[V.dual(q, 2)], 1u << (3 * lane + 2));
      }
    }
    __syncwarp();
    // DecompositionWithoutFaces: tet t of a vertex = (proj[t], proj[(t+5)%6], vertex)
    // with proj[2i] on plane dual[i] and proj[2i+1] on the line (dual[i+1], dual[i])
    for (int tt = lane; tt < 6 * nstep; tt += 32) {
      const int vl = tt / 6, t = tt - 6 * vl;
      const int q = base + vl;
      auto proj = [&](int qq) -> D3 {
        const int i = qq >> 1;
        if (qq & 1) return D3{Sc.ix[3 * vl + i], Sc.iy[3 * vl + i], Sc.iz[3 * vl + i]};
        return V.proj(V.dual(q, i));
      };
      const D3 v0 = proj(t), v1 = proj(t == 0 ? 5 : t - 1);
      const D3 vloc = V.loc(q);
      const double vol = signed_volume_tet(v0, v1, vloc, x);
      const D3 vc = scale(vol, add(add(add(v0, v1), vloc), x));
      const double ar = signed_area_tri(v0, v1, vloc, x);
      const D3 ac = scale(ar, add(add(v0, v1), vloc));
      Sc.val[0][tt] = vol;
      Sc.val[1][tt] = vc.x;
      Sc.val[2][tt] = vc.y;
      Sc.val[3][tt] = vc.z;
      Sc.val[4][tt] = ar;
      Sc.val[5][tt] = ac.x;
      Sc.val[6][tt] = ac.y;
      Sc.val[7][tt] = ac.z;
    }
    __syncwarp();
    const int ntet = 6 * nstep;
    if (lane < 4) {
      for (int s = 0; s < ntet; s += 2) {  // ntet is even
        const double2 v = *reinterpret_cast<const double2*>(&Sc.val[lane][s]);
        cacc = cacc + v.x;
        cacc = cacc + v.y;
      }
    }
    if constexpr (PM >= T::PMAX) {
      // face pl: its vertices of this step in vertex order (ascending bits)
#pragma unroll
      for (int k = 0; k < T::PMAX / 32; k++) {
        const int pl = lane + 32 * k;
        unsigned m = 0u;
        if (pl < np) {
          m = Sc.pm[pl];
          if (m) Sc.pm[pl] = 0u;
        }
        if (m) ftouched |= 1u << k;
        while (m) {
          const int b = __ffs(m) - 1;
          m &= m - 1u;
          const int vl = (b * 11) >> 5;  // b / 3 for b < 32
          const int s = 6 * vl + 2 * (b - 3 * vl);
          const double2 a2 = *reinterpret_cast<const double2*>(&Sc.val[4][s]);
          const double2 x2 = *reinterpret_cast<const double2*>(&Sc.val[5][s]);
          const double2 y2 = *reinterpret_cast<const double2*>(&Sc.val[6][s]);
          const double2 z2 = *reinterpret_cast<const double2*>(&Sc.val[7][s]);
          fa[k] = fa[k] + a2.x;
          fcx[k] = fcx[k] + x2.x;
          fcy[k] = fcy[k] + y2.x;
          fcz[k] = fcz[k] + z2.x;
          fa[k] = fa[k] + a2.y;
          fcx[k] = fcx[k] + x2.y;
          fcy[k] = fcy[k] + y2.y;
          fcz[k] = fcz[k] + z2.y;
        }
      }
    } else {
#pragma unroll
      for (int k = 0; k < T::PMAX / 32; k++) {
        const int pl = lane + 32 * k;
        if (pl < np) {
          for (int vl = 0; vl < nstep; vl++) {
            const int q = base + vl;
            const int kk = V.dual(q, 0) == pl ? 0 : (V.dual(q, 1) == pl ? 1 : (V.dual(q, 2) == pl ? 2 : -1));
            if (kk >= 0) {
              const int s = 6 * vl + 2 * kk;
              fa[k] = fa[k] + Sc.val[4][s];
              fcx[k] = fcx[k] + Sc.val[5][s];
              fcy[k] = fcy[k] + Sc.val[6][s];
              fcz[k] = fcz[k] + Sc.val[7][s];
              fa[k] = fa[k] + Sc.val[4][s + 1];
              fcx[k] = fcx[k] + Sc.val[5][s + 1];
              fcy[k] = fcy[k] + Sc.val[6][s + 1];
              fcz[k] = fcz[k] + Sc.val[7][s + 1];
              ftouched |= 1u << k;
            }
          }
        }
      }
    }
    __syncwarp();
  }
  // cell: VolumeCentroidIntegral::finalize (integrals.rs:97-105)
  const double vol = __shfl_sync(FULL, cacc, 0);
  const double nrm = vol > 0.0 ? 0.25 / vol : 0.0;
  if (lane < 4 && lane > 0) J.centroid[3 * (int64_t)self + (lane - 1)] = cacc * nrm;
  if (lane == 0) {
    J.volume[self] = vol;
    J.safety_radius[self] = sr;
  }
  // faces: ownership (voronoi_cell.rs:414-434) and emission in plane order
  unsigned emit = 0;
  int nf_mine = 0;
#pragma unroll
  for (int k = 0; k < T::PMAX / 32; k++) {
    const int pl = lane + 32 * k;
    bool e = false;
    if (pl < np && ((ftouched >> k) & 1u)) {
      const D3 nn = V.normal(pl);
      e = vector_is_valid(dim, nn);
      const int r = V.right(pl);
      if (e && J.face_mode == MV_FACES_OWNED && r >= 0 && V.code(pl) == 13)
        e = r > self || (J.mask != nullptr && J.mask[r] == 0);
    }
    emit |= (unsigned)e << k;
    nf_mine += e;
  }
  const int nf = __reduce_add_sync(FULL, (unsigned)nf_mine);
  unsigned long long base = 0;
  if (lane == 0) base = atomicAdd(J.face_counter, (unsigned long long)nf);
  base = __shfl_sync(FULL, base, 0);
  if ((long long)(base + nf) > J.face_cap) return CELL_FACE_OVERFLOW;  // host grows staging, reruns
  if (lane == 0) {
    J.face_count[self] = nf;
    J.stage_off[self] = (int64_t)base;
  }
  int rank_base = 0;
#pragma unroll
  for (int k = 0; k < T::PMAX / 32; k++) {
    const bool ek = (emit >> k) & 1u;
    const unsigned bal = __ballot_sync(FULL, ek);
    if (ek) {
      const int pl = lane + 32 * k;
      const int64_t f = (int64_t)base + rank_base + __popc(bal & lanemask_lt());
      const double na = fa[k] > 0.0 ? 1.0 / (3.0 * fa[k]) : 0.0;
      const D3 nn = V.normal(pl);
      J.f_left[f] = self + J.id_base;
      J.f_right[f] = V.right(pl);
      J.f_area[f] = fa[k];
      J.f_centroid[3 * f] = fcx[k] * na;
      J.f_centroid[3 * f + 1] = fcy[k] * na;
      J.f_centroid[3 * f + 2] = fcz[k] * na;
      J.f_normal[3 * f] = nn.x;
      J.f_normal[3 * f + 1] = nn.y;
      J.f_normal[3 * f + 2] = nn.z;
      J.f_code[f] = (uint8_t)V.code(pl);
    }
    rank_base += __popc(bal);
  }
  return CELL_DONE;
}

}  // namespace mv
