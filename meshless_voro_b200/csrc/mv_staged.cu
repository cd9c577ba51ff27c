// mv_staged.cu -- the staged cell pipeline: shell, clip and integral kernels.
//
// The same per-cell construction as the fused kernel (mv_cells.cu), split in three
// kernels over a chunk of cells so that each kernel keeps a small instruction
// footprint and its own occupancy:
//   1. shell_kernel gathers each cell's first neighbour shell (rtree_nn.rs:10-240
//      up to the initial radius) and writes it sorted to a candidate list;
//   2. clip_kernel runs ConvexCell::build (convex_cell.rs:316-356) over the list and
//      writes the finished cell (planes, vertices in the reference's order) to a
//      record;
//   3. integrate_kernel evaluates the integrals and emits the faces
//      (voronoi_cell.rs:40-100) from the record.
// A cell whose list does not decide it (the stream continues past the first shell,
// or the shell overflowed) goes to a retry list that the fused kernel builds from
// scratch afterwards, so every cell still sees the reference's full neighbour stream.
//
// Filtered clipping keeps 32 consecutive candidates in the warp, one per lane, with
// the division-free f32 test of the fused kernel.  A candidate is certified not to
// remove vertex v when s32(c, v) > T(c); a certificate depends only on the pair, so
// after a clip only the new vertices are tested against the waiting candidates and
// the next candidate needing the f64 plane is one ballot away.
#include <cfloat>
#include <cstdint>

#include "mv_cell_common.cuh"

namespace mv {

#ifndef MV_CLIP_MINB
#define MV_CLIP_MINB 7
#endif
#ifndef MV_CLIP_WARPS
#define MV_CLIP_WARPS 4
#endif
constexpr int SHELL_CMAX = 128;
constexpr int SHELL_MIN = 64;  // first shells below this many candidates are widened
constexpr int SHELL_WARPS = 4;
#ifndef MV_SHELL_MINB
#define MV_SHELL_MINB 8
#endif
constexpr int CLIP_WARPS = MV_CLIP_WARPS;
constexpr int INT_WARPS = 4;
#ifndef MV_INT_STEP
#define MV_INT_STEP 10
#endif
constexpr int INT_STEP = MV_INT_STEP;  // vertices per step of the integral kernel
#ifndef MV_INT_MINB
#define MV_INT_MINB 7
#endif
using TierClip = Tier<64, 64, SHELL_CMAX, 8, uint8_t, MV_CLIP_MINB>;

// sorted position of processing item `item` of a chunk
__device__ __forceinline__ int stage_pos(const StageJob& SJ, int item) {
  return SJ.order != nullptr ? __ldg(SJ.order + SJ.item0 + item) : SJ.item0 + item;
}

// ------------------------------------------------------------------- shell --
// Bitonic sort of 32 * EPL entries in registers (element i = lane + 32 e in slot e of
// every lane) by a 32-bit key alone, carrying the list word; as sort_regs.
template <int EPL>
__device__ __forceinline__ void sort_regs_key(uint32_t (&key)[EPL], uint32_t (&val)[EPL], int lane) {
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
            if ((key[e] > key[pe]) == asc) {
              const uint32_t tk = key[e];
              const uint32_t tv = val[e];
              key[e] = key[pe], val[e] = val[pe];
              key[pe] = tk, val[pe] = tv;
            }
          }
        }
      } else {
#pragma unroll
        for (int e = 0; e < EPL; e++) {
          const uint32_t ok = __shfl_xor_sync(FULL, key[e], j);
          const uint32_t ov = __shfl_xor_sync(FULL, val[e], j);
          const bool asc = (((lane + 32 * e) & k) == 0);
          const bool lower = (lane & j) == 0;
          if ((key[e] > ok) == (lower == asc)) key[e] = ok, val[e] = ov;
        }
      }
    }
  }
}

// Sorts the gathered shell (cnt <= 32 EPL entries; B.tie holds the shift codes) in
// registers and writes it as sorted position * 27 + shift code; returns whether the
// nearest entry is the generator itself (sorted position spos, no shift).  The entries are sorted by their
// squared distance rounded down to f32 (a monotone map, so distinct keys order the
// entries as their squared distances do); only when two keys are equal (distances
// within an f32 ulp, or equal as in lattice-like inputs) is the shell sorted again by
// (squared distance, original index, shift code), the stream's full order.
template <int EPL>
__device__ __forceinline__ bool sort_and_write(const Job& J, const ShellBuf<SHELL_CMAX>& B, int lane,
                                               int cnt, int self, int spos, uint32_t* out) {
  uint32_t key[EPL];
  uint32_t val[EPL];
#pragma unroll
  for (int e = 0; e < EPL; e++) {
    const int i = lane + 32 * e;
    // d2 >= 0 is finite: its f32 bit pattern orders as the value, below the padding
    key[e] = i < cnt ? __float_as_uint(__double2float_rd(__longlong_as_double((long long)B.key[i])))
                     : ~0u;
    val[e] = i < cnt ? (uint32_t)B.cpos[i] * 27u + B.tie[i] : 0u;
  }
  sort_regs_key<EPL>(key, val, lane);
  // equal keys end next to each other: element i against i + 1
  bool dup = false;
#pragma unroll
  for (int e = 0; e < EPL; e++) {
    const uint32_t nx = __shfl_down_sync(FULL, key[e], 1);
    const uint32_t wrap = __shfl_sync(FULL, key[e + 1 < EPL ? e + 1 : e], 0);
    const uint32_t next = lane < 31 ? nx : wrap;
    const int i = lane + 32 * e;
    dup |= (i + 1 < cnt) && (lane < 31 || e + 1 < EPL) && key[e] == next;
  }
  if (__any_sync(FULL, dup)) {
    unsigned long long dkey[EPL];
    uint32_t tie[EPL];
    int32_t pos[EPL];
#pragma unroll
    for (int e = 0; e < EPL; e++) {
      const int i = lane + 32 * e;
      dkey[e] = i < cnt ? B.key[i] : ~0ull;
      tie[e] = i < cnt ? (uint32_t)__ldg(J.sid + B.cpos[i]) * 27u + B.tie[i] : ~0u;
      pos[e] = i < cnt ? B.cpos[i] : 0;
    }
    sort_regs<EPL>(dkey, tie, pos, lane);
#pragma unroll
    for (int e = 0; e < EPL; e++) {
      const int i = lane + 32 * e;
      if (i < cnt) out[i] = (uint32_t)pos[e] * 27u + tie[e] % 27u;
    }
    return (int)(__shfl_sync(FULL, tie[0], 0) / 27u) == self;
  }
#pragma unroll
  for (int e = 0; e < EPL; e++) {
    const int i = lane + 32 * e;
    if (i < cnt) out[i] = val[e];
  }
  return __shfl_sync(FULL, val[0], 0) == (uint32_t)spos * 27u + 13u;
}

template <int WARPS, bool MULTI>
__global__ void __launch_bounds__(32 * WARPS, MV_SHELL_MINB)
    shell_kernel(const __grid_constant__ Job J0, const __grid_constant__ StageJob SJ,
                 const __grid_constant__ JobTable TB) {
  __shared__ ShellBuf<SHELL_CMAX> bufs[WARPS];
  __shared__ double ext_s[6];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  ShellBuf<SHELL_CMAX>& B = bufs[warp];
  if (threadIdx.x < 6) ext_s[threadIdx.x] = J0.ext[threadIdx.x];
  __syncthreads();
  for (;;) {
    int item = 0;
    if (lane == 0) item = (int)atomicAdd(SJ.work + 0, 1u);
    item = __shfl_sync(FULL, item, 0);
    if (item >= SJ.nitems) break;
    const int gpos = stage_pos(SJ, item);
    // the cell's tessellation (batch builds): its Job and its local position
    const int jb = MULTI ? job_of(TB, gpos) : 0;
    const Job& J = MULTI ? TB.jobs[jb] : J0;
    const int spos = MULTI ? gpos - __ldg(TB.pos_base + jb) : gpos;
    const double* ext = MULTI ? J.ext : ext_s;
    const int self = __ldg(J.sid + spos);
    if (J.mask != nullptr && J.mask[self] == 0) {
      if (lane == 0) SJ.info[item] = 0;
      continue;
    }
    const D3 x = load_gen(J, self);
    bool all = false;
    double R = first_radius(J, x, lane);
    int cnt = gather_shell<SHELL_CMAX, false, true>(J, B, lane, x, R, 0.0, ext, &all, 32 * SHELL_CMAX);
    // the density estimate behind R is rough where the density varies: a shell that
    // overflows the list is pulled in, one far below a uniform region's ~92 candidates
    // (too small to close most cells) is widened, a few times at most
    for (int it = 0; it < 6; it++) {
      double f;
      if (cnt > SHELL_CMAX)
        f = fmin(fmax(cbrt(0.6 * SHELL_CMAX / (double)cnt), 0.1), 0.9);
      else if (cnt < SHELL_MIN && !all)
        f = fmin(cbrt(96.0 / (double)max(cnt, 1)), 2.0);
      else
        break;
      R *= f;
      cnt = gather_shell<SHELL_CMAX, false, true>(J, B, lane, x, R, 0.0, ext, &all, 32 * SHELL_CMAX);
    }
    if (cnt > SHELL_CMAX || cnt == 0) {
      if (lane == 0) SJ.info[item] = -1;
      continue;
    }
    uint32_t* out = SJ.cand + (int64_t)item * SJ.cstride;
    bool self_first;
    if (cnt <= 32)
      self_first = sort_and_write<1>(J, B, lane, cnt, self, spos, out);
    else if (cnt <= 64)
      self_first = sort_and_write<2>(J, B, lane, cnt, self, spos, out);
    else
      self_first = sort_and_write<4>(J, B, lane, cnt, self, spos, out);
    // the first neighbour must be the generator itself (convex_cell.rs:325-329); the
    // fused kernel reports the error otherwise
    if (lane == 0) {
      SJ.info[item] = self_first ? (cnt | (all ? (1 << 30) : 0)) : -1;
      SJ.rad[item] = R;
    }
    __syncwarp();
  }
}

// The wide round: cells the first round could not close get a shell of up to WIDE_CMAX
// candidates (about eight times the first one), sorted in shared memory.  Cells the
// wide round cannot close either go to the fused kernel.
constexpr int WIDE_CMAX = 1024;
constexpr int WIDE_MIN = 384;
constexpr int WIDE_WARPS = 4;
constexpr size_t WIDE_SMEM = sizeof(ShellBuf<WIDE_CMAX>) * WIDE_WARPS;

// Sorts the wide shell [0, n) by the squared distance rounded down to f32 (as
// sort_and_write) in place of B.key: each key becomes that 32-bit key above the
// entry's index, so one 64-bit word is compared and moved per entry.  Returns false
// when two keys are equal (the order then needs the full (key, tie) sort, over the
// original keys, which this overwrote).
template <int CMAX>
__device__ __noinline__ bool sort_shell_key32(ShellBuf<CMAX>& B, int lane, int n) {
  int np2 = 32;
  while (np2 < n) np2 <<= 1;
  for (int i = lane; i < np2; i += 32) {
    unsigned long long w = ~0ull;
    if (i < n) {
      const float k = __double2float_rd(__longlong_as_double((long long)B.key[i]));
      w = ((unsigned long long)__float_as_uint(k) << 32) | (unsigned)i;
    }
    B.key[i] = w;
  }
  __syncwarp();
  for (int k = 2; k <= np2; k <<= 1) {
    for (int jl = __ffs(k) - 2; jl >= 0; jl--) {
      const int j = 1 << jl;
      for (int i = lane; i < (np2 >> 1); i += 32) {
        const int lo = ((i >> jl) << (jl + 1)) | (i & (j - 1));
        const int hi = lo + j;
        const unsigned long long ka = B.key[lo], kb = B.key[hi];
        if ((ka > kb) == ((lo & k) == 0)) B.key[lo] = kb, B.key[hi] = ka;
      }
      __syncwarp();
    }
  }
  bool dup = false;
  for (int i = lane; i + 1 < n; i += 32) dup |= (B.key[i] >> 32) == (B.key[i + 1] >> 32);
  return !__any_sync(FULL, dup);
}

template <int WARPS, bool MULTI>
__global__ void __launch_bounds__(32 * WARPS, 3)
    shell_wide_kernel(const __grid_constant__ Job J0, const __grid_constant__ StageJob SJ,
                      const __grid_constant__ JobTable TB) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ double ext_s[6];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  ShellBuf<WIDE_CMAX>& B = reinterpret_cast<ShellBuf<WIDE_CMAX>*>(smem_raw)[warp];
  if (threadIdx.x < 6) ext_s[threadIdx.x] = J0.ext[threadIdx.x];
  __syncthreads();
  for (;;) {
    int item = 0;
    if (lane == 0) item = (int)atomicAdd(SJ.work + 0, 1u);
    item = __shfl_sync(FULL, item, 0);
    if (item >= SJ.nitems) break;
    const int gpos = stage_pos(SJ, item);
    // the cell's tessellation (batch builds): its Job and its local position
    const int jb = MULTI ? job_of(TB, gpos) : 0;
    const Job& J = MULTI ? TB.jobs[jb] : J0;
    const int spos = MULTI ? gpos - __ldg(TB.pos_base + jb) : gpos;
    const double* ext = MULTI ? J.ext : ext_s;
    const int self = __ldg(J.sid + spos);
    if (J.mask != nullptr && J.mask[self] == 0) {
      if (lane == 0) SJ.info[item] = 0;
      continue;
    }
    const D3 x = load_gen(J, self);
    bool all = false;
    double R = 2.0 * first_radius(J, x, lane);
    int cnt = gather_shell<WIDE_CMAX>(J, B, lane, x, R, 0.0, ext, &all, 4 * WIDE_CMAX);
    for (int it = 0; it < 6; it++) {
      double f;
      if (cnt > WIDE_CMAX)
        f = fmin(fmax(cbrt(0.6 * WIDE_CMAX / (double)cnt), 0.1), 0.9);
      else if (cnt < WIDE_MIN && !all)
        f = fmin(cbrt(0.75 * WIDE_CMAX / (double)max(cnt, 1)), 2.0);
      else
        break;
      R *= f;
      cnt = gather_shell<WIDE_CMAX>(J, B, lane, x, R, 0.0, ext, &all, 4 * WIDE_CMAX);
    }
    if (cnt > WIDE_CMAX || cnt == 0) {
      if (lane == 0) SJ.info[item] = -1;
      continue;
    }
    uint32_t* out = SJ.cand + (int64_t)item * SJ.cstride;
    uint32_t first;  // the nearest entry's tie (original index * 27 + shift code)
    if (sort_shell_key32<WIDE_CMAX>(B, lane, cnt)) {
      for (int i = lane; i < cnt; i += 32) {
        const int e = (int)(uint32_t)B.key[i];
        out[i] = (uint32_t)B.cpos[e] * 27u + B.tie[e] % 27u;
      }
      first = B.tie[(uint32_t)B.key[0]];
    } else {
      // equal keys: the same shell again (the gather is deterministic), fully sorted
      cnt = gather_shell<WIDE_CMAX>(J, B, lane, x, R, 0.0, ext, &all, 4 * WIDE_CMAX);
      sort_shell<WIDE_CMAX>(B, lane, cnt);
      for (int i = lane; i < cnt; i += 32) out[i] = (uint32_t)B.cpos[i] * 27u + B.tie[i] % 27u;
      first = B.tie[0];
    }
    if (lane == 0) {
      const bool self_first = (int)(first / 27u) == self;
      SJ.info[item] = self_first ? (cnt | (all ? (1 << 30) : 0)) : -1;
      SJ.rad[item] = R;
    }
    __syncwarp();
  }
}

// -------------------------------------------------------------------- clip --
template <class T>
struct ClipSmem {
  using PIdx = typename T::PIdx;
  // clipping planes (half_space.rs:9-19); planes 0-5 are the boundary, the others
  // bisectors whose point p = (x + ngb) / 2 is recomputed from the right generator
  // (one f64 of padding after each coordinate array: the three lanes of a new vertex
  // read and write the same index of all three arrays, now in different banks)
  double pnx[T::PMAX], pad_nx, pny[T::PMAX], pad_ny, pnz[T::PMAX], pd[T::PMAX];
  int32_t pright[T::PMAX];  // original index of the right generator, -1: boundary
  uint8_t pcode[T::PMAX];   // periodic shift code, 13: none
  PIdx rptr[T::PMAX];       // ring successor (SimpleCycle::ptrs)
  // vertices (convex_cell.rs:16-25) in fixed slots
  double vx[T::VMAX], pad_vx, vy[T::VMAX], pad_vy, vz[T::VMAX];
  float4 f4[T::VMAX];  // f32 (v - x) for the filter
  uint32_t plm[T::PMAX];  // ring_ranked: lanes whose removed triangle holds the plane
  alignas(4) PIdx ord[T::VMAX];   // position -> slot; [0, nv) is the reference's order
  PIdx vd0[T::VMAX], vd1[T::VMAX], vd2[T::VMAX];
  PIdx ea[T::VMAX], eb[T::VMAX];  // ring edges in SimpleCycle iteration order
  // the window: 32 consecutive candidates of the list with their half-spaces as the
  // reference sets them up (HalfSpace::new: normal, offset d = n.p, error bound errb),
  // plus the f32 operands and bound coefficients of the filter
  double wnx[32], wny[32], wnz[32], wd[32], werr[32];
  float4 wf[32];  // filter operands: e = x - ngb in f32, |e|^2 / 2
  float2 wc[32];  // bound coefficients (c0, c1)
  uint32_t wpk[32];  // original index * 27 + shift code
  __device__ D3 plane_point(const Job& J, int k) const { return {J.bp[k][0], J.bp[k][1], J.bp[k][2]}; }
  // coordinate c (0: x, 1: y, 2: z) arrays of the plane normals and vertex locations
  __device__ const double* pn(int c) const { return c == 0 ? pnx : (c == 1 ? pny : pnz); }
  __device__ double* vc(int c) { return c == 0 ? vx : (c == 1 ? vy : vz); }
  // HalfSpace::p of plane k: the boundary point, or (x + ngb) / 2 recomputed as at the clip
  __device__ D3 bisector_point(const Job& J, int k, D3 x) const {
    const int rr = pright[k];
    if (rr < 0) return plane_point(J, k);
    D3 ngb = load_gen(J, rr);
    const int code = pcode[k];
    if (code != 13) ngb = add(ngb, D3{J.shift[code][0], J.shift[code][1], J.shift[code][2]});
    return scale(0.5, add(x, ngb));
  }
};

// Event counts of one clipped cell in warp-uniform registers: a = neighbours (16
// bits) | planes (8) | serial rings (8), b = f32-undecided tests, e = exact tests (all
// of them box-corner zeros).  A cell of the clip tier consumes at most 1023 neighbours
// and holds at most 64 planes and 64 vertices, so no field of a overflows.
struct ClipCount {
  unsigned a, b, e;
  __device__ void neighbours(unsigned v) { a += v; }
  __device__ void plane() { a += 1u << 16; }
  __device__ void serial_ring() { a += 1u << 24; }
  __device__ void undecided(unsigned v) { b += v; }
  __device__ void exact(unsigned v) { e += v; }
};

// Vertex::from_dual (convex_cell.rs:38-42) for the ring's E new vertices, three lanes
// per vertex: lane 3e + c computes coordinate c of intersect_planes (geometry.rs:68-76)
// of the planes (u, w, p_idx) of edge e, with the operations the whole-vector form
// performs for that coordinate (((d0 (n1 x n2)_c + d1 (n2 x n0)_c) + d2 (n0 x n1)_c) /
// det, det = n2 . (n0 x n1) on each of the three lanes), so every coordinate is the
// same binary64 number.  Lane e < E holds edge e in (eu, ew, erank) when `ranked`,
// otherwise the edges are S.ea / S.eb in ring order.  Stores the vertices at slots
// ord[nvf + rank] and raises *mk to their squared radii (on lanes 3e).  Returns false
// when a determinant is zero.
template <class T>
__device__ __forceinline__ bool new_vertices(ClipSmem<T>& S, int lane, int E, bool ranked, int eu,
                                             int ew, int erank, int nvf, int p_idx, D3 x, int dim,
                                             double* mk) {
  using PIdx = typename T::PIdx;
  const int el = (lane * 11) >> 5;  // lane / 3 for lane < 32
  const int c = lane - 3 * el;
  const int c1 = c == 2 ? 0 : c + 1, c2 = c == 0 ? 2 : c - 1;
  const double* P1 = S.pn(c1);
  const double* P2 = S.pn(c2);
  const double xc = c == 0 ? x.x : (c == 1 ? x.y : x.z);
  bool ok = true;
  for (int e0 = 0; e0 < E; e0 += 10) {
    const int e = e0 + el;
    const bool act = lane < 30 && e < E;
    int u, w, pos;
    if (ranked) {
      u = __shfl_sync(FULL, eu, e & 31);
      w = __shfl_sync(FULL, ew, e & 31);
      pos = __shfl_sync(FULL, erank, e & 31);
    } else {
      u = act ? (int)S.ea[e] : 0;
      w = act ? (int)S.eb[e] : 0;
      pos = e;
    }
    double coord = 0.0;
    int slot = 0;
    if (act) {
      slot = S.ord[nvf + pos];
      const int i = u, j = w, k = p_idx;
      const D3 n0 = {S.pnx[i], S.pny[i], S.pnz[i]};
      const D3 n1 = {S.pnx[j], S.pny[j], S.pnz[j]};
      const D3 n2 = {S.pnx[k], S.pny[k], S.pnz[k]};
      const double det = det_cols(n0, n1, n2);
      if (det == 0.0) {
        ok = false;
      } else {
        const double a1 = P1[i], a2 = P2[i], b1 = P1[j], b2 = P2[j], g1 = P1[k], g2 = P2[k];
        const double y12 = b1 * g2 - g1 * b2;  // (n1 x n2)_c
        const double y20 = g1 * a2 - a1 * g2;  // (n2 x n0)_c
        const double y01 = a1 * b2 - b1 * a2;  // (n0 x n1)_c
        coord = ((S.pd[i] * y12 + S.pd[j] * y20) + S.pd[k] * y01) / det;
        S.vc(c)[slot] = coord;
        reinterpret_cast<float*>(&S.f4[slot])[c] = __double2float_rn(coord - xc);
        (c == 0 ? S.vd0 : (c == 1 ? S.vd1 : S.vd2))[slot] = (PIdx)(c == 0 ? i : (c == 1 ? j : k));
      }
    }
    // squared radius (Vertex::from_dual) on lane 3e from the coordinates of lanes 3e + 1, 3e + 2
    const double cy = __shfl_down_sync(FULL, coord, 1), cz = __shfl_down_sync(FULL, coord, 2);
    if (act && c == 0) {
      const D3 dl = {coord, dim >= 2 ? cy : 0.0, dim == 3 ? cz : 0.0};
      const D3 r = sub(x, dl);
      *mk = fmax(*mk, dot(r, r));
    }
  }
  return __all_sync(FULL, ok);
}

// BOX: band tests that are box-corner zeros are decided here (the kernel used for
// lattice-like inputs; the check's registers slow the common kernel by about a tenth).
template <class T, int PREC, bool BOX>
__device__ int clip_cell(const Job& J, const StageJob& SJ, ClipSmem<T>& S, int lane, int item,
                         int self, int info, int* err_code, ClipCount& cc) {
  using PIdx = typename T::PIdx;
  static_assert(T::NW == 2, "the swap-remove permutation uses 64-bit position masks");
  const D3 x = load_gen(J, self);
  const int dim = J.dim;

  // ---- ConvexCell::init (convex_cell.rs:294-312) ----
  if (lane < 6) {
    S.pnx[lane] = J.bn[lane][0], S.pny[lane] = J.bn[lane][1], S.pnz[lane] = J.bn[lane][2];
    S.pd[lane] = J.bd[lane];
    S.pright[lane] = -1;
    S.pcode[lane] = 13;
  }
  for (int i = lane; i < T::VMAX; i += 32) S.ord[i] = (PIdx)i;
  for (int i = lane; i < T::PMAX; i += 32) S.plm[i] = 0u;
  __syncwarp();
  double r2init = 0.0;
  {
    int i0 = 0, i1 = 0, i2 = 0;
    cuboid_duals(lane, &i0, &i1, &i2);
    bool ok = true;
    if (lane < 8) ok = make_vertex<PIdx, false>(S, lane, i0, i1, i2, x, dim, &r2init);
    if (__any_sync(FULL, !ok)) {
      *err_code = MV_ERR_DET;
      return CELL_ERROR;
    }
  }
  __syncwarp();
  int nv = 8, np = 6;
  double max_r2 = warp_max_nonneg(lane < 8 ? r2init : 0.0);
  double sr = 2.0 * sqrt(max_r2);
  float A32 = amax32_of_sr(sr, dim);
  const double x1 = fabs(x.x) + fabs(x.y) + fabs(x.z);

  // ---- ConvexCell::build over the candidate list (convex_cell.rs:316-356) ----
  const int ncand = info & 0x3fffffff;
  const bool exhausted = (info >> 30) & 1;
  const uint32_t* list = SJ.cand + (int64_t)item * SJ.cstride;
  bool finished = false;
  for (int w0 = 1; w0 < ncand && !finished; w0 += 32) {
    const int wn = min(32, ncand - w0);
    const bool valid = lane < wn;
    // candidate w0 + lane: location and offset as the reference computes them
    // (convex_cell.rs:333-342), plus the f32 quantities of the filter
    bool bad = false, filt = false;
    double dist = 0.0;  // this lane's candidate's distance |x - ngb|
    if (valid) {
      const uint32_t pk = __ldg(list + w0 + lane);
      const int cp = (int)(pk / 27u);
      const int code = (int)(pk - (uint32_t)cp * 27u);
      D3 g = {__ldg(J.sx + cp), __ldg(J.sy + cp), __ldg(J.sz + cp)};
      const int orig = __ldg(J.sid + cp);
      if (code != 13) g = add(g, D3{J.shift[code][0], J.shift[code][1], J.shift[code][2]});
      const D3 dx = sub(x, g);
      dist = sqrt(dot(dx, dx));
      bad = !(dist > 0.0 && dist <= DBL_MAX);
      // HalfSpace::new (half_space.rs:24-34) for every candidate of the window at once
      const D3 n = divs(dx, dist);
      const D3 p = scale(0.5, add(x, g));
      S.wnx[lane] = n.x, S.wny[lane] = n.y, S.wnz[lane] = n.z;
      S.wd[lane] = dot(n, p);
      S.werr[lane] = 1e-13 * (1.0 + dot(vabs(n), vabs(p)));
      S.wpk[lane] = (uint32_t)orig * 27u + (uint32_t)code;
      if (PREC == MV_PRECISION_FILTERED) {
        // s = e.a + |e|^2 / 2 is certified by T = c0 + c1 A with A >= |v - x| over the
        // cell's vertices (the bound of setup_batch, split into its A-free and A parts)
        filt = !bad && dist >= 1e-15 && dist <= 1e15 && x1 <= 1e15;
        const float ex = __double2float_rn(dx.x), ey = __double2float_rn(dx.y),
                    ez = __double2float_rn(dx.z);
        const double e1 = fabs(dx.x) + fabs(dx.y) + fabs(dx.z);
        const double u32 = 5.9604644775390625e-08, u64 = 1.1102230246251565e-16;
        const double errb_up = 1e-13 * (1.0 + 1.001 * (x1 + e1)) * 1.0001;
        const double t0 = dist * (errb_up + u64 * (11.0 * e1 + 14.0 * x1) + u32 * (4.03 * dist));
        S.wf[lane] = make_float4(ex, ey, ez, 0.5f * fmaf(ez, ez, fmaf(ey, ey, ex * ex)));
        S.wc[lane] = make_float2(__double2float_ru(t0 * (1.0 + 1e-6) + 1e-40),
                                 __double2float_ru(dist * (u64 * 11.0 + u32 * 5.02) * (1.0 + 1e-6)));
      }
    }
    __syncwarp();
    // window-constant ballots: degenerate distance, f32 filter applicable
    const unsigned mbad = __ballot_sync(FULL, valid && bad);
    unsigned mfilt = 0u;
    if (PREC == MV_PRECISION_FILTERED) mfilt = __ballot_sync(FULL, valid && filt && A32 <= 1e15f);
    // beyond the safety radius (refreshed when a clip shrinks it)
    unsigned mstop = __ballot_sync(FULL, valid && !bad && sr < dist);
    // the f32 offset of this lane's vertex (position lane) for the filter
    float4 fv = make_float4(0.f, 0.f, 0.f, 0.f);
    if (PREC == MV_PRECISION_FILTERED && lane < nv) fv = S.f4[S.ord[lane]];
    int k = 0;
    for (;;) {
      const unsigned evt = (mbad | mstop) & (k < 32 ? (FULL << k) : 0u);
      const int limit = evt ? __ffs(evt) - 1 : wn;
      const int k0 = k;
      if (PREC == MV_PRECISION_FILTERED) {
        // candidates certified to remove no vertex are consumed without their plane
        while (k < limit && ((mfilt >> k) & 1u)) {
          const float4 fk = S.wf[k];
          const float2 ck = S.wc[k];
          const float exk = fk.x, eyk = fk.y, ezk = fk.z, hk = fk.w;
          const float Tk = __fmaf_ru(ck.y, A32, ck.x);
          bool need = lane < nv && !(fmaf(ezk, fv.z, fmaf(eyk, fv.y, fmaf(exk, fv.x, hk))) > Tk);
          if (nv > 32 && lane + 32 < nv) {
            const float4 f = S.f4[S.ord[lane + 32]];
            need = need || !(fmaf(ezk, f.z, fmaf(eyk, f.y, fmaf(exk, f.x, hk))) > Tk);
          }
          if (__any_sync(FULL, need)) break;
          k++;
        }
      }
      cc.neighbours(k - k0);
      if (k == limit) {
        if (limit == wn) break;  // window consumed
        if ((mbad >> k) & 1u) {
          *err_code = MV_ERR_DEGENERATE;  // convex_cell.rs:342
          return CELL_ERROR;
        }
        finished = true;  // safety radius reached (convex_cell.rs:343-345)
        break;
      }
      const int e = k++;
      cc.neighbours(1);
      // ---- candidate e: HalfSpace::new (half_space.rs:24-34) and clip_by_plane ----
      bool filt_e = false;
      float exe = 0.f, eye = 0.f, eze = 0.f, he = 0.f, Tk = 0.f;
      if (PREC == MV_PRECISION_FILTERED) {
        filt_e = (mfilt >> e) & 1u;
        const float4 fe = S.wf[e];
        const float2 ce = S.wc[e];
        exe = fe.x, eye = fe.y, eze = fe.z, he = fe.w;
        Tk = __fmaf_ru(ce.y, A32, ce.x);
      }
      const D3 n = {S.wnx[e], S.wny[e], S.wnz[e]};
      const double errb = S.werr[e];
      const double d = S.wd[e];
      unsigned rm[T::NW];
      int n_und = 0;
      int bsl[T::NW];  // slot of this lane's vertex when its f64 test is in the band, else -1
#pragma unroll
      for (int w = 0; w < T::NW; w++) {
        const int q = lane + 32 * w;
        bool removed = false;
        bsl[w] = -1;
        if (q < nv) {
          const int sl = S.ord[q];
          bool decided = false;
          if (PREC == MV_PRECISION_FILTERED && filt_e) {
            const float4 f = w == 0 ? fv : S.f4[sl];  // position lane: held in registers
            const float s = fmaf(eze, f.z, fmaf(eye, f.y, fmaf(exe, f.x, he)));
            if (fabsf(s) > Tk) {
              removed = s < 0.f;
              decided = true;
            }
          }
          if (!decided) {
            n_und++;
            const double c = dot(n, D3{S.vx[sl], S.vy[sl], S.vz[sl]}) - d;
            if (fabs(c) < errb)
              bsl[w] = sl;
            else
              removed = c < 0.0;
          }
        }
        rm[w] = __ballot_sync(FULL, removed);
      }
      // inside the f64 band the reference decides with the exact in-sphere predicate
      // (half_space.rs:40-47), a zero determinant keeping the vertex.  Five corners of
      // one axis-aligned box (every band test of a quantised lattice) are such a zero
      // without multi-limb arithmetic (BOX); any other band test sends the cell, before
      // any change here, to the fused kernel (the multi-limb predicate does not fit
      // this kernel's register budget)
      if (__any_sync(FULL, bsl[0] >= 0 || (T::NW > 1 && bsl[T::NW - 1] >= 0))) {
        if constexpr (BOX) {
          const uint32_t pk = S.wpk[e];
          const int cand = (int)(pk / 27u), code = (int)(pk % 27u);
          D3 ngb = load_gen(J, cand);
          if (code != 13) ngb = add(ngb, D3{J.shift[code][0], J.shift[code][1], J.shift[code][2]});
          bool hard = false;
          unsigned nb = 0;
#pragma unroll
          for (int w = 0; w < T::NW; w++)
            if (bsl[w] >= 0) hard |= !exact_clip_box_zero(J, S, bsl[w], x, ngb), nb++;
          if (__any_sync(FULL, hard)) return CELL_EXACT;
          cc.exact(__reduce_add_sync(FULL, nb));
        } else {
          return CELL_EXACT;
        }
      }
      n_und = (int)__reduce_add_sync(FULL, (unsigned)n_und);
      if (PREC == MV_PRECISION_FILTERED) cc.undecided(n_und);
      int nrem = 0;
#pragma unroll
      for (int w = 0; w < T::NW; w++) nrem += __popc(rm[w]);
      if (nrem == 0) continue;

      // ---- a vertex was clipped: add the plane (convex_cell.rs:393-418) ----
      if (np >= T::PMAX) return CELL_OVERFLOW;
      const int p_idx = np;
      if (lane == 0) {
        const uint32_t pk = S.wpk[e];
        S.pnx[p_idx] = n.x, S.pny[p_idx] = n.y, S.pnz[p_idx] = n.z;
        S.pd[p_idx] = d;
        S.pright[p_idx] = (int32_t)(pk / 27u);
        S.pcode[p_idx] = (uint8_t)(pk % 27u);
      }
      np++;
      cc.plane();

      // swap-remove loop (convex_cell.rs:365-390) as a closed-form permutation of ord
      // over masks of removed / kept positions; kept vertices before nvf stay.  The
      // s-th removed / kept position comes from inverse maps built in S.ea / S.eb (free
      // until the ring below).  Cells of at most 32 vertices (most clips) take 32-bit
      // masks, one position per lane.
      const unsigned long long rm64 = ((unsigned long long)rm[1] << 32) | rm[0];
      const unsigned long long km64 = ~rm64 & (nv >= 64 ? ~0ull : ((1ull << nv) - 1ull));
      const int totK = __popcll(km64);
      const int nvf = totK;
      if (nv <= 32) {
        const unsigned rm32 = rm[0], km32 = (unsigned)km64;
        const unsigned below = lanemask_lt();
        const bool in = lane < nv, gone = (rm32 >> lane) & 1u;
        const int rr = __popc(rm32 & below), rk = __popc(km32 & below);
        if (in) {
          if (gone)
            S.ea[rr] = (PIdx)lane;
          else
            S.eb[rk] = (PIdx)lane;
        }
        __syncwarp();
        int dd = -1;
        PIdx held = 0;
        if (in) {
          if (!gone) {
            if (lane >= nvf) dd = S.ea[totK - rk - 1];
          } else if (lane <= nvf) {
            dd = ((rr == 0) ? nv : (int)S.eb[totK - rr]) - 1;
          } else {
            dd = lane - 1;
          }
          if (dd >= 0) held = S.ord[lane];
        }
        __syncwarp();
        if (dd >= 0) S.ord[dd] = held;
        __syncwarp();
      } else {
#pragma unroll
        for (int w = 0; w < 2; w++) {
          const int q = lane + 32 * w;
          if (q < nv) {
            const unsigned long long below = (1ull << q) - 1ull;
            if ((rm64 >> q) & 1ull)
              S.ea[__popcll(rm64 & below)] = (PIdx)q;
            else
              S.eb[__popcll(km64 & below)] = (PIdx)q;
          }
        }
        __syncwarp();
        int dest[2];
        PIdx held[2];
#pragma unroll
        for (int w = 0; w < 2; w++) {
          const int q = lane + 32 * w;
          int dd = -1;
          held[w] = 0;
          if (q < nv) {
            const unsigned long long below = (1ull << q) - 1ull;
            if (!((rm64 >> q) & 1ull)) {
              if (q >= nvf) dd = S.ea[totK - __popcll(km64 & below) - 1];
            } else if (q <= nvf) {
              const int t = __popcll(rm64 & below) + 1;
              dd = ((t == 1) ? nv : (int)S.eb[totK - t + 1]) - 1;
            } else {
              dd = q - 1;
            }
            if (dd >= 0) held[w] = S.ord[q];
          }
          dest[w] = dd;
        }
        __syncwarp();
#pragma unroll
        for (int w = 0; w < 2; w++)
          if (dest[w] >= 0) S.ord[dest[w]] = held[w];
        __syncwarp();
      }
      double mk = 0.0;  // largest squared radius of this lane's vertices

      // ring of the removed region (compute_boundary + SimpleCycle iteration): lane e
      // gets the boundary edge at ring position erank and creates its vertex
      int eu = 0, ew = 0, erank = 0;
      int E = ring_ranked<T>(S, lane, nvf, nv, &eu, &ew, &erank);
      const bool replayed = E < 0;
      if (E < 0) {
        cc.serial_ring();
        E = ring_replay_lanes<T>(S, lane, nvf, nv, np);
        if (E == -2) return CELL_OVERFLOW;
        if (E < 0) {
          *err_code = MV_ERR_RING;
          return CELL_ERROR;
        }
      }
      if (nvf + E > T::VMAX) return CELL_OVERFLOW;
      if (!new_vertices<T>(S, lane, E, !replayed, eu, ew, erank, nvf, p_idx, x, dim, &mk)) {
        *err_code = MV_ERR_DET;
        return CELL_ERROR;
      }
      __syncwarp();
      nv = nvf + E;
      // update_safety_radius (convex_cell.rs:443-453): the maximum over the kept and the
      // new vertices
      for (int q = lane; q < nvf; q += 32) mk = fmax(mk, vertex_r2(S, S.ord[q], x, dim));
      const double mr = warp_max_nonneg(mk);
      if (__double_as_longlong(mr) != __double_as_longlong(max_r2)) {
        max_r2 = mr;
        sr = 2.0 * sqrt(max_r2);
        A32 = amax32_of_sr(sr, dim);
      }
      mstop = __ballot_sync(FULL, valid && !bad && sr < dist);
      if (PREC == MV_PRECISION_FILTERED && lane < nv) fv = S.f4[S.ord[lane]];
    }
  }
  // the list ends: the shell was complete up to the initial radius (as the fused
  // kernel's shell loop decides); otherwise the fused kernel continues the stream
  if (!finished && !(exhausted || sr < SJ.rad[item] * (1.0 - 1e-12))) return CELL_RETRY;

  // ---- the cell record for the integral kernel ----
  if (!write_record(J, SJ.rec, SJ.rec_cap, SJ.rec_counter, SJ.rec_off + item, S, lane, x, np, nv, sr,
                    SJ.full_records != 0))
    return CELL_RETRY;
  return CELL_DONE;
}

template <class T, int PREC, int WARPS, bool MULTI, bool BOX>
__global__ void __launch_bounds__(32 * WARPS, T::MINB)
    clip_kernel(const __grid_constant__ Job J0, const __grid_constant__ StageJob SJ,
                const __grid_constant__ JobTable TB) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  ClipSmem<T>& S = reinterpret_cast<ClipSmem<T>*>(smem_raw)[warp];
  __shared__ unsigned long long cnt[ST_COUNT];  // the block's event counts
  if (threadIdx.x < ST_COUNT) cnt[threadIdx.x] = 0ull;
  __syncthreads();
  for (;;) {
    int item = 0;
    if (lane == 0) item = (int)atomicAdd(SJ.work + 1, 1u);
    item = __shfl_sync(FULL, item, 0);
    if (item >= SJ.nitems) break;
    const int gpos = stage_pos(SJ, item);
    // the cell's tessellation (batch builds): its Job and its local position
    const int jb = MULTI ? job_of(TB, gpos) : 0;
    const Job& J = MULTI ? TB.jobs[jb] : J0;
    const int spos = MULTI ? gpos - __ldg(TB.pos_base + jb) : gpos;
    const int self = __ldg(J.sid + spos);
    if (J.mask != nullptr && J.mask[self] == 0) {
      // VoronoiCell::default() (voronoi.rs:303-305)
      if (lane < 3) J.centroid[3 * (int64_t)self + lane] = 0.0;
      if (lane == 0) {
        J.volume[self] = 0.0;
        J.safety_radius[self] = 0.0;
        J.face_count[self] = 0;
        J.stage_off[self] = 0;
        SJ.rec_off[item] = -1;
      }
      continue;
    }
    const int info = SJ.info[item];
    int res = CELL_RETRY;
    int err = 0;
    ClipCount cc{0u, 0u, 0u};
    if (info > 0) res = clip_cell<T, PREC, BOX>(J, SJ, S, lane, item, self, info, &err, cc);
    __syncwarp();
    if (lane == 0) {
      if (res == CELL_DONE) {
        const unsigned v[5] = {cc.a & 0xffffu, (cc.a >> 16) & 0xffu, cc.a >> 24, cc.b, cc.e};
        const int slot[5] = {ST_NEIGHBOURS, ST_PLANES, ST_SERIAL_RING, ST_F32_UNDECIDED, ST_EXACT};
#pragma unroll
        for (int i = 0; i < 5; i++)
          if (v[i]) atomicAdd(&cnt[slot[i]], (unsigned long long)v[i]);
      } else {
        SJ.rec_off[item] = -1;
        if (res == CELL_ERROR) {
          atomicCAS(J.status + STATUS_CODE, 0, err);
          atomicMin(J.status + STATUS_CELL, self + J.id_base);
        } else if (res == CELL_EXACT) {
          const unsigned k = atomicAdd(SJ.fused_count, 1u);
          SJ.fused_list[k] = gpos;
        } else {
          const unsigned k = atomicAdd(SJ.retry_count, 1u);
          SJ.retry_list[k] = gpos;
        }
      }
    }
    __syncwarp();
  }
  __syncwarp();
  __syncthreads();
  if (threadIdx.x < ST_COUNT && cnt[threadIdx.x]) atomicAdd(J0.stats + threadIdx.x, cnt[threadIdx.x]);
}

// --------------------------------------------------------------- integrals --
template <class T, int WARPS, bool MULTI>
__global__ void __launch_bounds__(32 * WARPS, MV_INT_MINB)
    integrate_kernel(const __grid_constant__ Job J0, const __grid_constant__ StageJob SJ,
                     const __grid_constant__ JobTable TB) {
  __shared__ TetScratch<INT_STEP, T::PMAX> scratch[WARPS];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int i = lane; i < T::PMAX; i += 32) scratch[warp].pm[i] = 0u;
  __syncwarp();
  unsigned done = 0;
  for (;;) {
    int item = 0;
    if (lane == 0) item = (int)atomicAdd(SJ.work + 2, 1u);
    item = __shfl_sync(FULL, item, 0);
    if (item >= SJ.nitems) break;
    const int64_t off = SJ.rec_off[item];
    if (off < 0) continue;
    const int gpos = stage_pos(SJ, item);
    const int jb = MULTI ? job_of(TB, gpos) : 0;
    const Job& J = MULTI ? TB.jobs[jb] : J0;
    const int spos = MULTI ? gpos - __ldg(TB.pos_base + jb) : gpos;
    const int self = __ldg(J.sid + spos);
    const D3 x = load_gen(J, self);
    const RecordView V(SJ.rec + off);
    int err = 0;
    const int res = integrate_view<T, INT_STEP>(J, V, scratch[warp], lane, self, x, V.nv, V.np, V.sr, &err);
    if (res == CELL_DONE) {
      done++;
    } else if (lane == 0) {
      if (res == CELL_FACE_OVERFLOW) {
        atomicExch(J.status + STATUS_FACE_OVERFLOW, 1);
      } else {
        atomicCAS(J.status + STATUS_CODE, 0, err);
        atomicMin(J.status + STATUS_CELL, self + J.id_base);
      }
    }
    __syncwarp();
  }
  if (lane == 0 && done) atomicAdd(J0.stats + ST_CELLS, (unsigned long long)done);
}

// ---------------------------------------------------------------- launchers --
template <class K>
static int occupancy(K k, int threads, size_t smem) {
  int nb = 0;
  if (smem > 0 &&
      cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
    return 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k, threads, smem) != cudaSuccess) return 0;
  return nb;
}

constexpr size_t CLIP_SMEM = sizeof(ClipSmem<TierClip>) * CLIP_WARPS;

int stage_blocks_per_sm(int kernel, int precision) {
  if (kernel == 0) return occupancy(shell_kernel<SHELL_WARPS, false>, 32 * SHELL_WARPS, 0);
  if (kernel == 3) return occupancy(shell_wide_kernel<WIDE_WARPS, false>, 32 * WIDE_WARPS, WIDE_SMEM);
  if (kernel == 1)
    return precision == MV_PRECISION_FILTERED
               ? occupancy(clip_kernel<TierClip, MV_PRECISION_FILTERED, CLIP_WARPS, false, false>,
                           32 * CLIP_WARPS, CLIP_SMEM)
               : occupancy(clip_kernel<TierClip, MV_PRECISION_FP64, CLIP_WARPS, false, false>,
                           32 * CLIP_WARPS, CLIP_SMEM);
  return occupancy(integrate_kernel<TierClip, INT_WARPS, false>, 32 * INT_WARPS, 0);
}

__global__ void append_range_kernel(int32_t* dst, int32_t first, int32_t count) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < count) dst[i] = first + i;
}

// dst[i] = first + i for i < count (processing positions handed to the fused kernel)
cudaError_t launch_append_range(int32_t* dst, int32_t first, int32_t count, cudaStream_t st) {
  if (count <= 0) return cudaSuccess;
  append_range_kernel<<<(count + 255) / 256, 256, 0, st>>>(dst, first, count);
  return cudaGetLastError();
}

int stage_list_stride() { return SHELL_CMAX; }
int stage_wide_stride() { return WIDE_CMAX; }

int64_t stage_record_words(int np, int nv) { return rec_words(np, nv); }

template <bool MULTI>
static cudaError_t launch_stage_t(int kernel, const Job& J, const StageJob& SJ, const JobTable& TB,
                                  int blocks, cudaStream_t st) {
  if (kernel == 0) {
    shell_kernel<SHELL_WARPS, MULTI><<<blocks, 32 * SHELL_WARPS, 0, st>>>(J, SJ, TB);
  } else if (kernel == 3) {
    auto k = shell_wide_kernel<WIDE_WARPS, MULTI>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)WIDE_SMEM);
    if (e != cudaSuccess) return e;
    k<<<blocks, 32 * WIDE_WARPS, WIDE_SMEM, st>>>(J, SJ, TB);
  } else if (kernel == 1) {
    auto k = J.precision == MV_PRECISION_FILTERED
                 ? clip_kernel<TierClip, MV_PRECISION_FILTERED, CLIP_WARPS, MULTI, false>
                 : clip_kernel<TierClip, MV_PRECISION_FP64, CLIP_WARPS, MULTI, false>;
    if constexpr (!MULTI) {
      if (SJ.box)
        k = J.precision == MV_PRECISION_FILTERED
                ? clip_kernel<TierClip, MV_PRECISION_FILTERED, CLIP_WARPS, false, true>
                : clip_kernel<TierClip, MV_PRECISION_FP64, CLIP_WARPS, false, true>;
    }
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)CLIP_SMEM);
    if (e != cudaSuccess) return e;
    k<<<blocks, 32 * CLIP_WARPS, CLIP_SMEM, st>>>(J, SJ, TB);
  } else {
    integrate_kernel<TierClip, INT_WARPS, MULTI><<<blocks, 32 * INT_WARPS, 0, st>>>(J, SJ, TB);
  }
  return cudaGetLastError();
}

// Launches stage kernel `kernel` (0 shell, 1 clip, 2 integrals, 3 wide shell); with a
// job table (TB.jobs != nullptr) over the cells of a batch.
cudaError_t launch_stage(int kernel, const Job& J, const StageJob& SJ, const JobTable& TB, int blocks,
                         cudaStream_t st) {
  if (blocks < 1) blocks = 1;
  return TB.jobs != nullptr ? launch_stage_t<true>(kernel, J, SJ, TB, blocks, st)
                            : launch_stage_t<false>(kernel, J, SJ, TB, blocks, st);
}

}  // namespace mv
