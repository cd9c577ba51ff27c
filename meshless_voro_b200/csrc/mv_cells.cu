// mv_cells.cu -- warp-per-cell Voronoi cell construction (sm_100a).
//
// Replaces the per-cell closure of Voronoi::build / VoronoiIntegrator::build
// (voronoi.rs:285-306, 582-602): the nearest-neighbour stream (rtree_nn.rs:10-240),
// ConvexCell::build / clip_by_plane / compute_boundary / update_safety_radius
// (convex_cell.rs:294-453, simple_cycle.rs), the half-space predicate with its exact
// fallback (half_space.rs:40-47, boundary.rs:49-64, geometry.rs:271-314) and the
// integrals of VoronoiCell::from_convex_cell (voronoi_cell.rs:40-100, integrals.rs).
//
// One warp builds one cell at a time, pulling cells from a global work queue.  The
// cell's clipping planes, vertices, neighbour shell and tet scratch live in shared
// memory.  Every step keeps the reference's sequential semantics:
//   * neighbours are consumed in ascending f64 squared distance (ties: original
//     index, then shift code) from nested shells of a uniform grid;
//   * vertices sit in fixed slots; a byte array `ord` carries the reference's vertex
//     order, and the swap-remove loop of clip_by_plane becomes a closed-form
//     permutation of `ord` derived from the ballot of removed vertices;
//   * the SimpleCycle ring is the boundary of the removed vertices' dual triangles,
//     started where the reference starts it (serial replay when that node vanished);
//   * cell and face integrals are summed in the reference's tet order.
// Hence vertices, topology and integrals are the same binary64 values the
// reference computes.
//
// Filtered precision tests a batch of upcoming neighbours at once with a
// division-free f32 predicate whose error bound certifies the reference's f64
// decision; neighbours certified to remove no vertex are consumed without building
// their f64 bisector plane, and the first neighbour that needs attention gets the
// reference's f64 (and, when undecided, exact integer) treatment.
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

// Resident blocks per SM the fast tier is compiled for (sets its register budget).
#ifndef MV_FAST_MINB
#define MV_FAST_MINB 4
#endif
#ifndef MV_FAST_KMAX
#define MV_FAST_KMAX 16
#endif
using TierFast = Tier<64, 64, 128, MV_FAST_KMAX, uint8_t, MV_FAST_MINB>;
using TierLarge = Tier<512, 512, 512, 32, uint16_t, 1>;

template <class T>
struct CellSmem {
  using PIdx = typename T::PIdx;
  // clipping planes (half_space.rs:9-19)
  double pnx[T::PMAX], pny[T::PMAX], pnz[T::PMAX];
  double ppx[T::PMAX], ppy[T::PMAX], ppz[T::PMAX];
  double pd[T::PMAX];
  int32_t pright[T::PMAX];  // original index of the right generator, -1: boundary
  uint8_t pcode[T::PMAX];   // periodic shift code, 13: none
  PIdx rptr[T::PMAX];       // ring successor (SimpleCycle::ptrs)
  // vertices (convex_cell.rs:16-25) in fixed slots
  double vx[T::VMAX], vy[T::VMAX], vz[T::VMAX], vr2[T::VMAX];
  float fx[T::VMAX], fy[T::VMAX], fz[T::VMAX];  // f32 (v - x) for the filter
  PIdx vd0[T::VMAX], vd1[T::VMAX], vd2[T::VMAX];
  PIdx ord[T::VMAX];              // position -> slot; [0, nv) is the reference's order
  PIdx ea[T::VMAX], eb[T::VMAX];  // ring edges in SimpleCycle iteration order
  unsigned long long cnt[ST_COUNT];  // per-warp event counts (flushed to global at exit)
  union {
    struct {  // clipping phase
      unsigned long long key[T::CMAX];  // f64 squared distance bits
      uint32_t tie[T::CMAX];            // original index * 27 + shift code
      int32_t cpos[T::CMAX];            // grid-sorted position of the generator
      int32_t sstart[96];
      int32_t spref[97];
      uint8_t scode[96];
      // neighbours of the current batch
      float bex[T::KMAX], bey[T::KMAX], bez[T::KMAX], bh[T::KMAX], bT[T::KMAX];
      double bdx[T::KMAX], bdy[T::KMAX], bdz[T::KMAX], bdist[T::KMAX];
      double bgx[T::KMAX], bgy[T::KMAX], bgz[T::KMAX];
      int32_t borig[T::KMAX];
      uint8_t bcode[T::KMAX];
      uint8_t bfilt[T::KMAX];
    } g;
    struct {  // integration phase
      double px[T::PMAX], py[T::PMAX], pz[T::PMAX];  // generator projected on each plane
      double ix[15], iy[15], iz[15];                 // on the plane-pair lines of 5 vertices
      double val[8][32];
    } t;
  } u;
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
template <class T>
__device__ __forceinline__ D3 right_loc(const Job& J, const CellSmem<T>& S, int k, D3 x) {
  int r = S.pright[k];
  if (r >= 0) {
    D3 l = load_gen(J, r);
    int code = S.pcode[k];
    if (code != 13) l = add(l, D3{J.shift[code][0], J.shift[code][1], J.shift[code][2]});
    return l;
  }
  D3 pr = plane_project({S.pnx[k], S.pny[k], S.pnz[k]}, {S.ppx[k], S.ppy[k], S.ppz[k]}, x);
  return sub(scale(2.0, pr), x);
}

// Exact decision of clip_by_plane for an undecided vertex in slot `s`
// (convex_cell.rs:370-382).
template <class T>
__device__ __noinline__ int exact_clip(const Job& J, const CellSmem<T>& S, int s, D3 x, D3 ngb) {
  int64_t A[3], B[3], C[3], Dd[3], W[3];
  iloc(J, x, A);
  iloc(J, right_loc(J, S, S.vd0[s], x), B);
  iloc(J, right_loc(J, S, S.vd1[s], x), C);
  iloc(J, right_loc(J, S, S.vd2[s], x), Dd);
  iloc(J, ngb, W);
  return in_sphere_exact_sign(A, B, C, Dd, W);
}

// Vertex::from_dual (convex_cell.rs:28-48) into slot `slot`.
template <class T>
__device__ __forceinline__ bool make_vertex(CellSmem<T>& S, int slot, int i, int j, int k, D3 x,
                                         int dim) {
  D3 loc;
  bool ok = intersect3({S.pnx[i], S.pny[i], S.pnz[i]}, S.pd[i], {S.pnx[j], S.pny[j], S.pnz[j]},
                       S.pd[j], {S.pnx[k], S.pny[k], S.pnz[k]}, S.pd[k], &loc);
  if (!ok) return false;
  D3 dl = loc;
  if (dim == 1) dl = {loc.x, 0.0, 0.0};
  if (dim == 2) dl = {loc.x, loc.y, 0.0};
  D3 r = sub(x, dl);
  S.vx[slot] = loc.x;
  S.vy[slot] = loc.y;
  S.vz[slot] = loc.z;
  S.vr2[slot] = dot(r, r);
  S.fx[slot] = __double2float_rn(loc.x - x.x);
  S.fy[slot] = __double2float_rn(loc.y - x.y);
  S.fz[slot] = __double2float_rn(loc.z - x.z);
  S.vd0[slot] = (typename T::PIdx)i;
  S.vd1[slot] = (typename T::PIdx)j;
  S.vd2[slot] = (typename T::PIdx)k;
  return true;
}

// Bound on |v - x| over the cell's vertices for the f32 filter: r2 omits the
// extruded dimensions, whose vertex coordinates are +-0.5.
__device__ __forceinline__ double amax_of(double max_r2, int dim) {
  return sqrt((max_r2 + 0.26 * (3 - dim)) * (1.0 + 1e-9)) * (1.0 + 1e-9);
}

enum CellResult { CELL_DONE = 0, CELL_OVERFLOW = 1, CELL_ERROR = 2, CELL_FACE_OVERFLOW = 3 };

// ------------------------------------------------------------- neighbour shell --
// Gathers every stream element (generator, periodic image) with lo2 <= d2 < R*R into
// S.u.g (unsorted) and returns how many there are (may exceed CMAX).  *exhausted is
// set when the enumerated cells cover every image and none lies beyond R, i.e. the
// stream ends with this shell.  d2 is the reference's squared distance:
// (g - q).length_squared() for nn_iter (rstar) and |(q + s) - g|^2 for
// wrapping_nn_iter (rtree_nn.rs:138-146).
template <class T>
__device__ __noinline__ int gather_shell(const Job& J, CellSmem<T>& S, int lane, D3 x, double R,
                                         double lo2, const double* ext, bool* exhausted) {
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

  // box-distance of unwrapped grid coordinate u along axis i
  auto box_d = [&](int i, int u) -> double {
    int G = J.G[i];
    bool wrap = J.periodic && i < J.dim;
    int m = u < 0 ? -1 : (u >= G ? 1 : 0);
    int c = u - m * G;
    double blo = J.ga[i] + c * J.gh[i], bhi = J.ga[i] + (c + 1) * J.gh[i];
    if (c == 0) blo = wrap ? fmin(blo, ext[i]) : -__longlong_as_double(0x7ff0000000000000ll);
    if (c == G - 1) bhi = wrap ? fmax(bhi, ext[3 + i]) : __longlong_as_double(0x7ff0000000000000ll);
    blo += m * J.gw[i] - J.geps[i];
    bhi += m * J.gw[i] + J.geps[i];
    return xa[i] < blo ? blo - xa[i] : (xa[i] > bhi ? xa[i] - bhi : 0.0);
  };

  for (int row0 = 0; row0 < nrows; row0 += 32) {
    const int row = row0 + lane;
    int nseg = 0;
    int32_t s0a = 0, s0b = 0, s0c = 0, sla = 0, slb = 0, slc = 0;
    int sca = 0, scb = 0, scc = 0;
    if (row < nrows) {
      const int uy = lo[1] + row % ny, uz = lo[2] + row / ny;
      const double dy = box_d(1, uy), dz = box_d(2, uz);
      const double byz2 = dy * dy + dz * dz;
      if (all || byz2 < R2v) {
        int first = 1 << 30, last = -(1 << 30);
        for (int ux = lo[0]; ux <= hi[0]; ux++) {
          double dx = box_d(0, ux);
          if (all || dx * dx + byz2 < R2v) {
            first = min(first, ux);
            last = max(last, ux);
          }
        }
        const int Gx = J.G[0], Gy = J.G[1], Gz = J.G[2];
        const int my = uy < 0 ? -1 : (uy >= Gy ? 1 : 0);
        const int mz = uz < 0 ? -1 : (uz >= Gz ? 1 : 0);
        const int cy = uy - my * Gy, cz = uz - mz * Gz;
        const int64_t rowbase = (int64_t)Gx * (cy + (int64_t)Gy * cz);
        for (int mx = -1; mx <= 1; mx++) {
          int a = max(first, mx * Gx), b = min(last, mx * Gx + Gx - 1);
          if (a > b) continue;
          int c0 = a - mx * Gx, c1 = b - mx * Gx;
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
      S.u.g.sstart[segoff] = s0a, S.u.g.spref[segoff] = lenoff, S.u.g.scode[segoff] = (uint8_t)sca;
    }
    if (nseg > 1) {
      S.u.g.sstart[segoff + 1] = s0b, S.u.g.spref[segoff + 1] = lenoff + sla;
      S.u.g.scode[segoff + 1] = (uint8_t)scb;
    }
    if (nseg > 2) {
      S.u.g.sstart[segoff + 2] = s0c, S.u.g.spref[segoff + 2] = lenoff + sla + slb;
      S.u.g.scode[segoff + 2] = (uint8_t)scc;
    }
    __syncwarp();
    for (int t0 = 0; t0 < total; t0 += 32) {
      const int t = t0 + lane;
      bool keep = false;
      double d2 = 0.0;
      uint32_t tie = 0;
      int s = 0;
      if (t < total) {
        int a = 0, b = nsegs_total - 1;
        while (a < b) {
          int mid = (a + b + 1) >> 1;
          if (S.u.g.spref[mid] <= t)
            a = mid;
          else
            b = mid - 1;
        }
        s = S.u.g.sstart[a] + (t - S.u.g.spref[a]);
        const int code = S.u.g.scode[a];
        const double px = __ldg(J.sx + s), py = __ldg(J.sy + s), pz = __ldg(J.sz + s);
        const int orig = __ldg(J.sid + s);
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
        tie = (uint32_t)orig * 27u + (uint32_t)code;
      }
      const unsigned bal = __ballot_sync(FULL, keep);
      const int pos = count + __popc(bal & lanemask_lt());
      if (keep && pos < T::CMAX) {
        S.u.g.key[pos] = (unsigned long long)__double_as_longlong(d2);
        S.u.g.tie[pos] = tie;
        S.u.g.cpos[pos] = s;
      }
      count += __popc(bal);
    }
    __syncwarp();
  }
  *exhausted = all && !__any_sync(FULL, beyond > 0);
  return count;
}

// Bitonic sort of the shell [0, n) by (key, tie) ascending, carrying cpos; n <= CMAX.
template <class T>
__device__ __noinline__ void sort_shell(CellSmem<T>& S, int lane, int n) {
  int np2 = 32;
  while (np2 < n) np2 <<= 1;
  for (int i = n + lane; i < np2; i += 32) {
    S.u.g.key[i] = ~0ull;
    S.u.g.tie[i] = ~0u;
    S.u.g.cpos[i] = 0;
  }
  __syncwarp();
  for (int k = 2; k <= np2; k <<= 1) {
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int i = lane; i < (np2 >> 1); i += 32) {
        const int lo = 2 * j * (i / j) + (i % j);
        const int hi = lo + j;
        const bool asc = (lo & k) == 0;
        const unsigned long long ka = S.u.g.key[lo], kb = S.u.g.key[hi];
        const uint32_t ta = S.u.g.tie[lo], tb = S.u.g.tie[hi];
        const bool gt = (ka > kb) || (ka == kb && ta > tb);
        if (gt == asc) {
          const int32_t pa = S.u.g.cpos[lo], pb = S.u.g.cpos[hi];
          S.u.g.key[lo] = kb;
          S.u.g.key[hi] = ka;
          S.u.g.tie[lo] = tb;
          S.u.g.tie[hi] = ta;
          S.u.g.cpos[lo] = pb;
          S.u.g.cpos[hi] = pa;
        }
      }
      __syncwarp();
    }
  }
}

// -------------------------------------------------------------------- ring --
// Serial replay of compute_boundary (convex_cell.rs:421-441) and SimpleCycle
// (simple_cycle.rs:17-78) on lane 0 for the removed vertices at positions [nvf, nv).
// Produces the edge list (S.ea, S.eb) and returns its length, -1 on failure, -2 when
// the ring exceeds the tier's vertex capacity.
template <class T>
__device__ __noinline__ int ring_serial(CellSmem<T>& S, int nvf, int nv, int np) {
  using PIdx = typename T::PIdx;
  for (int i = 0; i < np; i++) S.rptr[i] = (PIdx)i;
  auto contains = [&](int i) { return S.rptr[i] != (PIdx)i; };
  const int s0 = S.ord[nvf];
  int start = S.vd0[s0];
  int len = 3;
  {
    int a = S.vd0[s0], b = S.vd1[s0], c = S.vd2[s0];
    S.rptr[a] = (PIdx)b;
    S.rptr[b] = (PIdx)c;
    S.rptr[c] = (PIdx)a;
  }
  const int n = nv - nvf;
  for (int i = 1; i < n; i++) {
    int idx = i;
    for (;;) {
      if (idx >= n) return -1;
      const int sl = S.ord[nvf + idx];
      const int t0 = S.vd0[sl], t1 = S.vd1[sl], t2 = S.vd2[sl];
      const bool i0 = contains(t0), i1 = contains(t1), i2 = contains(t2);
      bool ok = false;
      for (int a = 0; a < 3 && !ok; a++) {
        // rotation (ta, tb, tc) = (tri[a], tri[a+1], tri[a+2])
        const int ta = a == 0 ? t0 : (a == 1 ? t1 : t2);
        const int tb = a == 0 ? t1 : (a == 1 ? t2 : t0);
        const int tc = a == 0 ? t2 : (a == 1 ? t0 : t1);
        const bool ia = a == 0 ? i0 : (a == 1 ? i1 : i2);
        const bool ib = a == 0 ? i1 : (a == 1 ? i2 : i0);
        const bool ic = a == 0 ? i2 : (a == 1 ? i0 : i1);
        if (!ia && ib && ic && S.rptr[tc] == (PIdx)tb) {
          S.rptr[tc] = (PIdx)ta;
          S.rptr[ta] = (PIdx)tb;
          len += 1;
          ok = true;
        } else if (ia && ib && ic && S.rptr[tc] == (PIdx)tb && S.rptr[tb] == (PIdx)ta) {
          S.rptr[tc] = (PIdx)ta;
          S.rptr[tb] = (PIdx)tb;
          if (start == tb) start = ta;
          len -= 1;
          ok = true;
        }
      }
      if (ok) {
        if (idx > i) {
          const PIdx tmp = S.ord[nvf + i];
          S.ord[nvf + i] = S.ord[nvf + idx];
          S.ord[nvf + idx] = tmp;
        }
        break;
      }
      idx++;
    }
  }
  if (len > T::VMAX) return -2;
  int cur = start;
  for (int e = 0; e < len; e++) {
    const int nxt = S.rptr[cur];
    S.ea[e] = (PIdx)cur;
    S.eb[e] = (PIdx)nxt;
    cur = nxt;
  }
  return len;
}

// Parallel ring: the boundary edges of the union of the removed dual triangles form
// the same cycle the serial algorithm builds; it starts at the first removed
// vertex's dual[0] whenever that node is still on the boundary.  Returns the edge
// count, or -1 when the serial replay must decide.
template <class T>
__device__ __forceinline__ int ring_parallel(CellSmem<T>& S, int lane, int nvf, int nv) {
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
  int E;
  warp_excl_scan((int)b01 + (int)b12 + (int)b20, lane, &E);
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

// ------------------------------------------------------------------ the cell --
// Event counts of one cell, kept in warp-uniform registers (a lane-0 branch inside
// the clip loop would split the warp) and flushed once per cell.
struct CellCount {
  unsigned c[ST_COUNT];
};
#define WCNT(CC, slot, v) ((CC).c[slot] += (unsigned)(v))

// Integrals and face emission of a finished cell (convex_cell.rs:131-187,
// voronoi_cell.rs:40-100).  The generator's projection on each plane is computed
// once per plane; each 5-vertex step projects on the 15 plane-pair lines, builds the
// 30 tets (one per lane) and accumulates them in the reference's tet order: lanes
// 0-3 the cell integrals, lane p (and p + 32k) the integrals of face p.
template <class T>
__device__ __noinline__ int integrate_cell(const Job& J, CellSmem<T>& S, int lane, int self, D3 x,
                                           int nv, int np, double sr, int* err_code) {
  // (the cell count is taken by the caller)
  const int dim = J.dim;
  for (int pl = lane; pl < np; pl += 32) {
    const D3 pr = plane_project({S.pnx[pl], S.pny[pl], S.pnz[pl]},
                                {S.ppx[pl], S.ppy[pl], S.ppz[pl]}, x);
    S.u.t.px[pl] = pr.x;
    S.u.t.py[pl] = pr.y;
    S.u.t.pz[pl] = pr.z;
  }
  double cacc = 0.0;  // lanes 0..3: volume, centroid x, y, z
  double fa[T::PMAX / 32], fcx[T::PMAX / 32], fcy[T::PMAX / 32], fcz[T::PMAX / 32];
  unsigned ftouched = 0;
#pragma unroll
  for (int k = 0; k < T::PMAX / 32; k++) fa[k] = 0.0, fcx[k] = 0.0, fcy[k] = 0.0, fcz[k] = 0.0;
  for (int base = 0; base < nv; base += 5) {
    const int nstep = min(5, nv - base);
    // projections on the lines dual[i] & dual[i+1]: project_onto_intersection
    // (geometry.rs:41-47) of plane dual[(i+1)%3] with dual[i]
    bool ok = true;
    if (lane < 3 * nstep) {
      const int vl = lane / 3, i = lane - 3 * vl;
      const int sl = S.ord[base + vl];
      const int d0 = S.vd0[sl], d1 = S.vd1[sl], d2 = S.vd2[sl];
      const int cur = i == 0 ? d0 : (i == 1 ? d1 : d2);
      const int nx = i == 0 ? d1 : (i == 1 ? d2 : d0);
      const D3 cn = {S.pnx[cur], S.pny[cur], S.pnz[cur]};
      const D3 nn = {S.pnx[nx], S.pny[nx], S.pnz[nx]};
      const D3 perp = cross(nn, cn);
      D3 pr = {0.0, 0.0, 0.0};
      ok = intersect3(nn, S.pd[nx], cn, S.pd[cur], perp, dot(x, perp), &pr);
      S.u.t.ix[lane] = pr.x;
      S.u.t.iy[lane] = pr.y;
      S.u.t.iz[lane] = pr.z;
    }
    if (__any_sync(FULL, !ok)) {
      *err_code = MV_ERR_DET;
      return CELL_ERROR;
    }
    __syncwarp();
    // DecompositionWithoutFaces: tet t of a vertex = (proj[t], proj[(t+5)%6], vertex)
    // with proj[2i] on plane dual[i] and proj[2i+1] on the line (dual[i+1], dual[i])
    if (lane < 6 * nstep) {
      const int vl = lane / 6, t = lane - 6 * vl;
      const int sl = S.ord[base + vl];
      const int d0 = S.vd0[sl], d1 = S.vd1[sl], d2 = S.vd2[sl];
      auto proj = [&](int q) -> D3 {
        const int i = q >> 1;
        if (q & 1) return D3{S.u.t.ix[3 * vl + i], S.u.t.iy[3 * vl + i], S.u.t.iz[3 * vl + i]};
        const int pl = i == 0 ? d0 : (i == 1 ? d1 : d2);
        return D3{S.u.t.px[pl], S.u.t.py[pl], S.u.t.pz[pl]};
      };
      const D3 v0 = proj(t), v1 = proj(t == 0 ? 5 : t - 1);
      const D3 vloc = {S.vx[sl], S.vy[sl], S.vz[sl]};
      const double vol = signed_volume_tet(v0, v1, vloc, x);
      const D3 vc = scale(vol, add(add(add(v0, v1), vloc), x));
      const double ar = signed_area_tri(v0, v1, vloc, x);
      const D3 ac = scale(ar, add(add(v0, v1), vloc));
      S.u.t.val[0][lane] = vol;
      S.u.t.val[1][lane] = vc.x;
      S.u.t.val[2][lane] = vc.y;
      S.u.t.val[3][lane] = vc.z;
      S.u.t.val[4][lane] = ar;
      S.u.t.val[5][lane] = ac.x;
      S.u.t.val[6][lane] = ac.y;
      S.u.t.val[7][lane] = ac.z;
    }
    __syncwarp();
    const int ntet = 6 * nstep;
    if (lane < 4) {
      for (int s = 0; s < ntet; s++) cacc = cacc + S.u.t.val[lane][s];
    }
#pragma unroll
    for (int k = 0; k < T::PMAX / 32; k++) {
      const int pl = lane + 32 * k;
      if (pl < np) {
        for (int vl = 0; vl < nstep; vl++) {
          const int sl = S.ord[base + vl];
          const int kk = S.vd0[sl] == pl ? 0 : (S.vd1[sl] == pl ? 1 : (S.vd2[sl] == pl ? 2 : -1));
          if (kk >= 0) {
            const int s = 6 * vl + 2 * kk;
            fa[k] = fa[k] + S.u.t.val[4][s];
            fcx[k] = fcx[k] + S.u.t.val[5][s];
            fcy[k] = fcy[k] + S.u.t.val[6][s];
            fcz[k] = fcz[k] + S.u.t.val[7][s];
            fa[k] = fa[k] + S.u.t.val[4][s + 1];
            fcx[k] = fcx[k] + S.u.t.val[5][s + 1];
            fcy[k] = fcy[k] + S.u.t.val[6][s + 1];
            fcz[k] = fcz[k] + S.u.t.val[7][s + 1];
            ftouched |= 1u << k;
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
      const D3 nn = {S.pnx[pl], S.pny[pl], S.pnz[pl]};
      e = vector_is_valid(dim, nn);
      const int r = S.pright[pl];
      if (e && J.face_mode == MV_FACES_OWNED && r >= 0 && S.pcode[pl] == 13)
        e = r > self || (J.mask != nullptr && J.mask[r] == 0);
    }
    emit |= (unsigned)e << k;
    nf_mine += e;
  }
  int nf;
  warp_excl_scan(nf_mine, lane, &nf);
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
      J.f_left[f] = self;
      J.f_right[f] = S.pright[pl];
      J.f_area[f] = fa[k];
      J.f_centroid[3 * f] = fcx[k] * na;
      J.f_centroid[3 * f + 1] = fcy[k] * na;
      J.f_centroid[3 * f + 2] = fcz[k] * na;
      J.f_normal[3 * f] = S.pnx[pl];
      J.f_normal[3 * f + 1] = S.pny[pl];
      J.f_normal[3 * f + 2] = S.pnz[pl];
      J.f_code[f] = S.pcode[pl];
    }
    rank_base += __popc(bal);
  }
  return CELL_DONE;
}

// Sets up neighbours [j, j + kb) of the sorted shell, one lane each: f64 location,
// offset and distance as the reference computes them (convex_cell.rs:333-342), plus
// the f32 quantities of the division-free filter.  Returns the ballots of neighbours
// whose distance is degenerate (*bad) and of those beyond the safety radius (*stop).
//
// Filter: for a vertex v = x + a and e = x - ngb,
//   s = e.a + |e|^2 / 2 = dist * M,   M = (n.v - d) up to the plane's rounding,
// and |s32| > T certifies sign(clip64) with |clip64| >= errb, where
//   T = dist * (errb_up + u64 (11 A + 11 |e|_1 + 14 |x|_1) + u32 (5.02 A + 4.03 dist))
// bounds the f64 rounding of n = e / dist, p = (x + ngb) / 2, d = n.p and n.v - d
// (u64 terms) and the f32 rounding of e, a and the three FMAs (u32 terms); A bounds
// |a| over the cell's vertices.
template <class T, int PREC>
__device__ __forceinline__ void setup_batch(const Job& J, CellSmem<T>& S, int lane, int j, int kb,
                                            D3 x, double x1, double sr, double A, unsigned* bad,
                                            unsigned* stop) {
  bool b = false, st = false;
  if (lane < kb) {
    const int c = j + lane;
    const uint32_t tie = S.u.g.tie[c];
    const int orig = (int)(tie / 27u);
    const int code = (int)(tie - (uint32_t)orig * 27u);
    const int sp = S.u.g.cpos[c];
    D3 ngb = {__ldg(J.sx + sp), __ldg(J.sy + sp), __ldg(J.sz + sp)};
    if (code != 13) ngb = add(ngb, D3{J.shift[code][0], J.shift[code][1], J.shift[code][2]});
    const D3 dx = sub(x, ngb);
    const double dist = sqrt(dot(dx, dx));
    b = !(dist > 0.0 && dist <= 1.7976931348623157e308);
    st = !b && sr < dist;
    S.u.g.bdx[lane] = dx.x, S.u.g.bdy[lane] = dx.y, S.u.g.bdz[lane] = dx.z;
    S.u.g.bdist[lane] = dist;
    S.u.g.bgx[lane] = ngb.x, S.u.g.bgy[lane] = ngb.y, S.u.g.bgz[lane] = ngb.z;
    S.u.g.borig[lane] = orig;
    S.u.g.bcode[lane] = (uint8_t)code;
    bool filt = false;
    if (PREC == MV_PRECISION_FILTERED) {
      filt = dist >= 1e-15 && dist <= 1e15 && A <= 1e15 && x1 <= 1e15;
      const float ex = __double2float_rn(dx.x), ey = __double2float_rn(dx.y),
                  ez = __double2float_rn(dx.z);
      const double e1 = fabs(dx.x) + fabs(dx.y) + fabs(dx.z);
      const double u32 = 5.9604644775390625e-08, u64 = 1.1102230246251565e-16;
      const double errb_up = 1e-13 * (1.0 + 1.001 * (x1 + e1)) * 1.0001;
      double Tb = dist * (errb_up + u64 * (11.0 * A + 11.0 * e1 + 14.0 * x1) +
                          u32 * (5.02 * A + 4.03 * dist));
      Tb = Tb * (1.0 + 1e-6) + 1e-40;
      S.u.g.bex[lane] = ex, S.u.g.bey[lane] = ey, S.u.g.bez[lane] = ez;
      S.u.g.bh[lane] = 0.5f * fmaf(ez, ez, fmaf(ey, ey, ex * ex));
      S.u.g.bT[lane] = __double2float_ru(Tb);
    }
    S.u.g.bfilt[lane] = filt;
  }
  *bad = __ballot_sync(FULL, b);
  *stop = __ballot_sync(FULL, st);
  __syncwarp();
}

template <class T, int PREC>
__device__ int build_cell(const Job& J, CellSmem<T>& S, int lane, int spos, const double* ext,
                          int* err_code, CellCount& cc) {
  using PIdx = typename T::PIdx;
  const int self = __ldg(J.sid + spos);
  const D3 x = load_gen(J, self);
  const int dim = J.dim;

  // ---- ConvexCell::init (convex_cell.rs:294-312) ----
  if (lane < 6) {
    S.pnx[lane] = J.bn[lane][0], S.pny[lane] = J.bn[lane][1], S.pnz[lane] = J.bn[lane][2];
    S.ppx[lane] = J.bp[lane][0], S.ppy[lane] = J.bp[lane][1], S.ppz[lane] = J.bp[lane][2];
    S.pd[lane] = J.bd[lane];
    S.pright[lane] = -1;
    S.pcode[lane] = 13;
  }
  for (int i = lane; i < T::VMAX; i += 32) S.ord[i] = (PIdx)i;
  __syncwarp();
  {
    // vertex duals of the cuboid (convex_cell.rs:298-307)
    int i0 = 0, i1 = 0, i2 = 0;
    switch (lane) {
      case 0: i0 = 2, i1 = 5, i2 = 0; break;
      case 1: i0 = 5, i1 = 3, i2 = 0; break;
      case 2: i0 = 1, i1 = 5, i2 = 2; break;
      case 3: i0 = 5, i1 = 1, i2 = 3; break;
      case 4: i0 = 4, i1 = 2, i2 = 0; break;
      case 5: i0 = 4, i1 = 0, i2 = 3; break;
      case 6: i0 = 2, i1 = 4, i2 = 1; break;
      default: i0 = 4, i1 = 3, i2 = 1; break;
    }
    bool ok = true;
    if (lane < 8) ok = make_vertex(S, lane, i0, i1, i2, x, dim);
    if (__any_sync(FULL, !ok)) {
      *err_code = MV_ERR_DET;
      return CELL_ERROR;
    }
  }
  __syncwarp();
  int nv = 8, np = 6;
  double max_r2 = warp_max(lane < 8 ? S.vr2[lane] : -1.0);
  double sr = 2.0 * sqrt(max_r2);
  double A = amax_of(max_r2, dim);
  const double x1 = fabs(x.x) + fabs(x.y) + fabs(x.z);

  // ---- ConvexCell::build neighbour loop (convex_cell.rs:316-356) ----
  double R = J.R0;
  double lo2 = 0.0;
  long long processed = 0;
  bool finished = false;
  int K = 1;  // neighbours set up per batch (adapts to runs of non-clipping neighbours)
  for (int shell = 0; !finished; shell++) {
    if (shell > 0) WCNT(cc, ST_SHELLS, 1);
    bool all;
    int cnt = gather_shell(J, S, lane, x, R, lo2, ext, &all);
    int shrink = 0;
    while (cnt > T::CMAX && shrink < 8) {
      // too many candidates for the shell buffer: pull the outer radius in
      const double rin = sqrt(lo2);
      R = rin + 0.5 * (R - rin);
      cnt = gather_shell(J, S, lane, x, R, lo2, ext, &all);
      shrink++;
    }
    if (cnt > T::CMAX) return CELL_OVERFLOW;
    sort_shell(S, lane, cnt);
    int j = 0;
    if (processed == 0 && cnt > 0) {
      // the first neighbour must be the generator itself (convex_cell.rs:325-329)
      if ((int)(S.u.g.tie[0] / 27u) != self) {
        *err_code = MV_ERR_DEGENERATE;
        return CELL_ERROR;
      }
      j = 1;
    }
    while (j < cnt) {
      const int kb = min(PREC == MV_PRECISION_FILTERED ? K : 1, cnt - j);
      unsigned bad, stop;
      setup_batch<T, PREC>(J, S, lane, j, kb, x, x1, sr, A, &bad, &stop);
      const int fb = bad ? __ffs(bad) - 1 : kb, fs = stop ? __ffs(stop) - 1 : kb;
      const int limit = min(fb, fs);
      // first neighbour in [0, limit) that may remove a vertex
      int kstar = limit;
      for (int k = 0; k < limit; k++) {
        bool need = !S.u.g.bfilt[k];
        if (!need) {
          const float ex = S.u.g.bex[k], ey = S.u.g.bey[k], ez = S.u.g.bez[k];
          const float h = S.u.g.bh[k], Tk = S.u.g.bT[k];
#pragma unroll
          for (int w = 0; w < T::NW; w++) {
            const int q = lane + 32 * w;
            if (q < nv) {
              const int sl = S.ord[q];
              const float s = fmaf(ez, S.fz[sl], fmaf(ey, S.fy[sl], fmaf(ex, S.fx[sl], h)));
              need = need || !(fabsf(s) > Tk) || s < 0.f;
            }
          }
        }
        if (__any_sync(FULL, need)) {
          kstar = k;
          break;
        }
      }
      WCNT(cc, ST_NEIGHBOURS, kstar);
      if (kstar == limit) {
        // neighbours [0, limit) remove nothing
        j += limit;
        if (limit < kb) {
          if (fb <= fs) {
            *err_code = MV_ERR_DEGENERATE;  // convex_cell.rs:342
            return CELL_ERROR;
          }
          finished = true;  // safety radius reached (convex_cell.rs:343-345)
          break;
        }
        K = min(2 * K, T::KMAX);
        continue;
      }
      WCNT(cc, ST_NEIGHBOURS, 1);
      // ---- neighbour kstar: HalfSpace::new (half_space.rs:24-34) and clip_by_plane ----
      const D3 dx = {S.u.g.bdx[kstar], S.u.g.bdy[kstar], S.u.g.bdz[kstar]};
      const double dist = S.u.g.bdist[kstar];
      const D3 ngb = {S.u.g.bgx[kstar], S.u.g.bgy[kstar], S.u.g.bgz[kstar]};
      const int orig = S.u.g.borig[kstar];
      const int code = S.u.g.bcode[kstar];
      const bool filt = S.u.g.bfilt[kstar];
      const float ex = S.u.g.bex[kstar], ey = S.u.g.bey[kstar], ez = S.u.g.bez[kstar];
      const float h = S.u.g.bh[kstar], Tk = S.u.g.bT[kstar];
      j += kstar + 1;
      K = 1;
      const D3 n = divs(dx, dist);
      const D3 p = scale(0.5, add(x, ngb));
      const double errb = 1e-13 * (1.0 + dot(vabs(n), vabs(p)));
      const double d = dot(n, p);
      unsigned rm[T::NW];
      int n_und = 0, n_ex = 0;
#pragma unroll
      for (int w = 0; w < T::NW; w++) {
        const int q = lane + 32 * w;
        bool removed = false;
        if (q < nv) {
          const int sl = S.ord[q];
          bool decided = false;
          if (PREC == MV_PRECISION_FILTERED && filt) {
            const float s = fmaf(ez, S.fz[sl], fmaf(ey, S.fy[sl], fmaf(ex, S.fx[sl], h)));
            if (fabsf(s) > Tk) {
              removed = s < 0.f;
              decided = true;
            }
          }
          if (!decided) {
            n_und++;
            const double c = dot(n, D3{S.vx[sl], S.vy[sl], S.vz[sl]}) - d;
            if (fabs(c) < errb) {
              removed = exact_clip(J, S, sl, x, ngb) < 0;
              n_ex++;
            } else {
              removed = c < 0.0;
            }
          }
        }
        rm[w] = __ballot_sync(FULL, removed);
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        n_und += __shfl_xor_sync(FULL, n_und, o);
        n_ex += __shfl_xor_sync(FULL, n_ex, o);
      }
      if (PREC == MV_PRECISION_FILTERED) WCNT(cc, ST_F32_UNDECIDED, n_und);
      WCNT(cc, ST_EXACT, n_ex);
      int nrem = 0;
#pragma unroll
      for (int w = 0; w < T::NW; w++) nrem += __popc(rm[w]);
      if (nrem == 0) continue;

      // ---- a vertex was clipped: add the plane (convex_cell.rs:393-418) ----
      if (np >= T::PMAX) return CELL_OVERFLOW;
      const int p_idx = np;
      if (lane == 0) {
        S.pnx[p_idx] = n.x, S.pny[p_idx] = n.y, S.pnz[p_idx] = n.z;
        S.ppx[p_idx] = p.x, S.ppy[p_idx] = p.y, S.ppz[p_idx] = p.z;
        S.pd[p_idx] = d;
        S.pright[p_idx] = orig;
        S.pcode[p_idx] = (uint8_t)code;
      }
      np++;
      WCNT(cc, ST_PLANES, 1);

      // swap-remove loop (convex_cell.rs:365-390) as a closed-form permutation of ord
      unsigned km[T::NW];
      int totK = 0;
#pragma unroll
      for (int w = 0; w < T::NW; w++) {
        km[w] = ~rm[w] & valid_bits(nv, w);
        totK += __popc(km[w]);
      }
      const int nvf = totK;
      {
        int dest[T::NW];
        PIdx held[T::NW];
#pragma unroll
        for (int w = 0; w < T::NW; w++) {
          const int q = lane + 32 * w;
          int dd = -1;
          held[w] = 0;
          if (q < nv) {
            held[w] = S.ord[q];
            if (!((rm[w] >> lane) & 1u)) {
              dd = q < nvf ? q : select_bit<T::NW>(rm, totK - rank_below<T::NW>(km, q));
            } else if (q <= nvf) {
              const int t = rank_below<T::NW>(rm, q) + 1;
              dd = ((t == 1) ? nv : select_bit<T::NW>(km, totK - t + 2)) - 1;
            } else {
              dd = q - 1;
            }
          }
          dest[w] = dd;
        }
        __syncwarp();
#pragma unroll
        for (int w = 0; w < T::NW; w++)
          if (dest[w] >= 0) S.ord[dest[w]] = held[w];
        __syncwarp();
      }

      // ring of the removed region (compute_boundary + SimpleCycle iteration)
      int E = ring_parallel(S, lane, nvf, nv);
      if (E < 0) {
        WCNT(cc, ST_SERIAL_RING, 1);
        int e2 = 0;
        if (lane == 0) e2 = ring_serial(S, nvf, nv, np);
        E = __shfl_sync(FULL, e2, 0);
        __syncwarp();
        if (E == -2) return CELL_OVERFLOW;
        if (E < 0) {
          *err_code = MV_ERR_RING;
          return CELL_ERROR;
        }
      }
      if (nvf + E > T::VMAX) return CELL_OVERFLOW;
      bool ok = true;
      for (int e = lane; e < E; e += 32)
        ok &= make_vertex(S, S.ord[nvf + e], S.ea[e], S.eb[e], p_idx, x, dim);
      if (__any_sync(FULL, !ok)) {
        *err_code = MV_ERR_DET;
        return CELL_ERROR;
      }
      __syncwarp();
      nv = nvf + E;
      // update_safety_radius (convex_cell.rs:443-453)
      double m = -1.0;
      for (int q = lane; q < nv; q += 32) m = fmax(m, S.vr2[S.ord[q]]);
      max_r2 = warp_max(m);
      sr = 2.0 * sqrt(max_r2);
      A = amax_of(max_r2, dim);
    }
    if (finished) break;
    processed += cnt;
    if (all) break;
    if (sr < R * (1.0 - 1e-12)) break;
    lo2 = R * R;
    R = fmax(R * 1.3, sr * 1.05);
  }
  return integrate_cell(J, S, lane, self, x, nv, np, sr, err_code);
}

template <class T, int PREC, int WARPS>
__global__ void __launch_bounds__(32 * WARPS, T::MINB) cells_kernel(const __grid_constant__ Job J) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  CellSmem<T>& S = reinterpret_cast<CellSmem<T>*>(smem_raw)[warp];
  __shared__ double ext_s[6];
  if (threadIdx.x < 6) ext_s[threadIdx.x] = J.ext[threadIdx.x];
  if (lane < ST_COUNT) S.cnt[lane] = 0ull;
  __syncthreads();
  const int total = J.order ? J.n_order : J.n;
  for (;;) {
    int item = 0;
    if (lane == 0) item = (int)atomicAdd(J.work_counter, 1u);
    item = __shfl_sync(FULL, item, 0);
    if (item >= total) break;
    const int spos = J.order ? J.order[item] : item;
    const int self = __ldg(J.sid + spos);
    if (J.mask != nullptr && J.mask[self] == 0) {
      // VoronoiCell::default() (voronoi.rs:303-305)
      if (lane < 3) J.centroid[3 * (int64_t)self + lane] = 0.0;
      if (lane == 0) {
        J.volume[self] = 0.0;
        J.safety_radius[self] = 0.0;
        J.face_count[self] = 0;
        J.stage_off[self] = 0;
      }
      continue;
    }
    int err = 0;
    CellCount cc;
#pragma unroll
    for (int i = 0; i < ST_COUNT; i++) cc.c[i] = 0u;
    const int res = build_cell<T, PREC>(J, S, lane, spos, ext_s, &err, cc);
    __syncwarp();
    if (res == CELL_DONE) cc.c[ST_CELLS]++;
    if (lane == 0) {
#pragma unroll
      for (int i = 0; i < ST_COUNT; i++) S.cnt[i] += cc.c[i];
    }
    __syncwarp();
    if (res == CELL_OVERFLOW) {
      if (lane == 0) {
        unsigned k = atomicAdd(J.ovf_count, 1u);
        J.ovf_list[k] = spos;
        S.cnt[ST_OVERFLOW]++;
      }
    } else if (res == CELL_FACE_OVERFLOW) {
      if (lane == 0) atomicExch(J.status + STATUS_FACE_OVERFLOW, 1);
    } else if (res == CELL_ERROR) {
      if (lane == 0) {
        atomicCAS(J.status + STATUS_CODE, 0, err);
        atomicMin(J.status + STATUS_CELL, self);
      }
    }
    __syncwarp();
  }
  __syncwarp();
  if (lane < ST_COUNT && S.cnt[lane]) atomicAdd(J.stats + lane, S.cnt[lane]);
}

// ---------------------------------------------------------------- launchers --
constexpr int FAST_WARPS = 4;
constexpr int LARGE_WARPS = 1;

template <class T, int PREC, int WARPS>
static int blocks_per_sm() {
  int nb = 0;
  const size_t smem = sizeof(CellSmem<T>) * WARPS;
  auto k = cells_kernel<T, PREC, WARPS>;
  if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
    return 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k, 32 * WARPS, smem) != cudaSuccess) return 0;
  return nb;
}

template <class T, int PREC, int WARPS>
static cudaError_t launch_tier(const Job& J, int blocks, cudaStream_t st) {
  const size_t smem = sizeof(CellSmem<T>) * WARPS;
  auto k = cells_kernel<T, PREC, WARPS>;
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  k<<<blocks, 32 * WARPS, smem, st>>>(J);
  return cudaGetLastError();
}

int cells_blocks_per_sm_fast(int precision) {
  return precision == MV_PRECISION_FILTERED
             ? blocks_per_sm<TierFast, MV_PRECISION_FILTERED, FAST_WARPS>()
             : blocks_per_sm<TierFast, MV_PRECISION_FP64, FAST_WARPS>();
}

int cells_blocks_per_sm_large(int precision) {
  return precision == MV_PRECISION_FILTERED
             ? blocks_per_sm<TierLarge, MV_PRECISION_FILTERED, LARGE_WARPS>()
             : blocks_per_sm<TierLarge, MV_PRECISION_FP64, LARGE_WARPS>();
}

cudaError_t launch_cells(const Job& J, bool large, int blocks, cudaStream_t st) {
  if (!large) {
    if (J.precision == MV_PRECISION_FILTERED)
      return launch_tier<TierFast, MV_PRECISION_FILTERED, FAST_WARPS>(J, blocks, st);
    return launch_tier<TierFast, MV_PRECISION_FP64, FAST_WARPS>(J, blocks, st);
  }
  if (J.precision == MV_PRECISION_FILTERED)
    return launch_tier<TierLarge, MV_PRECISION_FILTERED, LARGE_WARPS>(J, blocks, st);
  return launch_tier<TierLarge, MV_PRECISION_FP64, LARGE_WARPS>(J, blocks, st);
}

}  // namespace mv
