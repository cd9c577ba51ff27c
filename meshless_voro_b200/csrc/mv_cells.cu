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
//   * the swap-remove loop of clip_by_plane is applied as a closed-form permutation
//     derived from the ballot of removed vertices;
//   * the SimpleCycle ring is the boundary of the removed vertices' dual triangles,
//     started where the reference starts it (serial replay when that node vanished);
//   * cell and face integrals are summed in the reference's tet order.
// Hence vertices, topology and integrals are the same binary64 values the
// reference computes.
#include <cstdint>

#include "../../include/mvgpu.h"
#include "mv_exact.cuh"
#include "mv_geom.cuh"
#include "mv_internal.h"

namespace mv {

constexpr unsigned FULL = 0xffffffffu;

template <int VMAX_, int PMAX_, int CMAX_, typename PIdx_, int MINB_>
struct Tier {
  static constexpr int MINB = MINB_;  // min resident blocks per SM (register budget)
  static constexpr int VMAX = VMAX_;
  static constexpr int PMAX = PMAX_;
  static constexpr int CMAX = CMAX_;
  static constexpr int NW = VMAX / 32;  // vertex mask words
  using PIdx = PIdx_;
  static constexpr unsigned NONE = (unsigned)(PIdx)(~0u);
  static_assert(VMAX % 32 == 0 && PMAX % 32 == 0 && CMAX % 32 == 0, "tier sizes");
  static_assert(PMAX < (int)NONE, "plane index type too small");
};

// Resident blocks per SM the fast tier is compiled for (sets its register budget).
#ifndef MV_FAST_MINB
#define MV_FAST_MINB 4
#endif
using TierFast = Tier<64, 64, 128, uint8_t, MV_FAST_MINB>;
using TierLarge = Tier<512, 512, 512, uint16_t, 1>;

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
  // vertices (convex_cell.rs:16-25), reference order
  double vx[T::VMAX], vy[T::VMAX], vz[T::VMAX], vr2[T::VMAX];
  float fx[T::VMAX], fy[T::VMAX], fz[T::VMAX];  // f32 (v - x) for the filter
  PIdx vd0[T::VMAX], vd1[T::VMAX], vd2[T::VMAX];
  PIdx ea[T::VMAX], eb[T::VMAX];  // ring edges in SimpleCycle iteration order
  unsigned long long cnt[ST_COUNT];  // per-warp counters (flushed at exit)
  union {
    struct {
      unsigned long long key[T::CMAX];
      uint32_t tie[T::CMAX];
      int32_t sstart[96];
      int32_t spref[97];
      uint8_t scode[96];
    } g;
    struct {
      double val[8][32];
      int32_t plane[32];
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
    if (code != 13) l = add(l, shift_of_code(code, J.gw));
    return l;
  }
  D3 pr = plane_project({S.pnx[k], S.pny[k], S.pnz[k]}, {S.ppx[k], S.ppy[k], S.ppz[k]}, x);
  return sub(scale(2.0, pr), x);
}

// Exact decision of clip_by_plane for an undecided vertex (convex_cell.rs:370-382).
template <class T>
__device__ __noinline__ int exact_clip(const Job& J, const CellSmem<T>& S, int v, D3 x, D3 ngb) {
  int64_t A[3], B[3], C[3], Dd[3], W[3];
  iloc(J, x, A);
  iloc(J, right_loc(J, S, S.vd0[v], x), B);
  iloc(J, right_loc(J, S, S.vd1[v], x), C);
  iloc(J, right_loc(J, S, S.vd2[v], x), Dd);
  iloc(J, ngb, W);
  return in_sphere_exact_sign(A, B, C, Dd, W);
}

// Vertex::from_dual (convex_cell.rs:28-48); writes vertex slot `slot`.
template <class T>
__device__ __noinline__ bool make_vertex(CellSmem<T>& S, int slot, int i, int j, int k, D3 x,
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
__device__ __noinline__ int gather_shell(const Job& J, CellSmem<T>& S, int lane, D3 x, double R, double lo2,
                            const double* ext, bool* exhausted) {
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
    int32_t s0[3] = {0, 0, 0}, sl[3] = {0, 0, 0};
    int sc[3] = {0, 0, 0};
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
            s0[nseg] = ps;
            sl[nseg] = pe - ps;
            sc[nseg] = (mx + 1) + 3 * (my + 1) + 9 * (mz + 1);
            nseg++;
          }
        }
      }
    }
    int nsegs_total;
    const int segoff = warp_excl_scan(nseg, lane, &nsegs_total);
    const int mylen = sl[0] + sl[1] + sl[2];
    int total;
    const int lenoff = warp_excl_scan(mylen, lane, &total);
    {
      int run = lenoff;
      for (int k = 0; k < nseg; k++) {
        S.u.g.sstart[segoff + k] = s0[k];
        S.u.g.spref[segoff + k] = run;
        S.u.g.scode[segoff + k] = (uint8_t)sc[k];
        run += sl[k];
      }
    }
    __syncwarp();
    for (int t0 = 0; t0 < total; t0 += 32) {
      const int t = t0 + lane;
      bool keep = false;
      double d2 = 0.0;
      uint32_t tie = 0;
      if (t < total) {
        int a = 0, b = nsegs_total - 1;
        while (a < b) {
          int mid = (a + b + 1) >> 1;
          if (S.u.g.spref[mid] <= t)
            a = mid;
          else
            b = mid - 1;
        }
        const int s = S.u.g.sstart[a] + (t - S.u.g.spref[a]);
        const int code = S.u.g.scode[a];
        const double px = __ldg(J.sx + s), py = __ldg(J.sy + s), pz = __ldg(J.sz + s);
        const int orig = __ldg(J.sid + s);
        if (J.periodic) {
          const int mx = code % 3 - 1, my = (code / 3) % 3 - 1, mz = code / 9 - 1;
          const double ddx = (x.x + (double)(-mx) * J.gw[0]) - px;
          const double ddy = (x.y + (double)(-my) * J.gw[1]) - py;
          const double ddz = (x.z + (double)(-mz) * J.gw[2]) - pz;
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
      }
      count += __popc(bal);
    }
    __syncwarp();
  }
  *exhausted = all && !__any_sync(FULL, beyond > 0);
  return count;
}

// Bitonic sort of S.u.g.(key, tie)[0, n) ascending; n <= CMAX, padded to a power of 2.
template <class T>
__device__ __noinline__ void sort_shell(CellSmem<T>& S, int lane, int n) {
  int np2 = 32;
  while (np2 < n) np2 <<= 1;
  for (int i = n + lane; i < np2; i += 32) {
    S.u.g.key[i] = ~0ull;
    S.u.g.tie[i] = ~0u;
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
          S.u.g.key[lo] = kb;
          S.u.g.key[hi] = ka;
          S.u.g.tie[lo] = tb;
          S.u.g.tie[hi] = ta;
        }
      }
      __syncwarp();
    }
  }
}

// -------------------------------------------------------------------- ring --
// Serial replay of compute_boundary (convex_cell.rs:421-441) and SimpleCycle
// (simple_cycle.rs:17-78) on lane 0 for the removed vertices at [nvf, nv).
// Produces the edge list (S.ea, S.eb) and returns its length, or -1 on failure.
template <class T>
__device__ __noinline__ int ring_serial(CellSmem<T>& S, int nvf, int nv, int np) {
  using PIdx = typename T::PIdx;
  for (int i = 0; i < np; i++) S.rptr[i] = (PIdx)i;
  auto contains = [&](int i) { return S.rptr[i] != (PIdx)i; };
  int start = S.vd0[nvf];
  int len = 3;
  {
    int a = S.vd0[nvf], b = S.vd1[nvf], c = S.vd2[nvf];
    S.rptr[a] = (PIdx)b;
    S.rptr[b] = (PIdx)c;
    S.rptr[c] = (PIdx)a;
  }
  const int n = nv - nvf;
  for (int i = 1; i < n; i++) {
    int idx = i;
    for (;;) {
      if (idx >= n) return -1;
      const int v = nvf + idx;
      const int tri[3] = {S.vd0[v], S.vd1[v], S.vd2[v]};
      const bool in[3] = {contains(tri[0]), contains(tri[1]), contains(tri[2])};
      bool ok = false;
      for (int a = 0; a < 3 && !ok; a++) {
        const int b = (a + 1) % 3, c = (a + 2) % 3;
        if (!in[a] && in[b] && in[c] && S.rptr[tri[c]] == (PIdx)tri[b]) {
          S.rptr[tri[c]] = (PIdx)tri[a];
          S.rptr[tri[a]] = (PIdx)tri[b];
          len += 1;
          ok = true;
        } else if (in[a] && in[b] && in[c] && S.rptr[tri[c]] == (PIdx)tri[b] &&
                   S.rptr[tri[b]] == (PIdx)tri[a]) {
          S.rptr[tri[c]] = (PIdx)tri[a];
          S.rptr[tri[b]] = (PIdx)tri[b];
          if (start == tri[b]) start = tri[a];
          len -= 1;
          ok = true;
        }
      }
      if (ok) {
        if (idx > i) {
          const int w = nvf + i;
          PIdx t0 = S.vd0[w], t1 = S.vd1[w], t2 = S.vd2[w];
          S.vd0[w] = S.vd0[v], S.vd1[w] = S.vd1[v], S.vd2[w] = S.vd2[v];
          S.vd0[v] = t0, S.vd1[v] = t1, S.vd2[v] = t2;
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
__device__ __noinline__ int ring_parallel(CellSmem<T>& S, int lane, int nvf, int nv) {
  using PIdx = typename T::PIdx;
  const int r = nv - nvf;
  for (int q = lane; q < r; q += 32) {
    const int v = nvf + q;
    S.rptr[S.vd0[v]] = (PIdx)T::NONE;
    S.rptr[S.vd1[v]] = (PIdx)T::NONE;
    S.rptr[S.vd2[v]] = (PIdx)T::NONE;
  }
  __syncwarp();
  int myedges = 0;
  bool conflict = false;
  int eu[3], ew[3];
  for (int q = lane; q < r; q += 32) {
    const int v = nvf + q;
    const int t[3] = {S.vd0[v], S.vd1[v], S.vd2[v]};
    for (int e = 0; e < 3; e++) {
      const int u = t[e], w = t[(e + 1) % 3];
      bool internal = false;
      for (int k = 0; k < r && !internal; k++) {
        if (k == q) continue;
        const int o = nvf + k;
        const int a = S.vd0[o], b = S.vd1[o], c = S.vd2[o];
        internal = (a == w && b == u) || (b == w && c == u) || (c == w && a == u);
      }
      if (!internal) {
        S.rptr[u] = (PIdx)w;
        if (r <= 32) {
          eu[myedges] = u;
          ew[myedges] = w;
        }
        myedges++;
      }
    }
  }
  __syncwarp();
  if (r <= 32) {
    for (int e = 0; e < myedges; e++) conflict |= (S.rptr[eu[e]] != (PIdx)ew[e]);
  } else {
    conflict = true;  // large removal sets: let the serial replay decide
  }
  if (__any_sync(FULL, conflict)) return -1;
  int E;
  warp_excl_scan(myedges, lane, &E);
  const int start = S.vd0[nvf];
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
// Per-warp counters live in shared memory (lane 0 updates them).
#define WCNT(S, slot, v) \
  do {                   \
    if (lane == 0) (S).cnt[slot] += (unsigned long long)(v); \
  } while (0)

// Integrals and face emission of a finished cell (convex_cell.rs:131-187,
// voronoi_cell.rs:40-100).  Tets go through 30-lane steps (5 vertices x 6 tets);
// lanes 0-3 sum the cell integrals and lane p owns face p (and p + 32k), all in the
// reference's tet order.
template <class T>
__device__ __noinline__ int integrate_cell(const Job& J, CellSmem<T>& S, int lane, int self, D3 x,
                                           int nv, int np, double sr, int* err_code) {
  const int dim = J.dim;
  double cacc = 0.0;  // lanes 0..3: volume, centroid x, y, z
  double fa[T::PMAX / 32], fcx[T::PMAX / 32], fcy[T::PMAX / 32], fcz[T::PMAX / 32];
  unsigned ftouched = 0;
#pragma unroll
  for (int k = 0; k < T::PMAX / 32; k++) fa[k] = 0.0, fcx[k] = 0.0, fcy[k] = 0.0, fcz[k] = 0.0;
  const int vl = lane / 6, tt = lane - 6 * (lane / 6);
  for (int base = 0; base < nv; base += 5) {
    const int v = base + vl;
    const bool act = lane < 30 && v < nv;
    D3 pr = {0.0, 0.0, 0.0};
    bool ok = true;
    int plane = 0;
    D3 vloc = {0.0, 0.0, 0.0};
    if (act) {
      const int i = tt >> 1;
      const int d0 = S.vd0[v], d1 = S.vd1[v], d2 = S.vd2[v];
      const int cur = i == 0 ? d0 : (i == 1 ? d1 : d2);
      const D3 cn = {S.pnx[cur], S.pny[cur], S.pnz[cur]};
      if ((tt & 1) == 0) {
        pr = plane_project(cn, {S.ppx[cur], S.ppy[cur], S.ppz[cur]}, x);
      } else {
        const int nx = i == 0 ? d1 : (i == 1 ? d2 : d0);
        const D3 nn = {S.pnx[nx], S.pny[nx], S.pnz[nx]};
        const D3 perp = cross(nn, cn);
        ok = intersect3(nn, S.pd[nx], cn, S.pd[cur], perp, dot(x, perp), &pr);
      }
      plane = cur;
      vloc = {S.vx[v], S.vy[v], S.vz[v]};
    }
    if (__any_sync(FULL, !ok)) {
      *err_code = MV_ERR_DET;
      return CELL_ERROR;
    }
    // proj[(t + 5) % 6] lives on lane 6 vl + (t + 5) % 6
    const int src = 6 * vl + (tt + 5) % 6;
    const int srcl = src < 32 ? src : lane;
    D3 pq;
    pq.x = __shfl_sync(FULL, pr.x, srcl);
    pq.y = __shfl_sync(FULL, pr.y, srcl);
    pq.z = __shfl_sync(FULL, pr.z, srcl);
    if (act) {
      const double vol = signed_volume_tet(pr, pq, vloc, x);
      const D3 vc = scale(vol, add(add(add(pr, pq), vloc), x));
      const double ar = signed_area_tri(pr, pq, vloc, x);
      const D3 ac = scale(ar, add(add(pr, pq), vloc));
      S.u.t.val[0][lane] = vol;
      S.u.t.val[1][lane] = vc.x;
      S.u.t.val[2][lane] = vc.y;
      S.u.t.val[3][lane] = vc.z;
      S.u.t.val[4][lane] = ar;
      S.u.t.val[5][lane] = ac.x;
      S.u.t.val[6][lane] = ac.y;
      S.u.t.val[7][lane] = ac.z;
      S.u.t.plane[lane] = plane;
    }
    __syncwarp();
    const int ntet = 6 * min(5, nv - base);
    if (lane < 4) {
      for (int s = 0; s < ntet; s++) cacc = cacc + S.u.t.val[lane][s];
    }
#pragma unroll
    for (int k = 0; k < T::PMAX / 32; k++) {
      const int pl = lane + 32 * k;
      if (pl < np) {
        for (int s = 0; s < ntet; s++) {
          if (S.u.t.plane[s] == pl) {
            fa[k] = fa[k] + S.u.t.val[4][s];
            fcx[k] = fcx[k] + S.u.t.val[5][s];
            fcy[k] = fcy[k] + S.u.t.val[6][s];
            fcz[k] = fcz[k] + S.u.t.val[7][s];
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
  WCNT(S, ST_CELLS, 1);
  return CELL_DONE;
}


template <class T, int PREC>
__device__ int build_cell(const Job& J, CellSmem<T>& S, int lane, int spos, const double* ext,
                          int* err_code) {
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
  const double x1 = fabs(x.x) + fabs(x.y) + fabs(x.z);

  // ---- ConvexCell::build neighbour loop (convex_cell.rs:316-356) ----
  double R = J.R0;
  double lo2 = 0.0;
  long long processed = 0;
  bool finished = false;
  for (int shell = 0; !finished; shell++) {
    if (shell > 0) WCNT(S, ST_SHELLS, 1);
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
    for (int j = 0; j < cnt; j++) {
      const uint32_t tie = S.u.g.tie[j];
      const int orig = (int)(tie / 27u);
      const int code = (int)(tie - (uint32_t)orig * 27u);
      if (processed + j == 0) {
        if (orig != self) {
          *err_code = MV_ERR_DEGENERATE;
          return CELL_ERROR;
        }
        continue;
      }
      D3 ngb = load_gen(J, orig);
      if (code != 13) ngb = add(ngb, shift_of_code(code, J.gw));
      const D3 dx = sub(x, ngb);
      const double dist = sqrt(dot(dx, dx));
      if (!(dist > 0.0 && dist <= 1.7976931348623157e308)) {
        *err_code = MV_ERR_DEGENERATE;
        return CELL_ERROR;
      }
      if (sr < dist) {
        finished = true;
        break;
      }
      WCNT(S, ST_NEIGHBOURS, 1);

      // Per-vertex decisions of clip_by_plane (convex_cell.rs:365-390).  rm: removed,
      // und: not yet decided.  In filtered mode a division-free f32 test decides first:
      //   sign(n.v - d) == sign((x - ngb).(v - x) + |x - ngb|^2 / 2)
      // and |s32| > T certifies sign(clip64) with |clip64| >= errb, where T bounds the
      // rounding of both the f32 evaluation and the reference's f64 plane.
      unsigned rm[T::NW], und[T::NW];
      bool need_plane = true;
      const double A = amax_of(max_r2, dim);
      const bool filt = (PREC == MV_PRECISION_FILTERED) && dist >= 1e-15 && dist <= 1e15 &&
                        A <= 1e15 && x1 <= 1e15;
      if (filt) {
        const float ex = __double2float_rn(dx.x), ey = __double2float_rn(dx.y),
                    ez = __double2float_rn(dx.z);
        const float h32 = 0.5f * fmaf(ez, ez, fmaf(ey, ey, ex * ex));
        const double e1 = fabs(dx.x) + fabs(dx.y) + fabs(dx.z);
        const double u32 = 5.9604644775390625e-08, u64 = 1.1102230246251565e-16;
        const double errb_up = 1e-13 * (1.0 + 1.001 * (x1 + e1)) * 1.0001;
        double Tb = dist * (errb_up + u64 * (11.0 * A + 11.0 * e1 + 14.0 * x1) +
                            u32 * (5.02 * A + 4.03 * dist));
        Tb = Tb * (1.0 + 1e-6) + 1e-40;
        const float T32 = __double2float_ru(Tb);
        unsigned any = 0;
#pragma unroll
        for (int w = 0; w < T::NW; w++) {
          const int v = lane + 32 * w;
          bool rem = false, un = false;
          if (v < nv) {
            const float s = fmaf(ez, S.fz[v], fmaf(ey, S.fy[v], fmaf(ex, S.fx[v], h32)));
            const bool cert = fabsf(s) > T32;
            rem = cert && s < 0.f;
            un = !cert;
          }
          rm[w] = __ballot_sync(FULL, rem);
          und[w] = __ballot_sync(FULL, un);
          any |= rm[w] | und[w];
        }
        need_plane = any != 0;
      } else {
#pragma unroll
        for (int w = 0; w < T::NW; w++) {
          const int lim = nv - 32 * w;
          rm[w] = 0u;
          und[w] = lim >= 32 ? FULL : (lim <= 0 ? 0u : ((1u << lim) - 1u));
        }
      }
      if (!need_plane) continue;  // certified: the half-space removes no vertex

      // HalfSpace::new (half_space.rs:24-34)
      const D3 n = divs(dx, dist);
      const D3 p = scale(0.5, add(x, ngb));
      const double errb = 1e-13 * (1.0 + dot(vabs(n), vabs(p)));
      const double d = dot(n, p);
      int n_und = 0, n_ex = 0;
#pragma unroll
      for (int w = 0; w < T::NW; w++) {
        n_und += __popc(und[w]);
        const int v = lane + 32 * w;
        bool removed = false;
        if ((und[w] >> lane) & 1u) {
          const double c = dot(n, D3{S.vx[v], S.vy[v], S.vz[v]}) - d;
          if (fabs(c) < errb) {
            removed = exact_clip(J, S, v, x, ngb) < 0;
            n_ex++;
          } else {
            removed = c < 0.0;
          }
        }
        rm[w] |= __ballot_sync(FULL, removed);
      }
      if (PREC == MV_PRECISION_FILTERED) WCNT(S, ST_F32_UNDECIDED, filt ? n_und : 0);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) n_ex += __shfl_xor_sync(FULL, n_ex, o);
      WCNT(S, ST_EXACT, n_ex);
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
      WCNT(S, ST_PLANES, 1);

      // swap-remove permutation as a closed form of the ballot
      unsigned km[T::NW];
      int totK = 0;
#pragma unroll
      for (int w = 0; w < T::NW; w++) {
        const int lim = nv - 32 * w;
        const unsigned valid = lim >= 32 ? FULL : (lim <= 0 ? 0u : ((1u << lim) - 1u));
        km[w] = ~rm[w] & valid;
        totK += __popc(km[w]);
      }
      const int nvf = totK;
      int dest[T::NW];
#pragma unroll
      for (int w = 0; w < T::NW; w++) {
        const int v = lane + 32 * w;
        int dd = -1;
        if (v < nv) {
          const bool isrem = (rm[w] >> lane) & 1u;
          if (!isrem) {
            dd = v < nvf ? v : select_bit<T::NW>(rm, totK - rank_below<T::NW>(km, v));
          } else if (v <= nvf) {
            const int t = rank_below<T::NW>(rm, v) + 1;
            dd = ((t == 1) ? nv : select_bit<T::NW>(km, totK - t + 2)) - 1;
          } else {
            dd = v - 1;
          }
        }
        dest[w] = dd;
      }
      // scatter field by field (few live registers); removed vertices keep only duals
      auto scatter_d = [&](double* a, bool kept_only) {
        double t[T::NW];
#pragma unroll
        for (int w = 0; w < T::NW; w++) {
          const int v = lane + 32 * w;
          t[w] = v < nv ? a[v] : 0.0;
        }
        __syncwarp();
#pragma unroll
        for (int w = 0; w < T::NW; w++)
          if (dest[w] >= 0 && (!kept_only || dest[w] < nvf)) a[dest[w]] = t[w];
        __syncwarp();
      };
      auto scatter_f = [&](float* a) {
        float t[T::NW];
#pragma unroll
        for (int w = 0; w < T::NW; w++) {
          const int v = lane + 32 * w;
          t[w] = v < nv ? a[v] : 0.f;
        }
        __syncwarp();
#pragma unroll
        for (int w = 0; w < T::NW; w++)
          if (dest[w] >= 0 && dest[w] < nvf) a[dest[w]] = t[w];
        __syncwarp();
      };
      auto scatter_i = [&](PIdx* a) {
        PIdx t[T::NW];
#pragma unroll
        for (int w = 0; w < T::NW; w++) {
          const int v = lane + 32 * w;
          t[w] = v < nv ? a[v] : (PIdx)0;
        }
        __syncwarp();
#pragma unroll
        for (int w = 0; w < T::NW; w++)
          if (dest[w] >= 0) a[dest[w]] = t[w];
        __syncwarp();
      };
      scatter_d(S.vx, true);
      scatter_d(S.vy, true);
      scatter_d(S.vz, true);
      scatter_d(S.vr2, true);
      scatter_f(S.fx);
      scatter_f(S.fy);
      scatter_f(S.fz);
      scatter_i(S.vd0);
      scatter_i(S.vd1);
      scatter_i(S.vd2);

      // ring of the removed region (compute_boundary + SimpleCycle iteration)
      int E = ring_parallel(S, lane, nvf, nv);
      if (E < 0) {
        WCNT(S, ST_SERIAL_RING, 1);
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
        ok &= make_vertex(S, nvf + e, S.ea[e], S.eb[e], p_idx, x, dim);
      if (__any_sync(FULL, !ok)) {
        *err_code = MV_ERR_DET;
        return CELL_ERROR;
      }
      __syncwarp();
      nv = nvf + E;
      // update_safety_radius (convex_cell.rs:443-453)
      double m = -1.0;
      for (int v = lane; v < nv; v += 32) m = fmax(m, S.vr2[v]);
      max_r2 = warp_max(m);
      sr = 2.0 * sqrt(max_r2);
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
    const int res = build_cell<T, PREC>(J, S, lane, spos, ext_s, &err);
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


template <class T, int PREC, int WARPS>
static cudaError_t launch_tier(const Job& J, int blocks, cudaStream_t st) {
  const size_t smem = sizeof(CellSmem<T>) * WARPS;
  auto k = cells_kernel<T, PREC, WARPS>;
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  k<<<blocks, 32 * WARPS, smem, st>>>(J);
  return cudaGetLastError();
}

constexpr int FAST_WARPS = 4;
constexpr int LARGE_WARPS = 1;

size_t cells_smem_fast() { return sizeof(CellSmem<TierFast>) * FAST_WARPS; }
size_t cells_smem_large() { return sizeof(CellSmem<TierLarge>) * LARGE_WARPS; }

int cells_blocks_per_sm_fast(int precision) {
  int nb = 0;
  const size_t smem = cells_smem_fast();
  if (precision == MV_PRECISION_FILTERED) {
    cudaFuncSetAttribute(cells_kernel<TierFast, MV_PRECISION_FILTERED, FAST_WARPS>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &nb, cells_kernel<TierFast, MV_PRECISION_FILTERED, FAST_WARPS>, 32 * FAST_WARPS, smem);
  } else {
    cudaFuncSetAttribute(cells_kernel<TierFast, MV_PRECISION_FP64, FAST_WARPS>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &nb, cells_kernel<TierFast, MV_PRECISION_FP64, FAST_WARPS>, 32 * FAST_WARPS, smem);
  }
  return nb;
}

int cells_blocks_per_sm_large(int precision) {
  int nb = 0;
  const size_t smem = cells_smem_large();
  if (precision == MV_PRECISION_FILTERED) {
    cudaFuncSetAttribute(cells_kernel<TierLarge, MV_PRECISION_FILTERED, LARGE_WARPS>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &nb, cells_kernel<TierLarge, MV_PRECISION_FILTERED, LARGE_WARPS>, 32 * LARGE_WARPS, smem);
  } else {
    cudaFuncSetAttribute(cells_kernel<TierLarge, MV_PRECISION_FP64, LARGE_WARPS>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &nb, cells_kernel<TierLarge, MV_PRECISION_FP64, LARGE_WARPS>, 32 * LARGE_WARPS, smem);
  }
  return nb;
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
