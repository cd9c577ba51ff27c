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
#include <algorithm>
#include <cstdint>

#include "mv_cell_common.cuh"

namespace mv {

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
  float4 f4[T::VMAX];  // f32 (v - x) for the filter
  alignas(4) PIdx ord[T::VMAX];   // position -> slot; [0, nv) is the reference's order
  PIdx vd0[T::VMAX], vd1[T::VMAX], vd2[T::VMAX];
  PIdx ea[T::VMAX], eb[T::VMAX];  // ring edges in SimpleCycle iteration order
  unsigned long long cnt[ST_COUNT];  // per-warp event counts (flushed to global at exit)
  __device__ D3 plane_point(const Job&, int k) const { return {ppx[k], ppy[k], ppz[k]}; }
  __device__ D3 bisector_point(const Job&, int k, D3) const { return {ppx[k], ppy[k], ppz[k]}; }
  union {
    struct {  // clipping phase
      ShellBuf<T::CMAX> sh;
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
      TetScratch<5> ts;
    } t;
  } u;
};

// The finished cell as the integral step reads it (fused kernel: shared memory).
template <class T>
struct SmemView {
  const CellSmem<T>& S;
  __device__ D3 normal(int pl) const { return {S.pnx[pl], S.pny[pl], S.pnz[pl]}; }
  __device__ double d(int pl) const { return S.pd[pl]; }
  __device__ D3 proj(int pl) const { return {S.u.t.px[pl], S.u.t.py[pl], S.u.t.pz[pl]}; }
  __device__ int right(int pl) const { return S.pright[pl]; }
  __device__ int code(int pl) const { return S.pcode[pl]; }
  __device__ int dual(int q, int i) const {
    const int sl = S.ord[q];
    return i == 0 ? S.vd0[sl] : (i == 1 ? S.vd1[sl] : S.vd2[sl]);
  }
  __device__ D3 loc(int q) const {
    const int sl = S.ord[q];
    return {S.vx[sl], S.vy[sl], S.vz[sl]};
  }
};

// Integrals of a finished cell held in shared memory: the generator's projection on
// each plane is computed once per plane, then integrate_view sums the tets.
template <class T>
__device__ __noinline__ int integrate_cell(const Job& J, CellSmem<T>& S, int lane, int self, D3 x,
                                           int nv, int np, double sr, int* err_code) {
  for (int pl = lane; pl < np; pl += 32) {
    const D3 pr = plane_project({S.pnx[pl], S.pny[pl], S.pnz[pl]},
                                {S.ppx[pl], S.ppy[pl], S.ppz[pl]}, x);
    S.u.t.px[pl] = pr.x;
    S.u.t.py[pl] = pr.y;
    S.u.t.pz[pl] = pr.z;
  }
  __syncwarp();
  const SmemView<T> V{S};
  return integrate_view<T, 5>(J, V, S.u.t.ts, lane, self, x, nv, np, sr, err_code);
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
    const uint32_t tie = S.u.g.sh.tie[c];
    const int orig = (int)(tie / 27u);
    const int code = (int)(tie - (uint32_t)orig * 27u);
    const int sp = S.u.g.sh.cpos[c];
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
    cuboid_duals(lane, &i0, &i1, &i2);
    bool ok = true;
    double r2 = 0.0;
    if (lane < 8) ok = make_vertex<PIdx>(S, lane, i0, i1, i2, x, dim, &r2);
    if (__any_sync(FULL, !ok)) {
      *err_code = MV_ERR_DET;
      return CELL_ERROR;
    }
  }
  __syncwarp();
  int nv = 8, np = 6;
  double max_r2 = warp_max_nonneg(lane < 8 ? S.vr2[lane] : 0.0);
  double sr = 2.0 * sqrt(max_r2);
  double A = amax_of(max_r2, dim);
  const double x1 = fabs(x.x) + fabs(x.y) + fabs(x.z);

  // ---- ConvexCell::build neighbour loop (convex_cell.rs:316-356) ----
  double R = first_radius(J, x, lane);
  double lo2 = 0.0;
  long long processed = 0;
  bool finished = false;
  int K = 1;  // neighbours set up per batch (adapts to runs of non-clipping neighbours)
  for (int shell = 0; !finished; shell++) {
    if (shell > 0) WCNT(cc, ST_SHELLS, 1);
    bool all;
    // what this shell may hold: the shared buffer, or a staging slot
    const int fits = big_fits<T::CMAX>(J);
    int cnt = gather_shell<T::CMAX, true>(J, S.u.g.sh, lane, x, R, lo2, ext, &all, fits, big_slot(J));
    int shrink = 0;
    bool staged = false;
    for (;;) {
      if (cnt <= T::CMAX) break;
      if (J.big != nullptr && cnt <= fits &&
          big_bucket<T::CMAX>(S.u.g.sh, big_slot(J), lane, cnt, lo2, R * R) <= T::CMAX) {
        staged = true;
        break;
      }
      if (shrink >= 48) break;
      // too many candidates: pull the outer radius in, so that the shell keeps about
      // half of what fits (by volume, at the density just seen)
      const double rin3 = lo2 * sqrt(lo2);
      const double g = fmin(fmax(0.5 * (double)(J.big != nullptr ? fits : T::CMAX) / (double)cnt, 1e-3), 0.7);
      R = cbrt(rin3 + (R * R * R - rin3) * g);
      cnt = gather_shell<T::CMAX, true>(J, S.u.g.sh, lane, x, R, lo2, ext, &all, fits, big_slot(J));
      shrink++;
    }
    if (cnt > T::CMAX && !staged) return CELL_OVERFLOW;
    // a staged shell is consumed in groups of bins (the cursor lives in shared memory)
    if (lane == 0) {
      S.u.g.sh.gbin = staged ? 0 : -1;
      S.u.g.sh.total = cnt;
    }
    __syncwarp();
    if (staged) cnt = big_group<T::CMAX>(S.u.g.sh, big_slot(J), lane);
    for (;;) {
      sort_shell<T::CMAX>(S.u.g.sh, lane, cnt);
      int j = 0;
      if (processed == 0 && cnt > 0) {
        // the first neighbour must be the generator itself (convex_cell.rs:325-329)
        if ((int)(S.u.g.sh.tie[0] / 27u) != self) {
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
                const float4 f = S.f4[sl];
                const float s = fmaf(ez, f.z, fmaf(ey, f.y, fmaf(ex, f.x, h)));
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
              const float4 f = S.f4[sl];
              const float s = fmaf(ez, f.z, fmaf(ey, f.y, fmaf(ex, f.x, h)));
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
        int E = ring_parallel<T>(S, lane, nvf, nv);
        if (E < 0) {
          WCNT(cc, ST_SERIAL_RING, 1);
          E = ring_replay_warp<T>(S, lane, nvf, nv, np);
          if (E == -2) return CELL_OVERFLOW;
          if (E < 0) {
            *err_code = MV_ERR_RING;
            return CELL_ERROR;
          }
        }
        if (nvf + E > T::VMAX) return CELL_OVERFLOW;
        bool ok = true;
        double r2n = 0.0;
        for (int e = lane; e < E; e += 32)
          ok &= make_vertex<PIdx>(S, S.ord[nvf + e], S.ea[e], S.eb[e], p_idx, x, dim, &r2n);
        if (__any_sync(FULL, !ok)) {
          *err_code = MV_ERR_DET;
          return CELL_ERROR;
        }
        __syncwarp();
        nv = nvf + E;
        // update_safety_radius (convex_cell.rs:443-453)
        double m = 0.0;
        for (int q = lane; q < nv; q += 32) m = fmax(m, S.vr2[S.ord[q]]);
        max_r2 = warp_max_nonneg(m);
        sr = 2.0 * sqrt(max_r2);
        A = amax_of(max_r2, dim);
      }
      processed += cnt;
      if (finished || S.u.g.sh.gbin < 0) break;
      cnt = big_group<T::CMAX>(S.u.g.sh, big_slot(J), lane);
    }
    if (finished) break;
    if (all) break;
    if (sr < R * (1.0 - 1e-12)) break;
    // next shell: reach the safety radius, but at most double the radius, so that a
    // cell that is still open does not gather (and then shrink) a domain-wide shell;
    // after a staged shell, no further than the density just seen fills about half a
    // slot (a cell on a dense clump's surface streams the clump in many such shells)
    double Rn = fmin(fmax(R * 1.3, sr * 1.05), 2.0 * R);
    const int total = S.u.g.sh.total;
    if (J.big != nullptr && total > T::CMAX) {
      const double R3 = R * R * R, rin3 = lo2 * sqrt(lo2);
      const double Rd = cbrt(R3 + (R3 - rin3) * (0.5 * (double)BIG_CAP / (double)total));
      Rn = fmin(Rn, fmax(Rd, R * 1.0001));
    }
    lo2 = R * R;
    R = Rn;
  }
  const int res = integrate_cell(J, S, lane, self, x, nv, np, sr, err_code);
  if (res == CELL_DONE && J.rec != nullptr &&
      !write_record(J, J.rec, J.rec_cap, J.rec_counter, J.rec_off + spos, S, lane, x, np, nv, sr, true))
    return CELL_REC_OVERFLOW;
  return res;
}

template <class T, int PREC, int WARPS, bool MULTI>
__global__ void __launch_bounds__(32 * WARPS, T::MINB)
    cells_kernel(const __grid_constant__ Job J0, const __grid_constant__ JobTable TB) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  CellSmem<T>& S = reinterpret_cast<CellSmem<T>*>(smem_raw)[warp];
  __shared__ double ext_s[6];
  if (threadIdx.x < 6) ext_s[threadIdx.x] = J0.ext[threadIdx.x];
  if (lane < ST_COUNT) S.cnt[lane] = 0ull;
  __syncthreads();
  const int total = J0.order ? J0.n_order : J0.n;
  for (;;) {
    int item = 0;
    if (lane == 0) item = (int)atomicAdd(J0.work_counter, 1u);
    item = __shfl_sync(FULL, item, 0);
    if (item >= total) break;
    const int gpos = J0.order ? J0.order[item] : item;
    // the cell's tessellation (batch builds): its Job and its local position
    const int jb = MULTI ? job_of(TB, gpos) : 0;
    const Job& J = MULTI ? TB.jobs[jb] : J0;
    const int spos = MULTI ? gpos - __ldg(TB.pos_base + jb) : gpos;
    const double* ext = MULTI ? J.ext : ext_s;
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
    const int res = build_cell<T, PREC>(J, S, lane, spos, ext, &err, cc);
    __syncwarp();
    if (res == CELL_DONE) cc.c[ST_CELLS]++;
    if (lane == 0) {
#pragma unroll
      for (int i = 0; i < ST_COUNT; i++) S.cnt[i] += cc.c[i];
    }
    __syncwarp();
    if (res == CELL_OVERFLOW) {
      if (lane == 0) {
        unsigned k = atomicAdd(J0.ovf_count, 1u);
        J0.ovf_list[k] = gpos;
        S.cnt[ST_OVERFLOW]++;
      }
    } else if (res == CELL_FACE_OVERFLOW) {
      if (lane == 0) atomicExch(J.status + STATUS_FACE_OVERFLOW, 1);
    } else if (res == CELL_REC_OVERFLOW) {
      if (lane == 0) atomicExch(J.status + STATUS_REC_OVERFLOW, 1);
    } else if (res == CELL_ERROR) {
      if (lane == 0) {
        atomicCAS(J.status + STATUS_CODE, 0, err);
        atomicMin(J.status + STATUS_CELL, self + J.id_base);
      }
    }
    __syncwarp();
  }
  __syncwarp();
  if (lane < ST_COUNT && S.cnt[lane]) atomicAdd(J0.stats + lane, S.cnt[lane]);
}

// ---------------------------------------------------------------- launchers --
#ifndef MV_FAST_WARPS
#define MV_FAST_WARPS 4
#endif
constexpr int FAST_WARPS = MV_FAST_WARPS;
constexpr int LARGE_WARPS = 1;

template <class T, int PREC, int WARPS>
static int blocks_per_sm() {
  int nb = 0;
  const size_t smem = sizeof(CellSmem<T>) * WARPS;
  auto k = cells_kernel<T, PREC, WARPS, false>;
  if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
    return 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k, 32 * WARPS, smem) != cudaSuccess) return 0;
  return nb;
}

template <class T, int PREC, int WARPS>
static cudaError_t launch_tier(const Job& J, const JobTable& TB, int blocks, cudaStream_t st) {
  const size_t smem = sizeof(CellSmem<T>) * WARPS;
  auto k = TB.jobs != nullptr ? cells_kernel<T, PREC, WARPS, true> : cells_kernel<T, PREC, WARPS, false>;
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  k<<<blocks, 32 * WARPS, smem, st>>>(J, TB);
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

// Bytes of the staging slots (one per warp) of fast-tier and large-tier grids of the
// given sizes; the tiers run one after the other, so they share the slots.
size_t cells_big_bytes(int blocks_fast, int blocks_large) {
  const size_t warps = std::max((size_t)blocks_fast * FAST_WARPS, (size_t)blocks_large * LARGE_WARPS);
  return warps * BIG_SLOT_BYTES;
}

// The fused kernel over J's cells (J.order / J.n); with a job table (TB.jobs != nullptr)
// over the cells of a batch.
cudaError_t launch_cells(const Job& J, bool large, int blocks, cudaStream_t st, const JobTable& TB) {
  if (!large) {
    if (J.precision == MV_PRECISION_FILTERED)
      return launch_tier<TierFast, MV_PRECISION_FILTERED, FAST_WARPS>(J, TB, blocks, st);
    return launch_tier<TierFast, MV_PRECISION_FP64, FAST_WARPS>(J, TB, blocks, st);
  }
  if (J.precision == MV_PRECISION_FILTERED)
    return launch_tier<TierLarge, MV_PRECISION_FILTERED, LARGE_WARPS>(J, TB, blocks, st);
  return launch_tier<TierLarge, MV_PRECISION_FP64, LARGE_WARPS>(J, TB, blocks, st);
}

}  // namespace mv
