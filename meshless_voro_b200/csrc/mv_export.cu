// mv_export.cu -- export of the built convex cells (VoronoiIntegrator's cell view).
//
// Replaces the parts of VoronoiIntegrator that hand out the cells themselves:
// get_cell_at / cells_iter (voronoi.rs:640-657), the decomposition every custom
// integral consumes (ConvexCellDecomposition, convex_cell.rs:89-187; compute_cell_integral
// and compute_face_integrals(_sym), convex_cell.rs:583-664) and with_faces with
// sort_face_vertices (convex_cell.rs:461-543).  An export build keeps every finished
// cell as a record (planes, vertices in the reference's order, see write_record); these
// kernels turn the records into CSR arrays indexed by generator:
//   * the cell's clipping planes (normal, point, right generator, shift code) and
//     vertices (location, dual planes);
//   * the oriented tets of the decomposition, in the reference's order: per vertex the
//     six tets (proj[t], proj[(t+5)%6], vertex) of DecompositionWithoutFaces, or per
//     face the fan (v0, v_i, v_i+1) of DecompositionWithFaces;
//   * with faces: per cell the planes holding at least one vertex, each with its vertex
//     list sorted as sort_face_vertices sorts it.
// Every value is computed with the operations of the reference (the projections are
// the integral kernel's), so the tets are the same binary64 numbers.
#include <cstdint>

#include "mv_cell_common.cuh"

namespace mv {

struct ExportCounts {
  int32_t* planes;
  int32_t* verts;
  int32_t* tets;
  int32_t* faces;
  int32_t* face_verts;
};

struct ExportOut {
  const int64_t* plane_off;      // [n + 1]
  const int64_t* vert_off;       // [n + 1]
  const int64_t* tet_off;        // [n + 1]
  const int64_t* face_off;       // [n + 1]
  const int64_t* face_vert_base; // [n + 1] (per cell)
  double* plane_normal;          // [P][3]
  double* plane_point;           // [P][3]
  int32_t* plane_right;          // [P]
  uint8_t* plane_code;           // [P]
  double* vert_loc;              // [V][3]
  int32_t* vert_dual;            // [V][3]
  double* tet_v;                 // [T][3][3]
  int32_t* tet_plane;            // [T]
  int32_t* face_plane;           // [Fc]
  int64_t* face_vert_off;        // [Fc + 1]
  int32_t* face_verts;           // [3 V]
  int32_t* status;               // [STATUS_WORDS]
};

enum { EXP_TETS = 1, EXP_FACES = 2 };

// Number of the cell's vertices whose duals contain plane pl.
__device__ __forceinline__ int plane_vertex_count(const RecordView& V, int pl) {
  int k = 0;
  for (int q = 0; q < V.nv; q++)
    k += (V.dual(q, 0) == pl) + (V.dual(q, 1) == pl) + (V.dual(q, 2) == pl);
  return k;
}

// Warp per sorted position: the record of each generator and its export sizes.
__global__ void export_count_kernel(const int32_t* __restrict__ sid, const int64_t* __restrict__ rec_off,
                                    const double* __restrict__ rec, int n, int flags,
                                    int64_t* __restrict__ rec_by_orig, ExportCounts c) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t spos = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; spos < n; spos += warps) {
    const int k = __ldg(sid + spos);
    const int64_t off = rec_off[spos];
    int np = 0, nv = 0, tets = 0, faces = 0;
    if (off >= 0) {
      const RecordView V(rec + off);
      np = V.np, nv = V.nv;
      if ((flags & EXP_FACES) || (flags & EXP_TETS)) {
        if (flags & EXP_FACES) {
          for (int pl = lane; pl < np; pl += 32) {
            const int m = plane_vertex_count(V, pl);
            faces += m > 0;
            tets += m > 2 ? m - 2 : 0;
          }
          faces = (int)__reduce_add_sync(FULL, (unsigned)faces);
          tets = (int)__reduce_add_sync(FULL, (unsigned)tets);
        } else {
          tets = 6 * nv;
        }
      }
    }
    if (lane == 0) {
      rec_by_orig[k] = off;
      c.planes[k] = np;
      c.verts[k] = nv;
      c.tets[k] = (flags & EXP_TETS) ? tets : 0;
      c.faces[k] = (flags & EXP_FACES) ? faces : 0;
      c.face_verts[k] = (flags & EXP_FACES) ? 3 * nv : 0;
    }
  }
}

// sort_face_vertices (convex_cell.rs:508-543) on the list v[0, m) of plane pl, in place.
// Returns false when no vertex continues the face (the reference panics).
__device__ bool sort_face(const RecordView& V, int pl, int32_t* v, int m) {
  auto slot = [&](int q) { return V.dual(q, 0) == pl ? 0 : (V.dual(q, 1) == pl ? 1 : 2); };
  int cur = v[0];
  int next_plane = V.dual(cur, (slot(cur) + 1) % 3);
  int ci = 1;
  while (ci + 1 < m) {
    int ti = ci;
    for (; ti < m; ti++) {
      const int q = v[ti];
      if (V.dual(q, 0) == next_plane || V.dual(q, 1) == next_plane || V.dual(q, 2) == next_plane) {
        next_plane = V.dual(q, (slot(q) + 1) % 3);
        const int32_t t = v[ci];
        v[ci] = v[ti];
        v[ti] = t;
        ci++;
        break;
      }
    }
    if (ti >= m) return false;
  }
  return true;
}

__device__ __forceinline__ void put3(double* p, D3 v) { p[0] = v.x, p[1] = v.y, p[2] = v.z; }

// Warp per generator: planes, vertices, tets and face lists at the scanned offsets.
__global__ void export_write_kernel(const __grid_constant__ Job J, const int64_t* __restrict__ rec_by_orig,
                                    const double* __restrict__ rec, int n, int flags, ExportOut o) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t k = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; k < n; k += warps) {
    const int64_t off = rec_by_orig[k];
    if (off < 0) continue;
    const RecordView V(rec + off);
    const D3 x = load_gen(J, (int)k);
    const int np = V.np, nv = V.nv;
    // ConvexCell::clipping_planes: HalfSpace n and p (half_space.rs:24-34)
    const int64_t p0 = o.plane_off[k];
    for (int pl = lane; pl < np; pl += 32) {
      const int r = V.right(pl);
      D3 p;
      if (r < 0) {
        p = {J.bp[pl][0], J.bp[pl][1], J.bp[pl][2]};
      } else {
        D3 ngb = load_gen(J, r);
        const int code = V.code(pl);
        if (code != 13) ngb = add(ngb, D3{J.shift[code][0], J.shift[code][1], J.shift[code][2]});
        p = scale(0.5, add(x, ngb));
      }
      put3(o.plane_normal + 3 * (p0 + pl), V.normal(pl));
      put3(o.plane_point + 3 * (p0 + pl), p);
      o.plane_right[p0 + pl] = r;
      o.plane_code[p0 + pl] = (uint8_t)V.code(pl);
    }
    // ConvexCell::vertices
    const int64_t v0 = o.vert_off[k];
    for (int q = lane; q < nv; q += 32) {
      put3(o.vert_loc + 3 * (v0 + q), V.loc(q));
      o.vert_dual[3 * (v0 + q)] = V.dual(q, 0);
      o.vert_dual[3 * (v0 + q) + 1] = V.dual(q, 1);
      o.vert_dual[3 * (v0 + q) + 2] = V.dual(q, 2);
    }
    if ((flags & EXP_TETS) && !(flags & EXP_FACES)) {
      // DecompositionWithoutFaces (convex_cell.rs:131-187): six tets per vertex
      const int64_t t0 = o.tet_off[k];
      bool ok = true;
      for (int q = lane; q < nv; q += 32) {
        D3 proj[6];
        for (int i = 0; i < 3; i++) {
          proj[2 * i] = V.proj(V.dual(q, i));
          ok = ok && line_projection(V, q, i, x, &proj[2 * i + 1]);
        }
        const D3 vl = V.loc(q);
        for (int t = 0; t < 6; t++) {
          double* tv = o.tet_v + 9 * (t0 + 6 * q + t);
          put3(tv, proj[t]);
          put3(tv + 3, proj[t == 0 ? 5 : t - 1]);
          put3(tv + 6, vl);
          o.tet_plane[t0 + 6 * q + t] = V.dual(q, t / 2);
        }
      }
      if (!ok) atomicCAS(o.status + STATUS_CODE, 0, MV_ERR_DET);
    }
    if (flags & EXP_FACES) {
      // with_faces (convex_cell.rs:461-506): the planes holding vertices, in plane order,
      // each with its vertices in vertex order, then sorted counter-clockwise
      int64_t f_base = o.face_off[k], fv_base = o.face_vert_base[k], t_base = o.tet_off[k];
      bool ok = true;
      for (int pl0 = 0; pl0 < np; pl0 += 32) {
        const int pl = pl0 + lane;
        const int m = pl < np ? plane_vertex_count(V, pl) : 0;
        const int ft = m > 2 ? m - 2 : 0;
        const unsigned lt = lanemask_lt();
        const unsigned has = __ballot_sync(FULL, m > 0);
        int fvx, fvt, ftx, ftt;
        fvx = warp_excl_scan(m, lane, &fvt);
        ftx = warp_excl_scan(ft, lane, &ftt);
        if (m > 0) {
          const int64_t f = f_base + __popc(has & lt);
          int32_t* v = o.face_verts + fv_base + fvx;
          int c = 0;
          for (int q = 0; q < nv; q++)
            if (V.dual(q, 0) == pl || V.dual(q, 1) == pl || V.dual(q, 2) == pl) v[c++] = q;
          ok = ok && sort_face(V, pl, v, m);
          o.face_plane[f] = pl;
          o.face_vert_off[f] = fv_base + fvx;
          if (flags & EXP_TETS) {
            // DecompositionWithFaces (convex_cell.rs:104-128): the face's fan
            const D3 a = V.loc(v[0]);
            for (int i = 1; i + 1 < m; i++) {
              double* tv = o.tet_v + 9 * (t_base + ftx + i - 1);
              put3(tv, a);
              put3(tv + 3, V.loc(v[i]));
              put3(tv + 6, V.loc(v[i + 1]));
              o.tet_plane[t_base + ftx + i - 1] = pl;
            }
          }
        }
        f_base += __popc(has);
        fv_base += fvt;
        t_base += ftt;
      }
      if (!__all_sync(FULL, ok) && lane == 0) atomicCAS(o.status + STATUS_CODE, 0, MV_ERR_RING);
    }
  }
}

// face_vert_off[Fc] = total face vertices
__global__ void export_close_kernel(int64_t* face_vert_off, int64_t nfaces, int64_t total) {
  face_vert_off[nfaces] = total;
}

static int export_blocks(int64_t n) {
  const int64_t b = (n + 7) / 8;  // 8 warps of 256 threads
  return (int)(b < 1 ? 1 : (b > 65535 * 16 ? 65535 * 16 : b));
}

void launch_export_count(const int32_t* sid, const int64_t* rec_off, const double* rec, int n,
                         int flags, int64_t* rec_by_orig, int32_t* planes, int32_t* verts,
                         int32_t* tets, int32_t* faces, int32_t* face_verts, cudaStream_t st) {
  ExportCounts c{planes, verts, tets, faces, face_verts};
  if (n > 0) export_count_kernel<<<export_blocks(n), 256, 0, st>>>(sid, rec_off, rec, n, flags, rec_by_orig, c);
}

void launch_export_write(const Job& J, const int64_t* rec_by_orig, const double* rec, int n, int flags,
                         const int64_t* plane_off, const int64_t* vert_off, const int64_t* tet_off,
                         const int64_t* face_off, const int64_t* face_vert_base, double* plane_normal,
                         double* plane_point, int32_t* plane_right, uint8_t* plane_code,
                         double* vert_loc, int32_t* vert_dual, double* tet_v, int32_t* tet_plane,
                         int32_t* face_plane, int64_t* face_vert_off, int32_t* face_verts,
                         int64_t n_faces, int64_t n_face_verts, int32_t* status, cudaStream_t st) {
  ExportOut o{plane_off, vert_off, tet_off, face_off, face_vert_base, plane_normal, plane_point,
              plane_right, plane_code, vert_loc, vert_dual, tet_v, tet_plane, face_plane,
              face_vert_off, face_verts, status};
  if (n > 0) export_write_kernel<<<export_blocks(n), 256, 0, st>>>(J, rec_by_orig, rec, n, flags, o);
  if (flags & EXP_FACES) export_close_kernel<<<1, 1, 0, st>>>(face_vert_off, n_faces, n_face_verts);
}

}  // namespace mv
