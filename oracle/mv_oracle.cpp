// mv_oracle.cpp -- TEST INFRASTRUCTURE ONLY.
//
// CPU restatement of the per-cell Voronoi construction of the Rust crate
// meshless_voronoi 0.7.2 (yuyttenhove/meshless_voro).  It is the parity checker
// for the CUDA library and the timed CPU baseline in bench.py; nothing in the
// product links it.  Build: oracle/build_oracle.py (g++ -O2 -ffp-contract=off).
//
// Each function cites the reference file:line it restates.  Floating point
// follows the reference's operation order: glam 0.27 scalar DVec3 semantics
// (dot = (x*x' + y*y') + z*z'; cross; DMat3::determinant = z.dot(x.cross(y));
// Vec/scalar division; project_onto = rhs * self.dot(rhs) * recip(rhs.dot(rhs)))
// with IEEE binary64 and no FMA contraction.
//
// Pinning: the oracle is checked against the reference's own known-answer tests
// (volumes of lattice cells, the two/five-cell cases, partial builds, 2-D area
// sums, the 40-point thin-box fixture, in-sphere equivalence, SimpleCycle ring,
// signed volume/area) in tests/test_oracle_kat.py.  Two aspects are parity
// unpinned because the Rust reference cannot be built here (no cargo/rustc):
//   * the exact rounding of glam 0.27's vector ops (restated from its documented
//     semantics above), and
//   * the order among neighbours at exactly equal f64 squared distance (rstar 0.12 /
//     std BinaryHeap order); this oracle breaks such ties by (index, shift code).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <limits>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// ----------------------------------------------------------------- vectors --
struct V3 {
  double x, y, z;
};
inline V3 vadd(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 vsub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 vscale(double s, V3 a) { return {s * a.x, s * a.y, s * a.z}; }
inline V3 vdivs(V3 a, double s) { return {a.x / s, a.y / s, a.z / s}; }
inline V3 vabs(V3 a) { return {std::fabs(a.x), std::fabs(a.y), std::fabs(a.z)}; }
inline double vdot(V3 a, V3 b) {
  double r = a.x * b.x;
  r = r + a.y * b.y;
  r = r + a.z * b.z;
  return r;
}
inline V3 vcross(V3 a, V3 b) {
  return {a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y};
}
inline double vlen(V3 a) { return std::sqrt(vdot(a, a)); }
// DMat3::from_cols(c0, c1, c2).determinant() == c2 . (c0 x c1)
inline double det_cols(V3 c0, V3 c1, V3 c2) { return vdot(c2, vcross(c0, c1)); }
// f64::signum for non-NaN input
inline double signum(double x) { return std::copysign(1.0, x); }

enum Err : int {
  OK = 0,
  ERR_ARG = 1,
  ERR_DEGENERATE = 2,  // duplicate generator / first NN not self (convex_cell.rs:325-342)
  ERR_RING = 3,        // convex_cell.rs:428
  ERR_DET = 4,         // geometry.rs:70
};

// ------------------------------------------------------------------ planes --
// geometry.rs:22-47 Plane + HalfSpace fields of half_space.rs:9-19.
struct HalfSpace {
  V3 n, p;
  double d, errb;
  int64_t right;   // -1 == None (boundary)
  int shift_code;  // 13 == None; else (mx+1) + 3(my+1) + 9(mz+1)
  V3 shift;        // valid when shift_code != 13
};

// half_space.rs:24-34
HalfSpace make_half_space(V3 n, V3 p, int64_t right, int shift_code, V3 shift) {
  HalfSpace h;
  h.n = n;
  h.p = p;
  h.errb = 1e-13 * (1.0 + vdot(vabs(n), vabs(p)));
  h.d = vdot(n, p);
  h.right = right;
  h.shift_code = shift_code;
  h.shift = shift;
  return h;
}

// half_space.rs:40-47
inline double hs_clip(const HalfSpace& h, V3 v) {
  double c = vdot(h.n, v) - h.d;
  if (std::fabs(c) < h.errb) return 0.0;
  return signum(c);
}

// geometry.rs:36-38 (+ glam project_onto)
inline V3 plane_project(V3 n, V3 p, V3 point) {
  V3 v = vsub(p, point);
  double rcp = 1.0 / vdot(n, n);
  double s = vdot(v, n);
  V3 proj = {(n.x * s) * rcp, (n.y * s) * rcp, (n.z * s) * rcp};
  return vadd(point, proj);
}

// geometry.rs:68-76
inline bool intersect3(V3 n0, V3 p0, V3 n1, V3 p1, V3 n2, V3 p2, V3* out) {
  double det = det_cols(n0, n1, n2);
  if (det == 0.0) return false;
  V3 a = vscale(vdot(p0, n0), vcross(n1, n2));
  V3 b = vscale(vdot(p1, n1), vcross(n2, n0));
  V3 c = vscale(vdot(p2, n2), vcross(n0, n1));
  *out = vdivs(vadd(vadd(a, b), c), det);
  return true;
}

// geometry.rs:41-47
inline bool project_onto_intersection(const HalfSpace& self, const HalfSpace& other, V3 point,
                                      V3* out) {
  V3 nperp = vcross(self.n, other.n);
  return intersect3(self.n, self.p, other.n, other.p, nperp, point, out);
}

// geometry.rs:82-88
inline double signed_volume_tet(V3 v0, V3 v1, V3 v2, V3 v3) {
  return det_cols(vsub(v1, v0), vsub(v2, v0), vsub(v3, v0)) / 6.0;
}
// geometry.rs:95-100
inline double signed_area_tri(V3 v0, V3 v1, V3 v2, V3 t) {
  V3 n = vscale(0.5, vcross(vsub(v1, v0), vsub(v2, v0)));
  double sign = signum(vdot(vsub(t, v0), n));
  return vlen(n) * sign;
}

// ------------------------------------------------------------ exact sign --
// geometry.rs:232-314: sign of the 4x4 determinant with columns
// (b-a, |b-a|^2), (c-a, ..), (d-a, ..), (v-a, ..) expanded along the last column.
// Fixed-width two's complement integers (6 x 64 bit) replace the bignum crate;
// every intermediate fits in < 280 bits so arithmetic mod 2^384 is exact.
struct I384 {
  uint64_t w[6];
};
inline I384 i_from(int64_t v) {
  I384 r;
  uint64_t fill = v < 0 ? ~0ull : 0ull;
  r.w[0] = (uint64_t)v;
  for (int i = 1; i < 6; i++) r.w[i] = fill;
  return r;
}
inline I384 i_add(const I384& a, const I384& b) {
  I384 r;
  unsigned __int128 c = 0;
  for (int i = 0; i < 6; i++) {
    c += (unsigned __int128)a.w[i] + b.w[i];
    r.w[i] = (uint64_t)c;
    c >>= 64;
  }
  return r;
}
inline I384 i_neg(const I384& a) {
  I384 r;
  unsigned __int128 c = 1;
  for (int i = 0; i < 6; i++) {
    c += (unsigned __int128)(~a.w[i]);
    r.w[i] = (uint64_t)c;
    c >>= 64;
  }
  return r;
}
inline I384 i_sub(const I384& a, const I384& b) { return i_add(a, i_neg(b)); }
inline I384 i_mul(const I384& a, const I384& b) {
  uint64_t r[6] = {0, 0, 0, 0, 0, 0};
  for (int i = 0; i < 6; i++) {
    unsigned __int128 carry = 0;
    for (int j = 0; i + j < 6; j++) {
      unsigned __int128 t = (unsigned __int128)a.w[i] * b.w[j] + r[i + j] + carry;
      r[i + j] = (uint64_t)t;
      carry = t >> 64;
    }
  }
  I384 o;
  for (int i = 0; i < 6; i++) o.w[i] = r[i];
  return o;
}
inline int i_sign(const I384& a) {
  if ((int64_t)a.w[5] < 0) return -1;
  for (int i = 0; i < 6; i++)
    if (a.w[i]) return 1;
  return 0;
}
inline I384 det2(const I384& a, const I384& b, const I384& c, const I384& d) {
  return i_sub(i_mul(a, d), i_mul(b, c));
}
inline I384 det3(const I384& a0, const I384& a1, const I384& a2, const I384& b0, const I384& b1,
                 const I384& b2, const I384& c0, const I384& c1, const I384& c2) {
  I384 r = i_mul(a0, det2(b1, b2, c1, c2));
  r = i_sub(r, i_mul(a1, det2(b0, b2, c0, c2)));
  r = i_add(r, i_mul(a2, det2(b0, b1, c0, c1)));
  return r;
}
double in_sphere_exact(const int64_t* a, const int64_t* b, const int64_t* c, const int64_t* d,
                       const int64_t* v) {
  I384 B[4], C[4], D[4], W[4];
  const int64_t* src[4] = {b, c, d, v};
  I384* dst[4] = {B, C, D, W};
  for (int k = 0; k < 4; k++) {
    for (int i = 0; i < 3; i++) dst[k][i] = i_from(src[k][i] - a[i]);
    dst[k][3] = i_add(i_add(i_mul(dst[k][0], dst[k][0]), i_mul(dst[k][1], dst[k][1])),
                      i_mul(dst[k][2], dst[k][2]));
  }
  I384 det = i_from(0);
  det = i_sub(det, i_mul(W[0], det3(B[1], C[1], D[1], B[2], C[2], D[2], B[3], C[3], D[3])));
  det = i_add(det, i_mul(W[1], det3(B[0], C[0], D[0], B[2], C[2], D[2], B[3], C[3], D[3])));
  det = i_sub(det, i_mul(W[2], det3(B[0], C[0], D[0], B[1], C[1], D[1], B[3], C[3], D[3])));
  det = i_add(det, i_mul(W[3], det3(B[0], C[0], D[0], B[1], C[1], D[1], B[2], C[2], D[2])));
  return (double)i_sign(det);
}

// geometry.rs:223-230 (f64 in-sphere, used by the equivalence KAT only)
double in_sphere_f64(V3 a, V3 b, V3 c, V3 d, V3 v) {
  auto ext = [&](V3 q, double out[4]) {
    V3 r = vsub(q, a);
    out[0] = r.x;
    out[1] = r.y;
    out[2] = r.z;
    out[3] = vdot(r, r);
  };
  double m[4][4];  // columns b, c, d, v
  ext(b, m[0]);
  ext(c, m[1]);
  ext(d, m[2]);
  ext(v, m[3]);
  // cofactor expansion with 2x2 sub-factors; only its sign is used (equivalence KAT)
  double a2323 = m[2][2] * m[3][3] - m[3][2] * m[2][3];
  double a1323 = m[1][2] * m[3][3] - m[3][2] * m[1][3];
  double a1223 = m[1][2] * m[2][3] - m[2][2] * m[1][3];
  double a0323 = m[0][2] * m[3][3] - m[3][2] * m[0][3];
  double a0223 = m[0][2] * m[2][3] - m[2][2] * m[0][3];
  double a0123 = m[0][2] * m[1][3] - m[1][2] * m[0][3];
  double d0 = m[1][1] * a2323 - m[2][1] * a1323 + m[3][1] * a1223;
  double d1 = m[0][1] * a2323 - m[2][1] * a0323 + m[3][1] * a0223;
  double d2 = m[0][1] * a1323 - m[1][1] * a0323 + m[3][1] * a0123;
  double d3 = m[0][1] * a1223 - m[1][1] * a0223 + m[2][1] * a0123;
  return m[0][0] * d0 - m[1][0] * d1 + m[2][0] * d2 - m[3][0] * d3;
}

// ---------------------------------------------------------------- boundary --
// boundary.rs:14-64, voronoi.rs:200-210 (dimension normalisation).
struct Boundary {
  double anchor[3], width[3];  // normalised (not tripled) simulation volume
  V3 iloc_anchor, iloc_inv;    // anchor - width, 1/(3 width) of the (tripled) box
  int dim;
  bool periodic;
  HalfSpace planes[6];
};

void make_boundary(const double* anchor_in, const double* width_in, int dim, bool periodic,
                   Boundary* b) {
  V3 anchor = {anchor_in[0], anchor_in[1], anchor_in[2]};
  V3 width = {width_in[0], width_in[1], width_in[2]};
  if (dim == 1) {
    anchor.y = -0.5;
    width.y = 1.0;
  }
  if (dim == 1 || dim == 2) {
    anchor.z = -0.5;
    width.z = 1.0;
  }
  b->anchor[0] = anchor.x, b->anchor[1] = anchor.y, b->anchor[2] = anchor.z;
  b->width[0] = width.x, b->width[1] = width.y, b->width[2] = width.z;
  b->dim = dim;
  b->periodic = periodic;
  if (periodic) {
    anchor.x -= width.x;
    width.x *= 3.0;
    if (dim >= 2) {
      anchor.y -= width.y;
      width.y *= 3.0;
    }
    if (dim == 3) {
      anchor.z -= width.z;
      width.z *= 3.0;
    }
  }
  V3 hi = vadd(anchor, width);
  V3 none = {0, 0, 0};
  b->planes[0] = make_half_space({1.0, 0.0, 0.0}, anchor, -1, 13, none);
  b->planes[1] = make_half_space({-1.0, 0.0, 0.0}, hi, -1, 13, none);
  b->planes[2] = make_half_space({0.0, 1.0, 0.0}, anchor, -1, 13, none);
  b->planes[3] = make_half_space({0.0, -1.0, 0.0}, hi, -1, 13, none);
  b->planes[4] = make_half_space({0.0, 0.0, 1.0}, anchor, -1, 13, none);
  b->planes[5] = make_half_space({0.0, 0.0, -1.0}, hi, -1, 13, none);
  b->iloc_anchor = vsub(anchor, width);
  b->iloc_inv = {1.0 / (3.0 * width.x), 1.0 / (3.0 * width.y), 1.0 / (3.0 * width.z)};
}

// boundary.rs:49-64
inline void iloc(const Boundary& b, V3 loc, int64_t out[3]) {
  const uint64_t mask = 0xFFFFFFFFFFFFFull;
  double c[3] = {1.0 + (loc.x - b.iloc_anchor.x) * b.iloc_inv.x,
                 1.0 + (loc.y - b.iloc_anchor.y) * b.iloc_inv.y,
                 1.0 + (loc.z - b.iloc_anchor.z) * b.iloc_inv.z};
  for (int i = 0; i < 3; i++) {
    uint64_t bits;
    std::memcpy(&bits, &c[i], 8);
    out[i] = (int64_t)(bits & mask);
  }
}

// voronoi.rs:42-49
inline bool vector_is_valid(int dim, V3 v) {
  if (dim == 1) return v.y == 0.0 && v.z == 0.0;
  if (dim == 2) return v.z == 0.0;
  return true;
}

// emitted periodic shift for shift code (rtree_nn.rs:27-33: shift = -(i w, j w, k w))
inline V3 shift_vec(int code, const double* width) {
  int m[3] = {code % 3 - 1, (code / 3) % 3 - 1, code / 9 - 1};
  double s[3];
  for (int i = 0; i < 3; i++) {
    double si = (double)(-m[i]) * width[i];  // the rtree's query shift
    s[i] = -si;
  }
  return {s[0], s[1], s[2]};
}

// ----------------------------------------------------------- simple cycle --
// simple_cycle.rs:1-101
struct SimpleCycle {
  std::vector<int> ptrs;
  int start = 0, len = 0;
  void reset(int n) {
    ptrs.resize(n);
    for (int i = 0; i < n; i++) ptrs[i] = i;
    start = 0;
    len = 0;
  }
  void grow() { ptrs.push_back((int)ptrs.size()); }
  void init(int a, int b, int c) {
    int cur = start;
    for (int i = 0; i < len; i++) {
      int nxt = ptrs[cur];
      ptrs[cur] = cur;
      cur = nxt;
    }
    len = 3;
    start = a;
    ptrs[a] = b;
    ptrs[b] = c;
    ptrs[c] = a;
  }
  bool contains(int i) const { return ptrs[i] != i; }
  bool try_extend(int a, int b, int c) {
    int tri[3] = {a, b, c};
    bool in[3] = {contains(a), contains(b), contains(c)};
    for (int i = 0; i < 3; i++) {
      int j = (i + 1) % 3, k = (i + 2) % 3;
      if (!in[i] && in[j] && in[k] && ptrs[tri[k]] == tri[j]) {
        ptrs[tri[k]] = tri[i];
        ptrs[tri[i]] = tri[j];
        len += 1;
        return true;
      } else if (in[i] && in[j] && in[k] && ptrs[tri[k]] == tri[j] && ptrs[tri[j]] == tri[i]) {
        ptrs[tri[k]] = tri[i];
        ptrs[tri[j]] = tri[j];
        if (start == tri[j]) start = tri[i];
        len -= 1;
        return true;
      }
    }
    return false;
  }
};

// ------------------------------------------------------------ convex cell --
struct Vertex {
  V3 loc;
  int dual[3];
  double r2;
};

struct Gen {
  const V3* loc;  // generators with unused dims zeroed (generator.rs:13-24)
  int64_t n;
};

struct CellStats {
  int32_t n_nn;        // neighbours consumed from the stream (incl. self)
  int32_t n_planes;    // clipping planes at the end (incl. 6 boundary)
  int32_t n_vert;      // final vertex count
  int32_t max_vert;    // max vertex count during construction
  int32_t n_exact;     // exact in-sphere evaluations
  int32_t n_shells;    // neighbour-stream shell expansions
  int32_t n_cand;      // candidates in the final shell list
  int32_t pad;
};

struct ConvexCell {
  int64_t idx;
  V3 loc;
  std::vector<HalfSpace> planes;
  std::vector<Vertex> verts;
  SimpleCycle ring;
  double safety_radius = 0;
  int dim = 3;
};

// convex_cell.rs:28-48
inline bool vertex_from_dual(const ConvexCell& cell, int i, int j, int k, Vertex* out) {
  const HalfSpace &a = cell.planes[i], &b = cell.planes[j], &c = cell.planes[k];
  V3 loc;
  if (!intersect3(a.n, a.p, b.n, b.p, c.n, c.p, &loc)) return false;
  V3 d = loc;
  if (cell.dim == 1) d = {loc.x, 0.0, 0.0};
  if (cell.dim == 2) d = {loc.x, loc.y, 0.0};
  V3 r = vsub(cell.loc, d);
  out->loc = loc;
  out->dual[0] = i, out->dual[1] = j, out->dual[2] = k;
  out->r2 = vdot(r, r);
  return true;
}

// convex_cell.rs:443-453
inline void update_safety_radius(ConvexCell& cell) {
  double m = -std::numeric_limits<double>::infinity();
  for (auto& v : cell.verts) m = std::max(m, v.r2);
  cell.safety_radius = 2.0 * std::sqrt(m);
}

// convex_cell.rs:294-312
int cell_init(ConvexCell& cell, V3 loc, int64_t idx, const Boundary& b) {
  static const int duals[8][3] = {{2, 5, 0}, {5, 3, 0}, {1, 5, 2}, {5, 1, 3},
                                  {4, 2, 0}, {4, 0, 3}, {2, 4, 1}, {4, 3, 1}};
  cell.idx = idx;
  cell.loc = loc;
  cell.dim = b.dim;
  cell.planes.assign(b.planes, b.planes + 6);
  cell.verts.resize(8);
  for (int i = 0; i < 8; i++)
    if (!vertex_from_dual(cell, duals[i][0], duals[i][1], duals[i][2], &cell.verts[i]))
      return ERR_DET;
  cell.ring.reset(6);
  update_safety_radius(cell);
  return OK;
}

// half_space.rs:53-65
inline V3 right_loc(const HalfSpace& h, const ConvexCell& cell, const Gen& g) {
  if (h.right >= 0) {
    V3 l = g.loc[h.right];
    if (h.shift_code != 13) l = vadd(l, h.shift);
    return l;
  }
  V3 left = g.loc[cell.idx];
  V3 pr = plane_project(h.n, h.p, left);
  return vsub(vscale(2.0, pr), left);
}

// convex_cell.rs:421-441
bool compute_boundary(SimpleCycle& ring, Vertex* v, int n) {
  ring.init(v[0].dual[0], v[0].dual[1], v[0].dual[2]);
  for (int i = 1; i < n; i++) {
    int idx = i;
    for (;;) {
      if (idx >= n) return false;
      if (ring.try_extend(v[idx].dual[0], v[idx].dual[1], v[idx].dual[2])) {
        if (idx > i) std::swap(v[i], v[idx]);
        break;
      }
      idx++;
    }
  }
  return true;
}

// convex_cell.rs:358-419
int clip_by_plane(ConvexCell& cell, const HalfSpace& p, const Gen& g, const Boundary& b,
                  CellStats* st) {
  int i = 0;
  int num_v = (int)cell.verts.size();
  int num_r = 0;
  while (i < num_v) {
    double clip = hs_clip(p, cell.verts[i].loc);
    if (clip == 0.0) {
      const int* dual = cell.verts[i].dual;
      int64_t A[3], B[3], C[3], D[3], W[3];
      iloc(b, cell.loc, A);
      iloc(b, right_loc(cell.planes[dual[0]], cell, g), B);
      iloc(b, right_loc(cell.planes[dual[1]], cell, g), C);
      iloc(b, right_loc(cell.planes[dual[2]], cell, g), D);
      iloc(b, right_loc(p, cell, g), W);
      clip = in_sphere_exact(A, B, C, D, W);
      st->n_exact++;
    }
    if (clip < 0.0) {
      num_v -= 1;
      num_r += 1;
      std::swap(cell.verts[i], cell.verts[num_v]);
    } else {
      i += 1;
    }
  }
  if (num_r > 0) {
    int p_idx = (int)cell.planes.size();
    cell.planes.push_back(p);
    cell.ring.grow();
    if (!compute_boundary(cell.ring, cell.verts.data() + num_v, num_r)) return ERR_RING;
    cell.verts.resize(num_v);
    int cur = cell.ring.start;
    for (int e = 0; e < cell.ring.len; e++) {
      int next = cell.ring.ptrs[cur];
      Vertex nv;
      if (!vertex_from_dual(cell, cur, next, p_idx, &nv)) return ERR_DET;
      cell.verts.push_back(nv);
      cur = next;
    }
    update_safety_radius(cell);
  }
  return OK;
}

// ------------------------------------------------------- neighbour stream --
// Nearest-first stream of (generator, periodic image) pairs with the semantics of
// rtree_nn.rs:10-36 (nn_iter / wrapping_nn_iter): ordered by the f64 squared
// distance the reference computes, self first, images restricted to shifts in
// {-1,0,1}^dims.  Realised as nested shells on a uniform grid: a shell of radius R
// holds exactly the stream elements with d2 < R*R (a prefix of the stream).
struct Grid {
  double a[3], h[3], inv_h[3], w[3];
  double lo_ext[3], hi_ext[3];  // point extent, so boundary cells cover stray points
  int G[3];
  bool wrap[3];
  std::vector<int64_t> start, items;
};

void build_grid(const Gen& g, const Boundary& b, double ppc, Grid* gr) {
  int dim = b.dim;
  double vol = 1.0;
  for (int i = 0; i < dim; i++) vol *= b.width[i];
  double n = (double)std::max<int64_t>(g.n, 1);
  double h = std::pow(vol * ppc / n, 1.0 / dim);
  for (int i = 0; i < 3; i++) {
    gr->a[i] = b.anchor[i];
    gr->w[i] = b.width[i];
    int G = 1;
    if (i < dim) {
      double gg = std::floor(b.width[i] / h);
      G = (int)std::max(1.0, std::min(gg, 2048.0));
    }
    gr->G[i] = G;
    gr->h[i] = b.width[i] / G;
    gr->inv_h[i] = G / b.width[i];
    gr->wrap[i] = b.periodic && i < dim;
  }
  for (int i = 0; i < 3; i++) gr->lo_ext[i] = gr->a[i], gr->hi_ext[i] = gr->a[i] + gr->w[i];
  for (int64_t k = 0; k < g.n; k++) {
    const double* q = &g.loc[k].x;
    for (int i = 0; i < 3; i++) {
      gr->lo_ext[i] = std::min(gr->lo_ext[i], q[i]);
      gr->hi_ext[i] = std::max(gr->hi_ext[i], q[i]);
    }
  }
  int64_t ncell = (int64_t)gr->G[0] * gr->G[1] * gr->G[2];
  std::vector<int64_t> cid(g.n);
  gr->start.assign(ncell + 1, 0);
  for (int64_t k = 0; k < g.n; k++) {
    const double* q = &g.loc[k].x;
    int64_t c[3];
    for (int i = 0; i < 3; i++) {
      double f = std::floor((q[i] - gr->a[i]) * gr->inv_h[i]);
      if (!(f >= 0)) f = 0;  // also maps NaN to 0
      if (f > gr->G[i] - 1) f = gr->G[i] - 1;
      c[i] = (int64_t)f;
    }
    cid[k] = c[0] + (int64_t)gr->G[0] * (c[1] + (int64_t)gr->G[1] * c[2]);
    gr->start[cid[k] + 1]++;
  }
  for (int64_t c = 0; c < ncell; c++) gr->start[c + 1] += gr->start[c];
  gr->items.resize(g.n);
  std::vector<int64_t> fill(gr->start.begin(), gr->start.end() - 1);
  for (int64_t k = 0; k < g.n; k++) gr->items[fill[cid[k]]++] = k;
}

struct Cand {
  double d2;
  int64_t idx;
  int code;
};
inline bool cand_less(const Cand& a, const Cand& b) {
  if (a.d2 != b.d2) return a.d2 < b.d2;
  if (a.idx != b.idx) return a.idx < b.idx;
  return a.code < b.code;
}

// Gathers all stream elements with d2 < R2 (R2 == inf: every element).
// Returns true when the gather covered the whole (image-restricted) point set.
bool gather_shell(const Gen& g, const Grid& gr, V3 q, double R, std::vector<Cand>& out) {
  out.clear();
  const double* qa = &q.x;
  int lo[3], hi[3];
  bool all = true;
  for (int i = 0; i < 3; i++) {
    int G = gr.G[i];
    int umin = gr.wrap[i] ? -G : 0, umax = gr.wrap[i] ? 2 * G - 1 : G - 1;
    double fl = std::floor((qa[i] - R - gr.a[i]) * gr.inv_h[i]) - 1;
    double fh = std::floor((qa[i] + R - gr.a[i]) * gr.inv_h[i]) + 1;
    lo[i] = fl < umin ? umin : (int)fl;
    hi[i] = fh > umax ? umax : (int)fh;
    if (lo[i] > umin || hi[i] < umax) all = false;
  }
  double R2 = all ? std::numeric_limits<double>::infinity() : R * R;
  for (int uz = lo[2]; uz <= hi[2]; uz++)
    for (int uy = lo[1]; uy <= hi[1]; uy++)
      for (int ux = lo[0]; ux <= hi[0]; ux++) {
        int u[3] = {ux, uy, uz}, c[3], m[3];
        double bd2 = 0;
        for (int i = 0; i < 3; i++) {
          int G = gr.G[i];
          m[i] = u[i] < 0 ? -1 : (u[i] >= G ? 1 : 0);
          c[i] = u[i] - m[i] * G;
          double eps = 1e-9 * gr.h[i] + 1e-13 * (std::fabs(gr.a[i]) + gr.w[i]);
          double blo = gr.a[i] + c[i] * gr.h[i], bhi = gr.a[i] + (c[i] + 1) * gr.h[i];
          if (c[i] == 0) blo = gr.wrap[i] ? std::min(blo, gr.lo_ext[i]) : -INFINITY;
          if (c[i] == G - 1) bhi = gr.wrap[i] ? std::max(bhi, gr.hi_ext[i]) : INFINITY;
          blo += m[i] * gr.w[i] - eps;
          bhi += m[i] * gr.w[i] + eps;
          double dd = qa[i] < blo ? blo - qa[i] : (qa[i] > bhi ? qa[i] - bhi : 0.0);
          bd2 += dd * dd;
        }
        if (!all && bd2 >= R2 * (1 + 1e-9)) continue;
        int64_t cell = c[0] + (int64_t)gr.G[0] * (c[1] + (int64_t)gr.G[1] * c[2]);
        int code = (m[0] + 1) + 3 * (m[1] + 1) + 9 * (m[2] + 1);
        double s[3];
        for (int i = 0; i < 3; i++) s[i] = (double)(-m[i]) * gr.w[i];
        for (int64_t t = gr.start[cell]; t < gr.start[cell + 1]; t++) {
          int64_t k = gr.items[t];
          V3 p = g.loc[k];
          double d2;
          if (code == 13 && !gr.wrap[0]) {
            // rstar distance_2: (g - q).length_squared()
            V3 dd = vsub(p, q);
            d2 = vdot(dd, dd);
          } else {
            // rtree_nn.rs:138-146: dx = q + shift - g
            double dx = (q.x + s[0]) - p.x, dy = (q.y + s[1]) - p.y, dz = (q.z + s[2]) - p.z;
            d2 = dx * dx + dy * dy + dz * dz;
          }
          if (d2 < R2) out.push_back({d2, k, code});
        }
      }
  std::sort(out.begin(), out.end(), cand_less);
  return all;
}

// convex_cell.rs:316-356 driven by the shell stream
int build_cell(ConvexCell& cell, int64_t idx, const Gen& g, const Grid& gr, const Boundary& b,
               double R0, CellStats* st, std::vector<Cand>& cand) {
  V3 x = g.loc[idx];
  int err = cell_init(cell, x, idx, b);
  if (err) return err;
  size_t processed = 0;
  double R = R0;
  for (int shell = 0;; shell++) {
    bool all = gather_shell(g, gr, x, R, cand);
    st->n_shells = shell + 1;
    st->n_cand = (int)cand.size();
    for (size_t j = processed; j < cand.size(); j++) {
      const Cand& c = cand[j];
      st->n_nn++;
      if (j == 0) {
        if (c.idx != idx) return ERR_DEGENERATE;
        continue;
      }
      V3 shift = shift_vec(c.code, b.width);
      V3 ngb = g.loc[c.idx];
      if (c.code != 13) ngb = vadd(ngb, shift);
      V3 dx = vsub(cell.loc, ngb);
      double dist = vlen(dx);
      if (!(std::isfinite(dist) && dist > 0.0)) return ERR_DEGENERATE;
      if (cell.safety_radius < dist) return OK;
      V3 n = vdivs(dx, dist);
      V3 p = vscale(0.5, vadd(cell.loc, ngb));
      HalfSpace hs = make_half_space(n, p, c.idx, c.code, shift);
      err = clip_by_plane(cell, hs, g, b, st);
      if (err) return err;
      st->max_vert = std::max<int32_t>(st->max_vert, (int32_t)cell.verts.size());
    }
    processed = cand.size();
    if (all) return OK;
    if (processed == 0) return ERR_DEGENERATE;
    if (cell.safety_radius < R * (1.0 - 1e-12)) return OK;
    R *= 1.5;
  }
}

// -------------------------------------------------------- decomposition --
struct Tet {
  V3 v0, v1, v2;
  int plane;
};

// convex_cell.rs:131-187 (DecompositionWithoutFaces)
template <class F>
bool decompose_without_faces(const ConvexCell& cell, F&& fn) {
  for (const Vertex& v : cell.verts) {
    V3 proj[6];
    for (int i = 0; i < 3; i++) {
      const HalfSpace& cur = cell.planes[v.dual[i]];
      const HalfSpace& nxt = cell.planes[v.dual[(i + 1) % 3]];
      proj[2 * i] = plane_project(cur.n, cur.p, cell.loc);
      if (!project_onto_intersection(nxt, cur, cell.loc, &proj[2 * i + 1])) return false;
    }
    for (int t = 0; t < 6; t++) fn(Tet{proj[t], proj[(t + 5) % 6], v.loc, v.dual[t / 2]});
  }
  return true;
}

// convex_cell.rs:461-543 (with_faces + sort_face_vertices)
struct FaceLists {
  std::vector<int> plane, count, offset, verts;  // faces with >= 1 vertex, plane order
};
bool with_faces(const ConvexCell& cell, FaceLists* fl) {
  size_t P = cell.planes.size();
  std::vector<std::vector<int>> conn(P);
  for (size_t k = 0; k < cell.verts.size(); k++)
    for (int i = 0; i < 3; i++) conn[cell.verts[k].dual[i]].push_back((int)k);
  for (size_t pl = 0; pl < P; pl++) {
    auto& vi = conn[pl];
    if (vi.empty()) continue;
    auto plane_slot = [&](const Vertex& v) {
      for (int s = 0; s < 3; s++)
        if (v.dual[s] == (int)pl) return s;
      return -1;
    };
    const Vertex* cur = &cell.verts[vi[0]];
    int next_plane = cur->dual[(plane_slot(*cur) + 1) % 3];
    size_t ci = 1;
    while (ci + 1 < vi.size()) {
      size_t ti = ci;
      while (ti < vi.size()) {
        cur = &cell.verts[vi[ti]];
        int s = plane_slot(*cur);
        if (cur->dual[0] == next_plane || cur->dual[1] == next_plane ||
            cur->dual[2] == next_plane) {
          next_plane = cur->dual[(s + 1) % 3];
          std::swap(vi[ci], vi[ti]);
          ci++;
          break;
        }
        ti++;
      }
      if (ti >= vi.size()) return false;
    }
  }
  fl->plane.clear(), fl->count.clear(), fl->offset.clear(), fl->verts.clear();
  int off = 0;
  for (size_t pl = 0; pl < P; pl++) {
    if (conn[pl].empty()) continue;
    fl->plane.push_back((int)pl);
    fl->count.push_back((int)conn[pl].size());
    fl->offset.push_back(off);
    off += (int)conn[pl].size();
  }
  for (size_t pl = 0; pl < P; pl++)
    for (int k : conn[pl]) fl->verts.push_back(k);
  return true;
}

// convex_cell.rs:104-128 (DecompositionWithFaces)
template <class F>
void decompose_with_faces(const ConvexCell& cell, const FaceLists& fl, F&& fn) {
  for (size_t f = 0; f < fl.plane.size(); f++) {
    const int* v = &fl.verts[fl.offset[f]];
    for (int i = 1; i + 1 < fl.count[f]; i++)
      fn(Tet{cell.verts[v[0]].loc, cell.verts[v[i]].loc, cell.verts[v[i + 1]].loc, fl.plane[f]});
  }
}

// --------------------------------------------------------------- outputs --
struct FaceRec {
  int64_t left, right;
  double area;
  V3 centroid, normal;
  int code;
};

struct CellOut {
  double volume = 0, sr = 0;
  V3 centroid{0, 0, 0}, loc{0, 0, 0};
  std::vector<FaceRec> faces;
};

enum FaceMode { FACES_OWNED = 0, FACES_ALL = 1 };

// voronoi_cell.rs:40-100 + integrals.rs:86-106, 300-320 + voronoi_face.rs:548-575
// (FACES_ALL: convex_cell.rs:604-622, every face of valid dimensionality).
bool cell_outputs(const ConvexCell& cell, const uint8_t* mask, int face_mode, bool use_faces,
                  CellOut* out) {
  size_t P = cell.planes.size();
  std::vector<int> state(P, 0);  // 0 undecided, 1 face, 2 skip
  std::vector<double> area(P, 0.0);
  std::vector<V3> cen(P, V3{0, 0, 0});
  double vol = 0;
  V3 vc = {0, 0, 0};
  auto collect = [&](const Tet& t) {
    double v = signed_volume_tet(t.v0, t.v1, t.v2, cell.loc);
    vol += v;
    vc = vadd(vc, vscale(v, vadd(vadd(vadd(t.v0, t.v1), t.v2), cell.loc)));
    int pl = t.plane;
    if (state[pl] == 0) {
      const HalfSpace& h = cell.planes[pl];
      bool ok = vector_is_valid(cell.dim, h.n);
      if (ok && face_mode == FACES_OWNED && h.right >= 0 && h.shift_code == 13)
        ok = h.right > cell.idx || (mask && !mask[h.right]);
      state[pl] = ok ? 1 : 2;
    }
    if (state[pl] == 1) {
      double a = signed_area_tri(t.v0, t.v1, t.v2, cell.loc);
      area[pl] += a;
      cen[pl] = vadd(cen[pl], vscale(a, vadd(vadd(t.v0, t.v1), t.v2)));
    }
  };
  if (use_faces) {
    FaceLists fl;
    if (!with_faces(cell, &fl)) return false;
    decompose_with_faces(cell, fl, collect);
  } else {
    if (!decompose_without_faces(cell, collect)) return false;
  }
  double nv = vol > 0.0 ? 0.25 / vol : 0.0;
  out->volume = vol;
  out->centroid = {vc.x * nv, vc.y * nv, vc.z * nv};  // DVec3 *= f64
  out->loc = cell.loc;
  out->sr = cell.safety_radius;
  out->faces.clear();
  for (size_t pl = 0; pl < P; pl++) {
    if (state[pl] != 1) continue;
    const HalfSpace& h = cell.planes[pl];
    double na = area[pl] > 0.0 ? 1.0 / (3.0 * area[pl]) : 0.0;
    FaceRec f;
    f.left = cell.idx;
    f.right = h.right;
    f.area = area[pl];
    f.centroid = {cen[pl].x * na, cen[pl].y * na, cen[pl].z * na};
    f.normal = h.n;
    f.code = h.shift_code;
    out->faces.push_back(f);
  }
  return true;
}

}  // namespace

// ================================================================ C ABI ====
template <class T>
static void cp(const std::vector<T>& v, T* dst) {
  if (dst && !v.empty()) std::memcpy(dst, v.data(), v.size() * sizeof(T));
}

struct OrcResult {
  int status = 0;
  int64_t error_cell = -1;
  int64_t n = 0;
  std::vector<double> volume, centroid, loc, sr;
  std::vector<int64_t> face_offset, face_count;  // CSR into conn (voronoi.rs:241-263)
  std::vector<int64_t> cell_face_begin;          // first face emitted by each cell
  std::vector<int64_t> f_left, f_right;
  std::vector<double> f_area, f_centroid, f_normal;
  std::vector<int32_t> f_code;
  std::vector<int64_t> conn;
  std::vector<CellStats> stats;
  // convex-cell export (flag ORC_EXPORT_CELLS)
  std::vector<int64_t> pl_off, vx_off;
  std::vector<double> pl_n, pl_p, vx_loc;
  std::vector<int64_t> pl_right;
  std::vector<int32_t> pl_code, vx_dual;
  // decomposition export (flag ORC_EXPORT_TETS; the fan tets with ORC_WITH_FACES) and
  // sorted face-vertex lists (flag ORC_EXPORT_FACES)
  std::vector<int64_t> tet_off, cf_off, fv_off;
  std::vector<double> tet_v;
  std::vector<int32_t> tet_plane, cf_plane, fv;
  // wall seconds of the build's phases: setup (generators, boundary, grid), the
  // per-cell loop, flatten + finalize
  double t_setup = 0.0, t_cells = 0.0, t_finalize = 0.0;
};

static double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

enum {
  ORC_FACES_ALL = 1,      // compute_face_integrals (non-symmetric): every valid face
  ORC_WITH_FACES = 2,     // integrals through the with_faces fan decomposition
  ORC_BRUTE_FORCE = 4,    // one shell covering everything (checks the grid stream)
  ORC_EXPORT_CELLS = 8,   // keep planes/vertices of every built cell
  ORC_NO_CSR = 16,        // skip voronoi.rs finalize
  ORC_EXPORT_TETS = 32,   // keep the decomposition tets of every built cell
  ORC_EXPORT_FACES = 64,  // keep the with_faces vertex lists of every built cell
};

extern "C" {

void* orc_build(const double* xyz, int64_t n, const uint8_t* mask, const double* anchor,
                const double* width, int dim, int periodic, int nthreads, int flags,
                double ppc, double r0_factor) {
  OrcResult* R = new OrcResult();
  const double t0 = now_s();
  R->n = n;
  if (n < 0 || (dim < 1 || dim > 3)) {
    R->status = ERR_ARG;
    return R;
  }
  Boundary b;
  make_boundary(anchor, width, dim, periodic != 0, &b);
  std::vector<V3> locs(n);
  for (int64_t k = 0; k < n; k++) {
    V3 l = {xyz[3 * k], xyz[3 * k + 1], xyz[3 * k + 2]};
    if (dim == 1) l.y = 0.0, l.z = 0.0;
    if (dim == 2) l.z = 0.0;
    locs[k] = l;
  }
  Gen g{locs.data(), n};
  Grid gr;
  if (ppc <= 0) ppc = 2.0;
  build_grid(g, b, ppc, &gr);
  double vol = 1.0;
  for (int i = 0; i < dim; i++) vol *= b.width[i];
  double spacing = std::pow(vol / std::max<int64_t>(n, 1), 1.0 / dim);
  if (r0_factor <= 0) r0_factor = 2.6;
  double R0 = (flags & ORC_BRUTE_FORCE) ? 1e300 : r0_factor * spacing;

  std::vector<CellOut> outs(n);
  R->stats.assign(n, CellStats{});
  bool export_cells = flags & ORC_EXPORT_CELLS;
  std::vector<std::vector<HalfSpace>> ex_planes(export_cells ? n : 0);
  std::vector<std::vector<Vertex>> ex_verts(export_cells ? n : 0);
  const bool export_tets = flags & ORC_EXPORT_TETS, export_faces = flags & ORC_EXPORT_FACES;
  std::vector<std::vector<Tet>> ex_tets(export_tets ? n : 0);
  std::vector<FaceLists> ex_faces(export_faces ? n : 0);
  int status = 0;
  int64_t err_cell = -1;
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
  const double t1 = now_s();
  R->t_setup = t1 - t0;
#pragma omp parallel
  {
    ConvexCell cell;
    std::vector<Cand> cand;
#pragma omp for schedule(dynamic, 64)
    for (int64_t k = 0; k < n; k++) {
      if (mask && !mask[k]) continue;  // VoronoiCell::default() (voronoi.rs:303-305)
      int e = build_cell(cell, k, g, gr, b, R0, &R->stats[k], cand);
      if (!e && !cell_outputs(cell, mask, (flags & ORC_FACES_ALL) ? FACES_ALL : FACES_OWNED,
                              (flags & ORC_WITH_FACES) != 0, &outs[k]))
        e = ERR_DET;
      R->stats[k].n_planes = (int32_t)cell.planes.size();
      R->stats[k].n_vert = (int32_t)cell.verts.size();
      if (export_cells && !e) {
        ex_planes[k] = cell.planes;
        ex_verts[k] = cell.verts;
      }
      if ((export_tets || export_faces) && !e) {
        FaceLists fl;
        const bool fan = (flags & ORC_WITH_FACES) != 0;
        if ((fan || export_faces) && !with_faces(cell, &fl)) e = ERR_DET;
        if (!e && export_faces) ex_faces[k] = fl;
        if (!e && export_tets) {
          auto push = [&](const Tet& t) { ex_tets[k].push_back(t); };
          if (fan)
            decompose_with_faces(cell, fl, push);
          else if (!decompose_without_faces(cell, push))
            e = ERR_DET;
        }
      }
      if (e) {
#pragma omp critical
        {
          if (!status || k < err_cell) {
            status = e;
            err_cell = k;
          }
        }
      }
    }
  }
  R->status = status;
  R->error_cell = err_cell;
  const double t2 = now_s();
  R->t_cells = t2 - t1;
  if (status) return R;

  // flatten (voronoi.rs:226) and finalize (voronoi.rs:241-263)
  R->volume.resize(n), R->centroid.resize(3 * n), R->loc.resize(3 * n), R->sr.resize(n);
  R->cell_face_begin.resize(n + 1);
  int64_t F = 0;
  for (int64_t k = 0; k < n; k++) {
    R->cell_face_begin[k] = F;
    F += (int64_t)outs[k].faces.size();
  }
  R->cell_face_begin[n] = F;
  R->f_left.resize(F), R->f_right.resize(F), R->f_area.resize(F), R->f_centroid.resize(3 * F),
      R->f_normal.resize(3 * F), R->f_code.resize(F);
  for (int64_t k = 0; k < n; k++) {
    const CellOut& o = outs[k];
    R->volume[k] = o.volume;
    R->sr[k] = o.sr;
    R->centroid[3 * k] = o.centroid.x, R->centroid[3 * k + 1] = o.centroid.y,
                    R->centroid[3 * k + 2] = o.centroid.z;
    R->loc[3 * k] = o.loc.x, R->loc[3 * k + 1] = o.loc.y, R->loc[3 * k + 2] = o.loc.z;
    int64_t f0 = R->cell_face_begin[k];
    for (size_t j = 0; j < o.faces.size(); j++) {
      const FaceRec& f = o.faces[j];
      int64_t fi = f0 + (int64_t)j;
      R->f_left[fi] = f.left, R->f_right[fi] = f.right, R->f_area[fi] = f.area;
      R->f_centroid[3 * fi] = f.centroid.x, R->f_centroid[3 * fi + 1] = f.centroid.y,
                       R->f_centroid[3 * fi + 2] = f.centroid.z;
      R->f_normal[3 * fi] = f.normal.x, R->f_normal[3 * fi + 1] = f.normal.y,
                     R->f_normal[3 * fi + 2] = f.normal.z;
      R->f_code[fi] = f.code;
    }
  }
  if (!(flags & ORC_NO_CSR)) {
    std::vector<std::vector<int64_t>> lists(n);
    for (int64_t f = 0; f < F; f++) {
      lists[R->f_left[f]].push_back(f);
      if (R->f_right[f] >= 0 && R->f_code[f] == 13) lists[R->f_right[f]].push_back(f);
    }
    R->face_offset.resize(n), R->face_count.resize(n);
    int64_t off = 0;
    for (int64_t k = 0; k < n; k++) {
      R->face_offset[k] = off;
      R->face_count[k] = (int64_t)lists[k].size();
      off += (int64_t)lists[k].size();
    }
    R->conn.reserve(off);
    for (auto& l : lists) R->conn.insert(R->conn.end(), l.begin(), l.end());
  }
  R->t_finalize = now_s() - t2;
  if (export_cells) {
    R->pl_off.assign(n + 1, 0), R->vx_off.assign(n + 1, 0);
    for (int64_t k = 0; k < n; k++) {
      R->pl_off[k + 1] = R->pl_off[k] + (int64_t)ex_planes[k].size();
      R->vx_off[k + 1] = R->vx_off[k] + (int64_t)ex_verts[k].size();
    }
    for (int64_t k = 0; k < n; k++) {
      for (auto& h : ex_planes[k]) {
        R->pl_n.insert(R->pl_n.end(), {h.n.x, h.n.y, h.n.z});
        R->pl_p.insert(R->pl_p.end(), {h.p.x, h.p.y, h.p.z});
        R->pl_right.push_back(h.right);
        R->pl_code.push_back(h.shift_code);
      }
      for (auto& v : ex_verts[k]) {
        R->vx_loc.insert(R->vx_loc.end(), {v.loc.x, v.loc.y, v.loc.z});
        R->vx_dual.insert(R->vx_dual.end(), {v.dual[0], v.dual[1], v.dual[2]});
      }
    }
  }
  if (export_tets) {
    R->tet_off.assign(n + 1, 0);
    for (int64_t k = 0; k < n; k++) R->tet_off[k + 1] = R->tet_off[k] + (int64_t)ex_tets[k].size();
    for (int64_t k = 0; k < n; k++)
      for (const Tet& t : ex_tets[k]) {
        R->tet_v.insert(R->tet_v.end(), {t.v0.x, t.v0.y, t.v0.z, t.v1.x, t.v1.y, t.v1.z, t.v2.x,
                                         t.v2.y, t.v2.z});
        R->tet_plane.push_back(t.plane);
      }
  }
  if (export_faces) {
    R->cf_off.assign(n + 1, 0);
    for (int64_t k = 0; k < n; k++)
      R->cf_off[k + 1] = R->cf_off[k] + (int64_t)ex_faces[k].plane.size();
    R->fv_off.push_back(0);
    for (int64_t k = 0; k < n; k++) {
      const FaceLists& fl = ex_faces[k];
      for (size_t f = 0; f < fl.plane.size(); f++) {
        R->cf_plane.push_back(fl.plane[f]);
        for (int i = 0; i < fl.count[f]; i++) R->fv.push_back(fl.verts[fl.offset[f] + i]);
        R->fv_off.push_back((int64_t)R->fv.size());
      }
    }
  }
  return R;
}

int64_t orc_n_tets_total(void* h) { return (int64_t)((OrcResult*)h)->tet_plane.size(); }
int64_t orc_n_cell_faces_total(void* h) { return (int64_t)((OrcResult*)h)->cf_plane.size(); }
int64_t orc_n_face_vertices_total(void* h) { return (int64_t)((OrcResult*)h)->fv.size(); }
void orc_copy_tets(void* h, int64_t* tet_off, double* tet_v, int32_t* tet_plane) {
  OrcResult* R = (OrcResult*)h;
  cp(R->tet_off, tet_off), cp(R->tet_v, tet_v), cp(R->tet_plane, tet_plane);
}
void orc_copy_face_lists(void* h, int64_t* cf_off, int32_t* cf_plane, int64_t* fv_off,
                         int32_t* fv) {
  OrcResult* R = (OrcResult*)h;
  cp(R->cf_off, cf_off), cp(R->cf_plane, cf_plane), cp(R->fv_off, fv_off), cp(R->fv, fv);
}

int orc_status(void* h) { return ((OrcResult*)h)->status; }
void orc_times(void* h, double* out) {
  const OrcResult* R = (const OrcResult*)h;
  out[0] = R->t_setup, out[1] = R->t_cells, out[2] = R->t_finalize;
}
int64_t orc_error_cell(void* h) { return ((OrcResult*)h)->error_cell; }
int64_t orc_n_faces(void* h) { return (int64_t)((OrcResult*)h)->f_left.size(); }
int64_t orc_n_conn(void* h) { return (int64_t)((OrcResult*)h)->conn.size(); }
int64_t orc_n_planes_total(void* h) { return (int64_t)((OrcResult*)h)->pl_right.size(); }
int64_t orc_n_verts_total(void* h) { return (int64_t)((OrcResult*)h)->vx_dual.size() / 3; }

void orc_copy_cells(void* h, double* volume, double* centroid, double* loc, double* sr,
                    int64_t* face_offset, int64_t* face_count, int64_t* cell_face_begin) {
  OrcResult* R = (OrcResult*)h;
  cp(R->volume, volume), cp(R->centroid, centroid), cp(R->loc, loc), cp(R->sr, sr);
  cp(R->face_offset, face_offset), cp(R->face_count, face_count);
  cp(R->cell_face_begin, cell_face_begin);
}
void orc_copy_faces(void* h, int64_t* left, int64_t* right, double* area, double* centroid,
                    double* normal, int32_t* code) {
  OrcResult* R = (OrcResult*)h;
  cp(R->f_left, left), cp(R->f_right, right), cp(R->f_area, area);
  cp(R->f_centroid, centroid), cp(R->f_normal, normal), cp(R->f_code, code);
}
void orc_copy_conn(void* h, int64_t* conn) { cp(((OrcResult*)h)->conn, conn); }
void orc_copy_stats(void* h, int32_t* stats) {
  OrcResult* R = (OrcResult*)h;
  if (stats && !R->stats.empty())
    std::memcpy(stats, R->stats.data(), R->stats.size() * sizeof(CellStats));
}
void orc_copy_cells_export(void* h, int64_t* pl_off, double* pl_n, double* pl_p, int64_t* pl_right,
                           int32_t* pl_code, int64_t* vx_off, double* vx_loc, int32_t* vx_dual) {
  OrcResult* R = (OrcResult*)h;
  cp(R->pl_off, pl_off), cp(R->pl_n, pl_n), cp(R->pl_p, pl_p), cp(R->pl_right, pl_right);
  cp(R->pl_code, pl_code), cp(R->vx_off, vx_off), cp(R->vx_loc, vx_loc), cp(R->vx_dual, vx_dual);
}
void orc_free(void* h) { delete (OrcResult*)h; }

// ---- geometry entry points for the reference's unit-level known-answer tests ----
double orc_signed_volume_tet(const double* v0, const double* v1, const double* v2,
                             const double* v3) {
  return signed_volume_tet({v0[0], v0[1], v0[2]}, {v1[0], v1[1], v1[2]}, {v2[0], v2[1], v2[2]},
                           {v3[0], v3[1], v3[2]});
}
double orc_signed_area_tri(const double* v0, const double* v1, const double* v2,
                           const double* t) {
  return signed_area_tri({v0[0], v0[1], v0[2]}, {v1[0], v1[1], v1[2]}, {v2[0], v2[1], v2[2]},
                         {t[0], t[1], t[2]});
}
int orc_intersect_planes(const double* n0, const double* p0, const double* n1, const double* p1,
                         const double* n2, const double* p2, double* out) {
  V3 o;
  if (!intersect3({n0[0], n0[1], n0[2]}, {p0[0], p0[1], p0[2]}, {n1[0], n1[1], n1[2]},
                  {p1[0], p1[1], p1[2]}, {n2[0], n2[1], n2[2]}, {p2[0], p2[1], p2[2]}, &o))
    return ERR_DET;
  out[0] = o.x, out[1] = o.y, out[2] = o.z;
  return OK;
}
double orc_in_sphere_f64(const double* a, const double* b, const double* c, const double* d,
                         const double* v) {
  return in_sphere_f64({a[0], a[1], a[2]}, {b[0], b[1], b[2]}, {c[0], c[1], c[2]},
                       {d[0], d[1], d[2]}, {v[0], v[1], v[2]});
}
double orc_in_sphere_exact(const int64_t* a, const int64_t* b, const int64_t* c, const int64_t* d,
                           const int64_t* v) {
  return in_sphere_exact(a, b, c, d, v);
}
void orc_iloc(const double* anchor, const double* width, int dim, int periodic, const double* loc,
              int64_t* out) {
  Boundary b;
  make_boundary(anchor, width, dim, periodic != 0, &b);
  iloc(b, {loc[0], loc[1], loc[2]}, out);
}
// half_space.rs:24-47 on an arbitrary plane (n, p)
double orc_half_space_clip(const double* n, const double* p, const double* v) {
  V3 none = {0, 0, 0};
  HalfSpace h = make_half_space({n[0], n[1], n[2]}, {p[0], p[1], p[2]}, -1, 13, none);
  return hs_clip(h, {v[0], v[1], v[2]});
}
// simple_cycle.rs test harness: grow a ring from triangles with the compute_boundary search
int orc_simple_cycle(const int32_t* tris, int ntri, int capacity, int32_t* out, int* out_len) {
  SimpleCycle s;
  s.reset(capacity);
  std::vector<Vertex> v(ntri);
  for (int i = 0; i < ntri; i++)
    for (int k = 0; k < 3; k++) v[i].dual[k] = tris[3 * i + k];
  if (!compute_boundary(s, v.data(), ntri)) return ERR_RING;
  int cur = s.start;
  for (int i = 0; i < s.len; i++) {
    out[i] = cur;
    cur = s.ptrs[cur];
  }
  *out_len = s.len;
  return OK;
}
// convex_cell.rs:769-799 (test_init_cuboid / test_clipping): number of clipping planes of
// the cuboid cell of `loc` after clipping by the bisector with `ngb`.
int orc_clip_count(const double* anchor, const double* width, const double* loc,
                   const double* ngb) {
  Boundary b;
  make_boundary(anchor, width, 3, false, &b);
  V3 locs[2] = {{loc[0], loc[1], loc[2]}, {ngb[0], ngb[1], ngb[2]}};
  Gen g{locs, 2};
  ConvexCell cell;
  if (cell_init(cell, locs[0], 0, b)) return -1;
  V3 dx = vsub(locs[0], locs[1]);
  double dist = vlen(dx);
  CellStats st{};
  HalfSpace hs = make_half_space(vdivs(dx, dist), vscale(0.5, vadd(locs[0], locs[1])), 1, 13,
                                 V3{0, 0, 0});
  if (clip_by_plane(cell, hs, g, b, &st)) return -1;
  return (int)cell.planes.size();
}

}  // extern "C"
