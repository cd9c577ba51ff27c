// mv_geom.cuh -- f64 geometry primitives of the cell-construction path.
//
// Every function keeps the operation order of the reference crate (meshless_voronoi
// 0.7.2 on glam 0.27: dot = (x*x' + y*y') + z*z', cross, DMat3::determinant =
// z.dot(x.cross(y)), DVec3 / f64 as per-component division).  This translation unit
// is compiled with --fmad=false and IEEE division / square root, so each value is the
// same binary64 number the reference computes.
#pragma once
#include <cstdint>

namespace mv {

struct D3 {
  double x, y, z;
};

__host__ __device__ __forceinline__ D3 d3(double x, double y, double z) { return D3{x, y, z}; }
__host__ __device__ __forceinline__ D3 add(D3 a, D3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__host__ __device__ __forceinline__ D3 sub(D3 a, D3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__host__ __device__ __forceinline__ D3 scale(double s, D3 a) { return {s * a.x, s * a.y, s * a.z}; }
__host__ __device__ __forceinline__ D3 divs(D3 a, double s) { return {a.x / s, a.y / s, a.z / s}; }
__host__ __device__ __forceinline__ D3 vabs(D3 a) { return {fabs(a.x), fabs(a.y), fabs(a.z)}; }
__host__ __device__ __forceinline__ double dot(D3 a, D3 b) {
  double r = a.x * b.x;
  r = r + a.y * b.y;
  r = r + a.z * b.z;
  return r;
}
__host__ __device__ __forceinline__ D3 cross(D3 a, D3 b) {
  return {a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y};
}
// DMat3::from_cols(c0, c1, c2).determinant()
__host__ __device__ __forceinline__ double det_cols(D3 c0, D3 c1, D3 c2) {
  return dot(c2, cross(c0, c1));
}
// f64::signum for non-NaN input
__host__ __device__ __forceinline__ double signum(double x) { return copysign(1.0, x); }

// Plane::project_onto (geometry.rs:36-38) with glam's DVec3::project_onto.
__host__ __device__ __forceinline__ D3 plane_project(D3 n, D3 p, D3 point) {
  D3 v = sub(p, point);
  double rcp = 1.0 / dot(n, n);
  double s = dot(v, n);
  D3 proj = {(n.x * s) * rcp, (n.y * s) * rcp, (n.z * s) * rcp};
  return add(point, proj);
}

// intersect_planes (geometry.rs:68-76).  d_i == p_i . n_i.  Returns false on det == 0.
__host__ __device__ __forceinline__ bool intersect3(D3 n0, double d0, D3 n1, double d1, D3 n2,
                                                    double d2, D3* out) {
  double det = det_cols(n0, n1, n2);
  if (det == 0.0) return false;
  D3 a = scale(d0, cross(n1, n2));
  D3 b = scale(d1, cross(n2, n0));
  D3 c = scale(d2, cross(n0, n1));
  *out = divs(add(add(a, b), c), det);
  return true;
}

// signed_volume_tet (geometry.rs:82-88)
__host__ __device__ __forceinline__ double signed_volume_tet(D3 v0, D3 v1, D3 v2, D3 v3) {
  return det_cols(sub(v1, v0), sub(v2, v0), sub(v3, v0)) / 6.0;
}
// signed_area_tri (geometry.rs:95-100)
__host__ __device__ __forceinline__ double signed_area_tri(D3 v0, D3 v1, D3 v2, D3 t) {
  D3 n = scale(0.5, cross(sub(v1, v0), sub(v2, v0)));
  double sign = signum(dot(sub(t, v0), n));
  return sqrt(dot(n, n)) * sign;
}

// Dimensionality::vector_is_valid (voronoi.rs:42-49)
__host__ __device__ __forceinline__ bool vector_is_valid(int dim, D3 v) {
  if (dim == 1) return v.y == 0.0 && v.z == 0.0;
  if (dim == 2) return v.z == 0.0;
  return true;
}

// Shift vector of periodic image code (mx+1)+3(my+1)+9(mz+1): the reference emits
// -(i w0, j w1, k w2) for the query shift (i, j, k) = -m (rtree_nn.rs:27-33).
__host__ __device__ __forceinline__ D3 shift_of_code(int code, const double* w) {
  int mx = code % 3 - 1, my = (code / 3) % 3 - 1, mz = code / 9 - 1;
  double sx = (double)(-mx) * w[0], sy = (double)(-my) * w[1], sz = (double)(-mz) * w[2];
  return {-sx, -sy, -sz};
}

}  // namespace mv
