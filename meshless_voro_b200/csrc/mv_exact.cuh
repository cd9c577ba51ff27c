// mv_exact.cuh -- exact in-sphere sign on quantised coordinates (device).
//
// Replaces in_sphere_test_exact (geometry.rs:232-314), which evaluates with a heap
// bignum crate the sign of the 4x4 determinant whose columns are (b-a, |b-a|^2),
// (c-a, ..), (d-a, ..), (v-a, ..), expanded along the last column.  Inputs are the
// 52-bit integers produced by SimulationBoundary::iloc (boundary.rs:49-64), so
// differences have 53 bits, squared norms 106, the 3x3 minors at most 215 and the
// determinant at most 270 bits: fixed 5 x 64-bit two's-complement limbs (arithmetic
// mod 2^320) are exact.  The sign of an exact integer is unique, so any exact
// evaluation order agrees with the reference.  Five corners of one axis-aligned box
// (the undecided tests of lattice inputs) are recognised first: their determinant is
// exactly zero.
#pragma once
#include <cstdint>

namespace mv {

struct S5 {
  uint64_t w[5];
};

__device__ __forceinline__ S5 s5_from(int64_t v) {
  S5 r;
  uint64_t fill = v < 0 ? ~0ull : 0ull;
  r.w[0] = (uint64_t)v;
#pragma unroll
  for (int i = 1; i < 5; i++) r.w[i] = fill;
  return r;
}

__device__ __forceinline__ S5 s5_add(const S5& a, const S5& b) {
  S5 r;
  uint64_t c = 0;
#pragma unroll
  for (int i = 0; i < 5; i++) {
    uint64_t s = a.w[i] + b.w[i];
    uint64_t c1 = s < a.w[i];
    uint64_t t = s + c;
    uint64_t c2 = t < s;
    r.w[i] = t;
    c = c1 | c2;
  }
  return r;
}

__device__ __forceinline__ S5 s5_neg(const S5& a) {
  S5 r;
  uint64_t c = 1;
#pragma unroll
  for (int i = 0; i < 5; i++) {
    uint64_t t = ~a.w[i] + c;
    c = (c && t == 0) ? 1ull : 0ull;
    r.w[i] = t;
  }
  return r;
}

__device__ __forceinline__ S5 s5_sub(const S5& a, const S5& b) { return s5_add(a, s5_neg(b)); }

// (unsigned 64-bit) x (two's complement S5), mod 2^320
__device__ __forceinline__ S5 s5_mul_u64(uint64_t a, const S5& b) {
  S5 r;
  uint64_t carry = 0;
#pragma unroll
  for (int i = 0; i < 5; i++) {
    uint64_t lo = a * b.w[i];
    uint64_t hi = __umul64hi(a, b.w[i]);
    uint64_t t = lo + carry;
    hi += (t < lo);
    r.w[i] = t;
    carry = hi;
  }
  return r;
}

// (signed 64-bit, |a| < 2^63) x S5
__device__ __forceinline__ S5 s5_mul_i64(int64_t a, const S5& b) {
  S5 r = s5_mul_u64(a < 0 ? (uint64_t)(-a) : (uint64_t)a, b);
  return a < 0 ? s5_neg(r) : r;
}

// S5 x S5 truncated to 320 bits (two's complement ring product).
__device__ __forceinline__ S5 s5_mul(const S5& a, const S5& b) {
  S5 r = s5_mul_u64(a.w[0], b);
#pragma unroll
  for (int i = 1; i < 5; i++) {
    // add (a.w[i] * b) << (64 i)
    S5 t = s5_mul_u64(a.w[i], b);
    uint64_t c = 0;
#pragma unroll
    for (int k = i; k < 5; k++) {
      uint64_t x = t.w[k - i];
      uint64_t s = r.w[k] + x;
      uint64_t c1 = s < x;
      uint64_t u = s + c;
      uint64_t c2 = u < s;
      r.w[k] = u;
      c = c1 | c2;
    }
  }
  return r;
}

__device__ __forceinline__ int s5_sign(const S5& a) {
  if ((int64_t)a.w[4] < 0) return -1;
  return (a.w[0] | a.w[1] | a.w[2] | a.w[3] | a.w[4]) ? 1 : 0;
}

// 2x2 determinant a*d - b*c where a, b are small (|.| < 2^63) and c, d arbitrary.
__device__ __forceinline__ S5 det2_small(int64_t a, int64_t b, const S5& c, const S5& d) {
  return s5_sub(s5_mul_i64(a, d), s5_mul_i64(b, c));
}

// True when, on every axis, the five points take at most two values: they are then
// corners of one axis-aligned box (a flat one when an axis has a single value), so all
// five lie on the box's circumsphere or in one plane and the in-sphere determinant is
// exactly zero.  Quantised lattice inputs meet this in every undecided test: each
// coordinate is quantised on its own, so lattice neighbours stay box corners.
__device__ __forceinline__ bool box_corners(const int64_t a[3], const int64_t b[3],
                                            const int64_t c[3], const int64_t d[3],
                                            const int64_t v[3]) {
  bool ok = true;
#pragma unroll
  for (int i = 0; i < 3; i++) {
    const int64_t p0 = a[i];
    // the first value other than p0 (p0 itself when there is none)
    const int64_t p1 = b[i] != p0 ? b[i] : (c[i] != p0 ? c[i] : (d[i] != p0 ? d[i] : v[i]));
    ok = ok && (b[i] == p0 || b[i] == p1) && (c[i] == p0 || c[i] == p1) &&
         (d[i] == p0 || d[i] == p1) && (v[i] == p0 || v[i] == p1);
  }
  return ok;
}

// Sign of the exact in-sphere determinant (geometry.rs:271-314).  Returns -1, 0, 1.
static __device__ __noinline__ int in_sphere_exact_sign(const int64_t a[3], const int64_t b[3],
                                                 const int64_t c[3], const int64_t d[3],
                                                 const int64_t v[3]) {
  if (box_corners(a, b, c, d, v)) return 0;
  // rows: x, y, z (small, 53-bit) and n (squared norm); columns b, c, d, v
  int64_t X[4], Y[4], Z[4];
  S5 N[4];
  const int64_t* src[4] = {b, c, d, v};
#pragma unroll
  for (int k = 0; k < 4; k++) {
    X[k] = src[k][0] - a[0];
    Y[k] = src[k][1] - a[1];
    Z[k] = src[k][2] - a[2];
    N[k] = s5_add(s5_add(s5_mul_i64(X[k], s5_from(X[k])), s5_mul_i64(Y[k], s5_from(Y[k]))),
                  s5_mul_i64(Z[k], s5_from(Z[k])));
  }
  // 3x3 minors over columns (b, c, d), expanded along their first row.
  // M(yzn): rows y, z, n
  S5 zn01 = det2_small(Z[1], Z[2], N[1], N[2]);  // z_c n_d - z_d n_c
  S5 zn02 = det2_small(Z[0], Z[2], N[0], N[2]);
  S5 zn12 = det2_small(Z[0], Z[1], N[0], N[1]);
  S5 Myzn = s5_add(s5_sub(s5_mul_i64(Y[0], zn01), s5_mul_i64(Y[1], zn02)), s5_mul_i64(Y[2], zn12));
  S5 Mxzn = s5_add(s5_sub(s5_mul_i64(X[0], zn01), s5_mul_i64(X[1], zn02)), s5_mul_i64(X[2], zn12));
  S5 yn01 = det2_small(Y[1], Y[2], N[1], N[2]);
  S5 yn02 = det2_small(Y[0], Y[2], N[0], N[2]);
  S5 yn12 = det2_small(Y[0], Y[1], N[0], N[1]);
  S5 Mxyn = s5_add(s5_sub(s5_mul_i64(X[0], yn01), s5_mul_i64(X[1], yn02)), s5_mul_i64(X[2], yn12));
  S5 yz01 = det2_small(Y[1], Y[2], s5_from(Z[1]), s5_from(Z[2]));
  S5 yz02 = det2_small(Y[0], Y[2], s5_from(Z[0]), s5_from(Z[2]));
  S5 yz12 = det2_small(Y[0], Y[1], s5_from(Z[0]), s5_from(Z[1]));
  S5 Mxyz = s5_add(s5_sub(s5_mul_i64(X[0], yz01), s5_mul_i64(X[1], yz02)), s5_mul_i64(X[2], yz12));
  // det = -v_x M(yzn) + v_y M(xzn) - v_z M(xyn) + v_n M(xyz)
  S5 det = s5_neg(s5_mul_i64(X[3], Myzn));
  det = s5_add(det, s5_mul_i64(Y[3], Mxzn));
  det = s5_sub(det, s5_mul_i64(Z[3], Mxyn));
  det = s5_add(det, s5_mul(N[3], Mxyz));
  return s5_sign(det);
}

}  // namespace mv
