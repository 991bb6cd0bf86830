// TEST INFRASTRUCTURE ONLY — part of the CPU oracle that checks the CUDA path.
// Nothing in the product (vistio_b200/, include/) may include, link or call
// this code. Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
// leg use it, as the checker.
//
// Scalar vector algebra restating glam 0.29's Vec2/Vec3 (the reference's
// math types, vistio-math re-exports them) with the same operation order, plus
// the reference's Mat3x2 (crates/vistio-math/src/mat3x2.rs:16-91).
// Templated on the real type so the oracle runs in FP32 ("ref32", the
// reference's own precision) and in FP64 ("fp64", the truth run).
// Compile with -ffp-contract=off: Rust never fuses a*b+c.
#pragma once
#include <cmath>
#include <cstdint>
#include <algorithm>

namespace orc {

template <class R> struct V3 {
  R x, y, z;
  V3() : x(0), y(0), z(0) {}
  V3(R a, R b, R c) : x(a), y(b), z(c) {}
  V3 operator+(const V3& o) const { return V3(x + o.x, y + o.y, z + o.z); }
  V3 operator-(const V3& o) const { return V3(x - o.x, y - o.y, z - o.z); }
  V3 operator-() const { return V3(-x, -y, -z); }
  V3 operator*(R s) const { return V3(x * s, y * s, z * s); }
  V3 operator/(R s) const { return V3(x / s, y / s, z / s); }
  R dot(const V3& o) const { return x * o.x + y * o.y + z * o.z; }
  V3 cross(const V3& o) const {
    return V3(y * o.z - z * o.y, z * o.x - x * o.z, x * o.y - y * o.x);
  }
  R length_squared() const { return dot(*this); }
  R length() const { return std::sqrt(dot(*this)); }
  // glam: normalize = self * length().recip()
  V3 normalize() const { R r = R(1) / length(); return (*this) * r; }
};

template <class R> struct V2 {
  R x, y;
  V2() : x(0), y(0) {}
  V2(R a, R b) : x(a), y(b) {}
  R length() const { return std::sqrt(x * x + y * y); }
  V2 normalize() const { R r = R(1) / length(); return V2(x * r, y * r); }
};

// Rust f32::max / f32::min (IEEE maxNum/minNum) and f32::clamp.
template <class R> inline R rmax(R a, R b) { return std::fmax(a, b); }
template <class R> inline R rmin(R a, R b) { return std::fmin(a, b); }
template <class R> inline R rclamp(R v, R lo, R hi) {
  if (v < lo) return lo;
  if (v > hi) return hi;
  return v;
}

// crates/vistio-math/src/mat3x2.rs:16 — 3x2 column-major matrix.
template <class R> struct M32 {
  V3<R> c0, c1;
  M32() {}
  M32(V3<R> a, V3<R> b) : c0(a), c1(b) {}
  static M32 identity() { return M32(V3<R>(1, 0, 0), V3<R>(0, 1, 0)); }
  // mat3x2.rs:46 ftf
  void ftf(R out[4]) const {
    R a = c0.dot(c0), b = c0.dot(c1), d = c1.dot(c1);
    out[0] = a; out[1] = b; out[2] = b; out[3] = d;
  }
  R frob_sq() const { return c0.length_squared() + c1.length_squared(); }
  // mat3x2.rs:62 mul_mat2, m column-major [a, b, c, d]
  M32 mul2(const R m[4]) const {
    return M32(c0 * m[0] + c1 * m[1], c0 * m[2] + c1 * m[3]);
  }
  M32 operator-(const M32& o) const { return M32(c0 - o.c0, c1 - o.c1); }
};

// crates/vistio-math/src/decomposition.rs:21 PolarDecomposition
template <class R> struct Polar {
  M32<R> rot;
  R stretch[4];
  R s0, s1;
  V2<R> v0, v1;
};

// decomposition.rs:76-138 polar_decomposition_3x2
template <class R> Polar<R> polar_decomposition(const M32<R>& f) {
  R c[4];
  f.ftf(c);
  R a = c[0], b = c[1], d = c[3];
  R half_trace = R(0.5) * (a + d);
  R half_diff = R(0.5) * (a - d);
  R disc = std::sqrt(half_diff * half_diff + b * b);
  R lambda0 = rmax(half_trace + disc, R(0));
  R lambda1 = rmax(half_trace - disc, R(0));
  R s0 = std::sqrt(lambda0), s1 = std::sqrt(lambda1);
  const R eps = R(1.0e-10f);  // DEGENERATE_AREA_THRESHOLD (types/constants.rs:19)
  Polar<R> p;
  if (s0 < eps) {
    p.rot = M32<R>::identity();
    p.stretch[0] = p.stretch[1] = p.stretch[2] = p.stretch[3] = 0;
    p.s0 = p.s1 = 0;
    p.v0 = V2<R>(1, 0); p.v1 = V2<R>(0, 1);
    return p;
  }
  V2<R> v0, v1;
  if (std::fabs(b) > eps) {
    v0 = V2<R>(lambda0 - d, b).normalize();
    v1 = V2<R>(-v0.y, v0.x);
  } else if (a >= d) {
    v0 = V2<R>(1, 0); v1 = V2<R>(0, 1);
  } else {
    v0 = V2<R>(0, 1); v1 = V2<R>(1, 0);
  }
  R s00 = v0.x * v0.x * s0 + v1.x * v1.x * s1;
  R s01 = v0.x * v0.y * s0 + v1.x * v1.y * s1;
  R s11 = v0.y * v0.y * s0 + v1.y * v1.y * s1;
  R inv_s0 = R(1) / s0;
  R inv_s1 = s1 > eps ? R(1) / s1 : R(0);
  R si00 = v0.x * v0.x * inv_s0 + v1.x * v1.x * inv_s1;
  R si01 = v0.x * v0.y * inv_s0 + v1.x * v1.y * inv_s1;
  R si11 = v0.y * v0.y * inv_s0 + v1.y * v1.y * inv_s1;
  R sinv[4] = {si00, si01, si01, si11};
  p.rot = f.mul2(sinv);
  p.stretch[0] = s00; p.stretch[1] = s01; p.stretch[2] = s01; p.stretch[3] = s11;
  p.s0 = s0; p.s1 = s1; p.v0 = v0; p.v1 = v1;
  return p;
}

// decomposition.rs:50-66 clamp_stretch (tension-field theory)
template <class R> void clamp_stretch(const Polar<R>& p, R out[4]) {
  R cs0 = rmin(p.s0, R(1)), cs1 = rmin(p.s1, R(1));
  R s00 = p.v0.x * p.v0.x * cs0 + p.v1.x * p.v1.x * cs1;
  R s01 = p.v0.x * p.v0.y * cs0 + p.v1.x * p.v1.y * cs1;
  R s11 = p.v0.y * p.v0.y * cs0 + p.v1.y * p.v1.y * cs1;
  out[0] = s00; out[1] = s01; out[2] = s01; out[3] = s11;
}

// decomposition.rs:147-155 deformation_gradient: F = [p1-p0, p2-p0] * Dm_inv
template <class R>
M32<R> deformation_gradient(V3<R> p0, V3<R> p1, V3<R> p2, const R dm_inv[4]) {
  return M32<R>(p1 - p0, p2 - p0).mul2(dm_inv);
}

}  // namespace orc
