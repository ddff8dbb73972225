// Point/triangle arithmetic shared by the traversal kernels.
//
// The FP32 distance follows the same formulation as the reference's
// Triangle::distance_sq / closest_point / barycentric
// (atom3d/kernels/bvh_kernels.cu:101-222): inside the triangle's prism
// (all three edge-plane signs >= 0 and |n|^2 >= 1e-12) the squared plane
// distance, otherwise the minimum of the three clamped edge distances.
// Near-degenerate triangles (flagged at build time) are evaluated in FP64.
#pragma once

#include <math.h>

namespace a3d {

template <typename T>
struct V3 {
  T x, y, z;
};
template <typename T>
__device__ __forceinline__ V3<T> mk(T x, T y, T z) { return V3<T>{x, y, z}; }
template <typename T>
__device__ __forceinline__ V3<T> sub(V3<T> a, V3<T> b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
template <typename T>
__device__ __forceinline__ V3<T> add(V3<T> a, V3<T> b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
template <typename T>
__device__ __forceinline__ V3<T> scl(V3<T> a, T s) { return mk(a.x * s, a.y * s, a.z * s); }
template <typename T>
__device__ __forceinline__ T dot(V3<T> a, V3<T> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <typename T>
__device__ __forceinline__ V3<T> cross(V3<T> a, V3<T> b) {
  return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
template <typename T>
__device__ __forceinline__ T clamp01(T v) { return v < T(0) ? T(0) : (v > T(1) ? T(1) : v); }

// Division used by the FP32 evaluation: the fast approximate divide (max
// error 2 ulp); the FP64 evaluation divides exactly.
__device__ __forceinline__ float tdiv(float a, float b) { return __fdividef(a, b); }
__device__ __forceinline__ double tdiv(double a, double b) { return a / b; }

template <typename T>
struct TriEval {
  static constexpr T kDegen = T(1e-12);
  // squared distance; also reports whether the plane branch was taken
  __device__ static __forceinline__ T dist_sq(V3<T> p, V3<T> a, V3<T> b, V3<T> c) {
    const V3<T> v21 = sub(b, a), v32 = sub(c, b), v13 = sub(a, c);
    const V3<T> p1 = sub(p, a), p2 = sub(p, b), p3 = sub(p, c);
    const V3<T> nor = cross(v21, v13);
    const T nsq = dot(nor, nor);
    const bool inside = nsq >= kDegen && dot(cross(v21, nor), p1) >= T(0) && dot(cross(v32, nor), p2) >= T(0) &&
                        dot(cross(v13, nor), p3) >= T(0);
    if (inside) {
      const T d = dot(nor, p1);
      return tdiv(d * d, nsq);
    }
    const T e1 = edge_sq(v21, p1), e2 = edge_sq(v32, p2), e3 = edge_sq(v13, p3);
    return e1 < e2 ? (e1 < e3 ? e1 : e3) : (e2 < e3 ? e2 : e3);
  }
  __device__ static __forceinline__ T edge_sq(V3<T> v, V3<T> p) {
    const T vv = dot(v, v);
    const T t = clamp01(tdiv(dot(v, p), vv > kDegen ? vv : kDegen));
    const V3<T> d = sub(scl(v, t), p);
    return dot(d, d);
  }
  __device__ static __forceinline__ V3<T> closest(V3<T> p, V3<T> a, V3<T> b, V3<T> c) {
    const V3<T> v21 = sub(b, a), v32 = sub(c, b), v13 = sub(a, c);
    const V3<T> p1 = sub(p, a), p2 = sub(p, b), p3 = sub(p, c);
    const V3<T> nor = cross(v21, v13);
    const T nsq = dot(nor, nor);
    const bool inside = nsq >= kDegen && dot(cross(v21, nor), p1) >= T(0) && dot(cross(v32, nor), p2) >= T(0) &&
                        dot(cross(v13, nor), p3) >= T(0);
    if (inside) {
      const T d = tdiv(dot(nor, p1), nsq);
      return sub(p, scl(nor, d));
    }
    const V3<T> c1 = edge_pt(v21, p1, a), c2 = edge_pt(v32, p2, b), c3 = edge_pt(v13, p3, c);
    const V3<T> d1v = sub(c1, p), d2v = sub(c2, p), d3v = sub(c3, p);
    const T d1 = dot(d1v, d1v), d2 = dot(d2v, d2v), d3 = dot(d3v, d3v);
    if (d1 < d2 && d1 < d3) return c1;
    if (d2 < d3) return c2;
    return c3;
  }
  __device__ static __forceinline__ V3<T> edge_pt(V3<T> v, V3<T> p, V3<T> o) {
    const T vv = dot(v, v);
    const T t = clamp01(tdiv(dot(v, p), vv > kDegen ? vv : kDegen));
    return add(o, scl(v, t));
  }
  // barycentric coordinates (u, v, w) of q in (a, b, c), denominators clamped
  // at 1e-10 as in the reference
  __device__ static __forceinline__ V3<T> bary(V3<T> q, V3<T> a, V3<T> b, V3<T> c) {
    const V3<T> v0 = sub(b, a), v1 = sub(c, a), v2 = sub(q, a);
    const T d00 = dot(v0, v0), d01 = dot(v0, v1), d11 = dot(v1, v1), d20 = dot(v2, v0), d21 = dot(v2, v1);
    T den = d00 * d11 - d01 * d01;
    den = den > T(1e-10) ? den : T(1e-10);
    const T v = tdiv(d11 * d20 - d01 * d21, den);
    const T w = tdiv(d00 * d21 - d01 * d20, den);
    return mk(T(1) - v - w, v, w);
  }
};

// FP32 squared distance by barycentric projection.  p - a projects onto the
// plane at a + u e0 + w e1 (e0 = b - a, e1 = c - a) with u = A d1 - B d2,
// w = C d2 - B d1, d1 = (p - a).e0, d2 = (p - a).e1 and the triangle's
// precomputed dual-basis coefficients A, B, C; inside the triangle
// (u, w >= 0, u + w <= 1) the distance is that to the projection, else the
// nearest of the three clamped edge distances (edges a-b and a-c reuse d1
// and d2).  The same point-triangle distance as TriEval::dist_sq: the
// region test is made on the barycentrics instead of the three edge-plane
// signs, so the two agree to rounding where a point sits on a region border.
__device__ __forceinline__ float dist_sq_bary(V3<float> p, V3<float> a, V3<float> b, V3<float> c, float A, float B,
                                              float C, float inv_ab, float inv_bc, float inv_ca) {
  const V3<float> e0 = sub(b, a), e1 = sub(c, a), v = sub(p, a);
  const float d1 = dot(v, e0), d2 = dot(v, e1);
  const float u = A * d1 - B * d2, w = C * d2 - B * d1;
  if (u >= 0.f && w >= 0.f && u + w <= 1.f) {
    const V3<float> q = sub(v, add(scl(e0, u), scl(e1, w)));
    return dot(q, q);
  }
  const float t0 = clamp01(d1 * inv_ab), t2 = clamp01(d2 * inv_ca);
  const V3<float> r0 = sub(v, scl(e0, t0)), r2 = sub(v, scl(e1, t2));
  const V3<float> vb = sub(v, e0), ebc = sub(e1, e0);
  const float t1 = clamp01(dot(vb, ebc) * inv_bc);
  const V3<float> r1 = sub(vb, scl(ebc, t1));
  const float q0 = dot(r0, r0), q1 = dot(r1, r1), q2 = dot(r2, r2);
  return q0 < q1 ? (q0 < q2 ? q0 : q2) : (q1 < q2 ? q1 : q2);
}

}  // namespace a3d
