// Triangle/box SAT and the box query over the wide BVH, shared by the
// octree descent, MeshBVH.intersect_aabb's hit mask and its pair modes.
//
// SAT follows triangle_aabb_sat (atom3d/kernels/bvh_kernels.cu:285-353)
// operation by operation (box centre/half extents, 3 box axes, 9 edge cross
// axes, triangle plane, sat_eps = 1e-6).  Every multiply/add is an explicit
// round-to-nearest intrinsic so the compiler cannot contract it into an FMA:
// the result is then a pure function of IEEE single arithmetic and the CPU
// oracle (compiled with -ffp-contract=off) reproduces it bit for bit.
//
// The BVH only prunes: boxes are tested against child bounds grown by a
// margin that covers sat_eps and the rounding of the centre/half
// computation, so the set of triangles passing SAT does not depend on the
// tree.
#pragma once

#include <math.h>

#include "bvh_layout.cuh"

namespace a3d {

constexpr int kSatThreads = 128;
constexpr int kSatDepth = 48;
constexpr int kSatDeepDepth = 512;

__device__ __forceinline__ float fm(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fa(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fsb(float a, float b) { return __fsub_rn(a, b); }

__device__ __forceinline__ float dot3r(float ax, float ay, float az, float bx, float by, float bz) {
  return fa(fa(fm(ax, bx), fm(ay, by)), fm(az, bz));
}

__device__ __forceinline__ bool sat_test(const TriRec& t, float mnx, float mny, float mnz, float mxx, float mxy, float mxz) {
  const float eps = 1e-6f;
  const float cx = fm(fa(mnx, mxx), 0.5f), cy = fm(fa(mny, mxy), 0.5f), cz = fm(fa(mnz, mxz), 0.5f);
  const float hx = fm(fsb(mxx, mnx), 0.5f), hy = fm(fsb(mxy, mny), 0.5f), hz = fm(fsb(mxz, mnz), 0.5f);
  const float v0x = fsb(t.a.x, cx), v0y = fsb(t.a.y, cy), v0z = fsb(t.a.z, cz);
  const float v1x = fsb(t.b.x, cx), v1y = fsb(t.b.y, cy), v1z = fsb(t.b.z, cz);
  const float v2x = fsb(t.c.x, cx), v2y = fsb(t.c.y, cy), v2z = fsb(t.c.z, cz);
  float mn, mx;
  mn = fminf(fminf(v0x, v1x), v2x); mx = fmaxf(fmaxf(v0x, v1x), v2x);
  if (mn > fa(hx, eps) || mx < fsb(-hx, eps)) return false;
  mn = fminf(fminf(v0y, v1y), v2y); mx = fmaxf(fmaxf(v0y, v1y), v2y);
  if (mn > fa(hy, eps) || mx < fsb(-hy, eps)) return false;
  mn = fminf(fminf(v0z, v1z), v2z); mx = fmaxf(fmaxf(v0z, v1z), v2z);
  if (mn > fa(hz, eps) || mx < fsb(-hz, eps)) return false;
  const float e[3][3] = {{fsb(v1x, v0x), fsb(v1y, v0y), fsb(v1z, v0z)},
                         {fsb(v2x, v1x), fsb(v2y, v1y), fsb(v2z, v1z)},
                         {fsb(v0x, v2x), fsb(v0y, v2y), fsb(v0z, v2z)}};
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const float ex = e[k][0], ey = e[k][1], ez = e[k][2];
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) {
      float a0, a1, a2;
      if (ax == 0) { a0 = 0.f; a1 = ez; a2 = -ey; }
      else if (ax == 1) { a0 = -ez; a1 = 0.f; a2 = ex; }
      else { a0 = ey; a1 = -ex; a2 = 0.f; }
      const float p0 = dot3r(v0x, v0y, v0z, a0, a1, a2);
      const float p1 = dot3r(v1x, v1y, v1z, a0, a1, a2);
      const float p2 = dot3r(v2x, v2y, v2z, a0, a1, a2);
      const float mnp = fminf(fminf(p0, p1), p2), mxp = fmaxf(fmaxf(p0, p1), p2);
      const float rad = fa(fa(fa(fm(hx, fabsf(a0)), fm(hy, fabsf(a1))), fm(hz, fabsf(a2))), eps);
      if (mnp > rad || mxp < -rad) return false;
    }
  }
  // plane: normal = cross(e0, v2 - v0)
  const float wx = fsb(v2x, v0x), wy = fsb(v2y, v0y), wz = fsb(v2z, v0z);
  const float e0x = e[0][0], e0y = e[0][1], e0z = e[0][2];
  const float nx = fsb(fm(e0y, wz), fm(e0z, wy));
  const float ny = fsb(fm(e0z, wx), fm(e0x, wz));
  const float nz = fsb(fm(e0x, wy), fm(e0y, wx));
  const float d = -dot3r(nx, ny, nz, v0x, v0y, v0z);
  const float r = fa(fa(fa(fm(hx, fabsf(nx)), fm(hy, fabsf(ny))), fm(hz, fabsf(nz))), eps);
  if (fabsf(d) > r) return false;
  return true;
}

struct ShStack {
  uint32_t* base;
  int sp;
  static constexpr int kDepth = kSatDepth;
  __device__ __forceinline__ void push(uint32_t r) { base[sp++ * kSatThreads] = r; }
  __device__ __forceinline__ uint32_t pop() { return base[--sp * kSatThreads]; }
};
struct LcStack {
  uint32_t s[kSatDeepDepth];
  int sp;
  static constexpr int kDepth = kSatDeepDepth;
  __device__ __forceinline__ void push(uint32_t r) { s[sp++] = r; }
  __device__ __forceinline__ uint32_t pop() { return s[--sp]; }
};

// Visits every leaf triangle of the tree whose box may meet the query box;
// visit(const TriRec& t, uint32_t slot) returns true to stop.  Returns 0 =
// finished, 1 = stopped by visit, 2 = stack overflow.  Children are pushed
// last-first, so leaves are visited in a fixed (tree) order.
template <typename Stack, typename Visit>
__device__ __forceinline__ int box_traverse(const WideNode* __restrict__ nodes, const TriRec* __restrict__ tris,
                                            float mnx, float mny, float mnz, float mxx, float mxy, float mxz,
                                            Stack& st, Visit&& visit) {
  // pruning box: grown by a margin covering sat_eps and rounding
  const float mag = fmaxf(fmaxf(fmaxf(fabsf(mnx), fabsf(mxx)), fmaxf(fabsf(mny), fabsf(mxy))),
                          fmaxf(fabsf(mnz), fabsf(mxz)));
  const float g = 4e-6f + 4e-7f * mag;
  const float lx = mnx - g, ly = mny - g, lz = mnz - g, ux = mxx + g, uy = mxy + g, uz = mxz + g;
  uint32_t ref = 0;
  for (;;) {
    if (!ref_is_leaf(ref)) {
      const int4* np = reinterpret_cast<const int4*>(nodes + ref);
      const int4 w0 = __ldg(np), w1 = __ldg(np + 1), w2 = __ldg(np + 2), w3 = __ldg(np + 3);
      const float ox = __int_as_float(w0.x), oy = __int_as_float(w0.y), oz = __int_as_float(w0.z);
      const uint32_t meta = (uint32_t)w0.w;
      const float sx = __uint_as_float((meta & 0xffu) << 23);
      const float sy = __uint_as_float(((meta >> 8) & 0xffu) << 23);
      const float sz = __uint_as_float(((meta >> 16) & 0xffu) << 23);
      const int nch = (int)(meta >> 24);
      const uint32_t r[4] = {(uint32_t)w2.z, (uint32_t)w2.w, (uint32_t)w3.x, (uint32_t)w3.y};
      for (int c = nch - 1; c >= 0; --c) {
        const float clx = dequant((uint32_t)w1.x, c, sx, ox);
        const float cly = dequant((uint32_t)w1.y, c, sy, oy);
        const float clz = dequant((uint32_t)w1.z, c, sz, oz);
        const float chx = dequant((uint32_t)w1.w, c, sx, ox);
        const float chy = dequant((uint32_t)w2.x, c, sy, oy);
        const float chz = dequant((uint32_t)w2.y, c, sz, oz);
        const bool ov = clx <= ux && chx >= lx && cly <= uy && chy >= ly && clz <= uz && chz >= lz;
        if (ov) {
          if (st.sp >= Stack::kDepth) return 2;
          st.push(r[c]);
        }
      }
    } else {
      const uint32_t f0 = leaf_first(ref), cnt = leaf_count(ref);
      for (uint32_t i = 0; i < cnt; ++i) {
        const float4* p = reinterpret_cast<const float4*>(tris + f0 + i);
        TriRec t;
        t.a = __ldg(p); t.b = __ldg(p + 1); t.c = __ldg(p + 2); t.r = make_float4(0.f, 0.f, 0.f, 0.f);
        if (visit(t, f0 + i)) return 1;
      }
    }
    if (st.sp == 0) return 0;
    ref = st.pop();
  }
}


// any-hit SAT query; returns 0 = miss, 1 = hit, 2 = stack overflow
template <typename Stack>
__device__ int box_any_hit(const WideNode* __restrict__ nodes, const TriRec* __restrict__ tris, float mnx, float mny,
                           float mnz, float mxx, float mxy, float mxz, Stack& st) {
  return box_traverse(nodes, tris, mnx, mny, mnz, mxx, mxy, mxz, st, [&](const TriRec& t, uint32_t) {
    return sat_test(t, mnx, mny, mnz, mxx, mxy, mxz);
  });
}

}  // namespace a3d
