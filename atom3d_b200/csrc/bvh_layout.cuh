// Memory layout of the wide BVH shared by the builder and every traversal.
//
// WideNode (64 B, one aligned half cache line, read as 4 x 16-B loads):
//   [ 0..11] float origin[3]       quantisation frame minimum
//   [12..15] uint32 meta           ex | ey << 8 | ez << 16 | nchild << 24
//                                  (ex = biased float exponent of the axis
//                                   scale: scale = uint_as_float(ex << 23))
//   [16..39] uint32 q[6]           qlo_x, qlo_y, qlo_z, qhi_x, qhi_y, qhi_z,
//                                  each packs the 8-bit value of children
//                                  0..3 in bytes 0..3
//   [40..55] uint32 ref[4]         child reference:
//                                    internal: node index (bit 31 clear)
//                                    leaf:     0x80000000 | (count-1) << 28 | first
//   [56..63] uint32 pad[2]
// Child c's box is origin + q * scale per axis; quantisation rounds outward,
// so the decoded box always contains the exact one.
//
// TriRec (64 B): float4 a (xyz, w = original face id as int bits),
//                float4 b (xyz, w = B = d01 / |n|^2),
//                float4 c (xyz, w = A = d11 / |n|^2, or -1 for a
//                          near-degenerate triangle, evaluated in FP64),
//                float4 r (1 / max(|b-a|^2, 1e-12), 1 / max(|c-b|^2, 1e-12),
//                          1 / max(|a-c|^2, 1e-12), C = d00 / |n|^2)
// with e0 = b - a, e1 = c - a, d00 = e0.e0, d01 = e0.e1, d11 = e1.e1 and
// |n|^2 = d00 d11 - d01^2: the dual-basis coefficients of the barycentric
// projection and the edge reciprocals let the per-triangle distance test run
// without a cross product or a divide.  a, b, c are the mesh's own vertex
// coordinates (the bit-exact ray, SAT and clip tests read only them).
#pragma once

#include <stdint.h>

namespace a3d {

struct __align__(64) WideNode {
  float ox, oy, oz;
  uint32_t meta;
  uint32_t q[6];
  uint32_t ref[4];
  uint32_t pad[2];
};
static_assert(sizeof(WideNode) == 64, "WideNode must be 64 bytes");

struct __align__(16) TriRec {
  float4 a, b, c, r;
};
static_assert(sizeof(TriRec) == 64, "TriRec must be 64 bytes");

constexpr uint32_t kLeafBit = 0x80000000u;
constexpr uint32_t kTriFlagNearDegenerate = 1u;  // evaluate in FP64
constexpr int kMaxLeafTris = 8;

// Decoded child-box coordinate origin + q * scale for the 8-bit value q held
// in byte `byte` of `word`.  The byte is turned into a float without the
// conversion unit: placed in the mantissa of 2^23 (0x4B0000qq) and 2^23
// subtracted, which is exact for q < 2^23; q * scale is exact (scale is a
// power of two), so the result equals fmaf((float)q, scale, origin).
__device__ __forceinline__ float dequant(uint32_t word, int byte, float scale, float origin) {
  const uint32_t sel = (uint32_t)byte | (4u << 4) | (5u << 8) | (7u << 12);
  const float q = __uint_as_float(__byte_perm(word, 0x4B000000u, sel)) - 8388608.0f;
  return fmaf(q, scale, origin);
}

__host__ __device__ __forceinline__ bool ref_is_leaf(uint32_t r) { return (r & kLeafBit) != 0; }
__host__ __device__ __forceinline__ uint32_t leaf_first(uint32_t r) { return r & 0x0fffffffu; }
__host__ __device__ __forceinline__ uint32_t leaf_count(uint32_t r) { return ((r >> 28) & 7u) + 1u; }
__host__ __device__ __forceinline__ uint32_t make_leaf_ref(uint32_t first, uint32_t count) {
  return kLeafBit | ((count - 1u) << 28) | first;
}

}  // namespace a3d
