// Morton keys, triangle/box SAT queries and the coarse-to-fine octree
// descent.
//
// SAT follows triangle_aabb_sat (atom3d/kernels/bvh_kernels.cu:285-353)
// operation by operation (box centre/half extents, 3 box axes, 9 edge cross
// axes, triangle plane, sat_eps = 1e-6).  Every multiply/add is an explicit
// round-to-nearest intrinsic so the compiler cannot contract it into an FMA:
// the result is then a pure function of IEEE single arithmetic and the CPU
// oracle (compiled with -ffp-contract=off) reproduces it bit for bit.
//
// A box "hits" when some triangle passes SAT.  The BVH only prunes: boxes
// are tested against child bounds grown by a margin that covers sat_eps and
// the rounding of the centre/half computation, so the hit set does not
// depend on the tree.
#include <math.h>

#include "bvh_layout.cuh"
#include "primitives.cuh"

namespace a3d {

namespace {

constexpr int kSatThreads = 128;
constexpr int kSatDepth = 48;
constexpr int kSatDeepDepth = 512;

__device__ __forceinline__ float fm(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fa(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fsb(float a, float b) { return __fsub_rn(a, b); }

__device__ __forceinline__ float dot3r(float ax, float ay, float az, float bx, float by, float bz) {
  return fa(fa(fm(ax, bx), fm(ay, by)), fm(az, bz));
}

__device__ bool sat_test(const TriRec& t, float mnx, float mny, float mnz, float mxx, float mxy, float mxz) {
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

// any-hit SAT query; returns 0 = miss, 1 = hit, 2 = stack overflow
template <typename Stack>
__device__ int box_any_hit(const WideNode* __restrict__ nodes, const TriRec* __restrict__ tris, float mnx, float mny,
                           float mnz, float mxx, float mxy, float mxz, Stack& st) {
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
        if (sat_test(t, mnx, mny, mnz, mxx, mxy, mxz)) return 1;
      }
    }
    if (st.sp == 0) return 0;
    ref = st.pop();
  }
}

// ---- explicit boxes (MeshBVH.intersect_aabb mode 0) -----------------------
__global__ void __launch_bounds__(kSatThreads)
    aabb_hit_kernel(const WideNode* __restrict__ nodes, const TriRec* __restrict__ tris,
                    const float* __restrict__ bmin, const float* __restrict__ bmax, int64_t n,
                    uint8_t* __restrict__ hit, uint32_t* __restrict__ spill, uint32_t* __restrict__ nspill) {
  __shared__ uint32_t s_stack[kSatDepth * kSatThreads];
  const int64_t i = (int64_t)blockIdx.x * kSatThreads + threadIdx.x;
  if (i >= n) return;
  ShStack st{s_stack + threadIdx.x, 0};
  const int r = box_any_hit(nodes, tris, bmin[3 * i], bmin[3 * i + 1], bmin[3 * i + 2], bmax[3 * i], bmax[3 * i + 1],
                            bmax[3 * i + 2], st);
  if (r == 2) {
    spill[atomicAdd(nspill, 1u)] = (uint32_t)i;
  } else {
    hit[i] = (uint8_t)r;
  }
}

__global__ void aabb_hit_spill_kernel(const WideNode* __restrict__ nodes, const TriRec* __restrict__ tris,
                                      const float* __restrict__ bmin, const float* __restrict__ bmax,
                                      uint8_t* __restrict__ hit, const uint32_t* __restrict__ spill,
                                      const uint32_t* __restrict__ nspill, int* __restrict__ overflow) {
  const uint32_t m = *nspill;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < m; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = spill[t];
    LcStack st;
    st.sp = 0;
    const int r = box_any_hit(nodes, tris, bmin[3 * i], bmin[3 * i + 1], bmin[3 * i + 2], bmax[3 * i],
                              bmax[3 * i + 1], bmax[3 * i + 2], st);
    if (r == 2) atomicExch(overflow, 1);
    hit[i] = r == 1 ? 1 : 0;
  }
}

// ---- octree levels ----------------------------------------------------------
struct LevelGeom {
  float lo[3];
  float cell[3];
};

__device__ __forceinline__ void cube_box(int x, int y, int z, const LevelGeom& g, float* mn, float* mx) {
  // aabb_min = float(ijk) * cell + lo ; aabb_max = aabb_min + cell  (two roundings, no FMA)
  const int ijk[3] = {x, y, z};
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    mn[a] = fa(fm((float)ijk[a], g.cell[a]), g.lo[a]);
    mx[a] = fa(mn[a], g.cell[a]);
  }
}

// candidate k of this level: either cube k of the full min_level grid
// (meshgrid 'ij': x slowest, z fastest) or child (k & 7) of parent k >> 3
__device__ __forceinline__ void candidate_ijk(int64_t k, bool first_level, int res, const int32_t* parents, int& x,
                                              int& y, int& z) {
  if (first_level) {
    x = (int)(k / ((int64_t)res * res));
    y = (int)((k / res) % res);
    z = (int)(k % res);
  } else {
    const int64_t p = k >> 3;
    const int c = (int)(k & 7);
    x = 2 * parents[3 * p] + (c & 1);
    y = 2 * parents[3 * p + 1] + ((c >> 1) & 1);
    z = 2 * parents[3 * p + 2] + ((c >> 2) & 1);
  }
}

__global__ void __launch_bounds__(kSatThreads)
    octree_level_kernel(const WideNode* __restrict__ nodes, const TriRec* __restrict__ tris, int64_t ncand,
                        bool first_level, int res, const int32_t* __restrict__ parents, LevelGeom g,
                        uint32_t* __restrict__ flags, uint32_t* __restrict__ spill, uint32_t* __restrict__ nspill) {
  __shared__ uint32_t s_stack[kSatDepth * kSatThreads];
  const int64_t k = (int64_t)blockIdx.x * kSatThreads + threadIdx.x;
  if (k >= ncand) return;
  int x, y, z;
  candidate_ijk(k, first_level, res, parents, x, y, z);
  float mn[3], mx[3];
  cube_box(x, y, z, g, mn, mx);
  ShStack st{s_stack + threadIdx.x, 0};
  const int r = box_any_hit(nodes, tris, mn[0], mn[1], mn[2], mx[0], mx[1], mx[2], st);
  if (r == 2) {
    flags[k] = 0;
    spill[atomicAdd(nspill, 1u)] = (uint32_t)k;
  } else {
    flags[k] = (uint32_t)r;
  }
}

__global__ void octree_spill_kernel(const WideNode* __restrict__ nodes, const TriRec* __restrict__ tris,
                                    bool first_level, int res, const int32_t* __restrict__ parents, LevelGeom g,
                                    uint32_t* __restrict__ flags, const uint32_t* __restrict__ spill,
                                    const uint32_t* __restrict__ nspill, int* __restrict__ overflow) {
  const uint32_t m = *nspill;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < m; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t k = spill[t];
    int x, y, z;
    candidate_ijk(k, first_level, res, parents, x, y, z);
    float mn[3], mx[3];
    cube_box(x, y, z, g, mn, mx);
    LcStack st;
    st.sp = 0;
    const int r = box_any_hit(nodes, tris, mn[0], mn[1], mn[2], mx[0], mx[1], mx[2], st);
    if (r == 2) atomicExch(overflow, 1);
    flags[k] = r == 1 ? 1u : 0u;
  }
}

// stable compaction of the hit candidates (flags hold the exclusive scan
// after the scan pass; hit tested again from the candidate's own flag copy)
__global__ void octree_compact_kernel(int64_t ncand, bool first_level, int res, const int32_t* __restrict__ parents,
                                      const uint8_t* __restrict__ hit, const uint32_t* __restrict__ offs,
                                      int32_t* __restrict__ out32, int64_t* __restrict__ out64) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= ncand || !hit[k]) return;
  int x, y, z;
  candidate_ijk(k, first_level, res, parents, x, y, z);
  const int64_t o = offs[k];
  if (out64) {
    out64[3 * o] = x; out64[3 * o + 1] = y; out64[3 * o + 2] = z;
  } else {
    out32[3 * o] = x; out32[3 * o + 1] = y; out32[3 * o + 2] = z;
  }
}

__global__ void flags_to_u8_kernel(const uint32_t* __restrict__ f, int64_t n, uint8_t* __restrict__ h) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) h[i] = (uint8_t)f[i];
}

// ---- Morton ------------------------------------------------------------------
__global__ void morton_encode_kernel(const int64_t* __restrict__ ijk, int64_t n, int64_t* __restrict__ out) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  // bits 0..20 of each coordinate (two's complement bits, like the
  // reference's shift-and-mask loop)
  const uint64_t x = (uint64_t)ijk[3 * i], y = (uint64_t)ijk[3 * i + 1], z = (uint64_t)ijk[3 * i + 2];
  out[i] = (int64_t)(spread3_21(x) | (spread3_21(y) << 1) | (spread3_21(z) << 2));
}

__global__ void morton_decode_kernel(const int64_t* __restrict__ m, int64_t n, int level, int64_t* __restrict__ ijk) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint64_t v = (uint64_t)m[i];
  const int bits = level + 1 < 21 ? level + 1 : 21;
  const uint64_t mask = bits >= 64 ? ~0ull : ((1ull << bits) - 1);
  ijk[3 * i] = (int64_t)(compact3_21(v) & mask);
  ijk[3 * i + 1] = (int64_t)(compact3_21(v >> 1) & mask);
  ijk[3 * i + 2] = (int64_t)(compact3_21(v >> 2) & mask);
}

}  // namespace
}  // namespace a3d

using namespace a3d;

extern "C" int a3d_morton_encode(const int64_t* ijk, int64_t n, int64_t* morton, a3d_stream_t stream) {
  A3D_REQUIRE(n >= 0, A3D_ERR_ARGUMENT, "morton_encode: bad size");
  if (n == 0) return A3D_OK;
  morton_encode_kernel<<<(unsigned)ceil_div(n, 256), 256, 0, (cudaStream_t)stream>>>(ijk, n, morton);
  A3D_LAUNCH_CHECK();
  return A3D_OK;
}

extern "C" int a3d_morton_decode(const int64_t* morton, int64_t n, int level, int64_t* ijk, a3d_stream_t stream) {
  A3D_REQUIRE(n >= 0 && level >= 0, A3D_ERR_ARGUMENT, "morton_decode: bad argument");
  if (n == 0) return A3D_OK;
  morton_decode_kernel<<<(unsigned)ceil_div(n, 256), 256, 0, (cudaStream_t)stream>>>(morton, n, level, ijk);
  A3D_LAUNCH_CHECK();
  return A3D_OK;
}

extern "C" size_t a3d_aabb_hit_workspace_bytes(int64_t n) {
  Workspace ws(nullptr, 0);
  ws.take<uint32_t>(n);
  ws.take<uint32_t>(4);
  return ws.used + 256;
}

extern "C" int a3d_aabb_hit(const a3d_bvh_view* bvh, const float* box_min, const float* box_max, int64_t n,
                            uint8_t* hit, void* workspace, size_t workspace_bytes, a3d_stream_t stream) {
  cudaStream_t s = (cudaStream_t)stream;
  A3D_REQUIRE(bvh && bvh->nodes && bvh->tris, A3D_ERR_ARGUMENT, "aabb_hit: invalid bvh");
  A3D_REQUIRE(n >= 0 && n < (1ll << 32), A3D_ERR_ARGUMENT, "aabb_hit: bad size");
  if (n == 0) return A3D_OK;
  Workspace ws(workspace, workspace_bytes);
  uint32_t* spill = ws.take<uint32_t>(n);
  uint32_t* nspill = ws.take<uint32_t>(4);
  A3D_REQUIRE(workspace && ws.ok(), A3D_ERR_WORKSPACE, "aabb_hit: workspace too small");
  A3D_CUDA_TRY(cudaMemsetAsync(nspill, 0, 4 * sizeof(uint32_t), s));
  aabb_hit_kernel<<<(unsigned)ceil_div(n, kSatThreads), kSatThreads, 0, s>>>(
      (const WideNode*)bvh->nodes, (const TriRec*)bvh->tris, box_min, box_max, n, hit, spill, nspill);
  A3D_LAUNCH_CHECK();
  aabb_hit_spill_kernel<<<kNumSMs * 4, 64, 0, s>>>((const WideNode*)bvh->nodes, (const TriRec*)bvh->tris, box_min,
                                                   box_max, hit, spill, nspill, (int*)(nspill + 1));
  A3D_LAUNCH_CHECK();
  int ov = 0;
  A3D_CUDA_TRY(cudaMemcpyAsync(&ov, nspill + 1, sizeof(int), cudaMemcpyDeviceToHost, s));
  A3D_CUDA_TRY(cudaStreamSynchronize(s));
  A3D_REQUIRE(ov == 0, A3D_ERR_OVERFLOW, "aabb_hit: traversal stack overflow");
  return A3D_OK;
}

namespace {
struct OctWs {
  int32_t* list_a;
  int32_t* list_b;
  uint32_t* flags;
  uint8_t* hit;
  uint32_t* scan_tmp;
  uint32_t* spill;
  uint32_t* misc;  // [0] total, [1] spill count, [2] overflow
};
size_t carve_oct(OctWs& w, Workspace& ws, int64_t cap) {
  const int64_t ncap = 8 * cap;
  w.list_a = ws.take<int32_t>(3 * cap);
  w.list_b = ws.take<int32_t>(3 * cap);
  w.flags = ws.take<uint32_t>(ncap);
  w.hit = ws.take<uint8_t>(ncap);
  w.scan_tmp = ws.take<uint32_t>((int64_t)scan_workspace_elems(ncap));
  w.spill = ws.take<uint32_t>(ncap);
  w.misc = ws.take<uint32_t>(8);
  return ws.used;
}
}  // namespace

extern "C" size_t a3d_octree_workspace_bytes(int min_level, int max_level, int64_t cap) {
  (void)max_level;
  const int64_t first = 1ll << (3 * min_level);
  const int64_t c = cap > first ? cap : first;
  Workspace ws(nullptr, 0);
  OctWs w;
  return carve_oct(w, ws, c) + 256;
}

extern "C" int a3d_octree_traverse(const a3d_bvh_view* bvh, const float* grid_lo, const float* cell_sizes,
                                   int min_level, int max_level, int64_t* out_ijk, int64_t cap, int64_t* count_out,
                                   void* workspace, size_t workspace_bytes, a3d_stream_t stream) {
  cudaStream_t s = (cudaStream_t)stream;
  A3D_REQUIRE(bvh && bvh->nodes && bvh->tris, A3D_ERR_ARGUMENT, "octree: invalid bvh");
  A3D_REQUIRE(min_level >= 0 && max_level >= min_level && max_level <= 20, A3D_ERR_ARGUMENT,
              "octree: bad levels");
  A3D_REQUIRE(min_level <= 9, A3D_ERR_ARGUMENT, "octree: min_level above 9 (2^27 cubes) not supported");
  A3D_REQUIRE(count_out && grid_lo && cell_sizes, A3D_ERR_ARGUMENT, "octree: null argument");
  const int64_t first = 1ll << (3 * min_level);
  const int64_t c = cap > first ? cap : first;
  Workspace ws(workspace, workspace_bytes);
  OctWs w;
  carve_oct(w, ws, c);
  A3D_REQUIRE(workspace && ws.ok(), A3D_ERR_WORKSPACE, "octree: workspace too small");
  const WideNode* nodes = (const WideNode*)bvh->nodes;
  const TriRec* tris = (const TriRec*)bvh->tris;
  int64_t ncand = first;
  const int32_t* parents = nullptr;
  int32_t* next = w.list_a;
  *count_out = 0;
  for (int level = min_level; level <= max_level; ++level) {
    const bool first_level = level == min_level;
    const int res = 1 << level;
    LevelGeom g;
    for (int a = 0; a < 3; ++a) {
      g.lo[a] = grid_lo[a];
      g.cell[a] = cell_sizes[3 * level + a];
    }
    if (ncand > 8 * c) {
      *count_out = -1;
      A3D_REQUIRE(false, A3D_ERR_WORKSPACE, "octree: candidate capacity exceeded");
    }
    A3D_CUDA_TRY(cudaMemsetAsync(w.misc, 0, 8 * sizeof(uint32_t), s));
    const unsigned gk = (unsigned)ceil_div(ncand, kSatThreads);
    octree_level_kernel<<<gk, kSatThreads, 0, s>>>(nodes, tris, ncand, first_level, res, parents, g, w.flags, w.spill,
                                                   w.misc + 1);
    A3D_LAUNCH_CHECK();
    octree_spill_kernel<<<kNumSMs * 4, 64, 0, s>>>(nodes, tris, first_level, res, parents, g, w.flags, w.spill,
                                                   w.misc + 1, (int*)(w.misc + 2));
    A3D_LAUNCH_CHECK();
    flags_to_u8_kernel<<<(unsigned)ceil_div(ncand, 256), 256, 0, s>>>(w.flags, ncand, w.hit);
    A3D_LAUNCH_CHECK();
    A3D_TRY((device_exclusive_scan<uint32_t, uint32_t>(w.flags, w.flags, ncand, w.scan_tmp, w.misc, s)));
    uint32_t hm[3];
    A3D_CUDA_TRY(cudaMemcpyAsync(hm, w.misc, 3 * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    A3D_CUDA_TRY(cudaStreamSynchronize(s));
    A3D_REQUIRE(hm[2] == 0, A3D_ERR_OVERFLOW, "octree: traversal stack overflow");
    const int64_t total = hm[0];
    const bool last = level == max_level;
    if (last) {
      *count_out = total;
      if (total > cap) {
        A3D_REQUIRE(false, A3D_ERR_WORKSPACE, "octree: output capacity exceeded");
      }
    } else if (total > c) {
      *count_out = -1;
      A3D_REQUIRE(false, A3D_ERR_WORKSPACE, "octree: level capacity exceeded");
    }
    octree_compact_kernel<<<(unsigned)ceil_div(ncand, 256), 256, 0, s>>>(ncand, first_level, res, parents, w.hit,
                                                                         w.flags, last ? nullptr : next,
                                                                         last ? out_ijk : nullptr);
    A3D_LAUNCH_CHECK();
    if (last || total == 0) {
      if (!last) *count_out = 0;
      break;
    }
    parents = next;
    next = (next == w.list_a) ? w.list_b : w.list_a;
    ncand = total * 8;
  }
  return A3D_OK;
}
