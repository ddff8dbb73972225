// Morton keys, triangle/box SAT any-hit queries and the coarse-to-fine
// octree descent.  A box "hits" when some triangle passes SAT (the test and
// the tree walk are in box_query.cuh).
#include <math.h>

#include "box_query.cuh"
#include "primitives.cuh"

namespace a3d {

namespace {

// ---- explicit boxes (MeshBVH.intersect_aabb mode 0) -----------------------
__global__ void __launch_bounds__(kSatThreads)
    aabb_hit_kernel(const WideNode* __restrict__ nodes, const TriRec* __restrict__ tris,
                    const float* __restrict__ bmin, const float* __restrict__ bmax, int64_t n,
                    uint8_t* __restrict__ hit, uint32_t* __restrict__ spill, uint32_t* __restrict__ nspill) {
  pdl_wait();
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
  pdl_wait();
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

constexpr uint32_t kNoHint = 0xffffffffu;  // no triangle to try first

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

// A candidate's hit decision: the triangle that hit its parent first (most
// children of a hit voxel meet the same triangle, which is several voxels
// wide at the finest levels), else an any-hit walk from the root.  The SAT
// predicate does not depend on the tree (the walk's pruning box is grown to
// cover sat_eps and rounding), so a hint that hits gives the decision the
// walk would give.  The hitting triangle's slot goes to ctri for the
// candidate's own children.
template <typename Stack>
__device__ __forceinline__ int candidate_hit(const WideNode* __restrict__ nodes, const TriRec* __restrict__ tris,
                                             const float* mn, const float* mx, uint32_t hint, Stack& st,
                                             uint32_t& hit_slot) {
  if (hint != kNoHint) {
    const float4* p = reinterpret_cast<const float4*>(tris + hint);
    TriRec t;
    t.a = __ldg(p); t.b = __ldg(p + 1); t.c = __ldg(p + 2); t.r = make_float4(0.f, 0.f, 0.f, 0.f);
    if (sat_test(t, mn[0], mn[1], mn[2], mx[0], mx[1], mx[2])) {
      hit_slot = hint;
      return 1;
    }
  }
  return box_traverse(nodes, tris, mn[0], mn[1], mn[2], mx[0], mx[1], mx[2], st, [&](const TriRec& t, uint32_t slot) {
    if (!sat_test(t, mn[0], mn[1], mn[2], mx[0], mx[1], mx[2])) return false;
    hit_slot = slot;
    return true;
  });
}

__global__ void __launch_bounds__(kSatThreads)
    octree_level_kernel(const WideNode* __restrict__ nodes, const TriRec* __restrict__ tris, int64_t ncand,
                        bool first_level, int res, const int32_t* __restrict__ parents,
                        const uint32_t* __restrict__ parent_hint, LevelGeom g, uint32_t* __restrict__ flags,
                        uint32_t* __restrict__ ctri, uint32_t* __restrict__ spill, uint32_t* __restrict__ nspill) {
  pdl_wait();
  __shared__ uint32_t s_stack[kSatDepth * kSatThreads];
  const int64_t k = (int64_t)blockIdx.x * kSatThreads + threadIdx.x;
  if (k >= ncand) return;
  int x, y, z;
  candidate_ijk(k, first_level, res, parents, x, y, z);
  float mn[3], mx[3];
  cube_box(x, y, z, g, mn, mx);
  ShStack st{s_stack + threadIdx.x, 0};
  uint32_t slot = kNoHint;
  const uint32_t hint = parent_hint ? parent_hint[k >> 3] : kNoHint;
  const int r = candidate_hit(nodes, tris, mn, mx, hint, st, slot);
  if (r == 2) {
    flags[k] = 0;
    spill[atomicAdd(nspill, 1u)] = (uint32_t)k;
  } else {
    flags[k] = (uint32_t)r;
    ctri[k] = slot;
  }
}

__global__ void octree_spill_kernel(const WideNode* __restrict__ nodes, const TriRec* __restrict__ tris,
                                    bool first_level, int res, const int32_t* __restrict__ parents,
                                    const uint32_t* __restrict__ parent_hint, LevelGeom g,
                                    uint32_t* __restrict__ flags, uint32_t* __restrict__ ctri,
                                    const uint32_t* __restrict__ spill, const uint32_t* __restrict__ nspill,
                                    int* __restrict__ overflow) {
  pdl_wait();
  const uint32_t m = *nspill;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < m; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t k = spill[t];
    int x, y, z;
    candidate_ijk(k, first_level, res, parents, x, y, z);
    float mn[3], mx[3];
    cube_box(x, y, z, g, mn, mx);
    LcStack st;
    st.sp = 0;
    uint32_t slot = kNoHint;
    // the hint was tested in the level kernel; the walk decides
    const int r = candidate_hit(nodes, tris, mn, mx, kNoHint, st, slot);
    (void)parent_hint;
    if (r == 2) atomicExch(overflow, 1);
    flags[k] = r == 1 ? 1u : 0u;
    ctri[k] = slot;
  }
}

// stable compaction of the hit candidates (flags hold the exclusive scan
// after the scan pass; hit tested again from the candidate's own flag copy)
__global__ void octree_compact_kernel(int64_t ncand, bool first_level, int res, const int32_t* __restrict__ parents,
                                      const uint8_t* __restrict__ hit, const uint32_t* __restrict__ offs,
                                      const uint32_t* __restrict__ ctri, int32_t* __restrict__ out32,
                                      uint32_t* __restrict__ hint_out, int64_t* __restrict__ out64) {
  pdl_wait();
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= ncand || !hit[k]) return;
  int x, y, z;
  candidate_ijk(k, first_level, res, parents, x, y, z);
  const int64_t o = offs[k];
  if (out64) {
    out64[3 * o] = x; out64[3 * o + 1] = y; out64[3 * o + 2] = z;
  } else {
    out32[3 * o] = x; out32[3 * o + 1] = y; out32[3 * o + 2] = z;
    hint_out[o] = ctri[k];
  }
}

__global__ void flags_to_u8_kernel(const uint32_t* __restrict__ f, int64_t n, uint8_t* __restrict__ h) {
  pdl_wait();
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) h[i] = (uint8_t)f[i];
}

// ---- Morton ------------------------------------------------------------------
__global__ void morton_encode_kernel(const int64_t* __restrict__ ijk, int64_t n, int64_t* __restrict__ out) {
  pdl_wait();
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  // bits 0..20 of each coordinate (two's complement bits, like the
  // reference's shift-and-mask loop)
  const uint64_t x = (uint64_t)ijk[3 * i], y = (uint64_t)ijk[3 * i + 1], z = (uint64_t)ijk[3 * i + 2];
  out[i] = (int64_t)(spread3_21(x) | (spread3_21(y) << 1) | (spread3_21(z) << 2));
}

__global__ void morton_decode_kernel(const int64_t* __restrict__ m, int64_t n, int level, int64_t* __restrict__ ijk) {
  pdl_wait();
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
  A3D_PDL(morton_encode_kernel, dim3((unsigned)ceil_div(n, 256)), dim3(256), 0, (cudaStream_t)stream, ijk, n, morton);
  return A3D_OK;
}

extern "C" int a3d_morton_decode(const int64_t* morton, int64_t n, int level, int64_t* ijk, a3d_stream_t stream) {
  A3D_REQUIRE(n >= 0 && level >= 0, A3D_ERR_ARGUMENT, "morton_decode: bad argument");
  if (n == 0) return A3D_OK;
  A3D_PDL(morton_decode_kernel, dim3((unsigned)ceil_div(n, 256)), dim3(256), 0, (cudaStream_t)stream, morton, n, level,
          ijk);
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
  A3D_PDL(aabb_hit_kernel, dim3((unsigned)ceil_div(n, kSatThreads)), dim3(kSatThreads), 0, s,
          (const WideNode*)bvh->nodes, (const TriRec*)bvh->tris, box_min, box_max, n, hit, spill, nspill);
  A3D_PDL(aabb_hit_spill_kernel, dim3(num_sms() * 4), dim3(64), 0, s, (const WideNode*)bvh->nodes,
          (const TriRec*)bvh->tris, box_min, box_max, hit, spill, nspill, (int*)(nspill + 1));
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
  uint32_t* hint_a;  // per entry of list_a: the triangle that hit it
  uint32_t* hint_b;
  uint32_t* ctri;    // per candidate: the triangle that hit it
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
  w.hint_a = ws.take<uint32_t>(cap);
  w.hint_b = ws.take<uint32_t>(cap);
  w.ctri = ws.take<uint32_t>(ncap);
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
  const uint32_t* parent_hint = nullptr;
  int32_t* next = w.list_a;
  uint32_t* next_hint = w.hint_a;
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
    A3D_PDL(octree_level_kernel, dim3(gk), dim3(kSatThreads), 0, s, nodes, tris, ncand, first_level, res, parents,
            parent_hint, g, w.flags, w.ctri, w.spill, w.misc + 1);
    A3D_PDL(octree_spill_kernel, dim3(num_sms() * 4), dim3(64), 0, s, nodes, tris, first_level, res, parents,
            parent_hint, g, w.flags, w.ctri, w.spill, w.misc + 1, (int*)(w.misc + 2));
    A3D_PDL(flags_to_u8_kernel, dim3((unsigned)ceil_div(ncand, 256)), dim3(256), 0, s, w.flags, ncand, w.hit);
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
    A3D_PDL(octree_compact_kernel, dim3((unsigned)ceil_div(ncand, 256)), dim3(256), 0, s, ncand, first_level, res,
            parents, w.hit, w.flags, w.ctri, last ? nullptr : next, last ? nullptr : next_hint,
            last ? out_ijk : nullptr);
    if (last || total == 0) {
      if (!last) *count_out = 0;
      break;
    }
    parents = next;
    parent_hint = next_hint;
    next = (next == w.list_a) ? w.list_b : w.list_a;
    next_hint = (next_hint == w.hint_a) ? w.hint_b : w.hint_a;
    ncand = total * 8;
  }
  return A3D_OK;
}
