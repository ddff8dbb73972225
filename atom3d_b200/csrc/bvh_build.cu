// GPU construction of the wide BVH, for one mesh or a batch of meshes.
//
// Replaces the reference's single-threaded host SAH builder
// (atom3d/kernels/bvh_kernels.cu:616-925).  Pipeline, all on the stream and
// without a host synchronisation, so a whole (batched) build can be captured
// in a CUDA graph:
//   1. per-triangle AABB/centroid; per-mesh scene and centroid bounds
//      (block reduce, one atomic per block and mesh)
//   2. sort key = mesh id in the high bits | Morton code of the centroid in
//      its mesh's centroid box (21 bits per axis for one mesh; fewer when
//      the mesh id needs bits)
//   3. stable radix sort of (key, face) with the in-house sort; mesh m's
//      faces then occupy sorted positions [face_off[m], face_off[m+1])
//   4. one binary radix tree per mesh over its sorted range [s, e): internal
//      nodes s..e-2 with root s, leaf j at N + j (duplicate codes
//      disambiguated by index)
//   4b. SAH refinement: every subtree of at most 16384 triangles below the
//      top of the tree is rebuilt top-down with binned SAH by one thread
//      block (bvh_sah.cuh), in place and within its own index range
//   5. bottom-up refit (second arriving child computes the union box)
//   6. SAH-optimal collapse into 4-wide quantised nodes: the refit also
//      computes, bottom-up, the cheapest cover of every subtree by 1..4 wide
//      slots (leaf or wide node, weighted by surface area); a wide node's
//      children are the subtrees that cover chose, leaves hold at most
//      leaf_max triangles.  Level-synchronous over device-side worklists; a wide node is
//      written at the slot of its binary node, so the order in which a
//      level's work is done does not matter
//   7. layout: wide nodes stably sorted by level -- breadth first, each
//      node's children contiguous, mesh roots at 0..M-1 -- and child
//      references renumbered
//   8. triangle records in sorted order (64 B, with reciprocals)
#include <math.h>
#include <string.h>

#include "bvh_layout.cuh"
#include "bvh_sah.cuh"
#include "primitives.cuh"

namespace a3d {

namespace {

constexpr int kThreads = 256;
constexpr int kMaxLevels = 64;  // wide levels; deeper trees report A3D_ERR_OVERFLOW
constexpr uint32_t kNoLevel = 255u;
// leaves of up to 8 triangles: fewer, larger leaves trade node tests for
// cheaper triangle tests (16M-query closest-point workload on a 1.31M-
// triangle mesh: 201 ms at 8 vs 226 ms at 4)
constexpr int kDefaultLeafMax = 8;

struct BuildWs {
  int64_t* face_off;    // single-mesh builds: offsets written on the device
  int64_t* vert_off;
  float4* tri_lo;
  float4* tri_hi;
  float4* centroid;
  uint32_t* mesh_of;    // mesh id per (original) face
  uint32_t* bounds;     // [M][12] flipped floats: scene lo, scene hi, cent lo, cent hi
  int32_t* err;         // [0] face index out of range / empty mesh, [1] depth overflow
  uint64_t* keys;
  uint64_t* keys_alt;
  uint32_t* vals;
  uint32_t* vals_alt;
  uint32_t* rs_scratch;
  int32_t* left;
  int32_t* right;
  int32_t* parent;      // [2N]
  int32_t* first;
  int32_t* last;
  float4* box_lo;       // [2N]: internal 0..N-1 (per-mesh ranges), leaf j at N+j
  float4* box_hi;
  uint32_t* visit;
  int32_t* work_a;
  int32_t* work_b;
  uint32_t* counters;   // [kMaxLevels + 1] worklist sizes per level
  WideNode* tmp_nodes;  // [N] wide node at the slot of its binary node
  uint32_t* lvl;        // [N] level of the wide node at a slot, kNoLevel if none
  uint32_t* lvl_alt;
  uint32_t* slot;
  uint32_t* slot_alt;
  uint32_t* newidx;     // [N] slot -> final node index
  int64_t* count;       // single-mesh builds: node count
  int32_t* clusters;    // [N] roots of the subtrees the SAH pass rebuilds
  uint32_t* ncl;        // their count
  float4* dp_cost;      // [N] collapse cost of each internal node spread over 1..4 wide slots
  uint32_t* dp_dec;     // [N] the decisions behind dp_cost (see refit_kernel)
  uint32_t* sah_tmp;    // [N] partition scratch of the SAH pass
  SahNode* sah_small;   // [N] its lists of small nodes
};

size_t carve(BuildWs& w, Workspace& ws, int64_t n, int64_t m) {
  w.face_off = ws.take<int64_t>(2);
  w.vert_off = ws.take<int64_t>(2);
  w.tri_lo = ws.take<float4>(n);
  w.tri_hi = ws.take<float4>(n);
  w.centroid = ws.take<float4>(n);
  w.mesh_of = ws.take<uint32_t>(n);
  w.bounds = ws.take<uint32_t>(12 * m);
  w.err = ws.take<int32_t>(4);
  w.keys = ws.take<uint64_t>(n);
  w.keys_alt = ws.take<uint64_t>(n);
  w.vals = ws.take<uint32_t>(n);
  w.vals_alt = ws.take<uint32_t>(n);
  w.rs_scratch = ws.take<uint32_t>((int64_t)radix_sort_scratch_elems(n));
  w.left = ws.take<int32_t>(n);
  w.right = ws.take<int32_t>(n);
  w.parent = ws.take<int32_t>(2 * n);
  w.first = ws.take<int32_t>(n);
  w.last = ws.take<int32_t>(n);
  w.box_lo = ws.take<float4>(2 * n);
  w.box_hi = ws.take<float4>(2 * n);
  w.visit = ws.take<uint32_t>(n);
  w.work_a = ws.take<int32_t>(n);
  w.work_b = ws.take<int32_t>(n);
  w.counters = ws.take<uint32_t>(kMaxLevels + 1);
  w.tmp_nodes = ws.take<WideNode>(n);
  w.lvl = ws.take<uint32_t>(n);
  w.lvl_alt = ws.take<uint32_t>(n);
  w.slot = ws.take<uint32_t>(n);
  w.slot_alt = ws.take<uint32_t>(n);
  w.newidx = ws.take<uint32_t>(n);
  w.count = ws.take<int64_t>(1);
  w.clusters = ws.take<int32_t>(n);
  w.ncl = ws.take<uint32_t>(1);
  w.dp_cost = ws.take<float4>(n);
  w.dp_dec = ws.take<uint32_t>(n);
  w.sah_tmp = ws.take<uint32_t>(n);
  w.sah_small = ws.take<SahNode>(n);
  return ws.used;
}

__device__ __forceinline__ float3 ld3(const float* p, int64_t i) {
  return make_float3(p[3 * i], p[3 * i + 1], p[3 * i + 2]);
}

// index m with off[m] <= i < off[m+1] (off ascending, off[0] = 0)
__device__ __forceinline__ int segment_of(const int64_t* __restrict__ off, int nseg, int64_t i) {
  int lo = 0, hi = nseg - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (off[mid] <= i) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

__global__ void single_offsets_kernel(int64_t* face_off, int64_t* vert_off, int64_t nf, int64_t nv) {
  pdl_wait();
  if (threadIdx.x == 0) {
    face_off[0] = 0;
    face_off[1] = nf;
    vert_off[0] = 0;
    vert_off[1] = nv;
  }
}

// per-mesh bounds, error words, level counters and the level-0 worklist
// (the mesh roots: internal node s, or the lone leaf N + s)
__global__ void init_kernel(const int64_t* __restrict__ face_off, int nmesh, int64_t n, uint32_t* bounds,
                            int32_t* err, uint32_t* counters, int32_t* work0) {
  pdl_wait();
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < 12 * (int64_t)nmesh) bounds[t] = (((t % 12) / 3) % 2 == 0) ? 0xffffffffu : 0u;
  if (t < 4) err[t] = 0;
  if (t <= kMaxLevels) counters[t] = t == 0 ? (uint32_t)nmesh : 0u;
  if (t < nmesh) {
    const int64_t s = face_off[t], e = face_off[t + 1];
    if (e <= s) atomicExch(err, 1);
    work0[t] = (int32_t)(e - s > 1 ? s : n + s);
  }
}

// v[0..5]: minima (scene lo, centroid lo), v[6..11]: maxima (scene hi, centroid hi)
__device__ __forceinline__ void bounds_atomic(uint32_t* b, const float* v) {
#pragma unroll
  for (int k = 0; k < 12; ++k) {
    const int slot = k < 3 ? k : (k < 6 ? 6 + (k - 3) : (k < 9 ? 3 + (k - 6) : 9 + (k - 9)));
    if (isfinite(v[k])) {
      if (k < 6) atomicMin(&b[slot], float_flip(v[k]));
      else atomicMax(&b[slot], float_flip(v[k]));
    }
  }
}

// 1. triangle boxes, centroids, mesh ids, per-mesh bounds
__global__ void __launch_bounds__(kThreads)
    tri_prep_kernel(const float* __restrict__ V, const int64_t* __restrict__ vert_off, const int32_t* __restrict__ F,
                    const int64_t* __restrict__ face_off, int nmesh, int64_t nf, float4* __restrict__ tri_lo,
                    float4* __restrict__ tri_hi, float4* __restrict__ cen, uint32_t* __restrict__ mesh_of,
                    uint32_t* __restrict__ bounds, int32_t* __restrict__ err) {
  pdl_wait();
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t i0b = (int64_t)blockIdx.x * blockDim.x;
  __shared__ int s_m0;
  if (threadIdx.x == 0) s_m0 = segment_of(face_off, nmesh, i0b);
  __syncthreads();
  const int m0 = s_m0;
  float v[12];
#pragma unroll
  for (int k = 0; k < 6; ++k) { v[k] = INFINITY; v[k + 6] = -INFINITY; }
  if (i < nf) {
    const int m = segment_of(face_off, nmesh, i);
    mesh_of[i] = (uint32_t)m;
    const int64_t vb = vert_off[m], nv = vert_off[m + 1] - vb;
    int32_t i0 = F[3 * i], i1 = F[3 * i + 1], i2 = F[3 * i + 2];
    if (i0 < 0 || i1 < 0 || i2 < 0 || i0 >= nv || i1 >= nv || i2 >= nv) {
      atomicExch(err, 1);
      i0 = i1 = i2 = 0;
    }
    const float3 a = ld3(V, vb + i0), b = ld3(V, vb + i1), c = ld3(V, vb + i2);
    const float3 lo = make_float3(fminf(fminf(a.x, b.x), c.x), fminf(fminf(a.y, b.y), c.y), fminf(fminf(a.z, b.z), c.z));
    const float3 hi = make_float3(fmaxf(fmaxf(a.x, b.x), c.x), fmaxf(fmaxf(a.y, b.y), c.y), fmaxf(fmaxf(a.z, b.z), c.z));
    const float3 ce = make_float3((a.x + b.x + c.x) * (1.0f / 3.0f), (a.y + b.y + c.y) * (1.0f / 3.0f),
                                  (a.z + b.z + c.z) * (1.0f / 3.0f));
    tri_lo[i] = make_float4(lo.x, lo.y, lo.z, 0.f);
    tri_hi[i] = make_float4(hi.x, hi.y, hi.z, 0.f);
    cen[i] = make_float4(ce.x, ce.y, ce.z, 0.f);
    v[0] = lo.x; v[1] = lo.y; v[2] = lo.z;
    v[3] = ce.x; v[4] = ce.y; v[5] = ce.z;
    v[6] = hi.x; v[7] = hi.y; v[8] = hi.z;
    v[9] = ce.x; v[10] = ce.y; v[11] = ce.z;
    if (m != m0) {
      // a block straddling meshes: faces not of the block's first mesh
      // contribute directly
      bounds_atomic(bounds + 12 * (int64_t)m, v);
#pragma unroll
      for (int k = 0; k < 6; ++k) { v[k] = INFINITY; v[k + 6] = -INFINITY; }
    }
  }
  // block reduce for the block's first mesh
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      v[k] = fminf(v[k], __shfl_xor_sync(0xffffffffu, v[k], o));
      v[k + 6] = fmaxf(v[k + 6], __shfl_xor_sync(0xffffffffu, v[k + 6], o));
    }
  }
  __shared__ float s[kThreads / 32][12];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0)
    for (int k = 0; k < 12; ++k) s[warp][k] = v[k];
  __syncthreads();
  if (threadIdx.x == 0 && i0b < nf) {
    float r[12];
    for (int k = 0; k < 12; ++k) {
      r[k] = s[0][k];
      for (int w = 1; w < kThreads / 32; ++w) r[k] = k < 6 ? fminf(r[k], s[w][k]) : fmaxf(r[k], s[w][k]);
    }
    bounds_atomic(bounds + 12 * (int64_t)m0, r);
  }
}

// 2. sort keys: mesh id above the Morton code of the centroid
__global__ void morton_kernel(const float4* __restrict__ cen, const uint32_t* __restrict__ mesh_of, int64_t n,
                              const uint32_t* __restrict__ bounds, int bits, uint64_t* __restrict__ keys,
                              uint32_t* __restrict__ vals) {
  pdl_wait();
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t m = mesh_of[i];
  const uint32_t* b = bounds + 12 * (int64_t)m;
  const float lo[3] = {float_unflip(b[6]), float_unflip(b[7]), float_unflip(b[8])};
  const float hi[3] = {float_unflip(b[9]), float_unflip(b[10]), float_unflip(b[11])};
  const float4 c = cen[i];
  const float cc[3] = {c.x, c.y, c.z};
  const float qmax = (float)((1u << bits) - 1u);
  uint64_t code = 0;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const float ext = hi[a] - lo[a];
    float t = ext > 0.f ? (cc[a] - lo[a]) / ext : 0.f;
    t = fminf(fmaxf(t, 0.f), 1.f);
    const uint64_t q = (uint64_t)(t * qmax);
    code |= spread3_21(q) << a;
  }
  keys[i] = ((uint64_t)m << (3 * bits)) | code;
  vals[i] = (uint32_t)i;
}

// 4. binary radix tree of each mesh's sorted range
__device__ __forceinline__ int delta(const uint64_t* keys, int64_t s, int64_t e, int i, int j) {
  if (j < s || j >= e) return -1;
  const uint64_t a = keys[i], b = keys[j];
  if (a != b) return __clzll((long long)(a ^ b));
  return 64 + __clz(i ^ j);
}

__global__ void radix_tree_kernel(const uint64_t* __restrict__ keys, const int64_t* __restrict__ face_off, int nmesh,
                                  int64_t n, int32_t* __restrict__ left, int32_t* __restrict__ right,
                                  int32_t* __restrict__ parent, int32_t* __restrict__ first,
                                  int32_t* __restrict__ last) {
  pdl_wait();
  const int64_t ii = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (ii >= n) return;
  const int i = (int)ii;
  const int m = segment_of(face_off, nmesh, ii);
  const int64_t s = face_off[m], e = face_off[m + 1];
  if (ii == e - 1) {
    // the last position of a range carries no internal node; a lone leaf
    // is its mesh's root
    if (e - s == 1) parent[n + s] = -1;
    return;
  }
  const int d = (delta(keys, s, e, i, i + 1) - delta(keys, s, e, i, i - 1)) >= 0 ? 1 : -1;
  const int dmin = delta(keys, s, e, i, i - d);
  int lmax = 2;
  while (delta(keys, s, e, i, i + lmax * d) > dmin) lmax <<= 1;
  int l = 0;
  for (int t = lmax >> 1; t > 0; t >>= 1)
    if (delta(keys, s, e, i, i + (l + t) * d) > dmin) l += t;
  const int j = i + l * d;
  const int dnode = delta(keys, s, e, i, j);
  int sp = 0;
  int t = l;
  do {
    t = (t + 1) >> 1;
    if (delta(keys, s, e, i, i + (sp + t) * d) > dnode) sp += t;
  } while (t > 1);
  const int gamma = i + sp * d + (d < 0 ? -1 : 0);
  const int lo = min(i, j), hi = max(i, j);
  const int lc = (lo == gamma) ? (int)n + gamma : gamma;
  const int rc = (hi == gamma + 1) ? (int)n + gamma + 1 : gamma + 1;
  left[i] = lc;
  right[i] = rc;
  parent[lc] = i;
  parent[rc] = i;
  first[i] = lo;
  last[i] = hi;
  if (ii == s) parent[i] = -1;
}

__device__ __forceinline__ float half_area(float4 lo, float4 hi) {
  const float dx = hi.x - lo.x, dy = hi.y - lo.y, dz = hi.z - lo.z;
  return dx * dy + dy * dz + dz * dx;
}

// Cost weights of the SAH-optimal collapse: a wide-node visit against one
// triangle test, as measured on the closest-point traversal.  With the
// barycentric triangle test a 4-box node visit costs more triangle tests than
// before: on the 16M-query workload the traversal time is flat for weights
// 12-24 and lowest near 16 (148.4 ms; 150.6 ms at the 6.7 fitted for the
// cross-product test, 156.3 ms at 5)
#ifndef A3D_SAH_NODE_COST
#define A3D_SAH_NODE_COST 16.0f
#endif
constexpr float kCostNode = A3D_SAH_NODE_COST, kCostTri = 1.0f;

// 5. refit: leaf boxes from sorted triangles, unions bottom-up; and, at each
// internal node, the SAH-optimal collapse costs.  cost[i] (i = 1..4) is the
// cheapest way to cover the node's subtree with i slots of a wide node:
//   cost[1] = min(leaf: kCostTri * A * count   (count <= leaf_max, not a root),
//                 wide node: kCostNode * A + min over j = 2..4 of split[j])
//   split[j] = min over k of cost_left[k] + cost_right[j - k]
//   cost[i > 1] = min(cost[i - 1], split[i])
// with A the node's half surface area (a binary leaf costs kCostTri * A for
// any i).  dec bytes: [0] = 0 for a leaf, else (slots << 2) | k of the best
// wide node; [i-1] (i = 2..4) = k of split[i], or 0xff when cost[i-1] wins.
__device__ __forceinline__ void child_costs(int c, int64_t n, const float4* box_lo, const float4* box_hi,
                                            const float4* cost, float out[5]) {
  if (c >= n) {
    const float a = kCostTri * half_area(__ldcg(&box_lo[c]), __ldcg(&box_hi[c]));
    out[1] = out[2] = out[3] = out[4] = a;
  } else {
    const float4 v = __ldcg(&cost[c]);
    out[1] = v.x; out[2] = v.y; out[3] = v.z; out[4] = v.w;
  }
}

__global__ void refit_kernel(const uint32_t* __restrict__ order, const float4* __restrict__ tri_lo,
                             const float4* __restrict__ tri_hi, int64_t n, const int32_t* __restrict__ left,
                             const int32_t* __restrict__ right, const int32_t* __restrict__ parent,
                             const int32_t* __restrict__ first, const int32_t* __restrict__ last, int leaf_max,
                             float4* box_lo, float4* box_hi, float4* cost, uint32_t* dec, uint32_t* visit) {
  pdl_wait();
  const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const int64_t leaf = n + j;
  const uint32_t f = order[j];
  box_lo[leaf] = tri_lo[f];
  box_hi[leaf] = tri_hi[f];
  __threadfence();
  int p = parent[leaf];
  while (p >= 0) {
    if (atomicAdd(&visit[p], 1u) == 0u) return;  // sibling not done yet
    __threadfence();
    const int l = left[p], r = right[p];
    const float4 al = __ldcg(&box_lo[l]), ah = __ldcg(&box_hi[l]);
    const float4 bl = __ldcg(&box_lo[r]), bh = __ldcg(&box_hi[r]);
    const float4 lo = make_float4(fminf(al.x, bl.x), fminf(al.y, bl.y), fminf(al.z, bl.z), 0.f);
    const float4 hi = make_float4(fmaxf(ah.x, bh.x), fmaxf(ah.y, bh.y), fmaxf(ah.z, bh.z), 0.f);
    __stcg(&box_lo[p], lo);
    __stcg(&box_hi[p], hi);
    // collapse costs
    float cl[5], cr[5];
    child_costs(l, n, box_lo, box_hi, cost, cl);
    child_costs(r, n, box_lo, box_hi, cost, cr);
    float split[5] = {INFINITY, INFINITY, INFINITY, INFINITY, INFINITY};
    int sk[5] = {0, 0, 0, 0, 0};
    for (int i = 2; i <= 4; ++i)
      for (int k = 1; k < i; ++k) {
        const float c = cl[k] + cr[i - k];
        if (c < split[i]) { split[i] = c; sk[i] = k; }
      }
    const float area = half_area(lo, hi);
    int wi = 2;
    for (int i = 3; i <= 4; ++i)
      if (split[i] < split[wi]) wi = i;
    const float wide = kCostNode * area + split[wi];
    const int count = last[p] - first[p] + 1;
    const float leafc = (count <= leaf_max && parent[p] >= 0) ? kCostTri * area * (float)count : INFINITY;
    float c[5];
    uint32_t d = 0;
    if (leafc <= wide) {
      c[1] = leafc;
    } else {
      c[1] = wide;
      d = (uint32_t)((wi << 2) | sk[wi]);
    }
    for (int i = 2; i <= 4; ++i) {
      if (c[i - 1] <= split[i]) {
        c[i] = c[i - 1];
        d |= 0xffu << (8 * (i - 1));
      } else {
        c[i] = split[i];
        d |= (uint32_t)sk[i] << (8 * (i - 1));
      }
    }
    __stcg(&cost[p], make_float4(c[1], c[2], c[3], c[4]));
    __stcg(&dec[p], d);
    __threadfence();
    p = parent[p];
  }
}

__device__ __forceinline__ uint32_t scale_exponent(float ext) {
  // smallest power of two s with 255*s >= ext; returned as biased exponent
  int e = 0;
  float m = frexpf(fmaxf(ext, 1e-30f) * (1.0f / 255.0f), &e);  // value = m * 2^e, m in [0.5,1)
  (void)m;
  uint32_t be = (uint32_t)(e + 127);
  be = be < 1u ? 1u : (be > 254u ? 254u : be);
  while (be < 254u && 255.0f * __uint_as_float(be << 23) < ext) ++be;
  return be;
}

__device__ __forceinline__ void quantize_axis(float o, float s, float lo, float hi, uint32_t& qlo, uint32_t& qhi) {
  int ql = (int)floorf((lo - o) / s);
  int qh = (int)ceilf((hi - o) / s);
  ql = max(0, min(255, ql));
  qh = max(0, min(255, qh));
  while (ql > 0 && fmaf((float)ql, s, o) > lo) --ql;
  while (qh < 255 && fmaf((float)qh, s, o) < hi) ++qh;
  qlo = (uint32_t)ql;
  qhi = (uint32_t)qh;
}

// 6. one collapse level: each worklist entry becomes a wide node at the slot
// of its binary node; its internal children (binary node indices, which are
// also their slots) form the next level's worklist
__global__ void __launch_bounds__(kThreads)
    collapse_level_kernel(int level, uint32_t* __restrict__ counters, const int32_t* __restrict__ cur,
                          int32_t* __restrict__ nxt, int64_t n, int leaf_max, const int32_t* __restrict__ left,
                          const int32_t* __restrict__ right, const int32_t* __restrict__ first,
                          const int32_t* __restrict__ last, const float4* __restrict__ box_lo,
                          const float4* __restrict__ box_hi, const uint32_t* __restrict__ dec,
                          WideNode* __restrict__ tmp, uint32_t* __restrict__ lvl) {
  pdl_wait();
  const uint32_t cnt = counters[level];
  const int nn = (int)n;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < cnt; k += (int64_t)gridDim.x * blockDim.x) {
    const int b = cur[k];
    int c[4];
    int nc;
    if (b >= nn) {  // a lone leaf as root (single-triangle mesh)
      c[0] = b;
      nc = 1;
    } else {
      // the subtrees the SAH-optimal collapse chose for this node's slots,
      // expanded left to right (a pending (node, slots) pair per entry)
      const uint32_t d0 = dec[b];
      int pn[4], ps[4], np = 0;
      const int slots = (int)((d0 & 0xffu) >> 2), k0 = (int)(d0 & 3u);
      if (slots >= 2 && k0 >= 1 && k0 < slots) {
        pn[0] = right[b]; ps[0] = slots - k0;  // stack: right pushed first
        pn[1] = left[b]; ps[1] = k0;
        np = 2;
      } else {  // a root the cost model would have made a leaf: two slots
        pn[0] = right[b]; ps[0] = 1;
        pn[1] = left[b]; ps[1] = 1;
        np = 2;
      }
      nc = 0;
      while (np > 0 && nc < 4) {
        --np;
        const int x = pn[np];
        int i = ps[np];
        if (x < nn) {
          const uint32_t dx = dec[x];
          while (i > 1 && ((dx >> (8 * (i - 1))) & 0xffu) == 0xffu) --i;
        }
        if (i <= 1 || x >= nn) {
          c[nc++] = x;
        } else {
          const int k = (int)((dec[x] >> (8 * (i - 1))) & 0xffu);
          pn[np] = right[x]; ps[np] = i - k; ++np;
          pn[np] = left[x]; ps[np] = k; ++np;
        }
      }
    }
    const float4 plo = box_lo[b], phi = box_hi[b];
    WideNode nd;
    nd.ox = plo.x; nd.oy = plo.y; nd.oz = plo.z;
    const uint32_t ex = scale_exponent(phi.x - plo.x);
    const uint32_t ey = scale_exponent(phi.y - plo.y);
    const uint32_t ez = scale_exponent(phi.z - plo.z);
    const float sx = __uint_as_float(ex << 23), sy = __uint_as_float(ey << 23), sz = __uint_as_float(ez << 23);
    nd.meta = ex | (ey << 8) | (ez << 16) | ((uint32_t)nc << 24);
    for (int a = 0; a < 6; ++a) nd.q[a] = 0;
    const int slot = b < nn ? b : b - nn;
    nd.pad[0] = (uint32_t)slot;
    nd.pad[1] = 0;
    for (int j = 0; j < 4; ++j) {
      if (j >= nc) {
        // empty slot: inverted box (lo = 255, hi = 0) never passes a test
        nd.q[0] |= 255u << (8 * j); nd.q[1] |= 255u << (8 * j); nd.q[2] |= 255u << (8 * j);
        nd.ref[j] = 0xffffffffu;
        continue;
      }
      const int cj = c[j];
      const float4 lo = box_lo[cj], hi = box_hi[cj];
      uint32_t a0, a1;
      quantize_axis(nd.ox, sx, lo.x, hi.x, a0, a1); nd.q[0] |= a0 << (8 * j); nd.q[3] |= a1 << (8 * j);
      quantize_axis(nd.oy, sy, lo.y, hi.y, a0, a1); nd.q[1] |= a0 << (8 * j); nd.q[4] |= a1 << (8 * j);
      quantize_axis(nd.oz, sz, lo.z, hi.z, a0, a1); nd.q[2] |= a0 << (8 * j); nd.q[5] |= a1 << (8 * j);
      const int count = cj >= nn ? 1 : last[cj] - first[cj] + 1;
      if (cj >= nn || (dec[cj] & 0xffu) == 0u) {
        const uint32_t f0 = cj >= nn ? (uint32_t)(cj - nn) : (uint32_t)first[cj];
        nd.ref[j] = make_leaf_ref(f0, (uint32_t)count);
      } else {
        nd.ref[j] = (uint32_t)cj;  // slot; renumbered by the layout pass
        const uint32_t at = atomicAdd(&counters[level + 1], 1u);
        if (level + 1 < kMaxLevels) nxt[at] = cj;
      }
    }
    tmp[slot] = nd;
    lvl[slot] = (uint32_t)level;
  }
}

__global__ void depth_check_kernel(const uint32_t* counters, int32_t* err) {
  pdl_wait();
  if (threadIdx.x == 0 && counters[kMaxLevels] != 0u) err[1] = 1;
}

// 7a. final index of each wide node
__global__ void layout_index_kernel(const uint32_t* __restrict__ sorted_lvl, const uint32_t* __restrict__ sorted_slot,
                                    int64_t n, uint32_t* __restrict__ newidx) {
  pdl_wait();
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  if ((sorted_lvl[r] & 0xffu) != kNoLevel) newidx[sorted_slot[r]] = (uint32_t)r;
}

// 7b. copy in the final order with child references renumbered
__global__ void layout_copy_kernel(const uint32_t* __restrict__ sorted_lvl, const uint32_t* __restrict__ sorted_slot,
                                   int64_t n, const uint32_t* __restrict__ newidx, const WideNode* __restrict__ tmp,
                                   WideNode* __restrict__ out) {
  pdl_wait();
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  if ((sorted_lvl[r] & 0xffu) == kNoLevel) return;
  WideNode nd = tmp[sorted_slot[r]];
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const uint32_t ref = nd.ref[j];
    if (ref != 0xffffffffu && !ref_is_leaf(ref)) nd.ref[j] = newidx[ref];
  }
  out[r] = nd;
}

// 7c. mesh roots, mesh bounds, node count
__global__ void finish_kernel(const int64_t* __restrict__ face_off, int nmesh, const uint32_t* __restrict__ counters,
                              const uint32_t* __restrict__ newidx, const uint32_t* __restrict__ bounds,
                              uint32_t* __restrict__ roots, float* __restrict__ bounds_out,
                              int64_t* __restrict__ num_nodes) {
  pdl_wait();
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t == 0 && num_nodes) {
    int64_t total = 0;
    for (int l = 0; l < kMaxLevels; ++l) total += counters[l];
    *num_nodes = total;
  }
  if (t >= nmesh) return;
  if (roots) roots[t] = newidx[face_off[t]];
  if (bounds_out) {
    for (int k = 0; k < 6; ++k) bounds_out[6 * t + k] = float_unflip(bounds[12 * t + k]);
  }
}

// 8. triangle records in leaf (sorted) order; the face id stored is the
// mesh-local one
__global__ void write_tris_kernel(const float* __restrict__ V, const int64_t* __restrict__ vert_off,
                                  const int32_t* __restrict__ F, const int64_t* __restrict__ face_off,
                                  const uint32_t* __restrict__ mesh_of, const uint32_t* __restrict__ order, int64_t n,
                                  TriRec* __restrict__ tris) {
  pdl_wait();
  const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const uint32_t f = order[j];
  const uint32_t m = mesh_of[f];
  const int64_t vb = vert_off[m], nv = vert_off[m + 1] - vb;
  int32_t i0 = F[3 * (int64_t)f], i1 = F[3 * (int64_t)f + 1], i2 = F[3 * (int64_t)f + 2];
  if (i0 < 0 || i1 < 0 || i2 < 0 || i0 >= nv || i1 >= nv || i2 >= nv) i0 = i1 = i2 = 0;  // reported by tri_prep
  const float3 a = ld3(V, vb + i0), b = ld3(V, vb + i1), c = ld3(V, vb + i2);
  // near-degenerate test in FP64: |n|^2 tiny in absolute terms (the
  // reference's 1e-12 cut) or relative to the longest edge (slivers)
  const double e0x = (double)b.x - a.x, e0y = (double)b.y - a.y, e0z = (double)b.z - a.z;
  const double e1x = (double)c.x - a.x, e1y = (double)c.y - a.y, e1z = (double)c.z - a.z;
  const double e2x = (double)c.x - b.x, e2y = (double)c.y - b.y, e2z = (double)c.z - b.z;
  const double nx = e0y * e1z - e0z * e1y, ny = e0z * e1x - e0x * e1z, nz = e0x * e1y - e0y * e1x;
  const double nsq = nx * nx + ny * ny + nz * nz;
  const double l0 = e0x * e0x + e0y * e0y + e0z * e0z, l1 = e1x * e1x + e1y * e1y + e1z * e1z,
               l2 = e2x * e2x + e2y * e2y + e2z * e2z;
  const double lm = fmax(l0, fmax(l1, l2));
  uint32_t flags = 0;
  if (nsq < 1e-12 || nsq < 1e-6 * lm * lm) flags |= kTriFlagNearDegenerate;
  // reciprocals of the quantities the FP32 test divides by, evaluated with
  // the test's own FP32 expressions
  const float v21x = b.x - a.x, v21y = b.y - a.y, v21z = b.z - a.z;
  const float v32x = c.x - b.x, v32y = c.y - b.y, v32z = c.z - b.z;
  const float v13x = a.x - c.x, v13y = a.y - c.y, v13z = a.z - c.z;
  const float nrx = v21y * v13z - v21z * v13y, nry = v21z * v13x - v21x * v13z, nrz = v21x * v13y - v21y * v13x;
  const float nsqf = nrx * nrx + nry * nry + nrz * nrz;
  const float e0 = v21x * v21x + v21y * v21y + v21z * v21z;
  const float e1 = v32x * v32x + v32y * v32y + v32z * v32z;
  const float e2 = v13x * v13x + v13y * v13y + v13z * v13z;
  const int local = (int)((int64_t)f - face_off[m]);
  // dual-basis coefficients of the barycentric projection (e0 = b - a,
  // e1 = c - a): u = A (v.e0) - B (v.e1), w = C (v.e1) - B (v.e0) with
  // A = d11 / |n|^2, B = d01 / |n|^2, C = d00 / |n|^2 (|n|^2 = d00 d11 - d01^2),
  // from the FP32 edge vectors the test forms, divided in FP64
  const float f0x = b.x - a.x, f0y = b.y - a.y, f0z = b.z - a.z;
  const float f1x = c.x - a.x, f1y = c.y - a.y, f1z = c.z - a.z;
  const double d00 = (double)f0x * f0x + (double)f0y * f0y + (double)f0z * f0z;
  const double d01 = (double)f0x * f1x + (double)f0y * f1y + (double)f0z * f1z;
  const double d11 = (double)f1x * f1x + (double)f1y * f1y + (double)f1z * f1z;
  const double den = (double)nsqf > 0.0 ? (double)nsqf : 1.0;
  const bool near_degenerate = (flags & kTriFlagNearDegenerate) != 0;
  TriRec r;
  r.a = make_float4(a.x, a.y, a.z, __int_as_float(local));
  r.b = make_float4(b.x, b.y, b.z, (float)(d01 / den));
  // a negative c.w marks a near-degenerate triangle (evaluated in FP64)
  r.c = make_float4(c.x, c.y, c.z, near_degenerate ? -1.0f : (float)(d11 / den));
  r.r = make_float4(1.0f / fmaxf(e0, 1e-12f), 1.0f / fmaxf(e1, 1e-12f), 1.0f / fmaxf(e2, 1e-12f),
                    (float)(d00 / den));
  tris[j] = r;
}

// resident blocks of the SAH kernel on the current device (its shared
// memory needs the opt-in above 48 KB), set up once per device and block size
template <int kThreads>
int sah_grid_size(int* grid) {
  static int cached[kMaxDevices] = {0};
  int dev = 0;
  A3D_CUDA_TRY(cudaGetDevice(&dev));
  if (dev >= 0 && dev < kMaxDevices && cached[dev] > 0) {
    *grid = cached[dev];
    return A3D_OK;
  }
  A3D_CUDA_TRY(cudaFuncSetAttribute(sah_cluster_kernel<kThreads>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)sizeof(SahSmem<kThreads>)));
  int sms = 0, per_sm = 0;
  A3D_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  A3D_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, sah_cluster_kernel<kThreads>, kThreads,
                                                             sizeof(SahSmem<kThreads>)));
  const int g = (sms > 0 ? sms : 1) * (per_sm > 0 ? per_sm : 1);
  if (dev >= 0 && dev < kMaxDevices) cached[dev] = g;
  *grid = g;
  return A3D_OK;
}

template <int kThreads>
int launch_sah(int64_t n, BuildWs& w, const uint32_t* order, cudaStream_t s) {
  int sah_grid = 0;
  A3D_TRY(sah_grid_size<kThreads>(&sah_grid));
  const int64_t max_clusters = n / 3 + 1;
  A3D_PDL(sah_cluster_kernel<kThreads>, dim3((unsigned)(max_clusters < sah_grid ? max_clusters : sah_grid)),
          dim3(kThreads), sizeof(SahSmem<kThreads>), s, w.clusters, w.ncl,
          SahTree{w.left, w.right, w.parent, w.first, w.last, n}, const_cast<uint32_t*>(order), w.sah_tmp,
          w.sah_small, SahPrims{w.centroid, w.tri_lo, w.tri_hi});
  return A3D_OK;
}

int mesh_bits_of(int nmesh) {
  int mbits = 0;
  while ((1ll << mbits) < nmesh) ++mbits;
  return mbits;
}

// The whole build, launches only.  Offsets are device arrays [nmesh + 1].
int build_wide_bvh(const float* V, const int64_t* vert_off, const int32_t* F, const int64_t* face_off, int nmesh,
                   int64_t n, int leaf_max, WideNode* nodes_out, TriRec* tris_out, uint32_t* roots_out,
                   float* bounds_out, int64_t* num_nodes_out, int32_t* status_out, BuildWs& w, cudaStream_t s) {
  const int mbits = mesh_bits_of(nmesh);
  const int bits = (64 - mbits) / 3 < 21 ? (64 - mbits) / 3 : 21;
  const int64_t init_threads = 12ll * nmesh > kMaxLevels + 1 ? 12ll * nmesh : kMaxLevels + 1;
  A3D_PDL(init_kernel, dim3((unsigned)ceil_div(init_threads, kThreads)), dim3(kThreads), 0, s, face_off, nmesh, n,
          w.bounds, w.err, w.counters, w.work_a);
  const unsigned g = (unsigned)ceil_div(n, kThreads);
  A3D_PDL(tri_prep_kernel, dim3(g), dim3(kThreads), 0, s, V, vert_off, F, face_off, nmesh, n, w.tri_lo, w.tri_hi,
          w.centroid, w.mesh_of, w.bounds, w.err);
  A3D_PDL(morton_kernel, dim3(g), dim3(kThreads), 0, s, w.centroid, w.mesh_of, n, w.bounds, bits, w.keys, w.vals);
  bool alt = false;
  A3D_TRY(radix_sort_pairs<uint64_t>(w.keys, w.vals, w.keys_alt, w.vals_alt, n, 0, 3 * bits + mbits, w.rs_scratch,
                                     &alt, s));
  const uint64_t* keys = alt ? w.keys_alt : w.keys;
  const uint32_t* order = alt ? w.vals_alt : w.vals;

  A3D_PDL(radix_tree_kernel, dim3(g), dim3(kThreads), 0, s, keys, face_off, nmesh, n, w.left, w.right, w.parent,
          w.first, w.last);
  // SAH refinement of every subtree of <= sah_max triangles below the top:
  // kSahMax from 64 x kSahMax triangles up, below it n / 64 rounded down to
  // a power of two (at least 2,048), so that a small mesh still has about
  // 64 clusters for the SMs
  int sah_max = kSahMax;
  while (sah_max > 2048 && (int64_t)sah_max * 64 > n) sah_max >>= 1;
  A3D_CUDA_TRY(cudaMemsetAsync(w.ncl, 0, sizeof(uint32_t), s));
  A3D_PDL(sah_find_kernel, dim3(g), dim3(kThreads), 0, s, face_off, nmesh, n, w.parent, w.first, w.last, sah_max,
          w.clusters, w.ncl);
  A3D_TRY(n <= (int64_t)kSahMax * num_sms()
              ? launch_sah<kSahThreadsWide>(n, w, order, s)
              : launch_sah<kSahThreadsNarrow>(n, w, order, s));
  A3D_CUDA_TRY(cudaMemsetAsync(w.visit, 0, sizeof(uint32_t) * n, s));
  A3D_PDL(refit_kernel, dim3(g), dim3(kThreads), 0, s, order, w.tri_lo, w.tri_hi, n, w.left, w.right, w.parent, w.first,
          w.last, leaf_max, w.box_lo, w.box_hi, w.dp_cost, w.dp_dec, w.visit);
  A3D_PDL(write_tris_kernel, dim3(g), dim3(kThreads), 0, s, V, vert_off, F, face_off, w.mesh_of, order, n, tris_out);

  // collapse: a fixed number of level launches (empty levels return at once)
  A3D_CUDA_TRY(cudaMemsetAsync(w.lvl, 0xff, sizeof(uint32_t) * n, s));
  const int64_t level_blocks = (int64_t)num_sms() * 8;
  const int64_t lb = ceil_div(n, kThreads) < level_blocks ? ceil_div(n, kThreads) : level_blocks;
  int32_t *cur = w.work_a, *nxt = w.work_b;
  for (int level = 0; level < kMaxLevels; ++level) {
    A3D_PDL(collapse_level_kernel, dim3((unsigned)lb), dim3(kThreads), 0, s, level, w.counters, cur, nxt, n, leaf_max,
            w.left, w.right, w.first, w.last, w.box_lo, w.box_hi, w.dp_dec, w.tmp_nodes, w.lvl);
    int32_t* t = cur;
    cur = nxt;
    nxt = t;
  }
  A3D_PDL(depth_check_kernel, dim3(1), dim3(32), 0, s, w.counters, w.err);
  // breadth-first layout: stable sort of the slots by level
  A3D_PDL(iota_u32_kernel, dim3(g), dim3(kThreads), 0, s, w.slot, n);
  bool lalt = false;
  A3D_TRY(radix_sort_pairs<uint32_t>(w.lvl, w.slot, w.lvl_alt, w.slot_alt, n, 0, 8, w.rs_scratch, &lalt, s));
  const uint32_t* slvl = lalt ? w.lvl_alt : w.lvl;
  const uint32_t* sslot = lalt ? w.slot_alt : w.slot;
  A3D_PDL(layout_index_kernel, dim3(g), dim3(kThreads), 0, s, slvl, sslot, n, w.newidx);
  A3D_PDL(layout_copy_kernel, dim3(g), dim3(kThreads), 0, s, slvl, sslot, n, w.newidx, w.tmp_nodes, nodes_out);
  A3D_PDL(finish_kernel, dim3((unsigned)ceil_div(nmesh, kThreads)), dim3(kThreads), 0, s, face_off, nmesh, w.counters,
          w.newidx, w.bounds, roots_out, bounds_out, num_nodes_out);
  if (status_out) A3D_CUDA_TRY(cudaMemcpyAsync(status_out, w.err, 2 * sizeof(int32_t), cudaMemcpyDeviceToDevice, s));
  return A3D_OK;
}

}  // namespace

}  // namespace a3d

using namespace a3d;

extern "C" size_t a3d_bvh_build_workspace_bytes(int64_t num_faces) {
  Workspace ws(nullptr, 0);
  BuildWs w;
  return carve(w, ws, num_faces > 0 ? num_faces : 1, 1) + 256;
}

extern "C" int a3d_bvh_build(const float* vertices, int64_t num_vertices, const int32_t* faces, int64_t num_faces,
                             int leaf_max, void* nodes_out, int64_t node_capacity, void* tris_out, void* workspace,
                             size_t workspace_bytes, int64_t* num_nodes_out, float* bounds_out,
                             a3d_stream_t stream_) {
  cudaStream_t s = (cudaStream_t)stream_;
  A3D_REQUIRE(num_faces > 0 && num_vertices > 0, A3D_ERR_ARGUMENT, "bvh_build: empty mesh");
  A3D_REQUIRE(num_faces < (1ll << 28), A3D_ERR_ARGUMENT, "bvh_build: more than 2^28 faces");
  A3D_REQUIRE(vertices && faces && nodes_out && tris_out && num_nodes_out, A3D_ERR_ARGUMENT,
              "bvh_build: null pointer");
  A3D_REQUIRE(((uintptr_t)nodes_out & 63) == 0 && ((uintptr_t)tris_out & 15) == 0, A3D_ERR_ARGUMENT,
              "bvh_build: nodes must be 64-B and triangles 16-B aligned");
  const int64_t n = num_faces;
  A3D_REQUIRE(node_capacity >= n, A3D_ERR_WORKSPACE, "bvh_build: node capacity must be at least num_faces");
  Workspace ws(workspace, workspace_bytes);
  BuildWs w;
  carve(w, ws, n, 1);
  A3D_REQUIRE(workspace && ws.ok(), A3D_ERR_WORKSPACE, "bvh_build: workspace too small");
  if (leaf_max == 0) leaf_max = kDefaultLeafMax;
  A3D_REQUIRE(leaf_max >= 1 && leaf_max <= kMaxLeafTris, A3D_ERR_ARGUMENT, "bvh_build: leaf_max must be in 1..8");
  A3D_PDL(single_offsets_kernel, dim3(1), dim3(32), 0, s, w.face_off, w.vert_off, n, num_vertices);
  A3D_TRY(build_wide_bvh(vertices, w.vert_off, faces, w.face_off, 1, n, leaf_max, (WideNode*)nodes_out,
                         (TriRec*)tris_out, nullptr, nullptr, w.count, nullptr, w, s));
  uint32_t hb[12];
  int32_t herr[4];
  int64_t count = 0;
  A3D_CUDA_TRY(cudaMemcpyAsync(hb, w.bounds, sizeof(hb), cudaMemcpyDeviceToHost, s));
  A3D_CUDA_TRY(cudaMemcpyAsync(herr, w.err, sizeof(herr), cudaMemcpyDeviceToHost, s));
  A3D_CUDA_TRY(cudaMemcpyAsync(&count, w.count, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
  A3D_CUDA_TRY(cudaStreamSynchronize(s));
  A3D_REQUIRE(herr[0] == 0, A3D_ERR_ARGUMENT, "bvh_build: face index out of range");
  A3D_REQUIRE(herr[1] == 0, A3D_ERR_OVERFLOW, "bvh_build: tree deeper than the collapse's level limit");
  if (bounds_out) {
    for (int k = 0; k < 6; ++k) {
      const uint32_t u = hb[k];
      const uint32_t f = (u & 0x80000000u) ? (u & 0x7fffffffu) : ~u;
      memcpy(&bounds_out[k], &f, 4);
    }
  }
  *num_nodes_out = count;
  return A3D_OK;
}

extern "C" size_t a3d_batch_build_workspace_bytes(int64_t num_faces, int32_t num_meshes) {
  Workspace ws(nullptr, 0);
  BuildWs w;
  return carve(w, ws, num_faces > 0 ? num_faces : 1, num_meshes > 0 ? num_meshes : 1) + 256;
}

extern "C" int a3d_batch_build(const float* vertices, const int64_t* vertex_offsets, const int32_t* faces,
                               const int64_t* face_offsets, int32_t num_meshes, int64_t num_faces, int leaf_max,
                               void* nodes_out, void* tris_out, uint32_t* roots_out, float* bounds_out,
                               int64_t* num_nodes_out, int32_t* status_out, void* workspace, size_t workspace_bytes,
                               a3d_stream_t stream_) {
  cudaStream_t s = (cudaStream_t)stream_;
  A3D_REQUIRE(num_meshes > 0 && num_faces >= num_meshes, A3D_ERR_ARGUMENT,
              "batch_build: needs at least one face per mesh");
  A3D_REQUIRE(num_faces < (1ll << 28), A3D_ERR_ARGUMENT, "batch_build: more than 2^28 faces in the batch");
  A3D_REQUIRE(vertices && vertex_offsets && faces && face_offsets && nodes_out && tris_out && roots_out,
              A3D_ERR_ARGUMENT, "batch_build: null pointer");
  A3D_REQUIRE(((uintptr_t)nodes_out & 63) == 0 && ((uintptr_t)tris_out & 15) == 0, A3D_ERR_ARGUMENT,
              "batch_build: nodes must be 64-B and triangles 16-B aligned");
  if (leaf_max == 0) leaf_max = kDefaultLeafMax;
  A3D_REQUIRE(leaf_max >= 1 && leaf_max <= kMaxLeafTris, A3D_ERR_ARGUMENT, "batch_build: leaf_max must be in 1..8");
  Workspace ws(workspace, workspace_bytes);
  BuildWs w;
  carve(w, ws, num_faces, num_meshes);
  A3D_REQUIRE(workspace && ws.ok(), A3D_ERR_WORKSPACE, "batch_build: workspace too small");
  return build_wide_bvh(vertices, vertex_offsets, faces, face_offsets, num_meshes, num_faces, leaf_max,
                        (WideNode*)nodes_out, (TriRec*)tris_out, roots_out, bounds_out, num_nodes_out, status_out, w,
                        s);
}
