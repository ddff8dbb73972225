// GPU construction of the wide BVH.
//
// Replaces the reference's single-threaded host SAH builder
// (atom3d/kernels/bvh_kernels.cu:616-925).  Pipeline, all on the stream:
//   1. per-triangle AABB/centroid + scene and centroid bounds (block reduce,
//      one atomic per block)
//   2. 63-bit Morton code of each centroid
//   3. stable radix sort of (code, face id) with the in-house sort
//   4. binary radix tree over the sorted codes (one thread per internal node,
//      duplicate codes disambiguated by index)
//   5. bottom-up refit (second arriving child computes the union box)
//   6. surface-area-guided collapse into 4-wide quantised nodes: starting
//      from a binary node, the child with the largest surface area is opened
//      until four slots are used; subtrees of <= leaf_max triangles become
//      leaves.  Level-synchronous, node indices assigned by prefix sum so the
//      layout is deterministic.
#include <math.h>

#include "bvh_layout.cuh"
#include "primitives.cuh"

namespace a3d {

namespace {

constexpr int kThreads = 256;

struct BuildWs {
  float4* tri_lo;
  float4* tri_hi;
  float4* centroid;
  uint32_t* bounds;  // 12 flipped floats: scene lo, scene hi, cent lo, cent hi
  int32_t* err;
  uint64_t* keys;
  uint64_t* keys_alt;
  uint32_t* vals;
  uint32_t* vals_alt;
  uint32_t* rs_scratch;
  int32_t* left;
  int32_t* right;
  int32_t* parent;
  int32_t* first;
  int32_t* last;
  float4* box_lo;  // [2n-1]: internal 0..n-2, leaf j at n-1+j
  float4* box_hi;
  uint32_t* visit;
  int32_t* work_a_bin;
  int32_t* work_a_node;
  int32_t* work_b_bin;
  int32_t* work_b_node;
  int32_t* child_bin;  // [n*4]
  uint8_t* child_leaf; // [n*4]
  int32_t* nchild;
  uint32_t* nwide;
  uint32_t* nwide_off;
  uint32_t* scan_tmp;
  uint32_t* total;
};

size_t carve(BuildWs& w, Workspace& ws, int64_t n) {
  const int64_t nn = n > 1 ? 2 * n - 1 : 1;
  w.tri_lo = ws.take<float4>(n);
  w.tri_hi = ws.take<float4>(n);
  w.centroid = ws.take<float4>(n);
  w.bounds = ws.take<uint32_t>(12);
  w.err = ws.take<int32_t>(4);
  w.keys = ws.take<uint64_t>(n);
  w.keys_alt = ws.take<uint64_t>(n);
  w.vals = ws.take<uint32_t>(n);
  w.vals_alt = ws.take<uint32_t>(n);
  w.rs_scratch = ws.take<uint32_t>((int64_t)radix_sort_scratch_elems(n));
  w.left = ws.take<int32_t>(n);
  w.right = ws.take<int32_t>(n);
  w.parent = ws.take<int32_t>(nn);
  w.first = ws.take<int32_t>(n);
  w.last = ws.take<int32_t>(n);
  w.box_lo = ws.take<float4>(nn);
  w.box_hi = ws.take<float4>(nn);
  w.visit = ws.take<uint32_t>(n);
  w.work_a_bin = ws.take<int32_t>(n);
  w.work_a_node = ws.take<int32_t>(n);
  w.work_b_bin = ws.take<int32_t>(n);
  w.work_b_node = ws.take<int32_t>(n);
  w.child_bin = ws.take<int32_t>(4 * n);
  w.child_leaf = ws.take<uint8_t>(4 * n);
  w.nchild = ws.take<int32_t>(n);
  w.nwide = ws.take<uint32_t>(n);
  w.nwide_off = ws.take<uint32_t>(n);
  w.scan_tmp = ws.take<uint32_t>((int64_t)scan_workspace_elems(n));
  w.total = ws.take<uint32_t>(2);
  return ws.used;
}

__device__ __forceinline__ float3 ld3(const float* p, int64_t i) {
  return make_float3(p[3 * i], p[3 * i + 1], p[3 * i + 2]);
}

__global__ void init_bounds_kernel(uint32_t* bounds, int32_t* err) {
  int t = threadIdx.x;
  if (t < 12) bounds[t] = ((t / 3) % 2 == 0) ? 0xffffffffu : 0u;  // lo slots: min, hi slots: max
  if (t < 4) err[t] = 0;
}

// 1. triangle boxes, centroids, bounds, triangle records (original order)
__global__ void __launch_bounds__(kThreads)
    tri_prep_kernel(const float* __restrict__ V, int64_t nv, const int32_t* __restrict__ F, int64_t nf,
                    float4* __restrict__ tri_lo, float4* __restrict__ tri_hi, float4* __restrict__ cen,
                    uint32_t* __restrict__ bounds, int32_t* __restrict__ err) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  float v[12];
#pragma unroll
  for (int k = 0; k < 6; ++k) { v[k] = INFINITY; v[k + 6] = -INFINITY; }
  if (i < nf) {
    int32_t i0 = F[3 * i], i1 = F[3 * i + 1], i2 = F[3 * i + 2];
    if (i0 < 0 || i1 < 0 || i2 < 0 || i0 >= nv || i1 >= nv || i2 >= nv) {
      atomicExch(err, 1);
      i0 = i1 = i2 = 0;
    }
    float3 a = ld3(V, i0), b = ld3(V, i1), c = ld3(V, i2);
    float3 lo = make_float3(fminf(fminf(a.x, b.x), c.x), fminf(fminf(a.y, b.y), c.y), fminf(fminf(a.z, b.z), c.z));
    float3 hi = make_float3(fmaxf(fmaxf(a.x, b.x), c.x), fmaxf(fmaxf(a.y, b.y), c.y), fmaxf(fmaxf(a.z, b.z), c.z));
    float3 ce = make_float3((a.x + b.x + c.x) * (1.0f / 3.0f), (a.y + b.y + c.y) * (1.0f / 3.0f),
                            (a.z + b.z + c.z) * (1.0f / 3.0f));
    tri_lo[i] = make_float4(lo.x, lo.y, lo.z, 0.f);
    tri_hi[i] = make_float4(hi.x, hi.y, hi.z, 0.f);
    cen[i] = make_float4(ce.x, ce.y, ce.z, 0.f);
    v[0] = lo.x; v[1] = lo.y; v[2] = lo.z;
    v[3] = ce.x; v[4] = ce.y; v[5] = ce.z;
    v[6] = hi.x; v[7] = hi.y; v[8] = hi.z;
    v[9] = ce.x; v[10] = ce.y; v[11] = ce.z;
  }
  // block reduce: min of v[0..5], max of v[6..11]
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
  if (threadIdx.x < 12) {
    const int k = threadIdx.x;
    float r = s[0][k];
    for (int w = 1; w < kThreads / 32; ++w) r = k < 6 ? fminf(r, s[w][k]) : fmaxf(r, s[w][k]);
    // bounds layout: [0..2] scene lo, [3..5] scene hi, [6..8] cent lo, [9..11] cent hi
    const int slot = k < 3 ? k : (k < 6 ? 6 + (k - 3) : (k < 9 ? 3 + (k - 6) : 9 + (k - 9)));
    if (isfinite(r)) {
      if (k < 6) atomicMin(&bounds[slot], float_flip(r));
      else atomicMax(&bounds[slot], float_flip(r));
    }
  }
}

// 2. Morton codes of centroids
__global__ void morton_kernel(const float4* __restrict__ cen, int64_t n, const uint32_t* __restrict__ bounds,
                              uint64_t* __restrict__ keys, uint32_t* __restrict__ vals) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float lo[3] = {float_unflip(bounds[6]), float_unflip(bounds[7]), float_unflip(bounds[8])};
  const float hi[3] = {float_unflip(bounds[9]), float_unflip(bounds[10]), float_unflip(bounds[11])};
  const float4 c = cen[i];
  const float cc[3] = {c.x, c.y, c.z};
  uint64_t code = 0;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const float ext = hi[a] - lo[a];
    float t = ext > 0.f ? (cc[a] - lo[a]) / ext : 0.f;
    t = fminf(fmaxf(t, 0.f), 1.f);
    const uint64_t q = (uint64_t)(t * 2097151.0f);
    code |= spread3_21(q) << a;
  }
  keys[i] = code;
  vals[i] = (uint32_t)i;
}

// 4. binary radix tree
__device__ __forceinline__ int delta(const uint64_t* keys, int64_t n, int i, int j) {
  if (j < 0 || j >= n) return -1;
  const uint64_t a = keys[i], b = keys[j];
  if (a != b) return __clzll((long long)(a ^ b));
  return 64 + __clz(i ^ j);
}

__global__ void radix_tree_kernel(const uint64_t* __restrict__ keys, int64_t n, int32_t* __restrict__ left,
                                  int32_t* __restrict__ right, int32_t* __restrict__ parent,
                                  int32_t* __restrict__ first, int32_t* __restrict__ last) {
  const int i = (int)((int64_t)blockIdx.x * blockDim.x + threadIdx.x);
  if (i >= n - 1) return;
  const int d = (delta(keys, n, i, i + 1) - delta(keys, n, i, i - 1)) >= 0 ? 1 : -1;
  const int dmin = delta(keys, n, i, i - d);
  int lmax = 2;
  while (delta(keys, n, i, i + lmax * d) > dmin) lmax <<= 1;
  int l = 0;
  for (int t = lmax >> 1; t > 0; t >>= 1)
    if (delta(keys, n, i, i + (l + t) * d) > dmin) l += t;
  const int j = i + l * d;
  const int dnode = delta(keys, n, i, j);
  int s = 0;
  int t = l;
  do {
    t = (t + 1) >> 1;
    if (delta(keys, n, i, i + (s + t) * d) > dnode) s += t;
  } while (t > 1);
  const int gamma = i + s * d + (d < 0 ? -1 : 0);
  const int lo = min(i, j), hi = max(i, j);
  const int nm1 = (int)(n - 1);
  const int lc = (lo == gamma) ? nm1 + gamma : gamma;
  const int rc = (hi == gamma + 1) ? nm1 + gamma + 1 : gamma + 1;
  left[i] = lc;
  right[i] = rc;
  parent[lc] = i;
  parent[rc] = i;
  first[i] = lo;
  last[i] = hi;
  if (i == 0) parent[0] = -1;
}

// 5. refit: leaf boxes from sorted triangles, unions bottom-up
__global__ void refit_kernel(const uint32_t* __restrict__ order, const float4* __restrict__ tri_lo,
                             const float4* __restrict__ tri_hi, int64_t n, const int32_t* __restrict__ left,
                             const int32_t* __restrict__ right, const int32_t* __restrict__ parent,
                             float4* box_lo, float4* box_hi, uint32_t* visit) {
  const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const int64_t leaf = (n - 1) + j;
  const uint32_t f = order[j];
  box_lo[leaf] = tri_lo[f];
  box_hi[leaf] = tri_hi[f];
  if (n == 1) return;
  __threadfence();
  int p = parent[leaf];
  while (p >= 0) {
    if (atomicAdd(&visit[p], 1u) == 0u) return;  // sibling not done yet
    __threadfence();
    const int l = left[p], r = right[p];
    const float4 al = __ldcg(&box_lo[l]), ah = __ldcg(&box_hi[l]);
    const float4 bl = __ldcg(&box_lo[r]), bh = __ldcg(&box_hi[r]);
    __stcg(&box_lo[p], make_float4(fminf(al.x, bl.x), fminf(al.y, bl.y), fminf(al.z, bl.z), 0.f));
    __stcg(&box_hi[p], make_float4(fmaxf(ah.x, bh.x), fmaxf(ah.y, bh.y), fmaxf(ah.z, bh.z), 0.f));
    __threadfence();
    p = parent[p];
  }
}

__device__ __forceinline__ float half_area(float4 lo, float4 hi) {
  const float dx = hi.x - lo.x, dy = hi.y - lo.y, dz = hi.z - lo.z;
  return dx * dy + dy * dz + dz * dx;
}

// 6a. choose the (up to 4) children of each wide node of this level
__global__ void collapse_select_kernel(const int32_t* __restrict__ work_bin, int64_t nwork, int64_t n,
                                       int leaf_max, const int32_t* __restrict__ left,
                                       const int32_t* __restrict__ right, const int32_t* __restrict__ first,
                                       const int32_t* __restrict__ last, const float4* __restrict__ box_lo,
                                       const float4* __restrict__ box_hi, int32_t* __restrict__ child_bin,
                                       uint8_t* __restrict__ child_leaf, int32_t* __restrict__ nchild,
                                       uint32_t* __restrict__ nwide) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nwork) return;
  const int nm1 = (int)(n - 1);
  const int b = work_bin[k];
  int c[4];
  int cnt;
  if (b >= nm1) {  // a lone leaf as root (single-triangle mesh)
    c[0] = b;
    cnt = 1;
  } else {
    c[0] = left[b];
    c[1] = right[b];
    cnt = 2;
    while (cnt < 4) {
      int best = -1;
      float best_a = -1.f;
      for (int j = 0; j < cnt; ++j) {
        if (c[j] < nm1) {
          const float a = half_area(box_lo[c[j]], box_hi[c[j]]);
          if (a > best_a) { best_a = a; best = j; }
        }
      }
      if (best < 0) break;
      const int x = c[best];
      for (int j = cnt; j > best + 1; --j) c[j] = c[j - 1];
      c[best] = left[x];
      c[best + 1] = right[x];
      ++cnt;
    }
  }
  uint32_t w = 0;
  for (int j = 0; j < 4; ++j) {
    if (j < cnt) {
      const int cj = c[j];
      const int count = cj >= nm1 ? 1 : last[cj] - first[cj] + 1;
      const bool leaf = count <= leaf_max;
      child_bin[4 * k + j] = cj;
      child_leaf[4 * k + j] = leaf ? 1 : 0;
      if (!leaf) ++w;
    } else {
      child_bin[4 * k + j] = -1;
      child_leaf[4 * k + j] = 0;
    }
  }
  nchild[k] = cnt;
  nwide[k] = w;
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

// 6b. write the wide nodes of this level and the next worklist
__global__ void collapse_emit_kernel(const int32_t* __restrict__ work_bin, const int32_t* __restrict__ work_node,
                                     int64_t nwork, int64_t n, const int32_t* __restrict__ first,
                                     const int32_t* __restrict__ last, const float4* __restrict__ box_lo,
                                     const float4* __restrict__ box_hi, const int32_t* __restrict__ child_bin,
                                     const uint8_t* __restrict__ child_leaf, const int32_t* __restrict__ nchild,
                                     const uint32_t* __restrict__ nwide_off, int64_t level_base,
                                     WideNode* __restrict__ nodes, int32_t* __restrict__ next_bin,
                                     int32_t* __restrict__ next_node) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nwork) return;
  const int nm1 = (int)(n - 1);
  const int b = work_bin[k];
  const float4 plo = box_lo[b], phi = box_hi[b];
  WideNode nd;
  nd.ox = plo.x; nd.oy = plo.y; nd.oz = plo.z;
  const uint32_t ex = scale_exponent(phi.x - plo.x);
  const uint32_t ey = scale_exponent(phi.y - plo.y);
  const uint32_t ez = scale_exponent(phi.z - plo.z);
  const float sx = __uint_as_float(ex << 23), sy = __uint_as_float(ey << 23), sz = __uint_as_float(ez << 23);
  const int cnt = nchild[k];
  nd.meta = ex | (ey << 8) | (ez << 16) | ((uint32_t)cnt << 24);
  for (int a = 0; a < 6; ++a) nd.q[a] = 0;
  nd.pad[0] = (uint32_t)b;
  nd.pad[1] = 0;
  uint32_t m = nwide_off[k];
  for (int j = 0; j < 4; ++j) {
    if (j >= cnt) {
      // empty slot: inverted box (lo = 255, hi = 0) never passes a test
      nd.q[0] |= 255u << (8 * j); nd.q[1] |= 255u << (8 * j); nd.q[2] |= 255u << (8 * j);
      nd.ref[j] = 0xffffffffu;
      continue;
    }
    const int cj = child_bin[4 * k + j];
    const float4 lo = box_lo[cj], hi = box_hi[cj];
    uint32_t a0, a1;
    quantize_axis(nd.ox, sx, lo.x, hi.x, a0, a1); nd.q[0] |= a0 << (8 * j); nd.q[3] |= a1 << (8 * j);
    quantize_axis(nd.oy, sy, lo.y, hi.y, a0, a1); nd.q[1] |= a0 << (8 * j); nd.q[4] |= a1 << (8 * j);
    quantize_axis(nd.oz, sz, lo.z, hi.z, a0, a1); nd.q[2] |= a0 << (8 * j); nd.q[5] |= a1 << (8 * j);
    if (child_leaf[4 * k + j]) {
      const uint32_t f0 = cj >= nm1 ? (uint32_t)(cj - nm1) : (uint32_t)first[cj];
      const uint32_t c0 = cj >= nm1 ? 1u : (uint32_t)(last[cj] - first[cj] + 1);
      nd.ref[j] = make_leaf_ref(f0, c0);
    } else {
      const int64_t idx = level_base + m;
      nd.ref[j] = (uint32_t)idx;
      next_bin[m] = cj;
      next_node[m] = (int32_t)idx;
      ++m;
    }
  }
  nodes[work_node[k]] = nd;
}

// 7. triangle records in leaf (sorted) order
__global__ void write_tris_kernel(const float* __restrict__ V, const int32_t* __restrict__ F,
                                  const uint32_t* __restrict__ order, int64_t n, TriRec* __restrict__ tris) {
  const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const uint32_t f = order[j];
  const int32_t i0 = F[3 * f], i1 = F[3 * f + 1], i2 = F[3 * f + 2];
  const float3 a = ld3(V, i0), b = ld3(V, i1), c = ld3(V, i2);
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
  TriRec r;
  r.a = make_float4(a.x, a.y, a.z, __int_as_float((int)f));
  r.b = make_float4(b.x, b.y, b.z, __uint_as_float(flags));
  r.c = make_float4(c.x, c.y, c.z, nsqf > 0.f ? 1.0f / nsqf : 0.f);
  r.r = make_float4(1.0f / fmaxf(e0, 1e-12f), 1.0f / fmaxf(e1, 1e-12f), 1.0f / fmaxf(e2, 1e-12f), 0.f);
  tris[j] = r;
}

}  // namespace

}  // namespace a3d

using namespace a3d;

extern "C" size_t a3d_bvh_build_workspace_bytes(int64_t num_faces) {
  Workspace ws(nullptr, 0);
  BuildWs w;
  return carve(w, ws, num_faces > 0 ? num_faces : 1) + 256;
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
  A3D_REQUIRE(node_capacity >= 1, A3D_ERR_WORKSPACE, "bvh_build: node capacity");
  const int64_t n = num_faces;
  Workspace ws(workspace, workspace_bytes);
  BuildWs w;
  carve(w, ws, n);
  A3D_REQUIRE(workspace && ws.ok(), A3D_ERR_WORKSPACE, "bvh_build: workspace too small");
  if (leaf_max == 0) leaf_max = 4;
  A3D_REQUIRE(leaf_max >= 1 && leaf_max <= kMaxLeafTris, A3D_ERR_ARGUMENT, "bvh_build: leaf_max must be in 1..8");

  init_bounds_kernel<<<1, 32, 0, s>>>(w.bounds, w.err);
  A3D_LAUNCH_CHECK();
  const unsigned g = (unsigned)ceil_div(n, kThreads);
  tri_prep_kernel<<<g, kThreads, 0, s>>>(vertices, num_vertices, faces, n, w.tri_lo, w.tri_hi, w.centroid, w.bounds,
                                         w.err);
  A3D_LAUNCH_CHECK();
  morton_kernel<<<g, kThreads, 0, s>>>(w.centroid, n, w.bounds, w.keys, w.vals);
  A3D_LAUNCH_CHECK();
  bool alt = false;
  A3D_TRY(radix_sort_pairs<uint64_t>(w.keys, w.vals, w.keys_alt, w.vals_alt, n, 0, 64, w.rs_scratch, &alt, s));
  const uint64_t* keys = alt ? w.keys_alt : w.keys;
  const uint32_t* order = alt ? w.vals_alt : w.vals;

  if (n > 1) {
    radix_tree_kernel<<<(unsigned)ceil_div(n - 1, kThreads), kThreads, 0, s>>>(keys, n, w.left, w.right, w.parent,
                                                                              w.first, w.last);
    A3D_LAUNCH_CHECK();
    A3D_CUDA_TRY(cudaMemsetAsync(w.visit, 0, sizeof(uint32_t) * (n - 1), s));
  }
  refit_kernel<<<g, kThreads, 0, s>>>(order, w.tri_lo, w.tri_hi, n, w.left, w.right, w.parent, w.box_lo, w.box_hi,
                                      w.visit);
  A3D_LAUNCH_CHECK();
  write_tris_kernel<<<g, kThreads, 0, s>>>(vertices, faces, order, n, (TriRec*)tris_out);
  A3D_LAUNCH_CHECK();

  // level-synchronous collapse
  int32_t root_bin = 0;  // internal root, or the single leaf when n == 1 (index n-1 == 0)
  A3D_CUDA_TRY(cudaMemcpyAsync(w.work_a_bin, &root_bin, sizeof(int32_t), cudaMemcpyHostToDevice, s));
  A3D_CUDA_TRY(cudaMemsetAsync(w.work_a_node, 0, sizeof(int32_t), s));
  int64_t nwork = 1, level_base = 1;
  int32_t *cur_bin = w.work_a_bin, *cur_node = w.work_a_node, *nxt_bin = w.work_b_bin, *nxt_node = w.work_b_node;
  while (nwork > 0) {
    const unsigned gw = (unsigned)ceil_div(nwork, kThreads);
    collapse_select_kernel<<<gw, kThreads, 0, s>>>(cur_bin, nwork, n, leaf_max, w.left, w.right, w.first, w.last,
                                                   w.box_lo, w.box_hi, w.child_bin, w.child_leaf, w.nchild, w.nwide);
    A3D_LAUNCH_CHECK();
    A3D_TRY((device_exclusive_scan<uint32_t, uint32_t>(w.nwide, w.nwide_off, nwork, w.scan_tmp, w.total, s)));
    uint32_t total = 0;
    A3D_CUDA_TRY(cudaMemcpyAsync(&total, w.total, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    A3D_CUDA_TRY(cudaStreamSynchronize(s));
    A3D_REQUIRE(level_base + (int64_t)total <= node_capacity, A3D_ERR_WORKSPACE, "bvh_build: node capacity exceeded");
    collapse_emit_kernel<<<gw, kThreads, 0, s>>>(cur_bin, cur_node, nwork, n, w.first, w.last, w.box_lo, w.box_hi,
                                                 w.child_bin, w.child_leaf, w.nchild, w.nwide_off, level_base,
                                                 (WideNode*)nodes_out, nxt_bin, nxt_node);
    A3D_LAUNCH_CHECK();
    level_base += total;
    nwork = total;
    int32_t* t0 = cur_bin; cur_bin = nxt_bin; nxt_bin = t0;
    int32_t* t1 = cur_node; cur_node = nxt_node; nxt_node = t1;
  }
  uint32_t hb[12];
  int32_t herr[4];
  A3D_CUDA_TRY(cudaMemcpyAsync(hb, w.bounds, sizeof(hb), cudaMemcpyDeviceToHost, s));
  A3D_CUDA_TRY(cudaMemcpyAsync(herr, w.err, sizeof(herr), cudaMemcpyDeviceToHost, s));
  A3D_CUDA_TRY(cudaStreamSynchronize(s));
  A3D_REQUIRE(herr[0] == 0, A3D_ERR_ARGUMENT, "bvh_build: face index out of range");
  if (bounds_out) {
    for (int k = 0; k < 6; ++k) {
      uint32_t u = hb[k];
      uint32_t f = (u & 0x80000000u) ? (u & 0x7fffffffu) : ~u;
      memcpy(&bounds_out[k], &f, 4);
    }
  }
  *num_nodes_out = level_base;
  return A3D_OK;
}
