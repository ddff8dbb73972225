// Ray queries over the wide BVH: nearest hit, all hits, ray-parity inside
// votes.
//
// Replaces bvh_ray_intersect_kernel and bvh_ray_all_hit_kernel
// (atom3d/kernels/bvh_kernels.cu:469-553, :935-1022) and the host-side
// coalescing / vote loop of MeshBVH._sdf_parity and _signed_crossing_count
// (atom3d/core/mesh_bvh.py:850-948), which here is one fused kernel.
//
// The per-triangle maths is the reference's (Triangle::ray_intersect,
// ::normal, ::barycentric at bvh_kernels.cu:89-221) restated operation by
// operation with round-to-nearest intrinsics, so t values, hit decisions and
// signs are bit-identical to the oracle's restatement.  Child boxes are the
// outward-rounded quantised ones and a box is skipped only when its entry
// distance exceeds the current bound by a relative 2e-6, so pruning never
// drops a hit.  A triangle miss is +inf (the reference uses a 1e10 sentinel,
// which a max_t above 1e10 would count as a hit).
#include <math.h>

#include "bvh_layout.cuh"
#include "primitives.cuh"

namespace a3d {

namespace {

constexpr int kRayThreads = 128;
// shared-memory stack entries per ray: 20 KB per 128-thread block, and the
// nearest-hit kernel bounded to 48 registers, so that 10 blocks (40 warps)
// are resident per SM; a ray that needs more entries is re-run with a deep
// local stack
constexpr int kRayShared = 20;
constexpr int kRayBlocksPerSm = 10;
constexpr int kRayDeep = 256;    // local-memory stack of the re-run kernel
constexpr int kAllDepth = 192;   // node stack of the all-hit traversals
constexpr int kParityCap = 256;  // hits per (point, direction) kept by the parity kernel
constexpr float kPruneSlack = 1.000002f;

struct V3 {
  float x, y, z;
};

__device__ __forceinline__ V3 ld3(const float* p, int64_t i) { return V3{p[3 * i], p[3 * i + 1], p[3 * i + 2]}; }
__device__ __forceinline__ V3 vsub(V3 a, V3 b) {
  return V3{__fsub_rn(a.x, b.x), __fsub_rn(a.y, b.y), __fsub_rn(a.z, b.z)};
}
__device__ __forceinline__ float vdot(V3 a, V3 b) {
  return __fadd_rn(__fadd_rn(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y)), __fmul_rn(a.z, b.z));
}
__device__ __forceinline__ V3 vcross(V3 a, V3 b) {
  return V3{__fsub_rn(__fmul_rn(a.y, b.z), __fmul_rn(a.z, b.y)), __fsub_rn(__fmul_rn(a.z, b.x), __fmul_rn(a.x, b.z)),
            __fsub_rn(__fmul_rn(a.x, b.y), __fmul_rn(a.y, b.x))};
}
__device__ __forceinline__ V3 vpoint(V3 o, V3 d, float t) {
  return V3{__fadd_rn(o.x, __fmul_rn(d.x, t)), __fadd_rn(o.y, __fmul_rn(d.y, t)), __fadd_rn(o.z, __fmul_rn(d.z, t))};
}

struct Tri {
  V3 a, b, c;
  int32_t face;
};

__device__ __forceinline__ Tri load_tri(const TriRec* __restrict__ tris, uint32_t i) {
  const float4* p = reinterpret_cast<const float4*>(tris + i);
  const float4 a = __ldg(p), b = __ldg(p + 1), c = __ldg(p + 2);
  return Tri{V3{a.x, a.y, a.z}, V3{b.x, b.y, b.z}, V3{c.x, c.y, c.z}, __float_as_int(a.w)};
}

// Moller-Trumbore as Triangle::ray_intersect; +inf for a miss
__device__ __forceinline__ float ray_tri(const Tri& t, V3 ro, V3 rd) {
  const double eps_edge = 1.19209290e-7;
  const V3 e1 = vsub(t.b, t.a), e2 = vsub(t.c, t.a);
  const V3 h = vcross(rd, e2);
  const float det = vdot(e1, h);
  if (fabsf(det) < 1e-8f) return INFINITY;
  const float f = __fdiv_rn(1.0f, det);
  const V3 s = vsub(ro, t.a);
  const double u = __dmul_rn((double)f, (double)vdot(s, h));
  if (u < -eps_edge || u > 1.0 + eps_edge) return INFINITY;
  const V3 q = vcross(s, e1);
  const double v = __dmul_rn((double)f, (double)vdot(rd, q));
  if (v < -eps_edge || __dadd_rn(u, v) > 1.0 + eps_edge) return INFINITY;
  const float tt = __fmul_rn(f, vdot(e2, q));
  return tt > 1e-8f ? tt : INFINITY;
}

// Triangle::normal: unit normal of (b - a) x (c - a), (0, 0, 1) if degenerate
__device__ __forceinline__ V3 tri_normal(const Tri& t) {
  const V3 n = vcross(vsub(t.b, t.a), vsub(t.c, t.a));
  const float len = __fsqrt_rn(vdot(n, n));
  if (len > 1e-10f) {
    const float inv = __fdiv_rn(1.0f, len);
    return V3{__fmul_rn(n.x, inv), __fmul_rn(n.y, inv), __fmul_rn(n.z, inv)};
  }
  return V3{0.f, 0.f, 1.f};
}

// barycentrics of a point on the triangle: floor `dfloor` on the
// denominator (Triangle::barycentric, 1e-10) or additive `dadd`
// (MeshBVH._bary_from_hit, 1e-12)
__device__ __forceinline__ V3 tri_bary(const Tri& t, V3 p, bool additive) {
  const V3 v0 = vsub(t.b, t.a), v1 = vsub(t.c, t.a), v2 = vsub(p, t.a);
  const float d00 = vdot(v0, v0), d01 = vdot(v0, v1), d11 = vdot(v1, v1), d20 = vdot(v2, v0), d21 = vdot(v2, v1);
  float denom = __fsub_rn(__fmul_rn(d00, d11), __fmul_rn(d01, d01));
  denom = additive ? __fadd_rn(denom, 1e-12f) : fmaxf(denom, 1e-10f);
  const float v = __fdiv_rn(__fsub_rn(__fmul_rn(d11, d20), __fmul_rn(d01, d21)), denom);
  const float w = __fdiv_rn(__fsub_rn(__fmul_rn(d00, d21), __fmul_rn(d01, d20)), denom);
  return V3{__fsub_rn(__fsub_rn(1.0f, v), w), v, w};
}

struct Ray {
  V3 o, d, inv;
};

__device__ __forceinline__ Ray make_ray(V3 o, V3 d) {
  auto safe = [](float x) { return fabsf(x) > 1e-8f ? x : (x >= 0.f ? 1e-8f : -1e-8f); };
  return Ray{o, d, V3{__fdiv_rn(1.0f, safe(d.x)), __fdiv_rn(1.0f, safe(d.y)), __fdiv_rn(1.0f, safe(d.z))}};
}

// entry distances of a node's four children (+inf for a miss or an empty
// slot) and their references
__device__ __forceinline__ void child_entries(const WideNode* __restrict__ nodes, uint32_t ref, const Ray& r,
                                              float* tc, uint32_t* rc) {
  const int4* np = reinterpret_cast<const int4*>(nodes + ref);
  const int4 w0 = __ldg(np), w1 = __ldg(np + 1), w2 = __ldg(np + 2), w3 = __ldg(np + 3);
  const float ox = __int_as_float(w0.x), oy = __int_as_float(w0.y), oz = __int_as_float(w0.z);
  const uint32_t meta = (uint32_t)w0.w;
  const float sx = __uint_as_float((meta & 0xffu) << 23);
  const float sy = __uint_as_float(((meta >> 8) & 0xffu) << 23);
  const float sz = __uint_as_float(((meta >> 16) & 0xffu) << 23);
  const int nch = (int)(meta >> 24);
  rc[0] = (uint32_t)w2.z;
  rc[1] = (uint32_t)w2.w;
  rc[2] = (uint32_t)w3.x;
  rc[3] = (uint32_t)w3.y;
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    const float lx = dequant((uint32_t)w1.x, c, sx, ox), ly = dequant((uint32_t)w1.y, c, sy, oy);
    const float lz = dequant((uint32_t)w1.z, c, sz, oz), hx = dequant((uint32_t)w1.w, c, sx, ox);
    const float hy = dequant((uint32_t)w2.x, c, sy, oy), hz = dequant((uint32_t)w2.y, c, sz, oz);
    float t1 = (lx - r.o.x) * r.inv.x, t2 = (hx - r.o.x) * r.inv.x;
    float tmin = fminf(t1, t2), tmax = fmaxf(t1, t2);
    t1 = (ly - r.o.y) * r.inv.y;
    t2 = (hy - r.o.y) * r.inv.y;
    tmin = fmaxf(tmin, fminf(t1, t2));
    tmax = fminf(tmax, fmaxf(t1, t2));
    t1 = (lz - r.o.z) * r.inv.z;
    t2 = (hz - r.o.z) * r.inv.z;
    tmin = fmaxf(tmin, fminf(t1, t2));
    tmax = fminf(tmax, fmaxf(t1, t2));
    tc[c] = (c < nch && tmax >= tmin && tmax >= 0.f) ? fmaxf(tmin, 0.f) : INFINITY;
  }
}

__device__ __forceinline__ void cswap(float& ta, uint32_t& ra, float& tb, uint32_t& rb) {
  if (tb < ta || (tb == ta && rb < ra)) {
    const float t = ta;
    ta = tb;
    tb = t;
    const uint32_t x = ra;
    ra = rb;
    rb = x;
  }
}

struct SharedStack {
  uint2* base;
  int sp;
  static constexpr int kDepth = kRayShared;
  __device__ __forceinline__ void push(uint32_t ref, float t) {
    base[sp * kRayThreads] = make_uint2(ref, __float_as_uint(t));
    ++sp;
  }
  __device__ __forceinline__ uint2 pop() {
    --sp;
    return base[sp * kRayThreads];
  }
};

struct LocalStack {
  uint2 s[kRayDeep];
  int sp;
  static constexpr int kDepth = kRayDeep;
  __device__ __forceinline__ void push(uint32_t ref, float t) { s[sp++] = make_uint2(ref, __float_as_uint(t)); }
  __device__ __forceinline__ uint2 pop() { return s[--sp]; }
};

// Nearest hit: children in ascending entry distance, strict "<" on t.
// Returns false when the stack would overflow (the ray is re-run).
template <typename Stack>
__device__ bool nearest(const WideNode* __restrict__ nodes, const TriRec* __restrict__ tris, const Ray& r,
                        float& mint, uint32_t& best, Stack& st) {
  uint32_t ref = 0;
  bool have = true;
  for (;;) {
    if (have) {
      if (!ref_is_leaf(ref)) {
        float tc[4];
        uint32_t rc[4];
        child_entries(nodes, ref, r, tc, rc);
        cswap(tc[0], rc[0], tc[1], rc[1]);
        cswap(tc[2], rc[2], tc[3], rc[3]);
        cswap(tc[0], rc[0], tc[2], rc[2]);
        cswap(tc[1], rc[1], tc[3], rc[3]);
        cswap(tc[1], rc[1], tc[2], rc[2]);
        const float lim = mint * kPruneSlack;
        int q = 0;
#pragma unroll
        for (int c = 0; c < 4; ++c) q += tc[c] <= lim ? 1 : 0;
        if (q > 0) {
          if (st.sp + (q - 1) > Stack::kDepth) return false;
#pragma unroll
          for (int c = 3; c >= 1; --c)
            if (c < q) st.push(rc[c], tc[c]);
          ref = rc[0];
          continue;
        }
      } else {
        const uint32_t f0 = leaf_first(ref), cnt = leaf_count(ref);
        for (uint32_t i = 0; i < cnt; ++i) {
          const float t = ray_tri(load_tri(tris, f0 + i), r.o, r.d);
          if (t < mint) {
            mint = t;
            best = f0 + i;
          }
        }
      }
    }
    have = false;
    while (st.sp > 0) {
      const uint2 e = st.pop();
      if (__uint_as_float(e.y) <= mint * kPruneSlack) {
        ref = e.x;
        have = true;
        break;
      }
    }
    if (!have) return true;
  }
}

struct RayOut {
  uint8_t* hit;
  float* t;
  int32_t* face;
  float* point;
  float* normal;
  float* uvw;
};

__device__ void write_nearest(const TriRec* __restrict__ tris, const float* __restrict__ face_normals, const Ray& r,
                              int64_t i, float mint, uint32_t best, const RayOut& out) {
  const bool hit = best != 0xffffffffu;
  out.hit[i] = hit ? 1 : 0;
  out.t[i] = mint;
  V3 p{0.f, 0.f, 0.f}, nrm{0.f, 0.f, 0.f}, bc{0.f, 0.f, 0.f};
  int32_t face = -1;
  if (hit) {
    const Tri t = load_tri(tris, best);
    face = t.face;
    p = vpoint(r.o, r.d, mint);
    if (out.uvw) bc = tri_bary(t, p, true);
    if (face_normals) nrm = ld3(face_normals, face);
  }
  out.face[i] = face;
  if (out.point) {
    out.point[3 * i] = p.x;
    out.point[3 * i + 1] = p.y;
    out.point[3 * i + 2] = p.z;
  }
  if (out.normal) {
    out.normal[3 * i] = nrm.x;
    out.normal[3 * i + 1] = nrm.y;
    out.normal[3 * i + 2] = nrm.z;
  }
  if (out.uvw) {
    out.uvw[3 * i] = bc.x;
    out.uvw[3 * i + 1] = bc.y;
    out.uvw[3 * i + 2] = bc.z;
  }
}

__global__ void __launch_bounds__(kRayThreads, kRayBlocksPerSm)
    ray_nearest_kernel(const WideNode* __restrict__ nodes, const TriRec* __restrict__ tris,
                       const float* __restrict__ face_normals, const float* __restrict__ ro,
                       const float* __restrict__ rd, int64_t n, float max_t, RayOut out, uint32_t* __restrict__ rerun,
                       uint32_t* __restrict__ nrerun) {
  pdl_wait();
  __shared__ uint2 s_stack[kRayShared * kRayThreads];
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const Ray r = make_ray(ld3(ro, i), ld3(rd, i));
  float mint = max_t;
  uint32_t best = 0xffffffffu;
  SharedStack st{s_stack + threadIdx.x, 0};
  if (!nearest(nodes, tris, r, mint, best, st)) {
    rerun[atomicAdd(nrerun, 1u)] = (uint32_t)i;
    return;
  }
  write_nearest(tris, face_normals, r, i, mint, best, out);
}

__global__ void __launch_bounds__(64)
    ray_nearest_rerun_kernel(const WideNode* __restrict__ nodes, const TriRec* __restrict__ tris,
                             const float* __restrict__ face_normals, const float* __restrict__ ro,
                             const float* __restrict__ rd, float max_t, RayOut out,
                             const uint32_t* __restrict__ rerun, const uint32_t* __restrict__ nrerun,
                             uint32_t* __restrict__ overflow) {
  pdl_wait();
  const uint32_t m = *nrerun;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < m; k += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = rerun[k];
    const Ray r = make_ray(ld3(ro, i), ld3(rd, i));
    float mint = max_t;
    uint32_t best = 0xffffffffu;
    LocalStack st;
    st.sp = 0;
    if (!nearest(nodes, tris, r, mint, best, st)) atomicExch(overflow, 1u);
    write_nearest(tris, face_normals, r, i, mint, best, out);
  }
}

// All hits of one ray in traversal order; `emit(t, tri)` for each
// non-grazing hit with 0 < t < max_t.  Returns false on stack overflow.
template <typename Emit>
__device__ bool all_hits(const WideNode* __restrict__ nodes, const TriRec* __restrict__ tris, const Ray& r,
                         float max_t, Emit emit) {
  uint32_t stack[kAllDepth];
  int sp = 0;
  stack[sp++] = 0u;
  const float lim = max_t * kPruneSlack;
  bool ok = true;
  while (sp > 0) {
    const uint32_t ref = stack[--sp];
    if (!ref_is_leaf(ref)) {
      float tc[4];
      uint32_t rc[4];
      child_entries(nodes, ref, r, tc, rc);
#pragma unroll
      for (int c = 3; c >= 0; --c) {
        if (tc[c] <= lim) {
          if (sp < kAllDepth) stack[sp++] = rc[c];
          else ok = false;
        }
      }
    } else {
      const uint32_t f0 = leaf_first(ref), cnt = leaf_count(ref);
      for (uint32_t k = 0; k < cnt; ++k) {
        const Tri t = load_tri(tris, f0 + k);
        const float th = ray_tri(t, r.o, r.d);
        if (th > 0.0f && th < max_t) {
          const float ndotd = vdot(tri_normal(t), r.d);
          if (ndotd > -1e-4f && ndotd < 1e-4f) continue;  // grazing
          emit(th, t, ndotd > 0.0f ? 1 : -1);
        }
      }
    }
  }
  return ok;
}

__global__ void ray_all_count_kernel(const WideNode* __restrict__ nodes, const TriRec* __restrict__ tris,
                                     const float* __restrict__ ro, const float* __restrict__ rd, int64_t n,
                                     float max_t, int32_t* __restrict__ counts, uint32_t* __restrict__ overflow) {
  pdl_wait();
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const Ray r = make_ray(ld3(ro, i), ld3(rd, i));
  int32_t c = 0;
  if (!all_hits(nodes, tris, r, max_t, [&](float, const Tri&, int) { ++c; })) atomicExch(overflow, 1u);
  counts[i] = c;
}

struct AllOut {
  int32_t* ray;
  float* t;
  int32_t* face;
  int32_t* sign;
  float* point;
  float* uvw;
};

__global__ void ray_all_collect_kernel(const WideNode* __restrict__ nodes, const TriRec* __restrict__ tris,
                                       const float* __restrict__ ro, const float* __restrict__ rd, int64_t n,
                                       float max_t, const int64_t* __restrict__ offsets, AllOut out) {
  pdl_wait();
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const Ray r = make_ray(ld3(ro, i), ld3(rd, i));
  int64_t w = offsets[i];
  const int64_t wend = offsets[i + 1];
  all_hits(nodes, tris, r, max_t, [&](float th, const Tri& t, int s) {
    if (w >= wend) return;  // the count pass saw the same hits; kept as a bound
    out.ray[w] = (int32_t)i;
    out.t[w] = th;
    out.face[w] = t.face;
    out.sign[w] = s;
    const V3 p = vpoint(r.o, r.d, th);
    if (out.point) {
      out.point[3 * w] = p.x;
      out.point[3 * w + 1] = p.y;
      out.point[3 * w + 2] = p.z;
    }
    if (out.uvw) {
      const V3 b = tri_bary(t, p, false);
      out.uvw[3 * w] = b.x;
      out.uvw[3 * w + 1] = b.y;
      out.uvw[3 * w + 2] = b.z;
    }
    ++w;
  });
}

// Per point: for each direction, the signed crossing count of the ray with
// near-coincident hits (|dt| < coalesce, after sorting by t) merged -- a
// group whose hits all share a sign counts as one crossing of that sign, a
// mixed group as (|sum| mod 2) * sign(sum) -- and a vote when it is odd.
__global__ void __launch_bounds__(64)
    ray_parity_kernel(const WideNode* __restrict__ nodes, const TriRec* __restrict__ tris,
                      const float* __restrict__ pts, int64_t n, const float* __restrict__ dirs, int ndir, float max_t,
                      float coalesce, int32_t* __restrict__ votes, uint32_t* __restrict__ overflow) {
  pdl_wait();
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const V3 o = ld3(pts, i);
  float ts[kParityCap];
  int8_t sg[kParityCap];
  int32_t vote = 0;
  for (int d = 0; d < ndir; ++d) {
    const Ray r = make_ray(o, ld3(dirs, d));
    int k = 0;
    bool lost = false;
    if (!all_hits(nodes, tris, r, max_t, [&](float th, const Tri&, int s) {
          // insertion by t keeps the buffer sorted (stable for equal t)
          if (k >= kParityCap) {
            lost = true;
            return;
          }
          int j = k;
          while (j > 0 && ts[j - 1] > th) {
            ts[j] = ts[j - 1];
            sg[j] = sg[j - 1];
            --j;
          }
          ts[j] = th;
          sg[j] = (int8_t)s;
          ++k;
        }))
      lost = true;
    if (lost) atomicExch(overflow, 1u);
    int32_t sc = 0;
    int a = 0;
    while (a < k) {
      int b = a + 1;
      int32_t cnt = 1, sum = sg[a];
      while (b < k && fabsf(__fsub_rn(ts[b], ts[b - 1])) < coalesce) {
        ++cnt;
        sum += sg[b];
        ++b;
      }
      const int32_t sgn = sum > 0 ? 1 : (sum < 0 ? -1 : 0);
      const int32_t asum = sum < 0 ? -sum : sum;
      sc += asum == cnt ? sgn : (asum % 2) * sgn;
      a = b;
    }
    vote += ((sc < 0 ? -sc : sc) % 2) == 1 ? 1 : 0;
  }
  votes[i] = vote;
}

}  // namespace

}  // namespace a3d

using namespace a3d;

extern "C" size_t a3d_ray_workspace_bytes(int64_t num_rays) {
  Workspace ws(nullptr, 0);
  ws.take<uint32_t>(4);
  ws.take<uint32_t>(num_rays > 0 ? num_rays : 1);
  ws.take<int32_t>(num_rays > 0 ? num_rays : 1);
  ws.take<uint32_t>((int64_t)scan_workspace_elems(num_rays > 0 ? num_rays : 1) * 2);
  return ws.used + 256;
}

namespace {
struct RayWs {
  uint32_t* status;  // [0] re-run count, [1] stack / buffer overflow
  uint32_t* rerun;
  int32_t* counts;
  int64_t* scan_tmp;
};
bool carve_ray(RayWs& w, void* p, size_t bytes, int64_t n) {
  Workspace ws(p, bytes);
  w.status = ws.take<uint32_t>(4);
  w.rerun = ws.take<uint32_t>(n > 0 ? n : 1);
  w.counts = ws.take<int32_t>(n > 0 ? n : 1);
  w.scan_tmp = ws.take<int64_t>((int64_t)scan_workspace_elems(n > 0 ? n : 1));
  return p && ws.ok();
}
}  // namespace

extern "C" int a3d_ray_nearest(const a3d_bvh_view* bvh, const float* rays_o, const float* rays_d, int64_t num_rays,
                               float max_t, const float* face_normals, uint8_t* hit, float* t, int32_t* face_ids,
                               float* hit_points, float* normals, float* uvw, void* workspace,
                               size_t workspace_bytes, a3d_stream_t stream_) {
  cudaStream_t s = (cudaStream_t)stream_;
  A3D_REQUIRE(bvh && bvh->nodes && bvh->tris, A3D_ERR_ARGUMENT, "ray_nearest: invalid bvh");
  A3D_REQUIRE(num_rays >= 0 && num_rays < (1ll << 32), A3D_ERR_ARGUMENT, "ray_nearest: bad number of rays");
  RayWs w;
  A3D_REQUIRE(carve_ray(w, workspace, workspace_bytes, num_rays), A3D_ERR_WORKSPACE, "ray_nearest: workspace");
  A3D_CUDA_TRY(cudaMemsetAsync(w.status, 0, 4 * sizeof(uint32_t), s));
  if (num_rays == 0) return A3D_OK;
  A3D_REQUIRE(rays_o && rays_d && hit && t && face_ids, A3D_ERR_ARGUMENT, "ray_nearest: null pointer");
  A3D_REQUIRE(normals == nullptr || face_normals != nullptr, A3D_ERR_ARGUMENT,
              "ray_nearest: normals need the face normals");
  const WideNode* nodes = (const WideNode*)bvh->nodes;
  const TriRec* tris = (const TriRec*)bvh->tris;
  const RayOut out{hit, t, face_ids, hit_points, normals, uvw};
  A3D_PDL(ray_nearest_kernel, dim3((unsigned)ceil_div(num_rays, kRayThreads)), dim3(kRayThreads), 0, s, nodes, tris,
          face_normals, rays_o, rays_d, num_rays, max_t, out, w.rerun, w.status);
  A3D_PDL(ray_nearest_rerun_kernel, dim3(num_sms() * 4), dim3(64), 0, s, nodes, tris, face_normals, rays_o, rays_d,
          max_t, out, w.rerun, w.status, w.status + 1);
  return A3D_OK;
}

extern "C" int a3d_ray_all_count(const a3d_bvh_view* bvh, const float* rays_o, const float* rays_d, int64_t num_rays,
                                 float max_t, int64_t* offsets_out, void* workspace, size_t workspace_bytes,
                                 a3d_stream_t stream_) {
  cudaStream_t s = (cudaStream_t)stream_;
  A3D_REQUIRE(bvh && bvh->nodes && bvh->tris, A3D_ERR_ARGUMENT, "ray_all: invalid bvh");
  A3D_REQUIRE(num_rays >= 0 && num_rays < (1ll << 32) && offsets_out, A3D_ERR_ARGUMENT, "ray_all: bad argument");
  RayWs w;
  A3D_REQUIRE(carve_ray(w, workspace, workspace_bytes, num_rays), A3D_ERR_WORKSPACE, "ray_all: workspace");
  A3D_CUDA_TRY(cudaMemsetAsync(w.status, 0, 4 * sizeof(uint32_t), s));
  if (num_rays == 0) return cudaMemsetAsync(offsets_out, 0, sizeof(int64_t), s) == cudaSuccess ? A3D_OK : A3D_ERR_CUDA;
  A3D_REQUIRE(rays_o && rays_d, A3D_ERR_ARGUMENT, "ray_all: null pointer");
  A3D_PDL(ray_all_count_kernel, dim3((unsigned)ceil_div(num_rays, 128)), dim3(128), 0, s, (const WideNode*)bvh->nodes,
          (const TriRec*)bvh->tris, rays_o, rays_d, num_rays, max_t, w.counts, w.status + 1);
  A3D_TRY((device_exclusive_scan<int32_t, int64_t>(w.counts, offsets_out, num_rays, w.scan_tmp,
                                                   offsets_out + num_rays, s)));
  return A3D_OK;
}

extern "C" int a3d_ray_all_collect(const a3d_bvh_view* bvh, const float* rays_o, const float* rays_d,
                                   int64_t num_rays, float max_t, const int64_t* offsets, int32_t* ray_idx,
                                   float* t, int32_t* face_ids, int32_t* sign, float* hit_points, float* uvw,
                                   a3d_stream_t stream_) {
  cudaStream_t s = (cudaStream_t)stream_;
  A3D_REQUIRE(bvh && bvh->nodes && bvh->tris, A3D_ERR_ARGUMENT, "ray_all: invalid bvh");
  A3D_REQUIRE(num_rays >= 0 && num_rays < (1ll << 32), A3D_ERR_ARGUMENT, "ray_all: bad number of rays");
  if (num_rays == 0) return A3D_OK;
  A3D_REQUIRE(rays_o && rays_d && offsets && ray_idx && t && face_ids && sign, A3D_ERR_ARGUMENT,
              "ray_all: null pointer");
  const AllOut out{ray_idx, t, face_ids, sign, hit_points, uvw};
  A3D_PDL(ray_all_collect_kernel, dim3((unsigned)ceil_div(num_rays, 128)), dim3(128), 0, s, (const WideNode*)bvh->nodes,
          (const TriRec*)bvh->tris, rays_o, rays_d, num_rays, max_t, offsets, out);
  return A3D_OK;
}

extern "C" int a3d_ray_parity_votes(const a3d_bvh_view* bvh, const float* points, int64_t num_points,
                                    const float* dirs, int32_t num_dirs, float max_t, float coalesce_t,
                                    int32_t* votes, void* workspace, size_t workspace_bytes, a3d_stream_t stream_) {
  cudaStream_t s = (cudaStream_t)stream_;
  A3D_REQUIRE(bvh && bvh->nodes && bvh->tris, A3D_ERR_ARGUMENT, "ray_parity: invalid bvh");
  A3D_REQUIRE(num_points >= 0 && num_dirs > 0 && num_dirs <= 1024, A3D_ERR_ARGUMENT, "ray_parity: bad argument");
  RayWs w;
  A3D_REQUIRE(carve_ray(w, workspace, workspace_bytes, 0), A3D_ERR_WORKSPACE, "ray_parity: workspace");
  A3D_CUDA_TRY(cudaMemsetAsync(w.status, 0, 4 * sizeof(uint32_t), s));
  if (num_points == 0) return A3D_OK;
  A3D_REQUIRE(points && dirs && votes, A3D_ERR_ARGUMENT, "ray_parity: null pointer");
  A3D_PDL(ray_parity_kernel, dim3((unsigned)ceil_div(num_points, 64)), dim3(64), 0, s, (const WideNode*)bvh->nodes,
          (const TriRec*)bvh->tris, points, num_points, dirs, num_dirs, max_t, coalesce_t, votes, w.status + 1);
  return A3D_OK;
}

extern "C" int a3d_ray_status(const void* workspace, uint32_t* status_out, a3d_stream_t stream) {
  A3D_REQUIRE(workspace && status_out, A3D_ERR_ARGUMENT, "ray_status: null pointer");
  A3D_CUDA_TRY(cudaMemcpyAsync(status_out, workspace, 2 * sizeof(uint32_t), cudaMemcpyDeviceToHost,
                               (cudaStream_t)stream));
  A3D_CUDA_TRY(cudaStreamSynchronize((cudaStream_t)stream));
  return A3D_OK;
}
