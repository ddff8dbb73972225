// MeshBVH.intersect_aabb modes 1-3: (box, face) pairs, optionally clipped.
//
// Replaces the pair output of bvh_aabb_intersect_kernel
// (atom3d/kernels/bvh_kernels.cu:555-610, host :1192-1242) and
// sat_clip_polygon_kernel / clip_with_plane (atom3d/kernels/cumtv_kernels.cu:
// 209-460) behind atom3d/core/mesh_bvh.py:297-479:
//   mode 1  every face passing SAT (sat_eps 1e-6) against the box
//   mode 2  those whose Sutherland-Hodgman clip against the box's 6 planes
//           (eps 1e-8) is non-empty, with the polygon's vertex count, its
//           centroid projected onto the triangle, and its fan area
//   mode 3  mode 2 plus the polygon's vertices (8 slots, zero padded)
//
// The tree walk finds the faces passing SAT, in two passes over the boxes:
// a count pass, an exclusive scan of the counts, and a write pass that puts
// each box's pairs at its offset -- exact-size outputs, no truncation (the
// reference keeps at most min(100 N, 5e7) candidates and drops the rest
// silently).  Mode 1 writes the pairs directly.  Modes 2-3 write them as a
// candidate list (box, triangle slot) and clip it one thread per candidate,
// converged: a flag pass (clip, hit mask), an exclusive scan of the flags,
// and an emit pass that clips again and writes the outputs at their
// compacted index.  (Clipping inside the divergent walk ran with one or two
// active lanes per warp and was 10x slower.)  Pairs come grouped by box in
// ascending order, in tree order within a box; the reference's order is
// that of an atomic counter.
//
// The clip is restated operation by operation with round-to-nearest
// intrinsics (IEEE divide and square root, no contraction), so the CPU
// oracle built with -ffp-contract=off reproduces it bit for bit.  An
// emitted vertex past the 8-slot polygon buffer is dropped (the reference
// writes it past its local array) and the count saturates at 8.
#include "box_query.cuh"
#include "primitives.cuh"

namespace a3d {
namespace {

constexpr int kClipMaxV = 8;
constexpr float kClipEps = 1e-8f;

struct Poly {
  float v[kClipMaxV][3];
};

// one clip step against n.p - d <= eps, n = sign * e_axis
__device__ __forceinline__ int clip_plane(const Poly& in, int n_in, int axis, float sign, float d, Poly& out) {
  if (n_in <= 0) return 0;
  const float n0 = axis == 0 ? sign : 0.0f, n1 = axis == 1 ? sign : 0.0f, n2 = axis == 2 ? sign : 0.0f;
  float dist[kClipMaxV];
#pragma unroll
  for (int i = 0; i < kClipMaxV; ++i)
    if (i < n_in) dist[i] = fsb(fa(fa(fm(in.v[i][0], n0), fm(in.v[i][1], n1)), fm(in.v[i][2], n2)), d);
  int m = 0;
#pragma unroll
  for (int i = 0; i < kClipMaxV; ++i) {
    if (i >= n_in) break;
    const int j = (i + 1 == n_in) ? 0 : i + 1;
    const float dP = dist[i], dQ = dist[j];
    const bool inP = dP <= kClipEps, inQ = dQ <= kClipEps;
    if (inP && inQ) {
      if (m < kClipMaxV) {
        out.v[m][0] = in.v[j][0]; out.v[m][1] = in.v[j][1]; out.v[m][2] = in.v[j][2];
      }
      ++m;
    } else if (inP != inQ) {
      const float den = fsb(dP, dQ);
      if (fabsf(den) > kClipEps) {
        const float t = __fdiv_rn(dP, den);
        if (m < kClipMaxV) {
#pragma unroll
          for (int a = 0; a < 3; ++a) out.v[m][a] = fa(in.v[i][a], fm(t, fsb(in.v[j][a], in.v[i][a])));
        }
        ++m;
      }
      if (inQ) {
        if (m < kClipMaxV) {
          out.v[m][0] = in.v[j][0]; out.v[m][1] = in.v[j][1]; out.v[m][2] = in.v[j][2];
        }
        ++m;
      }
    }
    if (m >= kClipMaxV) return kClipMaxV;
  }
  return m;
}

struct ClipOut {
  int count;
  float cx, cy, cz;  // centroid (projected onto the triangle)
  float area;
};

// Clips triangle t against the box; returns the vertex count (0 = empty).
// The polygon ends in pa.
__device__ __forceinline__ int clip_tri(const TriRec& t, const float mn[3], const float mx[3], Poly& pa, Poly& pb) {
  pa.v[0][0] = t.a.x; pa.v[0][1] = t.a.y; pa.v[0][2] = t.a.z;
  pa.v[1][0] = t.b.x; pa.v[1][1] = t.b.y; pa.v[1][2] = t.b.z;
  pa.v[2][0] = t.c.x; pa.v[2][1] = t.c.y; pa.v[2][2] = t.c.z;
  int n = 3;
  n = clip_plane(pa, n, 0, 1.0f, mx[0], pb);
  if (!n) return 0;
  n = clip_plane(pb, n, 0, -1.0f, -mn[0], pa);
  if (!n) return 0;
  n = clip_plane(pa, n, 1, 1.0f, mx[1], pb);
  if (!n) return 0;
  n = clip_plane(pb, n, 1, -1.0f, -mn[1], pa);
  if (!n) return 0;
  n = clip_plane(pa, n, 2, 1.0f, mx[2], pb);
  if (!n) return 0;
  n = clip_plane(pb, n, 2, -1.0f, -mn[2], pa);
  return n > kClipMaxV ? kClipMaxV : n;
}

// centroid (mean clamped to the box, projected onto the triangle with
// clamped barycentrics) and fan area about the clamped mean
__device__ __forceinline__ ClipOut clip_measure(const TriRec& t, const float mn[3], const float mx[3], const Poly& p,
                                                int cnt) {
  ClipOut o;
  o.count = cnt;
  o.area = 0.0f;
  float c[3] = {0.0f, 0.0f, 0.0f};
  for (int i = 0; i < cnt; ++i) {
    c[0] = fa(c[0], p.v[i][0]);
    c[1] = fa(c[1], p.v[i][1]);
    c[2] = fa(c[2], p.v[i][2]);
  }
#pragma unroll
  for (int a = 0; a < 3; ++a) c[a] = fminf(fmaxf(__fdiv_rn(c[a], (float)cnt), mn[a]), mx[a]);
  const float ax = t.a.x, ay = t.a.y, az = t.a.z, bx = t.b.x, by = t.b.y, bz = t.b.z;
  const float qx = t.c.x, qy = t.c.y, qz = t.c.z;
  const float e1x = fsb(bx, ax), e1y = fsb(by, ay), e1z = fsb(bz, az);
  const float e2x = fsb(qx, ax), e2y = fsb(qy, ay), e2z = fsb(qz, az);
  const float vx = fsb(c[0], ax), vy = fsb(c[1], ay), vz = fsb(c[2], az);
  const float d00 = dot3r(e1x, e1y, e1z, e1x, e1y, e1z);
  const float d01 = dot3r(e1x, e1y, e1z, e2x, e2y, e2z);
  const float d11 = dot3r(e2x, e2y, e2z, e2x, e2y, e2z);
  const float d20 = dot3r(vx, vy, vz, e1x, e1y, e1z);
  const float d21 = dot3r(vx, vy, vz, e2x, e2y, e2z);
  const float den = fsb(fm(d00, d11), fm(d01, d01));
  if (fabsf(den) < fm(kClipEps, kClipEps)) {
    o.cx = ax; o.cy = ay; o.cz = az;  // degenerate triangle: area stays 0
    return o;
  }
  float v = __fdiv_rn(fsb(fm(d11, d20), fm(d01, d21)), den);
  float w = __fdiv_rn(fsb(fm(d00, d21), fm(d01, d20)), den);
  float u = fsb(fsb(1.0f, v), w);
  if (u < 0.0f) u = 0.0f;
  if (v < 0.0f) v = 0.0f;
  if (w < 0.0f) w = 0.0f;
  float nn = fa(fa(u, v), w);
  if (nn <= kClipEps) { u = 1.0f; v = 0.0f; w = 0.0f; nn = 1.0f; }
  u = __fdiv_rn(u, nn); v = __fdiv_rn(v, nn); w = __fdiv_rn(w, nn);
  o.cx = fa(fa(fm(u, ax), fm(v, bx)), fm(w, qx));
  o.cy = fa(fa(fm(u, ay), fm(v, by)), fm(w, qy));
  o.cz = fa(fa(fm(u, az), fm(v, bz)), fm(w, qz));
  float ar = 0.0f;
  for (int i = 0; i < cnt; ++i) {
    const int j = (i + 1) % cnt;
    const float p0 = fsb(p.v[i][0], c[0]), p1 = fsb(p.v[i][1], c[1]), p2 = fsb(p.v[i][2], c[2]);
    const float q0 = fsb(p.v[j][0], c[0]), q1 = fsb(p.v[j][1], c[1]), q2 = fsb(p.v[j][2], c[2]);
    const float x = fsb(fm(p1, q2), fm(p2, q1)), y = fsb(fm(p2, q0), fm(p0, q2)), z = fsb(fm(p0, q1), fm(p1, q0));
    ar = fa(ar, fm(0.5f, __fsqrt_rn(dot3r(x, y, z, x, y, z))));
  }
  o.area = ar < kClipEps ? 0.0f : ar;
  return o;
}

struct PairOut {
  void* aabb_ids;  // int32 (mode 1) or int64 (modes 2-3)
  void* face_ids;
  int32_t* poly_counts;
  float* centroids;
  float* areas;
  float* poly_verts;  // mode 3
};

// Clips candidate k (box cand_box[k], triangle record cand_slot[k]).
template <bool kEmit, int kMode>
__device__ __forceinline__ void clip_candidate(const TriRec* __restrict__ tris, const float* __restrict__ bmin,
                                               const float* __restrict__ bmax, const uint32_t* __restrict__ cand_box,
                                               const uint32_t* __restrict__ cand_slot, int64_t k,
                                               uint32_t* __restrict__ flags, uint8_t* __restrict__ hit,
                                               const int64_t* __restrict__ coffs, const PairOut& out,
                                               int64_t n, int64_t num_slots, int64_t num_pairs,
                                               unsigned long long* __restrict__ faults) {
  const int64_t i = cand_box[k];
  const uint32_t slot = cand_slot[k];
  if (i >= n || slot >= num_slots) {  // never for a candidate list written by the walk
    atomicAdd(faults, 1ull);
    if (!kEmit) flags[k] = 0;
    return;
  }
  const float4* p = reinterpret_cast<const float4*>(tris + slot);
  TriRec t;
  t.a = __ldg(p); t.b = __ldg(p + 1); t.c = __ldg(p + 2); t.r = make_float4(0.f, 0.f, 0.f, 0.f);
  const float mn[3] = {bmin[3 * i], bmin[3 * i + 1], bmin[3 * i + 2]};
  const float mx[3] = {bmax[3 * i], bmax[3 * i + 1], bmax[3 * i + 2]};
  Poly pa, pb;
  const int cnt = clip_tri(t, mn, mx, pa, pb);
  if (!kEmit) {
    flags[k] = cnt > 0;
    if (cnt > 0) hit[i] = 1;
    return;
  }
  if (!cnt) return;
  const int64_t o = coffs[k];
  if (!flags[k] || o < 0 || o >= num_pairs) {  // the flag pass decided this clip differently
    atomicAdd(faults, 1ull);
    return;
  }
  const ClipOut c = clip_measure(t, mn, mx, pa, cnt);
  reinterpret_cast<int64_t*>(out.aabb_ids)[o] = i;
  reinterpret_cast<int64_t*>(out.face_ids)[o] = __float_as_int(t.a.w);
  out.poly_counts[o] = c.count;
  out.centroids[3 * o] = c.cx;
  out.centroids[3 * o + 1] = c.cy;
  out.centroids[3 * o + 2] = c.cz;
  out.areas[o] = c.area;
  if (kMode == 3) {
    float4* pv = reinterpret_cast<float4*>(out.poly_verts + 24 * o);
#pragma unroll
    for (int q = 0; q < 6; ++q) {
      float e[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int f = 4 * q + u, vi = f / 3, ax = f % 3;
        e[u] = vi < cnt ? pa.v[vi][ax] : 0.0f;
      }
      pv[q] = make_float4(e[0], e[1], e[2], e[3]);
    }
  }
}

__global__ void clip_flags_kernel(const TriRec* __restrict__ tris, const float* __restrict__ bmin,
                                  const float* __restrict__ bmax, const uint32_t* __restrict__ cand_box,
                                  const uint32_t* __restrict__ cand_slot, int64_t m, uint32_t* __restrict__ flags,
                                  uint8_t* __restrict__ hit, int64_t n, int64_t num_slots,
                                  unsigned long long* __restrict__ faults) {
  pdl_wait();
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < m)
    clip_candidate<false, 2>(tris, bmin, bmax, cand_box, cand_slot, k, flags, hit, nullptr, PairOut{}, n, num_slots,
                             0, faults);
}

template <int kMode>
__global__ void clip_emit_kernel(const TriRec* __restrict__ tris, const float* __restrict__ bmin,
                                 const float* __restrict__ bmax, const uint32_t* __restrict__ cand_box,
                                 const uint32_t* __restrict__ cand_slot, int64_t m, uint32_t* __restrict__ flags,
                                 const int64_t* __restrict__ coffs, PairOut out, int64_t n, int64_t num_slots,
                                 unsigned long long* __restrict__ faults) {
  pdl_wait();
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < m)
    clip_candidate<true, kMode>(tris, bmin, bmax, cand_box, cand_slot, k, flags, nullptr, coffs, out, n, num_slots,
                                coffs[m], faults);
}

// Walks the tree for box i; counts (kWrite false) or writes (true) its
// SAT pairs from slot base: kSlots false writes int32 (box, face id) pairs,
// kSlots true the candidate list (box, triangle record slot).  Returns the
// traversal status (2 = overflow); *count = pairs.
template <bool kWrite, bool kSlots, typename Stack>
__device__ __forceinline__ int box_pairs(const WideNode* __restrict__ nodes, const TriRec* __restrict__ tris,
                                         const float* __restrict__ bmin, const float* __restrict__ bmax, int64_t i,
                                         Stack& st, int64_t base, int64_t end, int32_t* __restrict__ out_box,
                                         int32_t* __restrict__ out_face, uint32_t* count,
                                         unsigned long long* __restrict__ faults) {
  const float mnx = bmin[3 * i], mny = bmin[3 * i + 1], mnz = bmin[3 * i + 2];
  const float mxx = bmax[3 * i], mxy = bmax[3 * i + 1], mxz = bmax[3 * i + 2];
  uint32_t k = 0;
  const int r = box_traverse(nodes, tris, mnx, mny, mnz, mxx, mxy, mxz, st, [&](const TriRec& t, uint32_t slot) {
    if (!sat_test(t, mnx, mny, mnz, mxx, mxy, mxz)) return false;
    if (kWrite) {
      if (base + k < end) {  // the count pass found the same pairs
        out_box[base + k] = (int32_t)i;
        out_face[base + k] = kSlots ? (int32_t)slot : __float_as_int(t.a.w);
      } else {
        atomicAdd(faults, 1ull);
      }
    }
    ++k;
    return false;
  });
  *count = k;
  return r;
}

struct PairsWs {
  uint32_t* counts;
  int64_t* offs;
  int64_t* scan_tmp;
  uint32_t* spill;
  unsigned long long* misc;  // [0] spill count, [1] overflow, [2] guard faults
};

size_t carve_pairs(PairsWs& w, Workspace& ws, int64_t n) {
  w.counts = ws.take<uint32_t>(n);
  w.offs = ws.take<int64_t>(n + 1);
  w.scan_tmp = ws.take<int64_t>((int64_t)scan_workspace_elems(n));
  w.spill = ws.take<uint32_t>(n);
  w.misc = ws.take<unsigned long long>(4);
  return ws.used;
}

struct ClipWs {
  uint32_t* cand_box;
  uint32_t* cand_slot;
  uint32_t* flags;
  int64_t* coffs;
  int64_t* scan_tmp;
};

size_t carve_clip(ClipWs& w, Workspace& ws, int64_t m) {
  w.cand_box = ws.take<uint32_t>(m);
  w.cand_slot = ws.take<uint32_t>(m);
  w.flags = ws.take<uint32_t>(m);
  w.coffs = ws.take<int64_t>(m + 1);
  w.scan_tmp = ws.take<int64_t>((int64_t)scan_workspace_elems(m));
  return ws.used;
}

__global__ void __launch_bounds__(kSatThreads)
    pairs_count_kernel(const WideNode* __restrict__ nodes, const TriRec* __restrict__ tris,
                       const float* __restrict__ bmin, const float* __restrict__ bmax, int64_t n,
                       uint32_t* __restrict__ counts, uint8_t* __restrict__ hit, uint32_t* __restrict__ spill,
                       unsigned long long* __restrict__ misc) {
  pdl_wait();
  __shared__ uint32_t s_stack[kSatDepth * kSatThreads];
  const int64_t i = (int64_t)blockIdx.x * kSatThreads + threadIdx.x;
  if (i >= n) return;
  ShStack st{s_stack + threadIdx.x, 0};
  uint32_t c = 0;
  if (box_pairs<false, false>(nodes, tris, bmin, bmax, i, st, 0, 0, nullptr, nullptr, &c, nullptr) == 2) {
    spill[atomicAdd(misc, 1ull)] = (uint32_t)i;
    c = 0;
  }
  counts[i] = c;
  if (hit) hit[i] = c > 0;
}

__global__ void pairs_count_spill_kernel(const WideNode* __restrict__ nodes, const TriRec* __restrict__ tris,
                                         const float* __restrict__ bmin, const float* __restrict__ bmax,
                                         uint32_t* __restrict__ counts, uint8_t* __restrict__ hit,
                                         const uint32_t* __restrict__ spill, unsigned long long* __restrict__ misc) {
  pdl_wait();
  const uint64_t m = misc[0];
  for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < m; t += (uint64_t)gridDim.x * blockDim.x) {
    const int64_t i = spill[t];
    LcStack st;
    st.sp = 0;
    uint32_t c = 0;
    if (box_pairs<false, false>(nodes, tris, bmin, bmax, i, st, 0, 0, nullptr, nullptr, &c, nullptr) == 2) {
      atomicExch(misc + 1, 1ull);
      c = 0;
    }
    counts[i] = c;
    if (hit) hit[i] = c > 0;
  }
}

template <bool kSlots>
__global__ void __launch_bounds__(kSatThreads)
    pairs_write_kernel(const WideNode* __restrict__ nodes, const TriRec* __restrict__ tris,
                       const float* __restrict__ bmin, const float* __restrict__ bmax, int64_t n,
                       const int64_t* __restrict__ offs, int32_t* __restrict__ out_box,
                       int32_t* __restrict__ out_face, unsigned long long* __restrict__ misc) {
  pdl_wait();
  __shared__ uint32_t s_stack[kSatDepth * kSatThreads];
  const int64_t i = (int64_t)blockIdx.x * kSatThreads + threadIdx.x;
  if (i >= n) return;
  ShStack st{s_stack + threadIdx.x, 0};
  uint32_t c;
  // a box whose walk overflows here overflowed in the count pass too (same
  // walk): the spill kernel rewrites its whole segment
  box_pairs<true, kSlots>(nodes, tris, bmin, bmax, i, st, offs[i], offs[i + 1], out_box, out_face, &c, misc + 2);
}

template <bool kSlots>
__global__ void pairs_write_spill_kernel(const WideNode* __restrict__ nodes, const TriRec* __restrict__ tris,
                                         const float* __restrict__ bmin, const float* __restrict__ bmax,
                                         const int64_t* __restrict__ offs, const uint32_t* __restrict__ spill,
                                         unsigned long long* __restrict__ misc, int32_t* __restrict__ out_box,
                                         int32_t* __restrict__ out_face) {
  pdl_wait();
  const uint64_t m = misc[0];
  for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < m; t += (uint64_t)gridDim.x * blockDim.x) {
    const int64_t i = spill[t];
    LcStack st;
    st.sp = 0;
    uint32_t c;
    box_pairs<true, kSlots>(nodes, tris, bmin, bmax, i, st, offs[i], offs[i + 1], out_box, out_face, &c, misc + 2);
  }
}

template <bool kSlots>
int launch_write(const a3d_bvh_view* bvh, const float* bmin, const float* bmax, int64_t n, const PairsWs& w,
                 int32_t* out_box, int32_t* out_face, cudaStream_t s) {
  const WideNode* nodes = (const WideNode*)bvh->nodes;
  const TriRec* tris = (const TriRec*)bvh->tris;
  A3D_PDL(pairs_write_kernel<kSlots>, dim3((unsigned)ceil_div(n, kSatThreads)), dim3(kSatThreads), 0, s, nodes, tris,
          bmin, bmax, n, w.offs, out_box, out_face, w.misc);
  A3D_PDL(pairs_write_spill_kernel<kSlots>, dim3(num_sms() * 4), dim3(64), 0, s, nodes, tris, bmin, bmax, w.offs,
          w.spill, w.misc, out_box, out_face);
  return A3D_OK;
}

}  // namespace
}  // namespace a3d

using namespace a3d;

extern "C" size_t a3d_aabb_pairs_workspace_bytes(int64_t n) {
  Workspace ws(nullptr, 0);
  PairsWs w;
  return carve_pairs(w, ws, n > 0 ? n : 1) + 256;
}

extern "C" size_t a3d_aabb_clip_workspace_bytes(int64_t num_candidates) {
  Workspace ws(nullptr, 0);
  ClipWs w;
  return carve_clip(w, ws, num_candidates > 0 ? num_candidates : 1) + 256;
}

namespace {
int check_pairs_args(const a3d_bvh_view* bvh, int mode, int64_t n) {
  A3D_REQUIRE(bvh && bvh->nodes && bvh->tris, A3D_ERR_ARGUMENT, "aabb_pairs: invalid bvh");
  A3D_REQUIRE(mode >= 1 && mode <= 3, A3D_ERR_ARGUMENT, "aabb_pairs: mode must be 1, 2 or 3");
  A3D_REQUIRE(n >= 0 && n < (1ll << 31), A3D_ERR_ARGUMENT, "aabb_pairs: bad size");
  return A3D_OK;
}
}  // namespace

extern "C" int a3d_aabb_pairs_count(const a3d_bvh_view* bvh, const float* box_min, const float* box_max, int64_t n,
                                    int mode, uint8_t* hit, void* workspace, size_t workspace_bytes,
                                    int64_t* num_candidates_out, a3d_stream_t stream) {
  cudaStream_t s = (cudaStream_t)stream;
  A3D_TRY(check_pairs_args(bvh, mode, n));
  A3D_REQUIRE(num_candidates_out, A3D_ERR_ARGUMENT, "aabb_pairs: null count output");
  *num_candidates_out = 0;
  if (n == 0) return A3D_OK;
  A3D_REQUIRE(box_min && box_max && hit, A3D_ERR_ARGUMENT, "aabb_pairs: null pointer");
  Workspace ws(workspace, workspace_bytes);
  PairsWs w;
  carve_pairs(w, ws, n);
  A3D_REQUIRE(workspace && ws.ok(), A3D_ERR_WORKSPACE, "aabb_pairs: workspace too small");
  A3D_CUDA_TRY(cudaMemsetAsync(w.misc, 0, 4 * sizeof(unsigned long long), s));
  // modes 2-3: the hit mask comes from the clip
  uint8_t* h = mode == 1 ? hit : nullptr;
  const WideNode* nodes = (const WideNode*)bvh->nodes;
  const TriRec* tris = (const TriRec*)bvh->tris;
  A3D_PDL(pairs_count_kernel, dim3((unsigned)ceil_div(n, kSatThreads)), dim3(kSatThreads), 0, s, nodes, tris, box_min,
          box_max, n, w.counts, h, w.spill, w.misc);
  A3D_PDL(pairs_count_spill_kernel, dim3(num_sms() * 4), dim3(64), 0, s, nodes, tris, box_min, box_max, w.counts, h,
          w.spill, w.misc);
  A3D_TRY((device_exclusive_scan<uint32_t, int64_t>(w.counts, w.offs, n, w.scan_tmp, w.offs + n, s)));
  unsigned long long misc[4];
  int64_t total = 0;
  A3D_CUDA_TRY(cudaMemcpyAsync(misc, w.misc, sizeof(misc), cudaMemcpyDeviceToHost, s));
  A3D_CUDA_TRY(cudaMemcpyAsync(&total, w.offs + n, sizeof(total), cudaMemcpyDeviceToHost, s));
  A3D_CUDA_TRY(cudaStreamSynchronize(s));
  A3D_REQUIRE(misc[1] == 0, A3D_ERR_OVERFLOW, "aabb_pairs: traversal stack overflow");
  *num_candidates_out = total;
  return A3D_OK;
}

extern "C" int a3d_aabb_pairs_clip(const a3d_bvh_view* bvh, const float* box_min, const float* box_max, int64_t n,
                                   void* workspace, size_t workspace_bytes, void* clip_workspace,
                                   size_t clip_workspace_bytes, int64_t num_candidates, uint8_t* hit,
                                   int64_t* num_pairs_out, a3d_stream_t stream) {
  cudaStream_t s = (cudaStream_t)stream;
  A3D_TRY(check_pairs_args(bvh, 2, n));
  A3D_REQUIRE(num_pairs_out && num_candidates >= 0 && num_candidates < (1ll << 32), A3D_ERR_ARGUMENT,
              "aabb_pairs_clip: bad argument");
  *num_pairs_out = 0;
  if (n == 0) return A3D_OK;
  A3D_REQUIRE(box_min && box_max && hit, A3D_ERR_ARGUMENT, "aabb_pairs_clip: null pointer");
  Workspace ws(workspace, workspace_bytes);
  PairsWs w;
  carve_pairs(w, ws, n);
  Workspace cws(clip_workspace, clip_workspace_bytes);
  ClipWs c;
  carve_clip(c, cws, num_candidates);
  A3D_REQUIRE(workspace && ws.ok() && clip_workspace && cws.ok(), A3D_ERR_WORKSPACE,
              "aabb_pairs_clip: workspace too small");
  A3D_CUDA_TRY(cudaMemsetAsync(hit, 0, n, s));
  if (num_candidates == 0) return A3D_OK;
  A3D_TRY(launch_write<true>(bvh, box_min, box_max, n, w, (int32_t*)c.cand_box, (int32_t*)c.cand_slot, s));
  A3D_PDL(clip_flags_kernel, dim3((unsigned)ceil_div(num_candidates, 256)), dim3(256), 0, s, (const TriRec*)bvh->tris,
          box_min, box_max, c.cand_box, c.cand_slot, num_candidates, c.flags, hit, n, bvh->num_tris, w.misc + 2);
  A3D_TRY((device_exclusive_scan<uint32_t, int64_t>(c.flags, c.coffs, num_candidates, c.scan_tmp,
                                                     c.coffs + num_candidates, s)));
  int64_t total = 0;
  unsigned long long faults = 0;
  A3D_CUDA_TRY(cudaMemcpyAsync(&total, c.coffs + num_candidates, sizeof(total), cudaMemcpyDeviceToHost, s));
  A3D_CUDA_TRY(cudaMemcpyAsync(&faults, w.misc + 2, sizeof(faults), cudaMemcpyDeviceToHost, s));
  A3D_CUDA_TRY(cudaStreamSynchronize(s));
  A3D_REQUIRE(faults == 0, A3D_ERR_OVERFLOW, "aabb_pairs_clip: a candidate index guard fired");
  *num_pairs_out = total;
  return A3D_OK;
}

extern "C" int a3d_aabb_pairs_write(const a3d_bvh_view* bvh, const float* box_min, const float* box_max, int64_t n,
                                    int mode, void* workspace, size_t workspace_bytes, void* clip_workspace,
                                    size_t clip_workspace_bytes, int64_t num_candidates, void* aabb_ids,
                                    void* face_ids, int32_t* poly_counts, float* centroids, float* areas,
                                    float* poly_verts, a3d_stream_t stream) {
  cudaStream_t s = (cudaStream_t)stream;
  A3D_TRY(check_pairs_args(bvh, mode, n));
  if (n == 0) return A3D_OK;
  A3D_REQUIRE(box_min && box_max && aabb_ids && face_ids, A3D_ERR_ARGUMENT, "aabb_pairs: null output");
  Workspace ws(workspace, workspace_bytes);
  PairsWs w;
  carve_pairs(w, ws, n);
  A3D_REQUIRE(workspace && ws.ok(), A3D_ERR_WORKSPACE, "aabb_pairs: workspace too small");
  if (mode == 1) {
    A3D_TRY(launch_write<false>(bvh, box_min, box_max, n, w, (int32_t*)aabb_ids, (int32_t*)face_ids, s));
  } else {
    A3D_REQUIRE(poly_counts && centroids && areas, A3D_ERR_ARGUMENT, "aabb_pairs: null clip output");
    A3D_REQUIRE(mode != 3 || (poly_verts && ((uintptr_t)poly_verts & 15) == 0), A3D_ERR_ARGUMENT,
                "aabb_pairs: poly_verts must be a 16-byte aligned [P,8,3] buffer");
    Workspace cws(clip_workspace, clip_workspace_bytes);
    ClipWs c;
    carve_clip(c, cws, num_candidates);
    A3D_REQUIRE(clip_workspace && cws.ok() && num_candidates >= 0, A3D_ERR_WORKSPACE,
                "aabb_pairs: clip workspace too small");
    if (num_candidates == 0) return A3D_OK;
    const PairOut out{aabb_ids, face_ids, poly_counts, centroids, areas, poly_verts};
    const unsigned g = (unsigned)ceil_div(num_candidates, 256);
    if (mode == 2)
      A3D_PDL(clip_emit_kernel<2>, dim3(g), dim3(256), 0, s, (const TriRec*)bvh->tris, box_min, box_max, c.cand_box,
              c.cand_slot, num_candidates, c.flags, c.coffs, out, n, bvh->num_tris, w.misc + 2);
    else
      A3D_PDL(clip_emit_kernel<3>, dim3(g), dim3(256), 0, s, (const TriRec*)bvh->tris, box_min, box_max, c.cand_box,
              c.cand_slot, num_candidates, c.flags, c.coffs, out, n, bvh->num_tris, w.misc + 2);
  }
  unsigned long long faults = 0;
  A3D_CUDA_TRY(cudaMemcpyAsync(&faults, w.misc + 2, sizeof(faults), cudaMemcpyDeviceToHost, s));
  A3D_CUDA_TRY(cudaStreamSynchronize(s));
  A3D_REQUIRE(faults == 0, A3D_ERR_OVERFLOW, "aabb_pairs_write: an output index guard fired");
  return A3D_OK;
}
