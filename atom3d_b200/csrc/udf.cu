// Closest-triangle queries over the wide BVH: UDF, fused pseudo-normal SDF
// sign, learned-bound seeding, and the distance adjoints.
//
// Replaces bvh_udf_kernel (atom3d/kernels/bvh_kernels.cu:363-463) and the
// PyTorch sign gathers of MeshBVH._compute_sign (atom3d/core/mesh_bvh.py:
// 759-827).  Design:
//   * queries are Morton-sorted (30-bit key, in-house radix sort) so a warp
//     walks neighbouring regions of the tree together;
//   * one 64-B node = four 16-B loads; the four child boxes are decoded from
//     8-bit offsets, sorted by distance with a 5-exchange network, the
//     nearest qualifying child is visited next and the others pushed;
//   * the traversal stack lives in shared memory ([depth][thread] layout, no
//     bank conflicts); a query that would overflow it is re-run by a
//     fallback launch with a deep local-memory stack, never truncated;
//   * a per-query bound (learned upper bound on the distance) seeds the
//     pruning radius; a query whose bound proves too small is re-run
//     without it, so results are identical with and without the bound.
#include <math.h>

#include "bvh_layout.cuh"
#include "primitives.cuh"
#include "tri_math.cuh"

namespace a3d {

namespace {

constexpr int kUdfThreads = 128;
constexpr int kSharedDepth = 32;
constexpr int kDeepDepth = 256;

struct SignArgs {
  const float* face_normals;
  const float* vertex_pn;
  const float* edge_pn;
  const int64_t* he_edge_idx;
  const int32_t* faces;
};

struct QueryOut {
  float* dist;
  int32_t* fid;
  float* cp;
  float* uvw;
};

struct Counters {
  unsigned long long nodes;
  unsigned long long tris;
};

// Which tree a query walks.  One mesh: the root is node 0.  A batch: query
// qi (index qbase + qi in the caller's array) belongs to mesh m with
// qoff[m] <= qbase + qi < qoff[m+1], whose root is roots[m].
struct MeshSel {
  const int64_t* qoff;
  const uint32_t* roots;
  int nmesh;
  int64_t qbase;
  __device__ __forceinline__ uint32_t root_of(int64_t qi) const {
    if (qoff == nullptr) return 0u;
    const int64_t g = qbase + qi;
    int lo = 0, hi = nmesh - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (__ldg(qoff + mid) <= g) lo = mid;
      else hi = mid - 1;
    }
    return __ldg(roots + lo);
  }
};

// children are visited in ascending (distance, ref) order: a total order, so
// every traversal variant (single lane, quad of lanes) walks the same
// sequence and breaks distance ties identically
__device__ __forceinline__ bool child_less(float da, uint32_t ra, float db, uint32_t rb) {
  return da < db || (da == db && ra < rb);
}

__device__ __forceinline__ void cswap(float& da, uint32_t& ra, float& db, uint32_t& rb) {
  if (child_less(db, rb, da, ra)) {
    float t = da; da = db; db = t;
    uint32_t u = ra; ra = rb; rb = u;
  }
}

__device__ __forceinline__ float box_dist_sq(float px, float py, float pz, float lx, float ly, float lz, float hx,
                                             float hy, float hz) {
  const float dx = fmaxf(fmaxf(lx - px, px - hx), 0.f);
  const float dy = fmaxf(fmaxf(ly - py, py - hy), 0.f);
  const float dz = fmaxf(fmaxf(lz - pz, pz - hz), 0.f);
  return dx * dx + dy * dy + dz * dz;
}

// FP64 evaluation for near-degenerate triangles, kept out of line so the
// hot loop does not carry its registers.
__device__ __noinline__ float tri_dist_sq_f64(float ax, float ay, float az, float bx, float by, float bz, float cx,
                                              float cy, float cz, float px, float py, float pz) {
  const double d = TriEval<double>::dist_sq(mk<double>(px, py, pz), mk<double>(ax, ay, az), mk<double>(bx, by, bz),
                                            mk<double>(cx, cy, cz));
  return (float)d;
}

__device__ __forceinline__ float tri_dist_sq(const TriRec& t, float px, float py, float pz) {
  if (t.c.w < 0.f)  // near-degenerate
    return tri_dist_sq_f64(t.a.x, t.a.y, t.a.z, t.b.x, t.b.y, t.b.z, t.c.x, t.c.y, t.c.z, px, py, pz);
  return dist_sq_bary(mk(px, py, pz), mk(t.a.x, t.a.y, t.a.z), mk(t.b.x, t.b.y, t.b.z), mk(t.c.x, t.c.y, t.c.z),
                      t.c.w, t.b.w, t.r.w, t.r.x, t.r.y, t.r.z);
}

__device__ __forceinline__ TriRec load_tri(const TriRec* tris, uint32_t i) {
  const float4* p = reinterpret_cast<const float4*>(tris + i);
  TriRec r;
  r.a = __ldg(p);
  r.b = __ldg(p + 1);
  r.c = __ldg(p + 2);
  r.r = __ldg(p + 3);
  return r;
}

// The arrays a traversal reads.  With kGuard (batches, whose node count is
// only known on the device) a node or triangle index outside the arrays is
// recorded in *fault (kFaultNode / kFaultTri) and replaced by 0, so no
// access leaves them whatever the tree holds.
constexpr uint32_t kFaultNode = 1u, kFaultTri = 2u;

template <bool kGuard>
struct TreeT {
  const WideNode* __restrict__ nodes;
  const TriRec* __restrict__ tris;
  uint32_t num_nodes;
  uint32_t num_tris;
  uint32_t* fault;
  __device__ __forceinline__ const int4* node(uint32_t ref) const {
    if (kGuard && ref >= num_nodes) {
      atomicOr(fault, kFaultNode);
      ref = 0;
    }
    return reinterpret_cast<const int4*>(nodes + ref);
  }
  __device__ __forceinline__ TriRec tri(uint32_t i) const {
    if (kGuard && i >= num_tris) {
      atomicOr(fault, kFaultTri);
      i = 0;
    }
    return load_tri(tris, i);
  }
};

// Stack in shared memory, [depth][blockDim] layout.
struct SharedStack {
  uint2* base;  // points at s[0][threadIdx.x]
  int sp;
  static constexpr int kDepth = kSharedDepth;
  __device__ __forceinline__ void push(uint32_t ref, float d) {
    base[sp * kUdfThreads] = make_uint2(ref, __float_as_uint(d));
    ++sp;
  }
  __device__ __forceinline__ uint2 pop() {
    --sp;
    return base[sp * kUdfThreads];
  }
};

struct LocalStack {
  uint2 s[kDeepDepth];
  int sp;
  static constexpr int kDepth = kDeepDepth;
  __device__ __forceinline__ void push(uint32_t ref, float d) { s[sp++] = make_uint2(ref, __float_as_uint(d)); }
  __device__ __forceinline__ uint2 pop() { return s[--sp]; }
};

// Core traversal.  Returns false when the stack would overflow (result then
// invalid).  best_sq: in = initial pruning radius^2, out = best distance^2.
template <typename Stack, typename Tree>
__device__ __forceinline__ bool traverse(const Tree& T, float px, float py, float pz, Stack& st, float& best_sq,
                                         uint32_t& best_tri, Counters& ctr, uint32_t root = 0u) {
  uint32_t ref = root;  // a root is always an internal node (a single-leaf tree still has one)
  bool have = true;
  for (;;) {
    if (have) {
      if (!ref_is_leaf(ref)) {
        ++ctr.nodes;
        const int4* np = T.node(ref);
        const int4 w0 = __ldg(np), w1 = __ldg(np + 1), w2 = __ldg(np + 2), w3 = __ldg(np + 3);
        const float ox = __int_as_float(w0.x), oy = __int_as_float(w0.y), oz = __int_as_float(w0.z);
        const uint32_t meta = (uint32_t)w0.w;
        const float sx = __uint_as_float((meta & 0xffu) << 23);
        const float sy = __uint_as_float(((meta >> 8) & 0xffu) << 23);
        const float sz = __uint_as_float(((meta >> 16) & 0xffu) << 23);
        const uint32_t qlx = (uint32_t)w1.x, qly = (uint32_t)w1.y, qlz = (uint32_t)w1.z;
        const uint32_t qhx = (uint32_t)w1.w, qhy = (uint32_t)w2.x, qhz = (uint32_t)w2.y;
        float d[4];
        uint32_t r[4] = {(uint32_t)w2.z, (uint32_t)w2.w, (uint32_t)w3.x, (uint32_t)w3.y};
        const int nch = (int)(meta >> 24);
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const float lx = dequant(qlx, c, sx, ox);
          const float ly = dequant(qly, c, sy, oy);
          const float lz = dequant(qlz, c, sz, oz);
          const float hx = dequant(qhx, c, sx, ox);
          const float hy = dequant(qhy, c, sy, oy);
          const float hz = dequant(qhz, c, sz, oz);
          d[c] = c < nch ? box_dist_sq(px, py, pz, lx, ly, lz, hx, hy, hz) : INFINITY;
        }
        cswap(d[0], r[0], d[1], r[1]);
        cswap(d[2], r[2], d[3], r[3]);
        cswap(d[0], r[0], d[2], r[2]);
        cswap(d[1], r[1], d[3], r[3]);
        cswap(d[1], r[1], d[2], r[2]);
        int q = 0;
#pragma unroll
        for (int c = 0; c < 4; ++c) q += d[c] < best_sq ? 1 : 0;
        if (q > 0) {
          if (st.sp + (q - 1) > Stack::kDepth) return false;
#pragma unroll
          for (int c = 3; c >= 1; --c)
            if (c < q) st.push(r[c], d[c]);
          ref = r[0];
          continue;
        }
      } else {
        const uint32_t f0 = leaf_first(ref), cnt = leaf_count(ref);
        for (uint32_t i = 0; i < cnt; ++i) {
          const TriRec t = T.tri(f0 + i);
          ++ctr.tris;
          const float dsq = tri_dist_sq(t, px, py, pz);
          if (dsq < best_sq) {
            best_sq = dsq;
            best_tri = f0 + i;
          }
        }
      }
    }
    // pop the next candidate that can still beat best_sq
    have = false;
    while (st.sp > 0) {
      const uint2 e = st.pop();
      if (__uint_as_float(e.y) < best_sq) {
        ref = e.x;
        have = true;
        break;
      }
    }
    if (!have) return true;
  }
}

__device__ __noinline__ void finish_query(const TriRec* __restrict__ tris, uint32_t num_tris, uint32_t best_tri,
                                          float best_sq,
                                             float px, float py, float pz, int64_t qi, const QueryOut& out,
                                             const SignArgs& sg, bool do_sign) {
  float cx = px, cy = py, cz = pz;
  int32_t face = -1;
  float u = 0.f, v = 0.f, w = 0.f;
  float dist = sqrtf(best_sq);
  if (best_tri != 0xffffffffu) {
    const TriRec t = load_tri(tris, best_tri < num_tris ? best_tri : 0u);
    face = __float_as_int(t.a.w);
    const V3<float> a = mk(t.a.x, t.a.y, t.a.z), b = mk(t.b.x, t.b.y, t.b.z), c = mk(t.c.x, t.c.y, t.c.z);
    const V3<float> p = mk(px, py, pz);
    V3<float> cp;
    if (t.c.w < 0.f) {  // near-degenerate
      const V3<double> cd = TriEval<double>::closest(mk<double>(px, py, pz), mk<double>(a.x, a.y, a.z),
                                                     mk<double>(b.x, b.y, b.z), mk<double>(c.x, c.y, c.z));
      cp = mk((float)cd.x, (float)cd.y, (float)cd.z);
    } else {
      cp = TriEval<float>::closest(p, a, b, c);
    }
    cx = cp.x; cy = cp.y; cz = cp.z;
    const V3<float> bc = TriEval<float>::bary(cp, a, b, c);
    u = bc.x; v = bc.y; w = bc.z;
    if (do_sign) {
      // Baerentzen-Aanaes pseudo-normal selected from the barycentrics
      const float eps = 1e-4f;
      const bool z0 = u < eps, z1 = v < eps, z2 = w < eps;
      const int nz = (int)z0 + (int)z1 + (int)z2;
      const float* nrm = sg.face_normals + 3 * (int64_t)face;
      if (sg.edge_pn == nullptr) {
        // face normals only (caller supplied vertex normals)
      } else if (nz == 2) {
        const int dom = !z0 ? 0 : (!z1 ? 1 : 2);
        const int64_t vid = sg.faces[3 * (int64_t)face + dom];
        nrm = sg.vertex_pn + 3 * vid;
      } else if (nz == 1) {
        const int zi = z0 ? 0 : (z1 ? 1 : 2);
        const int he = zi == 0 ? 1 : (zi == 1 ? 2 : 0);
        const int64_t eid = sg.he_edge_idx[3 * (int64_t)face + he];
        nrm = sg.edge_pn + 3 * eid;
      }
      const float nx = __ldg(nrm), ny = __ldg(nrm + 1), nzv = __ldg(nrm + 2);
      float s;
      if (dist < 1e-3f) {
        // near the surface the sign is decided in FP64 from an FP64 closest point
        const V3<double> cd = TriEval<double>::closest(mk<double>(px, py, pz), mk<double>(a.x, a.y, a.z),
                                                       mk<double>(b.x, b.y, b.z), mk<double>(c.x, c.y, c.z));
        const double dd = ((double)px - cd.x) * nx + ((double)py - cd.y) * ny + ((double)pz - cd.z) * nzv;
        s = dd < 0.0 ? -1.f : 1.f;
      } else {
        const float dd = (px - cx) * nx + (py - cy) * ny + (pz - cz) * nzv;
        s = dd < 0.f ? -1.f : 1.f;
      }
      dist *= s;
    }
  }
  out.dist[qi] = dist;
  out.fid[qi] = face;
  out.cp[3 * qi] = cx;
  out.cp[3 * qi + 1] = cy;
  out.cp[3 * qi + 2] = cz;
  if (out.uvw && best_tri != 0xffffffffu) {
    out.uvw[3 * qi] = u;
    out.uvw[3 * qi + 1] = v;
    out.uvw[3 * qi + 2] = w;
  }
}

__device__ __forceinline__ void flush_counters(const Counters& c, unsigned long long* stats) {
  unsigned long long a = warp_reduce_sum(c.nodes), b = warp_reduce_sum(c.tris);
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(stats, a);
    atomicAdd(stats + 1, b);
  }
}

// Greedy root-to-leaf probe: follows the nearest child and tests that
// leaf's triangles.  Gives a real triangle (and its distance) that seeds the
// pruning radius of the full traversal.
template <typename Tree>
__device__ __forceinline__ void probe(const Tree& T, float px, float py, float pz, uint32_t& tri, float& dsq,
                                     Counters& ctr, uint32_t root = 0u) {
  uint32_t ref = root;
  while (!ref_is_leaf(ref)) {
    ++ctr.nodes;
    const int4* np = T.node(ref);
    const int4 w0 = __ldg(np), w1 = __ldg(np + 1), w2 = __ldg(np + 2), w3 = __ldg(np + 3);
    const float ox = __int_as_float(w0.x), oy = __int_as_float(w0.y), oz = __int_as_float(w0.z);
    const uint32_t meta = (uint32_t)w0.w;
    const float sx = __uint_as_float((meta & 0xffu) << 23);
    const float sy = __uint_as_float(((meta >> 8) & 0xffu) << 23);
    const float sz = __uint_as_float(((meta >> 16) & 0xffu) << 23);
    const uint32_t r[4] = {(uint32_t)w2.z, (uint32_t)w2.w, (uint32_t)w3.x, (uint32_t)w3.y};
    const int nch = (int)(meta >> 24);
    float bd = INFINITY;
    uint32_t br = r[0];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const float lx = dequant((uint32_t)w1.x, c, sx, ox);
      const float ly = dequant((uint32_t)w1.y, c, sy, oy);
      const float lz = dequant((uint32_t)w1.z, c, sz, oz);
      const float hx = dequant((uint32_t)w1.w, c, sx, ox);
      const float hy = dequant((uint32_t)w2.x, c, sy, oy);
      const float hz = dequant((uint32_t)w2.y, c, sz, oz);
      const float d = c < nch ? box_dist_sq(px, py, pz, lx, ly, lz, hx, hy, hz) : INFINITY;
      if (d < bd) { bd = d; br = r[c]; }
    }
    ref = br;
  }
  const uint32_t f0 = leaf_first(ref), cnt = leaf_count(ref);
  dsq = INFINITY;
  tri = f0;
  for (uint32_t i = 0; i < cnt; ++i) {
    ++ctr.tris;
    const float d = tri_dist_sq(T.tri(f0 + i), px, py, pz);
    if (d < dsq) { dsq = d; tri = f0 + i; }
  }
}

// Each thread walks `chunk` consecutive Morton-sorted queries.  The pruning
// radius of a query starts just above its distance to the previous query's
// closest triangle (a greedy probe for the first one), so a valid triangle
// always lies inside it and the traversal returns exactly what an
// unbounded traversal returns: the nodes it skips all lie at or beyond a
// distance some tested triangle already beats or ties earlier in the same
// nearest-first order.  An external bound, when given, tightens the radius
// further; if it excludes every triangle the query is re-run unbounded.
template <bool kSign, bool kStats>
__global__ void __launch_bounds__(kUdfThreads)
    udf_kernel(TreeT<false> T, const float* __restrict__ pts,
               int64_t n, int chunk, const uint32_t* __restrict__ perm, const float* __restrict__ bound,
               QueryOut out, SignArgs sg, unsigned long long* stats, uint32_t* __restrict__ rerun,
               uint32_t* __restrict__ nrerun) {
  pdl_wait();
  __shared__ uint2 s_stack[kSharedDepth * kUdfThreads];
  __shared__ uint32_t s_next[kUdfThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  // each warp owns 32 * chunk consecutive (sorted) queries and hands them out
  // to its lanes as they finish, so fast lanes do not idle behind slow ones
  const int64_t w0 = ((int64_t)blockIdx.x * (kUdfThreads / 32) + warp) * 32 * chunk;
  const int64_t w1 = w0 + 32 * chunk < n ? w0 + 32 * chunk : n;
  if (lane == 0) s_next[warp] = 32;
  __syncwarp();
  Counters ctr{0, 0};
  uint32_t prev = 0xffffffffu;
  int64_t k = w0 + lane;
  while (k < w1) {
    const int64_t qi = perm ? (int64_t)perm[k] : k;
    const float px = pts[3 * qi], py = pts[3 * qi + 1], pz = pts[3 * qi + 2];
    uint32_t seed_tri;
    float seed_sq;
    if (prev != 0xffffffffu) {
      seed_tri = prev;
      ++ctr.tris;
      seed_sq = tri_dist_sq(T.tri(prev), px, py, pz);
    } else {
      probe(T, px, py, pz, seed_tri, seed_sq, ctr);
    }
    // strictly above the seed distance so the seed triangle itself qualifies
    float best_sq = seed_sq < INFINITY ? nextafterf(seed_sq, INFINITY) : INFINITY;
    if (bound) {
      const float b = bound[qi];
      const float bsq = b * b;
      if (bsq >= 0.f && bsq < best_sq) best_sq = bsq;
    }
    uint32_t best_tri = 0xffffffffu;
    SharedStack st{s_stack + threadIdx.x, 0};
    const bool ok = traverse(T, px, py, pz, st, best_sq, best_tri, ctr);
    if (!ok || best_tri == 0xffffffffu) {
      // stack overflow, or an external bound excluded every triangle
      const uint32_t slot = atomicAdd(nrerun, 1u);
      rerun[slot] = (uint32_t)qi;
      prev = 0xffffffffu;
    } else {
      finish_query(T.tris, T.num_tris, best_tri, best_sq, px, py, pz, qi, out, sg, kSign);
      prev = best_tri;
    }
    k = w0 + (int64_t)atomicAdd(&s_next[warp], 1u);
  }
  if (kStats) {
    __syncwarp();
    flush_counters(ctr, stats);
  }
}



template <typename Tree>
__device__ __forceinline__ void quad_child_box(const Tree& T, uint32_t ref, int c, float px,
                                               float py, float pz, float& d, uint32_t& r) {
  const int4* np = T.node(ref);
  const int4 w0 = __ldg(np), w1 = __ldg(np + 1), w2 = __ldg(np + 2), w3 = __ldg(np + 3);
  const uint32_t meta = (uint32_t)w0.w;
  const int nch = (int)(meta >> 24);
  const float sx = __uint_as_float((meta & 0xffu) << 23);
  const float sy = __uint_as_float(((meta >> 8) & 0xffu) << 23);
  const float sz = __uint_as_float(((meta >> 16) & 0xffu) << 23);
  const float ox = __int_as_float(w0.x), oy = __int_as_float(w0.y), oz = __int_as_float(w0.z);
  const float lx = dequant((uint32_t)w1.x, c, sx, ox);
  const float ly = dequant((uint32_t)w1.y, c, sy, oy);
  const float lz = dequant((uint32_t)w1.z, c, sz, oz);
  const float hx = dequant((uint32_t)w1.w, c, sx, ox);
  const float hy = dequant((uint32_t)w2.x, c, sy, oy);
  const float hz = dequant((uint32_t)w2.y, c, sz, oz);
  r = c == 0 ? (uint32_t)w2.z : (c == 1 ? (uint32_t)w2.w : (c == 2 ? (uint32_t)w3.x : (uint32_t)w3.y));
  d = c < nch ? box_dist_sq(px, py, pz, lx, ly, lz, hx, hy, hz) : INFINITY;
}

// ---------------------------------------------------------------------------
// warp task traversal
// ---------------------------------------------------------------------------
// Each lane owns one query (its point, best distance and a stack in shared
// memory).  Every round, each owner contributes the work of its current item:
// four child-box tests for an internal node, one triangle test per triangle
// of a leaf (or of the seed triangle).  The tasks of all 32 owners are packed
// into dense lists and evaluated by all lanes in lockstep, then each owner
// consumes its results: sorts the four children by (distance, ref) and
// pushes the qualifying ones, or folds its triangle distances in order with a
// strict "<".  The per-query visiting order is therefore the one of the
// single-lane traversal above and results are identical; only the lane that
// evaluates each test changes.
constexpr int kTaskWarps = 2;
constexpr int kTaskDepth = 32;
constexpr int kSpillCap = 96;    // per-owner global overflow stack (entries)
constexpr int kSpillChunk = 16;  // entries moved per spill / refill
// A spill happens when a node's q <= 4 qualifying children do not fit, i.e.
// with at least kTaskDepth - 2 entries on the stack, and moves a whole chunk:
// the stack must then hold a chunk.
static_assert(kTaskDepth - 2 >= kSpillChunk, "a spill needs a full chunk on the shared stack");
constexpr int kTaskTriCap = 32 * kMaxLeafTris;
constexpr int kTaskPool = 64;  // queries per pool taken from the global counter
// register cap of the task kernel: each of the SM's four sub-partitions
// holds 16K registers, so 64-thread blocks reach 8 resident blocks (16
// warps) at <= 128 registers a thread and 9 (18 warps, also the 24 KB
// shared-memory limit) at <= 96
#ifndef A3D_TASK_MAX_REGS
#define A3D_TASK_MAX_REGS 128
#endif
constexpr int kTaskMaxRegs = A3D_TASK_MAX_REGS;

// Per-warp shared state.  Child-box results sit at node rank * 5 + child and
// triangle results at position-in-leaf * 33 + owner, so that the owners'
// reads in the consume step fall in distinct banks.  Finished queries wait
// in fin_* and are written out 32 at a time by the whole warp.
constexpr int kBoxStride = 5;
constexpr int kTriRow = 33;
constexpr int kFinCap = 64;

struct TaskSmem {
  uint2 stack[kTaskDepth][32];
  float4 p[32];  // owners' query points (w unused): one 16-B read per task
  uint32_t nref[32];
  uint8_t nown[32];
  uint2 box[32 * kBoxStride];  // (distance bits, child ref) per child-box task
  uint32_t tidx[kTaskTriCap];
  uint8_t town[kTaskTriCap];  // owner lane | position in its leaf << 5
  float trid[kMaxLeafTris * kTriRow];
  uint32_t fin_q[kFinCap];
  uint32_t fin_tri[kFinCap];
  float fin_sq[kFinCap];
};

enum : int { kIdle = 0, kProbe = 1, kSeed = 2, kTrav = 3, kAbandon = 4 };
// radius seeding of the task kernel
enum : uint32_t { kSeedReuse = 1u, kSeedBoundOnly = 2u };

template <bool kSign, bool kStats, bool kBatch>
__global__ void __maxnreg__(kTaskMaxRegs)
    udf_task_kernel(TreeT<kBatch> T, const float* __restrict__ pts, int64_t n, const uint32_t* __restrict__ perm,
                    const float* __restrict__ bound, QueryOut out, SignArgs sg, unsigned long long* stats,
                    uint32_t* __restrict__ rerun, uint32_t* __restrict__ nrerun, uint32_t* __restrict__ pool_counter,
                    uint2* __restrict__ spill, int64_t spill_owners, uint32_t seeding, MeshSel sel, int pool) {
  pdl_wait();
  __shared__ TaskSmem smem[kTaskWarps];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  TaskSmem& S = smem[warp];
  const unsigned FULL = 0xffffffffu;
  const unsigned lt_mask = (1u << lane) - 1u;
  // persistent warps: pools of kTaskPool consecutive (sorted) queries are
  // taken from a global counter; inside a pool, lanes take queries as they
  // finish their previous one
  int64_t pos = 0, end = 0;
  bool exhausted = false;
  Counters ctr{0, 0};

  // owner state
  int64_t qi = -1, kprev = -(1ll << 40);
  int phase = kIdle;
  uint32_t ref = 0, prev = 0xffffffffu, best_tri = 0xffffffffu, root = 0u, prev_root = 0u;
  float best_sq = INFINITY, px = 0.f, py = 0.f, pz = 0.f, bsq = INFINITY;
  bool have = false;
  bool reused = false;  // the query's radius is seeded by the previous query's triangle
  int sp = 0;
  // overflow stack in global memory (the workspace's spill region), used
  // when the shared stack is full; owners beyond the region have none
  const int64_t owner = ((int64_t)blockIdx.x * kTaskWarps + warp) * 32 + lane;
  uint2* my_spill = (spill != nullptr && owner < spill_owners) ? spill + owner * kSpillCap : nullptr;
  int gsp = 0;
  int nfin = 0;  // finished queries waiting in S.fin_* (warp-uniform)
  unsigned long long rounds = 0;

  // writes out finished query e of S.fin_*
  auto finish_entry = [&](int e) {
    const int64_t q = (int64_t)S.fin_q[e];
    finish_query(T.tris, T.num_tris, S.fin_tri[e], S.fin_sq[e], pts[3 * q], pts[3 * q + 1], pts[3 * q + 2], q, out,
                 sg, kSign);
  };

  auto start = [&](int64_t k) {
    qi = perm ? (int64_t)perm[k] : k;
    root = kBatch ? sel.root_of(qi) : 0u;
    px = pts[3 * qi]; py = pts[3 * qi + 1]; pz = pts[3 * qi + 2];
    S.p[lane] = make_float4(px, py, pz, 0.f);
    bsq = INFINITY;
    if (bound) {
      const float b = bound[qi];
      if (b * b >= 0.f) bsq = b * b;
    }
    best_sq = INFINITY;
    best_tri = 0xffffffffu;
    sp = 0;
    gsp = 0;
    // a finite caller bound alone seeds the radius when asked to (no probe
    // descent); else the previous result seeds it for a nearby query in the
    // sorted order; otherwise a greedy probe does
    reused = false;
    if ((seeding & kSeedBoundOnly) && bsq < INFINITY) {
      best_sq = bsq;
      phase = kTrav;
      ref = root;
      have = true;
    } else if ((seeding & kSeedReuse) && prev != 0xffffffffu && (!kBatch || root == prev_root) &&
               k - kprev <= 64 && k > kprev) {
      phase = kSeed;
      reused = true;
    } else {
      prev = 0xffffffffu;
      phase = kProbe;
      ref = root;
      have = true;
    }
    kprev = k;
    if (kBatch) prev_root = root;
  };

  // hands new queries to the lanes in `want` (warp-uniform bookkeeping)
  auto distribute = [&](unsigned want) {
    while (want) {
      if (pos >= end) {
        if (exhausted) break;
        uint32_t p = 0;
        if (lane == 0) p = atomicAdd(pool_counter, 1u);
        p = __shfl_sync(FULL, p, 0);
        const int psize = kBatch ? pool : kTaskPool;
        pos = (int64_t)p * psize;
        end = pos + psize < n ? pos + psize : n;
        if (pos >= n) { exhausted = true; break; }
      }
      const int64_t avail = end - pos;
      const int cnt = __popc(want);
      const int take = (int)(avail < cnt ? avail : cnt);
      const int rank = __popc(want & lt_mask);
      const bool mine = ((want >> lane) & 1u) && rank < take;
      if (mine) start(pos + rank);
      pos += take;
      want &= ~__ballot_sync(FULL, mine);
    }
  };
  distribute(FULL);

  while (__any_sync(FULL, phase != kIdle)) {
    ++rounds;
    // (a) traversing owners without an item pop; finished owners emit and refetch
    bool done = false;
    if (phase == kTrav && !have) {
      for (;;) {
        while (sp > 0) {
          --sp;
          const uint2 e = S.stack[sp][lane];
          if (__uint_as_float(e.y) < best_sq) { ref = e.x; have = true; break; }
        }
        if (have || gsp == 0) break;
        // shared stack empty: bring back the most recently spilled chunk
        const int k = gsp < kSpillChunk ? gsp : kSpillChunk;
        gsp -= k;
        for (int i = 0; i < k; ++i) S.stack[i][lane] = my_spill[gsp + i];
        sp = k;
      }
      done = !have;
    }
    if (done && best_tri == 0xffffffffu && bsq < INFINITY) {
      // the caller's bound excluded every triangle: run the query again in
      // place, unbounded, seeded as the plain method seeds it (the previous
      // query's triangle when that seeded it, else a greedy probe), instead
      // of handing it to the deep-stack re-run kernel
      bsq = INFINITY;
      best_sq = INFINITY;
      sp = 0;
      gsp = 0;
      if (reused) {
        phase = kSeed;
        have = false;
      } else {
        phase = kProbe;
        ref = root;
        have = true;
      }
      done = false;
    }
    if (phase == kAbandon) done = true;
    const bool found = done && phase != kAbandon && best_tri != 0xffffffffu;
    if (done && !found) {
      rerun[atomicAdd(nrerun, 1u)] = (uint32_t)qi;
      prev = 0xffffffffu;
    }
    {
      // queue the finished queries; once 32 wait, every lane writes one out
      const unsigned fmask = __ballot_sync(FULL, found);
      if (found) {
        const int at = nfin + __popc(fmask & lt_mask);
        S.fin_q[at] = (uint32_t)qi;
        S.fin_tri[at] = best_tri;
        S.fin_sq[at] = best_sq;
        prev = best_tri;
      }
      nfin += __popc(fmask);
      if (nfin >= 32) {
        __syncwarp();
        finish_entry(nfin - 32 + lane);
        nfin -= 32;
        __syncwarp();
      }
    }
    if (done) phase = kIdle;
    distribute(__ballot_sync(FULL, done));
    // (b) classify this round's item
    const bool is_node = (phase == kProbe || phase == kTrav) && have && !ref_is_leaf(ref);
    const bool is_leaf = (phase == kProbe || phase == kTrav) && have && ref_is_leaf(ref);
    const bool is_seed = phase == kSeed;
    const unsigned nmask = __ballot_sync(FULL, is_node);
    const int nrank = __popc(nmask & lt_mask);
    const int nnodes = __popc(nmask);
    if (is_node) {
      S.nref[nrank] = ref;
      S.nown[nrank] = (uint8_t)lane;
      if (kStats) ++ctr.nodes;
    }
    const int tcnt = is_leaf ? (int)leaf_count(ref) : (is_seed ? 1 : 0);
    int toff = tcnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int v = __shfl_up_sync(FULL, toff, o);
      if (lane >= o) toff += v;
    }
    const int ttotal = __shfl_sync(FULL, toff, 31);
    toff -= tcnt;
    const uint32_t f0 = is_seed ? prev : leaf_first(ref);
    if (tcnt > 0) {
      for (int i = 0; i < tcnt; ++i) {
        S.tidx[toff + i] = f0 + i;
        S.town[toff + i] = (uint8_t)(lane | (i << 5));
      }
      if (kStats) ctr.tris += tcnt;
    }
    __syncwarp();
    // (c) dense evaluation: child boxes, then triangles
    for (int t = lane; t < 4 * nnodes; t += 32) {
      const int r = t >> 2, c = t & 3;
      const int o = S.nown[r];
      float d;
      uint32_t cr;
      const float4 q = S.p[o];
      quad_child_box(T, S.nref[r], c, q.x, q.y, q.z, d, cr);
      S.box[r * kBoxStride + c] = make_uint2(__float_as_uint(d), cr);
    }
    for (int t = lane; t < ttotal; t += 32) {
      const uint32_t op = S.town[t];
      const int o = (int)(op & 31u);
      const float4 q = S.p[o];
      S.trid[(op >> 5) * kTriRow + o] = tri_dist_sq(T.tri(S.tidx[t]), q.x, q.y, q.z);
    }
    __syncwarp();
    // (d) owners consume their results
    if (is_node) {
      float d[4];
      uint32_t r[4];
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        const uint2 e = S.box[kBoxStride * nrank + c];
        d[c] = __uint_as_float(e.x);
        r[c] = e.y;
      }
      if (phase == kProbe) {
        // greedy: the (distance, ref)-smallest child
        float bd = d[0];
        uint32_t br = r[0];
#pragma unroll
        for (int c = 1; c < 4; ++c)
          if (child_less(d[c], r[c], bd, br)) { bd = d[c]; br = r[c]; }
        ref = br;
      } else {
        cswap(d[0], r[0], d[1], r[1]);
        cswap(d[2], r[2], d[3], r[3]);
        cswap(d[0], r[0], d[2], r[2]);
        cswap(d[1], r[1], d[3], r[3]);
        cswap(d[1], r[1], d[2], r[2]);
        int q = 0;
#pragma unroll
        for (int c = 0; c < 4; ++c) q += d[c] < best_sq ? 1 : 0;
        if (q > 0) {
          if (sp + (q - 1) > kTaskDepth && my_spill != nullptr && gsp + kSpillChunk <= kSpillCap) {
            // move the oldest entries (visited last) to the global overflow stack
            for (int i = 0; i < kSpillChunk; ++i) my_spill[gsp + i] = S.stack[i][lane];
            for (int i = kSpillChunk; i < sp; ++i) S.stack[i - kSpillChunk][lane] = S.stack[i][lane];
            gsp += kSpillChunk;
            sp -= kSpillChunk;
          }
          if (sp + (q - 1) > kTaskDepth) {
            // still no room: the deep-stack kernel re-runs the query
            phase = kAbandon;
            have = false;
          } else {
#pragma unroll
            for (int c = 3; c >= 1; --c)
              if (c < q) S.stack[sp++][lane] = make_uint2(r[c], __float_as_uint(d[c]));
            ref = r[0];
          }
        } else {
          have = false;
        }
      }
    } else if (is_leaf || is_seed) {
      float dmin = INFINITY;
      uint32_t imin = 0xffffffffu;
      for (int i = 0; i < tcnt; ++i) {
        const float dd = S.trid[i * kTriRow + lane];
        if (dd < dmin) { dmin = dd; imin = f0 + (uint32_t)i; }
      }
      if (phase == kTrav) {
        if (dmin < best_sq) { best_sq = dmin; best_tri = imin; }
        have = false;
      } else {
        // probe leaf or seed triangle: radius just above its distance
        float b = dmin < INFINITY ? nextafterf(dmin, INFINITY) : INFINITY;
        if (bsq < b) b = bsq;
        best_sq = b;
        phase = kTrav;
        ref = root;
        have = true;
      }
    }
    __syncwarp();
  }
  // queries still waiting to be written out
  __syncwarp();
  if (lane < nfin) finish_entry(lane);
  if (kStats) {
    flush_counters(ctr, stats);
    if (lane == 0) atomicAdd(stats + 3, rounds);
  }
}


template <bool kSign, bool kStats, bool kBatch>
__global__ void __launch_bounds__(64)
    udf_rerun_kernel(TreeT<kBatch> T, const float* __restrict__ pts, const uint32_t* __restrict__ rerun,
                     const uint32_t* __restrict__ nrerun, QueryOut out, SignArgs sg, unsigned long long* stats,
                     uint32_t* __restrict__ overflow, uint32_t* __restrict__ total_reruns, MeshSel sel) {
  pdl_wait();
  const uint32_t m = *nrerun;
  if (blockIdx.x == 0 && threadIdx.x == 0 && m > 0) atomicAdd(total_reruns, m);
  Counters ctr{0, 0};
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < m; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t qi = rerun[t];
    const float px = pts[3 * qi], py = pts[3 * qi + 1], pz = pts[3 * qi + 2];
    uint32_t seed_tri;
    float seed_sq;
    const uint32_t root = kBatch ? sel.root_of(qi) : 0u;
    probe(T, px, py, pz, seed_tri, seed_sq, ctr, root);
    float best_sq = seed_sq < INFINITY ? nextafterf(seed_sq, INFINITY) : INFINITY;
    uint32_t best_tri = 0xffffffffu;
    LocalStack st;
    st.sp = 0;
    if (!traverse(T, px, py, pz, st, best_sq, best_tri, ctr, root)) atomicExch(overflow, 1u);
    finish_query(T.tris, T.num_tris, best_tri, best_sq, px, py, pz, qi, out, sg, kSign);
  }
  if (kStats && (ctr.nodes | ctr.tris)) {
    atomicAdd(stats, ctr.nodes);
    atomicAdd(stats + 1, ctr.tris);
  }
}

__global__ void query_morton_kernel(const float* __restrict__ pts, int64_t n, float lox, float loy, float loz,
                                    float ix, float iy, float iz, uint32_t* __restrict__ keys,
                                    uint32_t* __restrict__ vals) {
  pdl_wait();
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float q[3] = {(pts[3 * i] - lox) * ix, (pts[3 * i + 1] - loy) * iy, (pts[3 * i + 2] - loz) * iz};
  uint32_t code = 0;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    float t = fminf(fmaxf(q[a], 0.f), 1023.f);
    if (!(t == t)) t = 0.f;
    code |= (uint32_t)spread3_21((uint64_t)t) << a;
  }
  keys[i] = code;
  vals[i] = (uint32_t)i;
}

constexpr int kStatusWords = 8;

struct UdfWs {
  uint32_t* keys;
  uint32_t* keys_alt;
  uint32_t* vals;
  uint32_t* vals_alt;
  uint32_t* rs_scratch;
  uint32_t* rerun;
  uint32_t* nrerun;  // status words: [0] re-run list length, [1] deep-stack overflow, [2] pool counter,
                     // [3] guard faults, [4] queries re-run in total
  uint2* spill;      // optional overflow stacks (trailing workspace)
  int64_t spill_owners;
};

size_t carve_udf(UdfWs& w, Workspace& ws, int64_t n, uint32_t flags) {
  // status words at the start of the workspace (read by a3d_udf_status)
  w.nrerun = ws.take<uint32_t>(kStatusWords);
  if (flags & A3D_UDF_SORT_QUERIES) {
    w.keys = ws.take<uint32_t>(n);
    w.keys_alt = ws.take<uint32_t>(n);
    w.vals = ws.take<uint32_t>(n);
    w.vals_alt = ws.take<uint32_t>(n);
    w.rs_scratch = ws.take<uint32_t>((int64_t)radix_sort_scratch_elems(n));
  } else {
    w.keys = w.keys_alt = w.vals = w.vals_alt = w.rs_scratch = nullptr;
  }
  w.rerun = ws.take<uint32_t>(n);
  return ws.used;
}

// owners of the persistent traversal that get an overflow stack when the
// workspace has room for it (bounded: 148 SMs x 10 blocks x 64 lanes)
int64_t spill_owner_bound(int64_t n) {
  const int64_t cap = (int64_t)148 * 10 * 64;  // overflow stacks for the resident owners of a 148-SM part
  return n + 128 < cap ? n + 128 : cap;
}

// launch shape of the persistent traversal: queries per pool, resident
// blocks per SM (0 = as many as fit)
struct TaskShape {
  int pool;
  int blocks_per_sm;
};

template <bool kSign, bool kStats, bool kBatch>
int task_blocks_per_sm(int* out) {
  // per device: a process may drive GPUs of different kinds
  static int cached[kMaxDevices] = {0};
  int dev = 0;
  A3D_CUDA_TRY(cudaGetDevice(&dev));
  if (dev >= 0 && dev < kMaxDevices && cached[dev] > 0) {
    *out = cached[dev];
    return A3D_OK;
  }
  int b = 0;
  A3D_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, udf_task_kernel<kSign, kStats, kBatch>,
                                                             kTaskWarps * 32, 0));
  b = b < 1 ? 1 : b;
  if (dev >= 0 && dev < kMaxDevices) cached[dev] = b;
  *out = b;
  return A3D_OK;
}

template <bool kSign, bool kStats, bool kBatch>
int launch_udf(const TreeT<kBatch>& T, const float* pts, int64_t n, const uint32_t* perm, bool coherent,
               const float* bound, const QueryOut& out, const SignArgs& sg, unsigned long long* stats, UdfWs& w,
               uint32_t seeding, const MeshSel& sel, TaskShape shape, cudaStream_t s) {
  if (coherent) {
    int bps = 0;
    A3D_TRY((task_blocks_per_sm<kSign, kStats, kBatch>(&bps)));
    if (shape.blocks_per_sm > 0 && shape.blocks_per_sm < bps) bps = shape.blocks_per_sm;
    const int pool = shape.pool > 0 ? shape.pool : kTaskPool;
    const int sms = num_sms();
    const int64_t pools = ceil_div(n, pool);
    const int64_t want_blocks = ceil_div(pools, kTaskWarps);
    const int64_t grid = want_blocks < (int64_t)sms * bps ? want_blocks : (int64_t)sms * bps;
    A3D_PDL((udf_task_kernel<kSign, kStats, kBatch>), dim3((unsigned)grid), dim3(kTaskWarps * 32), 0, s, T, pts, n,
            perm, bound, out, sg, stats, w.rerun, w.nrerun, w.nrerun + 2, w.spill, w.spill_owners, seeding, sel, pool);
  } else {
    if constexpr (!kBatch) {
      A3D_PDL((udf_kernel<kSign, kStats>), dim3((unsigned)ceil_div(n, kUdfThreads)), dim3(kUdfThreads), 0, s, T, pts, n,
              1, perm, bound, out, sg, stats, w.rerun, w.nrerun);
    } else {
      A3D_REQUIRE(false, A3D_ERR_ARGUMENT, "udf: batches are always sorted");
    }
  }
  A3D_LAUNCH_CHECK();
  // the re-run list length is only known on the device: launch enough
  // threads for a few percent of the queries, each thread strides
  const int64_t rr_min = (int64_t)num_sms() * 256;
  const int64_t rr_threads = n / 16 > rr_min ? n / 16 : rr_min;
  A3D_PDL((udf_rerun_kernel<kSign, kStats, kBatch>), dim3((unsigned)ceil_div(rr_threads, 64)), dim3(64), 0, s, T, pts,
          w.rerun, w.nrerun, out, sg, stats, w.nrerun + 1, w.nrerun + 4, sel);
  return A3D_OK;
}

// ---------------------------------------------------------------------------
// adjoints
// ---------------------------------------------------------------------------
__global__ void udf_backward_kernel(const float* __restrict__ pts, int64_t n, const float* __restrict__ cp,
                                    const int32_t* __restrict__ fid, const float* __restrict__ uvw,
                                    const float* __restrict__ gd, const int32_t* __restrict__ faces,
                                    float* __restrict__ gp, float* __restrict__ gv) {
  pdl_wait();
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float dx = pts[3 * i] - cp[3 * i], dy = pts[3 * i + 1] - cp[3 * i + 1], dz = pts[3 * i + 2] - cp[3 * i + 2];
  const float d = sqrtf(dx * dx + dy * dy + dz * dz);
  const float g = gd[i];
  // d|p-c|/dp = (p-c)/|p-c| (zero at the surface, like norm's subgradient)
  const float inv = d > 0.f ? g / d : 0.f;
  const float gx = dx * inv, gy = dy * inv, gz = dz * inv;
  if (gp) {
    gp[3 * i] = gx;
    gp[3 * i + 1] = gy;
    gp[3 * i + 2] = gz;
  }
  const int32_t f = fid[i];
  if (gv && f >= 0 && uvw) {
    // closest-point barycentrics clamped to the simplex (they are exact
    // for the closest point up to rounding)
    float w0 = fmaxf(uvw[3 * i], 0.f), w1 = fmaxf(uvw[3 * i + 1], 0.f), w2 = fmaxf(uvw[3 * i + 2], 0.f);
    const float sw = w0 + w1 + w2;
    if (sw > 0.f) { w0 /= sw; w1 /= sw; w2 /= sw; }
    const float ws[3] = {w0, w1, w2};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const int64_t v = faces[3 * (int64_t)f + k];
      atomicAdd(&gv[3 * v], -ws[k] * gx);
      atomicAdd(&gv[3 * v + 1], -ws[k] * gy);
      atomicAdd(&gv[3 * v + 2], -ws[k] * gz);
    }
  }
}

}  // namespace

}  // namespace a3d

using namespace a3d;

namespace a3d {
// Workspace a3d_udf needs at least (without the optional overflow stacks).
size_t udf_required_workspace_bytes(int64_t num_points, uint32_t flags) {
  Workspace ws(nullptr, 0);
  UdfWs w;
  return carve_udf(w, ws, num_points > 0 ? num_points : 1, flags) + 256;
}
}  // namespace a3d

extern "C" size_t a3d_udf_workspace_bytes(int64_t num_points, uint32_t flags) {
  Workspace ws(nullptr, 0);
  UdfWs w;
  const int64_t n = num_points > 0 ? num_points : 1;
  const size_t base = carve_udf(w, ws, n, flags);
  return base + (size_t)spill_owner_bound(n) * kSpillCap * sizeof(uint2) + 512;
}

extern "C" int a3d_udf(const a3d_bvh_view* bvh, const float* points, int64_t num_points, float* distances,
                       int32_t* face_ids, float* closest_points, float* uvw, const a3d_sign_data* sign,
                       const float* bound, unsigned long long* stats, uint32_t flags, void* workspace,
                       size_t workspace_bytes, a3d_stream_t stream_) {
  cudaStream_t s = (cudaStream_t)stream_;
  A3D_REQUIRE(bvh && bvh->nodes && bvh->tris && bvh->num_nodes > 0, A3D_ERR_ARGUMENT, "udf: invalid bvh");
  A3D_REQUIRE(num_points >= 0 && num_points < (1ll << 32), A3D_ERR_ARGUMENT, "udf: bad number of points");
  if (num_points == 0) return A3D_OK;
  A3D_REQUIRE(points && distances && face_ids && closest_points, A3D_ERR_ARGUMENT, "udf: null output");
  if (sign) {
    A3D_REQUIRE(sign->face_normals && sign->faces, A3D_ERR_ARGUMENT, "udf: sign data needs face normals and faces");
    const bool all = sign->vertex_pn && sign->edge_pn && sign->he_edge_idx;
    const bool none = !sign->vertex_pn && !sign->edge_pn && !sign->he_edge_idx;
    A3D_REQUIRE(all || none, A3D_ERR_ARGUMENT, "udf: pseudo-normal data must be all present or all absent");
  }
  Workspace ws(workspace, workspace_bytes);
  UdfWs w;
  carve_udf(w, ws, num_points, flags);
  A3D_REQUIRE(workspace && ws.ok(), A3D_ERR_WORKSPACE, "udf: workspace too small");
  // whatever trails the required part holds per-owner overflow stacks
  {
    const uintptr_t base = ((uintptr_t)workspace + ws.used + 255) & ~(uintptr_t)255;
    const uintptr_t endp = (uintptr_t)workspace + workspace_bytes;
    const int64_t owners = base < endp ? (int64_t)((endp - base) / (kSpillCap * sizeof(uint2))) : 0;
    w.spill = owners > 0 ? (uint2*)base : nullptr;
    w.spill_owners = owners;
  }
  const int64_t n = num_points;
  const uint32_t* perm = nullptr;
  if (flags & A3D_UDF_SORT_QUERIES) {
    const float ext[3] = {bvh->hi[0] - bvh->lo[0], bvh->hi[1] - bvh->lo[1], bvh->hi[2] - bvh->lo[2]};
    float emax = fmaxf(ext[0], fmaxf(ext[1], ext[2]));
    emax = emax > 0.f ? emax : 1.f;
    // queries may lie outside the mesh box: use a cube of twice its extent
    const float lo[3] = {0.5f * (bvh->lo[0] + bvh->hi[0]) - emax, 0.5f * (bvh->lo[1] + bvh->hi[1]) - emax,
                         0.5f * (bvh->lo[2] + bvh->hi[2]) - emax};
    const float inv = 1023.0f / (2.0f * emax);
    A3D_PDL(query_morton_kernel, dim3((unsigned)ceil_div(n, 256)), dim3(256), 0, s, points, n, lo[0], lo[1], lo[2], inv,
            inv, inv, w.keys, w.vals);
    bool alt = false;
    A3D_TRY(radix_sort_pairs<uint32_t>(w.keys, w.vals, w.keys_alt, w.vals_alt, n, 0, 32, w.rs_scratch, &alt, s));
    perm = alt ? w.vals_alt : w.vals;
  }
  const bool coherent = perm != nullptr || (flags & A3D_UDF_ASSUME_SORTED) != 0;
  const uint32_t seeding = ((flags & A3D_UDF_NO_REUSE) ? 0u : kSeedReuse) |
                           ((flags & A3D_UDF_BOUND_SEEDS) && bound ? kSeedBoundOnly : 0u);
  A3D_CUDA_TRY(cudaMemsetAsync(w.nrerun, 0, kStatusWords * sizeof(uint32_t), s));
  const TreeT<false> T{(const WideNode*)bvh->nodes, (const TriRec*)bvh->tris, (uint32_t)bvh->num_nodes,
                       (uint32_t)bvh->num_tris, w.nrerun + 3};
  const MeshSel sel{nullptr, nullptr, 1, 0};
  const TaskShape shape{kTaskPool, 0};
  QueryOut out{distances, face_ids, closest_points, uvw};
  SignArgs sg{nullptr, nullptr, nullptr, nullptr, nullptr};
  if (sign) {
    const bool pn = sign->edge_pn != nullptr;
    sg = SignArgs{sign->face_normals, pn ? sign->vertex_pn : nullptr, pn ? sign->edge_pn : nullptr,
                  pn ? sign->he_edge_idx : nullptr, sign->faces};
  }
  if (sign) {
    if (stats) A3D_TRY((launch_udf<true, true, false>(T, points, n, perm, coherent, bound, out, sg, stats, w, seeding, sel, shape, s)));
    else A3D_TRY((launch_udf<true, false, false>(T, points, n, perm, coherent, bound, out, sg, stats, w, seeding, sel, shape, s)));
  } else {
    if (stats) A3D_TRY((launch_udf<false, true, false>(T, points, n, perm, coherent, bound, out, sg, stats, w, seeding, sel, shape, s)));
    else A3D_TRY((launch_udf<false, false, false>(T, points, n, perm, coherent, bound, out, sg, stats, w, seeding, sel, shape, s)));
  }
  if (stats) {
    // reruns are reported as bound misses / spills (same counter: re-run queries)
    A3D_CUDA_TRY(cudaMemcpyAsync(stats + 2, w.nrerun + 4, sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
  }
  return A3D_OK;
}

extern "C" int a3d_udf_backward(const float* points, int64_t num_points, const float* closest_points,
                                const int32_t* face_ids, const float* uvw, const float* grad_dist,
                                const int32_t* faces, float* grad_points, float* grad_vertices,
                                a3d_stream_t stream_) {
  cudaStream_t s = (cudaStream_t)stream_;
  A3D_REQUIRE(num_points >= 0, A3D_ERR_ARGUMENT, "udf_backward: bad size");
  if (num_points == 0) return A3D_OK;
  A3D_REQUIRE(points && closest_points && grad_dist, A3D_ERR_ARGUMENT, "udf_backward: null input");
  A3D_REQUIRE(!grad_vertices || (face_ids && uvw && faces), A3D_ERR_ARGUMENT,
              "udf_backward: vertex adjoint needs face ids, uvw and faces");
  A3D_PDL(udf_backward_kernel, dim3((unsigned)ceil_div(num_points, 256)), dim3(256), 0, s, points, num_points,
          closest_points, face_ids, uvw, grad_dist, faces, grad_points, grad_vertices);
  return A3D_OK;
}

// ---------------------------------------------------------------------------
// batches of meshes: one sort and one persistent traversal per chunk of
// queries, all meshes together
// ---------------------------------------------------------------------------
namespace a3d {
namespace {

// queries per traversal launch of a batch (bounds the scratch: ~380 MB)
constexpr int64_t kBatchChunk = 1ll << 24;

__device__ __forceinline__ int segment_of64(const int64_t* __restrict__ off, int nseg, int64_t i) {
  int lo = 0, hi = nseg - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (off[mid] <= i) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// key = mesh id above the Morton code of the query in a cube of twice its
// mesh's extent about the mesh centre; i is local to the chunk at qbase
__global__ void batch_query_morton_kernel(const float* __restrict__ pts, int64_t n, int64_t qbase,
                                          const int64_t* __restrict__ qoff, int nmesh,
                                          const float* __restrict__ bounds, int bits, uint32_t* __restrict__ keys,
                                          uint32_t* __restrict__ vals) {
  pdl_wait();
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int m = segment_of64(qoff, nmesh, qbase + i);
  const float* b = bounds + 6 * (int64_t)m;
  float emax = fmaxf(b[3] - b[0], fmaxf(b[4] - b[1], b[5] - b[2]));
  emax = emax > 0.f ? emax : 1.f;
  const float qmax = (float)((1u << bits) - 1u);
  const float inv = qmax / (2.0f * emax);
  const float q[3] = {(pts[3 * i] - (0.5f * (b[0] + b[3]) - emax)) * inv,
                      (pts[3 * i + 1] - (0.5f * (b[1] + b[4]) - emax)) * inv,
                      (pts[3 * i + 2] - (0.5f * (b[2] + b[5]) - emax)) * inv};
  uint32_t code = 0;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    float t = fminf(fmaxf(q[a], 0.f), qmax);
    if (!(t == t)) t = 0.f;
    code |= (uint32_t)spread3_21((uint64_t)t) << a;
  }
  keys[i] = ((uint32_t)m << (3 * bits)) | code;
  vals[i] = (uint32_t)i;
}

int mesh_bits(int nmesh) {
  int mbits = 0;
  while ((1ll << mbits) < nmesh) ++mbits;
  return mbits;
}

size_t batch_udf_bytes(int64_t n) {
  const int64_t c = n < kBatchChunk ? (n > 0 ? n : 1) : kBatchChunk;
  Workspace ws(nullptr, 0);
  UdfWs w;
  const size_t base = carve_udf(w, ws, c, A3D_UDF_SORT_QUERIES);
  return base + (size_t)spill_owner_bound(c) * kSpillCap * sizeof(uint2) + 512;
}

int batch_udf(const a3d_bvh_batch* bvh, const float* points, const int64_t* qoff, int64_t n, float* distances,
              int32_t* face_ids, float* closest_points, float* uvw, TaskShape shape, unsigned long long* stats,
              void* workspace, size_t workspace_bytes, cudaStream_t s) {
  A3D_REQUIRE(bvh && bvh->nodes && bvh->tris && bvh->roots && bvh->bounds && bvh->num_meshes > 0 &&
                  bvh->num_faces > 0 && bvh->num_faces < (1ll << 28),
              A3D_ERR_ARGUMENT, "batch_udf: invalid batch");
  A3D_REQUIRE(n >= 0 && n < (1ll << 40), A3D_ERR_ARGUMENT, "batch_udf: bad number of queries");
  A3D_REQUIRE(workspace, A3D_ERR_WORKSPACE, "batch_udf: no workspace");
  const int mbits = mesh_bits(bvh->num_meshes);
  A3D_REQUIRE(mbits <= 26, A3D_ERR_ARGUMENT, "batch_udf: too many meshes");
  int bits = (32 - mbits) / 3;
  bits = bits < 10 ? bits : 10;
  const int64_t c = n < kBatchChunk ? (n > 0 ? n : 1) : kBatchChunk;
  Workspace ws(workspace, workspace_bytes);
  UdfWs w;
  carve_udf(w, ws, c, A3D_UDF_SORT_QUERIES);
  A3D_REQUIRE(ws.ok(), A3D_ERR_WORKSPACE, "batch_udf: workspace too small");
  {
    const uintptr_t base = ((uintptr_t)workspace + ws.used + 255) & ~(uintptr_t)255;
    const uintptr_t endp = (uintptr_t)workspace + workspace_bytes;
    const int64_t owners = base < endp ? (int64_t)((endp - base) / (kSpillCap * sizeof(uint2))) : 0;
    w.spill = owners > 0 ? (uint2*)base : nullptr;
    w.spill_owners = owners;
  }
  A3D_CUDA_TRY(cudaMemsetAsync(w.nrerun, 0, kStatusWords * sizeof(uint32_t), s));
  if (n == 0) return A3D_OK;
  A3D_REQUIRE(points && qoff && distances && face_ids && closest_points, A3D_ERR_ARGUMENT, "batch_udf: null pointer");
  // the node count is only known on the device: guard with the capacity
  const TreeT<true> T{(const WideNode*)bvh->nodes, (const TriRec*)bvh->tris, (uint32_t)bvh->num_faces,
                      (uint32_t)bvh->num_faces, w.nrerun + 3};
  const SignArgs sg{nullptr, nullptr, nullptr, nullptr, nullptr};
  for (int64_t base = 0; base < n; base += kBatchChunk) {
    const int64_t cn = n - base < kBatchChunk ? n - base : kBatchChunk;
    const float* pts = points + 3 * base;
    A3D_PDL(batch_query_morton_kernel, dim3((unsigned)ceil_div(cn, 256)), dim3(256), 0, s, pts, cn, base, qoff,
            bvh->num_meshes, bvh->bounds, bits, w.keys, w.vals);
    bool alt = false;
    A3D_TRY(radix_sort_pairs<uint32_t>(w.keys, w.vals, w.keys_alt, w.vals_alt, cn, 0, 3 * bits + mbits,
                                       w.rs_scratch, &alt, s));
    const uint32_t* perm = alt ? w.vals_alt : w.vals;
    // per chunk: the re-run list and the pool counter start at zero
    A3D_CUDA_TRY(cudaMemsetAsync(w.nrerun, 0, sizeof(uint32_t), s));
    A3D_CUDA_TRY(cudaMemsetAsync(w.nrerun + 2, 0, sizeof(uint32_t), s));
    const QueryOut out{distances + base, face_ids + base, closest_points + 3 * base, uvw ? uvw + 3 * base : nullptr};
    const MeshSel sel{qoff, bvh->roots, bvh->num_meshes, base};
    if (stats)
      A3D_TRY((launch_udf<false, true, true>(T, pts, cn, perm, true, nullptr, out, sg, stats, w, kSeedReuse, sel,
                                             shape, s)));
    else
      A3D_TRY((launch_udf<false, false, true>(T, pts, cn, perm, true, nullptr, out, sg, stats, w, kSeedReuse, sel,
                                              shape, s)));
  }
  if (stats) A3D_CUDA_TRY(cudaMemcpyAsync(stats + 2, w.nrerun + 4, sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
  return A3D_OK;
}

// every stride-th query, with the offsets of the sample per mesh
__global__ void sample_queries_kernel(const float* __restrict__ pts, int64_t stride, const int64_t* __restrict__ qoff,
                                      int nmesh, float* __restrict__ spts, int64_t ns, int64_t* __restrict__ sqoff) {
  pdl_wait();
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < ns) {
    const int64_t j = i * stride;
    spts[3 * i] = pts[3 * j];
    spts[3 * i + 1] = pts[3 * j + 1];
    spts[3 * i + 2] = pts[3 * j + 2];
  }
  if (i <= nmesh) sqoff[i] = (qoff[i] + stride - 1) / stride;  // first sample at or after qoff[i]
}

struct TuneWs {
  float* pts;
  int64_t* qoff;
  float* dist;
  int32_t* fid;
  float* cp;
  void* udf_ws;
  size_t udf_bytes;
};

size_t carve_tune(TuneWs& t, Workspace& ws, int64_t ns, int nmesh) {
  t.pts = ws.take<float>(3 * ns);
  t.qoff = ws.take<int64_t>(nmesh + 1);
  t.dist = ws.take<float>(ns);
  t.fid = ws.take<int32_t>(ns);
  t.cp = ws.take<float>(3 * ns);
  t.udf_bytes = batch_udf_bytes(ns);
  t.udf_ws = ws.take<unsigned char>((int64_t)t.udf_bytes);
  return ws.used;
}

}  // namespace
}  // namespace a3d

extern "C" int a3d_udf_status(const void* workspace, uint32_t* status_out, a3d_stream_t stream) {
  A3D_REQUIRE(workspace && status_out, A3D_ERR_ARGUMENT, "udf_status: null pointer");
  uint32_t w[a3d::kStatusWords];
  A3D_CUDA_TRY(cudaMemcpyAsync(w, workspace, sizeof(w), cudaMemcpyDeviceToHost, (cudaStream_t)stream));
  A3D_CUDA_TRY(cudaStreamSynchronize((cudaStream_t)stream));
  status_out[0] = w[4];  // queries re-run by the deep-stack kernel
  status_out[1] = w[1];  // deep-stack overflow
  status_out[2] = 0u;
  status_out[3] = w[3];  // guard faults
  return A3D_OK;
}

extern "C" size_t a3d_batch_udf_workspace_bytes(int64_t num_queries, int32_t num_meshes) {
  (void)num_meshes;
  return a3d::batch_udf_bytes(num_queries);
}

extern "C" int a3d_batch_udf(const a3d_bvh_batch* bvh, const float* points, const int64_t* query_offsets,
                             int64_t num_queries, float* distances, int32_t* face_ids, float* closest_points,
                             float* uvw, const a3d_udf_tuning* tuning, unsigned long long* stats, void* workspace,
                             size_t workspace_bytes, a3d_stream_t stream) {
  a3d::TaskShape shape{a3d::kTaskPool, 0};
  if (tuning) {
    A3D_REQUIRE(tuning->pool >= 0 && tuning->pool <= 4096 && tuning->blocks_per_sm >= 0, A3D_ERR_ARGUMENT,
                "batch_udf: bad tuning");
    if (tuning->pool > 0) shape.pool = tuning->pool;
    shape.blocks_per_sm = tuning->blocks_per_sm;
  }
  return a3d::batch_udf(bvh, points, query_offsets, num_queries, distances, face_ids, closest_points, uvw, shape,
                        stats, workspace, workspace_bytes, (cudaStream_t)stream);
}

extern "C" size_t a3d_batch_autotune_workspace_bytes(int64_t sample_queries, int32_t num_meshes) {
  a3d::Workspace ws(nullptr, 0);
  a3d::TuneWs t;
  return a3d::carve_tune(t, ws, sample_queries > 0 ? sample_queries : 1, num_meshes > 0 ? num_meshes : 1) + 256;
}

extern "C" int a3d_batch_autotune(const a3d_bvh_batch* bvh, const float* points, const int64_t* query_offsets,
                                  int64_t num_queries, int64_t sample_queries, void* workspace,
                                  size_t workspace_bytes, a3d_udf_tuning* best, float* best_ms,
                                  a3d_stream_t stream_) {
  using namespace a3d;
  cudaStream_t s = (cudaStream_t)stream_;
  A3D_REQUIRE(bvh && points && query_offsets && best && num_queries > 0 && sample_queries > 0, A3D_ERR_ARGUMENT,
              "batch_autotune: bad argument");
  A3D_REQUIRE(sample_queries <= kBatchChunk, A3D_ERR_ARGUMENT, "batch_autotune: sample larger than one launch");
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  A3D_CUDA_TRY(cudaStreamIsCapturing(s, &cap));
  A3D_REQUIRE(cap == cudaStreamCaptureStatusNone, A3D_ERR_ARGUMENT,
              "batch_autotune: times launches on the host; call it outside stream capture");
  const int64_t stride = (num_queries + sample_queries - 1) / sample_queries;
  const int64_t ns = (num_queries + stride - 1) / stride;
  Workspace ws(workspace, workspace_bytes);
  TuneWs t;
  carve_tune(t, ws, ns, bvh->num_meshes);
  A3D_REQUIRE(workspace && ws.ok(), A3D_ERR_WORKSPACE, "batch_autotune: workspace too small");
  const int64_t th = ns > (int64_t)bvh->num_meshes + 1 ? ns : (int64_t)bvh->num_meshes + 1;
  A3D_PDL(sample_queries_kernel, dim3((unsigned)ceil_div(th, 256)), dim3(256), 0, s, points, stride, query_offsets,
          bvh->num_meshes, t.pts, ns, t.qoff);
  int occ = 0;
  A3D_TRY((task_blocks_per_sm<false, false, true>(&occ)));
  const int pools[4] = {32, 64, 128, 256};
  const int bpss[3] = {occ, occ * 3 / 4, occ / 2};
  cudaEvent_t e0, e1;
  A3D_CUDA_TRY(cudaEventCreate(&e0));
  A3D_CUDA_TRY(cudaEventCreate(&e1));
  float best_t = INFINITY;
  a3d_udf_tuning bt{kTaskPool, occ, 0, 0};
  int rc = A3D_OK;
  for (int pi = 0; pi < 4 && rc == A3D_OK; ++pi) {
    for (int bi = 0; bi < 3 && rc == A3D_OK; ++bi) {
      const int bps = bpss[bi];
      if (bps < 1 || (bi > 0 && bps == bpss[bi - 1])) continue;
      const TaskShape shape{pools[pi], bps};
      // one warm-up run, then two timed
      for (int rep = 0; rep < 3 && rc == A3D_OK; ++rep) {
        if (rep == 1 && cudaEventRecord(e0, s) != cudaSuccess) rc = A3D_ERR_CUDA;
        if (rc == A3D_OK)
          rc = batch_udf(bvh, t.pts, t.qoff, ns, t.dist, t.fid, t.cp, nullptr, shape, nullptr, t.udf_ws, t.udf_bytes,
                         s);
      }
      float ms = 0.f;
      if (rc == A3D_OK && (cudaEventRecord(e1, s) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
                           cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess))
        rc = A3D_ERR_CUDA;
      if (rc != A3D_OK) break;
      ms *= 0.5f;
      if (ms < best_t) {
        best_t = ms;
        bt = a3d_udf_tuning{pools[pi], bps, 0, 0};
      }
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc != A3D_OK) return rc;
  *best = bt;
  if (best_ms) *best_ms = best_t;
  return A3D_OK;
}
