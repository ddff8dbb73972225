// SAH refinement of the binary radix tree, one thread block per cluster.
//
// The Morton radix tree splits space at the midpoint planes of the centroid
// cube, which gives loose boxes near the leaves.  Every subtree of the radix
// tree with at most kSahMax triangles whose parent holds more (a "cluster")
// is rebuilt top-down with a binned surface-area heuristic (16 bins per
// axis, centroid binning, cost = A_left N_left + A_right N_right, ties to
// the lower axis and bin), down to single triangles:
//   * nodes of more than kSahWarpMax triangles are split by the whole block
//     (shared-memory bins, block scans for a stable partition);
//   * smaller nodes are handed to the block's warps, each building its
//     subtrees alone (warp shuffles and ballots, per-warp bins).
// The triangles' centroids and boxes are read from global memory (L2
// resident); the cluster's slice of the sorted face order is partitioned in
// place.  Partitions are stable, reductions are min/max/integer sums, so the
// result is deterministic.  A node with no valid split (coincident centroids) or
// deeper than kSahMaxDepth inside its cluster is split at its median position.
//
// Node numbering stays within the cluster's own index set.  A radix-tree
// subtree over sorted positions [f, l] uses the internal indices [f, l]
// except the end that is not its root; here the node whose split falls
// between local positions m-1 and m gets index f + m - 1 (+1 when the old
// root sat at l), which enumerates exactly that set, and the new root takes
// the old root's index (swapping with the node that would have had it), so
// the cluster's parent needs no update.  Leaves stay N + position; the
// cluster's slice of the sorted face order is rewritten.  Boxes are computed
// afterwards by the ordinary refit.
#pragma once

#include "a3d_common.cuh"

namespace a3d {
namespace {

constexpr int kSahMax = 16384;
constexpr int kSahBins = 16;
constexpr int kSahWarpMax = 128;
// block size of the cluster kernel: 1024 threads when the clusters are
// about as many as the SMs (one mesh up to kSahMax x SMs triangles: each
// block's 32 warps share out its small nodes), 256 when there are many
// (batches: more blocks per SM, cheaper block-wide steps)
constexpr int kSahThreadsWide = 1024;
constexpr int kSahThreadsNarrow = 256;
constexpr int kSahMaxDepth = 48;
// nodes this small split at their median position: 2 = SAH all the way down
// (median splits at 8 and below cut a third of the 256-thread build time of
// the 1.31M-triangle tree but cost 21 more triangle tests per query, +1.2%
// query time)
constexpr int kSahTiny = 2;
constexpr int kSahCand = 3 * (kSahBins - 1);            // 45 split candidates
constexpr int kBinWords = 3 * kSahBins * 7;              // count, lo xyz, hi xyz
constexpr int kSahWarpStack = kSahWarpMax / 2;           // disjoint ranges of >= 2
constexpr int kSahBlockStack = kSahMax / (kSahWarpMax + 1) + 2;

// a node to split: local range [b, e) of its cluster, parent index (-1 for
// the cluster root), side in the parent, depth inside the cluster
struct SahNode {
  int b, e, parent, sd;  // sd = side | depth << 1
};

template <int kThreads>
struct SahSmem {
  static constexpr int kWarps = kThreads / 32;
  uint32_t bins[kWarps + 1][kBinWords];  // per warp, then the block's
  SahNode wstack[kWarps][kSahWarpStack];
  SahNode bstack[kSahBlockStack];
  float red[kWarps][6];
  uint32_t wsum[kWarps];
  float cb[6];
  int nsmall, nb, m, axis, kk, root_nat;
};

struct SahTree {
  int32_t* left;
  int32_t* right;
  int32_t* parent;
  int32_t* first;
  int32_t* last;
  int64_t n;  // total triangles (leaf j is n + j)
};

__device__ __forceinline__ float sah_half_area(float x0, float y0, float z0, float x1, float y1, float z1) {
  const float dx = x1 - x0, dy = y1 - y0, dz = z1 - z0;
  return dx * dy + dy * dz + dz * dx;
}

__device__ __forceinline__ int sah_bin(float c, float lo, float scale) {
  const int k = (int)((c - lo) * scale);
  return k < kSahBins - 1 ? k : kSahBins - 1;
}

// candidate `cand` (axis cand / 15, split after bin cand % 15) of the bins:
// cost and left count; cost = +inf when a side is empty or the axis is flat
__device__ __forceinline__ void sah_candidate(const uint32_t* bins, const float* cb, int cand, float& cost, int& nl) {
  cost = INFINITY;
  nl = 0;
  if (cand >= kSahCand) return;
  const int axis = cand / (kSahBins - 1), k = cand % (kSahBins - 1) + 1;
  if (!(cb[3 + axis] > cb[axis])) return;
  float l0 = INFINITY, l1 = INFINITY, l2 = INFINITY, u0 = -INFINITY, u1 = -INFINITY, u2 = -INFINITY;
  float r0 = INFINITY, r1 = INFINITY, r2 = INFINITY, v0 = -INFINITY, v1 = -INFINITY, v2 = -INFINITY;
  int cl = 0, cr = 0;
  for (int j = 0; j < kSahBins; ++j) {
    const uint32_t* w = bins + (axis * kSahBins + j) * 7;
    const int cnt = (int)w[0];
    if (cnt == 0) continue;
    const float a0 = float_unflip(w[1]), a1 = float_unflip(w[2]), a2 = float_unflip(w[3]);
    const float b0 = float_unflip(w[4]), b1 = float_unflip(w[5]), b2 = float_unflip(w[6]);
    if (j < k) {
      cl += cnt;
      l0 = fminf(l0, a0); l1 = fminf(l1, a1); l2 = fminf(l2, a2);
      u0 = fmaxf(u0, b0); u1 = fmaxf(u1, b1); u2 = fmaxf(u2, b2);
    } else {
      cr += cnt;
      r0 = fminf(r0, a0); r1 = fminf(r1, a1); r2 = fminf(r2, a2);
      v0 = fmaxf(v0, b0); v1 = fmaxf(v1, b1); v2 = fmaxf(v2, b2);
    }
  }
  if (cl == 0 || cr == 0) return;
  cost = sah_half_area(l0, l1, l2, u0, u1, u2) * (float)cl + sah_half_area(r0, r1, r2, v0, v1, v2) * (float)cr;
  nl = cl;
}

// the warp's best candidate (lowest cost, then lowest candidate index);
// returns the left count, 0 when no candidate is valid
__device__ __forceinline__ int sah_pick(const uint32_t* bins, const float* cb, int lane, int& axis, int& kk) {
  float cost0, cost1;
  int nl0, nl1;
  sah_candidate(bins, cb, lane, cost0, nl0);
  sah_candidate(bins, cb, lane + 32, cost1, nl1);
  float best = cost0;
  int bc = lane, bn = nl0;
  if (cost1 < best) { best = cost1; bc = lane + 32; bn = nl1; }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const float oc = __shfl_xor_sync(0xffffffffu, best, o);
    const int oi = __shfl_xor_sync(0xffffffffu, bc, o);
    const int on = __shfl_xor_sync(0xffffffffu, bn, o);
    if (oc < best || (oc == best && oi < bc)) { best = oc; bc = oi; bn = on; }
  }
  if (!(best < INFINITY)) return 0;
  axis = bc / (kSahBins - 1);
  kk = bc % (kSahBins - 1) + 1;
  return bn;
}

// the triangles' centroids and boxes, indexed by face id
struct SahPrims {
  const float4* __restrict__ cen;
  const float4* __restrict__ lo;
  const float4* __restrict__ hi;
};

__device__ __forceinline__ float sah_c(const float4& c, int a) { return a == 0 ? c.x : (a == 1 ? c.y : c.z); }

__device__ __forceinline__ void sah_bin_prim(uint32_t* bins, const SahPrims& P, uint32_t face, const float* cb,
                                             const float* scale) {
  const float4 c = __ldg(P.cen + face), lo = __ldg(P.lo + face), hi = __ldg(P.hi + face);
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    if (!(cb[3 + a] > cb[a])) continue;
    uint32_t* w = bins + (a * kSahBins + sah_bin(sah_c(c, a), cb[a], scale[a])) * 7;
    atomicAdd(&w[0], 1u);
    atomicMin(&w[1], float_flip(lo.x));
    atomicMin(&w[2], float_flip(lo.y));
    atomicMin(&w[3], float_flip(lo.z));
    atomicMax(&w[4], float_flip(hi.x));
    atomicMax(&w[5], float_flip(hi.y));
    atomicMax(&w[6], float_flip(hi.z));
  }
}

__device__ __forceinline__ void sah_clear_bins(uint32_t* bins, int t, int nt) {
  for (int i = t; i < kBinWords; i += nt) {
    const int f = i % 7;
    bins[i] = f == 0 ? 0u : (f <= 3 ? 0xffffffffu : 0u);  // flipped +inf / -inf
  }
}

// index of the node of a cluster rooted at R over [f, l] that splits at local m
__device__ __forceinline__ int sah_label(int f, int m, int shift, int R, int root_nat, bool is_root) {
  const int nat = f + m - 1 + shift;
  if (is_root) return R;
  return nat == R ? root_nat : nat;
}

// writes the node's topology and the leaf children; returns the children
// that need processing through `push(b, e, side)`
template <typename Push>
__device__ __forceinline__ void sah_emit(const SahTree& T, int f, int b, int m, int e, int label, int plabel,
                                         int side, Push&& push) {
  T.first[label] = f + b;
  T.last[label] = f + e - 1;
  if (plabel >= 0) {
    T.parent[label] = plabel;
    if (side) T.right[plabel] = label;
    else T.left[plabel] = label;
  }
  if (m - b == 1) {
    const int leaf = (int)(T.n + f + b);
    T.left[label] = leaf;
    T.parent[leaf] = label;
  } else {
    push(b, m, 0);
  }
  if (e - m == 1) {
    const int leaf = (int)(T.n + f + m);
    T.right[label] = leaf;
    T.parent[leaf] = label;
  } else {
    push(m, e, 1);
  }
}

// One block per cluster (grid-stride over the device-side cluster list).
// The cluster's slice of the sorted face order is partitioned in place
// (tmp: a scratch slice of the same positions); small nodes waiting for the
// warps are listed in `small` at the cluster's positions (a cluster of n
// triangles has fewer than n of them).
template <int kThreads>
__global__ void __launch_bounds__(kThreads)
    sah_cluster_kernel(const int32_t* __restrict__ clusters, const uint32_t* __restrict__ ncl, SahTree T,
                       uint32_t* __restrict__ order, uint32_t* __restrict__ tmp_all, SahNode* __restrict__ small_all,
                       SahPrims P) {
  pdl_wait();
  extern __shared__ __align__(16) unsigned char sah_raw[];
  constexpr int kWarps = kThreads / 32;
  SahSmem<kThreads>& S = *reinterpret_cast<SahSmem<kThreads>*>(sah_raw);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const unsigned FULL = 0xffffffffu;
  const uint32_t count = *ncl;
  for (uint32_t ci = blockIdx.x; ci < count; ci += gridDim.x) {
    const int R = clusters[ci];
    const int f = T.first[R], l = T.last[R];
    const int n = l - f + 1;
    const int shift = (R == l) ? 1 : 0;
    uint32_t* ord = order + f;
    uint32_t* tmp = tmp_all + f;
    SahNode* small = small_all + f;
    if (tid == 0) {
      S.nsmall = 0;
      S.nb = 0;
      const SahNode root{0, n, -1, 0};
      if (n > kSahWarpMax) S.bstack[S.nb++] = root;
      else small[S.nsmall++] = root;
    }
    __syncthreads();
    // ---- stage A: nodes above kSahWarpMax, split by the whole block
    for (;;) {
      __syncthreads();
      const int nb = S.nb;
      if (nb == 0) break;
      const SahNode en = S.bstack[nb - 1];
      const int b = en.b, e = en.e, side = en.sd & 1, depth = en.sd >> 1;
      const int plabel = en.parent;
      const bool is_root = plabel < 0;
      // centroid bounds
      float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
      for (int i = b + tid; i < e; i += kThreads) {
        const float4 c = __ldg(P.cen + ord[i]);
        mn[0] = fminf(mn[0], c.x); mn[1] = fminf(mn[1], c.y); mn[2] = fminf(mn[2], c.z);
        mx[0] = fmaxf(mx[0], c.x); mx[1] = fmaxf(mx[1], c.y); mx[2] = fmaxf(mx[2], c.z);
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1)
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          mn[a] = fminf(mn[a], __shfl_xor_sync(FULL, mn[a], o));
          mx[a] = fmaxf(mx[a], __shfl_xor_sync(FULL, mx[a], o));
        }
      if (lane == 0)
        for (int a = 0; a < 3; ++a) { S.red[warp][a] = mn[a]; S.red[warp][3 + a] = mx[a]; }
      sah_clear_bins(S.bins[kWarps], tid, kThreads);
      __syncthreads();
      if (tid < 6) {
        float v = S.red[0][tid];
        for (int w = 1; w < kWarps; ++w) v = tid < 3 ? fminf(v, S.red[w][tid]) : fmaxf(v, S.red[w][tid]);
        S.cb[tid] = v;
      }
      __syncthreads();
      float cb[6], scale[3];
#pragma unroll
      for (int k = 0; k < 6; ++k) cb[k] = S.cb[k];
#pragma unroll
      for (int a = 0; a < 3; ++a) scale[a] = cb[3 + a] > cb[a] ? (float)kSahBins / (cb[3 + a] - cb[a]) : 0.f;
      const bool median = depth >= kSahMaxDepth;
      if (!median)
        for (int i = b + tid; i < e; i += kThreads) sah_bin_prim(S.bins[kWarps], P, ord[i], cb, scale);
      __syncthreads();
      if (warp == 0) {
        int axis = 0, kk = 0, nl = 0;
        if (!median) nl = sah_pick(S.bins[kWarps], cb, lane, axis, kk);
        if (lane == 0) {
          S.m = nl > 0 ? b + nl : b + (e - b) / 2;
          S.axis = nl > 0 ? axis : -1;
          S.kk = kk;
        }
      }
      __syncthreads();
      const int m = S.m, axis = S.axis, kk = S.kk;
      if (axis >= 0) {
        // stable partition: block-wide ranks of the left flags, chunk by chunk
        int lbase = b, rbase = m;
        for (int i0 = b; i0 < e; i0 += kThreads) {
          const int i = i0 + tid;
          uint32_t p = 0;
          bool lft = false;
          if (i < e) {
            p = ord[i];
            lft = sah_bin(sah_c(__ldg(P.cen + p), axis), cb[axis], scale[axis]) < kk;
          }
          const unsigned bl = __ballot_sync(FULL, lft), br = __ballot_sync(FULL, i < e && !lft);
          __syncthreads();
          if (lane == 0) S.wsum[warp] = (uint32_t)__popc(bl) | ((uint32_t)__popc(br) << 16);
          __syncthreads();
          int lb = 0, rb = 0, lt = 0, rt = 0;
          for (int w = 0; w < kWarps; ++w) {
            const uint32_t v = S.wsum[w];
            if (w < warp) { lb += (int)(v & 0xffffu); rb += (int)(v >> 16); }
            lt += (int)(v & 0xffffu);
            rt += (int)(v >> 16);
          }
          const unsigned below = (1u << lane) - 1u;
          if (i < e) {
            if (lft) tmp[lbase + lb + __popc(bl & below)] = p;
            else tmp[rbase + rb + __popc(br & below)] = p;
          }
          lbase += lt;
          rbase += rt;
        }
        __syncthreads();
        for (int i = b + tid; i < e; i += kThreads) ord[i] = tmp[i];
      }
      __syncthreads();
      if (tid == 0) {
        --S.nb;
        if (is_root) S.root_nat = f + m - 1 + shift;
        const int label = sah_label(f, m, shift, R, S.root_nat, is_root);
        sah_emit(T, f, b, m, e, label, plabel, side, [&](int cb0, int ce0, int cs) {
          const SahNode ch{cb0, ce0, label, cs | ((depth + 1) << 1)};
          if (ce0 - cb0 > kSahWarpMax) S.bstack[S.nb++] = ch;
          else small[S.nsmall++] = ch;
        });
      }
    }
    __syncthreads();
    // ---- stage B: each warp builds the subtrees of its small nodes
    uint32_t* wb = S.bins[warp];
    SahNode* ws = S.wstack[warp];
    const int nsmall = S.nsmall;
    for (int si = warp; si < nsmall; si += kWarps) {
      if (lane == 0) ws[0] = small[si];
      int sp = 1;
      __syncwarp();
      while (sp > 0) {
        const SahNode en = ws[sp - 1];
        --sp;
        __syncwarp();
        const int b = en.b, e = en.e, side = en.sd & 1, depth = en.sd >> 1;
        const int plabel = en.parent;
        const bool is_root = plabel < 0;
        int m = b + 1;
        // at most kSahTiny triangles: split at the median position
        if (e - b > kSahTiny) {
          float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
          for (int i = b + lane; i < e; i += 32) {
            const float4 c = __ldg(P.cen + ord[i]);
            mn[0] = fminf(mn[0], c.x); mn[1] = fminf(mn[1], c.y); mn[2] = fminf(mn[2], c.z);
            mx[0] = fmaxf(mx[0], c.x); mx[1] = fmaxf(mx[1], c.y); mx[2] = fmaxf(mx[2], c.z);
          }
          float cb[6], scale[3];
#pragma unroll
          for (int o = 16; o > 0; o >>= 1)
#pragma unroll
            for (int a = 0; a < 3; ++a) {
              mn[a] = fminf(mn[a], __shfl_xor_sync(FULL, mn[a], o));
              mx[a] = fmaxf(mx[a], __shfl_xor_sync(FULL, mx[a], o));
            }
#pragma unroll
          for (int a = 0; a < 3; ++a) {
            cb[a] = mn[a];
            cb[3 + a] = mx[a];
            scale[a] = mx[a] > mn[a] ? (float)kSahBins / (mx[a] - mn[a]) : 0.f;
          }
          int nl = 0, axis = 0, kk = 0;
          if (depth < kSahMaxDepth) {
            sah_clear_bins(wb, lane, 32);
            __syncwarp();
            for (int i = b + lane; i < e; i += 32) sah_bin_prim(wb, P, ord[i], cb, scale);
            __syncwarp();
            nl = sah_pick(wb, cb, lane, axis, kk);
            __syncwarp();
          }
          if (nl > 0) {
            m = b + nl;
            int lbase = b, rbase = m;
            for (int i0 = b; i0 < e; i0 += 32) {
              const int i = i0 + lane;
              uint32_t p = 0;
              bool lft = false;
              if (i < e) {
                p = ord[i];
                lft = sah_bin(sah_c(__ldg(P.cen + p), axis), cb[axis], scale[axis]) < kk;
              }
              const unsigned bl = __ballot_sync(FULL, lft), br = __ballot_sync(FULL, i < e && !lft);
              const unsigned below = (1u << lane) - 1u;
              if (i < e) {
                if (lft) tmp[lbase + __popc(bl & below)] = p;
                else tmp[rbase + __popc(br & below)] = p;
              }
              lbase += __popc(bl);
              rbase += __popc(br);
            }
            __syncwarp();
            for (int i = b + lane; i < e; i += 32) ord[i] = tmp[i];
            __syncwarp();
          } else {
            m = b + (e - b) / 2;
          }
        } else {
          m = b + (e - b) / 2;
        }
        if (lane == 0) {
          if (is_root) S.root_nat = f + m - 1 + shift;
          const int label = sah_label(f, m, shift, R, S.root_nat, is_root);
          sah_emit(T, f, b, m, e, label, plabel, side, [&](int cb0, int ce0, int cs) {
            ws[sp++] = SahNode{cb0, ce0, label, cs | ((depth + 1) << 1)};
          });
        }
        sp = __shfl_sync(FULL, sp, 0);
        __syncwarp();
      }
    }
    __syncthreads();
  }
}

// clusters: internal nodes of 3..sah_max triangles whose parent has more (or
// that are a mesh root); sah_max <= kSahMax
__global__ void sah_find_kernel(const int64_t* __restrict__ face_off, int nmesh, int64_t n,
                                const int32_t* __restrict__ parent, const int32_t* __restrict__ first,
                                const int32_t* __restrict__ last, int sah_max, int32_t* __restrict__ clusters,
                                uint32_t* __restrict__ ncl) {
  pdl_wait();
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int lo = 0, hi = nmesh - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (face_off[mid] <= i) lo = mid;
    else hi = mid - 1;
  }
  if (i >= face_off[lo + 1] - 1) return;  // the last position of a range has no internal node
  const int cnt = last[i] - first[i] + 1;
  if (cnt < 3 || cnt > sah_max) return;
  const int p = parent[i];
  if (p >= 0 && last[p] - first[p] + 1 <= sah_max) return;
  clusters[atomicAdd(ncl, 1u)] = (int32_t)i;
}

}  // namespace
}  // namespace a3d
