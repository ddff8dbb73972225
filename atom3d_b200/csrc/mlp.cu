// Learned distance bound: a Fourier-feature MLP (3 -> 64 Fourier features
// -> 128 -> 128 -> 128 -> 1, ReLU) with BF16 operands and FP32
// accumulation: inference on the tcgen05 tensor cores (accumulators in
// tensor memory), training with mma.sync GEMM kernels.
//
// No counterpart in the reference.  The network predicts the unsigned
// distance of a query (or its logarithm); a calibrated scale and margin turn
// the prediction into a per-query upper bound that seeds the closest-point
// traversal's pruning radius (a3d_udf's `bound` argument).  The traversal
// re-runs any query whose bound proves too small, so results never depend
// on the network.
//
// Kernels:
//   mlp_bound_tc_kernel  fused inference: Fourier features, three hidden
//                        layers as tcgen05.mma (M = 128 queries, N = 128,
//                        K = 16 per instruction, weights staged once per
//                        CTA), epilogues from tensor memory, head
//   gemm_bf16_kernel     C = op(A) op(B) (+bias)(relu)(mask) for training,
//                        arbitrary strides, 64x64 tiles, 4 warps
//   small kernels        Fourier features, head forward/backward, column
//                        sums, Adam
#include <math.h>

#include <algorithm>

#include <cuda_bf16.h>

#include "a3d_common.cuh"

namespace a3d {
namespace {

constexpr int kIn = 64, kHid = 128;
constexpr float kTwoPi = 6.283185307179586f;

__device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], const uint32_t (&b)[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const uint32_t*>(&v);
}

// ---------------------------------------------------------------------------
// generic training GEMM
// ---------------------------------------------------------------------------
constexpr int kBM = 64, kBN = 64, kBK = 32, kPad = 8;

struct GemmArgs {
  const __nv_bfloat16* A;  // element (m, k) at A[m*sam + k*sak]
  const __nv_bfloat16* B;  // element (k, n) at B[k*sbk + n*sbn]
  int64_t sam, sak, sbk, sbn;
  int m, n, k;
  const float* bias;       // [n] or null
  const __nv_bfloat16* mask;  // [m, n] row-major: out *= (mask > 0), or null
  int relu;
  float* Cf;               // fp32 [m, n] row-major or null
  int accumulate;          // Cf += result
  __nv_bfloat16* Cb;       // bf16 [m, n] row-major or null
};

__global__ void __launch_bounds__(128) gemm_bf16_kernel(GemmArgs g) {
  __shared__ __align__(16) __nv_bfloat16 As[kBM][kBK + kPad];
  __shared__ __align__(16) __nv_bfloat16 Bs[kBN][kBK + kPad];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
  const int m0 = blockIdx.y * kBM, n0 = blockIdx.x * kBN;
  const int gid = lane >> 2, tig = lane & 3;
  float acc[2][4][4];
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int r = 0; r < 4; ++r) acc[i][j][r] = 0.f;
  const __nv_bfloat16 zero = __float2bfloat16(0.f);
  // split-K: slice z of gridDim.z covers [k_begin, k_end) and adds into Cf
  const int k_per = (int)((((int64_t)g.k + gridDim.z - 1) / gridDim.z + kBK - 1) / kBK) * kBK;
  const int k_begin = blockIdx.z * k_per, k_end = min(g.k, k_begin + k_per);
  for (int k0 = k_begin; k0 < k_end; k0 += kBK) {
    for (int e = tid; e < kBM * kBK; e += 128) {
      const int mm = e / kBK, kk = e % kBK;
      const int gm = m0 + mm, gk = k0 + kk;
      As[mm][kk] = (gm < g.m && gk < k_end) ? g.A[(int64_t)gm * g.sam + (int64_t)gk * g.sak] : zero;
      const int gn = n0 + mm;
      Bs[mm][kk] = (gn < g.n && gk < k_end) ? g.B[(int64_t)gk * g.sbk + (int64_t)gn * g.sbn] : zero;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < kBK; kk += 16) {
      uint32_t a[2][4], b[4][2];
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const int r = wm + i * 16 + gid;
        a[i][0] = *reinterpret_cast<const uint32_t*>(&As[r][kk + 2 * tig]);
        a[i][1] = *reinterpret_cast<const uint32_t*>(&As[r + 8][kk + 2 * tig]);
        a[i][2] = *reinterpret_cast<const uint32_t*>(&As[r][kk + 2 * tig + 8]);
        a[i][3] = *reinterpret_cast<const uint32_t*>(&As[r + 8][kk + 2 * tig + 8]);
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int c = wn + j * 8 + gid;
        b[j][0] = *reinterpret_cast<const uint32_t*>(&Bs[c][kk + 2 * tig]);
        b[j][1] = *reinterpret_cast<const uint32_t*>(&Bs[c][kk + 2 * tig + 8]);
      }
#pragma unroll
      for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) mma_bf16(acc[i][j], a[i], b[j]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        const int mm = m0 + wm + i * 16 + gid + (r >= 2 ? 8 : 0);
        const int nn = n0 + wn + j * 8 + 2 * tig + (r & 1);
        if (mm >= g.m || nn >= g.n) continue;
        float v = acc[i][j][r];
        if (g.bias) v += g.bias[nn];
        if (g.relu) v = fmaxf(v, 0.f);
        const int64_t o = (int64_t)mm * g.n + nn;
        if (g.mask && !(__bfloat162float(g.mask[o]) > 0.f)) v = 0.f;
        if (gridDim.z > 1) atomicAdd(g.Cf + o, v);
        else if (g.Cf) g.Cf[o] = g.accumulate ? g.Cf[o] + v : v;
        if (g.Cb) g.Cb[o] = __float2bfloat16(v);
      }
}

// ---------------------------------------------------------------------------
// small training kernels
// ---------------------------------------------------------------------------
struct Normalise {
  float cx, cy, cz, inv;  // x_hat = (x - c) * inv
};

// Fourier feature pair j of a point.  The hardware sine/cosine (__sincosf):
// its absolute error, about 1e-5 for the arguments here (|t| < ~50), is far
// below the BF16 rounding the features get next, and training and inference
// both use it, so the network sees the features it was trained on.
__device__ __forceinline__ void fourier(float x, float y, float z, const Normalise& nz, const float* __restrict__ freq,
                                        int j, float& s, float& c) {
  const float u = (x - nz.cx) * nz.inv, v = (y - nz.cy) * nz.inv, w = (z - nz.cz) * nz.inv;
  const float t = kTwoPi * (freq[3 * j] * u + freq[3 * j + 1] * v + freq[3 * j + 2] * w);
  __sincosf(t, &s, &c);
}

__global__ void fourier_kernel(const float* __restrict__ x, int64_t n, Normalise nz, const float* __restrict__ freq,
                               __nv_bfloat16* __restrict__ feat) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n * (kIn / 2)) return;
  const int64_t i = t / (kIn / 2);
  const int j = (int)(t % (kIn / 2));
  float s, c;
  fourier(x[3 * i], x[3 * i + 1], x[3 * i + 2], nz, freq, j, s, c);
  feat[i * kIn + 2 * j] = __float2bfloat16(s);
  feat[i * kIn + 2 * j + 1] = __float2bfloat16(c);
}

// y = h w4 + b4; dy = w * 2 (y - d) / n  (w = under_weight when y < d);
// dh = dy * w4 (bf16); dw4 += dy h, db4 += dy; loss += w (y - d)^2 / n
__global__ void head_kernel(const __nv_bfloat16* __restrict__ h, int64_t n, const float* __restrict__ w4,
                            const float* __restrict__ b4, const float* __restrict__ target, float under_weight,
                            float* __restrict__ y_out, __nv_bfloat16* __restrict__ dh, float* __restrict__ dw4,
                            float* __restrict__ db4, float* __restrict__ loss) {
  const int64_t i = (int64_t)blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (i >= n) return;
  float acc = 0.f;
  for (int k = lane; k < kHid; k += 32) acc += __bfloat162float(h[i * kHid + k]) * w4[k];
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  const float y = acc + b4[0];
  if (lane == 0 && y_out) y_out[i] = y;
  if (!target) return;
  const float e = y - target[i];
  const float wgt = e < 0.f ? under_weight : 1.f;
  const float dy = wgt * 2.f * e / (float)n;
  for (int k = lane; k < kHid; k += 32) {
    const float hv = __bfloat162float(h[i * kHid + k]);
    dh[i * kHid + k] = __float2bfloat16(dy * w4[k] * (hv > 0.f ? 1.f : 0.f));
    atomicAdd(&dw4[k], dy * hv);
  }
  if (lane == 0) {
    atomicAdd(db4, dy);
    atomicAdd(loss, wgt * e * e / (float)n);
  }
}

__global__ void colsum_kernel(const __nv_bfloat16* __restrict__ g, int64_t n, int cols, float* __restrict__ out) {
  const int c = blockIdx.x;
  float acc = 0.f;
  for (int64_t i = threadIdx.x; i < n; i += blockDim.x) acc += __bfloat162float(g[i * cols + c]);
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  __shared__ float s[32];
  if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    float t = 0.f;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += s[w];
    out[c] = t;
  }
}

__global__ void adam_kernel(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, int64_t n, float lr, float b1, float b2, float eps, float bc1,
                            float bc2) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  p[i] -= lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
}

__global__ void f32_to_bf16_kernel(const float* __restrict__ in, int64_t n, __nv_bfloat16* __restrict__ out) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = __float2bfloat16(in[i]);
}

// ---------------------------------------------------------------------------
// fused inference on the fifth-generation tensor cores (tcgen05 + TMEM)
// ---------------------------------------------------------------------------
// One CTA per SM, four warpgroups.  The three hidden-layer weight matrices
// are staged once per CTA in shared memory (W^T, K-major, 128-B swizzle:
// 80 KB); each warpgroup owns a tile of 128 queries at a time: its threads
// write the tile's Fourier features (one query row per thread) into the
// group's A operand, one thread issues the layer's tcgen05.mma.kind::f16
// (M = 128 queries, N = 128 outputs, K = 16 per instruction) into the
// group's 128 TMEM columns and commits to the group's mbarrier; the 128
// threads then read their own row back with tcgen05.ld (warp w of the group
// owns TMEM lanes 32w..32w+31), add the bias, apply ReLU, round to bf16 and
// write the next layer's A operand in place.  The last layer folds into the
// head dot product in registers.  The groups run independently (named
// barriers), so one group's MMAs overlap another group's epilogue.
constexpr int kTcGroups = 4;
constexpr int kTcThreads = kTcGroups * 128;
constexpr int kTcRows = 128;                   // queries per tile (MMA M)
constexpr uint32_t kAtom = kTcRows * 128u;     // 128 rows x 128 B: one swizzle column of K = 64 bf16
constexpr uint32_t kTmemCols = 512;            // 4 groups x 128 fp32 columns
constexpr uint32_t kWaitLimit = 1u << 22;      // mbarrier polls before a group gives up

struct TcSmem {  // placed at a 1024-B aligned address (the 128-B swizzle repeats every 1 KB)
  uint8_t w1[kAtom];                  // W1^T: N = 128, K = 64
  uint8_t w2[2 * kAtom];              // W2^T: K = 128 as two 64-wide columns
  uint8_t w3[2 * kAtom];
  uint8_t act[kTcGroups][2 * kAtom];  // per-group A operand (features, then hidden activations)
  float b1[kHid], b2[kHid], b3[kHid], w4[kHid];
  float freq[kIn / 2 * 3];
  unsigned long long mbar[kTcGroups];
  uint32_t tmem_base;
};

struct InfParams {
  const __nv_bfloat16* w1t;  // [128][64] (out-major)
  const __nv_bfloat16* w2t;  // [128][128]
  const __nv_bfloat16* w3t;
  const float* b1;
  const float* b2;
  const float* b3;
  const float* w4;
  float b4;
  const float* freq;  // [32][3]
  Normalise nz;
  float scale, margin;  // bound = max(y, 0) * scale + margin, or exp(y) * scale + margin
  int log_space;        // the network predicts log(distance)
};

// byte offset of 16-B chunk c (0..7) of row r inside one K-major 128-B
// swizzle column: 8-row groups 1 KB apart, rows 128 B apart, the chunk index
// XORed with the row's position in its 8-row group
__device__ __forceinline__ uint32_t sw128(uint32_t r, uint32_t c) {
  return (r >> 3) * 1024u + (r & 7u) * 128u + ((c ^ (r & 7u)) << 4);
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// shared-memory matrix descriptor: K-major, 128-B swizzle, 8-row groups
// 1024 B apart (stride byte offset), leading byte offset unused (1),
// descriptor version 1
__device__ __forceinline__ uint64_t sw128_desc(uint32_t addr) {
  return (uint64_t)((addr & 0x3FFFFu) >> 4) | ((uint64_t)1u << 16) | ((uint64_t)(1024u >> 4) << 32) |
         ((uint64_t)1u << 46) | ((uint64_t)2u << 61);
}

// instruction descriptor: BF16 x BF16 -> FP32, A and B K-major, M = 128, N = 128
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((128u >> 3) << 17) | ((128u >> 4) << 24);

__device__ __forceinline__ void umma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(kIdesc), "r"(accumulate));
}

__device__ __forceinline__ void umma_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
               : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void proxy_fence() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void group_sync(int g) {
  asm volatile("bar.sync %0, %1;" ::"r"(1 + g), "r"(128) : "memory");
}

// AND of a predicate over the 128 threads of warpgroup g (a named barrier)
__device__ __forceinline__ bool group_all(int g, bool v) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.u32 q, %1, 0;\n\t"
      "bar.red.and.pred p, %2, %3, q;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(r)
      : "r"((uint32_t)v), "r"(1 + g), "r"(128)
      : "memory");
  return r != 0;
}

// bounded wait for the mbarrier phase with the given parity; false when the
// poll limit ran out
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity) {
  for (uint32_t i = 0; i < kWaitLimit; ++i) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(mbar), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  return false;
}

// 32 consecutive fp32 columns of this thread's TMEM lane
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// stage W^T ([128 out][K] bf16, out-major) into K-major 128-B swizzle columns
__device__ __forceinline__ void stage_weights(uint8_t* dst, const __nv_bfloat16* src, int K, int tid) {
  const int chunks = K / 8;  // 16-B chunks per row
  for (int e = tid; e < kHid * chunks; e += kTcThreads) {
    const int n = e / chunks, c = e % chunks;
    const uint4 v = __ldg(reinterpret_cast<const uint4*>(src + (size_t)n * K) + c);
    *reinterpret_cast<uint4*>(dst + (c >> 3) * kAtom + sw128(n, c & 7)) = v;
  }
}

// one layer's epilogue: relu(acc + b) -> bf16 -> this thread's row of the
// next A operand (K = 128: two swizzle columns)
__device__ __forceinline__ void epilogue_to_act(uint32_t tmem_row, const float* b, uint8_t* act, uint32_t row) {
#pragma unroll
  for (int cb = 0; cb < kHid / 32; ++cb) {
    float v[32];
    tmem_ld32(tmem_row + cb * 32, v);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int c0 = cb * 32 + q * 8;
      uint4 w;
      w.x = pack_bf16(fmaxf(v[q * 8 + 0] + b[c0 + 0], 0.f), fmaxf(v[q * 8 + 1] + b[c0 + 1], 0.f));
      w.y = pack_bf16(fmaxf(v[q * 8 + 2] + b[c0 + 2], 0.f), fmaxf(v[q * 8 + 3] + b[c0 + 3], 0.f));
      w.z = pack_bf16(fmaxf(v[q * 8 + 4] + b[c0 + 4], 0.f), fmaxf(v[q * 8 + 5] + b[c0 + 5], 0.f));
      w.w = pack_bf16(fmaxf(v[q * 8 + 6] + b[c0 + 6], 0.f), fmaxf(v[q * 8 + 7] + b[c0 + 7], 0.f));
      *reinterpret_cast<uint4*>(act + (c0 >> 6) * kAtom + sw128(row, (c0 & 63) >> 3)) = w;
    }
  }
}

__global__ void __launch_bounds__(kTcThreads, 1)
    mlp_bound_tc_kernel(const float* __restrict__ x, int64_t n, InfParams p, float* __restrict__ bound,
                        unsigned int* __restrict__ status) {
  extern __shared__ unsigned char smem_raw[];
  TcSmem& S = *reinterpret_cast<TcSmem*>(smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u));
  const int tid = threadIdx.x, g = tid >> 7, t = tid & 127, wg = t >> 5;

  stage_weights(S.w1, p.w1t, kIn, tid);
  stage_weights(S.w2, p.w2t, kHid, tid);
  stage_weights(S.w3, p.w3t, kHid, tid);
  for (int e = tid; e < kHid; e += kTcThreads) {
    S.b1[e] = p.b1[e]; S.b2[e] = p.b2[e]; S.b3[e] = p.b3[e]; S.w4[e] = p.w4[e];
  }
  for (int e = tid; e < kIn / 2 * 3; e += kTcThreads) S.freq[e] = p.freq[e];
  if (tid < kTcGroups) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&S.mbar[tid])), "r"(1) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (tid < 32) {  // warp 0 allocates the CTA's TMEM columns
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&S.tmem_base)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  proxy_fence();  // staged weights visible to the tensor cores
  tc_fence_before();
  __syncthreads();
  tc_fence_after();

  const uint32_t tmem_group = S.tmem_base + (uint32_t)g * kHid;        // this group's 128 columns
  const uint32_t tmem_row = tmem_group + ((uint32_t)(wg * 32) << 16);  // this warp's 32 lanes
  uint8_t* act = S.act[g];
  const uint32_t act_a = smem_u32(act), w1_a = smem_u32(S.w1), w2_a = smem_u32(S.w2), w3_a = smem_u32(S.w3);
  const uint32_t mbar = smem_u32(&S.mbar[g]);
  uint32_t parity = 0;
  bool ok = true;

  const int64_t tiles = ceil_div(n, (int64_t)kTcRows);
  for (int64_t tile = (int64_t)blockIdx.x * kTcGroups + g; tile < tiles && ok;
       tile += (int64_t)gridDim.x * kTcGroups) {
    const int64_t q = tile * kTcRows + t;
    // Fourier features of query q -> row t (K = 64: one swizzle column)
    {
      float px = 0.f, py = 0.f, pz = 0.f;
      if (q < n) { px = x[3 * q]; py = x[3 * q + 1]; pz = x[3 * q + 2]; }
#pragma unroll
      for (int c = 0; c < kIn / 8; ++c) {
        uint32_t w[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          float s, co;
          fourier(px, py, pz, p.nz, S.freq, 4 * c + k, s, co);
          w[k] = pack_bf16(s, co);
        }
        *reinterpret_cast<uint4*>(act + sw128(t, c)) = make_uint4(w[0], w[1], w[2], w[3]);
      }
    }
    float y = 0.f;
#pragma unroll 1
    for (int layer = 0; layer < 3 && ok; ++layer) {
      proxy_fence();       // this thread's A-operand row visible to the tensor cores
      tc_fence_before();   // and its earlier TMEM reads ordered before the barrier
      group_sync(g);
      if (t == 0) {
        tc_fence_after();
        const int ksteps = layer == 0 ? kIn / 16 : kHid / 16;
        const uint32_t w_a = layer == 0 ? w1_a : (layer == 1 ? w2_a : w3_a);
        for (int j = 0; j < ksteps; ++j) {
          const uint32_t off = (uint32_t)(j >> 2) * kAtom + (uint32_t)(j & 3) * 32u;
          umma_bf16(tmem_group, sw128_desc(act_a + off), sw128_desc(w_a + off), j > 0 ? 1u : 0u);
        }
        umma_commit(mbar);
      }
      // the group goes on only if every thread saw the phase complete, so
      // its named barriers stay matched when a wait runs out
      ok = group_all(g, mbar_wait(mbar, parity));
      parity ^= 1u;
      if (!ok) break;
      tc_fence_after();
      if (layer < 2) {
        epilogue_to_act(tmem_row, layer == 0 ? S.b1 : S.b2, act, (uint32_t)t);
      } else {
        // last hidden layer: h rounded to bf16 like training, folded into the head
#pragma unroll
        for (int cb = 0; cb < kHid / 32; ++cb) {
          float v[32];
          tmem_ld32(tmem_row + cb * 32, v);
#pragma unroll
          for (int i = 0; i < 32; ++i) {
            const int c = cb * 32 + i;
            const float h = __bfloat162float(__float2bfloat16(fmaxf(v[i] + S.b3[c], 0.f)));
            y += h * S.w4[c];
          }
        }
      }
    }
    if (ok && q < n) {
      const float z = y + p.b4;
      bound[q] = (p.log_space ? expf(z) : fmaxf(z, 0.f)) * p.scale + p.margin;
    }
  }
  if (!ok) {
    atomicOr(status, 1u);
    // a group that gave up may still have MMAs in flight: wait once more
    // (bounded) for its last commit before the columns are released
    mbar_wait(mbar, parity ^ 1u);
  }
  tc_fence_before();
  __syncthreads();
  if (tid < 32) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(S.tmem_base), "r"(kTmemCols)
                 : "memory");
  }
}

}  // namespace
}  // namespace a3d

using namespace a3d;

// status word of the inference kernel, per device (bit 0: a warpgroup's
// tensor-core wait ran out and its remaining tiles were left unwritten)
__device__ unsigned int g_mlp_status;

extern "C" int a3d_gemm_bf16(const a3d_gemm_args* a, a3d_stream_t stream) {
  A3D_REQUIRE(a && a->A && a->B && (a->Cf || a->Cb), A3D_ERR_ARGUMENT, "gemm_bf16: null operand");
  A3D_REQUIRE(a->m > 0 && a->n > 0 && a->k > 0, A3D_ERR_ARGUMENT, "gemm_bf16: empty shape");
  GemmArgs g{(const __nv_bfloat16*)a->A, (const __nv_bfloat16*)a->B, a->sam, a->sak, a->sbk, a->sbn, a->m, a->n, a->k,
             a->bias, (const __nv_bfloat16*)a->mask, a->relu, a->Cf, a->accumulate, (__nv_bfloat16*)a->Cb};
  dim3 grid((unsigned)ceil_div(a->n, kBN), (unsigned)ceil_div(a->m, kBM));
  // weight gradients (small m x n, long k): split k over the SMs and add
  // into Cf atomically; only for a plain accumulate into Cf
  const bool plain_acc = a->Cf && a->accumulate && !a->Cb && !a->bias && !a->mask && !a->relu;
  const int64_t tiles = (int64_t)grid.x * grid.y;
  const int sms = a3d::num_sms();
  if (plain_acc && tiles < sms && a->k >= 4 * kBK) {
    const int64_t want = (2 * (int64_t)sms + tiles - 1) / tiles;
    grid.z = (unsigned)std::max<int64_t>(1, std::min<int64_t>(want, a->k / (2 * kBK)));
  }
  A3D_REQUIRE(grid.y < 65536, A3D_ERR_ARGUMENT, "gemm_bf16: m too large for one launch");
  gemm_bf16_kernel<<<grid, 128, 0, (cudaStream_t)stream>>>(g);
  A3D_LAUNCH_CHECK();
  return A3D_OK;
}

extern "C" int a3d_mlp_fourier(const float* x, int64_t n, const float* norm4, const float* freq, void* feat_bf16,
                               a3d_stream_t stream) {
  A3D_REQUIRE(n >= 0 && norm4 && freq, A3D_ERR_ARGUMENT, "mlp_fourier: bad argument");
  if (n == 0) return A3D_OK;
  Normalise nz{norm4[0], norm4[1], norm4[2], norm4[3]};
  fourier_kernel<<<(unsigned)ceil_div(n * (kIn / 2), 256), 256, 0, (cudaStream_t)stream>>>(
      x, n, nz, freq, (__nv_bfloat16*)feat_bf16);
  A3D_LAUNCH_CHECK();
  return A3D_OK;
}

extern "C" int a3d_mlp_head(const void* h_bf16, int64_t n, const float* w4, const float* b4, const float* target,
                            float under_weight, float* y, void* dh_bf16, float* dw4, float* db4, float* loss,
                            a3d_stream_t stream) {
  A3D_REQUIRE(n >= 0 && h_bf16 && w4 && b4, A3D_ERR_ARGUMENT, "mlp_head: bad argument");
  if (n == 0) return A3D_OK;
  head_kernel<<<(unsigned)ceil_div(n, 8), 256, 0, (cudaStream_t)stream>>>(
      (const __nv_bfloat16*)h_bf16, n, w4, b4, target, under_weight, y, (__nv_bfloat16*)dh_bf16, dw4, db4, loss);
  A3D_LAUNCH_CHECK();
  return A3D_OK;
}

extern "C" int a3d_mlp_colsum(const void* g_bf16, int64_t n, int cols, float* out, a3d_stream_t stream) {
  A3D_REQUIRE(n > 0 && cols > 0, A3D_ERR_ARGUMENT, "mlp_colsum: bad argument");
  colsum_kernel<<<cols, 256, 0, (cudaStream_t)stream>>>((const __nv_bfloat16*)g_bf16, n, cols, out);
  A3D_LAUNCH_CHECK();
  return A3D_OK;
}

extern "C" int a3d_adam(float* p, const float* g, float* m, float* v, int64_t n, float lr, float beta1, float beta2,
                        float eps, int step, a3d_stream_t stream) {
  A3D_REQUIRE(n > 0 && step > 0, A3D_ERR_ARGUMENT, "adam: bad argument");
  const float bc1 = 1.f - powf(beta1, (float)step), bc2 = 1.f - powf(beta2, (float)step);
  adam_kernel<<<(unsigned)ceil_div(n, 256), 256, 0, (cudaStream_t)stream>>>(p, g, m, v, n, lr, beta1, beta2, eps, bc1,
                                                                           bc2);
  A3D_LAUNCH_CHECK();
  return A3D_OK;
}

extern "C" int a3d_to_bf16(const float* in, int64_t n, void* out, a3d_stream_t stream) {
  if (n <= 0) return A3D_OK;
  f32_to_bf16_kernel<<<(unsigned)ceil_div(n, 256), 256, 0, (cudaStream_t)stream>>>(in, n, (__nv_bfloat16*)out);
  A3D_LAUNCH_CHECK();
  return A3D_OK;
}

extern "C" int a3d_mlp_bound(const a3d_mlp_weights* wts, const float* x, int64_t n, float* bound,
                             a3d_stream_t stream) {
  A3D_REQUIRE(wts && x && bound && n >= 0, A3D_ERR_ARGUMENT, "mlp_bound: null argument");
  if (n == 0) return A3D_OK;
  InfParams p;
  p.w1t = (const __nv_bfloat16*)wts->w1t; p.w2t = (const __nv_bfloat16*)wts->w2t;
  p.w3t = (const __nv_bfloat16*)wts->w3t;
  p.b1 = wts->b1; p.b2 = wts->b2; p.b3 = wts->b3; p.w4 = wts->w4; p.b4 = wts->b4;
  p.freq = wts->freq;
  p.nz = Normalise{wts->norm[0], wts->norm[1], wts->norm[2], wts->norm[3]};
  p.scale = wts->scale; p.margin = wts->margin;
  p.log_space = wts->log_space;
  // the staged weight rows are read as 16-B vectors
  A3D_REQUIRE(((uintptr_t)p.w1t | (uintptr_t)p.w2t | (uintptr_t)p.w3t) % 16 == 0, A3D_ERR_ARGUMENT,
              "mlp_bound: weight matrices must be 16-byte aligned");
  const size_t smem = sizeof(TcSmem) + 1024;  // + alignment of the swizzled operands
  // the shared-memory opt-in and the status word's address are per device
  static bool attr_set[kMaxDevices] = {false};
  static unsigned int* status_ptr[kMaxDevices] = {nullptr};
  int dev = 0;
  A3D_CUDA_TRY(cudaGetDevice(&dev));
  A3D_REQUIRE(dev >= 0 && dev < kMaxDevices, A3D_ERR_ARGUMENT, "mlp_bound: device ordinal out of range");
  if (!attr_set[dev]) {
    A3D_CUDA_TRY(cudaFuncSetAttribute(mlp_bound_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    A3D_CUDA_TRY(cudaGetSymbolAddress((void**)&status_ptr[dev], g_mlp_status));
    attr_set[dev] = true;
  }
  A3D_CUDA_TRY(cudaMemsetAsync(status_ptr[dev], 0, sizeof(unsigned int), (cudaStream_t)stream));
  const int sms = num_sms();
  const int64_t tiles = ceil_div(n, (int64_t)kTcRows);
  const int64_t want = ceil_div(tiles, (int64_t)kTcGroups);
  const int64_t grid = want < (int64_t)sms ? want : (int64_t)sms;
  mlp_bound_tc_kernel<<<(unsigned)grid, kTcThreads, smem, (cudaStream_t)stream>>>(x, n, p, bound,
                                                                                 status_ptr[dev]);
  A3D_LAUNCH_CHECK();
  return A3D_OK;
}

extern "C" int a3d_mlp_bound_status(unsigned int* status, a3d_stream_t stream) {
  A3D_REQUIRE(status, A3D_ERR_ARGUMENT, "mlp_bound_status: null argument");
  A3D_CUDA_TRY(cudaMemcpyFromSymbolAsync(status, g_mlp_status, sizeof(unsigned int), 0, cudaMemcpyDeviceToHost,
                                         (cudaStream_t)stream));
  A3D_CUDA_TRY(cudaStreamSynchronize((cudaStream_t)stream));
  return A3D_OK;
}
