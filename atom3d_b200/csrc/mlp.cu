// Learned distance bound: a Fourier-feature MLP (3 -> 64 Fourier features
// -> 128 -> 128 -> 128 -> 1, ReLU) evaluated and trained with hand-written
// BF16 tensor-core kernels (mma.sync m16n8k16, FP32 accumulation).
//
// No counterpart in the reference.  The network predicts the unsigned
// distance of a query; a calibrated margin turns the prediction into a
// per-query upper bound that seeds the closest-point traversal's pruning
// radius (a3d_udf's `bound` argument).  The traversal re-runs any query
// whose bound proves too small, so results never depend on the network.
//
// Kernels:
//   mlp_bound_kernel   fused inference: features, three hidden layers and
//                      the head for 128 queries per CTA, weights and
//                      activations in shared memory
//   gemm_bf16_kernel   C = op(A) op(B) (+bias)(relu)(mask) for training,
//                      arbitrary strides, 64x64 tiles, 4 warps
//   small kernels      Fourier features, head forward/backward, column
//                      sums, Adam
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

__device__ __forceinline__ void fourier(float x, float y, float z, const Normalise& nz, const float* __restrict__ freq,
                                        int j, float& s, float& c) {
  const float u = (x - nz.cx) * nz.inv, v = (y - nz.cy) * nz.inv, w = (z - nz.cz) * nz.inv;
  const float t = kTwoPi * (freq[3 * j] * u + freq[3 * j + 1] * v + freq[3 * j + 2] * w);
  sincosf(t, &s, &c);
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
// fused inference
// ---------------------------------------------------------------------------
constexpr int kInfWarps = 4;
constexpr int kRowsPerWarp = 32;
constexpr int kRows = kInfWarps * kRowsPerWarp;  // 128 queries per CTA
constexpr int kLd1 = kIn + 8;                    // padded row strides (bf16)
constexpr int kLdH = kHid + 8;

struct InfSmem {
  __nv_bfloat16 w1t[kHid][kLd1];   // W1 transposed: [out][in]
  __nv_bfloat16 w2t[kHid][kLdH];
  __nv_bfloat16 w3t[kHid][kLdH];
  float b1[kHid], b2[kHid], b3[kHid], w4[kHid];
  float freq[kIn / 2 * 3];
  __nv_bfloat16 act[kInfWarps][2][kRowsPerWarp][kLdH];  // ping-pong activations per warp
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
  float scale, margin;  // bound = max(y, 0) * scale + margin
};

// one warp: out[32 x 128] = relu(in[32 x K] W + b), written as bf16 to `out`
// (or, for the last layer, folded into the head dot product)
template <int K, int LDA, int LDW>
__device__ __forceinline__ void warp_layer(const __nv_bfloat16 (*in)[kLdH], const __nv_bfloat16 (*w)[LDW],
                                           const float* b, __nv_bfloat16 (*out)[kLdH], const float* w4,
                                           float* head_rows, int lane) {
  const int gid = lane >> 2, tig = lane & 3;
  const __nv_bfloat16* inb = &in[0][0];
#pragma unroll
  for (int half = 0; half < 2; ++half) {
    float acc[2][8][4];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
      for (int j = 0; j < 8; ++j)
#pragma unroll
        for (int r = 0; r < 4; ++r) acc[i][j][r] = 0.f;
#pragma unroll
    for (int k0 = 0; k0 < K; k0 += 16) {
      uint32_t a[2][4];
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const int r = i * 16 + gid;
        a[i][0] = *reinterpret_cast<const uint32_t*>(inb + r * LDA + k0 + 2 * tig);
        a[i][1] = *reinterpret_cast<const uint32_t*>(inb + (r + 8) * LDA + k0 + 2 * tig);
        a[i][2] = *reinterpret_cast<const uint32_t*>(inb + r * LDA + k0 + 2 * tig + 8);
        a[i][3] = *reinterpret_cast<const uint32_t*>(inb + (r + 8) * LDA + k0 + 2 * tig + 8);
      }
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const int c = half * 64 + j * 8 + gid;
        uint32_t bb[2];
        bb[0] = *reinterpret_cast<const uint32_t*>(&w[c][k0 + 2 * tig]);
        bb[1] = *reinterpret_cast<const uint32_t*>(&w[c][k0 + 2 * tig + 8]);
        mma_bf16(acc[0][j], a[0], bb);
        mma_bf16(acc[1][j], a[1], bb);
      }
    }
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const int c = half * 64 + j * 8 + 2 * tig;
        const float v0 = fmaxf(acc[i][j][0] + b[c], 0.f), v1 = fmaxf(acc[i][j][1] + b[c + 1], 0.f);
        const float v2 = fmaxf(acc[i][j][2] + b[c], 0.f), v3 = fmaxf(acc[i][j][3] + b[c + 1], 0.f);
        const int r = i * 16 + gid;
        if (head_rows) {
          // last hidden layer: fold into the head, h rounded to bf16 like training
          const float h0 = __bfloat162float(__float2bfloat16(v0)), h1 = __bfloat162float(__float2bfloat16(v1));
          const float h2 = __bfloat162float(__float2bfloat16(v2)), h3 = __bfloat162float(__float2bfloat16(v3));
          head_rows[i * 2] += h0 * w4[c] + h1 * w4[c + 1];
          head_rows[i * 2 + 1] += h2 * w4[c] + h3 * w4[c + 1];
        } else {
          *reinterpret_cast<uint32_t*>(&out[r][c]) = pack_bf16(v0, v1);
          *reinterpret_cast<uint32_t*>(&out[r + 8][c]) = pack_bf16(v2, v3);
        }
      }
  }
}

__global__ void __launch_bounds__(kInfWarps * 32) mlp_bound_kernel(const float* __restrict__ x, int64_t n,
                                                                 InfParams p, float* __restrict__ bound) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  InfSmem& S = *reinterpret_cast<InfSmem*>(smem_raw);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  // weights into shared memory (padded rows)
  for (int e = tid; e < kHid * kIn; e += blockDim.x) S.w1t[e / kIn][e % kIn] = p.w1t[e];
  for (int e = tid; e < kHid * kHid; e += blockDim.x) {
    S.w2t[e / kHid][e % kHid] = p.w2t[e];
    S.w3t[e / kHid][e % kHid] = p.w3t[e];
  }
  for (int e = tid; e < kHid; e += blockDim.x) {
    S.b1[e] = p.b1[e]; S.b2[e] = p.b2[e]; S.b3[e] = p.b3[e]; S.w4[e] = p.w4[e];
  }
  for (int e = tid; e < kIn / 2 * 3; e += blockDim.x) S.freq[e] = p.freq[e];
  __syncthreads();
  const int64_t tiles = ceil_div(n, kRows);
  for (int64_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
    const int64_t r0 = tile * kRows + warp * kRowsPerWarp;
    // Fourier features of this warp's 32 queries (lane = query)
    {
      const int64_t q = r0 + lane;
      float px = 0.f, py = 0.f, pz = 0.f;
      if (q < n) { px = x[3 * q]; py = x[3 * q + 1]; pz = x[3 * q + 2]; }
      for (int j = 0; j < kIn / 2; ++j) {
        float s, c;
        fourier(px, py, pz, p.nz, S.freq, j, s, c);
        *reinterpret_cast<uint32_t*>(&S.act[warp][0][lane][2 * j]) = pack_bf16(s, c);
      }
    }
    __syncwarp();
    warp_layer<kIn, kLdH, kLd1>(S.act[warp][0], S.w1t, S.b1, S.act[warp][1], nullptr, nullptr, lane);
    __syncwarp();
    warp_layer<kHid, kLdH, kLdH>(S.act[warp][1], S.w2t, S.b2, S.act[warp][0], nullptr, nullptr, lane);
    __syncwarp();
    float head[4] = {0.f, 0.f, 0.f, 0.f};  // rows gid, gid+8, 16+gid, 24+gid
    warp_layer<kHid, kLdH, kLdH>(S.act[warp][0], S.w3t, S.b3, nullptr, S.w4, head, lane);
    // reduce the head's partial sums over the 4 lanes of a row group
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      head[r] += __shfl_xor_sync(0xffffffffu, head[r], 1);
      head[r] += __shfl_xor_sync(0xffffffffu, head[r], 2);
    }
    if ((lane & 3) == 0) {
      const int gid = lane >> 2;
      const int rows[4] = {gid, gid + 8, 16 + gid, 24 + gid};
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        const int64_t q = r0 + rows[r];
        if (q < n) bound[q] = fmaxf(head[r] + p.b4, 0.f) * p.scale + p.margin;
      }
    }
    __syncwarp();
  }
}

}  // namespace
}  // namespace a3d

using namespace a3d;

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
  const size_t smem = sizeof(InfSmem);
  // the shared-memory opt-in is a per-device setting
  static bool attr_set[kMaxDevices] = {false};
  int dev = 0;
  A3D_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices || !attr_set[dev]) {
    A3D_CUDA_TRY(cudaFuncSetAttribute(mlp_bound_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    if (dev >= 0 && dev < kMaxDevices) attr_set[dev] = true;
  }
  const int sms = num_sms();
  const int64_t tiles = ceil_div(n, kRows);
  const int64_t grid = tiles < (int64_t)sms ? tiles : (int64_t)sms;
  mlp_bound_kernel<<<(unsigned)grid, kInfWarps * 32, smem, (cudaStream_t)stream>>>(x, n, p, bound);
  A3D_LAUNCH_CHECK();
  return A3D_OK;
}
