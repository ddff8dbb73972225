// Device-wide building blocks written for this library: exclusive scan and a
// stable LSD radix sort (8-bit digits, warp-match ranking).  Used by the BVH
// build, the query sort, octree compaction, the flood-fill extraction and
// the DMC edge sort.
#pragma once

#include "a3d_common.cuh"

namespace a3d {

// ---------------------------------------------------------------------------
// warp / block scans
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ T warp_inclusive_scan(T v) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    T n = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += n;
  }
  return v;
}

template <typename T>
__device__ __forceinline__ T warp_reduce_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Block-wide exclusive scan for blockDim.x <= 1024 (multiple of 32).
// s_warp must hold kBlockScanSlots elements: one exclusive offset per warp
// and, in its own slot, the block total (with 32 warps the last warp's
// offset and the total would otherwise share a slot).  Returns the
// exclusive prefix; *total = block sum.
constexpr int kBlockScanSlots = 33;
template <typename T>
__device__ __forceinline__ T block_exclusive_scan(T v, T* s_warp, T* total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nwarps = blockDim.x >> 5;
  T inc = warp_inclusive_scan(v);
  if (lane == 31) s_warp[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    T w = lane < nwarps ? s_warp[lane] : T(0);
    T wi = warp_inclusive_scan(w);
    if (lane < nwarps) s_warp[lane] = wi - w;
    if (lane == nwarps - 1) s_warp[32] = wi;
  }
  __syncthreads();
  T res = inc - v + s_warp[warp];
  if (total) *total = s_warp[32];
  __syncthreads();
  return res;
}

// ---------------------------------------------------------------------------
// device-wide exclusive scan: reduce tiles -> scan tile sums -> scan tiles
// ---------------------------------------------------------------------------
constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

template <typename TIn, typename T>
__global__ void scan_tile_reduce_kernel(const TIn* __restrict__ in, int64_t n, T* __restrict__ tile_sums) {
  pdl_wait();
  __shared__ T s_warp[kBlockScanSlots];
  const int64_t base = (int64_t)blockIdx.x * kScanTile;
  T acc = 0;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    int64_t idx = base + (int64_t)i * kScanThreads + threadIdx.x;
    if (idx < n) acc += (T)in[idx];
  }
  T total;
  block_exclusive_scan<T>(acc, s_warp, &total);
  if (threadIdx.x == 0) tile_sums[blockIdx.x] = total;
}

// Single block: exclusive scan of tile sums in place, total -> *total.
template <typename T>
__global__ void scan_tile_sums_kernel(T* __restrict__ sums, int64_t nb, T* __restrict__ total) {
  pdl_wait();
  __shared__ T s_warp[kBlockScanSlots];
  const int64_t per = ceil_div(nb, (int64_t)blockDim.x);
  const int64_t lo = (int64_t)threadIdx.x * per;
  const int64_t hi = lo + per < nb ? lo + per : nb;
  T local = 0;
  for (int64_t i = lo; i < hi; ++i) local += sums[i];
  T tot;
  T run = block_exclusive_scan<T>(local, s_warp, &tot);
  for (int64_t i = lo; i < hi; ++i) {
    T v = sums[i];
    sums[i] = run;
    run += v;
  }
  if (threadIdx.x == 0 && total) *total = tot;
}

// The tile passes through shared memory: loaded and stored with consecutive
// threads on consecutive elements (coalesced), scanned with each thread
// owning kScanItems consecutive elements (one padding slot per 32 keeps the
// per-thread reads off a single bank).  out may alias in: a block reads its
// whole tile before writing it.
//
// kFused: tile_offsets holds the raw tile sums of scan_tile_reduce_kernel and
// each block adds up those before its own (at most kScanFuseTiles of them,
// read from L2), so the single-block scan of the tile sums is skipped; the
// last block writes the total.
__host__ __device__ constexpr int scan_pad(int i) { return i + (i >> 5); }
constexpr int64_t kScanFuseTiles = 2048;

template <typename TIn, typename T, bool kFused>
__global__ void scan_tile_down_kernel(const TIn* __restrict__ in, T* __restrict__ out, int64_t n,
                                      const T* __restrict__ tile_offsets, T* __restrict__ total) {
  pdl_wait();
  __shared__ T s_warp[kBlockScanSlots];
  __shared__ T s_tile[scan_pad(kScanTile)];
  const int64_t base = (int64_t)blockIdx.x * kScanTile;
  T offset;
  if constexpr (kFused) {
    T part = 0;
    for (int64_t b = threadIdx.x; b < (int64_t)blockIdx.x; b += kScanThreads) part += tile_offsets[b];
    block_exclusive_scan<T>(part, s_warp, &offset);
  } else {
    offset = tile_offsets[blockIdx.x];
  }
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    const int li = i * kScanThreads + threadIdx.x;
    const int64_t idx = base + li;
    s_tile[scan_pad(li)] = idx < n ? (T)in[idx] : T(0);
  }
  __syncthreads();
  // each thread owns kScanItems consecutive elements
  T vals[kScanItems];
  T acc = 0;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    vals[i] = s_tile[scan_pad(threadIdx.x * kScanItems + i)];
    acc += vals[i];
  }
  T tile_total;
  T run = block_exclusive_scan<T>(acc, s_warp, &tile_total) + offset;
  if (kFused && total && blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) *total = offset + tile_total;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    s_tile[scan_pad(threadIdx.x * kScanItems + i)] = run;
    run += vals[i];
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    const int li = i * kScanThreads + threadIdx.x;
    const int64_t idx = base + li;
    if (idx < n) out[idx] = s_tile[scan_pad(li)];
  }
}

inline size_t scan_workspace_elems(int64_t n) { return (size_t)ceil_div(n > 0 ? n : 1, kScanTile) + 1; }

// Exclusive scan of in[0..n) into out (may alias in).  tmp must hold
// scan_workspace_elems(n) elements of T; the total goes to total_dev on the
// device, or to tmp[num_tiles] when total_dev is null.  Up to
// kScanFuseTiles tiles (4M elements) the scan is two launches (tile sums,
// then the tiles with their offsets summed in each block), above it three
// (the tile sums scanned by one block in between).
template <typename TIn, typename T>
int device_exclusive_scan(const TIn* in, T* out, int64_t n, T* tmp, T* total_dev, cudaStream_t s) {
  if (n <= 0) {
    if (total_dev) A3D_CUDA_TRY(cudaMemsetAsync(total_dev, 0, sizeof(T), s));
    return A3D_OK;
  }
  const int64_t nb = ceil_div(n, kScanTile);
  // The down pass reads thread-contiguous items, the reduce pass strided
  // items: both cover the same tile so tile sums agree.
  // the passes back to back with programmatic dependent launch
  T* total = total_dev ? total_dev : tmp + nb;
  A3D_PDL(scan_tile_reduce_kernel<TIn, T>, dim3((unsigned)nb), dim3(kScanThreads), 0, s, in, n, tmp);
  if (nb <= kScanFuseTiles) {
    A3D_PDL((scan_tile_down_kernel<TIn, T, true>), dim3((unsigned)nb), dim3(kScanThreads), 0, s, in, out, n,
            (const T*)tmp, total);
  } else {
    A3D_PDL(scan_tile_sums_kernel<T>, dim3(1), dim3(1024), 0, s, tmp, nb, total);
    A3D_PDL((scan_tile_down_kernel<TIn, T, false>), dim3((unsigned)nb), dim3(kScanThreads), 0, s, in, out, n,
            (const T*)tmp, (T*)nullptr);
  }
  return A3D_OK;
}

// n copies of v at p, a grid-stride kernel launched with programmatic
// dependent launch (a memset between two kernels would break the chain)
template <typename T>
__global__ void fill_kernel(T* __restrict__ p, int64_t n, T v) {
  pdl_wait();
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    p[i] = v;
}

template <typename T>
int fill_async(T* p, int64_t n, T v, cudaStream_t s) {
  if (n <= 0) return A3D_OK;
  const int64_t want = ceil_div(n, 256);
  const int64_t cap = (int64_t)num_sms() * 8;
  A3D_PDL(fill_kernel<T>, dim3((unsigned)(want < cap ? want : cap)), dim3(256), 0, s, p, n, v);
  return A3D_OK;
}

// ---------------------------------------------------------------------------
// stable LSD radix sort of (key, uint32 value) pairs, 8-bit digits
// ---------------------------------------------------------------------------
constexpr int kRsThreads = 256;
constexpr int kRsItems = 16;
constexpr int kRsTile = kRsThreads * kRsItems;

template <typename K>
__global__ void __launch_bounds__(kRsThreads) rs_upsweep_kernel(const K* __restrict__ keys, int64_t n, int shift,
                                                                uint32_t* __restrict__ hist, int64_t num_tiles) {
  pdl_wait();
  __shared__ uint32_t s_hist[256];
  s_hist[threadIdx.x] = 0;
  __syncthreads();
  const int64_t base = (int64_t)blockIdx.x * kRsTile;
  const int lane = threadIdx.x & 31;
#pragma unroll 4
  for (int i = 0; i < kRsItems; ++i) {
    int64_t idx = base + (int64_t)i * kRsThreads + threadIdx.x;
    uint32_t d = idx < n ? (uint32_t)((keys[idx] >> shift) & 0xff) : 0x100u;
    unsigned peers = __match_any_sync(0xffffffffu, d);
    if (d < 256u && lane == __ffs(peers) - 1) atomicAdd(&s_hist[d], (uint32_t)__popc(peers));
  }
  __syncthreads();
  hist[(int64_t)threadIdx.x * num_tiles + blockIdx.x] = s_hist[threadIdx.x];
}

template <typename K>
__global__ void __launch_bounds__(kRsThreads)
    rs_downsweep_kernel(const K* __restrict__ keys_in, const uint32_t* __restrict__ vals_in, K* __restrict__ keys_out,
                        uint32_t* __restrict__ vals_out, int64_t n, int shift, const uint32_t* __restrict__ offsets,
                        int64_t num_tiles) {
  pdl_wait();
  __shared__ uint32_t s_base[256];
  __shared__ uint32_t s_warp[kRsThreads / 32][256];
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  s_base[t] = offsets[(int64_t)t * num_tiles + blockIdx.x];
  const int64_t base = (int64_t)blockIdx.x * kRsTile;
  for (int c = 0; c < kRsItems; ++c) {
#pragma unroll
    for (int w = 0; w < kRsThreads / 32; ++w) s_warp[w][t] = 0;
    __syncthreads();
    const int64_t idx = base + (int64_t)c * kRsThreads + t;
    const bool valid = idx < n;
    K k = 0;
    uint32_t v = 0, d = 0x100u;
    if (valid) {
      k = keys_in[idx];
      v = vals_in[idx];
      d = (uint32_t)((k >> shift) & 0xff);
    }
    const unsigned peers = __match_any_sync(0xffffffffu, d);
    const int rank = __popc(peers & ((1u << lane) - 1u));
    if (valid && lane == __ffs(peers) - 1) s_warp[warp][d] = (uint32_t)__popc(peers);
    __syncthreads();
    uint32_t run = s_base[t];
#pragma unroll
    for (int w = 0; w < kRsThreads / 32; ++w) {
      uint32_t cnt = s_warp[w][t];
      s_warp[w][t] = run;
      run += cnt;
    }
    s_base[t] = run;
    __syncthreads();
    if (valid) {
      const uint32_t pos = s_warp[warp][d] + (uint32_t)rank;
      keys_out[pos] = k;
      vals_out[pos] = v;
    }
    __syncthreads();
  }
}

inline int64_t radix_num_tiles(int64_t n) { return ceil_div(n > 0 ? n : 1, kRsTile); }
// uint32 elements of scratch needed by radix_sort_pairs
inline size_t radix_sort_scratch_elems(int64_t n) {
  const int64_t h = 256 * radix_num_tiles(n);
  return (size_t)h + scan_workspace_elems(h);
}

// Sorts (keys, vals) by bits [begin_bit, end_bit) of the key.  Ping-pongs
// between (keys, vals) and (keys_alt, vals_alt); *result_in_alt tells the
// caller which pair holds the sorted data.  n must be < 2^32.
template <typename K>
int radix_sort_pairs(K* keys, uint32_t* vals, K* keys_alt, uint32_t* vals_alt, int64_t n, int begin_bit,
                     int end_bit, uint32_t* scratch, bool* result_in_alt, cudaStream_t s) {
  *result_in_alt = false;
  if (n <= 1) return A3D_OK;
  A3D_REQUIRE(n < (int64_t)0xffffffffll, A3D_ERR_ARGUMENT, "radix sort: too many elements");
  const int64_t nt = radix_num_tiles(n);
  uint32_t* hist = scratch;
  uint32_t* tmp = scratch + 256 * nt;
  K *kin = keys, *kout = keys_alt;
  uint32_t *vin = vals, *vout = vals_alt;
  for (int shift = begin_bit; shift < end_bit; shift += 8) {
    A3D_PDL(rs_upsweep_kernel<K>, dim3((unsigned)nt), dim3(kRsThreads), 0, s, (const K*)kin, n, shift, hist, nt);
    A3D_TRY((device_exclusive_scan<uint32_t, uint32_t>(hist, hist, 256 * nt, tmp, (uint32_t*)nullptr, s)));
    A3D_PDL(rs_downsweep_kernel<K>, dim3((unsigned)nt), dim3(kRsThreads), 0, s, (const K*)kin, (const uint32_t*)vin,
            kout, vout, n, shift, (const uint32_t*)hist, nt);
    K* tk = kin; kin = kout; kout = tk;
    uint32_t* tv = vin; vin = vout; vout = tv;
    *result_in_alt = !*result_in_alt;
  }
  return A3D_OK;
}

__global__ void iota_u32_kernel(uint32_t* out, int64_t n);

}  // namespace a3d
