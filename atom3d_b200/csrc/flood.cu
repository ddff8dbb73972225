// Flood fill of the octree's dam voxels on a bit-packed crop, plus the dam
// neighbourhood classification.
//
// Replaces flood_fill_3d_sparse + flood_fill_kernel + the host BFS loop
// (atom3d/kernels/flood_fill.py:118-258, atom3d/kernels/flood_fill_kernels.cu:
// 21-175) and get_dam_neighborhood_signs (atom3d/apps/sparse_flood_fill.py:
// 34-100).  The reference's labels are set properties of the crop:
//   water W    the connected component (6/18/26-connectivity) of free voxels
//              containing the seed
//   collision  W voxels with an occupied neighbour
//   dam        occupied voxels with a W neighbour, plus (extension) occupied
//              voxels in the 6-cross (connectivity 6) or 3x3x3 (otherwise)
//              dilation of W
//   dry        everything else in the crop
// so they are computed here with bit operations instead of a BFS:
//   * volume: one bit per voxel, 32 z-voxels per word, rows (x, y) in raster
//     order, so extraction in word order is the reference's lexicographic
//     (x, y, z) nonzero order;
//   * W grows by monotone relaxation over 32x32-row bricks: a CTA loads its
//     brick and a one-row halo into shared memory and iterates (dilate in
//     x/y, flood whole free runs along z with a Kogge-Stone prefix) until
//     the brick is stable, then marks its neighbours dirty if it changed.
//     Bits only ever get set, so reading a neighbour's word while it is
//     being updated is safe; rounds repeat until no brick is dirty;
//   * labels and the k-ring dilation are word-parallel passes; one pass
//     counts every label per tile of kTileWords words (and in total), and a
//     label's coordinates are written by one block per tile after a scan of
//     that label's tile counts (words are ranked inside the tile).
#include <limits.h>

#include "primitives.cuh"

namespace a3d {
namespace {

constexpr int kBX = 32, kBY = 32;  // rows per brick (one word of 32 z each)

struct Geom {
  int nx, ny, nz, nw;      // volume size, words per row
  int vx, vy, vz;          // volume origin in grid coordinates
  int cx0, cy0, cz0;       // crop box (flood domain) in volume coordinates
  int cx1, cy1, cz1;       // inclusive
  int conn;
};

__device__ __forceinline__ int64_t widx(const Geom& g, int x, int y, int w) {
  return ((int64_t)x * g.ny + y) * g.nw + w;
}

// z bits of word w inside [lo, hi] (inclusive), volume coordinates
__device__ __forceinline__ uint32_t zmask(int w, int lo, int hi) {
  const int b0 = w * 32, b1 = b0 + 31;
  if (hi < b0 || lo > b1) return 0u;
  const int s = lo > b0 ? lo - b0 : 0;
  const int e = hi < b1 ? hi - b0 : 31;
  const uint32_t top = e == 31 ? 0xffffffffu : ((1u << (e + 1)) - 1u);
  return top & ~((1u << s) - 1u);
}

__device__ __forceinline__ uint32_t valid_mask(const Geom& g, int w) { return zmask(w, 0, g.nz - 1); }

__device__ __forceinline__ uint32_t crop_mask(const Geom& g, int x, int y, int w) {
  if (x < g.cx0 || x > g.cx1 || y < g.cy0 || y > g.cy1) return 0u;
  return zmask(w, g.cz0, g.cz1);
}

// all free bits connected (along z, inside this word) to a bit of r
__device__ __forceinline__ uint32_t fill_runs(uint32_t r, uint32_t f) {
  r &= f;
  uint32_t m = f;
  uint32_t u = r;
  u |= (u << 1) & m; m &= m << 1;
  u |= (u << 2) & m; m &= m << 2;
  u |= (u << 4) & m; m &= m << 4;
  u |= (u << 8) & m; m &= m << 8;
  u |= (u << 16) & m;
  m = f;
  uint32_t d = r;
  d |= (d >> 1) & m; m &= m >> 1;
  d |= (d >> 2) & m; m &= m >> 2;
  d |= (d >> 4) & m; m &= m >> 4;
  d |= (d >> 8) & m; m &= m >> 8;
  d |= (d >> 16) & m;
  return u | d;
}

// z-dilation of word c with its neighbours a (w-1) and b (w+1)
__device__ __forceinline__ uint32_t zdil(uint32_t a, uint32_t c, uint32_t b) {
  return c | (c << 1) | (c >> 1) | (a >> 31) | (b << 31);
}

__global__ void bbox_kernel(const int64_t* __restrict__ ijk, int64_t n, long long* __restrict__ bb) {
  pdl_wait();
  long long lo[3] = {LLONG_MAX, LLONG_MAX, LLONG_MAX}, hi[3] = {LLONG_MIN, LLONG_MIN, LLONG_MIN};
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const long long v = ijk[3 * i + a];
      lo[a] = v < lo[a] ? v : lo[a];
      hi[a] = v > hi[a] ? v : hi[a];
    }
  }
#pragma unroll
  for (int a = 0; a < 3; ++a) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const long long l = __shfl_xor_sync(0xffffffffu, lo[a], o), h = __shfl_xor_sync(0xffffffffu, hi[a], o);
      lo[a] = l < lo[a] ? l : lo[a];
      hi[a] = h > hi[a] ? h : hi[a];
    }
  }
  // one atomic per block and bound: warps meet in shared memory first
  __shared__ long long s_b[6][32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  if (lane == 0) {
    for (int a = 0; a < 3; ++a) {
      s_b[a][warp] = lo[a];
      s_b[3 + a][warp] = hi[a];
    }
  }
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      lo[a] = lane < nwarps ? s_b[a][lane] : LLONG_MAX;
      hi[a] = lane < nwarps ? s_b[3 + a][lane] : LLONG_MIN;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        const long long l = __shfl_xor_sync(0xffffffffu, lo[a], o), h = __shfl_xor_sync(0xffffffffu, hi[a], o);
        lo[a] = l < lo[a] ? l : lo[a];
        hi[a] = h > hi[a] ? h : hi[a];
      }
    }
    if (lane == 0) {
      for (int a = 0; a < 3; ++a) {
        atomicMin(&bb[a], lo[a]);
        atomicMax(&bb[3 + a], hi[a]);
      }
    }
  }
}

__global__ void set_bits_kernel(const int64_t* __restrict__ ijk, int64_t n, Geom g, uint32_t* __restrict__ vol) {
  pdl_wait();
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int x = (int)(ijk[3 * i] - g.vx), y = (int)(ijk[3 * i + 1] - g.vy), z = (int)(ijk[3 * i + 2] - g.vz);
  if (x < 0 || y < 0 || z < 0 || x >= g.nx || y >= g.ny || z >= g.nz) return;
  atomicOr(&vol[widx(g, x, y, z >> 5)], 1u << (z & 31));
}

// One relaxation round over the bricks queued for it: list `cur` with
// cnt[round % 3] entries, which the blocks stride over.  A brick whose water
// changed queues its 27 neighbours (itself included) for the next round,
// each once: mark[b] is the last round b was queued for, raised with
// atomicMax, and the first raiser appends b to `nxt` (count cnt[(round + 1)
// % 3]).  Block 0 clears cnt[(round + 2) % 3], the input count of the
// previous round, for the round after this one.  Rounds run back to back
// inside one kernel, so everything another block may have written in an
// earlier round (queue, counts, water) is read through L2 (ld.global.cg),
// never from a stale L1 line.
__device__ __forceinline__ void relax_round(const Geom& g, const uint32_t* __restrict__ occ, uint32_t* water,
                                            const uint32_t* cur, uint32_t* nxt, uint32_t* __restrict__ mark,
                                            uint32_t* cnt, int round, int nbx, int nby, int max_iters,
                                            uint32_t (*s_r)[kBX + 2][kBY + 2]) {
  const uint32_t nbricks = (uint32_t)nbx * (uint32_t)nby * (uint32_t)g.nw;
  const uint32_t n_cur = min(__ldcg(cnt + round % 3), nbricks);
  if (blockIdx.x == 0 && threadIdx.x == 0) cnt[(round + 2) % 3] = 0u;
  const uint32_t next_round = (uint32_t)round + 1u;
  for (uint32_t item = blockIdx.x; item < n_cur; item += gridDim.x) {
    const int bid = (int)__ldcg(cur + item);
    const int bw = bid / (nbx * nby);
    const int rem = bid % (nbx * nby);
    const int bxi = rem / nby, byi = rem % nby;
    const int x0 = bxi * kBX, y0 = byi * kBY;
    const int tx = threadIdx.x / kBY, ty = threadIdx.x % kBY;
    // load the halo'd water words (monotone: a racing update is harmless)
    for (int i = threadIdx.x; i < 3 * (kBX + 2) * (kBY + 2); i += blockDim.x) {
      const int k = i / ((kBX + 2) * (kBY + 2));
      const int r2 = i % ((kBX + 2) * (kBY + 2));
      const int hx = r2 / (kBY + 2), hy = r2 % (kBY + 2);
      const int x = x0 + hx - 1, y = y0 + hy - 1, w = bw + k - 1;
      uint32_t v = 0;
      if (x >= 0 && x < g.nx && y >= 0 && y < g.ny && w >= 0 && w < g.nw) v = __ldcg(&water[widx(g, x, y, w)]);
      s_r[k][hx][hy] = v;
    }
    const int x = x0 + tx, y = y0 + ty;
    const bool inside = x < g.nx && y < g.ny;
    uint32_t f = 0;
    if (inside) f = ~occ[widx(g, x, y, bw)] & crop_mask(g, x, y, bw);
    __syncthreads();
    const uint32_t orig = s_r[1][tx + 1][ty + 1];
    for (int it = 0; it < max_iters; ++it) {
      uint32_t acc = 0;
      const uint32_t self = s_r[1][tx + 1][ty + 1];
      // neighbours along z of this row (words of the adjacent bricks)
      acc |= (s_r[0][tx + 1][ty + 1] >> 31) | (s_r[2][tx + 1][ty + 1] << 31);
  #pragma unroll
      for (int dx = -1; dx <= 1; ++dx) {
  #pragma unroll
        for (int dy = -1; dy <= 1; ++dy) {
          if (dx == 0 && dy == 0) continue;
          const int l1 = (dx != 0) + (dy != 0);
          const uint32_t a = s_r[0][tx + 1 + dx][ty + 1 + dy];
          const uint32_t c = s_r[1][tx + 1 + dx][ty + 1 + dy];
          const uint32_t b = s_r[2][tx + 1 + dx][ty + 1 + dy];
          if (g.conn == 6) {
            if (l1 == 1) acc |= c;
          } else if (g.conn == 18) {
            acc |= (l1 == 1) ? zdil(a, c, b) : c;
          } else {
            acc |= zdil(a, c, b);
          }
        }
      }
      const uint32_t nw = inside ? fill_runs(self | (acc & f), f) | self : self;
      const bool ch = nw != self;
      if (ch) s_r[1][tx + 1][ty + 1] = nw;
      if (!__syncthreads_or(ch)) break;
    }
    const uint32_t fin = s_r[1][tx + 1][ty + 1];
    if (inside && fin != orig) water[widx(g, x, y, bw)] = fin;
    // the barrier also ends this brick's reads of s_r before the next item's
    // halo load
    if (__syncthreads_or(inside && fin != orig)) {
      if (threadIdx.x < 27) {
        const int dz = threadIdx.x / 9 - 1, dxx = (threadIdx.x / 3) % 3 - 1, dyy = threadIdx.x % 3 - 1;
        const int nbw = bw + dz, nbxx = bxi + dxx, nbyy = byi + dyy;
        if (nbw >= 0 && nbw < g.nw && nbxx >= 0 && nbxx < nbx && nbyy >= 0 && nbyy < nby) {
          const uint32_t nb = (uint32_t)((nbw * nbx + nbxx) * nby + nbyy);
          if (atomicMax(&mark[nb], next_round) < next_round) {
            const uint32_t slot = atomicAdd(&cnt[(round + 1) % 3], 1u);
            if (slot < nbricks) nxt[slot] = nb;
          }
        }
      }
    }
  }
}

// Grid-wide barrier of a cooperative launch (every block resident): bar[0]
// counts arrivals, bar[1] is the generation the last arrival advances.  A
// block reads the generation before it arrives, so the advance cannot be
// missed; the waiting spins are bounded (about a second), after which the
// barrier reports failure instead of waiting on.
constexpr uint32_t kBarrierSpins = 1u << 24;
__device__ __forceinline__ bool grid_barrier(uint32_t* bar) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile uint32_t* vgen = bar + 1;
    const uint32_t gen = *vgen;
    __threadfence();
    bool ok = true;
    if (atomicAdd(bar, 1u) == gridDim.x - 1) {
      atomicExch(bar, 0u);
      __threadfence();
      atomicAdd(bar + 1, 1u);
    } else {
      for (uint32_t spins = 0; *vgen == gen; ++spins) {
        if (spins >= kBarrierSpins) {
          ok = false;
          break;
        }
        __nanosleep(64);
      }
    }
    __threadfence();
    s_ok = ok ? 1 : 0;
  }
  __syncthreads();
  return s_ok != 0;
}

// All relaxation rounds in one cooperative launch of the resident blocks:
// round r relaxes the bricks queued for it, a grid barrier closes the round,
// and every block reads the next queue's length after the barrier, so all
// blocks stop together when it is empty.  sync: [0..1] barrier words, [2]
// status (bit 0: the round cap was reached with bricks still queued, bit 1:
// a barrier wait ran out), [3] the number of rounds run.
__global__ void __launch_bounds__(kBX * kBY)
    flood_rounds_kernel(Geom g, const uint32_t* __restrict__ occ, uint32_t* water, uint32_t* list_a, uint32_t* list_b,
                        uint32_t* __restrict__ mark, uint32_t* cnt, int nbx, int nby, int max_iters, int max_rounds,
                        uint32_t* sync) {
  pdl_wait();
  __shared__ uint32_t s_r[3][kBX + 2][kBY + 2];  // words w-1, w, w+1 of the rows with halo
  int round = 0;
  for (;;) {
    const uint32_t* cur = (round & 1) ? list_b : list_a;
    uint32_t* nxt = (round & 1) ? list_a : list_b;
    relax_round(g, occ, water, cur, nxt, mark, cnt, round, nbx, nby, max_iters, s_r);
    const bool ok = grid_barrier(sync);
    ++round;
    if (!ok) {
      if (threadIdx.x == 0) atomicOr(sync + 2, 2u);
      break;
    }
    if (__ldcg(cnt + round % 3) == 0u) break;
    if (round >= max_rounds) {
      if (blockIdx.x == 0 && threadIdx.x == 0) atomicOr(sync + 2, 1u);
      break;
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) sync[3] = (uint32_t)round;
}

// label volumes.  slot order: 0 water(pure) 1 dry 2 tide(collision) 3 dam
// 4 extended dam 5 extended tide 6 dry adjacent 7 ring (scratch)
enum { kWater = 0, kDry = 1, kTide = 2, kDam = 3, kExt = 4, kExtTide = 5, kDryAdj = 6, kRing = 7, kLabels = 8 };

template <int kConn>
__device__ __forceinline__ uint32_t dil_conn(const uint32_t* __restrict__ v, const Geom& g, int x, int y, int w) {
  uint32_t acc = 0;
  auto word = [&](int xx, int yy, int ww) -> uint32_t {
    if (xx < 0 || yy < 0 || ww < 0 || xx >= g.nx || yy >= g.ny || ww >= g.nw) return 0u;
    return v[widx(g, xx, yy, ww)];
  };
  const uint32_t c0 = word(x, y, w);
  acc |= (c0 << 1) | (c0 >> 1) | (word(x, y, w - 1) >> 31) | (word(x, y, w + 1) << 31);
#pragma unroll
  for (int dx = -1; dx <= 1; ++dx)
#pragma unroll
    for (int dy = -1; dy <= 1; ++dy) {
      if (dx == 0 && dy == 0) continue;
      const int l1 = (dx != 0) + (dy != 0);
      if (kConn == 6 && l1 != 1) continue;
      const uint32_t c = word(x + dx, y + dy, w);
      if (kConn == 6 || (kConn == 18 && l1 == 2)) {
        acc |= c;
      } else {
        acc |= zdil(word(x + dx, y + dy, w - 1), c, word(x + dx, y + dy, w + 1));
      }
    }
  return acc;
}

__global__ void labels_kernel(Geom g, const uint32_t* __restrict__ occ, const uint32_t* __restrict__ water,
                              uint32_t* __restrict__ lab, int64_t nwords) {
  pdl_wait();
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nwords) return;
  const int w = (int)(i % g.nw);
  const int64_t row = i / g.nw;
  const int y = (int)(row % g.ny), x = (int)(row / g.ny);
  const uint32_t crop = crop_mask(g, x, y, w);
  const uint32_t o = occ[i] & crop, r = water[i] & crop;
  uint32_t near_occ, near_w;
  if (g.conn == 6) {
    near_occ = dil_conn<6>(occ, g, x, y, w);
    near_w = dil_conn<6>(water, g, x, y, w);
  } else if (g.conn == 18) {
    near_occ = dil_conn<18>(occ, g, x, y, w);
    near_w = dil_conn<18>(water, g, x, y, w);
  } else {
    near_occ = dil_conn<26>(occ, g, x, y, w);
    near_w = dil_conn<26>(water, g, x, y, w);
  }
  const uint32_t near_w_ext = g.conn == 6 ? near_w : (g.conn == 18 ? dil_conn<26>(water, g, x, y, w) : near_w);
  const uint32_t tide = r & near_occ;
  const uint32_t dam0 = o & near_w;
  const uint32_t ext = o & ~dam0 & near_w_ext;
  const uint32_t dam = dam0 | ext;
  const int64_t nwv = nwords;
  lab[kWater * nwv + i] = r & ~tide;
  lab[kTide * nwv + i] = tide;
  lab[kDam * nwv + i] = dam;
  lab[kExt * nwv + i] = ext;
  lab[kDry * nwv + i] = crop & ~r & ~dam;
}

// 3x3x3 box dilation of src into dst (one ring of get_dam_neighborhood_signs)
__global__ void box_dilate_kernel(Geom g, const uint32_t* __restrict__ src, uint32_t* __restrict__ dst,
                                  int64_t nwords) {
  pdl_wait();
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nwords) return;
  const int w = (int)(i % g.nw);
  const int64_t row = i / g.nw;
  const int y = (int)(row % g.ny), x = (int)(row / g.ny);
  dst[i] = (src[i] | dil_conn<26>(src, g, x, y, w)) & valid_mask(g, w);
}

__global__ void ring_classify_kernel(const uint32_t* __restrict__ ring, uint32_t* __restrict__ lab, int64_t nwords) {
  pdl_wait();
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nwords) return;
  const uint32_t n = ring[i];
  const uint32_t dam = lab[kDam * nwords + i], dry = lab[kDry * nwords + i];
  lab[kExtTide * nwords + i] = n & ~dam & ~dry;
  lab[kDryAdj * nwords + i] = n & dry & ~dam;
}

// A tile is kTileWords consecutive words: 256 threads, each warp owning
// kTileWords / 8 consecutive words in chunks of 32 (one word per lane).
constexpr int kTileThreads = 256;
constexpr int kTileWords = 2048;
constexpr int kTileChunks = kTileWords / kTileThreads;  // chunks of 32 words per warp

// set voxels of every label per tile (label-major [kRing][ntiles]) and per
// label in total
__global__ void __launch_bounds__(kTileThreads) tile_counts_kernel(const uint32_t* __restrict__ lab, int64_t nwords,
                                                                   int64_t ntiles, uint32_t* __restrict__ tcnt,
                                                                   unsigned long long* __restrict__ tot) {
  pdl_wait();
  __shared__ uint32_t s_part[kRing][kTileThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t base = (int64_t)blockIdx.x * kTileWords;
#pragma unroll 1
  for (int k = 0; k < kRing; ++k) {
    const uint32_t* v = lab + (int64_t)k * nwords;
    uint32_t c = 0;
#pragma unroll
    for (int j = 0; j < kTileChunks; ++j) {
      const int64_t i = base + (int64_t)j * kTileThreads + threadIdx.x;
      if (i < nwords) c += (uint32_t)__popc(v[i]);
    }
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) c += __shfl_xor_sync(0xffffffffu, c, d);
    if (lane == 0) s_part[k][warp] = c;
  }
  __syncthreads();
  if (threadIdx.x < kRing) {
    uint32_t c = 0;
#pragma unroll
    for (int w = 0; w < kTileThreads / 32; ++w) c += s_part[threadIdx.x][w];
    tcnt[threadIdx.x * ntiles + blockIdx.x] = c;
    if (c) atomicAdd(&tot[threadIdx.x], (unsigned long long)c);
  }
}

// One block per tile.  Each lane takes one word per chunk and ranks it in
// the tile (warp scans of popcounts, then the warps' totals); then, for each
// non-empty word of a chunk, the 32 lanes take its 32 bits, so the set
// voxels' coordinates are written as one contiguous run in the word's bit
// order -- lexicographic (x, y, z) overall.  Positions at or past `count`
// are not written.  Needs nwords < 2^32 (word coordinates in 32 bits).
__global__ void __launch_bounds__(kTileThreads) extract_tile_kernel(Geom g, const uint32_t* __restrict__ v,
                                                                    const int64_t* __restrict__ toff, int64_t nwords,
                                                                    int64_t count, int32_t* __restrict__ out) {
  pdl_wait();
  __shared__ uint32_t s_warp[kTileThreads / 32];
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const unsigned lt = (1u << lane) - 1u;
  const int64_t base = (int64_t)blockIdx.x * kTileWords + (int64_t)warp * (kTileChunks * 32);
  uint32_t word[kTileChunks], incl[kTileChunks];
  uint32_t run = 0;
#pragma unroll
  for (int c = 0; c < kTileChunks; ++c) {
    const int64_t i = base + c * 32 + lane;
    word[c] = i < nwords ? v[i] : 0u;
    uint32_t p = (uint32_t)__popc(word[c]);
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const uint32_t t = __shfl_up_sync(FULL, p, d);
      if (lane >= d) p += t;
    }
    incl[c] = run + p;
    run += __shfl_sync(FULL, p, 31);
  }
  if (lane == 0) s_warp[warp] = run;
  __syncthreads();
  uint32_t before = 0;
  for (int w = 0; w < warp; ++w) before += s_warp[w];
  const int64_t start = toff[blockIdx.x] + before;
#pragma unroll
  for (int c = 0; c < kTileChunks; ++c) {
    unsigned nz = __ballot_sync(FULL, word[c] != 0u);
    if (!nz) continue;
    const uint32_t i = (uint32_t)(base + c * 32 + lane);
    const uint32_t row = i / (uint32_t)g.nw;
    const int wz = (int)(i - row * (uint32_t)g.nw);
    const int y = (int)(row % (uint32_t)g.ny), x = (int)(row / (uint32_t)g.ny);
    const uint32_t excl = incl[c] - (uint32_t)__popc(word[c]);
    while (nz) {
      const int j = __ffs(nz) - 1;
      nz &= nz - 1u;
      const uint32_t m = __shfl_sync(FULL, word[c], j);
      const uint32_t e = __shfl_sync(FULL, excl, j);
      const int xx = __shfl_sync(FULL, x, j), yy = __shfl_sync(FULL, y, j), ww = __shfl_sync(FULL, wz, j);
      const int64_t pos = start + e + __popc(m & lt);
      if (((m >> lane) & 1u) && pos < count) {
        int32_t* p = out + 3 * pos;
        p[0] = xx + g.vx;
        p[1] = yy + g.vy;
        p[2] = ww * 32 + lane + g.vz;
      }
    }
  }
}

__global__ void test_bits_kernel(Geom g, const uint32_t* __restrict__ v, const int64_t* __restrict__ ijk, int64_t n,
                                 uint8_t* __restrict__ out) {
  pdl_wait();
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int x = (int)(ijk[3 * i] - g.vx), y = (int)(ijk[3 * i + 1] - g.vy), z = (int)(ijk[3 * i + 2] - g.vz);
  uint8_t r = 0;
  if (x >= 0 && y >= 0 && z >= 0 && x < g.nx && y < g.ny && z < g.nz)
    r = (uint8_t)((v[widx(g, x, y, z >> 5)] >> (z & 31)) & 1u);
  out[i] = r;
}

// plants the seed voxel and queues its brick for round 0 (list[0], cnt[0]);
// status: 1 when the seed is occupied
__global__ void seed_kernel(Geom g, const uint32_t* __restrict__ occ, uint32_t* __restrict__ water, int sx, int sy,
                            int sz, uint32_t seed_brick, uint32_t* __restrict__ list, uint32_t* __restrict__ cnt,
                            uint32_t* __restrict__ status) {
  pdl_wait();
  const int64_t i = widx(g, sx, sy, sz >> 5);
  const uint32_t bit = 1u << (sz & 31);
  if (occ[i] & bit) {
    status[0] = 1u;  // seed occupied
  } else {
    water[i] |= bit;
    list[0] = seed_brick;
    cnt[0] = 1u;
    status[0] = 0u;
  }
}

// sign of each listed voxel (get_dam_neighborhood_signs priority: dam 0,
// then water +1, then dry -1, else +1), read from the membership volumes
__global__ void ring_sign_kernel(Geom g, const uint32_t* __restrict__ dam, const uint32_t* __restrict__ water,
                                 const uint32_t* __restrict__ dry, const int32_t* __restrict__ ijk, int64_t n,
                                 int8_t* __restrict__ sign) {
  pdl_wait();
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int x = ijk[3 * i] - g.vx, y = ijk[3 * i + 1] - g.vy, z = ijk[3 * i + 2] - g.vz;
  int8_t r = 1;
  if (x >= 0 && y >= 0 && z >= 0 && x < g.nx && y < g.ny && z < g.nz) {
    const int64_t k = widx(g, x, y, z >> 5);
    const uint32_t bit = 1u << (z & 31);
    if (dam[k] & bit) r = 0;
    else if (water[k] & bit) r = 1;
    else if (dry[k] & bit) r = -1;
  }
  sign[i] = r;
}

}  // namespace
}  // namespace a3d

using namespace a3d;

namespace {
Geom to_geom(const a3d_flood_geom* p) {
  Geom g;
  g.nx = p->vol_dims[0]; g.ny = p->vol_dims[1]; g.nz = p->vol_dims[2];
  g.nw = (g.nz + 31) / 32;
  g.vx = (int)p->vol_lo[0]; g.vy = (int)p->vol_lo[1]; g.vz = (int)p->vol_lo[2];
  g.cx0 = (int)(p->crop_lo[0] - p->vol_lo[0]); g.cy0 = (int)(p->crop_lo[1] - p->vol_lo[1]);
  g.cz0 = (int)(p->crop_lo[2] - p->vol_lo[2]);
  g.cx1 = (int)(p->crop_hi[0] - p->vol_lo[0]); g.cy1 = (int)(p->crop_hi[1] - p->vol_lo[1]);
  g.cz1 = (int)(p->crop_hi[2] - p->vol_lo[2]);
  g.conn = p->connectivity;
  return g;
}

struct FloodWs {
  uint32_t* occ;
  uint32_t* water;
  uint32_t* lab;     // kLabels volumes
  uint32_t* ring2;   // second ring buffer
  uint32_t* mark;    // [nbricks] last round each brick was queued for
  uint32_t* list_a;  // [nbricks] bricks queued for even rounds
  uint32_t* list_b;  // [nbricks] odd rounds
  uint32_t* tcnt;    // [kRing][ntiles] voxels per label and tile
  int64_t* toff;     // [ntiles + 1] one label's tile offsets
  int64_t* scan_tmp;
  uint32_t* misc;    // [0] seed status [2..4] queue counts (round % 3) [8..21] label totals (u64)
};

int64_t tiles_of(const Geom& g) { return ceil_div((int64_t)g.nx * g.ny * g.nw, kTileWords); }

size_t carve_flood(FloodWs& w, Workspace& ws, const Geom& g) {
  const int64_t nwords = (int64_t)g.nx * g.ny * g.nw;
  const int64_t nbricks = (int64_t)ceil_div(g.nx, kBX) * ceil_div(g.ny, kBY) * g.nw;
  w.occ = ws.take<uint32_t>(nwords);
  w.water = ws.take<uint32_t>(nwords);
  w.lab = ws.take<uint32_t>(kLabels * nwords);
  w.ring2 = ws.take<uint32_t>(nwords);
  w.mark = ws.take<uint32_t>(nbricks);
  w.list_a = ws.take<uint32_t>(nbricks);
  w.list_b = ws.take<uint32_t>(nbricks);
  const int64_t ntiles = tiles_of(g);
  w.tcnt = ws.take<uint32_t>(kRing * ntiles);
  w.toff = ws.take<int64_t>(ntiles + 1);
  w.scan_tmp = ws.take<int64_t>((int64_t)scan_workspace_elems(ntiles));
  w.misc = ws.take<uint32_t>(32);
  return ws.used;
}
}  // namespace

extern "C" int a3d_flood_bbox(const int64_t* ijk, int64_t n, int64_t* bbox_out, void* workspace,
                              size_t workspace_bytes, a3d_stream_t stream) {
  cudaStream_t s = (cudaStream_t)stream;
  A3D_REQUIRE(n > 0 && ijk && bbox_out, A3D_ERR_ARGUMENT, "flood_bbox: empty input");
  A3D_REQUIRE(workspace && workspace_bytes >= 6 * sizeof(long long), A3D_ERR_WORKSPACE, "flood_bbox: workspace");
  long long init[6] = {LLONG_MAX, LLONG_MAX, LLONG_MAX, LLONG_MIN, LLONG_MIN, LLONG_MIN};
  long long* bb = (long long*)workspace;
  A3D_CUDA_TRY(cudaMemcpyAsync(bb, init, sizeof(init), cudaMemcpyHostToDevice, s));
  const int64_t blocks = ceil_div(n, 256) < 4096 ? ceil_div(n, 256) : 4096;
  A3D_PDL(bbox_kernel, dim3((unsigned)blocks), dim3(256), 0, s, ijk, n, bb);
  long long h[6];
  A3D_CUDA_TRY(cudaMemcpyAsync(h, bb, sizeof(h), cudaMemcpyDeviceToHost, s));
  A3D_CUDA_TRY(cudaStreamSynchronize(s));
  for (int a = 0; a < 6; ++a) bbox_out[a] = h[a];
  return A3D_OK;
}

extern "C" size_t a3d_flood_workspace_bytes(const a3d_flood_geom* geom) {
  if (!geom) return 0;
  Geom g = to_geom(geom);
  Workspace ws(nullptr, 0);
  FloodWs w;
  return carve_flood(w, ws, g) + 256;
}

extern "C" int a3d_flood_fill(const int64_t* dam_ijk, int64_t n, const a3d_flood_geom* geom, void* workspace,
                              size_t workspace_bytes, int64_t* counts_out, int* rounds_out, a3d_stream_t stream) {
  cudaStream_t s = (cudaStream_t)stream;
  A3D_REQUIRE(geom && counts_out, A3D_ERR_ARGUMENT, "flood_fill: null argument");
  const int conn = geom->connectivity;
  A3D_REQUIRE(conn == 6 || conn == 18 || conn == 26, A3D_ERR_ARGUMENT, "flood_fill: connectivity must be 6, 18 or 26");
  A3D_REQUIRE(geom->k_ring >= 0, A3D_ERR_ARGUMENT, "flood_fill: k_ring must be >= 0");
  Geom g = to_geom(geom);
  A3D_REQUIRE(g.nx > 0 && g.ny > 0 && g.nz > 0, A3D_ERR_ARGUMENT, "flood_fill: empty volume");
  A3D_REQUIRE((int64_t)g.nx * g.ny * g.nw < (1ll << 32), A3D_ERR_ARGUMENT,
              "flood_fill: volume above 2^37 voxels (2^32 words)");
  Workspace ws(workspace, workspace_bytes);
  FloodWs w;
  carve_flood(w, ws, g);
  A3D_REQUIRE(workspace && ws.ok(), A3D_ERR_WORKSPACE, "flood_fill: workspace too small");
  const int64_t nwords = (int64_t)g.nx * g.ny * g.nw;
  const int nbx = (int)ceil_div(g.nx, kBX), nby = (int)ceil_div(g.ny, kBY);
  const int64_t nbricks = (int64_t)nbx * nby * g.nw;
  for (int k = 0; k < kLabels; ++k) counts_out[k] = 0;
  A3D_CUDA_TRY(cudaMemsetAsync(w.occ, 0, nwords * 4, s));
  A3D_CUDA_TRY(cudaMemsetAsync(w.water, 0, nwords * 4, s));
  A3D_CUDA_TRY(cudaMemsetAsync(w.misc, 0, 32 * sizeof(uint32_t), s));
  if (n > 0) {
    A3D_PDL(set_bits_kernel, dim3((unsigned)ceil_div(n, 256)), dim3(256), 0, s, dam_ijk, n, g, w.occ);
  }
  const int sx = (int)(geom->seed[0] - geom->vol_lo[0]), sy = (int)(geom->seed[1] - geom->vol_lo[1]),
            sz = (int)(geom->seed[2] - geom->vol_lo[2]);
  A3D_REQUIRE(sx >= g.cx0 && sx <= g.cx1 && sy >= g.cy0 && sy <= g.cy1 && sz >= g.cz0 && sz <= g.cz1,
              A3D_ERR_ARGUMENT, "flood_fill: seed outside the crop");
  // the queue of round 0 is the seed's brick; misc (queue counts included)
  // was cleared above and mark starts at round 0 for every brick
  const int64_t sb = ((int64_t)(sz >> 5) * nbx + sx / kBX) * nby + sy / kBY;
  uint32_t* qcnt = w.misc + 2;
  A3D_CUDA_TRY(cudaMemsetAsync(w.mark, 0, nbricks * sizeof(uint32_t), s));
  A3D_PDL(seed_kernel, dim3(1), dim3(1), 0, s, g, w.occ, w.water, sx, sy, sz, (uint32_t)sb, w.list_a, qcnt, w.misc);
  uint32_t seed_status = 0;
  A3D_CUDA_TRY(cudaMemcpyAsync(&seed_status, w.misc, 4, cudaMemcpyDeviceToHost, s));
  A3D_CUDA_TRY(cudaStreamSynchronize(s));
  if (seed_status) {
    counts_out[kLabels] = 1;  // seed occupied: empty result, like the reference
    return A3D_OK;
  }
  counts_out[kLabels] = 0;
  // Relaxation rounds over queued bricks, all in one cooperative launch of
  // the resident blocks (they stride over each round's queue, so a round
  // costs what its queue holds); the rounds end on the device when the next
  // queue is empty, and one host read takes the status and the round count.
  int dev = 0, sms = 0, per_sm = 0, coop = 0;
  A3D_CUDA_TRY(cudaGetDevice(&dev));
  A3D_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  A3D_CUDA_TRY(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
  A3D_REQUIRE(coop != 0, A3D_ERR_CUDA, "a3d_flood_fill: the device does not support cooperative launches");
  A3D_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, flood_rounds_kernel, kBX * kBY, 0));
  const int64_t resident = (int64_t)(sms > 0 ? sms : 1) * (per_sm > 0 ? per_sm : 1);
  const unsigned grid = (unsigned)(nbricks < resident ? nbricks : resident);
  // barrier, status and round words: misc[24..27] (cleared with misc
  // above; misc[8..21] collects the label totals below)
  uint32_t* sync = w.misc + 24;
  int max_rounds = 1 << 20;
  int max_iters = 4 * (kBX + kBY);
  void* args[] = {(void*)&g, (void*)&w.occ, (void*)&w.water, (void*)&w.list_a, (void*)&w.list_b, (void*)&w.mark,
                  (void*)&qcnt, (void*)&nbx, (void*)&nby, (void*)&max_iters, (void*)&max_rounds, (void*)&sync};
  A3D_CUDA_TRY(cudaLaunchCooperativeKernel((const void*)flood_rounds_kernel, dim3(grid), dim3(kBX * kBY), args, 0,
                                           s));
  uint32_t hs[2] = {0, 0};
  A3D_CUDA_TRY(cudaMemcpyAsync(hs, sync + 2, sizeof(hs), cudaMemcpyDeviceToHost, s));
  A3D_CUDA_TRY(cudaStreamSynchronize(s));
  A3D_REQUIRE(!(hs[0] & 2u), A3D_ERR_TIMEOUT, "a3d_flood_fill: a grid barrier of the relaxation timed out");
  // bricks still queued after the round cap: the water is incomplete
  A3D_REQUIRE(!(hs[0] & 1u), A3D_ERR_OVERFLOW, "a3d_flood_fill: relaxation did not converge within 2^20 rounds");
  const int rounds = (int)hs[1];
  if (rounds_out) *rounds_out = rounds;
  const unsigned gw = (unsigned)ceil_div(nwords, 256);
  A3D_PDL(labels_kernel, dim3(gw), dim3(256), 0, s, g, w.occ, w.water, w.lab, nwords);
  // k-ring box dilation of the dam, ping-ponging ring buffers
  uint32_t* ring_a = w.lab + (int64_t)kRing * nwords;
  A3D_CUDA_TRY(cudaMemcpyAsync(ring_a, w.lab + (int64_t)kDam * nwords, nwords * 4, cudaMemcpyDeviceToDevice, s));
  uint32_t* ring_b = w.ring2;
  for (int k = 0; k < geom->k_ring; ++k) {
    A3D_PDL(box_dilate_kernel, dim3(gw), dim3(256), 0, s, g, ring_a, ring_b, nwords);
    uint32_t* t = ring_a; ring_a = ring_b; ring_b = t;
  }
  A3D_PDL(ring_classify_kernel, dim3(gw), dim3(256), 0, s, ring_a, w.lab, nwords);
  // counts per label and tile, one pass and one host read
  const int64_t ntiles = tiles_of(g);
  unsigned long long* tot = reinterpret_cast<unsigned long long*>(w.misc + 8);
  A3D_PDL(tile_counts_kernel, dim3((unsigned)ntiles), dim3(kTileThreads), 0, s, w.lab, nwords, ntiles, w.tcnt, tot);
  unsigned long long h[kRing];
  A3D_CUDA_TRY(cudaMemcpyAsync(h, tot, sizeof(h), cudaMemcpyDeviceToHost, s));
  A3D_CUDA_TRY(cudaStreamSynchronize(s));
  for (int k = 0; k < kRing; ++k) counts_out[k] = (int64_t)h[k];
  return A3D_OK;
}

extern "C" int a3d_flood_extract(const a3d_flood_geom* geom, void* workspace, size_t workspace_bytes, int label,
                                 int32_t* out_ijk, int64_t count, a3d_stream_t stream) {
  cudaStream_t s = (cudaStream_t)stream;
  A3D_REQUIRE(geom && label >= 0 && label < kRing, A3D_ERR_ARGUMENT, "flood_extract: bad label");
  Geom g = to_geom(geom);
  Workspace ws(workspace, workspace_bytes);
  FloodWs w;
  carve_flood(w, ws, g);
  A3D_REQUIRE(workspace && ws.ok(), A3D_ERR_WORKSPACE, "flood_extract: workspace too small");
  if (count == 0) return A3D_OK;
  A3D_REQUIRE(out_ijk, A3D_ERR_ARGUMENT, "flood_extract: null output");
  const int64_t nwords = (int64_t)g.nx * g.ny * g.nw;
  const int64_t ntiles = tiles_of(g);
  const uint32_t* v = w.lab + (int64_t)label * nwords;
  A3D_TRY((device_exclusive_scan<uint32_t, int64_t>(w.tcnt + (int64_t)label * ntiles, w.toff, ntiles, w.scan_tmp,
                                                     w.toff + ntiles, s)));
  A3D_PDL(extract_tile_kernel, dim3((unsigned)ntiles), dim3(kTileThreads), 0, s, g, v, w.toff, nwords, count, out_ijk);
  return A3D_OK;
}

extern "C" int a3d_flood_test(const a3d_flood_geom* geom, void* workspace, size_t workspace_bytes, int label,
                              const int64_t* ijk, int64_t n, uint8_t* out, a3d_stream_t stream) {
  cudaStream_t s = (cudaStream_t)stream;
  A3D_REQUIRE(geom && label >= 0 && label < kRing, A3D_ERR_ARGUMENT, "flood_test: bad label");
  Geom g = to_geom(geom);
  Workspace ws(workspace, workspace_bytes);
  FloodWs w;
  carve_flood(w, ws, g);
  A3D_REQUIRE(workspace && ws.ok(), A3D_ERR_WORKSPACE, "flood_test: workspace too small");
  if (n == 0) return A3D_OK;
  const int64_t nwords = (int64_t)g.nx * g.ny * g.nw;
  A3D_PDL(test_bits_kernel, dim3((unsigned)ceil_div(n, 256)), dim3(256), 0, s, g, w.lab + (int64_t)label * nwords, ijk,
          n, out);
  return A3D_OK;
}

// ---- dam neighbourhood signs for caller-given lists -------------------------
// Volumes of the flood workspace reused: lab[kDam], lab[kWater], lab[kDry]
// hold the three lists' voxels inside the volume, lab[kExtTide] the dam grown
// by k_ring 3x3x3 dilations (clamped to the volume, which the caller clamps
// to the grid), lab[kRing] and ring2 are the dilation's ping-pong buffers.
extern "C" int a3d_ring_signs(const int64_t* dam_ijk, int64_t n_dam, const int64_t* water_ijk, int64_t n_water,
                              const int64_t* dry_ijk, int64_t n_dry, const a3d_flood_geom* geom, void* workspace,
                              size_t workspace_bytes, int64_t* count_out, a3d_stream_t stream) {
  cudaStream_t s = (cudaStream_t)stream;
  A3D_REQUIRE(geom && count_out && dam_ijk && n_dam > 0, A3D_ERR_ARGUMENT, "ring_signs: null argument or no dam");
  A3D_REQUIRE(geom->k_ring >= 0, A3D_ERR_ARGUMENT, "ring_signs: k_ring must be >= 0");
  A3D_REQUIRE((n_water == 0 || water_ijk) && (n_dry == 0 || dry_ijk), A3D_ERR_ARGUMENT, "ring_signs: null list");
  Geom g = to_geom(geom);
  A3D_REQUIRE(g.nx > 0 && g.ny > 0 && g.nz > 0, A3D_ERR_ARGUMENT, "ring_signs: empty volume");
  A3D_REQUIRE((int64_t)g.nx * g.ny * g.nw < (1ll << 32), A3D_ERR_ARGUMENT, "ring_signs: volume above 2^32 words");
  Workspace ws(workspace, workspace_bytes);
  FloodWs w;
  carve_flood(w, ws, g);
  A3D_REQUIRE(workspace && ws.ok(), A3D_ERR_WORKSPACE, "ring_signs: workspace too small");
  const int64_t nwords = (int64_t)g.nx * g.ny * g.nw;
  A3D_CUDA_TRY(cudaMemsetAsync(w.lab, 0, (size_t)kLabels * nwords * 4, s));
  A3D_CUDA_TRY(cudaMemsetAsync(w.misc, 0, 32 * sizeof(uint32_t), s));
  uint32_t* v_dam = w.lab + (int64_t)kDam * nwords;
  A3D_PDL(set_bits_kernel, dim3((unsigned)ceil_div(n_dam, 256)), dim3(256), 0, s, dam_ijk, n_dam, g, v_dam);
  if (n_water > 0) {
    A3D_PDL(set_bits_kernel, dim3((unsigned)ceil_div(n_water, 256)), dim3(256), 0, s, water_ijk, n_water, g,
            w.lab + (int64_t)kWater * nwords);
  }
  if (n_dry > 0) {
    A3D_PDL(set_bits_kernel, dim3((unsigned)ceil_div(n_dry, 256)), dim3(256), 0, s, dry_ijk, n_dry, g,
            w.lab + (int64_t)kDry * nwords);
  }
  const unsigned gw = (unsigned)ceil_div(nwords, 256);
  uint32_t* ring_out = w.lab + (int64_t)kExtTide * nwords;
  const uint32_t* src = v_dam;
  uint32_t* bufs[2] = {w.lab + (int64_t)kRing * nwords, w.ring2};
  for (int k = 0; k < geom->k_ring; ++k) {
    uint32_t* dst = (k == geom->k_ring - 1) ? ring_out : bufs[k & 1];
    A3D_PDL(box_dilate_kernel, dim3(gw), dim3(256), 0, s, g, src, dst, nwords);
    src = dst;
  }
  if (geom->k_ring == 0)
    A3D_CUDA_TRY(cudaMemcpyAsync(ring_out, v_dam, nwords * 4, cudaMemcpyDeviceToDevice, s));
  const int64_t ntiles = tiles_of(g);
  unsigned long long* tot = reinterpret_cast<unsigned long long*>(w.misc + 8);
  A3D_PDL(tile_counts_kernel, dim3((unsigned)ntiles), dim3(kTileThreads), 0, s, w.lab, nwords, ntiles, w.tcnt, tot);
  unsigned long long h = 0;
  A3D_CUDA_TRY(cudaMemcpyAsync(&h, tot + kExtTide, sizeof(h), cudaMemcpyDeviceToHost, s));
  A3D_CUDA_TRY(cudaStreamSynchronize(s));
  *count_out = (int64_t)h;
  return A3D_OK;
}

extern "C" int a3d_ring_signs_emit(const a3d_flood_geom* geom, void* workspace, size_t workspace_bytes,
                                   int32_t* out_ijk, int8_t* out_signs, int64_t count, a3d_stream_t stream) {
  cudaStream_t s = (cudaStream_t)stream;
  A3D_REQUIRE(geom, A3D_ERR_ARGUMENT, "ring_signs_emit: null geometry");
  if (count == 0) return A3D_OK;
  A3D_REQUIRE(out_ijk && out_signs, A3D_ERR_ARGUMENT, "ring_signs_emit: null output");
  A3D_TRY(a3d_flood_extract(geom, workspace, workspace_bytes, kExtTide, out_ijk, count, stream));
  Geom g = to_geom(geom);
  Workspace ws(workspace, workspace_bytes);
  FloodWs w;
  carve_flood(w, ws, g);
  const int64_t nwords = (int64_t)g.nx * g.ny * g.nw;
  A3D_PDL(ring_sign_kernel, dim3((unsigned)ceil_div(count, 256)), dim3(256), 0, s, g, w.lab + (int64_t)kDam * nwords,
          w.lab + (int64_t)kWater * nwords, w.lab + (int64_t)kDry * nwords, out_ijk, count, out_signs);
  return A3D_OK;
}
