// Surface dual graph of the flood-fill cells, and the dam "wet" masks.
//
// Replaces construct_surface_dual_graph and get_dam_wet_faces / _edges /
// _corners (atom3d/apps/sparse_flood_fill.py:169-291).  The reference builds
// the graph with torch.unique(dim=0) over the 8 corners of every cell (a
// lexicographic row sort) and torch.searchsorted on linear keys.  Here both
// sets live in bit volumes over the cells' bounding box (32 z-voxels per
// word, rows (x, y) in raster order, as in flood.cu):
//   * cells: one bit per active cell; the union of the input lists is a
//     plain OR, so duplicates vanish with no sort;
//   * vertices: the cell volume dilated by +1 along x, y and z (a cell marks
//     its 8 corners) -- one extra layer on the + sides holds the top corners;
//   * word-order extraction is the lexicographic (x, y, z) order of
//     torch.unique(dim=0), and the index of a cell or vertex in its unique
//     list is its rank: an exclusive scan of per-word popcounts plus the
//     popcount of the word's lower bits.
// cube_idx of a cell needs 4 rank lookups (the z+1 corner of a row is the
// next vertex of that row); adj_idx reproduces the reference's lookup of the
// linear key (x*R + y)*R + z exactly, including its wrap-around at the y and
// z faces of the grid (key of (x, y, R) == key of (x, y+1, 0)).
//
// The wet masks test 6 / 12 / 8 groups of neighbours of each dam cell
// against the collision set: one 27-bit neighbourhood mask per dam cell from
// a bit volume over the collision set's bounding box, then a constant mask
// per face, edge and corner (tables of atom3d/constants.py:50-110).

#include <climits>
#include <cstdint>

#include "a3d_common.cuh"
#include "atom3d_b200.h"
#include "primitives.cuh"

namespace a3d {
namespace {

struct VGeom {
  int nx, ny, nz, nw;  // volume size in voxels, words per row
  int lx, ly, lz;      // grid coordinates of the volume's voxel (0, 0, 0)
};

__device__ __forceinline__ int64_t vidx(const VGeom& g, int x, int y, int w) {
  return ((int64_t)x * g.ny + y) * g.nw + w;
}

__device__ __forceinline__ bool vbit(const VGeom& g, const uint32_t* __restrict__ v, int x, int y, int z) {
  if (x < 0 || y < 0 || z < 0 || x >= g.nx || y >= g.ny || z >= g.nz) return false;
  return (__ldg(v + vidx(g, x, y, z >> 5)) >> (z & 31)) & 1u;
}

// index of set voxel (x, y, z) in word order
__device__ __forceinline__ int64_t vrank(const VGeom& g, const uint32_t* __restrict__ v,
                                         const int64_t* __restrict__ offs, int x, int y, int z) {
  const int64_t w = vidx(g, x, y, z >> 5);
  return __ldg(offs + w) + __popc(__ldg(v + w) & ((1u << (z & 31)) - 1u));
}

__global__ void bbox32_kernel(const int32_t* __restrict__ ijk, int64_t n, int* __restrict__ bb) {
  pdl_wait();
  int lo[3] = {INT_MAX, INT_MAX, INT_MAX}, hi[3] = {INT_MIN, INT_MIN, INT_MIN};
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const int v = ijk[3 * i + a];
      lo[a] = min(lo[a], v);
      hi[a] = max(hi[a], v);
    }
  }
#pragma unroll
  for (int a = 0; a < 3; ++a) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      lo[a] = min(lo[a], __shfl_xor_sync(0xffffffffu, lo[a], o));
      hi[a] = max(hi[a], __shfl_xor_sync(0xffffffffu, hi[a], o));
    }
  }
  // one atomic per block and bound: warps meet in shared memory first
  __shared__ int s_b[6][32];
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
      lo[a] = lane < nwarps ? s_b[a][lane] : INT_MAX;
      hi[a] = lane < nwarps ? s_b[3 + a][lane] : INT_MIN;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        const int l = __shfl_xor_sync(0xffffffffu, lo[a], o), h = __shfl_xor_sync(0xffffffffu, hi[a], o);
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

__global__ void set_cells_kernel(const int32_t* __restrict__ ijk, int64_t n, VGeom g, uint32_t* __restrict__ vol) {
  pdl_wait();
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int x = ijk[3 * i] - g.lx, y = ijk[3 * i + 1] - g.ly, z = ijk[3 * i + 2] - g.lz;
  if (x < 0 || y < 0 || z < 0 || x >= g.nx || y >= g.ny || z >= g.nz) return;  // host checked the bounds
  atomicOr(&vol[vidx(g, x, y, z >> 5)], 1u << (z & 31));
}

// vertex word = OR over the 4 rows (x-a, y-b) of the cell word and its
// one-bit z shift; also the per-word popcounts of both volumes
__global__ void corners_kernel(VGeom g, const uint32_t* __restrict__ cells, uint32_t* __restrict__ verts,
                               uint32_t* __restrict__ ccnt, uint32_t* __restrict__ vcnt, int64_t nwords) {
  pdl_wait();
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nwords) return;
  const int w = (int)(i % g.nw);
  const int64_t row = i / g.nw;
  const int y = (int)(row % g.ny), x = (int)(row / g.ny);
  uint32_t v = 0;
#pragma unroll
  for (int a = 0; a < 2; ++a) {
#pragma unroll
    for (int b = 0; b < 2; ++b) {
      if (x - a < 0 || y - b < 0) continue;
      const int64_t j = vidx(g, x - a, y - b, w);
      const uint32_t c = __ldg(cells + j);
      const uint32_t p = w > 0 ? __ldg(cells + j - 1) : 0u;
      v |= c | (c << 1) | (p >> 31);
    }
  }
  verts[i] = v;
  vcnt[i] = (uint32_t)__popc(v);
  ccnt[i] = (uint32_t)__popc(__ldg(cells + i));
}

// One warp per 32 consecutive words; the 32 lanes take the bits of each
// non-empty word in turn, so the set voxels are written as contiguous runs in
// word order.  Each lane reads the offset and computes the coordinates of
// its own word; the warp visits only the non-empty words.
// Cells (kVerts false): int32 grid coordinates.  Vertices: int64 grid
// coordinates and world positions origin + ijk * cell (a product, then a
// sum: the reference's two separate tensor operations, no contraction).
template <bool kVerts>
__global__ void extract_kernel(VGeom g, const uint32_t* __restrict__ v, const int64_t* __restrict__ offs,
                               int64_t nwords, int32_t* __restrict__ out_cells, int64_t* __restrict__ out_verts,
                               float* __restrict__ out_world, float3 origin, float3 cell) {
  pdl_wait();
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const int64_t w0 = (((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 32;
  if (w0 >= nwords) return;
  const int64_t i = w0 + lane;
  const uint32_t mine = i < nwords ? v[i] : 0u;
  unsigned nz = __ballot_sync(FULL, mine != 0u);
  if (!nz) return;
  const int64_t my_off = mine ? offs[i] : 0;
  const int64_t row = i / g.nw;
  const int my_z = (int)(i - row * g.nw) * 32 + g.lz;
  const int my_y = (int)(row % g.ny) + g.ly, my_x = (int)(row / g.ny) + g.lx;
  const unsigned lt = (1u << lane) - 1u;
  while (nz) {
    const int j = __ffs(nz) - 1;
    nz &= nz - 1u;
    const uint32_t m = __shfl_sync(FULL, mine, j);
    const int64_t o = __shfl_sync(FULL, my_off, j);
    const int gx = __shfl_sync(FULL, my_x, j), gy = __shfl_sync(FULL, my_y, j);
    const int gz = __shfl_sync(FULL, my_z, j) + lane;
    if (!((m >> lane) & 1u)) continue;
    const int64_t r = o + __popc(m & lt);
    if (kVerts) {
      out_verts[3 * r] = gx;
      out_verts[3 * r + 1] = gy;
      out_verts[3 * r + 2] = gz;
      out_world[3 * r] = __fadd_rn(origin.x, __fmul_rn((float)gx, cell.x));
      out_world[3 * r + 1] = __fadd_rn(origin.y, __fmul_rn((float)gy, cell.y));
      out_world[3 * r + 2] = __fadd_rn(origin.z, __fmul_rn((float)gz, cell.z));
    } else {
      out_cells[3 * r] = gx;
      out_cells[3 * r + 1] = gy;
      out_cells[3 * r + 2] = gz;
    }
  }
}

// the reference's neighbour lookup: key = (x*R + y)*R + z of the offset
// coordinates, found when some active cell has that key
__device__ __forceinline__ int64_t adj_lookup(const VGeom& g, const uint32_t* __restrict__ cells,
                                              const int64_t* __restrict__ coffs, int64_t R, int64_t gx, int64_t gy,
                                              int64_t gz) {
  if (gx < 0 || gx >= R || gy < 0 || gy >= R || gz < 0 || gz >= R) {
    const int64_t key = (gx * R + gy) * R + gz;
    if (key < 0 || key >= R * R * R) return -1;
    gz = key % R;
    gy = (key / R) % R;
    gx = key / (R * R);
  }
  const int x = (int)(gx - g.lx), y = (int)(gy - g.ly), z = (int)(gz - g.lz);
  if (!vbit(g, cells, x, y, z)) return -1;
  return vrank(g, cells, coffs, x, y, z);
}

// one thread per active cell: cube_idx (CUBE_CORNERS order, corner c at
// (c&1, (c>>1)&1, (c>>2)&1)) and adj_idx (+x, -x, +y, -y, +z, -z)
__global__ void links_kernel(VGeom g, int64_t R, const int32_t* __restrict__ cells_ijk, int64_t ncells,
                             const uint32_t* __restrict__ cells, const int64_t* __restrict__ coffs,
                             const uint32_t* __restrict__ verts, const int64_t* __restrict__ voffs,
                             int64_t* __restrict__ cube_idx, int64_t* __restrict__ adj_idx) {
  pdl_wait();
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ncells) return;
  const int gx = cells_ijk[3 * i], gy = cells_ijk[3 * i + 1], gz = cells_ijk[3 * i + 2];
  const int x = gx - g.lx, y = gy - g.ly, z = gz - g.lz;
  int64_t c[8];
#pragma unroll
  for (int b = 0; b < 2; ++b) {
#pragma unroll
    for (int a = 0; a < 2; ++a) {
      // vertex (x+a, y+b, z) and its successor (x+a, y+b, z+1) in the row
      const int64_t r = vrank(g, verts, voffs, x + a, y + b, z);
      c[a + 2 * b] = r;
      c[a + 2 * b + 4] = r + 1;
    }
  }
  longlong2* cp = reinterpret_cast<longlong2*>(cube_idx + 8 * i);
#pragma unroll
  for (int k = 0; k < 4; ++k) cp[k] = make_longlong2(c[2 * k], c[2 * k + 1]);
  int64_t n[6];
  n[0] = adj_lookup(g, cells, coffs, R, (int64_t)gx + 1, gy, gz);
  n[1] = adj_lookup(g, cells, coffs, R, (int64_t)gx - 1, gy, gz);
  n[2] = adj_lookup(g, cells, coffs, R, gx, (int64_t)gy + 1, gz);
  n[3] = adj_lookup(g, cells, coffs, R, gx, (int64_t)gy - 1, gz);
  // +-z inside the grid: the row neighbours of cell i in word order
  n[4] = gz + 1 < R ? (vbit(g, cells, x, y, z + 1) ? i + 1 : -1)
                    : adj_lookup(g, cells, coffs, R, gx, gy, (int64_t)gz + 1);
  n[5] = gz > 0 ? (vbit(g, cells, x, y, z - 1) ? i - 1 : -1) : adj_lookup(g, cells, coffs, R, gx, gy, -1);
  longlong2* ap = reinterpret_cast<longlong2*>(adj_idx + 6 * i);
#pragma unroll
  for (int k = 0; k < 3; ++k) ap[k] = make_longlong2(n[2 * k], n[2 * k + 1]);
}

// ---- wet masks ------------------------------------------------------------
// neighbourhood bit of offset (dx, dy, dz) in {-1, 0, 1}^3
__host__ __device__ constexpr int nb_bit(int dx, int dy, int dz) { return (dx + 1) + 3 * (dy + 1) + 9 * (dz + 1); }

struct WetMasks {
  uint32_t face[6], edge[12], corner[8];
};

// Tables of atom3d/constants.py:50-110, as 27-bit neighbourhood masks.
// Faces: +x, -x, +y, -y, +z, -z.  Edge e (4 per axis, x-, y-, then
// z-aligned): its two perpendicular axes p < q get signs + or - by bit 0 and
// bit 1 of e % 4, and the neighbours are p, q and p+q.  Corner c with signs
// s = 2 * (c&1, (c>>1)&1, (c>>2)&1) - 1: the 7 nonzero sub-offsets of s.
WetMasks make_wet_masks() {
  WetMasks m{};
  const int f6[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
  for (int k = 0; k < 6; ++k) m.face[k] = 1u << nb_bit(f6[k][0], f6[k][1], f6[k][2]);
  for (int e = 0; e < 12; ++e) {
    const int axis = e / 4, k = e % 4;
    const int p = axis == 0 ? 1 : 0, q = axis == 2 ? 1 : 2;
    int op[3] = {0, 0, 0}, oq[3] = {0, 0, 0};
    op[p] = (k & 1) ? -1 : 1;
    oq[q] = (k & 2) ? -1 : 1;
    m.edge[e] = (1u << nb_bit(op[0], op[1], op[2])) | (1u << nb_bit(oq[0], oq[1], oq[2])) |
                (1u << nb_bit(op[0] + oq[0], op[1] + oq[1], op[2] + oq[2]));
  }
  for (int c = 0; c < 8; ++c) {
    const int s[3] = {(c & 1) ? 1 : -1, (c & 2) ? 1 : -1, (c & 4) ? 1 : -1};
    uint32_t bits = 0;
    for (int sub = 1; sub < 8; ++sub)
      bits |= 1u << nb_bit((sub & 1) ? s[0] : 0, (sub & 2) ? s[1] : 0, (sub & 4) ? s[2] : 0);
    m.corner[c] = bits;
  }
  return m;
}

__global__ void dam_wet_kernel(VGeom g, const uint32_t* __restrict__ coll, const int32_t* __restrict__ dam, int64_t n,
                               WetMasks wm, uint8_t* __restrict__ faces, uint8_t* __restrict__ edges,
                               uint8_t* __restrict__ corners) {
  pdl_wait();
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  // grid coordinates outside [0, R) are never in the collision volume, so
  // the reference's in-bounds test is implied by the volume test
  const int x = dam[3 * i] - g.lx, y = dam[3 * i + 1] - g.ly, z = dam[3 * i + 2] - g.lz;
  uint32_t nb = 0;
#pragma unroll
  for (int dy = -1; dy <= 1; ++dy) {
#pragma unroll
    for (int dx = -1; dx <= 1; ++dx) {
      const int xx = x + dx, yy = y + dy;
      if (xx < 0 || yy < 0 || xx >= g.nx || yy >= g.ny) continue;
#pragma unroll
      for (int dz = -1; dz <= 1; ++dz) {
        const int zz = z + dz;
        if (zz < 0 || zz >= g.nz) continue;
        if ((__ldg(coll + vidx(g, xx, yy, zz >> 5)) >> (zz & 31)) & 1u) nb |= 1u << nb_bit(dx, dy, dz);
      }
    }
  }
  if (faces)
    for (int k = 0; k < 6; ++k) faces[6 * i + k] = (nb & wm.face[k]) != 0u;
  if (edges)
    for (int k = 0; k < 12; ++k) edges[12 * i + k] = (nb & wm.edge[k]) != 0u;
  if (corners)
    for (int k = 0; k < 8; ++k) corners[8 * i + k] = (nb & wm.corner[k]) != 0u;
}

}  // namespace
}  // namespace a3d

using namespace a3d;

namespace {
constexpr int kMaxLists = 8;
constexpr int64_t kMaxVolumeWords = (int64_t)1 << 33;  // 32 GiB per bit volume

// volume over [lo, hi + extra] per axis
bool make_vgeom(const int64_t* lo, const int64_t* hi, int extra, VGeom* g) {
  int64_t d[3];
  for (int a = 0; a < 3; ++a) {
    d[a] = hi[a] - lo[a] + 1 + extra;
    if (hi[a] < lo[a] || d[a] > INT_MAX - 64) return false;
  }
  g->nx = (int)d[0]; g->ny = (int)d[1]; g->nz = (int)d[2];
  g->nw = (int)ceil_div(d[2], 32);
  g->lx = (int)lo[0]; g->ly = (int)lo[1]; g->lz = (int)lo[2];
  return (int64_t)g->nx * g->ny * g->nw <= kMaxVolumeWords;
}

struct DualWs {
  uint32_t* cells;
  uint32_t* verts;
  uint32_t* ccnt;
  uint32_t* vcnt;
  int64_t* coffs;
  int64_t* voffs;
  int64_t* scan_tmp;
};

size_t carve_dual(DualWs& w, Workspace& ws, const VGeom& g) {
  const int64_t nwords = (int64_t)g.nx * g.ny * g.nw;
  w.cells = ws.take<uint32_t>(nwords);
  w.verts = ws.take<uint32_t>(nwords);
  w.ccnt = ws.take<uint32_t>(nwords);
  w.vcnt = ws.take<uint32_t>(nwords);
  w.coffs = ws.take<int64_t>(nwords + 1);
  w.voffs = ws.take<int64_t>(nwords + 1);
  w.scan_tmp = ws.take<int64_t>((int64_t)scan_workspace_elems(nwords));
  return ws.used;
}

int dual_geom(const a3d_dual_geom* p, VGeom* g) {
  A3D_REQUIRE(p && p->resolution > 0 && p->resolution <= ((int64_t)1 << 21), A3D_ERR_ARGUMENT,
              "dual graph: resolution must be in [1, 2^21]");
  for (int a = 0; a < 3; ++a)
    A3D_REQUIRE(p->lo[a] >= 0 && p->lo[a] <= p->hi[a] && p->hi[a] < p->resolution, A3D_ERR_ARGUMENT,
                "dual graph: cells must lie in [0, resolution)");
  A3D_REQUIRE(make_vgeom(p->lo, p->hi, 1, g), A3D_ERR_ARGUMENT, "dual graph: bounding box too large");
  return A3D_OK;
}
}  // namespace

extern "C" int a3d_cells_bbox(const int32_t* const* lists, const int64_t* counts, int num_lists, int64_t* bbox_out,
                              void* workspace, size_t workspace_bytes, a3d_stream_t stream) {
  cudaStream_t s = (cudaStream_t)stream;
  A3D_REQUIRE(bbox_out && num_lists >= 0 && num_lists <= kMaxLists && (num_lists == 0 || (lists && counts)),
              A3D_ERR_ARGUMENT, "cells_bbox: bad argument");
  A3D_REQUIRE(workspace && workspace_bytes >= 6 * sizeof(int), A3D_ERR_WORKSPACE, "cells_bbox: workspace");
  int init[6] = {INT_MAX, INT_MAX, INT_MAX, INT_MIN, INT_MIN, INT_MIN};
  int* bb = (int*)workspace;
  A3D_CUDA_TRY(cudaMemcpyAsync(bb, init, sizeof(init), cudaMemcpyHostToDevice, s));
  for (int l = 0; l < num_lists; ++l) {
    A3D_REQUIRE(counts[l] >= 0 && (counts[l] == 0 || lists[l]), A3D_ERR_ARGUMENT, "cells_bbox: bad list");
    if (counts[l] == 0) continue;
    const int64_t blocks = ceil_div(counts[l], 256) < 4096 ? ceil_div(counts[l], 256) : 4096;
    A3D_PDL(bbox32_kernel, dim3((unsigned)blocks), dim3(256), 0, s, lists[l], counts[l], bb);
  }
  int h[6];
  A3D_CUDA_TRY(cudaMemcpyAsync(h, bb, sizeof(h), cudaMemcpyDeviceToHost, s));
  A3D_CUDA_TRY(cudaStreamSynchronize(s));
  for (int a = 0; a < 6; ++a) bbox_out[a] = h[a];
  return A3D_OK;
}

extern "C" size_t a3d_dual_workspace_bytes(const a3d_dual_geom* geom) {
  VGeom g;
  if (dual_geom(geom, &g) != A3D_OK) return 0;
  Workspace ws(nullptr, 0);
  DualWs w;
  return carve_dual(w, ws, g) + 256;
}

extern "C" int a3d_dual_graph_count(const int32_t* const* lists, const int64_t* counts, int num_lists,
                                    const a3d_dual_geom* geom, void* workspace, size_t workspace_bytes,
                                    int64_t* counts_out, a3d_stream_t stream) {
  cudaStream_t s = (cudaStream_t)stream;
  A3D_REQUIRE(counts_out && num_lists >= 0 && num_lists <= kMaxLists && (num_lists == 0 || (lists && counts)),
              A3D_ERR_ARGUMENT, "dual_graph_count: bad argument");
  VGeom g;
  A3D_TRY(dual_geom(geom, &g));
  Workspace ws(workspace, workspace_bytes);
  DualWs w;
  carve_dual(w, ws, g);
  A3D_REQUIRE(workspace && ws.ok(), A3D_ERR_WORKSPACE, "dual_graph_count: workspace too small");
  const int64_t nwords = (int64_t)g.nx * g.ny * g.nw;
  A3D_CUDA_TRY(cudaMemsetAsync(w.cells, 0, nwords * 4, s));
  for (int l = 0; l < num_lists; ++l) {
    A3D_REQUIRE(counts[l] >= 0 && (counts[l] == 0 || lists[l]), A3D_ERR_ARGUMENT, "dual_graph_count: bad list");
    if (counts[l] == 0) continue;
    A3D_PDL(set_cells_kernel, dim3((unsigned)ceil_div(counts[l], 256)), dim3(256), 0, s, lists[l], counts[l], g,
            w.cells);
  }
  A3D_PDL(corners_kernel, dim3((unsigned)ceil_div(nwords, 256)), dim3(256), 0, s, g, w.cells, w.verts, w.ccnt, w.vcnt,
          nwords);
  A3D_TRY((device_exclusive_scan<uint32_t, int64_t>(w.ccnt, w.coffs, nwords, w.scan_tmp, w.coffs + nwords, s)));
  A3D_TRY((device_exclusive_scan<uint32_t, int64_t>(w.vcnt, w.voffs, nwords, w.scan_tmp, w.voffs + nwords, s)));
  A3D_CUDA_TRY(cudaMemcpyAsync(counts_out, w.coffs + nwords, 8, cudaMemcpyDeviceToHost, s));
  A3D_CUDA_TRY(cudaMemcpyAsync(counts_out + 1, w.voffs + nwords, 8, cudaMemcpyDeviceToHost, s));
  A3D_CUDA_TRY(cudaStreamSynchronize(s));
  return A3D_OK;
}

extern "C" int a3d_dual_graph_emit(const a3d_dual_geom* geom, void* workspace, size_t workspace_bytes,
                                   int64_t num_cells, int64_t num_vertices, const float* origin, const float* cell,
                                   int32_t* cells_ijk, int64_t* vertices_ijk, float* vertices_world,
                                   int64_t* cube_idx, int64_t* adj_idx, a3d_stream_t stream) {
  cudaStream_t s = (cudaStream_t)stream;
  VGeom g;
  A3D_TRY(dual_geom(geom, &g));
  A3D_REQUIRE(origin && cell && num_cells >= 0 && num_vertices >= 0, A3D_ERR_ARGUMENT, "dual_graph_emit: bad argument");
  Workspace ws(workspace, workspace_bytes);
  DualWs w;
  carve_dual(w, ws, g);
  A3D_REQUIRE(workspace && ws.ok(), A3D_ERR_WORKSPACE, "dual_graph_emit: workspace too small");
  if (num_cells == 0) return A3D_OK;
  A3D_REQUIRE(cells_ijk && vertices_ijk && vertices_world && cube_idx && adj_idx, A3D_ERR_ARGUMENT,
              "dual_graph_emit: null output");
  A3D_REQUIRE(((uintptr_t)cube_idx & 15) == 0 && ((uintptr_t)adj_idx & 15) == 0, A3D_ERR_ARGUMENT,
              "dual_graph_emit: cube_idx / adj_idx must be 16-byte aligned");
  const int64_t nwords = (int64_t)g.nx * g.ny * g.nw;
  const unsigned gw = (unsigned)ceil_div(nwords, 256);
  const float3 o = make_float3(origin[0], origin[1], origin[2]), c = make_float3(cell[0], cell[1], cell[2]);
  A3D_PDL(extract_kernel<false>, dim3(gw), dim3(256), 0, s, g, w.cells, w.coffs, nwords, cells_ijk, nullptr, nullptr, o,
          c);
  A3D_PDL(extract_kernel<true>, dim3(gw), dim3(256), 0, s, g, w.verts, w.voffs, nwords, nullptr, vertices_ijk,
          vertices_world, o, c);
  A3D_PDL(links_kernel, dim3((unsigned)ceil_div(num_cells, 256)), dim3(256), 0, s, g, geom->resolution, cells_ijk,
          num_cells, w.cells, w.coffs, w.verts, w.voffs, cube_idx, adj_idx);
  return A3D_OK;
}

extern "C" size_t a3d_dam_wet_workspace_bytes(const int64_t* collision_bbox) {
  if (!collision_bbox) return 0;
  VGeom g;
  if (!make_vgeom(collision_bbox, collision_bbox + 3, 0, &g)) return 256;  // empty collision set
  return (((size_t)g.nx * g.ny * g.nw * 4 + 255) & ~(size_t)255) + 256;
}

extern "C" int a3d_dam_wet(const int32_t* dam_ijk, int64_t n, const int32_t* collision_ijk, int64_t m,
                           const int64_t* collision_bbox, int64_t resolution, void* workspace, size_t workspace_bytes,
                           uint8_t* wet_faces, uint8_t* wet_edges, uint8_t* wet_corners, a3d_stream_t stream) {
  cudaStream_t s = (cudaStream_t)stream;
  A3D_REQUIRE(n >= 0 && m >= 0 && resolution > 0 && (n == 0 || dam_ijk) && (m == 0 || (collision_ijk && collision_bbox)),
              A3D_ERR_ARGUMENT, "dam_wet: bad argument");
  if (n == 0) return A3D_OK;
  const size_t per = 6 * (wet_faces != nullptr) + 12 * (wet_edges != nullptr) + 8 * (wet_corners != nullptr);
  if (per == 0) return A3D_OK;
  if (m == 0) {  // nothing is wet
    if (wet_faces) A3D_CUDA_TRY(cudaMemsetAsync(wet_faces, 0, 6 * n, s));
    if (wet_edges) A3D_CUDA_TRY(cudaMemsetAsync(wet_edges, 0, 12 * n, s));
    if (wet_corners) A3D_CUDA_TRY(cudaMemsetAsync(wet_corners, 0, 8 * n, s));
    return A3D_OK;
  }
  for (int a = 0; a < 3; ++a)
    A3D_REQUIRE(collision_bbox[a] >= 0 && collision_bbox[a] <= collision_bbox[3 + a] &&
                    collision_bbox[3 + a] < resolution,
                A3D_ERR_ARGUMENT, "dam_wet: collision cells must lie in [0, resolution)");
  VGeom g;
  A3D_REQUIRE(make_vgeom(collision_bbox, collision_bbox + 3, 0, &g), A3D_ERR_ARGUMENT, "dam_wet: bounding box too large");
  const int64_t nwords = (int64_t)g.nx * g.ny * g.nw;
  A3D_REQUIRE(workspace && workspace_bytes >= (size_t)nwords * 4, A3D_ERR_WORKSPACE, "dam_wet: workspace too small");
  uint32_t* vol = (uint32_t*)workspace;
  A3D_CUDA_TRY(cudaMemsetAsync(vol, 0, nwords * 4, s));
  A3D_PDL(set_cells_kernel, dim3((unsigned)ceil_div(m, 256)), dim3(256), 0, s, collision_ijk, m, g, vol);
  static const WetMasks wm = make_wet_masks();
  A3D_PDL(dam_wet_kernel, dim3((unsigned)ceil_div(n, 256)), dim3(256), 0, s, g, vol, dam_ijk, n, wm, wet_faces,
          wet_edges, wet_corners);
  return A3D_OK;
}
