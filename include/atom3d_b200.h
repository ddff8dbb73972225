/*
 * atom3d_b200 — C ABI of the B200 geometry hot path.
 *
 * Every function takes raw device pointers, element counts and a CUDA
 * stream, allocates nothing itself (scratch comes from a caller-provided
 * workspace whose size is queried first), and returns an int status
 * (A3D_OK == 0).  No C++ exception or torch type crosses this boundary.
 * The host-side Python package (atom3d_b200) binds these with ctypes and
 * keeps the reference's Python signatures on top of them.
 *
 * Each entry point names the reference interface it replaces (file:line
 * inside the Luo-Yihao/Atom3d project).
 */
#ifndef ATOM3D_B200_H_
#define ATOM3D_B200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st* a3d_stream_t; /* == cudaStream_t */

/* ---- status codes ------------------------------------------------------ */
#define A3D_OK 0
#define A3D_ERR_ARGUMENT 1      /* bad size / null pointer / unsupported option */
#define A3D_ERR_WORKSPACE 2     /* workspace or output capacity too small       */
#define A3D_ERR_CUDA 3          /* a CUDA runtime call or launch failed         */
#define A3D_ERR_OVERFLOW 4      /* a device-side queue or stack overflowed      */
#define A3D_ERR_TIMEOUT 5       /* a bounded device-side wait gave up           */

/* Last error message of the calling host thread ("" when none). */
const char* a3d_last_error(void);
/* Library version string. */
const char* a3d_version(void);

/* ---- BVH ---------------------------------------------------------------- */
/* Device-resident wide BVH: 64-byte 4-wide quantised nodes (node 0 = root)
 * and 64-byte triangle records stored in leaf order.  The memory is owned by
 * the caller; a3d_bvh_build fills it. */
typedef struct a3d_bvh_view {
  const void* nodes;   /* num_nodes x 64 B, 64-B aligned                     */
  const void* tris;    /* num_tris  x 64 B, 16-B aligned                     */
  int64_t num_nodes;
  int64_t num_tris;
  float lo[3];         /* scene bounds (triangle AABB union)                 */
  float hi[3];
} a3d_bvh_view;

#define A3D_BVH_NODE_BYTES 64
#define A3D_BVH_TRI_BYTES 64

/* Replaces build_bvh_cuda / build_bvh_recursive
 * (atom3d/kernels/bvh_kernels.cu:860-925, :667-854) behind
 * BVHAccelerator.__init__ (atom3d/kernels/bvh.py:66-93).
 * GPU build: Morton codes -> in-house radix sort -> binary radix tree ->
 * bottom-up refit -> SAH-guided collapse into 4-wide quantised nodes.
 * node_capacity >= max(num_faces, 1) always suffices.  leaf_max (1..8, 0 =
 * default 8): subtrees with at most this many triangles become leaves. */
size_t a3d_bvh_build_workspace_bytes(int64_t num_faces);
int a3d_bvh_build(const float* vertices, int64_t num_vertices,
                  const int32_t* faces, int64_t num_faces, int leaf_max,
                  void* nodes_out, int64_t node_capacity, void* tris_out,
                  void* workspace, size_t workspace_bytes,
                  int64_t* num_nodes_out /* host */,
                  float* bounds_out /* host, 6 floats: lo xyz, hi xyz */,
                  a3d_stream_t stream);

/* ---- pseudo-normal precompute for the SDF sign -------------------------- */
/* Replaces MeshBVH._precompute_face_normals and
 * MeshBVH._precompute_pseudo_normal_data (atom3d/core/mesh_bvh.py:129-232).
 * Outputs: face_normals_sign [F,3] (n/(|n|+1e-8), used by the sign test),
 * face_angles [F,3], vertex_pn [V,3], edge_pn [edge_capacity,3],
 * he_edge_idx [3F] int64 (half-edge -> edge id, edges numbered in ascending
 * key lo*V+hi order like torch.unique). *num_edges_out receives E.
 * A face index outside [0, num_vertices) returns A3D_ERR_ARGUMENT (no kernel
 * reads or writes through it). */
size_t a3d_mesh_normals_workspace_bytes(int64_t num_vertices, int64_t num_faces);
int a3d_mesh_normals(const float* vertices, int64_t num_vertices,
                     const int32_t* faces, int64_t num_faces,
                     float* face_normals_sign, float* face_angles,
                     float* vertex_pn, float* edge_pn, int64_t edge_capacity,
                     int64_t* he_edge_idx, int64_t* num_edges_out /* host */,
                     void* workspace, size_t workspace_bytes, a3d_stream_t stream);

/* Sign inputs for a3d_udf (all device pointers). */
typedef struct a3d_sign_data {
  const float* face_normals;   /* [F,3]  */
  const float* vertex_pn;      /* [V,3]  */
  const float* edge_pn;        /* [E,3]  */
  const int64_t* he_edge_idx;  /* [3F]   */
  const int32_t* faces;        /* [F,3]  */
} a3d_sign_data;

/* ---- closest-point queries --------------------------------------------- */
/* Replaces bvh_udf_cuda + bvh_udf_kernel (atom3d/kernels/bvh_kernels.cu:
 * 1028-1066, :363-463) and, when sign != NULL, the pseudo-normal sign of
 * MeshBVH._compute_sign (atom3d/core/mesh_bvh.py:759-827) fused into the
 * same launch: distances then hold signed distances.
 * uvw may be NULL.  bound (nullable) is a per-query upper bound on the
 * unsigned distance that seeds the pruning radius; queries whose bound proves
 * too small are re-run unbounded, so results never depend on it.
 * flags: A3D_UDF_SORT_QUERIES (Morton-sort queries for warp coherence),
 * A3D_UDF_ASSUME_SORTED (caller's order is already coherent).
 * stats (nullable, device, 4 x uint64): node visits, triangle tests,
 * bound misses, stack spills.  */
#define A3D_UDF_SORT_QUERIES 1u
#define A3D_UDF_ASSUME_SORTED 2u  /* queries already spatially coherent: skip the sort */
/* radius seeding (results never depend on it): by default a query's pruning
 * radius starts just above the distance to the closest triangle of the
 * previous query in the sorted order, or of a greedy descent, capped by
 * `bound`.  NO_REUSE drops the previous-query seed; BOUND_SEEDS lets a
 * finite `bound` alone seed the radius (no greedy descent).  A query with
 * no triangle inside a too-small bound is re-run without it. */
#define A3D_UDF_NO_REUSE 4u
#define A3D_UDF_BOUND_SEEDS 8u
size_t a3d_udf_workspace_bytes(int64_t num_points, uint32_t flags);
int a3d_udf(const a3d_bvh_view* bvh, const float* points, int64_t num_points,
            float* distances, int32_t* face_ids, float* closest_points,
            float* uvw, const a3d_sign_data* sign, const float* bound,
            unsigned long long* stats, uint32_t flags,
            void* workspace, size_t workspace_bytes, a3d_stream_t stream);

/* Allocation-free variant of a3d_udf (no counterpart in the reference).
 * For callers that may not call cudaMalloc (a host application owning all
 * device memory, or a latency-critical loop where an allocation would
 * synchronise the device): scratch lives in a 24 MiB file-scope device
 * array held by every GPU that loads the library.  At most 1,048,576
 * queries per call (larger: A3D_ERR_ARGUMENT).  The first call on a device
 * looks up the array's address; make it before any stream capture.  Calls
 * share the array: calls that overlap on the GPU race.  Queries are
 * Morton-sorted; results equal a3d_udf's. */
int a3d_udf_noalloc(const a3d_bvh_view* bvh, const float* points, int64_t num_points,
                    float* distances, int32_t* face_ids, float* closest_points,
                    float* uvw, a3d_stream_t stream);
/* Status words of the last a3d_udf_noalloc call on the current device, in
 * a3d_udf_status's layout (re-runs, deep-stack overflow, 0, guard faults),
 * read from the shared static scratch after `stream` drains; a call that
 * overlapped on the GPU with another a3d_udf_noalloc call reads a mix of
 * both.  No counterpart in the reference. */
int a3d_udf_noalloc_status(uint32_t* status_out, a3d_stream_t stream);

/* Adjoint of the unsigned distance with respect to the mesh vertices:
 * grad_vertices[V,3] += sum_q grad_dist[q] * d dist_q / d vertex.
 * With closest point c = sum_i w_i v_i (w = clamped barycentrics of the
 * closest point) the envelope theorem gives d dist / d v_i = -w_i (p-c)/|p-c|.
 * grad_points[Q,3] (nullable) receives grad_dist * (p-c)/|p-c| like
 * MeshBVH._udf_with_grad (atom3d/core/mesh_bvh.py:685-700). */
int a3d_udf_backward(const float* points, int64_t num_points,
                     const float* closest_points, const int32_t* face_ids,
                     const float* uvw, const float* grad_dist,
                     const int32_t* faces, float* grad_points,
                     float* grad_vertices, a3d_stream_t stream);

/* ---- Morton keys -------------------------------------------------------- */
/* Replaces OctreeIndexer._ijk_to_morton / _morton_to_ijk
 * (atom3d/grid/octree_indexer.py:162-185): x -> bit 3i, y -> 3i+1,
 * z -> 3i+2, 21 bits per axis. decode keeps bits of levels 0..level. */
int a3d_morton_encode(const int64_t* ijk, int64_t n, int64_t* morton, a3d_stream_t stream);
int a3d_morton_decode(const int64_t* morton, int64_t n, int level, int64_t* ijk, a3d_stream_t stream);

/* ---- triangle/box SAT --------------------------------------------------- */
/* Replaces bvh_aabb_intersect_cuda / bvh_aabb_intersect_kernel in hit-mask
 * mode (atom3d/kernels/bvh_kernels.cu:1192-1242, :555-610; triangle_aabb_sat
 * :285-353) behind MeshBVH.intersect_aabb(mode=0). hit[n] = 1 when some
 * triangle passes the SAT test with sat_eps = 1e-6. */
size_t a3d_aabb_hit_workspace_bytes(int64_t n);
int a3d_aabb_hit(const a3d_bvh_view* bvh, const float* box_min, const float* box_max,
                 int64_t n, uint8_t* hit, void* workspace, size_t workspace_bytes,
                 a3d_stream_t stream);

/* Replaces the pair outputs of MeshBVH.intersect_aabb modes 1-3
 * (atom3d/core/mesh_bvh.py:297-479): bvh_aabb_intersect_kernel's
 * (box, face) pairs (atom3d/kernels/bvh_kernels.cu:555-610) and
 * sat_clip_polygon_kernel (atom3d/kernels/cumtv_kernels.cu:209-460).
 *   mode 1: faces passing SAT;  modes 2, 3: faces passing SAT whose clip
 *   against the box (eps 1e-8) is non-empty.
 * Protocol (each call synchronises once; the workspaces carry state from
 * call to call):
 *   1. a3d_aabb_pairs_count: per-box SAT counts; *num_candidates_out = the
 *      number of SAT pairs.  Mode 1 also fills hit[n] (uint8).
 *   2. modes 2, 3 only: a clip workspace of
 *      a3d_aabb_clip_workspace_bytes(num_candidates) bytes, then
 *      a3d_aabb_pairs_clip: hit[n] and *num_pairs_out (clip survivors).
 *   3. a3d_aabb_pairs_write into outputs sized by the pair count, grouped
 *      by box (ascending), in tree order within a box:
 *        aabb_ids, face_ids  int32 [P] (mode 1) or int64 [P] (modes 2, 3)
 *        poly_counts int32 [P], centroids f32 [P,3], areas f32 [P]  (2, 3)
 *        poly_verts f32 [P,8,3], 16-byte aligned, zero padded       (3)
 *      (mode 1 ignores the clip workspace). */
size_t a3d_aabb_pairs_workspace_bytes(int64_t n);
size_t a3d_aabb_clip_workspace_bytes(int64_t num_candidates);
int a3d_aabb_pairs_count(const a3d_bvh_view* bvh, const float* box_min, const float* box_max,
                         int64_t n, int mode, uint8_t* hit, void* workspace,
                         size_t workspace_bytes, int64_t* num_candidates_out, a3d_stream_t stream);
int a3d_aabb_pairs_clip(const a3d_bvh_view* bvh, const float* box_min, const float* box_max,
                        int64_t n, void* workspace, size_t workspace_bytes, void* clip_workspace,
                        size_t clip_workspace_bytes, int64_t num_candidates, uint8_t* hit,
                        int64_t* num_pairs_out, a3d_stream_t stream);
int a3d_aabb_pairs_write(const a3d_bvh_view* bvh, const float* box_min, const float* box_max,
                         int64_t n, int mode, void* workspace, size_t workspace_bytes,
                         void* clip_workspace, size_t clip_workspace_bytes, int64_t num_candidates,
                         void* aabb_ids, void* face_ids, int32_t* poly_counts, float* centroids,
                         float* areas, float* poly_verts, a3d_stream_t stream);

/* Replaces OctreeIndexer.octree_traverse (atom3d/grid/octree_indexer.py:470-509):
 * coarse-to-fine candidate voxels at max_level in the reference's order
 * (meshgrid 'ij' at min_level, then parent-major x 8 CUBE_CORNERS children,
 * stable compaction).  grid_lo / cell sizes per level come from the caller
 * (cell_sizes[level] as float32 = (hi-lo)/2^level).  out_ijk [cap,3] int64.
 * *count_out (host) receives K; A3D_ERR_WORKSPACE when K > cap (count still
 * reported). */
size_t a3d_octree_workspace_bytes(int min_level, int max_level, int64_t cap);
int a3d_octree_traverse(const a3d_bvh_view* bvh, const float* grid_lo /* host[3] */,
                        const float* cell_sizes /* host [(max_level+1)*3] */,
                        int min_level, int max_level,
                        int64_t* out_ijk, int64_t cap, int64_t* count_out /* host */,
                        void* workspace, size_t workspace_bytes, a3d_stream_t stream);

/* ---- sparse flood fill ------------------------------------------------- */
/* Replaces flood_fill_3d_sparse / flood_fill_kernel / the host BFS loop
 * (atom3d/kernels/flood_fill.py:118-258, atom3d/kernels/flood_fill_kernels.cu:
 * 21-175) and get_dam_neighborhood_signs (atom3d/apps/sparse_flood_fill.py:
 * 34-100).  Work on a bit-packed volume: vol_lo/vol_dims (grid coordinates)
 * contains the flood domain crop_lo..crop_hi (inclusive); the k-ring needs
 * the volume to reach k voxels beyond the dam where the grid allows. */
typedef struct a3d_flood_geom {
  int64_t vol_lo[3];
  int32_t vol_dims[3];
  int64_t crop_lo[3];
  int64_t crop_hi[3];
  int64_t seed[3];        /* grid coordinates, inside the crop */
  int32_t connectivity;   /* 6, 18 or 26 */
  int32_t k_ring;         /* >= 0 */
} a3d_flood_geom;

/* label slots of a3d_flood_fill / _extract / _test */
#define A3D_FLOOD_WATER 0      /* pure water (reference mask == 2)          */
#define A3D_FLOOD_DRY 1        /* mask == -2                               */
#define A3D_FLOOD_TIDE 2       /* collision, mask == 1                     */
#define A3D_FLOOD_DAM 3        /* mask == -1 (extension included)          */
#define A3D_FLOOD_EXT_DAM 4    /* the extension alone                      */
#define A3D_FLOOD_EXT_TIDE 5   /* k-ring neighbours with sign +1           */
#define A3D_FLOOD_DRY_ADJ 6    /* k-ring neighbours with sign -1           */

/* bbox_out (host, 6): min xyz, max xyz of the n voxels (synchronises). */
int a3d_flood_bbox(const int64_t* ijk, int64_t n, int64_t* bbox_out,
                   void* workspace, size_t workspace_bytes, a3d_stream_t stream);
size_t a3d_flood_workspace_bytes(const a3d_flood_geom* geom);
/* Floods and labels; counts_out (host, 9): voxel count per label slot 0..6,
 * [7] = 0 and [8] = 1 when the seed is occupied (then nothing else is
 * computed, like the reference's empty result).  The labelled volumes and
 * their per-tile counts stay in the workspace for a3d_flood_extract /
 * a3d_flood_test.  rounds_out (nullable): relaxation rounds run; all rounds
 * run in one cooperative launch of the resident blocks, separated by grid
 * barriers and ended on the device when the next round's queue is empty (one
 * host read per call).  A3D_ERR_OVERFLOW when bricks are still queued after
 * 2^20 rounds (the water would be incomplete); A3D_ERR_TIMEOUT when a grid
 * barrier waited about a second.  The volume must hold fewer than 2^37 voxels (2^32
 * words). */
int a3d_flood_fill(const int64_t* dam_ijk, int64_t n, const a3d_flood_geom* geom,
                   void* workspace, size_t workspace_bytes, int64_t* counts_out,
                   int* rounds_out, a3d_stream_t stream);
/* Writes the voxels of one label as int32 [count,3] in lexicographic order;
 * count is the label's count from a3d_flood_fill (no position at or past
 * count is written). */
int a3d_flood_extract(const a3d_flood_geom* geom, void* workspace, size_t workspace_bytes,
                      int label, int32_t* out_ijk, int64_t count, a3d_stream_t stream);
/* out[i] = 1 when voxel ijk[i] carries the label. */
int a3d_flood_test(const a3d_flood_geom* geom, void* workspace, size_t workspace_bytes,
                   int label, const int64_t* ijk, int64_t n, uint8_t* out, a3d_stream_t stream);

/* Replaces get_dam_neighborhood_signs (atom3d/apps/sparse_flood_fill.py:
 * 34-100) for caller-given lists (sparse_flood_fill's fused pass covers its
 * own).  geom: vol_lo/vol_dims = the dam's bounding box grown by k_ring and
 * clamped to [0, resolution), crop = the volume, k_ring >= 1 (seed and
 * connectivity unused); workspace: a3d_flood_workspace_bytes(geom).
 * a3d_ring_signs marks the three lists (voxels outside the volume are
 * ignored), grows the dam by k_ring 3x3x3 dilations and returns the number
 * of ring voxels (one host read); a3d_ring_signs_emit writes them as int32
 * [count,3] in lexicographic order (torch.unique(dim=0) order) and their
 * signs: 0 dam, else +1 water, else -1 dry, else +1. */
int a3d_ring_signs(const int64_t* dam_ijk, int64_t n_dam, const int64_t* water_ijk, int64_t n_water,
                   const int64_t* dry_ijk, int64_t n_dry, const a3d_flood_geom* geom, void* workspace,
                   size_t workspace_bytes, int64_t* count_out, a3d_stream_t stream);
int a3d_ring_signs_emit(const a3d_flood_geom* geom, void* workspace, size_t workspace_bytes, int32_t* out_ijk,
                        int8_t* out_signs, int64_t count, a3d_stream_t stream);

/* ---- device-wide primitives (no reference counterpart) ------------------ */
/* The library's own exclusive scan and stable LSD radix sort, for callers
 * building their own compactions and orders.  out [n+1] int64: out[i] =
 * sum of in[0..i), out[n] = total.  The sort orders (keys, vals) in place by
 * key bits [begin_bit, end_bit), stably; n < 2^32. */
size_t a3d_exclusive_scan_workspace_bytes(int64_t n);
int a3d_exclusive_scan_u32(const uint32_t* in, int64_t n, int64_t* out, void* workspace,
                           size_t workspace_bytes, a3d_stream_t stream);
size_t a3d_sort_pairs_workspace_bytes(int64_t n);
int a3d_sort_pairs_u64(uint64_t* keys, uint32_t* vals, int64_t n, int begin_bit, int end_bit,
                       void* workspace, size_t workspace_bytes, a3d_stream_t stream);
/* Streams `bytes` (a multiple of 16) of `buf` `passes` times through L2 with
 * 16-byte loads from 4 blocks of 512 threads per SM; `sink` (device, one
 * word) keeps the loads live.  Timed with events on a buffer that fits in L2
 * it measures the L2 read bandwidth (the bench's L2 roofline denominator). */
int a3d_read_probe(const void* buf, int64_t bytes, int passes, uint32_t* sink, a3d_stream_t stream);

/* ---- surface dual graph and dam wet masks -------------------------------- */
/* Replace construct_surface_dual_graph and get_dam_wet_faces / _edges /
 * _corners (atom3d/apps/sparse_flood_fill.py:169-291).  Cells are int32
 * [n,3] grid coordinates in [0, resolution). */

/* bbox_out (host, 6): min xyz, max xyz over up to 8 cell lists (host arrays
 * of device pointers and counts); synchronises.  An all-empty union gives
 * min > max.  workspace >= 64 bytes. */
int a3d_cells_bbox(const int32_t* const* lists, const int64_t* counts, int num_lists,
                   int64_t* bbox_out, void* workspace, size_t workspace_bytes,
                   a3d_stream_t stream);

typedef struct a3d_dual_geom {
  int64_t lo[3];       /* bounding box of the active cells, inclusive */
  int64_t hi[3];
  int64_t resolution;  /* R = 2^max_level of the octree */
} a3d_dual_geom;

size_t a3d_dual_workspace_bytes(const a3d_dual_geom* geom);
/* Marks the union of the lists (the active cells) and their cube corners;
 * counts_out (host, 2): unique cells N, unique vertices V.  Synchronises.
 * The marked sets stay in the workspace for a3d_dual_graph_emit. */
int a3d_dual_graph_count(const int32_t* const* lists, const int64_t* counts, int num_lists,
                         const a3d_dual_geom* geom, void* workspace, size_t workspace_bytes,
                         int64_t* counts_out, a3d_stream_t stream);
/* Writes, in the reference's orders:
 *   cells_ijk      int32 [N,3]  active cells, lexicographic (x, y, z)
 *   vertices_ijk   int64 [V,3]  cube corners, lexicographic
 *   vertices_world f32   [V,3]  origin + ijk * cell (product, then sum)
 *   cube_idx       int64 [N,8]  corner c = (c&1, (c>>1)&1, (c>>2)&1)
 *   adj_idx        int64 [N,6]  +x,-x,+y,-y,+z,-z neighbour or -1, found by
 *                               the reference's linear key (x*R + y)*R + z
 * origin and cell are host float[3]; cube_idx and adj_idx 16-byte aligned. */
int a3d_dual_graph_emit(const a3d_dual_geom* geom, void* workspace, size_t workspace_bytes,
                        int64_t num_cells, int64_t num_vertices, const float* origin,
                        const float* cell, int32_t* cells_ijk, int64_t* vertices_ijk,
                        float* vertices_world, int64_t* cube_idx, int64_t* adj_idx,
                        a3d_stream_t stream);

/* collision_bbox: a3d_cells_bbox of the collision cells. */
size_t a3d_dam_wet_workspace_bytes(const int64_t* collision_bbox);
/* Per dam cell, whether a neighbour sharing each face [n,6] (+x,-x,+y,-y,
 * +z,-z), edge [n,12] or corner [n,8] is a collision cell (uint8 0/1; each
 * output nullable).  Neighbours outside [0, resolution) are never wet. */
int a3d_dam_wet(const int32_t* dam_ijk, int64_t n, const int32_t* collision_ijk, int64_t m,
                const int64_t* collision_bbox, int64_t resolution, void* workspace,
                size_t workspace_bytes, uint8_t* wet_faces, uint8_t* wet_edges,
                uint8_t* wet_corners, a3d_stream_t stream);

/* ---- sparse differentiable dual marching cubes ------------------------ */
/* Replaces SparseDiffDMC.forward in training mode (weighted-average dual
 * vertices, 4-triangle quad split) and its autograd backward
 * (atom3d/mesh_extractor/sparse_diffdmc.py:76-232, :234-287, :516-871).
 * All pointers are device memory; deform/alpha/beta may be NULL (then the
 * reference's defaults: no deformation, unit weights). */
typedef struct a3d_dmc_inputs {
  const int64_t* voxel_coords;  /* [N,3]  */
  const float* sdf;             /* [M]    */
  const int64_t* cube_idx;      /* [N,8]  */
  const float* deform;          /* [M,3]  */
  const float* alpha;           /* [N,8]  raw (tanh-normalised inside) */
  const float* beta;            /* [N,12] raw */
  int64_t num_cubes;            /* N */
  int64_t num_corners;          /* M */
  int32_t resolution;
  float isovalue;
  float weight_scale;
} a3d_dmc_inputs;

size_t a3d_dmc_workspace_bytes(int64_t num_cubes, int64_t num_corners);
/* Topology pass.  counts (host, 6): surface cubes, groups G (crossing
 * cube-edges == L_dev/p_alpha/n_alpha rows), surface edges, quads Q, dual
 * vertices V; the workspace keeps the topology for _emit and _backward.
 * A cube_idx entry outside [0, num_corners) returns A3D_ERR_ARGUMENT (no
 * kernel reads or writes through it; the other DMC entry points read such
 * an entry as corner 0 and report nothing, so call this one first). */
int a3d_dmc_prepare(const a3d_dmc_inputs* in, void* workspace, size_t workspace_bytes,
                    int64_t* counts, a3d_stream_t stream);
/* Geometry pass: vertices [V+Q,3], faces [4Q,3] int64, L_dev [G],
 * p_alpha [G,3], n_alpha [G,3]. */
int a3d_dmc_emit(const a3d_dmc_inputs* in, void* workspace, size_t workspace_bytes,
                 const int64_t* counts, float* vertices, int64_t* faces, float* l_dev,
                 float* p_alpha, float* n_alpha, a3d_stream_t stream);
/* Adjoint: accumulates into g_sdf [M], g_deform [M,3], g_alpha [N,8],
 * g_beta [N,12] (each nullable, zero-initialised by the caller) from the
 * incoming gradients of the five outputs (each nullable).  Per-edge
 * quantities are recomputed, not stored. */
int a3d_dmc_backward(const a3d_dmc_inputs* in, void* workspace, size_t workspace_bytes,
                     const int64_t* counts, const float* g_vertices, const float* g_l_dev,
                     const float* g_p_alpha, const float* g_n_alpha, float* g_sdf,
                     float* g_deform, float* g_alpha, float* g_beta, a3d_stream_t stream);
/* Vertex features (SparseDiffDMC's v_features,
 * atom3d/mesh_extractor/sparse_diffdmc.py:658-663, :762-770, :815-818), after
 * a3d_dmc_emit or a3d_dmc_emit_qef on the same workspace: corner features
 * [M, channels] -> out [V (+Q with with_centres), channels], each dual
 * vertex's feature the beta-weighted mean of its crossings' alpha-weighted
 * interpolations (the weights of p_alpha); with_centres appends each quad's
 * mean (the training split's centre vertices).  The adjoint accumulates into
 * g_features [M, C], g_sdf [M], g_alpha [N, 8], g_beta [N, 12] (nullable,
 * zero-initialised by the caller); scratch [V, C], zeroed by the caller,
 * takes the centres' share when with_centres. */
int a3d_dmc_features(const a3d_dmc_inputs* in, void* workspace, size_t workspace_bytes,
                     const int64_t* counts, const float* features, int32_t channels,
                     int32_t with_centres, float* out, a3d_stream_t stream);
int a3d_dmc_features_backward(const a3d_dmc_inputs* in, void* workspace, size_t workspace_bytes,
                              const int64_t* counts, const float* features, int32_t channels,
                              int32_t with_centres, const float* g_out, float* scratch,
                              float* g_features, float* g_sdf, float* g_alpha, float* g_beta,
                              a3d_stream_t stream);
/* QEF inference mode (SparseDiffDMC in eval / inference_mode "qef",
 * atom3d/mesh_extractor/sparse_diffdmc.py:201-218, :289-513, :798-805).
 * Corner gradients: least-squares fit over every unique cube edge at each
 * corner (device [M,3]).  a3d_dmc_emit_qef runs after a3d_dmc_prepare on the
 * same workspace: vertices [V,3] (no quad centres), faces [2Q,3] (shorter
 * diagonal), L_dev / p_alpha / n_alpha [G] like a3d_dmc_emit; n_alpha holds
 * the crossing normals interpolated from the corner gradients.  The dual
 * vertex solves the least-squares system the reference's
 * _solve_qef_scatter assembles (its slot scatter places constraint j of k
 * in row (j - (k-1)) mod 10 of the 10 x 3 matrix). */
size_t a3d_dmc_corner_gradients_workspace_bytes(int64_t num_cubes, int64_t num_corners);
int a3d_dmc_corner_gradients(const a3d_dmc_inputs* in, void* workspace, size_t workspace_bytes,
                             float* gradients, a3d_stream_t stream);
int a3d_dmc_emit_qef(const a3d_dmc_inputs* in, void* workspace, size_t workspace_bytes,
                     const int64_t* counts, const float* corner_gradients, float qef_reg_scale,
                     float* vertices, int64_t* faces, float* l_dev, float* p_alpha, float* n_alpha,
                     a3d_stream_t stream);
/* Adjoint of a3d_dmc_emit_qef on the same workspace and the same corner
 * gradients: the reference differentiates the QEF vertices through
 * torch.linalg.lstsq, the crossings and the interpolated crossing normals
 * (atom3d/mesh_extractor/sparse_diffdmc.py:289-389, :610-650).  Gradients
 * w.r.t. vertices [V,3], L_dev [G], p_alpha [G,3], n_alpha [G,3] (each
 * nullable) are accumulated into g_sdf [M], g_deform [M,3], g_alpha [N,8]
 * and g_corner_gradients [M,3] (each nullable; the caller zeroes them).
 * Corner gradients the library estimated carry no gradient, as in the
 * reference (_estimate_corner_gradients runs under no_grad); pass
 * g_corner_gradients for gradients the caller supplied. */
int a3d_dmc_backward_qef(const a3d_dmc_inputs* in, void* workspace, size_t workspace_bytes,
                         const int64_t* counts, const float* corner_gradients, float qef_reg_scale,
                         const float* g_vertices, const float* g_l_dev, const float* g_p_alpha,
                         const float* g_n_alpha, float* g_sdf, float* g_deform, float* g_alpha,
                         float* g_corner_gradients, a3d_stream_t stream);

/* Status words of the last a3d_udf / a3d_batch_udf call that used
 * `workspace`, copied to the host after the stream drains:
 * [0] queries re-run by the deep-stack kernel, [1] deep-stack overflow (a
 * re-run query's result may be inexact), [2] 0, [3] guard faults of batch
 * queries (bit 0: a node index outside the node array, bit 1: a triangle
 * index outside the triangle array; the access was skipped).  No
 * counterpart in the reference. */
int a3d_udf_status(const void* workspace, uint32_t* status_out, a3d_stream_t stream);

/* ---- ray queries ---------------------------------------------------------
 * Replace bvh_ray_intersect_kernel / bvh_ray_all_hit_kernel
 * (atom3d/kernels/bvh_kernels.cu:469-553, :935-1022) behind
 * MeshBVH.intersect_ray (atom3d/core/mesh_bvh.py:1076-1160) and the
 * crossing-count loop of MeshBVH._sdf_parity (:850-948).  Triangle test:
 * Moller-Trumbore with the reference's thresholds (|det| >= 1e-8, FP64
 * u, v with FLT_EPSILON slack, t > 1e-8). */
size_t a3d_ray_workspace_bytes(int64_t num_rays);
/* Nearest hit per ray: hit flag, t (max_t on a miss), face id (-1 on a
 * miss), hit point (0 on a miss; nullable), normal = face_normals[face]
 * (nullable; needs face_normals), barycentrics as MeshBVH._bary_from_hit
 * (nullable). */
int a3d_ray_nearest(const a3d_bvh_view* bvh, const float* rays_o, const float* rays_d, int64_t num_rays,
                    float max_t, const float* face_normals, uint8_t* hit, float* t, int32_t* face_ids,
                    float* hit_points, float* normals, float* uvw, void* workspace,
                    size_t workspace_bytes, a3d_stream_t stream);
/* All non-grazing hits (|n.d| >= 1e-4) with 0 < t < max_t: the count pass
 * writes exclusive offsets [num_rays + 1] (device; total at the end), the
 * collect pass fills ray index, t, face id, sign(n.d), point and
 * barycentrics (Triangle::barycentric; both nullable), grouped by ray. */
int a3d_ray_all_count(const a3d_bvh_view* bvh, const float* rays_o, const float* rays_d, int64_t num_rays,
                      float max_t, int64_t* offsets_out, void* workspace, size_t workspace_bytes,
                      a3d_stream_t stream);
int a3d_ray_all_collect(const a3d_bvh_view* bvh, const float* rays_o, const float* rays_d, int64_t num_rays,
                        float max_t, const int64_t* offsets, int32_t* ray_idx, float* t, int32_t* face_ids,
                        int32_t* sign, float* hit_points, float* uvw, a3d_stream_t stream);
/* Per point, the number of directions whose signed crossing count, after
 * merging hits closer than coalesce_t along the ray, is odd. */
int a3d_ray_parity_votes(const a3d_bvh_view* bvh, const float* points, int64_t num_points, const float* dirs,
                         int32_t num_dirs, float max_t, float coalesce_t, int32_t* votes, void* workspace,
                         size_t workspace_bytes, a3d_stream_t stream);
/* [0] rays re-run with the deep stack, [1] stack or hit-buffer overflow
 * (results of some ray may be incomplete) of the last ray call on workspace. */
int a3d_ray_status(const void* workspace, uint32_t* status_out, a3d_stream_t stream);

/* ---- batches of meshes (no counterpart in the reference) ---------------- */
/* Many meshes of uneven size built into one wide-BVH array and queried by
 * persistent traversal launches shared by all meshes, with no host
 * synchronisation (build + query can be captured in a CUDA graph).  Mesh m
 * owns vertices [vertex_offsets[m], vertex_offsets[m+1]), faces
 * [face_offsets[m], face_offsets[m+1]) (vertex indices local to the mesh)
 * and queries [query_offsets[m], query_offsets[m+1]); the offset arrays live
 * on the device.  Face ids returned are local to the query's mesh.  Queries
 * are processed in launches of at most 16,777,216. */
typedef struct a3d_bvh_batch {
  const void* nodes;           /* num_faces x 64 B (capacity; the build writes the count) */
  const void* tris;            /* num_faces x 64 B */
  int64_t num_faces;
  int32_t num_meshes;
  const uint32_t* roots;       /* device [M]: root node of each mesh */
  const float* bounds;         /* device [M][6]: lo xyz, hi xyz */
} a3d_bvh_batch;

size_t a3d_batch_build_workspace_bytes(int64_t num_faces, int32_t num_meshes);
/* status_out (device int32[2], nullable): [0] bad face index or empty mesh,
 * [1] tree deeper than the collapse's level limit; read after the stream. */
int a3d_batch_build(const float* vertices, const int64_t* vertex_offsets, const int32_t* faces,
                    const int64_t* face_offsets, int32_t num_meshes, int64_t num_faces, int leaf_max,
                    void* nodes_out, void* tris_out, uint32_t* roots_out, float* bounds_out,
                    int64_t* num_nodes_out, int32_t* status_out, void* workspace,
                    size_t workspace_bytes, a3d_stream_t stream);

/* launch shape of the persistent traversal (0 = default) */
typedef struct a3d_udf_tuning {
  int32_t pool;           /* queries taken per work request */
  int32_t blocks_per_sm;  /* resident blocks per SM */
  int32_t leaf_max;       /* informational: the build's leaf size */
  int32_t reserved;
} a3d_udf_tuning;

size_t a3d_batch_udf_workspace_bytes(int64_t num_queries, int32_t num_meshes);
int a3d_batch_udf(const a3d_bvh_batch* bvh, const float* points, const int64_t* query_offsets,
                  int64_t num_queries, float* distances, int32_t* face_ids, float* closest_points,
                  float* uvw, const a3d_udf_tuning* tuning, unsigned long long* stats,
                  void* workspace, size_t workspace_bytes, a3d_stream_t stream);
/* Times the traversal's launch shapes on every ceil(Q/sample)-th query
 * (sample <= 16,777,216) and returns the fastest (host-synchronous; not
 * inside stream capture). */
size_t a3d_batch_autotune_workspace_bytes(int64_t sample_queries, int32_t num_meshes);
int a3d_batch_autotune(const a3d_bvh_batch* bvh, const float* points, const int64_t* query_offsets,
                       int64_t num_queries, int64_t sample_queries, void* workspace,
                       size_t workspace_bytes, a3d_udf_tuning* best, float* best_ms,
                       a3d_stream_t stream);

/* ---- learned distance bound (no counterpart in the reference) ----------- */
/* A Fourier-feature MLP (3 -> 64 -> 128 -> 128 -> 128 -> 1, ReLU) predicts
 * a query's unsigned distance (or its logarithm); bound = max(y, 0) * scale
 * + margin (exp(y) * scale + margin in log space) seeds a3d_udf's pruning
 * radius (results never depend on it).  Inference is one fused kernel on the
 * tcgen05 tensor cores (BF16 operands in shared memory, FP32 accumulators in
 * tensor memory, one CTA per SM, 128 queries per warpgroup tile); the weight
 * matrices must be 16-byte aligned.  Training uses the kernels below. */
typedef struct a3d_mlp_weights {
  const void* w1t;   /* bf16 [128][64]  (W1 transposed, out-major) */
  const void* w2t;   /* bf16 [128][128] */
  const void* w3t;   /* bf16 [128][128] */
  const float* b1;   /* [128] */
  const float* b2;
  const float* b3;
  const float* w4;   /* [128] head weights */
  float b4;
  const float* freq; /* [32][3] Fourier frequencies */
  float norm[4];     /* x_hat = (x - norm[0..2]) * norm[3] */
  float scale;
  float margin;
  int32_t log_space; /* nonzero: y predicts log(distance), bound = exp(y) * scale + margin */
} a3d_mlp_weights;

int a3d_mlp_bound(const a3d_mlp_weights* w, const float* x, int64_t n, float* bound,
                  a3d_stream_t stream);
/* Status of the last a3d_mlp_bound launch on the current device (waits for
 * `stream`): bit 0 set when a tile's tensor-core wait ran out, in which case
 * bounds of the tiles not reached were left unwritten.  Calls that overlap
 * on the GPU share the word. */
int a3d_mlp_bound_status(unsigned int* status, a3d_stream_t stream);

/* training building blocks (BF16 operands, FP32 accumulation) */
typedef struct a3d_gemm_args {
  const void* A;           /* bf16, element (m,k) at A[m*sam + k*sak] */
  const void* B;           /* bf16, element (k,n) at B[k*sbk + n*sbn] */
  int64_t sam, sak, sbk, sbn;
  int32_t m, n, k;
  const float* bias;       /* [n] or NULL */
  const void* mask;        /* bf16 [m,n]: result zeroed where mask <= 0, or NULL */
  int32_t relu;
  float* Cf;               /* fp32 [m,n] or NULL */
  int32_t accumulate;      /* Cf += result */
  void* Cb;                /* bf16 [m,n] or NULL */
} a3d_gemm_args;
int a3d_gemm_bf16(const a3d_gemm_args* args, a3d_stream_t stream);
int a3d_mlp_fourier(const float* x, int64_t n, const float* norm4, const float* freq,
                    void* feat_bf16, a3d_stream_t stream);
int a3d_mlp_head(const void* h_bf16, int64_t n, const float* w4, const float* b4,
                 const float* target, float under_weight, float* y, void* dh_bf16,
                 float* dw4, float* db4, float* loss, a3d_stream_t stream);
int a3d_mlp_colsum(const void* g_bf16, int64_t n, int cols, float* out, a3d_stream_t stream);
int a3d_adam(float* p, const float* g, float* m, float* v, int64_t n, float lr, float beta1,
             float beta2, float eps, int step, a3d_stream_t stream);
int a3d_to_bf16(const float* in, int64_t n, void* out, a3d_stream_t stream);

#ifdef __cplusplus
}
#endif

#endif /* ATOM3D_B200_H_ */
