// Pseudo-normal precompute for the SDF sign (Baerentzen & Aanaes).
//
// Replaces MeshBVH._precompute_face_normals and
// MeshBVH._precompute_pseudo_normal_data (atom3d/core/mesh_bvh.py:129-232):
//   face normal for the sign       n / (|n| + 1e-8)
//   unit face normal               n / (|n| + 1e-12)
//   interior angles                acos(clamp(a.b / (|a||b| + 1e-12), -1, 1))
//   vertex pseudo-normal           normalise(sum angle * unit face normal)
//   edge pseudo-normal             normalise(sum of the adjacent unit normals)
// Edges are keyed lo*V + hi; sorting the 3F half-edge keys with the in-house
// radix sort numbers the edges in ascending key order, which is the order
// torch.unique produces, so he_edge_idx matches the reference's inverse map.
#include <math.h>

#include "primitives.cuh"

namespace a3d {
namespace {

__global__ void face_kernel(const float* __restrict__ V, const int32_t* __restrict__ F, int64_t nf, int64_t nv,
                            float* __restrict__ fn_sign, float* __restrict__ fn_unit, float* __restrict__ ang,
                            float* __restrict__ vacc, uint64_t* __restrict__ keys, uint32_t* __restrict__ vals,
                            uint32_t* __restrict__ bad_face) {
  pdl_wait();
  const int64_t f = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= nf) return;
  int64_t id[3] = {F[3 * f], F[3 * f + 1], F[3 * f + 2]};
  // a face index outside [0, nv) is reported after the edge count is read;
  // until then the face reads as a point at vertex 0
  if (id[0] < 0 || id[1] < 0 || id[2] < 0 || id[0] >= nv || id[1] >= nv || id[2] >= nv) {
    *bad_face = 1u;
    id[0] = id[1] = id[2] = 0;
  }
  float p[3][3];
#pragma unroll
  for (int k = 0; k < 3; ++k)
#pragma unroll
    for (int a = 0; a < 3; ++a) p[k][a] = V[3 * id[k] + a];
  float e01[3], e02[3], e10[3], e12[3], e20[3], e21[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    e01[a] = p[1][a] - p[0][a]; e02[a] = p[2][a] - p[0][a];
    e10[a] = p[0][a] - p[1][a]; e12[a] = p[2][a] - p[1][a];
    e20[a] = p[0][a] - p[2][a]; e21[a] = p[1][a] - p[2][a];
  }
  auto nrm = [](const float* v) { return sqrtf(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]); };
  auto angle = [&](const float* a, const float* b) {
    float c = (a[0] * b[0] + a[1] * b[1] + a[2] * b[2]) / (nrm(a) * nrm(b) + 1e-12f);
    c = fminf(fmaxf(c, -1.f), 1.f);
    return acosf(c);
  };
  const float a0 = angle(e01, e02), a1 = angle(e10, e12), a2 = angle(e20, e21);
  const float n[3] = {e01[1] * e02[2] - e01[2] * e02[1], e01[2] * e02[0] - e01[0] * e02[2],
                      e01[0] * e02[1] - e01[1] * e02[0]};
  const float ln = nrm(n);
  const float iu = 1.f / (ln + 1e-12f), is = 1.f / (ln + 1e-8f);
  float u[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    u[a] = n[a] / (ln + 1e-12f);
    fn_unit[3 * f + a] = u[a];
    fn_sign[3 * f + a] = n[a] / (ln + 1e-8f);
  }
  (void)iu; (void)is;
  ang[3 * f] = a0; ang[3 * f + 1] = a1; ang[3 * f + 2] = a2;
  const float w[3] = {a0, a1, a2};
#pragma unroll
  for (int k = 0; k < 3; ++k)
#pragma unroll
    for (int a = 0; a < 3; ++a) atomicAdd(&vacc[3 * id[k] + a], w[k] * u[a]);
  // half-edges 3f+0: v0v1, 3f+1: v1v2, 3f+2: v2v0
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const int64_t va = id[k], vb = id[(k + 1) % 3];
    const int64_t lo = va < vb ? va : vb, hi = va < vb ? vb : va;
    keys[3 * f + k] = (uint64_t)(lo * nv + hi);
    vals[3 * f + k] = (uint32_t)(3 * f + k);
  }
}

__global__ void normalize_rows_kernel(const float* __restrict__ in, float* __restrict__ out, int64_t n) {
  pdl_wait();
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float x = in[3 * i], y = in[3 * i + 1], z = in[3 * i + 2];
  const float l = sqrtf(x * x + y * y + z * z) + 1e-12f;
  out[3 * i] = x / l; out[3 * i + 1] = y / l; out[3 * i + 2] = z / l;
}

__global__ void run_start_kernel(const uint64_t* __restrict__ k, int64_t n, uint32_t* __restrict__ flag) {
  pdl_wait();
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  flag[i] = (i == 0 || k[i] != k[i - 1]) ? 1u : 0u;
}

// one thread per sorted half-edge that starts a run: sums the run's unit
// normals in sorted (half-edge index) order and writes the edge id of every
// half-edge of the run
__global__ void edge_kernel(const uint64_t* __restrict__ k, const uint32_t* __restrict__ he, int64_t n,
                            const uint32_t* __restrict__ start_flag, const uint32_t* __restrict__ edge_id,
                            const float* __restrict__ fn_unit, float* __restrict__ edge_pn,
                            int64_t* __restrict__ he_edge_idx) {
  pdl_wait();
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || !start_flag[i]) return;
  const uint32_t e = edge_id[i];
  float s[3] = {0.f, 0.f, 0.f};
  int64_t j = i;
  do {
    const uint32_t h = he[j];
    const int64_t f = h / 3;
    s[0] += fn_unit[3 * f]; s[1] += fn_unit[3 * f + 1]; s[2] += fn_unit[3 * f + 2];
    he_edge_idx[h] = e;
    ++j;
  } while (j < n && k[j] == k[i]);
  const float l = sqrtf(s[0] * s[0] + s[1] * s[1] + s[2] * s[2]) + 1e-12f;
  edge_pn[3 * e] = s[0] / l; edge_pn[3 * e + 1] = s[1] / l; edge_pn[3 * e + 2] = s[2] / l;
}

struct NrmWs {
  float* fn_unit;
  float* vacc;
  uint64_t* keys;
  uint64_t* keys_alt;
  uint32_t* vals;
  uint32_t* vals_alt;
  uint32_t* rs;
  uint32_t* flag;
  uint32_t* eid;
  uint32_t* scan_tmp;
  uint32_t* total;  // [0] unique edges, [1] out-of-range face flag
};
size_t carve_nrm(NrmWs& w, Workspace& ws, int64_t nv, int64_t nf) {
  const int64_t nh = 3 * nf;
  w.fn_unit = ws.take<float>(3 * nf);
  w.vacc = ws.take<float>(3 * nv);
  w.keys = ws.take<uint64_t>(nh);
  w.keys_alt = ws.take<uint64_t>(nh);
  w.vals = ws.take<uint32_t>(nh);
  w.vals_alt = ws.take<uint32_t>(nh);
  w.rs = ws.take<uint32_t>((int64_t)radix_sort_scratch_elems(nh));
  w.flag = ws.take<uint32_t>(nh);
  w.eid = ws.take<uint32_t>(nh);
  w.scan_tmp = ws.take<uint32_t>((int64_t)scan_workspace_elems(nh));
  w.total = ws.take<uint32_t>(2);
  return ws.used;
}

}  // namespace
}  // namespace a3d

using namespace a3d;

extern "C" size_t a3d_mesh_normals_workspace_bytes(int64_t num_vertices, int64_t num_faces) {
  Workspace ws(nullptr, 0);
  NrmWs w;
  return carve_nrm(w, ws, num_vertices > 0 ? num_vertices : 1, num_faces > 0 ? num_faces : 1) + 256;
}

extern "C" int a3d_mesh_normals(const float* vertices, int64_t num_vertices, const int32_t* faces, int64_t num_faces,
                                float* face_normals_sign, float* face_angles, float* vertex_pn, float* edge_pn,
                                int64_t edge_capacity, int64_t* he_edge_idx, int64_t* num_edges_out, void* workspace,
                                size_t workspace_bytes, a3d_stream_t stream) {
  cudaStream_t s = (cudaStream_t)stream;
  A3D_REQUIRE(num_vertices > 0 && num_faces > 0, A3D_ERR_ARGUMENT, "mesh_normals: empty mesh");
  A3D_REQUIRE(num_faces < (1ll << 30), A3D_ERR_ARGUMENT, "mesh_normals: too many faces");
  A3D_REQUIRE(num_vertices < (1ll << 31), A3D_ERR_ARGUMENT, "mesh_normals: too many vertices");
  A3D_REQUIRE(vertices && faces && face_normals_sign && face_angles && vertex_pn && he_edge_idx &&
                  (edge_pn || edge_capacity == 0),
              A3D_ERR_ARGUMENT, "mesh_normals: null pointer");
  Workspace ws(workspace, workspace_bytes);
  NrmWs w;
  carve_nrm(w, ws, num_vertices, num_faces);
  A3D_REQUIRE(workspace && ws.ok(), A3D_ERR_WORKSPACE, "mesh_normals: workspace too small");
  const int64_t nh = 3 * num_faces;
  A3D_CUDA_TRY(cudaMemsetAsync(w.vacc, 0, sizeof(float) * 3 * num_vertices, s));
  A3D_CUDA_TRY(cudaMemsetAsync(w.total, 0, sizeof(uint32_t) * 2, s));
  A3D_PDL(face_kernel, dim3((unsigned)ceil_div(num_faces, 256)), dim3(256), 0, s, vertices, faces, num_faces,
          num_vertices, face_normals_sign, w.fn_unit, face_angles, w.vacc, w.keys, w.vals, w.total + 1);
  A3D_PDL(normalize_rows_kernel, dim3((unsigned)ceil_div(num_vertices, 256)), dim3(256), 0, s, w.vacc, vertex_pn,
          num_vertices);
  // key bits: lo*V+hi < V^2
  int bits = 1;
  while (bits < 64 && ((unsigned __int128)1 << bits) < (unsigned __int128)num_vertices * num_vertices) ++bits;
  const int end_bit = ((bits + 7) / 8) * 8;
  bool alt = false;
  A3D_TRY(radix_sort_pairs<uint64_t>(w.keys, w.vals, w.keys_alt, w.vals_alt, nh, 0, end_bit, w.rs, &alt, s));
  const uint64_t* k = alt ? w.keys_alt : w.keys;
  const uint32_t* he = alt ? w.vals_alt : w.vals;
  A3D_PDL(run_start_kernel, dim3((unsigned)ceil_div(nh, 256)), dim3(256), 0, s, k, nh, w.flag);
  A3D_TRY((device_exclusive_scan<uint32_t, uint32_t>(w.flag, w.eid, nh, w.scan_tmp, w.total, s)));
  uint32_t h[2] = {0, 0};
  A3D_CUDA_TRY(cudaMemcpyAsync(h, w.total, sizeof(h), cudaMemcpyDeviceToHost, s));
  A3D_CUDA_TRY(cudaStreamSynchronize(s));
  A3D_REQUIRE(h[1] == 0u, A3D_ERR_ARGUMENT, "mesh_normals: face index outside [0, num_vertices)");
  const uint32_t ne = h[0];
  if (num_edges_out) *num_edges_out = ne;
  A3D_REQUIRE((int64_t)ne <= edge_capacity, A3D_ERR_WORKSPACE, "mesh_normals: edge capacity too small");
  A3D_PDL(edge_kernel, dim3((unsigned)ceil_div(nh, 256)), dim3(256), 0, s, k, he, nh, w.flag, w.eid, w.fn_unit, edge_pn,
          he_edge_idx);
  return A3D_OK;
}
