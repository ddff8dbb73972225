// The device-wide scan and radix sort (primitives.cuh) as C entry points:
// building blocks for callers writing their own compactions and orders,
// and the handle the tests use to check them at any size.
#include "primitives.cuh"

using namespace a3d;

extern "C" size_t a3d_exclusive_scan_workspace_bytes(int64_t n) {
  Workspace ws(nullptr, 0);
  ws.take<int64_t>((int64_t)scan_workspace_elems(n));
  return ws.used + 256;
}

extern "C" int a3d_exclusive_scan_u32(const uint32_t* in, int64_t n, int64_t* out, void* workspace,
                                      size_t workspace_bytes, a3d_stream_t stream) {
  A3D_REQUIRE(n >= 0 && out && (n == 0 || in), A3D_ERR_ARGUMENT, "exclusive_scan: bad argument");
  Workspace ws(workspace, workspace_bytes);
  int64_t* tmp = ws.take<int64_t>((int64_t)scan_workspace_elems(n));
  A3D_REQUIRE(workspace && ws.ok(), A3D_ERR_WORKSPACE, "exclusive_scan: workspace too small");
  return device_exclusive_scan<uint32_t, int64_t>(in, out, n, tmp, out + n, (cudaStream_t)stream);
}

extern "C" size_t a3d_sort_pairs_workspace_bytes(int64_t n) {
  Workspace ws(nullptr, 0);
  ws.take<uint64_t>(n);
  ws.take<uint32_t>(n);
  ws.take<uint32_t>((int64_t)radix_sort_scratch_elems(n));
  return ws.used + 256;
}

extern "C" int a3d_sort_pairs_u64(uint64_t* keys, uint32_t* vals, int64_t n, int begin_bit, int end_bit,
                                  void* workspace, size_t workspace_bytes, a3d_stream_t stream) {
  cudaStream_t s = (cudaStream_t)stream;
  A3D_REQUIRE(n >= 0 && n < (int64_t)0xffffffffll && (n == 0 || (keys && vals)), A3D_ERR_ARGUMENT,
              "sort_pairs: bad argument");
  A3D_REQUIRE(begin_bit >= 0 && begin_bit <= end_bit && end_bit <= 64, A3D_ERR_ARGUMENT, "sort_pairs: bad bit range");
  Workspace ws(workspace, workspace_bytes);
  uint64_t* keys_alt = ws.take<uint64_t>(n);
  uint32_t* vals_alt = ws.take<uint32_t>(n);
  uint32_t* scratch = ws.take<uint32_t>((int64_t)radix_sort_scratch_elems(n));
  A3D_REQUIRE(workspace && ws.ok(), A3D_ERR_WORKSPACE, "sort_pairs: workspace too small");
  bool in_alt = false;
  A3D_TRY(radix_sort_pairs<uint64_t>(keys, vals, keys_alt, vals_alt, n, begin_bit, end_bit, scratch, &in_alt, s));
  if (in_alt) {
    A3D_CUDA_TRY(cudaMemcpyAsync(keys, keys_alt, n * sizeof(uint64_t), cudaMemcpyDeviceToDevice, s));
    A3D_CUDA_TRY(cudaMemcpyAsync(vals, vals_alt, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
  }
  return A3D_OK;
}

namespace {

// Streams `n16` 16-byte words `passes` times through L2 only (ld.global.cg),
// folding them into one word per thread so no load is dead.  Timed on a
// buffer that fits in L2 it gives the L2 read bandwidth that an L2-resident
// working set (a BVH of a few tens of MB) is measured against.
__global__ void __launch_bounds__(512) read_probe_kernel(const uint4* __restrict__ p, int64_t n16, int passes,
                                                         uint32_t* __restrict__ sink) {
  uint32_t acc = 0;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int k = 0; k < passes; ++k) {
    // each pass starts at another block's slice, so no SM re-reads its own
    const int64_t start = (int64_t)((blockIdx.x + k * 37u) % gridDim.x) * blockDim.x + threadIdx.x;
    for (int64_t i = start; i < n16; i += stride) {
      const uint4 v = __ldcg(p + i);
      acc ^= v.x ^ v.y ^ v.z ^ v.w;
    }
  }
  if (acc == 0x9e3779b9u) sink[0] = acc;  // practically never taken; keeps the loads live
}

}  // namespace

extern "C" int a3d_read_probe(const void* buf, int64_t bytes, int passes, uint32_t* sink, a3d_stream_t stream) {
  A3D_REQUIRE(buf && sink && bytes >= 16 && bytes % 16 == 0 && passes > 0, A3D_ERR_ARGUMENT,
              "read_probe: bad argument");
  A3D_REQUIRE(((uintptr_t)buf & 15u) == 0, A3D_ERR_ARGUMENT, "read_probe: buffer must be 16-byte aligned");
  const int sms = num_sms();
  read_probe_kernel<<<(unsigned)(4 * sms), 512, 0, (cudaStream_t)stream>>>((const uint4*)buf, bytes / 16, passes,
                                                                          sink);
  A3D_LAUNCH_CHECK();
  return A3D_OK;
}
