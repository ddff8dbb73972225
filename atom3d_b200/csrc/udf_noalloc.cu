// Allocation-free closest-point query.
//
// Some callers cannot call cudaMalloc: code embedded in a host application
// that owns all device memory (a fixed budget or its own pool allocator), or
// a latency-critical loop where cudaMalloc/cudaFree would synchronise the
// device.  a3d_udf_noalloc serves them: the caller passes only the inputs
// and outputs, and the query's scratch (Morton keys, sort buffers, re-run
// list) lives in the file-scope device array below, which every GPU that
// loads this library holds until the process exits.
//
// Limits and rules:
//   * at most kNoAllocMaxQueries queries per call (longer batches: loop);
//   * the first call on a device looks up the array's device address with
//     cudaGetSymbolAddress (with that device current) and caches it; make
//     that first call before any stream capture;
//   * all calls share the array and it keeps the last call's contents; the
//     query clears the counters it needs itself; calls whose executions
//     overlap on the GPU (different streams without ordering) race on it.
#include <mutex>

#include "a3d_common.cuh"

namespace a3d {
size_t udf_required_workspace_bytes(int64_t num_points, uint32_t flags);
}

namespace {

constexpr int64_t kNoAllocMaxQueries = 1ll << 20;    // 1,048,576 queries per call
constexpr size_t kNoAllocScratchBytes = 24ull << 20;  // 24 MiB per GPU
constexpr int kMaxDevices = 64;

}  // namespace

static __device__ __align__(256) unsigned char g_udf_scratch[kNoAllocScratchBytes];

namespace {

std::mutex g_setup_mutex;
void* g_scratch_addr[kMaxDevices] = {nullptr};

// Device address of the scratch array on the current device (set-up on the
// first call per device).
int scratch_address(void** out) {
  int dev = 0;
  A3D_CUDA_TRY(cudaGetDevice(&dev));
  A3D_REQUIRE(dev >= 0 && dev < kMaxDevices, A3D_ERR_ARGUMENT, "udf_noalloc: device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (g_scratch_addr[dev] == nullptr) {
    void* p = nullptr;
    A3D_CUDA_TRY(cudaGetSymbolAddress(&p, g_udf_scratch));
    A3D_REQUIRE(p != nullptr, A3D_ERR_CUDA, "udf_noalloc: no device address for the scratch array");
    g_scratch_addr[dev] = p;
  }
  *out = g_scratch_addr[dev];
  return A3D_OK;
}

}  // namespace

extern "C" int a3d_udf_noalloc(const a3d_bvh_view* bvh, const float* points, int64_t num_points, float* distances,
                               int32_t* face_ids, float* closest_points, float* uvw, a3d_stream_t stream) {
  A3D_REQUIRE(num_points >= 0, A3D_ERR_ARGUMENT, "udf_noalloc: negative number of points");
  A3D_REQUIRE(num_points <= kNoAllocMaxQueries, A3D_ERR_ARGUMENT,
              "udf_noalloc: at most 1048576 queries per call; split larger batches");
  if (num_points == 0) return A3D_OK;
  // the query's required scratch; any remainder of the array serves as
  // optional overflow stacks
  const size_t need = a3d::udf_required_workspace_bytes(num_points, A3D_UDF_SORT_QUERIES);
  A3D_REQUIRE(need <= kNoAllocScratchBytes, A3D_ERR_WORKSPACE, "udf_noalloc: static scratch smaller than required");
  void* scratch = nullptr;
  A3D_TRY(scratch_address(&scratch));
  return a3d_udf(bvh, points, num_points, distances, face_ids, closest_points, uvw, nullptr, nullptr, nullptr,
                 A3D_UDF_SORT_QUERIES, scratch, kNoAllocScratchBytes, stream);
}

extern "C" int a3d_udf_noalloc_status(uint32_t* status_out, a3d_stream_t stream) {
  A3D_REQUIRE(status_out, A3D_ERR_ARGUMENT, "udf_noalloc_status: null output");
  void* scratch = nullptr;
  A3D_TRY(scratch_address(&scratch));
  return a3d_udf_status(scratch, status_out, stream);
}
