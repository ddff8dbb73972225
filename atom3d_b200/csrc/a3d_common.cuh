// Shared device helpers for the atom3d_b200 kernels (sm_100a).
//
// Every entry point of libatom3d_b200.so returns an int status (A3D_OK = 0)
// instead of throwing across the C ABI; the codes are declared in
// include/atom3d_b200.h.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include "../../include/atom3d_b200.h"

#define A3D_CUDA_TRY(expr)                                  \
  do {                                                      \
    cudaError_t _e = (expr);                                \
    if (_e != cudaSuccess) {                                \
      a3d_set_error(cudaGetErrorString(_e), __FILE__, __LINE__); \
      return A3D_ERR_CUDA;                                  \
    }                                                       \
  } while (0)

#define A3D_LAUNCH_CHECK()                                  \
  do {                                                      \
    cudaError_t _e = cudaGetLastError();                    \
    if (_e != cudaSuccess) {                                \
      a3d_set_error(cudaGetErrorString(_e), __FILE__, __LINE__); \
      return A3D_ERR_CUDA;                                  \
    }                                                       \
  } while (0)

#define A3D_TRY(expr)                                       \
  do {                                                      \
    int _s = (expr);                                        \
    if (_s != A3D_OK) return _s;                            \
  } while (0)

// launch `kernel` with programmatic dependent launch (see launch_pdl)
#define A3D_PDL(kernel, grid, block, smem, stream, ...) \
  A3D_CUDA_TRY(::a3d::launch_pdl(kernel, grid, block, smem, stream, __VA_ARGS__))

#define A3D_REQUIRE(cond, code, msg)                        \
  do {                                                      \
    if (!(cond)) {                                          \
      a3d_set_error(msg, __FILE__, __LINE__);               \
      return (code);                                        \
    }                                                       \
  } while (0)

// Records the last error message (thread-local, host side).
void a3d_set_error(const char* msg, const char* file, int line);

namespace a3d {

// streaming multiprocessors of the current device (queried once per device;
// 148 on B200), for sizing persistent and grid-stride launches
int num_sms();
constexpr int kMaxDevices = 64;

__host__ __device__ inline int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }

// Programmatic dependent launch.  A kernel started with launch_pdl may be
// scheduled while the previous kernel on the stream is still draining, which
// hides the launch gap between dependent kernels; it must call pdl_wait()
// (griddepcontrol.wait) before it touches memory, which returns once the
// previous kernel has completed and its writes are visible, so the effects
// keep the stream order.  pdl_wait() is a no-op in a kernel launched
// without the attribute.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

template <typename... KArgs, typename... Args>
cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                       Args... args) {
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
}

// Bump allocator over a caller-provided workspace.  Every sub-buffer is
// 256-byte aligned so that vector loads and bulk copies stay aligned.
struct Workspace {
  char* base;
  size_t size;
  size_t used;
  bool measuring;  // when true only sizes are accumulated (base may be null)

  __host__ Workspace(void* b, size_t s) : base((char*)b), size(s), used(0), measuring(b == nullptr) {}

  template <typename T>
  __host__ T* take(int64_t count) {
    size_t bytes = ((size_t)(count > 0 ? count : 1) * sizeof(T) + 255) & ~(size_t)255;
    size_t off = used;
    used += bytes;
    if (measuring || used > size) return nullptr;
    return reinterpret_cast<T*>(base + off);
  }
  __host__ bool ok() const { return measuring || used <= size; }
};

// float <-> order-preserving uint32 (for atomic min/max on floats)
__device__ __forceinline__ uint32_t float_flip(float f) {
  uint32_t u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float float_unflip(uint32_t u) {
  return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

// Spread the low 21 bits of v so that bit i lands on bit 3i.
__host__ __device__ __forceinline__ uint64_t spread3_21(uint64_t v) {
  v &= 0x1fffffull;
  v = (v | (v << 32)) & 0x1f00000000ffffull;
  v = (v | (v << 16)) & 0x1f0000ff0000ffull;
  v = (v | (v << 8)) & 0x100f00f00f00f00full;
  v = (v | (v << 4)) & 0x10c30c30c30c30c3ull;
  v = (v | (v << 2)) & 0x1249249249249249ull;
  return v;
}
__host__ __device__ __forceinline__ uint64_t compact3_21(uint64_t v) {
  v &= 0x1249249249249249ull;
  v = (v | (v >> 2)) & 0x10c30c30c30c30c3ull;
  v = (v | (v >> 4)) & 0x100f00f00f00f00full;
  v = (v | (v >> 8)) & 0x1f0000ff0000ffull;
  v = (v | (v >> 16)) & 0x1f00000000ffffull;
  v = (v | (v >> 32)) & 0x1fffffull;
  return v;
}

}  // namespace a3d
