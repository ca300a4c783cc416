// noalloc.cu — pyro_k_forces without any device allocation.
//
// pyro_k_forces needs one float4 of scratch per cell for the vorticity-
// confinement force of each cell; it allocates that scratch with cudaMalloc
// on every call.  Some callers cannot allocate: code that runs while a CUDA
// graph is being captured elsewhere in the process, hosts that hand the GPU's
// memory to their own pool allocator and forbid any other allocation, and
// real-time loops where cudaMalloc's implicit device synchronisation would
// stall the pipeline.  pyro_k_forces_noalloc gives them the same kernels with
// the scratch in a fixed array that this library owns for the lifetime of the
// process.
//
// The array lives in device global memory declared at file scope.  Its name
// is only a host-side stand-in in host code, so the device address is looked
// up with cudaGetSymbolAddress once per device (on the first call made with
// that device current) and then passed to the kernels.
#include <mutex>
#include <string>

#include "runtime.h"

using namespace pyro;

namespace {

constexpr size_t kNoAllocMaxCells = PYRO_NOALLOC_MAX_CELLS;

// One float4 of confinement force per cell: 8 MiB on every GPU that loads
// the library, held until the process exits.  Every call overwrites the
// cells it uses before reading them, so nothing needs to start at zero.
static __device__ __align__(256) float4 g_noalloc_scratch[kNoAllocMaxCells];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
float4* g_addr[kMaxDevices] = {};

// Device address of the scratch array on the current device.
int scratch_on_current_device(float4** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    set_error(std::string("pyro_k_forces_noalloc: cudaGetDevice: ") + cudaGetErrorString(e));
    return PYRO_E_CUDA;
  }
  if (dev < 0 || dev >= kMaxDevices) {
    set_error("pyro_k_forces_noalloc: device index out of range");
    return PYRO_E_INVALID;
  }
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr) {
      set_error(std::string("pyro_k_forces_noalloc: cudaGetSymbolAddress: ") +
                cudaGetErrorString(e));
      return PYRO_E_CUDA;
    }
    g_addr[dev] = static_cast<float4*>(p);
  }
  *out = g_addr[dev];
  return PYRO_OK;
}

}  // namespace

extern "C" int pyro_k_forces_noalloc(const PyroParams* params_dev, uint32_t nx, uint32_t ny,
                                     uint32_t nz, float* u, float* v, float* w, const float* s0,
                                     const float* s1, const float* curl, const uint32_t* flags,
                                     void* stream) {
  clear_error();
  PYRO_REQUIRE(params_dev, "pyro_k_forces_noalloc: null parameter block");
  PYRO_REQUIRE(nx >= 2 && ny >= 2 && nz >= 2 &&
                   (uint64_t)(nx + 1) * (ny + 1) * (nz + 1) < (1ull << 31),
               "pyro_k_forces_noalloc: invalid grid dimensions");
  PYRO_REQUIRE(u && v && w && s0 && s1 && curl && flags, "pyro_k_forces_noalloc: null buffer");
  uint64_t cells = (uint64_t)nx * ny * nz;
  if (cells > kNoAllocMaxCells) {
    set_error("pyro_k_forces_noalloc: grid of " + std::to_string(cells) +
              " cells exceeds the fixed scratch of " + std::to_string(kNoAllocMaxCells) +
              " cells; use pyro_k_forces");
    return PYRO_E_INVALID;
  }
  float4* scratch = nullptr;
  int rc = scratch_on_current_device(&scratch);
  if (rc != PYRO_OK) return rc;
  cudaError_t e = launch_forces(params_dev, Dims3{(int)nx, (int)ny, (int)nz}, u, v, w,
                                (const float4*)s0, (const float4*)s1, (const float4*)curl,
                                scratch, flags, reinterpret_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) {
    set_error(std::string("pyro_k_forces_noalloc: ") + cudaGetErrorString(e));
    return PYRO_E_CUDA;
  }
  return PYRO_OK;
}
