// runtime.h — internal host runtime: error state, device buffers, the
// multigrid hierarchy shared by the simulation and the stand-alone Poisson
// solver.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/pyro_sim.h"
#include "kernels.h"

namespace pyro {

// Thread-local last error text (pyro_last_error).
void set_error(const std::string& msg);
void clear_error();

#define PYRO_CU(call)                                                                   \
  do {                                                                                  \
    cudaError_t e_ = (call);                                                            \
    if (e_ != cudaSuccess) {                                                            \
      ::pyro::set_error(std::string(#call) + ": " + cudaGetErrorString(e_));            \
      return e_ == cudaErrorMemoryAllocation ? PYRO_E_NOMEM : PYRO_E_CUDA;              \
    }                                                                                   \
  } while (0)

#define PYRO_REQUIRE(cond, msg)        \
  do {                                 \
    if (!(cond)) {                     \
      ::pyro::set_error(msg);          \
      return PYRO_E_INVALID;           \
    }                                  \
  } while (0)

// Owning device allocation.
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  int alloc(size_t n);
  void release();
  ~DevBuf() { release(); }
  template <typename T>
  T* as() const { return reinterpret_cast<T*>(p); }
};

// Multigrid hierarchy (src/sim.rs:142-168): <= 4 levels, stop after the
// first level whose smallest dimension is < 16, halve with ceil, h doubles.
// Level 0 arrays are bound from outside; the coarse levels are owned.
struct Multigrid {
  int bc_mode = 0;
  std::vector<Dims3> dims;
  std::vector<float> h;
  std::vector<float*> phi, b;
  std::vector<const uint32_t*> f;
  std::vector<DevBuf> own_phi, own_b, own_f;
  std::vector<DevBuf> phi2;   // ping-pong partner of phi on every level
  std::vector<DevBuf> meta;   // per-cell neighbour mask (k_mgf.cu)
  bool coarse_one_cta = false;
  float* stats = nullptr;  // device, for mg_resid

  int init(Dims3 d0, float h0, int bc);
  void bind_level0(float* phi0, const float* b0, const uint32_t* f0) {
    phi[0] = phi0;
    b[0] = const_cast<float*>(b0);
    f[0] = f0;
  }
  size_t levels() const { return dims.size(); }
  // One smoother pass schedule (src/sim.rs:425-449), one launch per colour.
  cudaError_t smooth(int l, int iters, bool coarse, cudaStream_t st);
  // Coarse solid flags and neighbour masks of every level from the bound
  // level-0 flags; the V-cycles below need them (once per new flag field).
  cudaError_t prepare(cudaStream_t st);
  // `cycles` V-cycles (src/sim.rs:451-491) on the bound level-0 arrays with
  // the fused kernels (k_mgf.cu); calls prepare() first.
  cudaError_t vcycles(int cycles, cudaStream_t st);
  // Symmetric V-cycle for the CG preconditioner: pre-smoothing red-black,
  // post-smoothing black-red, restriction P^T/8 of the fluid-normalised
  // trilinear prolongation, coarsest level by alternating SOR sweeps.  With
  // bphi != nullptr phi and b are stored in BF16 (FP32 arithmetic).  The
  // initial guess is zero: level 0's phi must hold zeros in FP32 storage
  // and is not read in BF16 storage (the result overwrites all of it).
  // prep = false skips the per-level masks (valid while the level flags
  // are unchanged since the last prepare()).
  cudaError_t vcycle_sym(cudaStream_t st, DevBuf* bphi, DevBuf* bphi2, DevBuf* bb,
                         bool prep = true);
  size_t device_bytes() const;
};

// Level dims of the reference rule (shared with the C ABI).
std::vector<Dims3> mg_level_dims(Dims3 d0, int max_levels);

}  // namespace pyro
