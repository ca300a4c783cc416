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
// Launch classes of the V-cycle, for per-launch timing
// (pyro_sim_profile_pressure).
enum MgClass {
  MG_PREPARE = 0,  // coarse flags and neighbour masks of every level
  MG_PASS_L0,      // one colour pass of the smoother on level 0
  MG_RESTRICT_L0,  // restriction from level 0
  MG_PROLONG_L0,   // prolongation onto level 0
  MG_PASS_MID,     // a colour pass on a level between 0 and the coarsest
  MG_RESTRICT_MID,
  MG_PROLONG_MID,
  MG_COARSE,       // the coarsest-level solve
  MG_CG_VECTOR,    // a CG vector kernel (dot products, updates, q = A p)
  MG_CLASSES
};

// Per-launch timer of the V-cycle: start() records an event, then mark()
// after each launch records the next one and credits the interval to its
// class.  Read after the stream has finished.
struct MgTimer {
  std::vector<cudaEvent_t> ev;
  std::vector<int> cls;
  ~MgTimer();
  cudaError_t start(cudaStream_t st);
  cudaError_t mark(int c, cudaStream_t st);
  // per-class totals (ms) and launch counts
  cudaError_t read(float* ms, int* launches) const;
};

// The direct solve of the coarsest level of the CG preconditioner
// (solver.cu): phi = A^-1 b with b and phi in the level's storage (FP32 or
// BF16).
struct CoarseDirect {
  virtual ~CoarseDirect() = default;
  virtual cudaError_t apply(cudaStream_t st, const void* b, void* phi, bool bf16) = 0;
};

// Multigrid hierarchy.  Reference rule (src/sim.rs:142-168): <= 4 levels,
// stop after the first level whose smallest dimension is < 16, halve with
// ceil, h doubles.  Deep rule (the CG preconditioner): halve until the
// coarsest level has at most `direct_max` cells, which are then solved
// directly.  Level 0 arrays are bound from outside; the coarse levels are
// owned.
struct Multigrid {
  MgTimer* timer = nullptr;  // set only while pyro_sim_profile_pressure runs
  CoarseDirect* direct = nullptr;  // coarsest solve of vcycle_sym, when set
  int bc_mode = 0;
  std::vector<Dims3> dims;
  std::vector<float> h;
  std::vector<float*> phi, b;
  std::vector<const uint32_t*> f;
  std::vector<DevBuf> own_phi, own_b, own_f;
  std::vector<DevBuf> phi2;   // ping-pong partner of phi on every level
  std::vector<DevBuf> meta;   // per-cell neighbour mask (k_mgf.cu)
  std::vector<DevBuf> wq;     // 64 x prolongation weight sums (vcycle_sym, levels < last)
  bool coarse_one_cta = false;
  float* stats = nullptr;  // device, for mg_resid

  // direct_max == 0: the reference rule; else the deep rule.
  int init(Dims3 d0, float h0, int bc, size_t direct_max = 0);
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
  // prepare() and the weight sums of the symmetric V-cycle's restriction.
  cudaError_t prepare_sym(cudaStream_t st);
  // `cycles` V-cycles (src/sim.rs:451-491) on the bound level-0 arrays with
  // the fused kernels (k_mgf.cu); calls prepare() first.
  cudaError_t vcycles(int cycles, cudaStream_t st);
  // Symmetric V-cycle for the CG preconditioner: pre-smoothing red-black,
  // post-smoothing black-red, restriction P^T/8 of the fluid-normalised
  // trilinear prolongation, coarsest level by the direct solve when set,
  // else alternating SOR sweeps.  With bphi != nullptr phi and b are stored
  // in BF16 (FP32 arithmetic).  The initial guess is zero: level 0's phi is
  // not read, the result overwrites all of it (FP32), and level 0's b is the
  // FP32 right-hand side in both storages.
  // prep = false skips the per-level masks and weights (valid while the
  // level flags are unchanged since the last prepare_sym()).
  cudaError_t vcycle_sym(cudaStream_t st, DevBuf* bphi, DevBuf* bphi2, DevBuf* bb,
                         bool prep = true);
  size_t device_bytes() const;
};

// Level dims of the reference rule (shared with the C ABI).
std::vector<Dims3> mg_level_dims(Dims3 d0, int max_levels);
// Level dims of the deep rule: halve (ceil) until the level has at most
// direct_max cells or a dimension would drop below 2.
std::vector<Dims3> mg_level_dims_deep(Dims3 d0, size_t direct_max);

}  // namespace pyro
