// solver.h — pressure solvers on a multigrid hierarchy: fixed V-cycles,
// V-cycles to a tolerance, and flexible preconditioned CG (MGPCG) with an
// FP32 or BF16-storage V-cycle preconditioner.  Dot products and residual
// norms are accumulated in FP64.
#pragma once

#include "runtime.h"

namespace pyro {

struct DirectSolve;

// Cells of the preconditioner's coarsest level, which is solved directly in
// FP64 (a dense inverse of DIRECT_MAX^2 doubles at most: 75 MB).
constexpr size_t DIRECT_MAX = 3072;

struct Solver {
  Multigrid* mg = nullptr;  // the reference hierarchy (fixed V-cycle modes)
  Multigrid pc;             // the preconditioner's deep hierarchy (CG modes)
  DirectSolve* direct = nullptr;  // its coarsest-level solve (owned)
  Dims3 d{};
  DevBuf r, z, p, q;        // level-0 work vectors (FP32)
  DevBuf sc;                // FP64 device scalars
  double* host_sc = nullptr;  // pinned mirror
  // BF16 hierarchy for the low-precision preconditioner
  std::vector<DevBuf> bphi, bphi2, bb;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr, evl0 = nullptr, evl1 = nullptr;
  PyroNet* net = nullptr;   // learned stage of PYRO_SOLVER_MGPCG_LEARNED (not owned)
  // flags of the CG modes: fluid cells without a fluid path to a Dirichlet
  // face are marked solid (recomputed when the flag field changes)
  DevBuf fa, reach_dev;
  unsigned long long reach_hash = 0;
  const uint32_t* reach_flags = nullptr;
  bool reach_valid = false;

  int init(Multigrid* m);
  ~Solver();
  size_t device_bytes() const;
  // Solve A phi = b in place (phi = initial guess).  Returns PYRO_OK or
  // PYRO_E_NOCONV (info filled either way) or an error.
  int solve(cudaStream_t st, float* phi, const float* b, int mode, float tol, int max_iters,
            PyroSolveInfo* info);

 private:
  cudaError_t precond(cudaStream_t st, bool bf16, bool prep);
  int true_resid(cudaStream_t st, const float* phi, const float* b, double* rel, double* bn);
  // phi += alpha net(r) when that lowers |r| (r = b - A phi on entry, kept
  // consistent); *rr is |r|^2 in and out.
  int learned_stage(cudaStream_t st, float* phi, double* rr, PyroSolveInfo* info);
  int update_reach(cudaStream_t st);
};

}  // namespace pyro
