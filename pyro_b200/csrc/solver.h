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

// State of the device-driven CG loop: written by the host before the loop's
// graph is launched, updated by its check kernel after every iteration.
struct CgCtl {
  float* x;     // the solution array
  double bb2;   // |b|^2
  double tol;   // relative residual target
  double rr;    // |r|^2 after the last iteration
  int it;       // iterations done (across restarts)
  int max_it;   // iteration cap
  int first;    // 1: the next search direction is p = z
  int stalled;  // 1: |r|^2 not finite or <p, A p> = 0
};

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
  bool pc_ready = false;  // the hierarchy's flags and the coarsest inverse follow fa
  // The CG iterations as one CUDA graph: a conditional while node whose body
  // is one preconditioned iteration ending in k_cg_check, which decides on
  // the device whether another iteration follows.  One per preconditioner
  // storage (FP32, BF16), built on first use; the solution array is read
  // from the control block.
  cudaGraphExec_t cg_exec[2] = {nullptr, nullptr};
  cudaStream_t cap_st = nullptr;  // the stream the loop body is captured on
  DevBuf ctl;                     // CgCtl on the device
  CgCtl* host_ctl = nullptr;      // pinned mirror

  int init(Multigrid* m);
  ~Solver();
  size_t device_bytes() const;
  // Solve A phi = b in place (phi = initial guess).  Returns PYRO_OK or
  // PYRO_E_NOCONV (info filled either way) or an error.
  int solve(cudaStream_t st, float* phi, const float* b, int mode, float tol, int max_iters,
            PyroSolveInfo* info);
  // `iters` CG iterations of mode PYRO_SOLVER_MGPCG or _BF16 from phi, one
  // launch at a time with an event after each (no graph, no convergence
  // test), credited to the launch classes of MgTimer; ms / launches per
  // class out.  phi is updated like a solve's iterations update it.
  int profile_cg(cudaStream_t st, float* phi, const float* b, bool bf16, int iters, float* ms,
                 int* launches);

 private:
  cudaError_t precond(cudaStream_t st, bool bf16, bool prep);
  // |b - A phi| / |b| and |b|; cg: on the CG modes' reachable set (their
  // level-0 masks), else on the solid flags of level 0
  int true_resid(cudaStream_t st, const float* phi, const float* b, double* rel, double* bn,
                 bool cg);
  // phi += alpha net(r) when that lowers |r| (r = b - A phi on entry, kept
  // consistent); *rr is |r|^2 in and out.
  int learned_stage(cudaStream_t st, float* phi, double* rr, PyroSolveInfo* info);
  // The reachable-fluid flags fa, the preconditioner's levels and its
  // coarsest inverse for the current flag field, and r = b - A phi with
  // |r|^2, |b|^2 in host_sc (one host synchronisation when the flags did not
  // change).
  int begin_cg(cudaStream_t st, float* phi, const float* b);
  // fa from the current flag field, whose hash is h
  int update_reach(cudaStream_t st, unsigned long long h);
  // BF16 storage of every preconditioner level (allocated once)
  int alloc_bf16_levels();
  // Enqueue CG iterations from r (p = z first) until the recursive residual
  // meets tol, the count reaches max_it or the iteration stalls.
  int cg_loop(cudaStream_t st, float* phi, bool bf16, double bb2, float tol, int it0,
              int max_it);
};

}  // namespace pyro
