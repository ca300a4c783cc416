// runtime.cu — error state, device buffers, multigrid schedule.
#include <cstring>

#include "runtime.h"

namespace pyro {

namespace {
thread_local std::string g_last_error;
}

void set_error(const std::string& msg) { g_last_error = msg; }
void clear_error() { g_last_error.clear(); }
const std::string& last_error_text() { return g_last_error; }

int DevBuf::alloc(size_t n) {
  release();
  if (n == 0) return PYRO_OK;
  cudaError_t e = cudaMalloc(&p, n);
  if (e != cudaSuccess) {
    p = nullptr;
    set_error(std::string("cudaMalloc(") + std::to_string(n) + "): " + cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? PYRO_E_NOMEM : PYRO_E_CUDA;
  }
  bytes = n;
  // The zero fill runs on the default stream, which the library's own
  // (non-blocking) streams do not wait for: it must be finished before any
  // of them touches the buffer.
  e = cudaMemset(p, 0, n);
  if (e == cudaSuccess) e = cudaStreamSynchronize(0);
  if (e != cudaSuccess) {
    set_error(std::string("cudaMemset: ") + cudaGetErrorString(e));
    return PYRO_E_CUDA;
  }
  return PYRO_OK;
}

void DevBuf::release() {
  if (p) cudaFree(p);
  p = nullptr;
  bytes = 0;
}

MgTimer::~MgTimer() {
  for (auto e : ev) cudaEventDestroy(e);
}

cudaError_t MgTimer::start(cudaStream_t st) {
  for (auto e : ev) cudaEventDestroy(e);
  ev.clear();
  cls.clear();
  return mark(-1, st);
}

cudaError_t MgTimer::mark(int c, cudaStream_t st) {
  cudaEvent_t e;
  cudaError_t r = cudaEventCreate(&e);
  if (r != cudaSuccess) return r;
  ev.push_back(e);
  cls.push_back(c);
  return cudaEventRecord(e, st);
}

cudaError_t MgTimer::read(float* ms, int* launches) const {
  for (int c = 0; c < MG_CLASSES; c++) {
    ms[c] = 0.0f;
    launches[c] = 0;
  }
  for (size_t i = 1; i < ev.size(); i++) {
    float t = 0.0f;
    cudaError_t r = cudaEventElapsedTime(&t, ev[i - 1], ev[i]);
    if (r != cudaSuccess) return r;
    if (cls[i] >= 0 && cls[i] < MG_CLASSES) {
      ms[cls[i]] += t;
      launches[cls[i]] += 1;
    }
  }
  return cudaSuccess;
}

std::vector<Dims3> mg_level_dims(Dims3 d, int max_levels) {
  std::vector<Dims3> v;
  for (int l = 0; l < max_levels; l++) {
    v.push_back(d);
    if (std::min(std::min(d.nx, d.ny), d.nz) < 16) break;
    d = Dims3{(d.nx + 1) / 2, (d.ny + 1) / 2, (d.nz + 1) / 2};
  }
  return v;
}

std::vector<Dims3> mg_level_dims_deep(Dims3 d, size_t direct_max) {
  std::vector<Dims3> v{d};
  while (d.cells() > direct_max && std::min(std::min(d.nx, d.ny), d.nz) >= 4) {
    d = Dims3{(d.nx + 1) / 2, (d.ny + 1) / 2, (d.nz + 1) / 2};
    v.push_back(d);
  }
  return v;
}

int Multigrid::init(Dims3 d0, float h0, int bc, size_t direct_max) {
  bc_mode = bc;
  dims = direct_max ? mg_level_dims_deep(d0, direct_max) : mg_level_dims(d0, 4);
  size_t L = dims.size();
  h.resize(L);
  phi.assign(L, nullptr);
  b.assign(L, nullptr);
  f.assign(L, nullptr);
  own_phi.resize(L);
  own_b.resize(L);
  own_f.resize(L);
  phi2.resize(L);
  meta.resize(L);
  float hh = h0;
  for (size_t l = 0; l < L; l++) {
    h[l] = hh;
    hh *= 2.0f;
    size_t n = dims[l].cells();
    int rc;
    if ((rc = phi2[l].alloc(n * 4)) != PYRO_OK) return rc;
    if ((rc = meta[l].alloc(n)) != PYRO_OK) return rc;
    if (l == 0) continue;
    if ((rc = own_phi[l].alloc(n * 4)) != PYRO_OK) return rc;
    if ((rc = own_b[l].alloc(n * 4)) != PYRO_OK) return rc;
    if ((rc = own_f[l].alloc(n * 4)) != PYRO_OK) return rc;
    phi[l] = own_phi[l].as<float>();
    b[l] = own_b[l].as<float>();
    f[l] = own_f[l].as<uint32_t>();
  }
  coarse_one_cta = mg_coarse_fits(dims.back());
  return PYRO_OK;
}

size_t Multigrid::device_bytes() const {
  size_t s = 0;
  for (size_t l = 1; l < dims.size(); l++) s += own_phi[l].bytes + own_b[l].bytes + own_f[l].bytes;
  for (size_t l = 0; l < dims.size(); l++) s += phi2[l].bytes + meta[l].bytes;
  for (const DevBuf& w : wq) s += w.bytes;
  return s;
}

cudaError_t Multigrid::smooth(int l, int iters, bool coarse, cudaStream_t st) {
  float om = coarse ? 1.6f : 1.0f;
  if (coarse && coarse_one_cta)
    return launch_mg_coarse(dims[l], h[l], b[l], f[l], phi[l], iters, om, bc_mode, st);
  for (int it = 0; it < iters; it++)
    for (int c = 0; c < 2; c++) {
      cudaError_t e = launch_mg_pass(dims[l], h[l], b[l], meta[l].as<uint8_t>(), phi[l], c, om,
                                     bc_mode, st);
      if (e != cudaSuccess) return e;
    }
  return cudaSuccess;
}

cudaError_t Multigrid::prepare(cudaStream_t st) {
  int nl = (int)dims.size();
  cudaError_t e;
  for (int l = 1; l < nl; l++)
    if ((e = launch_mg_flags_down(dims[l - 1], f[l - 1], dims[l], const_cast<uint32_t*>(f[l]),
                                  st)) != cudaSuccess)
      return e;
  for (int l = 0; l < nl; l++)
    if ((e = launch_mg_meta(dims[l], f[l], meta[l].as<uint8_t>(), st)) != cudaSuccess) return e;
  return cudaSuccess;
}

cudaError_t Multigrid::prepare_sym(cudaStream_t st) {
  cudaError_t e = prepare(st);
  const int nl = (int)dims.size();
  if (wq.size() != dims.size()) wq.resize(dims.size());
  for (int l = 0; e == cudaSuccess && l + 1 < nl; l++) {
    if (!wq[l].p && wq[l].alloc(dims[l].cells()) != PYRO_OK) return cudaErrorMemoryAllocation;
    e = launch_mg_wsum(dims[l], meta[l].as<uint8_t>(), dims[l + 1], meta[l + 1].as<uint8_t>(),
                       wq[l].as<uint8_t>(), st);
  }
  return e;
}

cudaError_t Multigrid::vcycles(int cycles, cudaStream_t st) {
  int nl = (int)dims.size();
  cudaError_t e;
  // with a timer, an event after every launch credits it to its class
  auto tick = [&](int cls) -> cudaError_t { return timer ? timer->mark(cls, st) : cudaSuccess; };
  if (timer && (e = timer->start(st)) != cudaSuccess) return e;
  if ((e = prepare(st)) != cudaSuccess) return e;
  if ((e = tick(MG_PREPARE)) != cudaSuccess) return e;
  auto M = [&](int l) { return meta[l].as<uint8_t>(); };
  auto sm = [&](int l) -> cudaError_t {  // two red-black iterations, omega 1
    for (int it = 0; it < 2; it++)
      for (int c = 0; c < 2; c++) {
        cudaError_t e2 = launch_mg_pass(dims[l], h[l], b[l], M(l), phi[l], c, 1.0f, bc_mode, st);
        if (e2 == cudaSuccess) e2 = tick(l == 0 ? MG_PASS_L0 : MG_PASS_MID);
        if (e2 != cudaSuccess) return e2;
      }
    return cudaSuccess;
  };
  for (int cy = 0; cy < cycles; cy++) {
    for (int l = 0; l < nl - 1; l++) {
      if ((e = sm(l)) != cudaSuccess) return e;
      if ((e = launch_mg_restrict_m(dims[l], h[l], phi[l], b[l], M(l), dims[l + 1], b[l + 1],
                                    phi[l + 1], bc_mode, st)) != cudaSuccess)
        return e;
      if ((e = tick(l == 0 ? MG_RESTRICT_L0 : MG_RESTRICT_MID)) != cudaSuccess) return e;
    }
    if ((e = smooth(nl - 1, 80, true, st)) != cudaSuccess) return e;
    if ((e = tick(MG_COARSE)) != cudaSuccess) return e;
    for (int l = nl - 2; l >= 0; l--) {
      if ((e = launch_mg_prolong_m(dims[l], phi[l + 1], M(l), phi[l], dims[l + 1], M(l + 1), st)) !=
          cudaSuccess)
        return e;
      if ((e = tick(l == 0 ? MG_PROLONG_L0 : MG_PROLONG_MID)) != cudaSuccess) return e;
      if ((e = sm(l)) != cudaSuccess) return e;
    }
  }
  return cudaSuccess;
}

// Red-black sweeps before and after the coarse correction on level l of the
// symmetric V-cycle: 2 on level 0, 4 on the coarser levels, whose passes
// cost a fraction of level 0's.  Measured on the 2 cm pool's system and the
// 256^3 case against 1..4 sweeps on level 0 and 1..8 below: fewer CG
// iterations pay for the extra coarse passes (BF16 MGPCG to 1e-4 on the
// pool: 8 iterations, 4.6 ms with 2 / 2; 6 iterations, 3.9 ms with 2 / 4).
static int sym_sweeps(int l) { return l == 0 ? 2 : 4; }
// Relaxation factor of the symmetric V-cycle's red-black sweeps: over-
// relaxed (SOR) smoothing, the same factor before and after the coarse
// correction so the cycle stays symmetric.  Measured on the 2 cm pool's
// system, the 256^3 case with both boundary modes and the 150x365x150 step
// against 1.0, 1.1, 1.15, 1.2, 1.4, 1.5 and 1.6: 1.3 and 1.4 the fastest
// (BF16 MGPCG to 1e-4 on the pool: 6 iterations, 3.96 ms with 1.0; 5, 3.35
// ms with 1.3), 1.6 back to the 1.0 counts.
constexpr float kSymOmega = 1.3f;

cudaError_t Multigrid::vcycle_sym(cudaStream_t st, DevBuf* bphi, DevBuf* bphi2, DevBuf* bb,
                                   bool prep) {
  int nl = (int)dims.size();
  const bool lo = bphi != nullptr;
  cudaError_t e;
  if (lo) {
    for (int l = 0; l < nl; l++) {
      size_t need = dims[l].cells() * 2;
      if (bphi[l].bytes != need) {
        if (bphi[l].alloc(need) != PYRO_OK || bphi2[l].alloc(need) != PYRO_OK ||
            bb[l].alloc(need) != PYRO_OK)
          return cudaErrorMemoryAllocation;
      }
    }
  }
  // with a timer, an event after every step credits it to its class
  auto tick = [&](int cls) -> cudaError_t { return timer ? timer->mark(cls, st) : cudaSuccess; };
  if (prep && (e = prepare_sym(st)) != cudaSuccess) return e;
  if (prep && (e = tick(MG_PREPARE)) != cudaSuccess) return e;
  auto M = [&](int l) { return meta[l].as<uint8_t>(); };
  // storage of level l: phi, b, scratch
  auto P = [&](int l) -> void* { return lo ? bphi[l].p : (void*)phi[l]; };
  auto B = [&](int l) -> void* { return lo ? bb[l].p : (void*)b[l]; };
  auto T = [&](int l) -> void* { return lo ? bphi2[l].p : phi2[l].p; };
  size_t n0 = dims[0].cells();
  // The first and last level-0 passes take the zero guess, the FP32
  // right-hand side and (BF16) the FP32 result directly; a hierarchy of one
  // level (solved directly) clears and converts level 0 here and converts
  // back at the end.
  const bool fuse = nl > 1;
  if (!fuse) {
    if (lo) {
      if ((e = launch_f32_to_bf16(b[0], bb[0].p, n0, st)) != cudaSuccess) return e;
      if ((e = cudaMemsetAsync(bphi[0].p, 0, n0 * 2, st)) != cudaSuccess) return e;
    } else if ((e = cudaMemsetAsync(phi[0], 0, n0 * 4, st)) != cudaSuccess) {
      return e;
    }
  }
  auto pass = [&](int l, int c, float om) -> cudaError_t {
    return lo ? launch_mg_pass_bf16(dims[l], h[l], B(l), M(l), P(l), c, om, bc_mode, st)
              : launch_mg_pass(dims[l], h[l], (const float*)B(l), M(l), (float*)P(l), c, om,
                               bc_mode, st);
  };
  for (int l = 0; l < nl - 1; l++) {
    for (int it = 0; it < sym_sweeps(l); it++)
      for (int c = 0; c < 2; c++) {
        e = (fuse && l == 0 && it == 0 && c == 0)
                ? launch_mg_pass_first(dims[0], h[0], b[0], lo ? bb[0].p : nullptr, M(0), P(0), 0,
                                       kSymOmega, bc_mode, lo, st)
                : pass(l, c, kSymOmega);
        if (e == cudaSuccess) e = tick(l == 0 ? MG_PASS_L0 : MG_PASS_MID);
        if (e != cudaSuccess) return e;
      }
    const uint8_t* W = wq[l].as<uint8_t>();
    e = lo ? launch_mg_restrict_sym_bf16(dims[l], h[l], P(l), B(l), M(l), W, T(l), dims[l + 1],
                                         M(l + 1), B(l + 1), P(l + 1), bc_mode, st)
           : launch_mg_restrict_sym(dims[l], h[l], (const float*)P(l), (const float*)B(l), M(l),
                                    W, (float*)T(l), dims[l + 1], M(l + 1), (float*)B(l + 1),
                                    (float*)P(l + 1), bc_mode, st);
    if (e == cudaSuccess) e = tick(l == 0 ? MG_RESTRICT_L0 : MG_RESTRICT_MID);
    if (e != cudaSuccess) return e;
  }
  int lc = nl - 1;
  if (direct) {
    if ((e = direct->apply(st, B(lc), P(lc), lo)) != cudaSuccess) return e;
  } else if (coarse_one_cta) {
    e = lo ? launch_mg_coarse_sym_bf16(dims[lc], h[lc], B(lc), f[lc], P(lc), 80, 1.6f, bc_mode, st)
           : launch_mg_coarse_sym(dims[lc], h[lc], (const float*)B(lc), f[lc], (float*)P(lc), 80,
                                  1.6f, bc_mode, st);
    if (e != cudaSuccess) return e;
  } else {
    for (int it = 0; it < 80; it++)
      for (int cc = 0; cc < 2; cc++)
        if ((e = pass(lc, cc ^ (it & 1), 1.6f)) != cudaSuccess) return e;
  }
  if ((e = tick(MG_COARSE)) != cudaSuccess) return e;
  for (int l = nl - 2; l >= 0; l--) {
    e = lo ? launch_mg_prolong_m_bf16(dims[l], P(l + 1), M(l), P(l), dims[l + 1], M(l + 1), st)
           : launch_mg_prolong_m(dims[l], (const float*)P(l + 1), M(l), (float*)P(l),
                                 dims[l + 1], M(l + 1), st);
    if (e == cudaSuccess) e = tick(l == 0 ? MG_PROLONG_L0 : MG_PROLONG_MID);
    if (e != cudaSuccess) return e;
    for (int it = 0; it < sym_sweeps(l); it++)
      for (int c = 1; c >= 0; c--) {
        e = (fuse && lo && l == 0 && it == sym_sweeps(0) - 1 && c == 0)
                ? launch_mg_pass_last_f32(dims[0], h[0], B(0), M(0), P(0), phi[0], 0, kSymOmega,
                                          bc_mode, st)
                : pass(l, c, kSymOmega);
        if (e == cudaSuccess) e = tick(l == 0 ? MG_PASS_L0 : MG_PASS_MID);
        if (e != cudaSuccess) return e;
      }
  }
  if (lo && !fuse) return launch_bf16_to_f32(bphi[0].p, phi[0], n0, st);
  return cudaSuccess;
}

}  // namespace pyro
