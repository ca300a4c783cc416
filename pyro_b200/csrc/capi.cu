// capi.cu — C entry points for single kernels, the voxelizer and the error
// text (include/pyro_sim.h).  The simulation object lives in sim.cu, the
// Poisson solver in solver.cu.
#include <cstring>
#include <string>

#include "runtime.h"

using namespace pyro;

namespace {

thread_local std::string g_err_copy;

inline cudaStream_t S(void* s) { return reinterpret_cast<cudaStream_t>(s); }

int ret(cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    set_error(std::string(what) + ": " + cudaGetErrorString(e));
    return PYRO_E_CUDA;
  }
  return PYRO_OK;
}

bool dims_ok(uint32_t nx, uint32_t ny, uint32_t nz) {
  return nx >= 2 && ny >= 2 && nz >= 2 &&
         (uint64_t)(nx + 1) * (ny + 1) * (nz + 1) < (1ull << 31);
}

// light caches, ground cache and images: at least one texel, < 2^31 texels
bool cache_dims_ok(uint32_t lx, uint32_t ly, uint32_t lz) {
  return lx >= 1 && ly >= 1 && lz >= 1 && (uint64_t)lx * ly * lz < (1ull << 31);
}

}  // namespace

namespace pyro {
// defined in runtime.cu
const std::string& last_error_text();
}

extern "C" {

const char* pyro_last_error(void) {
  g_err_copy = pyro::last_error_text();
  return g_err_copy.c_str();
}

#define KDIMS(name)                                                  \
  clear_error();                                                     \
  PYRO_REQUIRE(params_dev, #name ": null parameter block");          \
  PYRO_REQUIRE(dims_ok(nx, ny, nz), #name ": invalid grid dimensions"); \
  Dims3 d{(int)nx, (int)ny, (int)nz};

int pyro_k_solid(const PyroParams* params_dev, uint32_t nx, uint32_t ny, uint32_t nz,
                 const float* sol_in, float* sol_out, float* pyr, uint32_t* flags,
                 const float* s0, float* stats, void* stream) {
  KDIMS(pyro_k_solid)
  PYRO_REQUIRE(sol_in && sol_out && pyr && flags && s0, "pyro_k_solid: null buffer");
  return ret(launch_solid(params_dev, d, (const float4*)sol_in, (float4*)sol_out, (float4*)pyr,
                          flags, (const float4*)s0, stats, S(stream)),
             "pyro_k_solid");
}

int pyro_k_curl(const PyroParams* params_dev, uint32_t nx, uint32_t ny, uint32_t nz,
                const float* u, const float* v, const float* w, float* curl, float* stats,
                void* stream) {
  KDIMS(pyro_k_curl)
  PYRO_REQUIRE(u && v && w && curl, "pyro_k_curl: null buffer");
  return ret(launch_curl(params_dev, d, u, v, w, (float4*)curl, stats, S(stream)), "pyro_k_curl");
}

int pyro_k_adv_vel(const PyroParams* params_dev, uint32_t nx, uint32_t ny, uint32_t nz,
                   const float* u, const float* v, const float* w, float* hu, float* hv,
                   float* hw, float* ou, float* ov, float* ow, const uint32_t* flags,
                   void* stream) {
  KDIMS(pyro_k_adv_vel)
  PYRO_REQUIRE(u && v && w && hu && hv && hw && ou && ov && ow && flags,
               "pyro_k_adv_vel: null buffer");
  // the predictor's min / max at the backtrace, handed to the corrector
  DevBuf lohi;
  int rc = lohi.alloc((size_t)(nx + 1) * (ny + 1) * (nz + 1) * 6 * 4);
  if (rc != PYRO_OK) return rc;
  cudaError_t e = launch_adv_vel1(params_dev, d, u, v, w, hu, hv, hw, lohi.as<float>(), S(stream));
  if (e == cudaSuccess)
    e = launch_adv_vel2(params_dev, d, u, v, w, hu, hv, hw, lohi.as<float>(), ou, ov, ow, flags,
                        S(stream));
  if (e == cudaSuccess) e = cudaStreamSynchronize(S(stream));  // before lohi is freed
  return ret(e, "pyro_k_adv_vel");
}

int pyro_k_adv_scalars(const PyroParams* params_dev, uint32_t nx, uint32_t ny, uint32_t nz,
                       const float* u, const float* v, const float* w, const float* s0,
                       const float* s1, float* h0, float* h1, float* o0, float* o1,
                       void* stream) {
  KDIMS(pyro_k_adv_scalars)
  PYRO_REQUIRE(u && v && w && s0 && s1 && h0 && h1 && o0 && o1,
               "pyro_k_adv_scalars: null buffer");
  // the predictor's backtrace, handed to the corrector
  DevBuf bt;
  int rc = bt.alloc((size_t)nx * ny * nz * 3 * 4);
  if (rc != PYRO_OK) return rc;
  cudaError_t e = launch_adv_s1(params_dev, d, u, v, w, (const float4*)s0, (const float4*)s1,
                                (float4*)h0, (float4*)h1, bt.as<float>(), S(stream));
  if (e == cudaSuccess)
    e = launch_adv_s2(params_dev, d, u, v, w, (const float4*)s0, (const float4*)s1,
                      (const float4*)h0, (const float4*)h1, bt.as<float>(), (float4*)o0,
                      (float4*)o1, S(stream));
  if (e == cudaSuccess) e = cudaStreamSynchronize(S(stream));  // before bt is freed
  return ret(e, "pyro_k_adv_scalars");
}

int pyro_k_react(const PyroParams* params_dev, uint32_t nx, uint32_t ny, uint32_t nz,
                 const float* s0in, const float* s1in, float* s0out, float* s1out,
                 const uint32_t* flags, const float* sol, const float* pyr, const float* curl,
                 float* stats, void* stream) {
  KDIMS(pyro_k_react)
  PYRO_REQUIRE(s0in && s1in && s0out && s1out && flags && sol && pyr && curl,
               "pyro_k_react: null buffer");
  return ret(launch_react(params_dev, d, (const float4*)s0in, (const float4*)s1in,
                          (float4*)s0out, (float4*)s1out, flags, (const float4*)sol,
                          (const float4*)pyr, (const float4*)curl, stats, S(stream)),
             "pyro_k_react");
}

int pyro_k_forces(const PyroParams* params_dev, uint32_t nx, uint32_t ny, uint32_t nz, float* u,
                  float* v, float* w, const float* s0, const float* s1, const float* curl,
                  const uint32_t* flags, void* stream) {
  KDIMS(pyro_k_forces)
  PYRO_REQUIRE(u && v && w && s0 && s1 && curl && flags, "pyro_k_forces: null buffer");
  DevBuf conf;
  int rc = conf.alloc(d.cells() * 16);
  if (rc != PYRO_OK) return rc;
  rc = ret(launch_forces(params_dev, d, u, v, w, (const float4*)s0, (const float4*)s1,
                         (const float4*)curl, conf.as<float4>(), flags, S(stream)),
           "pyro_k_forces");
  if (rc == PYRO_OK) PYRO_CU(cudaStreamSynchronize(S(stream)));
  return rc;
}

int pyro_k_divergence(const PyroParams* params_dev, uint32_t nx, uint32_t ny, uint32_t nz,
                      const float* u, const float* v, const float* w, const float* s1,
                      const uint32_t* flags, float* b, void* stream) {
  KDIMS(pyro_k_divergence)
  PYRO_REQUIRE(u && v && w && s1 && flags && b, "pyro_k_divergence: null buffer");
  return ret(launch_divergence(params_dev, d, u, v, w, (const float4*)s1, flags, b, S(stream)),
             "pyro_k_divergence");
}

int pyro_k_project(const PyroParams* params_dev, uint32_t nx, uint32_t ny, uint32_t nz,
                   float* u, float* v, float* w, const float* phi, const uint32_t* flags,
                   void* stream) {
  KDIMS(pyro_k_project)
  PYRO_REQUIRE(u && v && w && phi && flags, "pyro_k_project: null buffer");
  return ret(launch_project(params_dev, d, u, v, w, phi, flags, S(stream)), "pyro_k_project");
}

// The reference's per-flag multigrid dispatches (mg.wgsl) run here on the
// kernels the V-cycle itself launches: the level's neighbour masks are built
// into a temporary buffer (k_mg_meta), then the mask-driven pass,
// restriction or prolongation runs.  Each call waits for its stream before
// the temporaries are freed.
int pyro_k_mg_smooth(uint32_t nx, uint32_t ny, uint32_t nz, float h, const float* b,
                     const uint32_t* flags, float* phi, int color, float omega, void* stream) {
  clear_error();
  PYRO_REQUIRE(dims_ok(nx, ny, nz), "pyro_k_mg_smooth: invalid grid dimensions");
  PYRO_REQUIRE(b && flags && phi, "pyro_k_mg_smooth: null buffer");
  PYRO_REQUIRE(color == 0 || color == 1, "pyro_k_mg_smooth: color must be 0 or 1");
  Dims3 d{(int)nx, (int)ny, (int)nz};
  DevBuf meta;
  int rc = meta.alloc(d.cells());
  if (rc != PYRO_OK) return rc;
  cudaError_t e = launch_mg_meta(d, flags, meta.as<uint8_t>(), S(stream));
  if (e == cudaSuccess)
    e = launch_mg_pass(d, h, b, meta.as<uint8_t>(), phi, color, omega, 0, S(stream));
  if (e == cudaSuccess) e = cudaStreamSynchronize(S(stream));
  return ret(e, "pyro_k_mg_smooth");
}

int pyro_k_mg_restrict(uint32_t fnx, uint32_t fny, uint32_t fnz, float fh, const float* pf,
                       const float* bf, const uint32_t* ff, uint32_t cnx, uint32_t cny,
                       uint32_t cnz, float* bc, float* pc, uint32_t* fc, void* stream) {
  clear_error();
  PYRO_REQUIRE(dims_ok(fnx, fny, fnz) && cnx >= 1 && cny >= 1 && cnz >= 1,
               "pyro_k_mg_restrict: invalid grid dimensions");
  PYRO_REQUIRE(cnx == (fnx + 1) / 2 && cny == (fny + 1) / 2 && cnz == (fnz + 1) / 2,
               "pyro_k_mg_restrict: coarse dims must be ceil(fine / 2)");
  PYRO_REQUIRE(pf && bf && ff && bc && pc && fc, "pyro_k_mg_restrict: null buffer");
  Dims3 df{(int)fnx, (int)fny, (int)fnz}, dc{(int)cnx, (int)cny, (int)cnz};
  DevBuf meta;
  int rc = meta.alloc(df.cells());
  if (rc != PYRO_OK) return rc;
  cudaError_t e = launch_mg_meta(df, ff, meta.as<uint8_t>(), S(stream));
  if (e == cudaSuccess) e = launch_mg_flags_down(df, ff, dc, fc, S(stream));
  if (e == cudaSuccess)
    e = launch_mg_restrict_m(df, fh, pf, bf, meta.as<uint8_t>(), dc, bc, pc, 0, S(stream));
  if (e == cudaSuccess) e = cudaStreamSynchronize(S(stream));
  return ret(e, "pyro_k_mg_restrict");
}

int pyro_k_mg_prolong(uint32_t fnx, uint32_t fny, uint32_t fnz, const float* pc,
                      const uint32_t* ff, float* pf, uint32_t cnx, uint32_t cny, uint32_t cnz,
                      const uint32_t* fc, void* stream) {
  clear_error();
  PYRO_REQUIRE(dims_ok(fnx, fny, fnz), "pyro_k_mg_prolong: invalid grid dimensions");
  PYRO_REQUIRE(cnx == (fnx + 1) / 2 && cny == (fny + 1) / 2 && cnz == (fnz + 1) / 2,
               "pyro_k_mg_prolong: coarse dims must be ceil(fine / 2)");
  PYRO_REQUIRE(pc && ff && pf && fc, "pyro_k_mg_prolong: null buffer");
  Dims3 df{(int)fnx, (int)fny, (int)fnz}, dc{(int)cnx, (int)cny, (int)cnz};
  DevBuf mf, mc;
  int rc = mf.alloc(df.cells());
  if (rc == PYRO_OK) rc = mc.alloc(dc.cells());
  if (rc != PYRO_OK) return rc;
  cudaError_t e = launch_mg_meta(df, ff, mf.as<uint8_t>(), S(stream));
  if (e == cudaSuccess) e = launch_mg_meta(dc, fc, mc.as<uint8_t>(), S(stream));
  if (e == cudaSuccess)
    e = launch_mg_prolong_m(df, pc, mf.as<uint8_t>(), pf, dc, mc.as<uint8_t>(), S(stream));
  if (e == cudaSuccess) e = cudaStreamSynchronize(S(stream));
  return ret(e, "pyro_k_mg_prolong");
}

int pyro_k_mg_meta(uint32_t nx, uint32_t ny, uint32_t nz, const uint32_t* flags, uint8_t* meta,
                   void* stream) {
  clear_error();
  PYRO_REQUIRE(dims_ok(nx, ny, nz), "pyro_k_mg_meta: invalid grid dimensions");
  PYRO_REQUIRE(flags && meta, "pyro_k_mg_meta: null buffer");
  return ret(launch_mg_meta(Dims3{(int)nx, (int)ny, (int)nz}, flags, meta, S(stream)),
             "pyro_k_mg_meta");
}

int pyro_k_mg_flags_down(uint32_t fnx, uint32_t fny, uint32_t fnz, const uint32_t* ff,
                         uint32_t cnx, uint32_t cny, uint32_t cnz, uint32_t* fc, void* stream) {
  clear_error();
  PYRO_REQUIRE(dims_ok(fnx, fny, fnz), "pyro_k_mg_flags_down: invalid grid dimensions");
  PYRO_REQUIRE(cnx == (fnx + 1) / 2 && cny == (fny + 1) / 2 && cnz == (fnz + 1) / 2,
               "pyro_k_mg_flags_down: coarse dims must be ceil(fine / 2)");
  PYRO_REQUIRE(ff && fc, "pyro_k_mg_flags_down: null buffer");
  return ret(launch_mg_flags_down(Dims3{(int)fnx, (int)fny, (int)fnz}, ff,
                                  Dims3{(int)cnx, (int)cny, (int)cnz}, fc, S(stream)),
             "pyro_k_mg_flags_down");
}

int pyro_k_mg_pass(uint32_t nx, uint32_t ny, uint32_t nz, float h, const void* b,
                   const uint8_t* meta, void* phi, int color, float omega, int bc_mode,
                   int storage, void* stream) {
  clear_error();
  PYRO_REQUIRE(dims_ok(nx, ny, nz), "pyro_k_mg_pass: invalid grid dimensions");
  PYRO_REQUIRE(b && meta && phi, "pyro_k_mg_pass: null buffer");
  PYRO_REQUIRE(color == 0 || color == 1, "pyro_k_mg_pass: color must be 0 or 1");
  PYRO_REQUIRE(bc_mode == 0 || bc_mode == 1, "pyro_k_mg_pass: bc_mode must be 0 or 1");
  PYRO_REQUIRE(storage == PYRO_MG_F32 || storage == PYRO_MG_BF16,
               "pyro_k_mg_pass: storage must be PYRO_MG_F32 or PYRO_MG_BF16");
  Dims3 d{(int)nx, (int)ny, (int)nz};
  return ret(storage == PYRO_MG_BF16
                 ? launch_mg_pass_bf16(d, h, b, meta, phi, color, omega, bc_mode, S(stream))
                 : launch_mg_pass(d, h, (const float*)b, meta, (float*)phi, color, omega,
                                  bc_mode, S(stream)),
             "pyro_k_mg_pass");
}

int pyro_k_mg_pass_first(uint32_t nx, uint32_t ny, uint32_t nz, float h, const float* r,
                         void* bq, const uint8_t* meta, void* phi, int color, float omega,
                         int bc_mode, int storage, void* stream) {
  clear_error();
  PYRO_REQUIRE(dims_ok(nx, ny, nz), "pyro_k_mg_pass_first: invalid grid dimensions");
  Dims3 d{(int)nx, (int)ny, (int)nz};
  PYRO_REQUIRE(r && meta && phi && (storage != PYRO_MG_BF16 || bq),
               "pyro_k_mg_pass_first: null buffer");
  PYRO_REQUIRE(color == 0 || color == 1, "pyro_k_mg_pass_first: color must be 0 or 1");
  PYRO_REQUIRE(bc_mode == 0 || bc_mode == 1, "pyro_k_mg_pass_first: bc_mode must be 0 or 1");
  PYRO_REQUIRE(storage == PYRO_MG_F32 || storage == PYRO_MG_BF16,
               "pyro_k_mg_pass_first: storage must be PYRO_MG_F32 or PYRO_MG_BF16");
  return ret(launch_mg_pass_first(d, h, r, bq, meta, phi, color, omega, bc_mode,
                                  storage == PYRO_MG_BF16, S(stream)),
             "pyro_k_mg_pass_first");
}

int pyro_k_mg_pass_last(uint32_t nx, uint32_t ny, uint32_t nz, float h, const void* b,
                        const uint8_t* meta, void* phi, float* out, int color, float omega,
                        int bc_mode, void* stream) {
  clear_error();
  PYRO_REQUIRE(dims_ok(nx, ny, nz), "pyro_k_mg_pass_last: invalid grid dimensions");
  Dims3 d{(int)nx, (int)ny, (int)nz};
  PYRO_REQUIRE(b && meta && phi && out, "pyro_k_mg_pass_last: null buffer");
  PYRO_REQUIRE(color == 0 || color == 1, "pyro_k_mg_pass_last: color must be 0 or 1");
  PYRO_REQUIRE(bc_mode == 0 || bc_mode == 1, "pyro_k_mg_pass_last: bc_mode must be 0 or 1");
  return ret(launch_mg_pass_last_f32(d, h, b, meta, phi, out, color, omega, bc_mode, S(stream)),
             "pyro_k_mg_pass_last");
}

int pyro_k_mg_restrict_m(uint32_t fnx, uint32_t fny, uint32_t fnz, float fh, const void* pf,
                         const void* bf, const uint8_t* mf, uint32_t cnx, uint32_t cny,
                         uint32_t cnz, void* bc, void* pc, int bc_mode, int storage,
                         void* stream) {
  clear_error();
  PYRO_REQUIRE(dims_ok(fnx, fny, fnz), "pyro_k_mg_restrict_m: invalid grid dimensions");
  PYRO_REQUIRE(cnx == (fnx + 1) / 2 && cny == (fny + 1) / 2 && cnz == (fnz + 1) / 2,
               "pyro_k_mg_restrict_m: coarse dims must be ceil(fine / 2)");
  PYRO_REQUIRE(pf && bf && mf && bc && pc, "pyro_k_mg_restrict_m: null buffer");
  PYRO_REQUIRE(bc_mode == 0 || bc_mode == 1, "pyro_k_mg_restrict_m: bc_mode must be 0 or 1");
  PYRO_REQUIRE(storage == PYRO_MG_F32 || storage == PYRO_MG_BF16,
               "pyro_k_mg_restrict_m: storage must be PYRO_MG_F32 or PYRO_MG_BF16");
  Dims3 df{(int)fnx, (int)fny, (int)fnz}, dc{(int)cnx, (int)cny, (int)cnz};
  return ret(storage == PYRO_MG_BF16
                 ? launch_mg_restrict_m_bf16(df, fh, pf, bf, mf, dc, bc, pc, bc_mode, S(stream))
                 : launch_mg_restrict_m(df, fh, (const float*)pf, (const float*)bf, mf, dc,
                                        (float*)bc, (float*)pc, bc_mode, S(stream)),
             "pyro_k_mg_restrict_m");
}

int pyro_k_mg_prolong_m(uint32_t fnx, uint32_t fny, uint32_t fnz, const void* pc,
                        const uint8_t* mf, void* pf, uint32_t cnx, uint32_t cny, uint32_t cnz,
                        const uint8_t* mc, int storage, void* stream) {
  clear_error();
  PYRO_REQUIRE(dims_ok(fnx, fny, fnz), "pyro_k_mg_prolong_m: invalid grid dimensions");
  PYRO_REQUIRE(cnx == (fnx + 1) / 2 && cny == (fny + 1) / 2 && cnz == (fnz + 1) / 2,
               "pyro_k_mg_prolong_m: coarse dims must be ceil(fine / 2)");
  PYRO_REQUIRE(pc && mf && pf && mc, "pyro_k_mg_prolong_m: null buffer");
  PYRO_REQUIRE(storage == PYRO_MG_F32 || storage == PYRO_MG_BF16,
               "pyro_k_mg_prolong_m: storage must be PYRO_MG_F32 or PYRO_MG_BF16");
  Dims3 df{(int)fnx, (int)fny, (int)fnz}, dc{(int)cnx, (int)cny, (int)cnz};
  return ret(storage == PYRO_MG_BF16
                 ? launch_mg_prolong_m_bf16(df, pc, mf, pf, dc, mc, S(stream))
                 : launch_mg_prolong_m(df, (const float*)pc, mf, (float*)pf, dc, mc, S(stream)),
             "pyro_k_mg_prolong_m");
}

int pyro_k_mg_restrict_sym(uint32_t fnx, uint32_t fny, uint32_t fnz, float fh, const void* pf,
                           const void* bf, const uint8_t* mf, uint32_t cnx, uint32_t cny,
                           uint32_t cnz, const uint8_t* mc, void* bc, void* pc, int bc_mode,
                           int storage, void* stream) {
  clear_error();
  PYRO_REQUIRE(dims_ok(fnx, fny, fnz), "pyro_k_mg_restrict_sym: invalid grid dimensions");
  PYRO_REQUIRE(cnx == (fnx + 1) / 2 && cny == (fny + 1) / 2 && cnz == (fnz + 1) / 2,
               "pyro_k_mg_restrict_sym: coarse dims must be ceil(fine / 2)");
  PYRO_REQUIRE(pf && bf && mf && mc && bc && pc, "pyro_k_mg_restrict_sym: null buffer");
  PYRO_REQUIRE(bc_mode == 0 || bc_mode == 1, "pyro_k_mg_restrict_sym: bc_mode must be 0 or 1");
  PYRO_REQUIRE(storage == PYRO_MG_F32 || storage == PYRO_MG_BF16,
               "pyro_k_mg_restrict_sym: storage must be PYRO_MG_F32 or PYRO_MG_BF16");
  Dims3 df{(int)fnx, (int)fny, (int)fnz}, dc{(int)cnx, (int)cny, (int)cnz};
  const bool lo = storage == PYRO_MG_BF16;
  DevBuf wq, rt;
  int rc = wq.alloc(df.cells());
  if (rc == PYRO_OK) rc = rt.alloc(df.cells() * (lo ? 2 : 4));
  if (rc != PYRO_OK) return rc;
  cudaStream_t st = S(stream);
  PYRO_CU(launch_mg_wsum(df, mf, dc, mc, wq.as<uint8_t>(), st));
  PYRO_CU(lo ? launch_mg_restrict_sym_bf16(df, fh, pf, bf, mf, wq.as<uint8_t>(), rt.p, dc, mc, bc,
                                           pc, bc_mode, st)
             : launch_mg_restrict_sym(df, fh, (const float*)pf, (const float*)bf, mf,
                                      wq.as<uint8_t>(), rt.as<float>(), dc, mc, (float*)bc,
                                      (float*)pc, bc_mode, st));
  // the temporaries are freed on return
  PYRO_CU(cudaStreamSynchronize(st));
  return PYRO_OK;
}

int pyro_k_mg_resid(uint32_t nx, uint32_t ny, uint32_t nz, float h, const float* phi,
                    const float* b, const uint32_t* flags, float* stats, void* stream) {
  clear_error();
  PYRO_REQUIRE(dims_ok(nx, ny, nz), "pyro_k_mg_resid: invalid grid dimensions");
  PYRO_REQUIRE(phi && b && flags && stats, "pyro_k_mg_resid: null buffer");
  return ret(launch_mg_resid(Dims3{(int)nx, (int)ny, (int)nz}, h, phi, b, flags, 0, stats,
                             S(stream)),
             "pyro_k_mg_resid");
}

int pyro_k_mg_coarse(uint32_t nx, uint32_t ny, uint32_t nz, float h, const float* b,
                     const uint32_t* flags, float* phi, int iters, float omega, void* stream) {
  clear_error();
  PYRO_REQUIRE(dims_ok(nx, ny, nz), "pyro_k_mg_coarse: invalid grid dimensions");
  PYRO_REQUIRE(b && flags && phi, "pyro_k_mg_coarse: null buffer");
  PYRO_REQUIRE(iters >= 0, "pyro_k_mg_coarse: iters must be >= 0");
  Dims3 d{(int)nx, (int)ny, (int)nz};
  cudaError_t e = cudaSuccess;
  if (mg_coarse_fits(d)) {
    e = launch_mg_coarse(d, h, b, flags, phi, iters, omega, 0, S(stream));
  } else {  // the V-cycle's own fallback: one mask-driven launch per colour
    DevBuf meta;
    int rc = meta.alloc(d.cells());
    if (rc != PYRO_OK) return rc;
    e = launch_mg_meta(d, flags, meta.as<uint8_t>(), S(stream));
    for (int it = 0; it < iters && e == cudaSuccess; it++)
      for (int c = 0; c < 2 && e == cudaSuccess; c++)
        e = launch_mg_pass(d, h, b, meta.as<uint8_t>(), phi, c, omega, 0, S(stream));
    if (e == cudaSuccess) e = cudaStreamSynchronize(S(stream));
  }
  return ret(e, "pyro_k_mg_coarse");
}

int pyro_k_mg_coarse_sym(uint32_t nx, uint32_t ny, uint32_t nz, float h, const float* b,
                         const uint32_t* flags, float* phi, int iters, float omega, int bc_mode,
                         void* stream) {
  clear_error();
  PYRO_REQUIRE(dims_ok(nx, ny, nz), "pyro_k_mg_coarse_sym: invalid grid dimensions");
  PYRO_REQUIRE(b && flags && phi, "pyro_k_mg_coarse_sym: null buffer");
  PYRO_REQUIRE(iters >= 0, "pyro_k_mg_coarse_sym: iters must be >= 0");
  PYRO_REQUIRE(bc_mode == 0 || bc_mode == 1, "pyro_k_mg_coarse_sym: bc_mode must be 0 or 1");
  Dims3 d{(int)nx, (int)ny, (int)nz};
  PYRO_REQUIRE(mg_coarse_fits(d), "pyro_k_mg_coarse_sym: level too large for one cluster");
  return ret(launch_mg_coarse_sym(d, h, b, flags, phi, iters, omega, bc_mode, S(stream)),
             "pyro_k_mg_coarse_sym");
}

int pyro_k_render_pack(const PyroParams* params_dev, uint32_t nx, uint32_t ny, uint32_t nz,
                       const float* s0, const float* s1, const float* sol,
                       const uint32_t* flags, const float* u, const float* v, const float* w,
                       void* vol, void* sol_out, void* vel, void* stream) {
  KDIMS(pyro_k_render_pack)
  PYRO_REQUIRE(params_dev && s0 && s1 && sol && flags && u && v && w && vol && sol_out && vel,
               "pyro_k_render_pack: null buffer");
  return ret(launch_render_pack(params_dev, d, (const float4*)s0, (const float4*)s1,
                                (const float4*)sol, flags, u, v, w, vol, sol_out, vel,
                                S(stream)),
             "pyro_k_render_pack");
}

int pyro_k_render_bricks(uint32_t nx, uint32_t ny, uint32_t nz, const void* vol,
                         const void* sol_packed, float* bricks, void* stream) {
  clear_error();
  PYRO_REQUIRE(dims_ok(nx, ny, nz), "pyro_k_render_bricks: invalid grid dimensions");
  PYRO_REQUIRE(vol && sol_packed && bricks, "pyro_k_render_bricks: null buffer");
  Dims3 d{(int)nx, (int)ny, (int)nz};
  return ret(launch_render_bricks(d, vol, sol_packed, bricks, S(stream)), "pyro_k_render_bricks");
}

int pyro_k_render_ecells(const PyroParams* params_dev, uint32_t nx, uint32_t ny, uint32_t nz,
                         const void* vol, const float* lut, const float* chemi, float* ecell,
                         void* stream) {
  KDIMS(pyro_k_render_ecells)
  PYRO_REQUIRE(vol && lut && chemi && ecell, "pyro_k_render_ecells: null buffer");
  return ret(launch_render_ecells(params_dev, d, vol, lut, chemi, ecell, S(stream)),
             "pyro_k_render_ecells");
}

int pyro_k_render_cdf(uint64_t n, const float* ecell, float* cdf, void* stream) {
  clear_error();
  PYRO_REQUIRE(n >= 1 && n <= (uint64_t)1 << 34, "pyro_k_render_cdf: invalid length");
  PYRO_REQUIRE(ecell && cdf, "pyro_k_render_cdf: null buffer");
  DevBuf scratch;  // the scan's block sums
  int rc = scratch.alloc(render_cdf_scratch_bytes((long)n));
  if (rc != PYRO_OK) return rc;
  cudaError_t e = launch_render_cdf((long)n, ecell, cdf, scratch.p, S(stream));
  if (e == cudaSuccess) e = cudaStreamSynchronize(S(stream));  // before scratch is freed
  return ret(e, "pyro_k_render_cdf");
}

// The tracer's uniform block and the bindings every tracer kernel reads:
// the grid (as pyro_k_render_pack), dx, and the volumes and tables.
#define TRACE_COMMON(name)                                                                  \
  clear_error();                                                                            \
  PYRO_REQUIRE(rp, #name ": null render parameters");                                       \
  PYRO_REQUIRE(dims_ok(rp->dims[0], rp->dims[1], rp->dims[2]),                              \
               #name ": invalid grid dimensions");                                          \
  PYRO_REQUIRE(rp->a[0] > 0.0f, #name ": dx (a[0]) must be positive");                      \
  PYRO_REQUIRE(vol && sol && vel && bricks && lut && ecdf, #name ": null buffer");

int pyro_k_render_lightvol(const PyroRenderParams* rp, const void* vol, const void* sol,
                           const void* vel, const float* bricks, const float* lut,
                           const float* ecdf, uint32_t lx, uint32_t ly, uint32_t lz,
                           uint32_t rays, void* lvA, void* lvB, void* stream) {
  TRACE_COMMON(pyro_k_render_lightvol)
  PYRO_REQUIRE(cache_dims_ok(lx, ly, lz), "pyro_k_render_lightvol: invalid cache dimensions");
  PYRO_REQUIRE(rays >= 1 && rays <= 65536, "pyro_k_render_lightvol: rays must be 1 .. 65536");
  PYRO_REQUIRE(lvA && lvB && lvA != lvB, "pyro_k_render_lightvol: lvA, lvB must be distinct");
  return ret(launch_render_lightvol(*rp, vol, sol, vel, bricks, lut, ecdf, (int)lx, (int)ly,
                                    (int)lz, (int)rays, lvA, lvB, S(stream)),
             "pyro_k_render_lightvol");
}

int pyro_k_render_lightground(const PyroRenderParams* rp, const void* vol, const void* sol,
                              const void* vel, const float* bricks, const float* lut,
                              const float* ecdf, uint32_t gres, uint32_t rays, void* gE,
                              void* stream) {
  TRACE_COMMON(pyro_k_render_lightground)
  PYRO_REQUIRE(cache_dims_ok(gres, gres, 1), "pyro_k_render_lightground: invalid gres");
  PYRO_REQUIRE(rays >= 1 && rays <= 65536, "pyro_k_render_lightground: rays must be 1 .. 65536");
  PYRO_REQUIRE(rp->gc[2] > 0.0f, "pyro_k_render_lightground: ground side (gc[2]) must be positive");
  PYRO_REQUIRE(gE, "pyro_k_render_lightground: null gE");
  return ret(launch_render_lightground(*rp, vol, sol, vel, bricks, lut, ecdf, (int)gres,
                                       (int)rays, gE, S(stream)),
             "pyro_k_render_lightground");
}

int pyro_k_render_blur(const void* src, void* dst, uint32_t nx, uint32_t ny, uint32_t nz,
                       uint32_t axis, uint32_t radius, void* stream) {
  clear_error();
  PYRO_REQUIRE(cache_dims_ok(nx, ny, nz), "pyro_k_render_blur: invalid dimensions");
  PYRO_REQUIRE(axis <= 2, "pyro_k_render_blur: axis must be 0, 1 or 2");
  PYRO_REQUIRE(radius >= 1 && (int)radius <= render_blur_max_radius(),
               "pyro_k_render_blur: radius must be 1 .. 16");
  PYRO_REQUIRE(src && dst && src != dst, "pyro_k_render_blur: src, dst must be distinct buffers");
  return ret(launch_render_blur(src, dst, Dims3{(int)nx, (int)ny, (int)nz}, (int)axis,
                                (int)radius, S(stream)),
             "pyro_k_render_blur");
}

int pyro_k_render_trace(const PyroRenderParams* rp, const void* vol, const void* sol,
                        const void* vel, const float* bricks, const float* lut,
                        const float* ecdf, const void* lvA, const void* lvB, uint32_t lx,
                        uint32_t ly, uint32_t lz, const void* gE, uint32_t gres, float* accum,
                        void* stream) {
  TRACE_COMMON(pyro_k_render_trace)
  PYRO_REQUIRE(accum, "pyro_k_render_trace: null accum");
  PYRO_REQUIRE(cache_dims_ok(rp->res[0], rp->res[1], 1),
               "pyro_k_render_trace: invalid image size (res[0], res[1])");
  PYRO_REQUIRE(rp->res[3] <= 1024, "pyro_k_render_trace: at most 1024 samples per dispatch");
  PYRO_REQUIRE(rp->b[2] >= 0.0f && rp->b[2] <= 64.0f,
               "pyro_k_render_trace: bounces (b[2]) must be 0 .. 64");
  if (rp->gc[3] > 0.5f) {
    PYRO_REQUIRE(lvA && lvB && gE, "pyro_k_render_trace: light-cache mode needs lvA, lvB, gE");
    PYRO_REQUIRE(cache_dims_ok(lx, ly, lz) && cache_dims_ok(gres, gres, 1),
                 "pyro_k_render_trace: invalid cache dimensions");
    PYRO_REQUIRE(rp->gc[2] > 0.0f, "pyro_k_render_trace: ground side (gc[2]) must be positive");
  }
  return ret(launch_render_trace(*rp, vol, sol, vel, bricks, lut, ecdf, lvA, lvB, (int)lx,
                                 (int)ly, (int)lz, gE, (int)gres, accum, S(stream)),
             "pyro_k_render_trace");
}

int pyro_post_select(const float* accum, uint32_t w, uint32_t h, uint32_t k, float* img,
                     uint32_t* keys, uint32_t* sel, float* kth, void* stream) {
  clear_error();
  PYRO_REQUIRE(accum && img && keys && sel && kth, "pyro_post_select: null argument");
  PYRO_REQUIRE(w >= 1 && h >= 1 && (uint64_t)w * h * 3 < (1ull << 31),
               "pyro_post_select: invalid image size");
  PYRO_REQUIRE((uint64_t)k < (uint64_t)w * h, "pyro_post_select: rank k must be < w * h");
  cudaStream_t st = S(stream);
  PYRO_CU(launch_post_select(accum, (int)(w * h), (int)k, img, keys, sel, st));
  uint32_t key = 0;
  PYRO_CU(cudaMemcpyAsync(&key, sel + 3, 4, cudaMemcpyDeviceToHost, st));
  PYRO_CU(cudaStreamSynchronize(st));
  *kth = post_key_value(key);
  return PYRO_OK;
}

int pyro_post_develop(const float* img, uint32_t w, uint32_t h, float gain, float glare,
                      float* scratch, uint8_t* out, float* lin_out, void* stream) {
  clear_error();
  PYRO_REQUIRE(img && scratch && out, "pyro_post_develop: null argument");
  PYRO_REQUIRE(w >= 1 && h >= 1 && (uint64_t)w * h * 12 < (1ull << 31),
               "pyro_post_develop: invalid image size");
  PYRO_REQUIRE(glare >= 0.0f && glare <= 1.0f, "pyro_post_develop: glare must be in [0, 1]");
  return ret(launch_post_develop(img, (int)w, (int)h, gain, glare, scratch, out, lin_out,
                                 S(stream)),
             "pyro_post_develop");
}

int pyro_voxelize(const PyroShape* shapes, uint32_t n_shapes, uint32_t nx, uint32_t ny,
                  uint32_t nz, float dx, float t0, uint32_t seed, const float* slot_density,
                  const uint32_t* slot_kind, float* sol_out, void* stream) {
  clear_error();
  PYRO_REQUIRE(dims_ok(nx, ny, nz), "pyro_voxelize: invalid grid dimensions");
  PYRO_REQUIRE(sol_out && slot_density && slot_kind && (shapes || n_shapes == 0),
               "pyro_voxelize: null argument");
  PYRO_REQUIRE(dx > 0.0f, "pyro_voxelize: dx must be positive");
  // small set-up copy of the shape list and slot tables
  size_t sb = sizeof(PyroShape) * (n_shapes ? n_shapes : 1);
  DevBuf dshapes, dtab;
  int rc;
  if ((rc = dshapes.alloc(sb)) != PYRO_OK) return rc;
  if ((rc = dtab.alloc(64)) != PYRO_OK) return rc;
  cudaStream_t st = S(stream);
  if (n_shapes) PYRO_CU(cudaMemcpyAsync(dshapes.p, shapes, sizeof(PyroShape) * n_shapes,
                                        cudaMemcpyHostToDevice, st));
  PYRO_CU(cudaMemcpyAsync(dtab.p, slot_density, 32, cudaMemcpyHostToDevice, st));
  PYRO_CU(cudaMemcpyAsync((char*)dtab.p + 32, slot_kind, 32, cudaMemcpyHostToDevice, st));
  PYRO_CU(launch_voxelize(dshapes.as<PyroShape>(), n_shapes, Dims3{(int)nx, (int)ny, (int)nz},
                          dx, t0, seed, dtab.as<float>(),
                          reinterpret_cast<const uint32_t*>((char*)dtab.p + 32),
                          (float4*)sol_out, st));
  PYRO_CU(cudaStreamSynchronize(st));
  return PYRO_OK;
}

}  // extern "C"
