// kernels.h — host-side launchers of the simulation and multigrid kernels
// (internal to libpyro_b200; the C ABI is include/pyro_sim.h).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/pyro_sim.h"

namespace pyro {

struct Dims3 {
  int nx, ny, nz;
  size_t cells() const { return (size_t)nx * ny * nz; }
  size_t faces() const { return (size_t)(nx + 1) * (ny + 1) * (nz + 1); }
};

// Simulation kernels; P is a device pointer to the parameter block and
// stats (device, PYRO_STATS_N floats) may be null.  All return the launch
// status.
cudaError_t launch_solid(const PyroParams* P, Dims3 d, const float4* solIn, float4* solOut,
                         float4* pyr, uint32_t* flags, const float4* s0, float* stats,
                         cudaStream_t st);
cudaError_t launch_curl(const PyroParams* P, Dims3 d, const float* u, const float* v,
                        const float* w, float4* curl, float* stats, cudaStream_t st);
// lohi: 6 face arrays of (nx+1)(ny+1)(nz+1) floats, the predictor's
// per-component min (0..2) and max (3..5) of v at the backtrace, written by
// adv_vel1 and read by adv_vel2.
cudaError_t launch_adv_vel1(const PyroParams* P, Dims3 d, const float* u, const float* v,
                            const float* w, float* hu, float* hv, float* hw, float* lohi,
                            cudaStream_t st);
cudaError_t launch_adv_vel2(const PyroParams* P, Dims3 d, const float* u, const float* v,
                            const float* w, const float* hu, const float* hv, const float* hw,
                            const float* lohi, float* ou, float* ov, float* ow,
                            const uint32_t* flags, cudaStream_t st);
// bt: 3 cell arrays (x, y, z) of the cell-centred backtrace, written by
// adv_s1 and read by adv_s2.
cudaError_t launch_adv_s1(const PyroParams* P, Dims3 d, const float* u, const float* v,
                          const float* w, const float4* s0, const float4* s1, float4* h0,
                          float4* h1, float* bt, cudaStream_t st);
cudaError_t launch_adv_s2(const PyroParams* P, Dims3 d, const float* u, const float* v,
                          const float* w, const float4* s0, const float4* s1, const float4* h0,
                          const float4* h1, const float* bt, float4* o0, float4* o1,
                          cudaStream_t st);
cudaError_t launch_react(const PyroParams* P, Dims3 d, const float4* s0in, const float4* s1in,
                         float4* s0out, float4* s1out, const uint32_t* flags, const float4* sol,
                         const float4* pyr, const float4* curl, float* stats, cudaStream_t st);
// forces runs a per-cell confinement kernel into `conf` (N float4 scratch)
// and then the face kernel.
cudaError_t launch_forces(const PyroParams* P, Dims3 d, float* u, float* v, float* w,
                          const float4* s0, const float4* s1, const float4* curl,
                          float4* conf, const uint32_t* flags, cudaStream_t st);
cudaError_t launch_divergence(const PyroParams* P, Dims3 d, const float* u, const float* v,
                              const float* w, const float4* s1, const uint32_t* flags, float* b,
                              cudaStream_t st);
// Renderer input pack (k_render.cu): three volumes of 4 binary16 values per
// cell, and the 8^3 brick maxima read back from two of them.
cudaError_t launch_render_pack(const PyroParams* P, Dims3 d, const float4* s0, const float4* s1,
                               const float4* sol, const uint32_t* flags, const float* u,
                               const float* v, const float* w, void* vol, void* solp, void* vel,
                               cudaStream_t st);
cudaError_t launch_render_bricks(Dims3 d, const void* vol, const void* solp, float* bricks,
                                 cudaStream_t st);
// Emission power per cell from the packed vol and the soot colour table
// (1024 float4), chemi = 4 host floats; and its FP64 cumulative
// distribution (n + 1 floats) with render_cdf_scratch_bytes(n) of scratch.
cudaError_t launch_render_ecells(const PyroParams* P, Dims3 d, const void* vol, const float* lut,
                                 const float* chemi, float* ecell, cudaStream_t st);
size_t render_cdf_scratch_bytes(long n);
cudaError_t launch_render_cdf(long n, const float* ecell, float* cdf, void* scratch,
                              cudaStream_t st);
// The volume path tracer (k_trace.cu) on the packed volumes: camera rays
// into accum, the two light caches, and the caches' separable blur (radius
// 1 .. render_blur_max_radius()).
cudaError_t launch_render_trace(const PyroRenderParams& R, const void* vol, const void* sol,
                                const void* vel, const float* bricks, const float* lut,
                                const float* ecdf, const void* lvA, const void* lvB, int lx,
                                int ly, int lz, const void* gE, int gres, float* accum,
                                cudaStream_t st);
cudaError_t launch_render_lightvol(const PyroRenderParams& R, const void* vol, const void* sol,
                                   const void* vel, const float* bricks, const float* lut,
                                   const float* ecdf, int lx, int ly, int lz, int rays,
                                   void* lvA, void* lvB, cudaStream_t st);
cudaError_t launch_render_lightground(const PyroRenderParams& R, const void* vol,
                                      const void* sol, const void* vel, const float* bricks,
                                      const float* lut, const float* ecdf, int gres, int rays,
                                      void* gE, cudaStream_t st);
int render_blur_max_radius();
cudaError_t launch_render_blur(const void* src, void* dst, Dims3 d, int axis, int r,
                               cudaStream_t st);
cudaError_t launch_project(const PyroParams* P, Dims3 d, float* u, float* v, float* w,
                           const float* phi, const uint32_t* flags, cudaStream_t st);

// Frame development (k_post.cu): the mean radiance of n = w*h pixels from
// the tracer's accumulation image, each pixel's luminance key, and the
// radix select of the k-th smallest luminance (its key ends in sel[3]; sel
// holds POST_SEL_WORDS words); then the exposure, glare, tone curve and
// 8-bit image.  scratch: 4 * 3n floats.
constexpr int POST_SEL_WORDS = 260;
cudaError_t launch_post_select(const float* accum, int n, int k, float* img, uint32_t* keys,
                               uint32_t* sel, cudaStream_t st);
float post_key_value(uint32_t key);
cudaError_t launch_post_develop(const float* img, int w, int h, float gain, float glare,
                                float* scratch, uint8_t* out, float* lin_out, cudaStream_t st);

// Multigrid level kernels (src/shaders/mg.wgsl).  bc_mode 0 = reference
// boundaries, 1 = Dirichlet on the top face only.
// The same statistics from the level's neighbour masks, four cells per
// thread (k_mgf.cu); rows of a multiple of 4 cells, else
// cudaErrorNotSupported.
cudaError_t launch_mg_resid_m(Dims3 d, float h, const float* p, const float* b,
                              const uint8_t* meta, int bc_mode, float* stats, cudaStream_t st);
cudaError_t launch_mg_resid(Dims3 d, float h, const float* p, const float* b, const uint32_t* f,
                            int bc_mode, float* stats, cudaStream_t st);
// Whole coarsest-level solve in one CTA (shared memory); returns
// cudaErrorInvalidValue when the level does not fit.
bool mg_coarse_fits(Dims3 d);
cudaError_t launch_mg_coarse(Dims3 d, float h, const float* b, const uint32_t* f, float* p,
                             int iters, float omega, int bc_mode, cudaStream_t st);

// BF16-storage variants (phi and b as __nv_bfloat16, FP32 arithmetic) for
// the low-precision MGPCG preconditioner; pointers are bf16 arrays.
cudaError_t launch_f32_to_bf16(const float* a, void* b, size_t n, cudaStream_t st);
cudaError_t launch_bf16_to_f32(const void* a, float* b, size_t n, cudaStream_t st);

// Multigrid on neighbour masks (k_mgf.cu): per-level masks, coarse solid
// flags and the prolongation.
cudaError_t launch_mg_meta(Dims3 d, const uint32_t* f, uint8_t* meta, cudaStream_t st);
cudaError_t launch_mg_flags_down(Dims3 df, const uint32_t* ff, Dims3 dc, uint32_t* fc,
                                 cudaStream_t st);
cudaError_t launch_mg_prolong_m(Dims3 df, const float* pc, const uint8_t* mf, float* pf,
                                Dims3 dc, const uint8_t* mc, cudaStream_t st);
cudaError_t launch_mg_prolong_m_bf16(Dims3 df, const void* pc, const uint8_t* mf, void* pf,
                                     Dims3 dc, const uint8_t* mc, cudaStream_t st);

// Lean per-colour pass and restriction driven by the neighbour mask.
cudaError_t launch_mg_pass(Dims3 d, float h, const float* b, const uint8_t* meta, float* p,
                           int color, float omega, int bc_mode, cudaStream_t st);
cudaError_t launch_mg_pass_bf16(Dims3 d, float h, const void* b, const uint8_t* meta, void* p,
                                int color, float omega, int bc_mode, cudaStream_t st);
// The first and last colour pass on level 0 of the CG preconditioner's
// V-cycle (k_mg_pass4z / k_mg_pass2z): the first from the zero initial
// guess with the FP32 right-hand side r (with BF16 storage also written
// rounded into bq), writing every cell of p; the last on BF16 storage
// writing every cell widened to FP32 into out.
cudaError_t launch_mg_pass_first(Dims3 d, float h, const float* r, void* bq,
                                 const uint8_t* meta, void* p, int color, float omega,
                                 int bc_mode, bool bf16, cudaStream_t st);
cudaError_t launch_mg_pass_last_f32(Dims3 d, float h, const void* b, const uint8_t* meta,
                                    void* p, float* out, int color, float omega, int bc_mode,
                                    cudaStream_t st);
cudaError_t launch_mg_restrict_m(Dims3 df, float h, const float* pf, const float* bf,
                                 const uint8_t* mf, Dims3 dc, float* bc, float* pc, int bc_mode,
                                 cudaStream_t st);
cudaError_t launch_mg_restrict_m_bf16(Dims3 df, float h, const void* pf, const void* bf,
                                      const uint8_t* mf, Dims3 dc, void* bc, void* pc,
                                      int bc_mode, cudaStream_t st);

// Symmetric V-cycle pieces for the MGPCG preconditioner: wsum gives each
// fine cell 64 x its fluid prolongation weight sum (a byte, exact; once per
// flag field); the restriction divides the residual by that weight into
// `rt`, then applies the transpose (P^T / 8); the coarse solve alternates
// red-black / black-red.
cudaError_t launch_mg_wsum(Dims3 df, const uint8_t* mf, Dims3 dc, const uint8_t* mc,
                           uint8_t* wq, cudaStream_t st);
cudaError_t launch_mg_restrict_sym(Dims3 df, float h, const float* pf, const float* bf,
                                   const uint8_t* mf, const uint8_t* wq, float* rt, Dims3 dc,
                                   const uint8_t* mc, float* bc, float* pc, int bc_mode,
                                   cudaStream_t st);
cudaError_t launch_mg_restrict_sym_bf16(Dims3 df, float h, const void* pf, const void* bf,
                                        const uint8_t* mf, const uint8_t* wq, void* rt,
                                        Dims3 dc, const uint8_t* mc, void* bc, void* pc,
                                        int bc_mode, cudaStream_t st);
cudaError_t launch_mg_coarse_sym(Dims3 d, float h, const float* b, const uint32_t* f, float* p,
                                 int iters, float omega, int bc_mode, cudaStream_t st);
cudaError_t launch_mg_coarse_sym_bf16(Dims3 d, float h, const void* b, const uint32_t* f,
                                      void* p, int iters, float omega, int bc_mode,
                                      cudaStream_t st);

// Voxelizer.
cudaError_t launch_voxelize(const PyroShape* shapes_dev, uint32_t n, Dims3 d, float dx, float t0,
                            uint32_t seed, const float* dens_dev, const uint32_t* kind_dev,
                            float4* sol, cudaStream_t st);

}  // namespace pyro
