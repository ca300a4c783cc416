// k_mg.cu — geometric multigrid kernels for the pressure Poisson system.
//
// Operator on every level (src/shaders/mg.wgsl:2,25-35):
//   (sum over fluid neighbours of phi_n - cnt * phi) / h^2 = b
// A neighbour below the floor (y < 0) is skipped (Neumann floor), one outside
// the other faces counts in cnt with phi = 0 (Dirichlet sides and top), a
// solid neighbour is skipped (Neumann at solids).  bc_mode 1 keeps only the
// top face Dirichlet.  Neighbours are visited in the reference's order
// (+x, -x, +y, -y, +z, -z) so sums round identically.
//
//   mg_smooth    mg.wgsl:5-36   red-black Gauss-Seidel / SOR, one colour
//   mg_restrict  mg.wgsl:38-83  fine residual -> fluid-averaged coarse rhs
//   mg_prolong   mg.wgsl:85-120 fluid-weighted trilinear correction
//   mg_resid     mg.wgsl:122-158 sums of r^2 and b^2
//   mg_coarse    the whole coarsest-level solve (src/sim.rs:473: 80 SOR
//                sweeps at omega 1.6) in one CTA with the level in shared
//                memory, replacing 160 dispatches.
#include <cuda_bf16.h>

#include "common.cuh"
#include "kernels.h"

namespace pyro {

namespace {

// Storage of phi and b: FP32 (the reference) or BF16 (the low-precision
// preconditioner); arithmetic is FP32 either way.
__device__ __forceinline__ float ldv(const float* p) { return *p; }
__device__ __forceinline__ float ldv(const __nv_bfloat16* p) { return __bfloat162float(*p); }
__device__ __forceinline__ void stv(float* p, float v) { *p = v; }
__device__ __forceinline__ void stv(__nv_bfloat16* p, float v) { *p = __float2bfloat16_rn(v); }

constexpr int BX = 32, BY = 4, BZ = 2;

inline dim3 grid_for(int x, int y, int z) {
  return dim3((unsigned)((x + BX - 1) / BX), (unsigned)((y + BY - 1) / BY),
              (unsigned)((z + BZ - 1) / BZ));
}

struct Lvl {
  int nx, ny, nz;
  __device__ __forceinline__ bool inb(int x, int y, int z) const {
    return (unsigned)x < (unsigned)nx && (unsigned)y < (unsigned)ny && (unsigned)z < (unsigned)nz;
  }
  __device__ __forceinline__ int idx(int x, int y, int z) const { return x + nx * (y + ny * z); }
};

// Accumulate the 6-neighbour sum and count of cell (x,y,z).
template <typename PhiAt, typename SolidAt>
__device__ __forceinline__ void neigh_sum(const Lvl& d, int x, int y, int z, int bc_mode,
                                          PhiAt phi_at, SolidAt solid_at, float& sum,
                                          float& cnt) {
  sum = 0.0f;
  cnt = 0.0f;
#pragma unroll
  for (int k = 0; k < 6; k++) {
    int nx_ = x + (k == 0) - (k == 1);
    int ny_ = y + (k == 2) - (k == 3);
    int nz_ = z + (k == 4) - (k == 5);
    if (ny_ < 0) continue;
    if (!d.inb(nx_, ny_, nz_)) {
      if (bc_mode == 0 || ny_ >= d.ny) cnt += 1.0f;
      continue;
    }
    int j = d.idx(nx_, ny_, nz_);
    if (solid_at(j)) continue;
    sum += phi_at(j);
    cnt += 1.0f;
  }
}

template <typename TS>
__global__ void __launch_bounds__(256) k_mg_smooth(Lvl d, float h2, const TS* __restrict__ b,
                                                   const uint32_t* __restrict__ f,
                                                   TS* __restrict__ p, int color,
                                                   float omega, int bc_mode) {
  int y = blockIdx.y * BY + threadIdx.y;
  int z = blockIdx.z * BZ + threadIdx.z;
  int x = (int)(blockIdx.x * BX + threadIdx.x) * 2 + ((y + z + color) & 1);
  if (!d.inb(x, y, z)) return;
  int i = d.idx(x, y, z);
  if (__ldg(f + i) == 1u) return;
  float sum, cnt;
  neigh_sum(
      d, x, y, z, bc_mode, [&](int j) { return ldv(p + j); },
      [&](int j) { return __ldg(f + j) == 1u; }, sum, cnt);
  if (cnt < 0.5f) return;
  stv(p + i, wmix(ldv(p + i), (sum - h2 * ldv(b + i)) / cnt, omega));
}

template <typename TS>
__device__ __forceinline__ float resid_cell(const Lvl& d, float h2, const TS* __restrict__ p,
                                            const TS* __restrict__ b,
                                            const uint32_t* __restrict__ f, int x, int y, int z,
                                            int bc_mode) {
  int i = d.idx(x, y, z);
  if (__ldg(f + i) == 1u) return 0.0f;
  float pcen = ldv(p + i);
  float sum, cnt;
  neigh_sum(
      d, x, y, z, bc_mode, [&](int j) { return ldv(p + j); },
      [&](int j) { return __ldg(f + j) == 1u; }, sum, cnt);
  return ldv(b + i) - (sum - cnt * pcen) / h2;
}

template <typename TS>
__global__ void __launch_bounds__(256) k_mg_restrict(Lvl df, float h2f,
                                                     const TS* __restrict__ pf,
                                                     const TS* __restrict__ bf,
                                                     const uint32_t* __restrict__ ff, Lvl dc,
                                                     TS* __restrict__ bc,
                                                     TS* __restrict__ pc,
                                                     uint32_t* __restrict__ fc, int bc_mode) {
  int x = blockIdx.x * BX + threadIdx.x;
  int y = blockIdx.y * BY + threadIdx.y;
  int z = blockIdx.z * BZ + threadIdx.z;
  if (!dc.inb(x, y, z)) return;
  float r = 0.0f, nfl = 0.0f;
#pragma unroll
  for (int k = 0; k < 8; k++) {
    int cx = 2 * x + (k & 1), cy = 2 * y + ((k >> 1) & 1), cz = 2 * z + ((k >> 2) & 1);
    if (!df.inb(cx, cy, cz)) continue;
    if (__ldg(ff + df.idx(cx, cy, cz)) != 1u) {
      nfl += 1.0f;
      r += resid_cell(df, h2f, pf, bf, ff, cx, cy, cz, bc_mode);
    }
  }
  int i = dc.idx(x, y, z);
  stv(bc + i, (nfl > 0.0f) ? r / fmaxf(nfl, 1.0f) : 0.0f);
  stv(pc + i, 0.0f);
  fc[i] = (nfl > 0.0f) ? 0u : 1u;
}

template <typename TS>
__global__ void __launch_bounds__(256) k_mg_prolong(Lvl df, const TS* __restrict__ pc,
                                                    const uint32_t* __restrict__ ff,
                                                    TS* __restrict__ pf, Lvl dc,
                                                    const uint32_t* __restrict__ fc) {
  int x = blockIdx.x * BX + threadIdx.x;
  int y = blockIdx.y * BY + threadIdx.y;
  int z = blockIdx.z * BZ + threadIdx.z;
  if (!df.inb(x, y, z)) return;
  int i = df.idx(x, y, z);
  if (__ldg(ff + i) == 1u) return;
  // x = (c + 0.5) * 0.5 - 0.5: even c -> i0 = c/2 - 1, frac 0.75;
  // odd c -> i0 = (c-1)/2, frac 0.25 (exact in FP32).
  float gx = ((float)x + 0.5f) * 0.5f - 0.5f;
  float gy = ((float)y + 0.5f) * 0.5f - 0.5f;
  float gz = ((float)z + 0.5f) * 0.5f - 0.5f;
  int i0x = (int)floorf(gx), i0y = (int)floorf(gy), i0z = (int)floorf(gz);
  float frx = gx - (float)i0x, fry = gy - (float)i0y, frz = gz - (float)i0z;
  float acc = 0.0f, ws = 0.0f;
#pragma unroll
  for (int k = 0; k < 8; k++) {
    int ox = k & 1, oy = (k >> 1) & 1, oz = (k >> 2) & 1;
    int cx = min(max(i0x + ox, 0), dc.nx - 1);
    int cy = min(max(i0y + oy, 0), dc.ny - 1);
    int cz = min(max(i0z + oz, 0), dc.nz - 1);
    int j = dc.idx(cx, cy, cz);
    if (__ldg(fc + j) == 1u) continue;
    float wx = ox ? frx : 1.0f - frx;
    float wy = oy ? fry : 1.0f - fry;
    float wz = oz ? frz : 1.0f - frz;
    float w = wx * wy * wz;
    acc += w * ldv(pc + j);
    ws += w;
  }
  if (ws > 1e-4f) stv(pf + i, ldv(pf + i) + acc / ws);
}

__global__ void __launch_bounds__(256) k_mg_resid(Lvl d, float h2, const float* __restrict__ p,
                                                  const float* __restrict__ b,
                                                  const uint32_t* __restrict__ f, int bc_mode,
                                                  float* __restrict__ stats) {
  __shared__ float sh[32];
  int x = blockIdx.x * BX + threadIdx.x;
  int y = blockIdx.y * BY + threadIdx.y;
  int z = blockIdx.z * BZ + threadIdx.z;
  float r2 = 0.0f, b2 = 0.0f;
  if (d.inb(x, y, z)) {
    int i = d.idx(x, y, z);
    if (__ldg(f + i) != 1u) {
      float r = resid_cell(d, h2, p, b, f, x, y, z, bc_mode);
      float bi = __ldg(b + i);
      r2 = r * r;
      b2 = bi * bi;
    }
  }
  block_add(sh, r2, stats + 10);
  block_add(sh, b2, stats + 11);
}

// ------------------------------------------------------------ coarse solve
// One CTA of 1024 threads; thread t owns the (x, y) column t of the level
// and walks z over the cells of the colour being swept.  phi, h^2 b and the
// solid flags of the whole level live in shared memory (9 bytes per cell).
constexpr int COARSE_THREADS = 1024;
constexpr size_t COARSE_SMEM_CAP = 200 * 1024;

template <typename TS>
__global__ void __launch_bounds__(COARSE_THREADS, 1)
    k_mg_coarse(Lvl d, float h2, const TS* __restrict__ b, const uint32_t* __restrict__ f,
                TS* __restrict__ p, int iters, float omega, int bc_mode) {
  extern __shared__ float smem[];
  const int n = d.nx * d.ny * d.nz;
  float* sp = smem;
  float* sb = smem + n;
  uint8_t* sf = reinterpret_cast<uint8_t*>(smem + 2 * n);
  for (int j = threadIdx.x; j < n; j += COARSE_THREADS) {
    sp[j] = ldv(p + j);
    sb[j] = h2 * ldv(b + j);
    sf[j] = (uint8_t)(f[j] == 1u);
  }
  const int t = threadIdx.x;
  const bool own = t < d.nx * d.ny;
  const int x = own ? t % d.nx : 0;
  const int y = own ? t / d.nx : 0;
  const int plane = d.nx * d.ny;
  __syncthreads();
#pragma unroll 1
  for (int it = 0; it < iters; it++) {
#pragma unroll 1
    for (int c = 0; c < 2; c++) {
      if (own) {
        // colour c of cell (x,y,z) is (x+y+z)&1
#pragma unroll 1
        for (int z = (c + x + y) & 1; z < d.nz; z += 2) {
          int i = t + plane * z;
          if (sf[i]) continue;
          float sum, cnt;
          neigh_sum(
              d, x, y, z, bc_mode, [&](int j) { return sp[j]; },
              [&](int j) { return sf[j] != 0; }, sum, cnt);
          if (cnt >= 0.5f) sp[i] = wmix(sp[i], (sum - sb[i]) / cnt, omega);
        }
      }
      __syncthreads();
    }
  }
  for (int j = threadIdx.x; j < n; j += COARSE_THREADS) stv(p + j, sp[j]);
}

__global__ void k_f32_to_bf16(const float* __restrict__ a, __nv_bfloat16* __restrict__ b,
                              size_t n) {
  size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i < n) b[i] = __float2bfloat16_rn(a[i]);
}
__global__ void k_bf16_to_f32(const __nv_bfloat16* __restrict__ a, float* __restrict__ b,
                              size_t n) {
  size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i < n) b[i] = __bfloat162float(a[i]);
}

template <typename TS>
cudaError_t mg_smooth_t(Dims3 d, float h, const TS* b, const uint32_t* f, TS* p, int color,
                        float omega, int bc_mode, cudaStream_t st) {
  Lvl l{d.nx, d.ny, d.nz};
  k_mg_smooth<TS><<<grid_for((d.nx + 1) / 2, d.ny, d.nz), dim3(BX, BY, BZ), 0, st>>>(
      l, h * h, b, f, p, color, omega, bc_mode);
  return cudaGetLastError();
}

template <typename TS>
cudaError_t mg_restrict_t(Dims3 df, float hf, const TS* pf, const TS* bf, const uint32_t* ff,
                          Dims3 dc, TS* bc, TS* pc, uint32_t* fc, int bc_mode, cudaStream_t st) {
  k_mg_restrict<TS><<<grid_for(dc.nx, dc.ny, dc.nz), dim3(BX, BY, BZ), 0, st>>>(
      Lvl{df.nx, df.ny, df.nz}, hf * hf, pf, bf, ff, Lvl{dc.nx, dc.ny, dc.nz}, bc, pc, fc,
      bc_mode);
  return cudaGetLastError();
}

template <typename TS>
cudaError_t mg_prolong_t(Dims3 df, const TS* pc, const uint32_t* ff, TS* pf, Dims3 dc,
                         const uint32_t* fc, cudaStream_t st) {
  k_mg_prolong<TS><<<grid_for(df.nx, df.ny, df.nz), dim3(BX, BY, BZ), 0, st>>>(
      Lvl{df.nx, df.ny, df.nz}, pc, ff, pf, Lvl{dc.nx, dc.ny, dc.nz}, fc);
  return cudaGetLastError();
}

template <typename TS>
cudaError_t mg_coarse_t(Dims3 d, float h, const TS* b, const uint32_t* f, TS* p, int iters,
                        float omega, int bc_mode, cudaStream_t st) {
  if (!mg_coarse_fits(d)) return cudaErrorInvalidValue;
  cudaError_t e = cudaFuncSetAttribute(k_mg_coarse<TS>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)COARSE_SMEM_CAP);
  if (e != cudaSuccess) return e;
  k_mg_coarse<TS><<<1, COARSE_THREADS, d.cells() * 9, st>>>(Lvl{d.nx, d.ny, d.nz}, h * h, b, f,
                                                           p, iters, omega, bc_mode);
  return cudaGetLastError();
}

}  // namespace

bool mg_coarse_fits(Dims3 d) {
  size_t n = d.cells();
  return d.nx * d.ny <= COARSE_THREADS && n * 9 <= COARSE_SMEM_CAP;
}

cudaError_t launch_mg_smooth(Dims3 d, float h, const float* b, const uint32_t* f, float* p,
                             int color, float omega, int bc_mode, cudaStream_t st) {
  return mg_smooth_t<float>(d, h, b, f, p, color, omega, bc_mode, st);
}

cudaError_t launch_mg_restrict(Dims3 df, float hf, const float* pf, const float* bf,
                               const uint32_t* ff, Dims3 dc, float* bc, float* pc, uint32_t* fc,
                               int bc_mode, cudaStream_t st) {
  return mg_restrict_t<float>(df, hf, pf, bf, ff, dc, bc, pc, fc, bc_mode, st);
}

cudaError_t launch_mg_prolong(Dims3 df, const float* pc, const uint32_t* ff, float* pf, Dims3 dc,
                              const uint32_t* fc, cudaStream_t st) {
  return mg_prolong_t<float>(df, pc, ff, pf, dc, fc, st);
}

cudaError_t launch_mg_resid(Dims3 d, float h, const float* p, const float* b, const uint32_t* f,
                            int bc_mode, float* stats, cudaStream_t st) {
  k_mg_resid<<<grid_for(d.nx, d.ny, d.nz), dim3(BX, BY, BZ), 0, st>>>(
      Lvl{d.nx, d.ny, d.nz}, h * h, p, b, f, bc_mode, stats);
  return cudaGetLastError();
}

cudaError_t launch_mg_coarse(Dims3 d, float h, const float* b, const uint32_t* f, float* p,
                             int iters, float omega, int bc_mode, cudaStream_t st) {
  return mg_coarse_t<float>(d, h, b, f, p, iters, omega, bc_mode, st);
}

// ---- BF16-storage hierarchy (MGPCG preconditioner) -----------------------
cudaError_t launch_f32_to_bf16(const float* a, void* b, size_t n, cudaStream_t st) {
  k_f32_to_bf16<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(a, (__nv_bfloat16*)b, n);
  return cudaGetLastError();
}
cudaError_t launch_bf16_to_f32(const void* a, float* b, size_t n, cudaStream_t st) {
  k_bf16_to_f32<<<(unsigned)((n + 255) / 256), 256, 0, st>>>((const __nv_bfloat16*)a, b, n);
  return cudaGetLastError();
}
cudaError_t launch_mg_smooth_bf16(Dims3 d, float h, const void* b, const uint32_t* f, void* p,
                                  int color, float omega, int bc_mode, cudaStream_t st) {
  return mg_smooth_t<__nv_bfloat16>(d, h, (const __nv_bfloat16*)b, f, (__nv_bfloat16*)p, color,
                                    omega, bc_mode, st);
}
cudaError_t launch_mg_restrict_bf16(Dims3 df, float hf, const void* pf, const void* bf,
                                    const uint32_t* ff, Dims3 dc, void* bc, void* pc,
                                    uint32_t* fc, int bc_mode, cudaStream_t st) {
  return mg_restrict_t<__nv_bfloat16>(df, hf, (const __nv_bfloat16*)pf,
                                      (const __nv_bfloat16*)bf, ff, dc, (__nv_bfloat16*)bc,
                                      (__nv_bfloat16*)pc, fc, bc_mode, st);
}
cudaError_t launch_mg_prolong_bf16(Dims3 df, const void* pc, const uint32_t* ff, void* pf,
                                   Dims3 dc, const uint32_t* fc, cudaStream_t st) {
  return mg_prolong_t<__nv_bfloat16>(df, (const __nv_bfloat16*)pc, ff, (__nv_bfloat16*)pf, dc,
                                     fc, st);
}
cudaError_t launch_mg_coarse_bf16(Dims3 d, float h, const void* b, const uint32_t* f, void* p,
                                  int iters, float omega, int bc_mode, cudaStream_t st) {
  return mg_coarse_t<__nv_bfloat16>(d, h, (const __nv_bfloat16*)b, f, (__nv_bfloat16*)p, iters,
                                    omega, bc_mode, st);
}

}  // namespace pyro
