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
//   mg_resid     mg.wgsl:122-158 sums of r^2 and b^2
//   mg_coarse    the whole coarsest-level solve (src/sim.rs:473: 80 SOR
//                sweeps at omega 1.6) in one thread-block cluster with the
//                level in distributed shared memory, replacing 160 dispatches.
// The per-colour smoother, the restriction and the prolongation of every
// other level run on per-cell neighbour masks (k_mgf.cu).
#include <cooperative_groups.h>
#include <cstdlib>
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

__global__ void __launch_bounds__(256) k_mg_resid(Lvl d, float h2, const float* __restrict__ p,
                                                  const float* __restrict__ b,
                                                  const uint32_t* __restrict__ f, int bc_mode,
                                                  float* __restrict__ stats) {
  __shared__ float sh[2 * 32];
  int x = blockIdx.x * BX + threadIdx.x;
  int y = blockIdx.y * BY + threadIdx.y;
  int z = blockIdx.z * BZ + threadIdx.z;
  float vals[2] = {0.0f, 0.0f};  // r^2, b^2
  if (d.inb(x, y, z)) {
    int i = d.idx(x, y, z);
    if (__ldg(f + i) != 1u) {
      float r = resid_cell(d, h2, p, b, f, x, y, z, bc_mode);
      float bi = __ldg(b + i);
      vals[0] = r * r;
      vals[1] = bi * bi;
    }
  }
  block_stats<2>(sh, vals, stats, {10, 11}, 0u);
}

// ------------------------------------------------------------ coarse solve
// The coarsest level is swept 80 times per V-cycle (src/sim.rs:473), 160
// dependent red-black passes over ~10-30 k cells.  One thread-block cluster
// of up to 16 CTAs runs them all in a single launch: CTA r owns z-planes
// [r*nz/C, (r+1)*nz/C) of phi in its shared memory, a thread owns up to
// COARSE_K cells with their neighbour mask, count and h^2 b precomputed in
// registers, neighbours across a slab boundary are read from the owning
// CTA's shared memory (distributed shared memory), and the hardware cluster
// barrier separates the colour passes.  The arithmetic per cell is the
// reference's, in the same order, so the result equals 160 separate passes.
constexpr int COARSE_THREADS = 1024;
constexpr int COARSE_K = 2;
constexpr int COARSE_MAX_CLUSTER = 16;

struct CoarseCell {
  int j;             // index in the own slab (-1: none)
  uint32_t meta;     // bits 0-5: fluid in-domain neighbour, bit 6: colour, bit 7: skip
  float cnt;
  float hb;
  const float* zp;   // +z neighbour (local or remote), null when absent
  const float* zm;   // -z neighbour
};

template <typename TS>
__global__ void __launch_bounds__(COARSE_THREADS, 1)
    k_mg_coarse_cluster(Lvl d, float h2, const TS* __restrict__ b,
                        const uint32_t* __restrict__ f, TS* __restrict__ p, int iters,
                        float omega, int bc_mode, int symmetric) {
  namespace cg = cooperative_groups;
  pdl_trigger();
  pdl_wait();
  cg::cluster_group cl = cg::this_cluster();
  extern __shared__ float sp[];
  const int C = (int)cl.num_blocks();
  const int rank = (int)cl.block_rank();
  const int plane = d.nx * d.ny;
  const int z0 = rank * d.nz / C, z1 = (rank + 1) * d.nz / C;
  const int own = (z1 - z0) * plane;
  for (int j = threadIdx.x; j < own; j += COARSE_THREADS) sp[j] = ldv(p + z0 * plane + j);
  cl.sync();  // every slab is loaded before any remote read
  CoarseCell cell[COARSE_K];
#pragma unroll
  for (int r = 0; r < COARSE_K; r++) {
    int j = threadIdx.x + r * COARSE_THREADS;
    cell[r].j = -1;
    cell[r].meta = 0x80u;
    cell[r].cnt = 1.0f;
    cell[r].hb = 0.0f;
    cell[r].zp = nullptr;
    cell[r].zm = nullptr;
    if (j >= own) continue;
    int zl = j / plane, rem = j - zl * plane;
    int y = rem / d.nx, x = rem - y * d.nx, z = z0 + zl;
    int gi = d.idx(x, y, z);
    cell[r].j = j;
    uint32_t meta = (uint32_t)((x + y + z) & 1) << 6;
    float cnt = 0.0f;
#pragma unroll
    for (int k = 0; k < 6; k++) {
      int ax = x + (k == 0) - (k == 1), ay = y + (k == 2) - (k == 3), az = z + (k == 4) - (k == 5);
      if (ay < 0) continue;
      if (!d.inb(ax, ay, az)) {
        if (bc_mode == 0 || ay >= d.ny) cnt += 1.0f;
        continue;
      }
      if (f[d.idx(ax, ay, az)] == 1u) continue;
      meta |= 1u << k;
      cnt += 1.0f;
      if (k >= 4) {
        // owner of plane az and its slab-local index
        int o = 0;
        while (o + 1 < C && (o + 1) * d.nz / C <= az) o++;
        const float* base = (az >= z0 && az < z1) ? sp : cl.map_shared_rank(sp, o);
        int oz0 = o * d.nz / C;
        const float* q = base + (az - oz0) * plane + rem;
        if (k == 4) cell[r].zp = q; else cell[r].zm = q;
      }
    }
    if (f[gi] == 1u || cnt < 0.5f) meta |= 0x80u;
    cell[r].meta = meta;
    cell[r].cnt = cnt;
    cell[r].hb = h2 * ldv(b + gi);
  }
  const int nx = d.nx;
#pragma unroll 1
  for (int it = 0; it < iters; it++) {
    // symmetric: alternate red-black and black-red iterations (SSOR pairs)
    const int first = symmetric ? (it & 1) : 0;
#pragma unroll
    for (int cc = 0; cc < 2; cc++) {
      const int c = cc ^ first;
#pragma unroll
      for (int r = 0; r < COARSE_K; r++) {
        uint32_t m = cell[r].meta;
        if ((m & 0x80u) || ((m >> 6) & 1u) != (uint32_t)c) continue;
        int j = cell[r].j;
        float sum = 0.0f;
        if (m & 1u) sum += sp[j + 1];
        if (m & 2u) sum += sp[j - 1];
        if (m & 4u) sum += sp[j + nx];
        if (m & 8u) sum += sp[j - nx];
        if (m & 16u) sum += *cell[r].zp;
        if (m & 32u) sum += *cell[r].zm;
        sp[j] = wmix(sp[j], (sum - cell[r].hb) / cell[r].cnt, omega);
      }
      cl.sync();
    }
  }
  for (int j = threadIdx.x; j < own; j += COARSE_THREADS) stv(p + z0 * plane + j, sp[j]);
}

__global__ void k_f32_to_bf16(const float* __restrict__ a, __nv_bfloat16* __restrict__ b,
                              size_t n) {
  pdl_trigger();
  pdl_wait();
  size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i < n) b[i] = __float2bfloat16_rn(a[i]);
}
__global__ void k_bf16_to_f32(const __nv_bfloat16* __restrict__ a, float* __restrict__ b,
                              size_t n) {
  pdl_trigger();
  pdl_wait();
  size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i < n) b[i] = __bfloat162float(a[i]);
}

// Cluster size for a level: the largest of 16 / 8 whose slabs keep every
// CTA within COARSE_K cells per thread and the level fits the cluster.
int coarse_cluster_size(Dims3 d) {
  for (int C : {COARSE_MAX_CLUSTER, 8}) {
    if (d.nz < 1) return 0;
    int max_planes = (d.nz + C - 1) / C;
    size_t own = (size_t)max_planes * d.nx * d.ny;
    if (own <= (size_t)COARSE_K * COARSE_THREADS && own * 4 <= 200 * 1024) return C;
  }
  return 0;
}

template <typename TS>
cudaError_t mg_coarse_t(Dims3 d, float h, const TS* b, const uint32_t* f, TS* p, int iters,
                        float omega, int bc_mode, cudaStream_t st, int symmetric = 0) {
  static int attr_done = 0;  // attributes are per function, set once
  static int max_cluster = 0;
  cudaError_t e;
  if (!(attr_done & (1 << sizeof(TS)))) {
    e = cudaFuncSetAttribute(k_mg_coarse_cluster<TS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             200 * 1024);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k_mg_coarse_cluster<TS>,
                             cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    if (e != cudaSuccess) return e;
    attr_done |= 1 << sizeof(TS);
    // the largest cluster this device co-schedules at this CTA shape
    cudaLaunchConfig_t q = {};
    q.gridDim = dim3(COARSE_MAX_CLUSTER, 1, 1);
    q.blockDim = dim3(COARSE_THREADS, 1, 1);
    q.dynamicSmemBytes = 64 * 1024;
    int mc = 0;
    if (cudaOccupancyMaxPotentialClusterSize(&mc, k_mg_coarse_cluster<TS>, &q) != cudaSuccess)
      mc = 8;
    max_cluster = mc >= COARSE_MAX_CLUSTER ? COARSE_MAX_CLUSTER : 8;
    // tuning knob: PYRO_COARSE_CLUSTER=8 caps the cluster at 8 CTAs
    const char* env = getenv("PYRO_COARSE_CLUSTER");
    if (env && atoi(env) == 8) max_cluster = 8;
  }
  int C = coarse_cluster_size(d);
  if (C > max_cluster) C = (max_cluster >= 8 && coarse_cluster_size(d) != 0) ? 8 : 0;
  if (C == 0) return cudaErrorInvalidValue;
  {
    size_t own = (size_t)((d.nz + C - 1) / C) * d.nx * d.ny;
    if (own > (size_t)COARSE_K * COARSE_THREADS) return cudaErrorInvalidValue;
  }
  size_t smem = (size_t)((d.nz + C - 1) / C) * d.nx * d.ny * 4;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)C, 1, 1);
  cfg.blockDim = dim3(COARSE_THREADS, 1, 1);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[2];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = (unsigned)C;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  at[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;  // see launch_pdl
  at[1].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 2;
  return cudaLaunchKernelEx(&cfg, k_mg_coarse_cluster<TS>, Lvl{d.nx, d.ny, d.nz}, h * h, b, f, p,
                            iters, omega, bc_mode, symmetric);
}

}  // namespace

bool mg_coarse_fits(Dims3 d) { return coarse_cluster_size(d) != 0; }

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
  return launch_pdl(k_f32_to_bf16, dim3((unsigned)((n + 255) / 256)), dim3(256), 0, st, a,
                    (__nv_bfloat16*)b, n);
}
cudaError_t launch_bf16_to_f32(const void* a, float* b, size_t n, cudaStream_t st) {
  return launch_pdl(k_bf16_to_f32, dim3((unsigned)((n + 255) / 256)), dim3(256), 0, st,
                    (const __nv_bfloat16*)a, b, n);
}
cudaError_t launch_mg_coarse_sym(Dims3 d, float h, const float* b, const uint32_t* f, float* p,
                                 int iters, float omega, int bc_mode, cudaStream_t st) {
  return mg_coarse_t<float>(d, h, b, f, p, iters, omega, bc_mode, st, 1);
}
cudaError_t launch_mg_coarse_sym_bf16(Dims3 d, float h, const void* b, const uint32_t* f,
                                      void* p, int iters, float omega, int bc_mode,
                                      cudaStream_t st) {
  return mg_coarse_t<__nv_bfloat16>(d, h, (const __nv_bfloat16*)b, f, (__nv_bfloat16*)p, iters,
                                    omega, bc_mode, st, 1);
}

}  // namespace pyro
