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
// [r*nz/C, (r+1)*nz/C) of phi in its shared memory, neighbours across a
// slab boundary are read from the owning CTA's shared memory (distributed
// shared memory), and the hardware cluster barrier separates the colour
// passes.  Threads are sorted by colour: thread t holds, per colour c, the
// cells q = t + T k (k < K) of the slab in the reference smoother's own
// numbering (x = 2 hx + ((y + z + c) & 1), mg.wgsl:17-19), with the
// neighbour mask, count and h^2 b in registers, so every lane of a warp
// updates a cell of the pass's colour and a barrier waits on few warps.  A
// thread loads all neighbours of its cells of the pass before it computes
// any of them.  The arithmetic per cell is the reference's, in the same
// order, so the result equals 160 separate passes bit for bit.
constexpr int COARSE_MAX_CLUSTER = 16;
constexpr int COARSE_SMEM = 200 * 1024;

struct CoarseCell {
  int j;             // index in the own slab (0 for an empty slot)
  uint32_t meta;     // bits 0-5: fluid in-domain neighbour, bit 7: skip
  float cnt;
  float hb;
  const float* zp;   // +z neighbour (local or remote); the cell itself when absent
  const float* zm;   // -z neighbour
};

template <typename TS, int T, int K>
__global__ void __launch_bounds__(T, 1)
    k_mg_coarse_rb(Lvl d, float h2, const TS* __restrict__ b, const uint32_t* __restrict__ f,
                   TS* __restrict__ p, int iters, float omega, int bc_mode, int symmetric) {
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
  for (int j = threadIdx.x; j < own; j += T) sp[j] = ldv(p + z0 * plane + j);
  cl.sync();  // every slab is loaded before any remote read
  const int hxn = (d.nx + 1) / 2;
  const int vpc = hxn * d.ny * (z1 - z0);  // virtual cells per colour
  CoarseCell cell[2][K];
#pragma unroll
  for (int c = 0; c < 2; c++)
#pragma unroll
    for (int k = 0; k < K; k++) {
      CoarseCell& q = cell[c][k];
      q.j = 0;
      q.meta = 0x80u;
      q.cnt = 1.0f;
      q.hb = 0.0f;
      q.zp = sp;
      q.zm = sp;
      const int v = threadIdx.x + T * k;
      if (v >= vpc) continue;
      const int hx = v % hxn, r = v / hxn;
      const int y = r % d.ny, zl = r / d.ny, z = z0 + zl;
      const int x = 2 * hx + ((y + z + c) & 1);
      if (x >= d.nx) continue;
      const int rem = y * d.nx + x, j = zl * plane + rem;
      const int gi = d.idx(x, y, z);
      q.j = j;
      q.zp = sp + j;
      q.zm = sp + j;
      uint32_t meta = 0u;
      float cnt = 0.0f;
#pragma unroll
      for (int nb = 0; nb < 6; nb++) {
        int ax = x + (nb == 0) - (nb == 1), ay = y + (nb == 2) - (nb == 3),
            az = z + (nb == 4) - (nb == 5);
        if (ay < 0) continue;
        if (!d.inb(ax, ay, az)) {
          if (bc_mode == 0 || ay >= d.ny) cnt += 1.0f;
          continue;
        }
        if (f[d.idx(ax, ay, az)] == 1u) continue;
        meta |= 1u << nb;
        cnt += 1.0f;
        if (nb >= 4) {
          // owner of plane az and its slab-local index
          int o = 0;
          while (o + 1 < C && (o + 1) * d.nz / C <= az) o++;
          const float* base = (az >= z0 && az < z1) ? sp : cl.map_shared_rank(sp, o);
          const float* a = base + (az - o * d.nz / C) * plane + rem;
          if (nb == 4) q.zp = a; else q.zm = a;
        }
      }
      if (f[gi] == 1u || cnt < 0.5f) meta |= 0x80u;
      q.meta = meta;
      q.cnt = cnt;
      q.hb = h2 * ldv(b + gi);
    }
  const int nx = d.nx;
#pragma unroll 1
  for (int it = 0; it < iters; it++) {
    // symmetric: alternate red-black and black-red iterations (SSOR pairs)
    const int first = symmetric ? (it & 1) : 0;
#pragma unroll
    for (int cc = 0; cc < 2; cc++) {
      const int c = cc ^ first;
      float nbv[K][6], ownv[K];
      // every load of the pass first: absent neighbours read the cell itself
      // (a valid address) and are not added
#pragma unroll
      for (int k = 0; k < K; k++) {
        const CoarseCell& q = c ? cell[1][k] : cell[0][k];
        const int j = q.j;
        const uint32_t m = q.meta;
        nbv[k][0] = sp[(m & 1u) ? j + 1 : j];
        nbv[k][1] = sp[(m & 2u) ? j - 1 : j];
        nbv[k][2] = sp[(m & 4u) ? j + nx : j];
        nbv[k][3] = sp[(m & 8u) ? j - nx : j];
        nbv[k][4] = *q.zp;
        nbv[k][5] = *q.zm;
        ownv[k] = sp[j];
      }
#pragma unroll
      for (int k = 0; k < K; k++) {
        const CoarseCell& q = c ? cell[1][k] : cell[0][k];
        const uint32_t m = q.meta;
        if (m & 0x80u) continue;
        float sum = 0.0f;
        if (m & 1u) sum += nbv[k][0];
        if (m & 2u) sum += nbv[k][1];
        if (m & 4u) sum += nbv[k][2];
        if (m & 8u) sum += nbv[k][3];
        if (m & 16u) sum += nbv[k][4];
        if (m & 32u) sum += nbv[k][5];
        sp[q.j] = wmix(ownv[k], (sum - q.hb) / q.cnt, omega);
      }
      cl.sync();
    }
  }
  for (int j = threadIdx.x; j < own; j += T) stv(p + z0 * plane + j, sp[j]);
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

// Threads per CTA and cells per thread and colour of the coarse kernel, in
// the order tried: the first whose T * K covers a CTA's cells of one colour.
// Measured on the 2 cm pool's 20 x 40 x 20 level (16 CTAs, 800 cells of a
// colour per CTA, 80 sweeps): 512 threads x 2 cells 142 us, 256 x 4 154 us,
// 128 x 8 229 us -- the barrier and the remote loads of a pass set its
// length, and fewer warps hide less of it.
struct CoarseShape {
  int T, K;
};
constexpr CoarseShape COARSE_SHAPES[] = {{512, 2}, {512, 4}, {256, 8}};

// Cluster size and shape for a level: the largest cluster of 16 / 8 whose
// slabs fit a shape and the shared memory; {0, 0} when none does.
struct CoarsePlan {
  int C = 0;
  CoarseShape s{0, 0};
};
CoarsePlan coarse_plan(Dims3 d, int max_cluster) {
  CoarsePlan pl;
  if (d.nz < 1) return pl;
  for (int C : {COARSE_MAX_CLUSTER, 8}) {
    if (C > max_cluster) continue;
    const int planes = (d.nz + C - 1) / C;
    const size_t vpc = (size_t)((d.nx + 1) / 2) * d.ny * planes;
    if ((size_t)planes * d.nx * d.ny * 4 > (size_t)COARSE_SMEM) continue;
    for (const CoarseShape& s : COARSE_SHAPES)
      if ((size_t)s.T * s.K >= vpc) {
        pl.C = C;
        pl.s = s;
        return pl;
      }
  }
  return pl;
}

template <typename TS, int T, int K>
cudaError_t coarse_launch(const CoarsePlan& pl, Dims3 d, float h, const TS* b, const uint32_t* f,
                          TS* p, int iters, float omega, int bc_mode, cudaStream_t st,
                          int symmetric) {
  auto kern = k_mg_coarse_rb<TS, T, K>;
  static bool attr = false;  // attributes are per function, set once
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         COARSE_SMEM);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  const size_t smem = (size_t)((d.nz + pl.C - 1) / pl.C) * d.nx * d.ny * 4;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)pl.C, 1, 1);
  cfg.blockDim = dim3((unsigned)T, 1, 1);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[2];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = (unsigned)pl.C;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  at[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;  // see launch_pdl
  at[1].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 2;
  return cudaLaunchKernelEx(&cfg, kern, Lvl{d.nx, d.ny, d.nz}, h * h, b, f, p, iters, omega,
                            bc_mode, symmetric);
}

// The largest cluster this device co-schedules for the coarse kernel (16
// where non-portable cluster sizes are allowed, else 8), found once.
int coarse_max_cluster() {
  static int mc = 0;
  if (mc) return mc;
  auto kern = k_mg_coarse_rb<float, 256, 8>;
  int q = 8;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) ==
          cudaSuccess &&
      cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, COARSE_SMEM) ==
          cudaSuccess) {
    cudaLaunchConfig_t c = {};
    c.gridDim = dim3(COARSE_MAX_CLUSTER, 1, 1);
    c.blockDim = dim3(256, 1, 1);
    c.dynamicSmemBytes = 64 * 1024;
    if (cudaOccupancyMaxPotentialClusterSize(&q, kern, &c) != cudaSuccess) q = 8;
  }
  mc = q >= COARSE_MAX_CLUSTER ? COARSE_MAX_CLUSTER : 8;
  return mc;
}

int coarse_cluster_size(Dims3 d) { return coarse_plan(d, COARSE_MAX_CLUSTER).C; }

template <typename TS>
cudaError_t mg_coarse_t(Dims3 d, float h, const TS* b, const uint32_t* f, TS* p, int iters,
                        float omega, int bc_mode, cudaStream_t st, int symmetric = 0) {
  const CoarsePlan pl = coarse_plan(d, coarse_max_cluster());
  if (pl.C == 0) return cudaErrorInvalidValue;
  if (pl.s.K == 2)
    return coarse_launch<TS, 512, 2>(pl, d, h, b, f, p, iters, omega, bc_mode, st, symmetric);
  if (pl.s.K == 4)
    return coarse_launch<TS, 512, 4>(pl, d, h, b, f, p, iters, omega, bc_mode, st, symmetric);
  return coarse_launch<TS, 256, 8>(pl, d, h, b, f, p, iters, omega, bc_mode, st, symmetric);
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
