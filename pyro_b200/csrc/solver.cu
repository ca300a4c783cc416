// solver.cu — pressure solvers (fixed V-cycles as in src/sim.rs:451-491,
// V-cycles to a tolerance, and flexible MGPCG).
//
// MGPCG solves the reference system A phi = b (A negative semi-definite,
// src/shaders/mg.wgsl:25-35) by CG on -A: with r = b - A phi, z = V(r) one
// symmetric V-cycle from a zero guess (Multigrid::vcycle_sym), q = A p:
//   alpha = <r,z> / <p,q>,  phi += alpha p,  r -= alpha q,
//   beta  = <z_new, r_new - r_old> / <z_old, r_old> = -<z_new, q> / <p,q>
// (Polak-Ribiere form, valid for the non-symmetric V-cycle), p = z + beta p.
// Vectors are FP32; every dot product and norm is accumulated in FP64.
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>

#include "common.cuh"
#include "net.h"
#include "solver.h"

namespace pyro {

namespace {

__device__ __forceinline__ float cvt_load(const float* p) { return *p; }
__device__ __forceinline__ float cvt_load(const __nv_bfloat16* p) { return __bfloat162float(*p); }
__device__ __forceinline__ void cvt_store(float* p, float v) { *p = v; }
__device__ __forceinline__ void cvt_store(__nv_bfloat16* p, float v) {
  *p = __float2bfloat16_rn(v);
}

constexpr int BX = 32, BY = 4, BZ = 2;
inline dim3 grid_for(Dims3 d) {
  return dim3((unsigned)((d.nx + BX - 1) / BX), (unsigned)((d.ny + BY - 1) / BY),
              (unsigned)((d.nz + BZ - 1) / BZ));
}

enum { SC_RZ = 0, SC_PQ, SC_RR, SC_BB, SC_ZQ, SC_RZN, SC_N = 8 };
constexpr int VT = 256;  // threads per block of the CG vector kernels

// The FP64 scalars are followed in the same allocation by one row of block
// partial sums per scalar and one arrival counter per scalar (block_add_d).
constexpr int RED_MAXB = 4096;  // blocks of a reduction kernel at most
constexpr size_t SC_BYTES = SC_N * 8 + (size_t)SC_N * RED_MAXB * 8 + SC_N * 4;

unsigned vec_blocks(size_t n) {
  static int nsm = 0;
  if (nsm <= 0) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        nsm <= 0)
      nsm = 148;
  }
  return (unsigned)std::min<size_t>(std::min<size_t>((n + 255) / 256, (size_t)nsm * 8),
                                    (size_t)RED_MAXB);
}

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
// sc[slot] += the sum of v over every thread of the grid, in an order that
// does not depend on scheduling: each block writes its sum (a fixed tree
// over its threads) to the slot's row of partials; the block that arrives
// last adds the row in index order and resets the counter.  So a solve
// repeats bit for bit.  Every thread of every block must call; blocks of
// VT threads.
__device__ __forceinline__ void block_add_d(double* sh, double v, double* sc, int slot) {
  __shared__ bool s_last;
  const int t = threadIdx.x;
  double* part = sc + SC_N + (size_t)slot * RED_MAXB;
  unsigned* cnt = reinterpret_cast<unsigned*>(sc + SC_N + (size_t)SC_N * RED_MAXB) + slot;
  v = warp_sum_d(v);
  __syncthreads();
  if ((t & 31) == 0) sh[t >> 5] = v;
  __syncthreads();
  if (t < 32) {
    double s = t < VT / 32 ? sh[t] : 0.0;
    s = warp_sum_d(s);
    if (t == 0) {
      part[blockIdx.x] = s;
      __threadfence();
      s_last = atomicAdd(cnt, 1u) == gridDim.x - 1;
    }
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  double a = 0.0;
  for (unsigned k = t; k < gridDim.x; k += VT) a += __ldcg(part + k);
  a = warp_sum_d(a);
  if ((t & 31) == 0) sh[t >> 5] = a;
  __syncthreads();
  if (t == 0) {
    double s = 0.0;
    for (int w = 0; w < VT / 32; w++) s += sh[w];
    sc[slot] += s;
    *cnt = 0u;
  }
}

struct L3 {
  int nx, ny, nz;
  __device__ __forceinline__ bool inb(int x, int y, int z) const {
    return (unsigned)x < (unsigned)nx && (unsigned)y < (unsigned)ny && (unsigned)z < (unsigned)nz;
  }
  __device__ __forceinline__ int idx(int x, int y, int z) const { return x + nx * (y + ny * z); }
};

#define CELL_PROLOGUE                          \
  int x = blockIdx.x * BX + threadIdx.x;       \
  int y = blockIdx.y * BY + threadIdx.y;       \
  int z = blockIdx.z * BZ + threadIdx.z;       \
  bool in = d.inb(x, y, z);                    \
  int i = in ? d.idx(x, y, z) : 0;             \
  bool fluid = in && __ldg(f + i) != 1u;

// The CG vector kernels run on a 1-D grid capped at 8 blocks per SM; each
// thread strides over the cells, so a reduction adds ~1,200 block sums
// (one per 256 cells would be 32,000 at 8.2 M cells).
struct Cells {
  L3 d;
  FastDiv by_nx, by_plane;
  int n;
  __device__ __forceinline__ void coords(int i, int& x, int& y, int& z) const {
    z = (int)by_plane.div((uint32_t)i);
    const int r = i - z * d.nx * d.ny;
    y = (int)by_nx.div((uint32_t)r);
    x = r - y * d.nx;
  }
};
inline Cells cells_of(Dims3 d) {
  return Cells{L3{d.nx, d.ny, d.nz}, FastDiv((uint32_t)d.nx), FastDiv((uint32_t)(d.nx * d.ny)),
               (int)d.cells()};
}
#define CELL_LOOP(i) \
  for (int i = blockIdx.x * VT + threadIdx.x; i < c.n; i += gridDim.x * VT)

// The thread's cells of the grid-stride loop in order, CG_U at a time: the
// loads of a group (ld(cell, slot)) are all issued before any is used
// (use(cell, slot)), so a thread keeps CG_U cells' loads in flight instead
// of one.  The order of the cells, and so of any per-thread sum, is the
// plain loop's.
constexpr int CG_U = 4;
// k_update_xr holds five values per cell: two cells at a time keep its
// registers (and so its occupancy) lower, measured 0.5-0.8 % faster per
// solve than four.
constexpr int XR_U = 2;
template <int U = CG_U, typename LD, typename USE>
__device__ __forceinline__ void cells_grouped(const Cells& c, LD ld, USE use) {
  const int s = gridDim.x * VT;
  int i = blockIdx.x * VT + threadIdx.x;
  for (; i + (U - 1) * s < c.n; i += U * s) {
#pragma unroll
    for (int u = 0; u < U; u++) ld(i + u * s, u);
#pragma unroll
    for (int u = 0; u < U; u++) use(i + u * s, u);
  }
  for (; i < c.n; i += s) {
    ld(i, 0);
    use(i, 0);
  }
}

// (A v)_i = (sum fluid nbrs v - cnt v_i) / h^2, 0 in solids; evaluated in
// FP64 so residuals near 1e-6 of |b| are not lost to cancellation.  The
// fluid neighbours are added in the order +x, -x, +y, -y, +z, -z and cnt
// counts them and the Dirichlet faces (the top; with bc_mode 0 the sides).
// Two sources of the cells' solidity give the same sums:
//  * FlagMask: u32 solid flags (1 = solid), read at each neighbour (the
//    fixed V-cycle modes and pyro_k_mg_apply, whose masks are not built
//    yet when their residual is taken);
//  * MetaMask: the CG modes' level-0 neighbour masks (bit k = neighbour k
//    inside the grid and fluid, bit 6 = solid), one byte per cell.
struct FlagMask {
  static constexpr bool kLoadFirst = false;  // measured slower with the loads hoisted
  const uint32_t* f;
  __device__ __forceinline__ uint32_t load(int i) const { return __ldg(f + i); }
  __device__ __forceinline__ bool solid(uint32_t raw) const { return raw == 1u; }
  __device__ __forceinline__ double apply(const Cells& c, double ih2, const float* __restrict__ v,
                                         int i, int bc_mode, float vi, uint32_t) const {
    int x, y, z;
    c.coords(i, x, y, z);
    const L3& d = c.d;
    double sum = 0.0, cnt = 0.0;
#pragma unroll
    for (int k = 0; k < 6; k++) {
      int a = x + (k == 0) - (k == 1), b = y + (k == 2) - (k == 3), cz = z + (k == 4) - (k == 5);
      if (b < 0) continue;
      if (!d.inb(a, b, cz)) {
        if (bc_mode == 0 || b >= d.ny) cnt += 1.0;
        continue;
      }
      int j = d.idx(a, b, cz);
      if (__ldg(f + j) == 1u) continue;
      sum += (double)__ldg(v + j);
      cnt += 1.0;
    }
    return (sum - cnt * (double)vi) * ih2;
  }
};
struct MetaMask {
  static constexpr bool kLoadFirst = true;
  const uint8_t* m;
  __device__ __forceinline__ uint32_t load(int i) const { return __ldg(m + i); }
  __device__ __forceinline__ bool solid(uint32_t raw) const { return (raw & 0x40u) != 0; }
  // The six neighbour values are loaded from the cell's coordinates (an
  // in-grid index, the cell itself at the grid's edge) without waiting for
  // the mask, which then selects the ones that are added.
  __device__ __forceinline__ double apply(const Cells& c, double ih2, const float* __restrict__ v,
                                         int i, int bc_mode, float vi, uint32_t mi) const {
    int x, y, z;
    c.coords(i, x, y, z);
    const int nx = c.d.nx, ny = c.d.ny, nz = c.d.nz, sy = nx, sz = nx * ny;
    const float xp = __ldg(v + (x + 1 < nx ? i + 1 : i)), xm = __ldg(v + (x > 0 ? i - 1 : i));
    const float yp = __ldg(v + (y + 1 < ny ? i + sy : i)), ym = __ldg(v + (y > 0 ? i - sy : i));
    const float zp = __ldg(v + (z + 1 < nz ? i + sz : i)), zm = __ldg(v + (z > 0 ? i - sz : i));
    double sum = 0.0;
    if (mi & 1u) sum += (double)xp;
    if (mi & 2u) sum += (double)xm;
    if (mi & 4u) sum += (double)yp;
    if (mi & 8u) sum += (double)ym;
    if (mi & 16u) sum += (double)zp;
    if (mi & 32u) sum += (double)zm;
    int faces = (y == ny - 1);
    if (bc_mode == 0) faces += (x == 0) + (x == nx - 1) + (z == 0) + (z == nz - 1);
    const double cnt = (double)(__popc(mi & 63u) + faces);
    return (sum - cnt * (double)vi) * ih2;
  }
};

// In the kernels below every load of a cell is issued before its mask
// decides what is used (one memory round trip per cell, not two), for the
// mask bytes; with the u32 flags (the fixed V-cycle modes' residual) the
// loads stay behind the flag test, which measured faster there (the 2 cm
// system's V-cycles to their cap: 35.1 ms against 40.2 ms hoisted).
template <typename M>
__global__ void __launch_bounds__(VT) k_resid(Cells c, double ih2, const float* __restrict__ phi,
                                              const float* __restrict__ b, M mk, int bc_mode,
                                              float* __restrict__ r, double* __restrict__ sc) {
  pdl_trigger();
  pdl_wait();
  __shared__ double sh[32];
  double r2 = 0.0, b2 = 0.0;
  CELL_LOOP(i) {
    const uint32_t raw = mk.load(i);
    float bi = 0.0f, pi = 0.0f;
    if constexpr (M::kLoadFirst) {
      bi = __ldg(b + i);
      pi = __ldg(phi + i);
    }
    float ri = 0.0f;
    if (!mk.solid(raw)) {
      if constexpr (!M::kLoadFirst) {
        bi = __ldg(b + i);
        pi = __ldg(phi + i);
      }
      double rd = (double)bi - mk.apply(c, ih2, phi, i, bc_mode, pi, raw);
      ri = (float)rd;
      r2 += rd * rd;
      b2 += (double)bi * (double)bi;
    }
    if (r) r[i] = ri;
  }
  block_add_d(sh, r2, sc, SC_RR);
  block_add_d(sh, b2, sc, SC_BB);
}

template <typename M>
__global__ void __launch_bounds__(VT) k_apply_dot(Cells c, double ih2, const float* __restrict__ p,
                                                  M mk, int bc_mode, float* __restrict__ q,
                                                  double* __restrict__ sc) {
  pdl_trigger();
  pdl_wait();
  __shared__ double sh[32];
  double pq = 0.0;
  CELL_LOOP(i) {
    const uint32_t raw = mk.load(i);
    const float pi = __ldg(p + i);
    float qi = 0.0f;
    if (!mk.solid(raw)) {
      double qd = mk.apply(c, ih2, p, i, bc_mode, pi, raw);
      qi = (float)qd;
      pq += (double)pi * qd;
    }
    q[i] = qi;
  }
  block_add_d(sh, pq, sc, SC_PQ);
}

// q = A p (FP64 evaluation, rounded), 0 in solids.
__global__ void __launch_bounds__(VT) k_apply(Cells c, double ih2, const float* __restrict__ p,
                                              FlagMask mk, int bc_mode, float* __restrict__ q) {
  pdl_trigger();
  pdl_wait();
  CELL_LOOP(i) {
    const uint32_t raw = mk.load(i);
    float qi = 0.0f;
    if (!mk.solid(raw)) qi = (float)mk.apply(c, ih2, p, i, bc_mode, __ldg(p + i), raw);
    q[i] = qi;
  }
}

// phi += alpha p; r -= alpha q; accumulate |r|^2.  phi is ctl->x when
// the argument is null (the CG loop's graph, which serves any solution
// array).
template <typename M>
__global__ void __launch_bounds__(VT) k_update_xr(Cells c, M mk, float* phi_arg,
                                                  float* __restrict__ r,
                                                  const float* __restrict__ p,
                                                  const float* __restrict__ q,
                                                  double* __restrict__ sc,
                                                  const CgCtl* __restrict__ ctl) {
  pdl_trigger();
  pdl_wait();
  __shared__ double sh[32];
  __shared__ float s_alpha;
  if (threadIdx.x == 0) s_alpha = (float)(sc[SC_RZ] / sc[SC_PQ]);
  __syncthreads();
  const float alpha = s_alpha;
  float* __restrict__ phi = phi_arg ? phi_arg : ctl->x;
  double rr = 0.0;
  uint32_t raw[XR_U];
  float pv[XR_U], qv[XR_U], rv[XR_U], xv[XR_U];
  cells_grouped<XR_U>(
      c,
      [&](int i, int u) {
        raw[u] = mk.load(i);
        pv[u] = p[i];
        qv[u] = q[i];
        rv[u] = r[i];
        xv[u] = phi[i];
      },
      [&](int i, int u) {
        if (mk.solid(raw[u])) return;
        phi[i] = xv[u] + alpha * pv[u];
        const float ri = rv[u] - alpha * qv[u];
        r[i] = ri;
        rr += (double)ri * (double)ri;
      });
  block_add_d(sh, rr, sc, SC_RR);
}

// <z,r> -> SC_RZN and, when q is given, <z,q> -> SC_ZQ
template <typename M>
__global__ void __launch_bounds__(VT) k_dots(Cells c, M mk, const float* __restrict__ zv,
                                             const float* __restrict__ r,
                                             const float* __restrict__ q,
                                             double* __restrict__ sc) {
  pdl_trigger();
  pdl_wait();
  __shared__ double sh[32];
  double zr = 0.0, zq = 0.0;
  uint32_t raw[CG_U];
  float zv_[CG_U], rv[CG_U], qv[CG_U];
  cells_grouped(
      c,
      [&](int i, int u) {
        raw[u] = mk.load(i);
        zv_[u] = zv[i];
        rv[u] = r[i];
        qv[u] = q ? q[i] : 0.0f;
      },
      [&](int, int u) {
        if (mk.solid(raw[u])) return;
        zr += (double)zv_[u] * (double)rv[u];
        if (q) zq += (double)zv_[u] * (double)qv[u];
      });
  block_add_d(sh, zr, sc, SC_RZN);
  if (q) block_add_d(sh, zq, sc, SC_ZQ);
}

// p = z + beta p with beta = -<z,q>/<p,q>; p = z when ctl->first is set
// (the first iteration after a start or restart)
template <typename M>
__global__ void __launch_bounds__(VT) k_update_p(Cells c, M mk, float* __restrict__ p,
                                                 const float* __restrict__ zv,
                                                 const double* __restrict__ sc,
                                                 const CgCtl* __restrict__ ctl) {
  pdl_trigger();
  pdl_wait();
  __shared__ float s_beta;
  __shared__ int s_first;
  if (threadIdx.x == 0) {
    s_first = ctl->first;
    s_beta = s_first ? 0.0f : (float)(-sc[SC_ZQ] / sc[SC_PQ]);
  }
  __syncthreads();
  const float beta = s_beta;
  const bool first = s_first != 0;
  uint32_t raw[CG_U];
  float zv_[CG_U], pv[CG_U];
  cells_grouped(
      c,
      [&](int i, int u) {
        raw[u] = mk.load(i);
        zv_[u] = zv[i];
        pv[u] = first ? 0.0f : p[i];
      },
      [&](int i, int u) { p[i] = mk.solid(raw[u]) ? 0.0f : (first ? zv_[u] : zv_[u] + beta * pv[u]); });
}

// End of one CG iteration on the device: count it and let the loop's
// conditional node run another unless |r| / |b| <= tol, the count reached
// max_it, or the iteration stalled (|r|^2 not finite, <p, A p> = 0).  The
// count rises by one per iteration and the cap is a host-checked int, so
// the loop always ends.
__global__ void k_cg_check(CgCtl* __restrict__ ctl, const double* __restrict__ sc,
                           cudaGraphConditionalHandle h) {
  pdl_trigger();
  pdl_wait();
  const double rr = sc[SC_RR], pq = sc[SC_PQ];
  const int it = ctl->it + 1;
  const bool stalled = !(rr >= 0.0) || !(pq < 0.0 || pq > 0.0);
  const bool conv = ctl->bb2 > 0.0 && sqrt(rr / ctl->bb2) <= ctl->tol;
  ctl->it = it;
  ctl->rr = rr;
  ctl->first = 0;
  ctl->stalled = stalled ? 1 : 0;
  cudaGraphSetConditional(h, (!stalled && !conv && it < ctl->max_it) ? 1u : 0u);
}

__global__ void k_roll(double* sc) {
  pdl_trigger();
  pdl_wait();
  // rz <- rz_new, clear the accumulators of the next iteration
  sc[SC_RZ] = sc[SC_RZN];
  sc[SC_RZN] = 0.0;
  sc[SC_ZQ] = 0.0;
  sc[SC_PQ] = 0.0;
  sc[SC_RR] = 0.0;
}

// ---- cells the CG modes solve for ----------------------------------------
// A fluid region sealed by solids with no Dirichlet face makes A singular
// (its b need not sum to zero).  The CG modes solve only for fluid cells
// connected through fluid faces to a Dirichlet face; the others keep their
// initial phi and are treated as solid.  fa = 0 reached fluid, 1 solid or
// unreached fluid; 2 marks fluid not reached yet while propagating.

// order-independent 64-bit hash of the flag field
__global__ void __launch_bounds__(256) k_flag_hash(L3 d, const uint32_t* __restrict__ f,
                                                   unsigned long long* out) {
  CELL_PROLOGUE
  (void)fluid;
  unsigned long long h = 0;
  if (in && __ldg(f + i) == 1u) {
    unsigned long long k = (unsigned long long)i * 0x9E3779B97F4A7C15ull + 0x632BE59BD9B4E019ull;
    k ^= k >> 29;
    k *= 0xBF58476D1CE4E5B9ull;
    h = k ^ (k >> 32);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) h += __shfl_xor_sync(0xffffffffu, h, o);
  if ((threadIdx.x & 31) == 0 && h) atomicAdd(out, h);
}

__global__ void __launch_bounds__(256) k_reach_init(L3 d, const uint32_t* __restrict__ f,
                                                    int bc_mode, uint32_t* __restrict__ fa) {
  CELL_PROLOGUE
  if (!in) return;
  if (!fluid) {
    fa[i] = 1u;
    return;
  }
  bool seed = y == d.ny - 1 ||
              (bc_mode == 0 && (x == 0 || x == d.nx - 1 || z == 0 || z == d.nz - 1));
  fa[i] = seed ? 0u : 2u;
}

// One 8x8x8 tile per block: propagate "reached" (0) into fluid (2) cells
// through fluid faces until the tile stops changing (halo values read from
// global memory), then write back; *changed is set when a cell was reached.
constexpr int RT = 8;
__global__ void __launch_bounds__(RT * RT * RT) k_reach_tile(L3 d, uint32_t* __restrict__ fa,
                                                             int* __restrict__ changed) {
  __shared__ uint8_t t[RT + 2][RT + 2][RT + 2];
  const int lx = threadIdx.x % RT, ly = (threadIdx.x / RT) % RT, lz = threadIdx.x / (RT * RT);
  const int bx = blockIdx.x * RT, by = blockIdx.y * RT, bz = blockIdx.z * RT;
  for (int k = threadIdx.x; k < (RT + 2) * (RT + 2) * (RT + 2); k += RT * RT * RT) {
    int hx = k % (RT + 2), hy = (k / (RT + 2)) % (RT + 2), hz = k / ((RT + 2) * (RT + 2));
    int gx = bx + hx - 1, gy = by + hy - 1, gz = bz + hz - 1;
    t[hz][hy][hx] = d.inb(gx, gy, gz) ? (uint8_t)fa[d.idx(gx, gy, gz)] : (uint8_t)1;
  }
  __syncthreads();
  const int x = bx + lx, y = by + ly, z = bz + lz;
  const bool mine = d.inb(x, y, z) && t[lz + 1][ly + 1][lx + 1] == 2;
  bool got = false;
  for (int it = 0; it < RT * RT * RT; it++) {
    bool ch = false;
    if (mine && !got) {
      const int cx = lx + 1, cy = ly + 1, cz = lz + 1;
      if (t[cz][cy][cx - 1] == 0 || t[cz][cy][cx + 1] == 0 || t[cz][cy - 1][cx] == 0 ||
          t[cz][cy + 1][cx] == 0 || t[cz - 1][cy][cx] == 0 || t[cz + 1][cy][cx] == 0) {
        t[cz][cy][cx] = 0;
        got = true;
        ch = true;
      }
    }
    if (!__syncthreads_or(ch)) break;
  }
  if (got) {
    fa[d.idx(x, y, z)] = 0u;
    *changed = 1;
  }
}

__global__ void __launch_bounds__(256) k_reach_final(L3 d, uint32_t* __restrict__ fa) {
  int x = blockIdx.x * BX + threadIdx.x, y = blockIdx.y * BY + threadIdx.y,
      z = blockIdx.z * BZ + threadIdx.z;
  if (!d.inb(x, y, z)) return;
  int i = d.idx(x, y, z);
  if (fa[i] == 2u) fa[i] = 1u;
}

}  // namespace

// ---- coarsest level of the preconditioner: FP64 direct solve --------------
// The preconditioner's hierarchy halves the grid until its coarsest level
// has at most DIRECT_MAX cells (Multigrid deep rule).  That level is solved
// exactly: M = -A (symmetric positive definite on the fluid cells, the
// identity on solid ones) is assembled densely in FP64 and inverted in
// place by Gauss-Jordan elimination without pivoting (stable for SPD
// matrices), one pivot per step: with p = m_kk,
//   m_kk <- 1/p,  m_kj <- m_kj/p,  m_ik <- -m_ik/p,  m_ij <- m_ij - m_ik m_kj/p.
// The inverse is kept until the level's flags change; each application is
// one FP64 matrix-vector product, phi = -M^-1 b.  A pivot that is not
// positive (a fluid region with no Dirichlet face, which the CG modes'
// reachability flags exclude) is replaced by the cell's h^-2, as if the cell
// touched a Dirichlet face, and counted.
namespace {

__global__ void __launch_bounds__(256) k_dc_assemble(L3 d, double ih2,
                                                     const uint32_t* __restrict__ f, int bc_mode,
                                                     double* __restrict__ M) {
  const int n = d.nx * d.ny * d.nz;
  const int i = blockIdx.x * 256 + threadIdx.x;
  if (i >= n) return;
  const int x = i % d.nx, y = (i / d.nx) % d.ny, z = i / (d.nx * d.ny);
  double* row = M + (size_t)i * n;
  if (f[i] == 1u) {
    row[i] = 1.0;
    return;
  }
  double cnt = 0.0;
#pragma unroll
  for (int k = 0; k < 6; k++) {
    int a = x + (k == 0) - (k == 1), b = y + (k == 2) - (k == 3), c = z + (k == 4) - (k == 5);
    if (b < 0) continue;
    if (!d.inb(a, b, c)) {
      if (bc_mode == 0 || b >= d.ny) cnt += 1.0;
      continue;
    }
    const int j = d.idx(a, b, c);
    if (f[j] == 1u) continue;
    row[j] = -ih2;
    cnt += 1.0;
  }
  row[i] = cnt * ih2;
}

// The pivot row and column of step k (the matrix as the previous step left
// it), with the pivot itself checked.
__global__ void k_dc_pivot(double* __restrict__ M, int n, int k, double ih2,
                           double* __restrict__ col, double* __restrict__ row,
                           int* __restrict__ bad) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    col[t] = M[(size_t)t * n + k];
    double r = M[(size_t)k * n + t];
    if (t == k && !(r > 1e-9 * ih2)) {
      r = ih2;
      atomicAdd(bad, 1);
    }
    row[t] = r;
  }
}

__global__ void __launch_bounds__(256) k_dc_eliminate(double* __restrict__ M, int n, int k,
                                                      const double* __restrict__ col,
                                                      const double* __restrict__ row) {
  const int j = blockIdx.x * 32 + threadIdx.x;
  const int i = blockIdx.y * 8 + threadIdx.y;
  if (i >= n || j >= n) return;
  const double ip = 1.0 / row[k];
  double* m = M + (size_t)i * n + j;
  if (i == k) *m = (j == k) ? ip : row[j] * ip;
  else if (j == k) *m = -col[i] * ip;
  else *m = *m - col[i] * row[j] * ip;
}

// phi_i = -(M^-1 b)_i on fluid cells, 0 on solid ones: one warp per row,
// b staged in shared memory as FP64 (solid entries 0).
template <typename TS>
__global__ void __launch_bounds__(256) k_dc_apply(const double* __restrict__ Minv, int n,
                                                  const TS* __restrict__ b,
                                                  const uint32_t* __restrict__ f,
                                                  TS* __restrict__ phi) {
  extern __shared__ double sb[];
  pdl_trigger();
  pdl_wait();
  for (int t = threadIdx.x; t < n; t += blockDim.x)
    sb[t] = f[t] == 1u ? 0.0 : (double)cvt_load(b + t);
  __syncthreads();
  const int i = blockIdx.x * 8 + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (i >= n) return;
  const double* r = Minv + (size_t)i * n;
  double acc = 0.0;
  for (int j = lane; j < n; j += 32) acc += r[j] * sb[j];
  acc = warp_sum_d(acc);
  if (lane == 0) cvt_store(phi + i, f[i] == 1u ? 0.0f : (float)(-acc));
}

}  // namespace

struct DirectSolve : CoarseDirect {
  Dims3 dc{};
  float h = 1.0f;
  int bc_mode = 0;
  const uint32_t* f = nullptr;  // the level's flags (device, owned by the hierarchy)
  DevBuf minv, piv, bad;
  std::vector<uint32_t> flags_host, flags_now;
  bool valid = false;
  int singular = 0;  // pivots replaced at the last factorisation

  size_t n() const { return dc.cells(); }
  // Factor when the level's flags differ from those of the last
  // factorisation (they are compared on the host after a copy).
  int refresh(cudaStream_t st) {
    const size_t nn = n();
    if (!minv.p) {
      int rc;
      if ((rc = minv.alloc(nn * nn * 8)) != PYRO_OK || (rc = piv.alloc(nn * 16)) != PYRO_OK ||
          (rc = bad.alloc(16)) != PYRO_OK)
        return rc;
    }
    flags_now.resize(nn);
    PYRO_CU(cudaMemcpyAsync(flags_now.data(), f, nn * 4, cudaMemcpyDeviceToHost, st));
    PYRO_CU(cudaStreamSynchronize(st));
    if (valid && flags_now == flags_host) return PYRO_OK;
    const double ih2 = 1.0 / ((double)h * h);
    L3 l{dc.nx, dc.ny, dc.nz};
    PYRO_CU(cudaMemsetAsync(minv.p, 0, nn * nn * 8, st));
    PYRO_CU(cudaMemsetAsync(bad.p, 0, 4, st));
    k_dc_assemble<<<(unsigned)((nn + 255) / 256), 256, 0, st>>>(l, ih2, f, bc_mode,
                                                                minv.as<double>());
    PYRO_CU(cudaGetLastError());
    double* col = piv.as<double>();
    double* row = col + nn;
    dim3 eg((unsigned)((nn + 31) / 32), (unsigned)((nn + 7) / 8));
    for (size_t k = 0; k < nn; k++) {
      k_dc_pivot<<<(unsigned)((nn + 255) / 256), 256, 0, st>>>(minv.as<double>(), (int)nn, (int)k,
                                                                ih2, col, row, bad.as<int>());
      k_dc_eliminate<<<eg, dim3(32, 8), 0, st>>>(minv.as<double>(), (int)nn, (int)k, col, row);
    }
    PYRO_CU(cudaGetLastError());
    PYRO_CU(cudaMemcpyAsync(&singular, bad.p, 4, cudaMemcpyDeviceToHost, st));
    PYRO_CU(cudaStreamSynchronize(st));
    flags_host = flags_now;
    valid = true;
    return PYRO_OK;
  }
  cudaError_t apply(cudaStream_t st, const void* b, void* phi, bool bf16) override {
    const size_t nn = n();
    const unsigned blocks = (unsigned)((nn + 7) / 8);
    if (bf16)
      return launch_pdl(k_dc_apply<__nv_bfloat16>, dim3(blocks), dim3(256), nn * 8, st,
                        (const double*)minv.as<double>(), (int)nn, (const __nv_bfloat16*)b, f,
                        (__nv_bfloat16*)phi);
    return launch_pdl(k_dc_apply<float>, dim3(blocks), dim3(256), nn * 8, st,
                      (const double*)minv.as<double>(), (int)nn, (const float*)b, f, (float*)phi);
  }
};

int Solver::update_reach(cudaStream_t st, unsigned long long h) {
  const uint32_t* f0 = mg->f[0];
  L3 l{d.nx, d.ny, d.nz};
  unsigned long long* H = reach_dev.as<unsigned long long>();
  k_reach_init<<<grid_for(d), dim3(BX, BY, BZ), 0, st>>>(l, f0, mg->bc_mode, fa.as<uint32_t>());
  PYRO_CU(cudaGetLastError());
  dim3 tg((unsigned)((d.nx + RT - 1) / RT), (unsigned)((d.ny + RT - 1) / RT),
          (unsigned)((d.nz + RT - 1) / RT));
  int* C = reinterpret_cast<int*>(H + 1);
  // every launch reaches at least one more tile along each front; the
  // number of launches is bounded by the tile count
  const long max_rounds = (long)tg.x * tg.y * tg.z + 8;
  bool done = false;
  for (long r = 0; r < max_rounds && !done; r += 4) {
    PYRO_CU(cudaMemsetAsync(C, 0, 4, st));
    for (int k = 0; k < 4; k++) k_reach_tile<<<tg, RT * RT * RT, 0, st>>>(l, fa.as<uint32_t>(), C);
    PYRO_CU(cudaGetLastError());
    int c = 0;
    PYRO_CU(cudaMemcpyAsync(host_sc, C, 4, cudaMemcpyDeviceToHost, st));
    PYRO_CU(cudaStreamSynchronize(st));
    std::memcpy(&c, host_sc, 4);
    done = c == 0;
  }
  k_reach_final<<<grid_for(d), dim3(BX, BY, BZ), 0, st>>>(l, fa.as<uint32_t>());
  PYRO_CU(cudaGetLastError());
  reach_hash = h;
  reach_flags = f0;
  reach_valid = true;
  return PYRO_OK;
}

int Solver::begin_cg(cudaStream_t st, float* phi, const float* b) {
  const uint32_t* f0 = mg->f[0];
  L3 l{d.nx, d.ny, d.nz};
  const double ih2 = 1.0 / ((double)mg->h[0] * mg->h[0]);
  double* S = sc.as<double>();
  int rc;
  if (!fa.p) {
    if ((rc = fa.alloc(d.cells() * 4)) != PYRO_OK || (rc = reach_dev.alloc(16)) != PYRO_OK)
      return rc;
  }
  auto resid = [&]() -> cudaError_t {
    cudaError_t e = cudaMemsetAsync(sc.p, 0, SC_N * 8, st);
    if (e == cudaSuccess)
      e = launch_pdl(k_resid<MetaMask>, dim3(vec_blocks(d.cells())), dim3(VT), 0, st,
                     cells_of(d), ih2, (const float*)phi, b, MetaMask{pc.meta[0].as<uint8_t>()},
                     mg->bc_mode, r.as<float>(), S);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(host_sc, sc.p, SC_N * 8, cudaMemcpyDeviceToHost, st);
    return e;
  };
  // The hash of the flag field and, when the last solve's reachable set
  // and levels are still in place, the residual on them: one round trip.
  unsigned long long* H = reach_dev.as<unsigned long long>();
  PYRO_CU(cudaMemsetAsync(H, 0, 16, st));
  k_flag_hash<<<grid_for(d), dim3(BX, BY, BZ), 0, st>>>(l, f0, H);
  PYRO_CU(cudaGetLastError());
  const bool spec = reach_valid && reach_flags == f0 && pc_ready;
  if (spec) PYRO_CU(resid());
  PYRO_CU(cudaMemcpyAsync(host_sc + SC_N, H, 8, cudaMemcpyDeviceToHost, st));
  PYRO_CU(cudaStreamSynchronize(st));
  unsigned long long h;
  std::memcpy(&h, host_sc + SC_N, 8);
  if (spec && h == reach_hash) return PYRO_OK;
  // the flags changed (or first solve): reachable set, the
  // preconditioner's level flags and masks, its coarsest-level inverse
  pc_ready = false;
  if ((rc = update_reach(st, h)) != PYRO_OK) return rc;
  pc.bind_level0(z.as<float>(), r.as<float>(), fa.as<uint32_t>());
  PYRO_CU(pc.prepare_sym(st));
  if (direct) {
    direct->f = pc.f.back();  // level 0's flags when the grid is the coarsest level
    if ((rc = direct->refresh(st)) != PYRO_OK) return rc;
  }
  pc_ready = true;
  PYRO_CU(resid());
  PYRO_CU(cudaStreamSynchronize(st));
  return PYRO_OK;
}

int Solver::alloc_bf16_levels() {
  for (size_t l = 0; l < bphi.size(); l++) {
    const size_t need = pc.dims[l].cells() * 2;
    int rc;
    if (bphi[l].bytes != need &&
        ((rc = bphi[l].alloc(need)) != PYRO_OK || (rc = bphi2[l].alloc(need)) != PYRO_OK ||
         (rc = bb[l].alloc(need)) != PYRO_OK))
      return rc;
  }
  return PYRO_OK;
}

int Solver::cg_loop(cudaStream_t st, float* phi, bool bf16, double bb2, float tol, int it0,
                    int max_it) {
  cudaGraphExec_t& exec = cg_exec[bf16 ? 1 : 0];
  if (!exec) {
    const MetaMask mk{pc.meta[0].as<uint8_t>()};
    const double ih2 = 1.0 / ((double)mg->h[0] * mg->h[0]);
    double* S = sc.as<double>();
    CgCtl* C = ctl.as<CgCtl>();
    // the BF16 levels exist before their addresses are captured
    int rc;
    if (bf16 && (rc = alloc_bf16_levels()) != PYRO_OK) return rc;
    cudaGraph_t g = nullptr;
    PYRO_CU(cudaGraphCreate(&g, 0));
    struct Own {
      cudaGraph_t g;
      ~Own() { cudaGraphDestroy(g); }
    } own{g};
    cudaGraphConditionalHandle hc;
    PYRO_CU(cudaGraphConditionalHandleCreate(&hc, g, 1, cudaGraphCondAssignDefault));
    cudaGraphNodeParams np = {};
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = hc;
    np.conditional.type = cudaGraphCondTypeWhile;
    np.conditional.size = 1;
    cudaGraphNode_t node;
    PYRO_CU(cudaGraphAddNode(&node, g, nullptr, 0, &np));
    cudaGraph_t body = np.conditional.phGraph_out[0];
    // one iteration: z = V(r); <z,r>, <z,q>; p = z + beta p; roll the
    // scalars; q = A p, <p,q>; phi += alpha p, r -= alpha q, |r|^2; check
    PYRO_CU(cudaStreamBeginCaptureToGraph(cap_st, body, nullptr, nullptr, 0,
                                          cudaStreamCaptureModeRelaxed));
    const dim3 vb(vec_blocks(d.cells())), vt(VT);
    cudaError_t e = precond(cap_st, bf16, false);
    if (e == cudaSuccess)
      e = launch_pdl(k_dots<MetaMask>, vb, vt, 0, cap_st, cells_of(d), mk,
                     (const float*)z.as<float>(), (const float*)r.as<float>(),
                     (const float*)q.as<float>(), S);
    if (e == cudaSuccess)
      e = launch_pdl(k_update_p<MetaMask>, vb, vt, 0, cap_st, cells_of(d), mk, p.as<float>(),
                     (const float*)z.as<float>(), (const double*)S, (const CgCtl*)C);
    if (e == cudaSuccess) e = launch_pdl(k_roll, dim3(1), dim3(1), 0, cap_st, S);
    if (e == cudaSuccess)
      e = launch_pdl(k_apply_dot<MetaMask>, vb, vt, 0, cap_st, cells_of(d), ih2,
                     (const float*)p.as<float>(), mk, mg->bc_mode, q.as<float>(), S);
    if (e == cudaSuccess)
      e = launch_pdl(k_update_xr<MetaMask>, vb, vt, 0, cap_st, cells_of(d), mk, (float*)nullptr,
                     r.as<float>(), (const float*)p.as<float>(), (const float*)q.as<float>(), S,
                     (const CgCtl*)C);
    if (e == cudaSuccess)
      e = launch_pdl(k_cg_check, dim3(1), dim3(1), 0, cap_st, C, (const double*)S, hc);
    cudaGraph_t out = nullptr;
    const cudaError_t ec = cudaStreamEndCapture(cap_st, &out);
    PYRO_CU(e);
    PYRO_CU(ec);
    PYRO_CU(cudaGraphInstantiate(&exec, g, 0));
  }
  host_ctl->x = phi;
  host_ctl->bb2 = bb2;
  host_ctl->tol = (double)tol;
  host_ctl->rr = 0.0;
  host_ctl->it = it0;
  host_ctl->max_it = max_it;
  host_ctl->first = 1;
  host_ctl->stalled = 0;
  PYRO_CU(cudaMemcpyAsync(ctl.p, host_ctl, sizeof(CgCtl), cudaMemcpyHostToDevice, st));
  PYRO_CU(cudaGraphLaunch(exec, st));
  return PYRO_OK;
}

int Solver::init(Multigrid* m) {
  mg = m;
  d = m->dims[0];
  size_t n = d.cells();
  int rc;
  if ((rc = r.alloc(n * 4)) != PYRO_OK) return rc;
  if ((rc = z.alloc(n * 4)) != PYRO_OK) return rc;
  if ((rc = p.alloc(n * 4)) != PYRO_OK) return rc;
  if ((rc = q.alloc(n * 4)) != PYRO_OK) return rc;
  if ((rc = sc.alloc(SC_BYTES)) != PYRO_OK) return rc;
  PYRO_CU(cudaMemset(sc.p, 0, SC_BYTES));  // the reductions' counters start at 0
  if ((rc = ctl.alloc(sizeof(CgCtl))) != PYRO_OK) return rc;
  // the scalars and one 8-byte word (the flag hash)
  if (cudaMallocHost(&host_sc, (SC_N + 1) * 8) != cudaSuccess ||
      cudaMallocHost(&host_ctl, sizeof(CgCtl)) != cudaSuccess) {
    set_error("solver: pinned allocation failed");
    return PYRO_E_NOMEM;
  }
  // q is read (and its products discarded) by the first iteration's dots;
  // the clears run on the default stream, which the solve's non-blocking
  // stream does not wait for, so they finish here (a reduction counter
  // cleared while the first solve already counts would stay offset)
  PYRO_CU(cudaMemset(q.p, 0, n * 4));
  PYRO_CU(cudaStreamSynchronize(0));
  PYRO_CU(cudaStreamCreateWithFlags(&cap_st, cudaStreamNonBlocking));
  if (cudaEventCreate(&ev0) != cudaSuccess || cudaEventCreate(&ev1) != cudaSuccess ||
      cudaEventCreate(&evl0) != cudaSuccess || cudaEventCreate(&evl1) != cudaSuccess) {
    set_error("solver: cudaEventCreate failed");
    return PYRO_E_CUDA;
  }
  // the preconditioner's hierarchy: down to <= DIRECT_MAX cells, solved
  // directly when the coarsest level got there
  if ((rc = pc.init(d, m->h[0], m->bc_mode, DIRECT_MAX)) != PYRO_OK) return rc;
  const size_t L = pc.levels();
  bphi.resize(L);
  bphi2.resize(L);
  bb.resize(L);
  if (pc.dims.back().cells() <= DIRECT_MAX) {
    direct = new (std::nothrow) DirectSolve();
    if (!direct) {
      set_error("solver: host allocation failed");
      return PYRO_E_NOMEM;
    }
    direct->dc = pc.dims.back();
    direct->h = pc.h.back();
    direct->bc_mode = pc.bc_mode;
    direct->f = pc.f.back();
    pc.direct = direct;
  }
  return PYRO_OK;
}

Solver::~Solver() {
  for (cudaGraphExec_t x : cg_exec)
    if (x) cudaGraphExecDestroy(x);
  if (cap_st) cudaStreamDestroy(cap_st);
  delete direct;
  if (host_sc) cudaFreeHost(host_sc);
  if (host_ctl) cudaFreeHost(host_ctl);
  if (ev0) cudaEventDestroy(ev0);
  if (ev1) cudaEventDestroy(ev1);
  if (evl0) cudaEventDestroy(evl0);
  if (evl1) cudaEventDestroy(evl1);
}

size_t Solver::device_bytes() const {
  size_t s = r.bytes + z.bytes + p.bytes + q.bytes + sc.bytes + ctl.bytes + fa.bytes +
             reach_dev.bytes;
  for (size_t l = 0; l < bphi.size(); l++) s += bphi[l].bytes + bphi2[l].bytes + bb[l].bytes;
  s += pc.device_bytes();
  if (direct) s += direct->minv.bytes + direct->piv.bytes + direct->bad.bytes;
  return s;
}

int Solver::true_resid(cudaStream_t st, const float* phi, const float* b, double* rel,
                       double* bn, bool cg) {
  PYRO_CU(cudaMemsetAsync(sc.p, 0, SC_N * 8, st));
  const dim3 vb(vec_blocks(d.cells())), vt(VT);
  const double ih2 = 1.0 / ((double)mg->h[0] * mg->h[0]);
  float* none = nullptr;
  if (cg)
    launch_pdl(k_resid<MetaMask>, vb, vt, 0, st, cells_of(d), ih2, phi, b,
               MetaMask{pc.meta[0].as<uint8_t>()}, mg->bc_mode, none, sc.as<double>());
  else
    launch_pdl(k_resid<FlagMask>, vb, vt, 0, st, cells_of(d), ih2, phi, b,
               FlagMask{mg->f[0]}, mg->bc_mode, none, sc.as<double>());
  PYRO_CU(cudaGetLastError());
  PYRO_CU(cudaMemcpyAsync(host_sc, sc.p, SC_N * 8, cudaMemcpyDeviceToHost, st));
  PYRO_CU(cudaStreamSynchronize(st));
  double bb2 = host_sc[SC_BB];
  *bn = std::sqrt(bb2);
  *rel = bb2 > 0 ? std::sqrt(host_sc[SC_RR] / bb2) : 0.0;
  return PYRO_OK;
}

cudaError_t Solver::precond(cudaStream_t st, bool bf16, bool prep) {
  // z = V(r): one V-cycle from a zero initial guess (it writes every cell
  // of z and does not read it).
  pc.bind_level0(z.as<float>(), r.as<float>(), fa.as<uint32_t>());
  return bf16 ? pc.vcycle_sym(st, bphi.data(), bphi2.data(), bb.data(), prep)
              : pc.vcycle_sym(st, nullptr, nullptr, nullptr, prep);
}

int Solver::learned_stage(cudaStream_t st, float* phi, double* rr, PyroSolveInfo* info) {
  const uint32_t* f0 = mg->f[0];
  const double ih2 = 1.0 / ((double)mg->h[0] * mg->h[0]);
  double* S = sc.as<double>();
  PYRO_CU(cudaEventRecord(evl0, st));
  // e = net(r) into z, q = A e
  NetVol v{d.nx, d.ny, d.nz, 1};
  int rc;
  if ((rc = net->ensure(v, false)) || (rc = net->forward(r.as<float>(), f0, v, st)) ||
      (rc = net->output(f0, mg->h[0], z.as<float>(), v, st)) || (rc = net->check_err(st)))
    return rc;
  PYRO_CU(cudaMemsetAsync(sc.p, 0, SC_N * 8, st));
  const MetaMask mk{pc.meta[0].as<uint8_t>()};
  const dim3 vb(vec_blocks(d.cells())), vt(VT);
  launch_pdl(k_apply_dot<MetaMask>, vb, vt, 0, st, cells_of(d), ih2, (const float*)z.as<float>(),
             mk, mg->bc_mode, q.as<float>(), S);
  launch_pdl(k_dots<MetaMask>, vb, vt, 0, st, cells_of(d), mk, (const float*)z.as<float>(),
             (const float*)r.as<float>(), (const float*)nullptr, S);
  PYRO_CU(cudaGetLastError());
  PYRO_CU(cudaMemcpyAsync(host_sc, sc.p, SC_N * 8, cudaMemcpyDeviceToHost, st));
  PYRO_CU(cudaStreamSynchronize(st));
  const double re = host_sc[SC_RZN], eae = host_sc[SC_PQ];
  // <Ae, r>, <Ae, Ae>
  PYRO_CU(cudaMemsetAsync(sc.p, 0, SC_N * 8, st));
  launch_pdl(k_dots<MetaMask>, vb, vt, 0, st, cells_of(d), mk, (const float*)q.as<float>(),
             (const float*)r.as<float>(), (const float*)q.as<float>(), S);
  PYRO_CU(cudaGetLastError());
  PYRO_CU(cudaMemcpyAsync(host_sc, sc.p, SC_N * 8, cudaMemcpyDeviceToHost, st));
  PYRO_CU(cudaStreamSynchronize(st));
  const double rae = host_sc[SC_RZN], aeae = host_sc[SC_ZQ];
  double alpha = 0.0, rr_new = *rr;
  const int keep = pyro_learned_accept(re, eae, rae, aeae, *rr, &alpha, &rr_new);
  if (keep) {
    // phi += alpha e, r -= alpha A e with alpha = S[RZ] / S[PQ]
    std::memset(host_sc, 0, SC_N * 8);
    host_sc[SC_RZ] = re;
    host_sc[SC_PQ] = eae;
    PYRO_CU(cudaMemcpyAsync(sc.p, host_sc, SC_N * 8, cudaMemcpyHostToDevice, st));
    launch_pdl(k_update_xr<MetaMask>, vb, vt, 0, st, cells_of(d), mk, phi, r.as<float>(),
               (const float*)z.as<float>(), (const float*)q.as<float>(), S,
               (const CgCtl*)nullptr);
    PYRO_CU(cudaGetLastError());
    PYRO_CU(cudaMemcpyAsync(host_sc, sc.p, SC_N * 8, cudaMemcpyDeviceToHost, st));
  }
  PYRO_CU(cudaEventRecord(evl1, st));
  PYRO_CU(cudaEventSynchronize(evl1));
  if (keep) *rr = host_sc[SC_RR];
  // the CG accumulators start from zero (a discarded correction may have
  // left NaN in them)
  PYRO_CU(cudaMemsetAsync(sc.p, 0, SC_N * 8, st));
  float ms = 0.0f;
  PYRO_CU(cudaEventElapsedTime(&ms, evl0, evl1));
  info->learned = keep;
  info->learned_ms = ms;
  return PYRO_OK;
}

int Solver::profile_cg(cudaStream_t st, float* phi, const float* b, bool bf16, int iters,
                       float* ms, int* launches) {
  int rc;
  if ((rc = begin_cg(st, phi, b)) != PYRO_OK) return rc;
  float* save_phi = mg->phi[0];
  float* save_b = mg->b[0];
  const uint32_t* save_f0 = mg->f[0];
  mg->bind_level0(save_phi, save_b, fa.as<uint32_t>());
  struct Rebind {
    Multigrid* m;
    float* p;
    float* b;
    const uint32_t* f;
    ~Rebind() { m->bind_level0(p, b, f); }
  } rebind{mg, save_phi, save_b, save_f0};
  // the BF16 levels exist before the first event
  if (bf16 && (rc = alloc_bf16_levels()) != PYRO_OK) return rc;
  const MetaMask mk{pc.meta[0].as<uint8_t>()};
  const double ih2 = 1.0 / ((double)mg->h[0] * mg->h[0]);
  double* S = sc.as<double>();
  CgCtl* C = ctl.as<CgCtl>();
  const dim3 vb(vec_blocks(d.cells())), vt(VT);
  std::memset(host_ctl, 0, sizeof(CgCtl));
  host_ctl->x = phi;
  host_ctl->first = 1;
  PYRO_CU(cudaMemcpyAsync(ctl.p, host_ctl, sizeof(CgCtl), cudaMemcpyHostToDevice, st));
  MgTimer timer;
  PYRO_CU(timer.start(st));
  pc.timer = &timer;
  struct Untime {
    Multigrid* m;
    ~Untime() { m->timer = nullptr; }
  } untime{&pc};
  auto tick = [&]() { return timer.mark(MG_CG_VECTOR, st); };
  for (int it = 0; it < iters; it++) {
    PYRO_CU(precond(st, bf16, false));
    PYRO_CU(launch_pdl(k_dots<MetaMask>, vb, vt, 0, st, cells_of(d), mk,
                       (const float*)z.as<float>(), (const float*)r.as<float>(),
                       (const float*)q.as<float>(), S));
    PYRO_CU(tick());
    PYRO_CU(launch_pdl(k_update_p<MetaMask>, vb, vt, 0, st, cells_of(d), mk, p.as<float>(),
                       (const float*)z.as<float>(), (const double*)S, (const CgCtl*)C));
    if (it == 0) PYRO_CU(cudaMemsetAsync(&C->first, 0, sizeof(int), st));
    PYRO_CU(tick());
    PYRO_CU(launch_pdl(k_roll, dim3(1), dim3(1), 0, st, S));
    PYRO_CU(tick());
    PYRO_CU(launch_pdl(k_apply_dot<MetaMask>, vb, vt, 0, st, cells_of(d), ih2,
                       (const float*)p.as<float>(), mk, mg->bc_mode, q.as<float>(), S));
    PYRO_CU(tick());
    PYRO_CU(launch_pdl(k_update_xr<MetaMask>, vb, vt, 0, st, cells_of(d), mk, (float*)nullptr,
                       r.as<float>(), (const float*)p.as<float>(), (const float*)q.as<float>(),
                       S, (const CgCtl*)C));
    PYRO_CU(tick());
  }
  PYRO_CU(cudaStreamSynchronize(st));
  PYRO_CU(timer.read(ms, launches));
  return PYRO_OK;
}

int Solver::solve(cudaStream_t st, float* phi, const float* b, int mode, float tol,
                  int max_iters, PyroSolveInfo* info) {
  PYRO_REQUIRE(mode >= PYRO_SOLVER_VCYCLE && mode <= PYRO_SOLVER_MGPCG_LEARNED,
               "solve: unknown mode");
  PYRO_REQUIRE(max_iters > 0, "solve: max_iters must be positive");
  PYRO_REQUIRE(mode != PYRO_SOLVER_MGPCG_LEARNED || net,
               "solve: the learned mode needs a network (set_net)");
  std::memset(info, 0, sizeof(*info));
  info->mode = mode;
  info->learned = -1;
  float* save_phi = mg->phi[0];
  float* save_b = mg->b[0];
  const uint32_t* save_f0 = mg->f[0];
  const uint32_t* f0 = save_f0;
  PYRO_CU(cudaEventRecord(ev0, st));
  int iters = 0;
  double rel = 0, bn = 0;
  int rc = PYRO_OK;
  const double ih2 = 1.0 / ((double)mg->h[0] * mg->h[0]);
  if (mode == PYRO_SOLVER_VCYCLE || mode == PYRO_SOLVER_VCYCLE_TOL) {
    mg->bind_level0(phi, b, f0);
    if (mode == PYRO_SOLVER_VCYCLE) {
      cudaError_t e = mg->vcycles(max_iters, st);
      mg->bind_level0(save_phi, save_b, f0);
      PYRO_CU(e);
      iters = max_iters;
      if ((rc = true_resid(st, phi, b, &rel, &bn, false)) != PYRO_OK) return rc;
    } else {
      if ((rc = true_resid(st, phi, b, &rel, &bn, false)) != PYRO_OK) return rc;
      while (rel > tol && iters < max_iters) {
        mg->bind_level0(phi, b, f0);
        cudaError_t e = mg->vcycles(1, st);
        mg->bind_level0(save_phi, save_b, f0);
        PYRO_CU(e);
        iters++;
        if ((rc = true_resid(st, phi, b, &rel, &bn, false)) != PYRO_OK) return rc;
      }
    }
  } else {
    const bool bf16 = mode == PYRO_SOLVER_MGPCG_BF16 || mode == PYRO_SOLVER_MGPCG_LEARNED;
    double* S = sc.as<double>();
    // CG and its V-cycle run on the reachable fluid cells only; r = b - A phi
    if ((rc = begin_cg(st, phi, b)) != PYRO_OK) return rc;
    f0 = fa.as<uint32_t>();
    mg->bind_level0(save_phi, save_b, f0);
    struct Rebind {
      Multigrid* m;
      float* p;
      float* b;
      const uint32_t* f;
      ~Rebind() { m->bind_level0(p, b, f); }
    } rebind{mg, save_phi, save_b, save_f0};
    double bb2 = host_sc[SC_BB];
    bn = std::sqrt(bb2);
    rel = bb2 > 0 ? std::sqrt(host_sc[SC_RR] / bb2) : 0.0;
    info->rel_resid_start = rel;
    info->rel_resid_learned = rel;
    bool rel_true = true;  // rel is of the true residual
    if (mode == PYRO_SOLVER_MGPCG_LEARNED && bb2 > 0 && rel > tol) {
      double rr = host_sc[SC_RR];
      if ((rc = learned_stage(st, phi, &rr, info)) != PYRO_OK) return rc;
      rel = std::sqrt(rr / bb2);
      info->rel_resid_learned = rel;
      rel_true = false;
    }
    // CG with residual replacement: the iterations run on the device until
    // the recursively updated residual meets the tolerance; then the true
    // residual is recomputed and, if it does not meet it, CG restarts from it.
    int restarts = 0;
    while (rel > tol && iters < max_iters && restarts < 8) {
      if ((rc = cg_loop(st, phi, bf16, bb2, tol, iters, max_iters)) != PYRO_OK) return rc;
      // true residual into r (and |r|, |b|)
      PYRO_CU(cudaMemsetAsync(sc.p, 0, SC_N * 8, st));
      launch_pdl(k_resid<MetaMask>, dim3(vec_blocks(d.cells())), dim3(VT), 0, st, cells_of(d),
                 ih2, (const float*)phi, b, MetaMask{pc.meta[0].as<uint8_t>()}, mg->bc_mode,
                 r.as<float>(), S);
      PYRO_CU(cudaGetLastError());
      PYRO_CU(cudaMemcpyAsync(host_sc, sc.p, SC_N * 8, cudaMemcpyDeviceToHost, st));
      PYRO_CU(cudaMemcpyAsync(host_ctl, ctl.p, sizeof(CgCtl), cudaMemcpyDeviceToHost, st));
      PYRO_CU(cudaStreamSynchronize(st));
      iters = host_ctl->it;
      rel = bb2 > 0 ? std::sqrt(host_sc[SC_RR] / bb2) : 0.0;
      rel_true = true;
      restarts++;
      if (host_ctl->stalled) break;
    }
    if (!rel_true && (rc = true_resid(st, phi, b, &rel, &bn, true)) != PYRO_OK) return rc;
  }
  PYRO_CU(cudaEventRecord(ev1, st));
  PYRO_CU(cudaEventSynchronize(ev1));
  float ms = 0;
  PYRO_CU(cudaEventElapsedTime(&ms, ev0, ev1));
  info->iterations = iters;
  info->rel_resid = rel;
  info->b_norm = bn;
  info->ms = ms;
  info->converged = rel <= tol ? 1 : 0;
  if (mode != PYRO_SOLVER_VCYCLE && !info->converged) {
    set_error("solve: iteration cap reached before the tolerance");
    return PYRO_E_NOCONV;
  }
  return PYRO_OK;
}

cudaError_t launch_mg_apply(Dims3 d, float h, const uint32_t* f, const float* p, float* q,
                            int bc_mode, cudaStream_t st) {
  return launch_pdl(k_apply, dim3(vec_blocks(d.cells())), dim3(VT), 0, st, cells_of(d),
                    1.0 / ((double)h * h), p, FlagMask{f}, bc_mode, q);
}

}  // namespace pyro

// ------------------------------------------------------ stand-alone solver
using namespace pyro;

struct PyroPoisson {
  Dims3 d{};
  cudaStream_t stream = nullptr;
  DevBuf flags;
  Multigrid mg;
  Solver solver;
  ~PyroPoisson() {
    if (stream) {
      cudaStreamSynchronize(stream);
      cudaStreamDestroy(stream);
    }
  }
};

extern "C" {

int pyro_k_mg_apply(uint32_t nx, uint32_t ny, uint32_t nz, float h, const uint32_t* flags,
                    const float* p, float* q, int bc_mode, void* stream) {
  clear_error();
  PYRO_REQUIRE(nx && ny && nz && (size_t)nx * ny * nz < ((size_t)1 << 31),
               "pyro_k_mg_apply: invalid grid dimensions");
  PYRO_REQUIRE(flags && p && q && p != q, "pyro_k_mg_apply: null or aliased buffer");
  PYRO_REQUIRE(bc_mode == 0 || bc_mode == 1, "pyro_k_mg_apply: bc_mode must be 0 or 1");
  PYRO_CU(launch_mg_apply(Dims3{(int)nx, (int)ny, (int)nz}, h, flags, p, q, bc_mode,
                          static_cast<cudaStream_t>(stream)));
  return PYRO_OK;
}

int pyro_poisson_create(uint32_t nx, uint32_t ny, uint32_t nz, float h, int bc_mode,
                        PyroPoisson** out) {
  clear_error();
  PYRO_REQUIRE(out, "pyro_poisson_create: null argument");
  *out = nullptr;
  PYRO_REQUIRE(nx >= 2 && ny >= 2 && nz >= 2, "pyro_poisson_create: dims must be >= 2");
  PYRO_REQUIRE((uint64_t)nx * ny * nz < (1ull << 31), "pyro_poisson_create: grid too large");
  PYRO_REQUIRE(h > 0.0f, "pyro_poisson_create: h must be positive");
  PYRO_REQUIRE(bc_mode == 0 || bc_mode == 1, "pyro_poisson_create: bc_mode must be 0 or 1");
  PyroPoisson* ps = new PyroPoisson();
  ps->d = Dims3{(int)nx, (int)ny, (int)nz};
  int rc;
  if (cudaStreamCreateWithFlags(&ps->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete ps;
    set_error("pyro_poisson_create: cudaStreamCreate failed");
    return PYRO_E_CUDA;
  }
  if ((rc = ps->flags.alloc(ps->d.cells() * 4)) != PYRO_OK ||
      (rc = ps->mg.init(ps->d, h, bc_mode)) != PYRO_OK) {
    delete ps;
    return rc;
  }
  ps->mg.bind_level0(nullptr, nullptr, ps->flags.as<uint32_t>());
  if ((rc = ps->solver.init(&ps->mg)) != PYRO_OK) {
    delete ps;
    return rc;
  }
  *out = ps;
  return PYRO_OK;
}

int pyro_poisson_set_flags(PyroPoisson* ps, const uint32_t* flags) {
  clear_error();
  PYRO_REQUIRE(ps && flags, "pyro_poisson_set_flags: null argument");
  PYRO_CU(cudaMemcpyAsync(ps->flags.p, flags, ps->d.cells() * 4, cudaMemcpyDeviceToDevice,
                          ps->stream));
  PYRO_CU(cudaStreamSynchronize(ps->stream));
  return PYRO_OK;
}

int pyro_poisson_solve(PyroPoisson* ps, const float* b, float* phi, int mode, float tol,
                       int max_iters, PyroSolveInfo* info) {
  clear_error();
  PYRO_REQUIRE(ps && b && phi && info, "pyro_poisson_solve: null argument");
  return ps->solver.solve(ps->stream, phi, b, mode, tol, max_iters, info);
}

int pyro_poisson_profile_cg(PyroPoisson* ps, const float* b, float* phi, int mode, int iters,
                            float* ms_out, int* launches_out, int n) {
  clear_error();
  PYRO_REQUIRE(ps && b && phi && ms_out && launches_out && n >= 0,
               "pyro_poisson_profile_cg: null argument");
  PYRO_REQUIRE(mode == PYRO_SOLVER_MGPCG || mode == PYRO_SOLVER_MGPCG_BF16,
               "pyro_poisson_profile_cg: mode must be PYRO_SOLVER_MGPCG or _BF16");
  PYRO_REQUIRE(iters >= 1 && iters <= 1000, "pyro_poisson_profile_cg: iters must be 1..1000");
  float ms[MG_CLASSES];
  int cnt[MG_CLASSES];
  int rc = ps->solver.profile_cg(ps->stream, phi, b, mode == PYRO_SOLVER_MGPCG_BF16, iters, ms,
                                 cnt);
  if (rc != PYRO_OK) return rc;
  for (int i = 0; i < n && i < MG_CLASSES; i++) {
    ms_out[i] = ms[i];
    launches_out[i] = cnt[i];
  }
  return PYRO_OK;
}

int pyro_poisson_set_net(PyroPoisson* ps, PyroNet* net) {
  clear_error();
  PYRO_REQUIRE(ps, "pyro_poisson_set_net: null solver");
  ps->solver.net = net;
  return PYRO_OK;
}

int pyro_learned_accept(double re, double eae, double rae, double aeae, double rr,
                        double* alpha, double* rr_new) {
  double a = re / eae;
  double n = rr - 2.0 * a * rae + a * a * aeae;
  bool keep = std::isfinite(a) && std::isfinite(n) && std::isfinite(rr) && n < rr;
  if (alpha) *alpha = keep ? a : 0.0;
  if (rr_new) *rr_new = keep ? std::max(n, 0.0) : rr;
  return keep ? 1 : 0;
}

int pyro_poisson_stream(PyroPoisson* ps, void** stream) {
  clear_error();
  PYRO_REQUIRE(ps && stream, "pyro_poisson_stream: null argument");
  *stream = (void*)ps->stream;
  return PYRO_OK;
}

int pyro_poisson_destroy(PyroPoisson* ps) {
  clear_error();
  delete ps;
  return PYRO_OK;
}

}  // extern "C"
