// k_render.cu — the renderer's per-frame prologue: its input pack
// (src/shaders/render.wgsl:3-61) and its fire-light sampling tables
// (render.wgsl:63-98 and the CDF of src/render.rs:316-333), dispatched by
// src/render.rs:263-333.
//
// The reference packs the step's fields into three rgba16float 3D textures
// that the volume path tracer samples with hardware trilinear filtering,
// then marks the 8^3 bricks that hold anything visible.  Here the volumes
// are linear device buffers of 4 IEEE binary16 values per cell (x fastest,
// the cell index of the simulation grid), converted with round to nearest
// even; a CUDA consumer can sample them directly or copy them into a
// cudaArray for filtering.
//
//  * k_render_pack: one thread per cell, float4 loads of s0, s1 and sol,
//    the flag, the six faces of the cell, three 8-byte stores.  It is a
//    stream: 64 bytes in and 24 out per cell, bound by HBM.
//  * k_render_bricks: one CTA per brick, the maximum over the brick and a
//    one-cell shell (the reach of trilinear filtering) read back from the
//    half volumes, as the reference reads its textures.
//  * k_render_ecells: one thread per cell, the emission power with the
//    six-axis escape weighting, rays loaded eight samples ahead.
//  * k_cdf_sums / k_cdf_blocks / k_cdf_final: the emission CDF as a
//    deterministic FP64 scan on the device, where the reference reads the
//    emission back and sums it on the CPU.
//
// Per-cell arithmetic is the reference's in its order (--fmad=false keeps
// each product rounded), so the half values equal the oracle's bit for bit.
#include <cuda_fp16.h>

#include "common.cuh"
#include "kernels.h"

namespace pyro {

namespace {

constexpr int RP_BX = 32, RP_BY = 8;

__device__ __forceinline__ uint2 half4(float a, float b, float c, float d) {
  const __half2 lo = __floats2half2_rn(a, b), hi = __floats2half2_rn(c, d);
  return make_uint2(*reinterpret_cast<const uint32_t*>(&lo),
                    *reinterpret_cast<const uint32_t*>(&hi));
}

// vol = (soot volume fraction ppm, T K, smoke g/m^3, heat release kW/m^3),
// sol = (occupancy, Ts, char fraction, material slot) premultiplied by the
// occupancy, vel = (cell-centred velocity m/s, 0)  (render.wgsl:17-35).
__global__ void __launch_bounds__(RP_BX * RP_BY) k_render_pack(
    const PyroParams* __restrict__ Pp, Grid g, const float4* __restrict__ s0,
    const float4* __restrict__ s1, const float4* __restrict__ sol,
    const uint32_t* __restrict__ flags, const float* __restrict__ u,
    const float* __restrict__ v, const float* __restrict__ w, uint2* __restrict__ vol,
    uint2* __restrict__ solp, uint2* __restrict__ velp) {
  const int x = blockIdx.x * RP_BX + threadIdx.x, y = blockIdx.y * RP_BY + threadIdx.y;
  const int z = blockIdx.z;
  if (x >= g.nx || y >= g.ny) return;
  const I3 c{x, y, z};
  const int i = g.sidx(c), f = g.vidx(c);
  const float4 a = __ldg(s0 + i), b = __ldg(s1 + i), so = __ldg(sol + i);
  const bool solid = __ldg(flags + i) == 1u;
  const float rho = rhoOf(*Pp, a.x);
  vol[i] = solid ? half4(0.0f, a.x, 0.0f, 0.0f)
                 : half4(rho * a.w / RHO_SOOT * 1e6f, a.x, rho * b.x * 1e3f, b.y * 1e-3f);
  const float tot = so.y + so.z;
  const float oc = solid ? 1.0f : 0.0f;
  solp[i] = half4(oc, so.w * oc, so.z / fmaxf(tot, 1e-6f) * oc, so.x * oc);
  const int sy = g.nx + 1, sz = (g.nx + 1) * (g.ny + 1);
  velp[i] = half4(0.5f * (__ldg(u + f) + __ldg(u + f + 1)), 0.5f * (__ldg(v + f) + __ldg(v + f + sy)),
                  0.5f * (__ldg(w + f) + __ldg(w + f + sz)), 0.0f);
}

constexpr int RB_THREADS = 256;

__device__ __forceinline__ float4 unhalf4(uint2 q) {
  const float2 lo = __half22float2(*reinterpret_cast<const __half2*>(&q.x));
  const float2 hi = __half22float2(*reinterpret_cast<const __half2*>(&q.y));
  return make_float4(lo.x, lo.y, hi.x, hi.y);
}

// Brick b (x fastest over ceil(n / 8) bricks per axis): the maximum of
// max(max(vol.x * 10, vol.z * 2), max(vol.w * 0.1, sol.x * 10)) over the
// cells of [8 b - 1, 8 b + 9) inside the grid, at least 0
// (render.wgsl:38-61).
__global__ void __launch_bounds__(RB_THREADS) k_render_bricks(Grid g, int bnx, int bny,
                                                              const uint2* __restrict__ vol,
                                                              const uint2* __restrict__ solp,
                                                              float* __restrict__ bricks) {
  __shared__ float red[RB_THREADS / 32];
  const int b = blockIdx.x;
  const int bx = b % bnx, by = (b / bnx) % bny, bz = b / (bnx * bny);
  const int x0 = max(8 * bx - 1, 0), x1 = min(8 * bx + 9, g.nx);
  const int y0 = max(8 * by - 1, 0), y1 = min(8 * by + 9, g.ny);
  const int z0 = max(8 * bz - 1, 0), z1 = min(8 * bz + 9, g.nz);
  const int ex = x1 - x0, ey = y1 - y0, n = ex * ey * (z1 - z0);
  float m = 0.0f;
  for (int t = threadIdx.x; t < n; t += RB_THREADS) {
    const int r = t / ex, lx = t - r * ex;
    const int lz = r / ey, ly = r - lz * ey;
    const int i = g.sidx(I3{x0 + lx, y0 + ly, z0 + lz});
    const float4 vv = unhalf4(__ldg(vol + i)), ss = unhalf4(__ldg(solp + i));
    m = fmaxf(m, fmaxf(fmaxf(vv.x * 10.0f, vv.z * 2.0f), fmaxf(vv.w * 0.1f, ss.x * 10.0f)));
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    float r = red[0];
#pragma unroll
    for (int k = 1; k < RB_THREADS / 32; k++) r = fmaxf(r, red[k]);
    bricks[b] = r;
  }
}

// Emission power of each cell for the renderer's fire-light sampling
// (render.wgsl:63-98): soot emission from the first 1024 rows of the colour
// table at the cell's temperature plus chemiluminescence, luminance times
// the cell volume, weighted by the mean escape transmittance along the six
// axes (rays of up to 48 cells that stop once the optical depth passes 7).
// The ray samples are loaded eight at a time before the sequential sum,
// which keeps the reference's stopping rule and summation order.
__device__ __forceinline__ float ray_depth(const Grid& g, const uint2* __restrict__ vol, I3 c,
                                           I3 d, float ks, float km, float dx) {
  float od = 0.0f;
  for (int s0 = 1; s0 <= 48; s0 += 8) {
    float w[8];
    bool in[8];
#pragma unroll
    for (int j = 0; j < 8; j++) {
      const int s = s0 + j;
      const I3 p{c.x + s * d.x, c.y + s * d.y, c.z + s * d.z};
      in[j] = s <= 48 && g.inb(p);
      w[j] = 0.0f;
      if (in[j]) {
        const float4 v = unhalf4(__ldg(vol + g.sidx(p)));
        w[j] = ks * fmaxf(v.x, 0.0f) + km * fmaxf(v.z, 0.0f);
      }
    }
#pragma unroll
    for (int j = 0; j < 8; j++) {
      if (!in[j] || od > 7.0f) return od;
      od += w[j] * dx;
    }
  }
  return od;
}

__global__ void __launch_bounds__(RP_BX * RP_BY) k_render_ecells(
    const PyroParams* __restrict__ Pp, Grid g, const uint2* __restrict__ vol,
    const float4* __restrict__ lut, float4 chemi, float* __restrict__ ecell) {
  const int x = blockIdx.x * RP_BX + threadIdx.x, y = blockIdx.y * RP_BY + threadIdx.y;
  const int z = blockIdx.z;
  if (x >= g.nx || y >= g.ny) return;
  const I3 c{x, y, z};
  const int i = g.sidx(c);
  const float dx = Pp->dx;
  const float4 v = unhalf4(__ldg(vol + i));
  // lutAt(T): linear in the table's 1024 temperature rows
  const float xt = wclamp((v.y - 300.0f) / 3000.0f, 0.0f, 1.0f) * 1023.0f;
  const uint32_t li = (uint32_t)floorf(xt);
  const float4 l0 = __ldg(lut + li), l1 = __ldg(lut + min(li + 1u, 1023u));
  const float fr = xt - (float)li;
  const float sx = fmaxf(v.x, 0.0f);
  const float a = chemi.x * fmaxf(v.w, 0.0f) * expf(-20.0f * sx);
  const float er = wmix(l0.x, l1.x, fr) * sx * 1e-6f + a * 0.12f;
  const float eg = wmix(l0.y, l1.y, fr) * sx * 1e-6f + a * 0.28f;
  const float eb = wmix(l0.z, l1.z, fr) * sx * 1e-6f + a * 1.0f;
  float e = (er * 0.2126f + eg * 0.7152f + eb * 0.0722f) * dx * dx * dx;
  if (e > 0.0f) {
    float esc = 0.0f;
#pragma unroll 1
    for (int k = 0; k < 6; k++) esc += expf(-ray_depth(g, vol, c, dir6(k), chemi.y, chemi.z, dx));
    e *= fmaxf(esc / 6.0f, 0.02f);
  }
  ecell[i] = e;
}

// The emission CDF (src/render.rs:316-333, a CPU loop over a read-back
// buffer in the reference): cdf[i] = (sum_{j<=i} max(e_j, 0)) / total as
// float, cdf[n] = total, all sums in FP64.  Three deterministic passes:
// per-block sums, one block scanning those, per-block scan plus offset.
constexpr int CDF_T = 512, CDF_PER = 16, CDF_SPAN = CDF_T * CDF_PER;

// exclusive scan of one double per thread across the block (fixed order)
__device__ __forceinline__ double block_exscan(double v, double* sh, double* total) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  double inc = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const double t = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += t;
  }
  if (lane == 31) sh[wid] = inc;
  __syncthreads();
  if (wid == 0) {
    double w = lane < CDF_T / 32 ? sh[lane] : 0.0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const double t = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += t;
    }
    if (lane < CDF_T / 32) sh[lane] = w;  // inclusive warp prefixes
  }
  __syncthreads();
  const double off = wid > 0 ? sh[wid - 1] : 0.0;
  *total = sh[CDF_T / 32 - 1];
  return off + inc - v;
}

// A block's 8192 values staged in shared memory: global loads and stores
// coalesced (element j of the block at k * CDF_T + t for thread t), each
// thread then works on its own CDF_PER contiguous values.  One padding word
// per 32 keeps both access patterns free of bank conflicts.
__device__ __forceinline__ int cdf_pad(int j) { return j + (j >> 5); }
constexpr int CDF_SMEM = CDF_SPAN + CDF_SPAN / 32;

__device__ __forceinline__ void cdf_stage(const float* __restrict__ e, long n, float* se) {
  const long base = (long)blockIdx.x * CDF_SPAN;
#pragma unroll
  for (int k = 0; k < CDF_PER; k++) {
    const int j = k * CDF_T + threadIdx.x;
    se[cdf_pad(j)] = base + j < n ? fmaxf(__ldg(e + base + j), 0.0f) : 0.0f;
  }
  __syncthreads();
}

__global__ void __launch_bounds__(CDF_T) k_cdf_sums(const float* __restrict__ e, long n,
                                                    double* __restrict__ bsum) {
  __shared__ double sh[CDF_T / 32];
  __shared__ float se[CDF_SMEM];
  cdf_stage(e, n, se);
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < CDF_PER; k++) s += (double)se[cdf_pad(threadIdx.x * CDF_PER + k)];
  double tot;
  block_exscan(s, sh, &tot);
  if (threadIdx.x == 0) bsum[blockIdx.x] = tot;
}

// bsum[0..nb) -> exclusive prefixes in place, bsum[nb] = the total
__global__ void __launch_bounds__(CDF_T) k_cdf_blocks(double* __restrict__ bsum, int nb) {
  __shared__ double sh[CDF_T / 32];
  double carry = 0.0;
  for (int b0 = 0; b0 < nb; b0 += CDF_T) {
    const int b = b0 + threadIdx.x;
    const double v = b < nb ? bsum[b] : 0.0;
    double tot;
    const double ex = block_exscan(v, sh, &tot);
    __syncthreads();  // every thread has read sh before the next chunk writes it
    if (b < nb) bsum[b] = carry + ex;
    carry += tot;
  }
  if (threadIdx.x == 0) bsum[nb] = carry;
}

__global__ void __launch_bounds__(CDF_T) k_cdf_final(const float* __restrict__ e, long n,
                                                     const double* __restrict__ bsum, int nb,
                                                     float* __restrict__ cdf) {
  __shared__ double sh[CDF_T / 32];
  __shared__ float se[CDF_SMEM];
  cdf_stage(e, n, se);
  const int t0 = threadIdx.x * CDF_PER;
  float v[CDF_PER];
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < CDF_PER; k++) {
    v[k] = se[cdf_pad(t0 + k)];
    s += (double)v[k];
  }
  double tot;
  double acc = bsum[blockIdx.x] + block_exscan(s, sh, &tot);
  const double total = bsum[nb];
#pragma unroll
  for (int k = 0; k < CDF_PER; k++) {  // each thread rewrites only its own values
    acc += (double)v[k];
    se[cdf_pad(t0 + k)] = total > 0.0 ? (float)(acc / total) : 0.0f;
  }
  __syncthreads();
  const long base = (long)blockIdx.x * CDF_SPAN;
#pragma unroll
  for (int k = 0; k < CDF_PER; k++) {
    const int j = k * CDF_T + threadIdx.x;
    if (base + j < n) cdf[base + j] = se[cdf_pad(j)];
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) cdf[n] = (float)total;
}

}  // namespace

size_t render_cdf_scratch_bytes(long n) {
  return (size_t)((n + CDF_SPAN - 1) / CDF_SPAN + 1) * sizeof(double);
}

cudaError_t launch_render_ecells(const PyroParams* P, Dims3 d, const void* vol, const float* lut,
                                 const float* chemi, float* ecell, cudaStream_t st) {
  dim3 grid((d.nx + RP_BX - 1) / RP_BX, (d.ny + RP_BY - 1) / RP_BY, d.nz);
  k_render_ecells<<<grid, dim3(RP_BX, RP_BY), 0, st>>>(
      P, Grid{d.nx, d.ny, d.nz}, (const uint2*)vol, (const float4*)lut,
      make_float4(chemi[0], chemi[1], chemi[2], chemi[3]), ecell);
  return cudaGetLastError();
}

cudaError_t launch_render_cdf(long n, const float* ecell, float* cdf, void* scratch,
                              cudaStream_t st) {
  const int nb = (int)((n + CDF_SPAN - 1) / CDF_SPAN);
  double* bsum = (double*)scratch;
  k_cdf_sums<<<nb, CDF_T, 0, st>>>(ecell, n, bsum);
  k_cdf_blocks<<<1, CDF_T, 0, st>>>(bsum, nb);
  k_cdf_final<<<nb, CDF_T, 0, st>>>(ecell, n, bsum, nb, cdf);
  return cudaGetLastError();
}

cudaError_t launch_render_pack(const PyroParams* P, Dims3 d, const float4* s0, const float4* s1,
                               const float4* sol, const uint32_t* flags, const float* u,
                               const float* v, const float* w, void* vol, void* solp, void* vel,
                               cudaStream_t st) {
  dim3 grid((d.nx + RP_BX - 1) / RP_BX, (d.ny + RP_BY - 1) / RP_BY, d.nz);
  k_render_pack<<<grid, dim3(RP_BX, RP_BY), 0, st>>>(P, Grid{d.nx, d.ny, d.nz}, s0, s1, sol,
                                                      flags, u, v, w, (uint2*)vol, (uint2*)solp,
                                                      (uint2*)vel);
  return cudaGetLastError();
}

cudaError_t launch_render_bricks(Dims3 d, const void* vol, const void* solp, float* bricks,
                                 cudaStream_t st) {
  const int bnx = (d.nx + 7) / 8, bny = (d.ny + 7) / 8, bnz = (d.nz + 7) / 8;
  k_render_bricks<<<bnx * bny * bnz, RB_THREADS, 0, st>>>(Grid{d.nx, d.ny, d.nz}, bnx, bny,
                                                          (const uint2*)vol, (const uint2*)solp,
                                                          bricks);
  return cudaGetLastError();
}

}  // namespace pyro
