// common.cuh — device helpers shared by the simulation kernels.
//
// Field layout and physics helpers follow src/shaders/common.wgsl:1-89;
// WGSL builtins are written with their specified formulas (mix = a*(1-t) +
// b*t, smoothstep = t*t*(3-2t), clamp = min(max(x,lo),hi)).  The library is
// compiled with --fmad=false so FP32 expressions keep the reference's
// rounding (no contraction into fused multiply-adds).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/pyro_sim.h"

namespace pyro {

// ------------------------------------------------------------ small vectors
struct F3 { float x, y, z; };
struct I3 { int x, y, z; };

__device__ __forceinline__ F3 mkf3(float x, float y, float z) { return F3{x, y, z}; }
__device__ __forceinline__ F3 operator+(F3 a, F3 b) { return F3{a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ F3 operator-(F3 a, F3 b) { return F3{a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ F3 operator*(float s, F3 a) { return F3{s * a.x, s * a.y, s * a.z}; }
__device__ __forceinline__ F3 operator*(F3 a, float s) { return F3{a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ F3 operator/(F3 a, float s) { return F3{a.x / s, a.y / s, a.z / s}; }
__device__ __forceinline__ F3 tof3(I3 c) { return F3{(float)c.x, (float)c.y, (float)c.z}; }
__device__ __forceinline__ I3 operator+(I3 a, I3 b) { return I3{a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ I3 operator-(I3 a, I3 b) { return I3{a.x - b.x, a.y - b.y, a.z - b.z}; }

__device__ __forceinline__ float4 operator+(float4 a, float4 b) {
  return make_float4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w);
}
__device__ __forceinline__ float4 operator-(float4 a, float4 b) {
  return make_float4(a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w);
}
__device__ __forceinline__ float4 operator*(float s, float4 a) {
  return make_float4(s * a.x, s * a.y, s * a.z, s * a.w);
}

// ------------------------------------------------------------ WGSL builtins
__device__ __forceinline__ float wclamp(float x, float lo, float hi) {
  return fminf(fmaxf(x, lo), hi);
}
__device__ __forceinline__ float wmix(float a, float b, float t) { return a * (1.0f - t) + b * t; }
__device__ __forceinline__ float4 wmix4(float4 a, float4 b, float t) {
  return make_float4(wmix(a.x, b.x, t), wmix(a.y, b.y, t), wmix(a.z, b.z, t), wmix(a.w, b.w, t));
}
// Two mixes a*(1-t) + b*t at once (omt = 1 - t): the four products as two
// paired FP32 multiplies of sm_100 (FMUL2), the two sums as scalar adds.
// Each lane rounds as the scalar multiply does, so the pair equals two
// wmix calls bit for bit.  The sums stay scalar on purpose: a paired
// multiply feeding a paired add is contracted into a paired fused
// multiply-add even under --fmad=false (measured on B200), which would
// change the rounding.
__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ float2 mix2(float2 a, float2 b, float2 omt, float2 t) {
  const float2 p = __fmul2_rn(a, omt), q = __fmul2_rn(b, t);
  return f2(p.x + q.x, p.y + q.y);
}
__device__ __forceinline__ float4 min4(float4 a, float4 b) {
  return make_float4(fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z), fminf(a.w, b.w));
}
__device__ __forceinline__ float4 max4(float4 a, float4 b) {
  return make_float4(fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z), fmaxf(a.w, b.w));
}
__device__ __forceinline__ float smoothstep(float e0, float e1, float x) {
  float t = wclamp((x - e0) / (e1 - e0), 0.0f, 1.0f);
  return t * t * (3.0f - 2.0f * t);
}
__device__ __forceinline__ float len3(F3 v) { return sqrtf(v.x * v.x + v.y * v.y + v.z * v.z); }
__device__ __forceinline__ F3 cross3(F3 a, F3 b) {
  return F3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ float pow4(float x) { float y = x * x; return y * y; }

constexpr float SIGMA = 5.670374e-8f;
constexpr float RGAS = 8.314f;
constexpr float RHO_SOOT = 1800.0f;

__device__ __forceinline__ I3 dir6(int k) {
  // +x -x +y -y +z -z (common.wgsl:34)
  return I3{k == 0 ? 1 : (k == 1 ? -1 : 0), k == 2 ? 1 : (k == 3 ? -1 : 0),
            k == 4 ? 1 : (k == 5 ? -1 : 0)};
}

// ------------------------------------------------ programmatic dependent launch
// A kernel launched with launch_pdl may be scheduled while the kernel before
// it in the stream is still finishing.  It calls pdl_trigger() first (so
// that the next one may be scheduled once all of its own blocks are
// running) and pdl_wait() before its first global memory access (which
// returns once the previous kernel has completed and its writes are
// visible).  Without the launch attribute both are no-ops.
__device__ __forceinline__ void pdl_trigger() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

template <typename... KArgs, typename... Args>
inline cudaError_t launch_pdl(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem,
                              cudaStream_t st, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kern, args...);
}

// --------------------------------------------------------- integer division
// Division of unsigned 32-bit values by a divisor fixed at launch, by a
// multiply-high and shifts (Granlund and Montgomery, "Division by invariant
// integers using multiplication", PLDI 1994, fig. 4.1): with
// l = ceil(log2 d) and m = floor(2^32 (2^l - d) / d) + 1,
// n / d = (t + ((n - t) >> 1)) >> (l - 1), t = umulhi(m, n), for every n.
struct FastDiv {
  uint32_t d, m, s1, s2;
  FastDiv() = default;
  __host__ explicit FastDiv(uint32_t dv) : d(dv) {
    uint32_t l = 0;
    while ((1ull << l) < dv) l++;
    m = (uint32_t)(((1ull << 32) * ((1ull << l) - dv)) / dv + 1);
    s1 = l > 0 ? 1u : 0u;
    s2 = l > 0 ? l - 1u : 0u;
  }
  __device__ __forceinline__ uint32_t div(uint32_t n) const {
    const uint32_t t = __umulhi(m, n);
    return (t + ((n - t) >> s1)) >> s2;
  }
};

// ------------------------------------------------------------------- grid
struct Grid {
  int nx, ny, nz;
  __device__ __forceinline__ bool inb(I3 c) const {
    return (unsigned)c.x < (unsigned)nx && (unsigned)c.y < (unsigned)ny &&
           (unsigned)c.z < (unsigned)nz;
  }
  __device__ __forceinline__ int sidx(I3 c) const { return c.x + nx * (c.y + ny * c.z); }
  __device__ __forceinline__ int vidx(I3 c) const {
    return c.x + (nx + 1) * (c.y + (ny + 1) * c.z);
  }
  __device__ __forceinline__ I3 clampC(I3 c) const {
    return I3{min(max(c.x, 0), nx - 1), min(max(c.y, 0), ny - 1), min(max(c.z, 0), nz - 1)};
  }
  // staggered component k: offset and valid upper index (common.wgsl:61-72)
  __device__ __forceinline__ I3 compHi(int k) const {
    return I3{nx - 1 + (k == 0), ny - 1 + (k == 1), nz - 1 + (k == 2)};
  }
  __device__ __forceinline__ bool compValid(int k, I3 c) const {
    I3 h = compHi(k);
    return c.x >= 0 && c.y >= 0 && c.z >= 0 && c.x <= h.x && c.y <= h.y && c.z <= h.z;
  }
  // distance outside the open sides/top (common.wgsl:79-82)
  __device__ __forceinline__ float outside(F3 gc) const {
    float dx_ = (float)nx, dy_ = (float)ny, dz_ = (float)nz;
    return fmaxf(fmaxf(-0.5f - gc.x, gc.x - (dx_ - 0.5f)),
                 fmaxf(fmaxf(-0.5f - gc.z, gc.z - (dz_ - 0.5f)), gc.y - (dy_ - 0.5f)));
  }
};

__device__ __forceinline__ F3 compOff(int k) {
  return F3{k == 0 ? 0.0f : 0.5f, k == 1 ? 0.0f : 0.5f, k == 2 ? 0.0f : 0.5f};
}
__device__ __forceinline__ I3 unitI(int k) { return I3{k == 0, k == 1, k == 2}; }

// Physics helpers (common.wgsl:44-58,84-89) on a parameter block.
__device__ __forceinline__ float rhoOf(const PyroParams& P, float T) {
  return P.rho0 * P.t0 / fmaxf(T, 200.0f);
}
__device__ __forceinline__ float kapP(const PyroParams& P, float T, float yo, float ys) {
  float fv = rhoOf(P, T) * fmaxf(ys, 0.0f) / RHO_SOOT;
  return 1862.0f * fv * T + P.kap_gas * wclamp(1.0f - yo / P.yo2, 0.0f, 1.0f);
}
__device__ __forceinline__ float cpOf(float T) {
  return wclamp(1000.0f + 0.24f * (T - 300.0f), 1000.0f, 1450.0f);
}
__device__ __forceinline__ float spongeSide(const PyroParams& P, const Grid& g, I3 c) {
  float e = (float)min(min(c.x, g.nx - 1 - c.x), min(c.z, g.nz - 1 - c.z));
  return 1.0f - smoothstep(0.0f, P.sponge, e);
}
__device__ __forceinline__ float spongeTop(const PyroParams& P, const Grid& g, I3 c) {
  float h = (float)g.ny;
  return smoothstep(h - 1.5f * P.sponge, h - 1.0f, (float)c.y);
}

// --------------------------------------------------------------- samplers
// Trilinear sample of staggered component X at grid point g0
// (tmpl_comp.wgsl:2-15): clamp to [0, hi], base cell min(floor, hi - 1),
// mix along x, then y, then z, with the x and y stages as paired multiplies
// (mix2: the same value as the scalar mixes bit for bit).
__device__ __forceinline__ float triC_p(const float* __restrict__ X, const Grid& gr, F3 g0, I3 hi) {
  float gx = wclamp(g0.x, 0.0f, (float)hi.x);
  float gy = wclamp(g0.y, 0.0f, (float)hi.y);
  float gz = wclamp(g0.z, 0.0f, (float)hi.z);
  int bx = min((int)floorf(gx), hi.x - 1);
  int by = min((int)floorf(gy), hi.y - 1);
  int bz = min((int)floorf(gz), hi.z - 1);
  float fx = gx - (float)bx, fy = gy - (float)by, fz = gz - (float)bz;
  const int sy = gr.nx + 1, sz = (gr.nx + 1) * (gr.ny + 1);
  int i = bx + sy * by + sz * bz;
  const float ox = 1.0f - fx, oy = 1.0f - fy;
  const float2 c0010 = mix2(f2(__ldg(X + i), __ldg(X + i + sy)),
                            f2(__ldg(X + i + 1), __ldg(X + i + sy + 1)), f2(ox, ox), f2(fx, fx));
  const float2 c0111 = mix2(f2(__ldg(X + i + sz), __ldg(X + i + sy + sz)),
                            f2(__ldg(X + i + sz + 1), __ldg(X + i + sy + sz + 1)), f2(ox, ox),
                            f2(fx, fx));
  const float2 c01 = mix2(f2(c0010.x, c0111.x), f2(c0010.y, c0111.y), f2(oy, oy), f2(fy, fy));
  return wmix(c01.x, c01.y, fz);
}
// triC_p at g0 and the 8 corners' min / max (tmpl_comp.wgsl:16-25, in its
// expression order) from one set of corner loads.
__device__ __forceinline__ float triC_mm_p(const float* __restrict__ X, const Grid& gr, F3 g0,
                                          I3 hi, float& lo, float& hv) {
  float gx = wclamp(g0.x, 0.0f, (float)hi.x);
  float gy = wclamp(g0.y, 0.0f, (float)hi.y);
  float gz = wclamp(g0.z, 0.0f, (float)hi.z);
  int bx = min((int)floorf(gx), hi.x - 1);
  int by = min((int)floorf(gy), hi.y - 1);
  int bz = min((int)floorf(gz), hi.z - 1);
  float fx = gx - (float)bx, fy = gy - (float)by, fz = gz - (float)bz;
  const int sy = gr.nx + 1, sz = (gr.nx + 1) * (gr.ny + 1);
  int i = bx + sy * by + sz * bz;
  float v0 = __ldg(X + i), v1 = __ldg(X + i + 1), v2 = __ldg(X + i + sy),
        v3 = __ldg(X + i + sy + 1), v4 = __ldg(X + i + sz), v5 = __ldg(X + i + sz + 1),
        v6 = __ldg(X + i + sy + sz), v7 = __ldg(X + i + sy + sz + 1);
  lo = fminf(fminf(fminf(fminf(fminf(fminf(fminf(1e30f, v0), v1), v2), v3), v4), v5), fminf(v6, v7));
  hv = fmaxf(fmaxf(fmaxf(fmaxf(fmaxf(fmaxf(fmaxf(-1e30f, v0), v1), v2), v3), v4), v5), fmaxf(v6, v7));
  const float ox = 1.0f - fx, oy = 1.0f - fy;
  const float2 c0010 = mix2(f2(v0, v2), f2(v1, v3), f2(ox, ox), f2(fx, fx));
  const float2 c0111 = mix2(f2(v4, v6), f2(v5, v7), f2(ox, ox), f2(fx, fx));
  const float2 c01 = mix2(f2(c0010.x, c0111.x), f2(c0010.y, c0111.y), f2(oy, oy), f2(fy, fy));
  return wmix(c01.x, c01.y, fz);
}
// Cell-centred vec4 trilinear sample (tmpl_scalar.wgsl:2-15).
__device__ __forceinline__ float4 triS(const float4* __restrict__ X, const Grid& gr, F3 gc0) {
  float gx = wclamp(gc0.x, 0.0f, (float)(gr.nx - 1));
  float gy = wclamp(gc0.y, 0.0f, (float)(gr.ny - 1));
  float gz = wclamp(gc0.z, 0.0f, (float)(gr.nz - 1));
  int bx = min((int)floorf(gx), gr.nx - 2);
  int by = min((int)floorf(gy), gr.ny - 2);
  int bz = min((int)floorf(gz), gr.nz - 2);
  float fx = gx - (float)bx, fy = gy - (float)by, fz = gz - (float)bz;
  const int sy = gr.nx, sz = gr.nx * gr.ny;
  int i = bx + sy * by + sz * bz;
  float4 c00 = wmix4(__ldg(X + i), __ldg(X + i + 1), fx);
  float4 c10 = wmix4(__ldg(X + i + sy), __ldg(X + i + sy + 1), fx);
  float4 c01 = wmix4(__ldg(X + i + sz), __ldg(X + i + sz + 1), fx);
  float4 c11 = wmix4(__ldg(X + i + sy + sz), __ldg(X + i + sy + sz + 1), fx);
  return wmix4(wmix4(c00, c10, fy), wmix4(c01, c11, fy), fz);
}
// 8-corner vec4 min/max (tmpl_scalar.wgsl:20-32).
__device__ __forceinline__ void mmS(const float4* __restrict__ X, const Grid& gr, F3 gc0,
                                    float4& lo, float4& hi) {
  float gx = wclamp(gc0.x, 0.0f, (float)(gr.nx - 1));
  float gy = wclamp(gc0.y, 0.0f, (float)(gr.ny - 1));
  float gz = wclamp(gc0.z, 0.0f, (float)(gr.nz - 1));
  int bx = min((int)floorf(gx), gr.nx - 2);
  int by = min((int)floorf(gy), gr.ny - 2);
  int bz = min((int)floorf(gz), gr.nz - 2);
  const int sy = gr.nx, sz = gr.nx * gr.ny;
  int i = bx + sy * by + sz * bz;
  lo = make_float4(1e30f, 1e30f, 1e30f, 1e30f);
  hi = make_float4(-1e30f, -1e30f, -1e30f, -1e30f);
#pragma unroll
  for (int j = 0; j < 8; j++) {
    float4 v = __ldg(X + i + (j & 1) + sy * ((j >> 1) & 1) + sz * ((j >> 2) & 1));
    lo = min4(lo, v);
    hi = max4(hi, v);
  }
}

// One axis of a trilinear sample: clamp to [0, hi], base cell
// min(floor, hi - 1), fraction and its complement (tmpl_comp.wgsl:3-5).
struct Axis {
  int b;
  float f, omf;
};
__device__ __forceinline__ Axis axis(float g0, int hi) {
  float g = wclamp(g0, 0.0f, (float)hi);
  int b = min((int)floorf(g), hi - 1);
  float f = g - (float)b;
  return Axis{b, f, 1.0f - f};
}
// Trilinear sample of a staggered component from prepared axes
// (tmpl_comp.wgsl:6-14; mix(a,b,t) = a*(1-t) + b*t).
__device__ __forceinline__ float tri_axes(const float* __restrict__ X, const Grid& gr, Axis ax,
                                          Axis ay, Axis az) {
  const int sy = gr.nx + 1, sz = (gr.nx + 1) * (gr.ny + 1);
  int i = ax.b + sy * ay.b + sz * az.b;
  float c00 = __ldg(X + i) * ax.omf + __ldg(X + i + 1) * ax.f;
  float c10 = __ldg(X + i + sy) * ax.omf + __ldg(X + i + sy + 1) * ax.f;
  float c01 = __ldg(X + i + sz) * ax.omf + __ldg(X + i + sz + 1) * ax.f;
  float c11 = __ldg(X + i + sy + sz) * ax.omf + __ldg(X + i + sy + sz + 1) * ax.f;
  float c0 = c00 * ay.omf + c10 * ay.f;
  float c1 = c01 * ay.omf + c11 * ay.f;
  return c0 * az.omf + c1 * az.f;
}

// tri_axes with the x and y stages as paired multiplies (same value bit for bit).
__device__ __forceinline__ float tri_axes_p(const float* __restrict__ X, const Grid& gr, Axis ax,
                                            Axis ay, Axis az) {
  const int sy = gr.nx + 1, sz = (gr.nx + 1) * (gr.ny + 1);
  int i = ax.b + sy * ay.b + sz * az.b;
  const float2 OX = f2(ax.omf, ax.omf), FX = f2(ax.f, ax.f);
  const float2 c0010 = mix2(f2(__ldg(X + i), __ldg(X + i + sy)),
                            f2(__ldg(X + i + 1), __ldg(X + i + sy + 1)), OX, FX);
  const float2 c0111 = mix2(f2(__ldg(X + i + sz), __ldg(X + i + sy + sz)),
                            f2(__ldg(X + i + sz + 1), __ldg(X + i + sy + sz + 1)), OX, FX);
  const float2 c01 = mix2(f2(c0010.x, c0111.x), f2(c0010.y, c0111.y), f2(ay.omf, ay.omf),
                          f2(ay.f, ay.f));
  return c01.x * az.omf + c01.y * az.f;
}
// Two tri_axes samples (components X and Y, each with its own axes), every
// stage paired across the two.
__device__ __forceinline__ float2 tri_axes_p2(const float* __restrict__ X,
                                              const float* __restrict__ Y, const Grid& gr,
                                              Axis axX, Axis ayX, Axis azX, Axis axY, Axis ayY,
                                              Axis azY) {
  const int sy = gr.nx + 1, sz = (gr.nx + 1) * (gr.ny + 1);
  const int i = axX.b + sy * ayX.b + sz * azX.b, j = axY.b + sy * ayY.b + sz * azY.b;
  const float2 OX = f2(axX.omf, axY.omf), FX = f2(axX.f, axY.f);
  const float2 c00 = mix2(f2(__ldg(X + i), __ldg(Y + j)), f2(__ldg(X + i + 1), __ldg(Y + j + 1)),
                          OX, FX);
  const float2 c10 = mix2(f2(__ldg(X + i + sy), __ldg(Y + j + sy)),
                          f2(__ldg(X + i + sy + 1), __ldg(Y + j + sy + 1)), OX, FX);
  const float2 c01 = mix2(f2(__ldg(X + i + sz), __ldg(Y + j + sz)),
                          f2(__ldg(X + i + sz + 1), __ldg(Y + j + sz + 1)), OX, FX);
  const float2 c11 = mix2(f2(__ldg(X + i + sy + sz), __ldg(Y + j + sy + sz)),
                          f2(__ldg(X + i + sy + sz + 1), __ldg(Y + j + sy + sz + 1)), OX, FX);
  const float2 OY = f2(ayX.omf, ayY.omf), FY = f2(ayX.f, ayY.f);
  const float2 c0 = mix2(c00, c10, OY, FY);
  const float2 c1 = mix2(c01, c11, OY, FY);
  return mix2(c0, c1, f2(azX.omf, azY.omf), f2(azX.f, azY.f));
}

// Staggered velocity and RK2 traces in grid units (vel.wgsl:2-19).
struct Vel {
  const float* __restrict__ u;
  const float* __restrict__ v;
  const float* __restrict__ w;
  // velAt(p): u at p - (0,.5,.5) clamped to (nx, ny-1, nz-1), v at
  // p - (.5,0,.5) to (nx-1, ny, nz-1), w at p - (.5,.5,0) to
  // (nx-1, ny-1, nz).  Per axis only two offset/bound pairs occur, so six
  // axis set-ups serve the three samples.
  // PAIRED: the same values with paired FP32 multiplies (mix2), u paired
  // with v; it pays only where the FP32 pipe is the limit (the velocity
  // predictor; measured slower in the other advection kernels).
  template <bool PAIRED = false>
  __device__ __forceinline__ F3 at(const Grid& g, F3 p) const {
    Axis xu = axis(p.x - 0.0f, g.nx), xvw = axis(p.x - 0.5f, g.nx - 1);
    Axis yv = axis(p.y - 0.0f, g.ny), yuw = axis(p.y - 0.5f, g.ny - 1);
    Axis zw = axis(p.z - 0.0f, g.nz), zuv = axis(p.z - 0.5f, g.nz - 1);
    if constexpr (PAIRED) {
      const float2 uv = tri_axes_p2(u, v, g, xu, yuw, zuv, xvw, yv, zuv);
      return F3{uv.x, uv.y, tri_axes_p(w, g, xvw, yuw, zw)};
    }
    return F3{tri_axes(u, g, xu, yuw, zuv), tri_axes(v, g, xvw, yv, zuv),
              tri_axes(w, g, xvw, yuw, zw)};
  }
  __device__ __forceinline__ F3 back(const Grid& g, float k, F3 x) const {
    F3 u1 = at(g, x);
    F3 u2 = at(g, x - (0.5f * k) * u1);
    return x - k * u2;
  }
  __device__ __forceinline__ F3 fwd(const Grid& g, float k, F3 x) const {
    F3 u1 = at(g, x);
    F3 u2 = at(g, x + (0.5f * k) * u1);
    return x + k * u2;
  }
  // Both traces from x; the velocity at x (identical in the two traces)
  // is sampled once.
  __device__ __forceinline__ void both(const Grid& g, float k, F3 x, F3& b, F3& f) const {
    F3 u1 = at(g, x);
    F3 h = (0.5f * k) * u1;
    F3 ub = at(g, x - h);
    F3 uf = at(g, x + h);
    b = x - k * ub;
    f = x + k * uf;
  }

  // velAt at a face or cell centre, where every trilinear fraction is 0,
  // 1/2 or (clamped) 1: the same value as at() bit for bit (mix(a, b, 0) =
  // a, mix(a, b, 1/2) = a * 0.5 + b * 0.5, mix(a, b, 1) = b), with only
  // the loads and additions that remain, in at()'s x, y, z order.
  __device__ __forceinline__ F3 at_face(const Grid& g, int k, I3 c) const {
    return F3{face_comp(g, 0, k, c), face_comp(g, 1, k, c), face_comp(g, 2, k, c)};
  }
  __device__ __forceinline__ F3 at_center(const Grid& g, I3 c) const {
    const int sy = g.nx + 1, sz = (g.nx + 1) * (g.ny + 1);
    const int i = c.x + sy * c.y + sz * c.z;
    return F3{__ldg(u + i) * 0.5f + __ldg(u + i + 1) * 0.5f,
              __ldg(v + i) * 0.5f + __ldg(v + i + sy) * 0.5f,
              __ldg(w + i) * 0.5f + __ldg(w + i + sz) * 0.5f};
  }
  // back / both with the first sample at the k-face of cell c (k = 3: the
  // cell centre); x is that position.
  __device__ __forceinline__ F3 first(const Grid& g, int k, I3 c) const {
    return k == 3 ? at_center(g, c) : at_face(g, k, c);
  }
  template <bool PAIRED = false>
  __device__ __forceinline__ F3 back_at(const Grid& g, float kk, int k, I3 c, F3 x) const {
    F3 u1 = first(g, k, c);
    F3 u2 = at<PAIRED>(g, x - (0.5f * kk) * u1);
    return x - kk * u2;
  }
  __device__ __forceinline__ F3 fwd_at(const Grid& g, float kk, int k, I3 c, F3 x) const {
    F3 u1 = first(g, k, c);
    F3 h = (0.5f * kk) * u1;
    F3 uf = at(g, x + h);
    return x + kk * uf;
  }
  __device__ __forceinline__ void both_at(const Grid& g, float kk, int k, I3 c, F3 x, F3& b,
                                          F3& f) const {
    F3 u1 = first(g, k, c);
    F3 h = (0.5f * kk) * u1;
    F3 ub = at(g, x - h);
    F3 uf = at(g, x + h);
    b = x - kk * ub;
    f = x + kk * uf;
  }

 private:
  // Component j sampled at the k-face position of cell c.  Along axis k the
  // coordinate is c - 1/2 (clamped to [0, n - 1]: the lower value alone at
  // c = 0, the upper alone past the top), along axis j it is c + 1/2, along
  // the third axis c itself; for j == k the face value itself.
  __device__ __forceinline__ float face_comp(const Grid& g, int j, int k, I3 c) const {
    const float* X = j == 0 ? u : (j == 1 ? v : w);
    const int sy = g.nx + 1, sz = (g.nx + 1) * (g.ny + 1);
    const int cc[3] = {c.x, c.y, c.z}, n[3] = {g.nx, g.ny, g.nz}, st[3] = {1, sy, sz};
    if (j == k) return __ldg(X + c.x + sy * c.y + sz * c.z);
    // base index and the two averaged axes (ordered x < y < z)
    int two[3];
    int base = 0;
#pragma unroll
    for (int a = 0; a < 3; a++) {
      int b = cc[a];
      int t = 0;
      if (a == k) {
        if (b <= 0) b = 0;
        else if (b > n[a] - 1) b = n[a] - 1;
        else { b -= 1; t = 1; }
      } else if (a == j) {
        t = 1;
      }
      two[a] = t;
      base += st[a] * b;
    }
    const int a1 = j < k ? j : k, a2 = j < k ? k : j;
    const int s1 = st[a1], s2 = st[a2];
    auto avg1 = [&](int i) {
      return two[a1] ? __ldg(X + i) * 0.5f + __ldg(X + i + s1) * 0.5f : __ldg(X + i);
    };
    float r0 = avg1(base);
    if (!two[a2]) return r0;
    float r1 = avg1(base + s2);
    return r0 * 0.5f + r1 * 0.5f;
  }
};

// -------------------------------------------------------------- statistics
// Block-wide reductions then one global atomic per value and block (they
// replace the 64-lane tree + CAS add of stats.wgsl:1-36): block_max for one
// maximum (`sh`: 32 floats), block_stats for several sums and maxima at
// once.  Every thread of the block must call them.
__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ float warp_max(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ int lin_tid() {
  return threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
}
// N statistics of one block in one pass: each value is reduced over the
// warp (a sum, or for bit k of max_mask the maximum of non-negative values),
// the warps' results meet in shared memory (sh: N * 32 floats, not otherwise
// in use) behind a single barrier, and warp 0 reduces them and adds (or
// atomicMax-es) them into stats[slot[k]] (the reference's float atomics,
// stats.wgsl:1-36, as one atomic per block).  Every thread of the block must
// call it.
template <int N>
__device__ __forceinline__ void block_stats(float* sh, float (&v)[N], float* stats,
                                            const int (&slot)[N], uint32_t max_mask) {
  const int t = lin_tid();
  const int nw = (blockDim.x * blockDim.y * blockDim.z) >> 5;
#pragma unroll
  for (int k = 0; k < N; k++)
    v[k] = ((max_mask >> k) & 1u) ? warp_max(fmaxf(v[k], 0.0f)) : warp_sum(v[k]);
  if ((t & 31) == 0) {
#pragma unroll
    for (int k = 0; k < N; k++) sh[k * 32 + (t >> 5)] = v[k];
  }
  __syncthreads();
  if (t < 32) {
#pragma unroll
    for (int k = 0; k < N; k++) {
      const bool mx = ((max_mask >> k) & 1u) != 0;
      float s = t < nw ? sh[k * 32 + t] : 0.0f;
      s = mx ? warp_max(s) : warp_sum(s);
      if (t == 0) {
        if (mx) atomicMax(reinterpret_cast<unsigned int*>(stats + slot[k]), __float_as_uint(s));
        else if (s != 0.0f) atomicAdd(stats + slot[k], s);
      }
    }
  }
}
// max of non-negative values via integer atomicMax on the bits (stats.wgsl:14)
__device__ __forceinline__ void block_max(float* sh, float v, float* dst) {
  int t = lin_tid();
  int nthreads = blockDim.x * blockDim.y * blockDim.z;
  v = warp_max(fmaxf(v, 0.0f));
  __syncthreads();
  if ((t & 31) == 0) sh[t >> 5] = v;
  __syncthreads();
  if (t < 32) {
    float s = t < (nthreads >> 5) ? sh[t] : 0.0f;
    s = warp_max(s);
    if (t == 0) atomicMax(reinterpret_cast<unsigned int*>(dst), __float_as_uint(s));
  }
}

}  // namespace pyro
