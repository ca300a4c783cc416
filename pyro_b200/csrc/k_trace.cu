// k_trace.cu — the renderer's light caches and camera rays: the volume path
// tracer of src/shaders/trace_lib.wgsl and the trace, lightvol, lightground
// and blur kernels of src/shaders/render.wgsl:100-304, dispatched by
// src/render.rs:335-418.
//
// The reference samples rgba16float 3D textures through a linear,
// clamp-to-edge sampler.  Here the volumes stay the linear binary16 buffers
// of k_render.cu and filtering is done in FP32 from eight 8-byte texel
// loads (per axis p = u * n - 0.5, texels floor(p) and floor(p) + 1 clamped
// to the volume, weight p - floor(p); mixes along x, then y, then z).  The
// texture unit's filter keeps only 8 fractional bits of each weight; this
// keeps all of them, so the result is the exact trilinear interpolation of
// the texels.
//
//  * k_trace: one thread per pixel (8 x 8 pixels per CTA as the reference's
//    workgroup); each runs the dispatch's samples of its pixel in order and
//    adds their sum to its accum entry.
//  * k_lightvol / k_lightground: one thread per cache cell / ground texel;
//    cells of the volume cache far from any occupied brick are cleared
//    without tracing.
//  * k_blur: one thread per cell, the Gaussian weights of the radius
//    computed once on the host and passed in the launch.
//
// The random numbers are the reference's PCG hash seeded per pixel, sample
// and frame (per cell and frame for the caches), so every thread follows
// the reference's paths.  All arithmetic is FP32 in the reference's
// expression order (--fmad=false keeps products rounded); exp, sin, cos
// are CUDA's, so results match a CPU restatement to their rounding.
#include <cuda_fp16.h>

#include <cmath>

#include "common.cuh"
#include "kernels.h"

namespace pyro {

namespace {

struct V3 {
  float x, y, z;
};
__device__ __forceinline__ V3 v3(float a, float b, float c) { return V3{a, b, c}; }
__device__ __forceinline__ V3 operator+(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ V3 operator-(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ V3 operator*(V3 a, V3 b) { return v3(a.x * b.x, a.y * b.y, a.z * b.z); }
__device__ __forceinline__ V3 operator/(V3 a, V3 b) { return v3(a.x / b.x, a.y / b.y, a.z / b.z); }
__device__ __forceinline__ V3 operator*(V3 a, float s) { return v3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ V3 operator*(float s, V3 a) { return v3(s * a.x, s * a.y, s * a.z); }
__device__ __forceinline__ V3 operator/(V3 a, float s) { return v3(a.x / s, a.y / s, a.z / s); }
__device__ __forceinline__ V3 operator-(V3 a) { return v3(-a.x, -a.y, -a.z); }
__device__ __forceinline__ float dot3(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float len3(V3 a) { return sqrtf(a.x * a.x + a.y * a.y + a.z * a.z); }
__device__ __forceinline__ V3 normalize3(V3 a) { return a / len3(a); }
__device__ __forceinline__ V3 cross3(V3 a, V3 b) {
  return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
// WGSL min / max / clamp: a NaN operand gives NaN
__device__ __forceinline__ float wmin(float a, float b) {
  return (a != a || b != b) ? __int_as_float(0x7fc00000) : (a < b ? a : b);
}
__device__ __forceinline__ float wmax(float a, float b) {
  return (a != a || b != b) ? __int_as_float(0x7fc00000) : (a > b ? a : b);
}
__device__ __forceinline__ float wclamp(float x, float lo, float hi) { return wmin(wmax(x, lo), hi); }
__device__ __forceinline__ V3 vmax(V3 a, V3 b) { return v3(wmax(a.x, b.x), wmax(a.y, b.y), wmax(a.z, b.z)); }
__device__ __forceinline__ V3 vmin(V3 a, V3 b) { return v3(wmin(a.x, b.x), wmin(a.y, b.y), wmin(a.z, b.z)); }
__device__ __forceinline__ V3 vexp(V3 a) { return v3(expf(a.x), expf(a.y), expf(a.z)); }
__device__ __forceinline__ float mixf(float a, float b, float t) { return a * (1.0f - t) + b * t; }
__device__ __forceinline__ float4 mix4(float4 a, float4 b, float t) {
  return make_float4(mixf(a.x, b.x, t), mixf(a.y, b.y, t), mixf(a.z, b.z, t), mixf(a.w, b.w, t));
}
__device__ __forceinline__ float lum(V3 c) { return dot3(c, v3(0.2126f, 0.7152f, 0.0722f)); }
__device__ __forceinline__ float maxc(V3 c) { return wmax(c.x, wmax(c.y, c.z)); }

__device__ __forceinline__ float4 unhalf4(uint2 q) {
  const float2 lo = __half22float2(*reinterpret_cast<const __half2*>(&q.x));
  const float2 hi = __half22float2(*reinterpret_cast<const __half2*>(&q.y));
  return make_float4(lo.x, lo.y, hi.x, hi.y);
}
// The caches' rgba16float stores.  A value beyond the largest finite
// binary16 (65504) is stored as that value, not as an infinity: how an
// out-of-range store converts is left to the implementation by WGSL, and an
// infinite cache texel turns into NaN radiance where the tracer multiplies
// it by a zero weight.  A developed 2 cm pool flame reaches that range in
// the light caches' flux.
__device__ __forceinline__ float sat16(float v) { return fminf(fmaxf(v, -65504.0f), 65504.0f); }
__device__ __forceinline__ uint2 half4(float a, float b, float c, float d) {
  const __half2 lo = __floats2half2_rn(sat16(a), sat16(b)),
                hi = __floats2half2_rn(sat16(c), sat16(d));
  return make_uint2(*reinterpret_cast<const uint32_t*>(&lo),
                    *reinterpret_cast<const uint32_t*>(&hi));
}

// A volume of nx * ny * nz texels of 4 binary16 values, x fastest; every
// access is clamped into it.
struct HVol {
  const uint2* t;
  int nx, ny, nz;
  __device__ __forceinline__ float4 load(int x, int y, int z) const {
    return unhalf4(__ldg(t + ((uint32_t)x + (uint32_t)nx * ((uint32_t)y + (uint32_t)ny * (uint32_t)z))));
  }
  // textureSampleLevel with a linear clamp-to-edge sampler at mip 0
  __device__ __forceinline__ float4 sample(V3 uv) const {
    int x0, x1, y0, y1, z0, z1;
    float fx, fy, fz;
    axis(uv.x, nx, x0, x1, fx);
    axis(uv.y, ny, y0, y1, fy);
    axis(uv.z, nz, z0, z1, fz);
    const float4 c00 = mix4(load(x0, y0, z0), load(x1, y0, z0), fx);
    const float4 c10 = mix4(load(x0, y1, z0), load(x1, y1, z0), fx);
    const float4 c01 = mix4(load(x0, y0, z1), load(x1, y0, z1), fx);
    const float4 c11 = mix4(load(x0, y1, z1), load(x1, y1, z1), fx);
    return mix4(mix4(c00, c10, fy), mix4(c01, c11, fy), fz);
  }
  __device__ __forceinline__ static void axis(float u, int n, int& i0, int& i1, float& w) {
    const float p = u * (float)n - 0.5f;
    const float f0 = floorf(p);
    w = p - f0;
    const int k = (int)f0;
    i0 = min(max(k, 0), n - 1);
    i1 = min(max(k + 1, 0), n - 1);
  }
  __device__ __forceinline__ V3 dims() const { return v3((float)nx, (float)ny, (float)nz); }
};

// The bindings of one dispatch (trace_lib.wgsl:15-22, render.wgsl:101-106).
struct TraceBind {
  HVol vol, sol, vel, lvA, lvB, gE;
  const float* bricks;
  const float4* lut;
  const float* ecdf;
};

constexpr float PI = 3.14159265f;
constexpr float NEE_N = 2.0f;

struct Med {
  V3 st, ss, em;
};
struct Hit {
  float t;
  uint32_t kind;  // 0 sky, 1 solid, 2 ground, 3 opaque medium
  V3 n;
  float Ts, chr;
  uint32_t mat;
};
struct March {
  V3 L, Tr;
  float W;
  V3 selP, selThr;
  Hit hit;
};
struct NeeS {
  V3 c, w;
};

__device__ __forceinline__ uint32_t pcg(uint32_t v) {
  const uint32_t s = v * 747796405u + 2891336453u;
  const uint32_t w = ((s >> ((s >> 28u) + 4u)) ^ s) * 277803737u;
  return (w >> 22u) ^ w;
}

// One invocation: the uniform block, the bindings and its private RNG state.
struct Tracer {
  const PyroRenderParams& R;
  const TraceBind& B;
  bool cacheInscatter;  // the trace kernel's single-scattering lookup
  uint32_t rs;

  __device__ float rnd() {
    rs = pcg(rs);
    return (float)(rs >> 8u) * (1.0f / 16777216.0f);
  }
  __device__ V3 dimsF() const { return v3((float)R.dims[0], (float)R.dims[1], (float)R.dims[2]); }
  __device__ int dimV(int k) const { return (int)R.dims[k]; }

  // the colour table's row at temperature T (trace_lib.wgsl:31-38); off 0
  // soot emission, 1024 surface emission
  __device__ V3 lutAt(uint32_t off, float T) const {
    const float x = wclamp((T - 300.0f) / 3000.0f, 0.0f, 1.0f) * 1023.0f;
    const uint32_t i = min((uint32_t)floorf(x), 1023u);
    const uint32_t j = min(i + 1u, 1023u);
    const float4 a = __ldg(B.lut + off + i), b = __ldg(B.lut + off + j);
    const float t = x - (float)i;
    return v3(mixf(a.x, b.x, t), mixf(a.y, b.y, t), mixf(a.z, b.z, t));
  }
  // motion blur: the cell the fluid moved here from within tau seconds
  __device__ V3 blurSrc(V3 g, float tau) const {
    if (tau == 0.0f) return g;
    const float4 v = B.vel.sample(g / dimsF());
    return g - v3(v.x, v.y, v.z) * tau / R.a[0];
  }
  __device__ Med medium(V3 g, float tau) const {
    const V3 gp = blurSrc(g, tau);
    const float4 s = B.vol.sample(gp / dimsF());
    const float fv = wmax(s.x, 0.0f);
    const float aer = wmax(s.z, 0.0f);
    Med m;
    const V3 sootT = v3(R.soot[0], R.soot[1], R.soot[2]) * fv;
    const float ae = R.c[0] * aer;
    const V3 aerT = v3(ae, ae, ae);
    m.st = sootT + aerT;
    m.ss = sootT * R.soot[3] + aerT * R.c[1];
    const float ch = R.b[3] * wmax(s.w, 0.0f) * expf(-20.0f * fv);
    m.em = lutAt(0u, s.y) * fv * 1e-6f + ch * v3(0.12f, 0.28f, 1.0f);
    return m;
  }
  __device__ static void boxHit(V3 ro, V3 rd, V3 bmax, float& tn_out, float& tf_out) {
    const V3 inv = v3(1.0f / rd.x, 1.0f / rd.y, 1.0f / rd.z);
    const V3 t0 = (v3(0.0f, 0.0f, 0.0f) - ro) * inv;
    const V3 t1 = (bmax - ro) * inv;
    const V3 tn = vmin(t0, t1), tf = vmax(t0, t1);
    tn_out = wmax(wmax(tn.x, tn.y), wmax(tn.z, 0.0f));
    tf_out = wmin(wmin(tf.x, tf.y), tf.z);
  }
  __device__ float solidOcc(V3 g) const { return B.sol.sample(g / dimsF()).x; }
  __device__ float neePdf(V3 g) const {
    const int dx = dimV(0), dy = dimV(1), dz = dimV(2);
    const int cx = (int)floorf(g.x), cy = (int)floorf(g.y), cz = (int)floorf(g.z);
    if (cx < 0 || cy < 0 || cz < 0 || cx >= dx || cy >= dy || cz >= dz) return 0.0f;
    const uint32_t i = (uint32_t)(cx + dx * (cy + dy * cz));
    const float pb = __ldg(B.ecdf + i) - (i > 0u ? __ldg(B.ecdf + (i - 1u)) : 0.0f);
    return pb / (R.a[0] * R.a[0] * R.a[0]);
  }
  __device__ void brickOf(V3 g, int& cx, int& cy, int& cz, int& bx, int& by) const {
    bx = (dimV(0) + 7) / 8;
    by = (dimV(1) + 7) / 8;
    const int bz = (dimV(2) + 7) / 8;
    cx = min(max((int)floorf(g.x / 8.0f), 0), bx - 1);
    cy = min(max((int)floorf(g.y / 8.0f), 0), by - 1);
    cz = min(max((int)floorf(g.z / 8.0f), 0), bz - 1);
  }
  __device__ float brickAt(V3 g) const {
    int cx, cy, cz, bx, by;
    brickOf(g, cx, cy, cz, bx, by);
    return __ldg(B.bricks + (cx + bx * (cy + by * cz)));
  }
  // the exit distance of the brick holding g along rdg (grid units)
  __device__ float brickExit(V3 g, V3 rdg) const {
    int cx, cy, cz, bx, by;
    brickOf(g, cx, cy, cz, bx, by);
    const V3 lo = v3((float)(cx * 8), (float)(cy * 8), (float)(cz * 8));
    const V3 hi = lo + v3(8.0f, 8.0f, 8.0f);
    const V3 sel = v3(rdg.x > 0.0f ? hi.x : lo.x, rdg.y > 0.0f ? hi.y : lo.y,
                      rdg.z > 0.0f ? hi.z : lo.z);
    const V3 te = (sel - g) / rdg;
    const float ex = fabsf(rdg.x) > 1e-9f ? te.x : 1e30f;
    const float ey = fabsf(rdg.y) > 1e-9f ? te.y : 1e30f;
    const float ez = fabsf(rdg.z) > 1e-9f ? te.z : 1e30f;
    return wmin(wmin(ex, ey), ez);
  }
  __device__ static float hgPdf(float ct, float g) {
    const float d = 1.0f + g * g - 2.0f * g * ct;
    return (1.0f - g * g) / (4.0f * PI * d * sqrtf(d));
  }
  // the light cache as "isotropic + one beam along the mean direction"
  // (render.wgsl:108-125): returns A and the lobe weight a and direction d
  __device__ V3 cacheAt(V3 g, float& a, V3& d) const {
    const V3 uv = g / (2.0f * B.lvA.dims());
    const float4 a4 = B.lvA.sample(uv), b4 = B.lvB.sample(uv);
    const V3 Bv = v3(b4.x, b4.y, b4.z);
    a = wclamp(len3(Bv), 0.0f, 1.0f);
    d = a > 1e-4f ? Bv / wmax(len3(Bv), 1e-6f) : v3(0.0f, 1.0f, 0.0f);
    return v3(a4.x, a4.y, a4.z);
  }
  __device__ V3 inscatter(V3 g, V3 rd) const {
    if (!cacheInscatter) return v3(0.0f, 0.0f, 0.0f);
    float a;
    V3 d;
    const V3 A = cacheAt(g, a, d);
    return A * ((1.0f - a) / (4.0f * PI) + a * hgPdf(dot3(rd, d), R.c[2]));
  }
  __device__ V3 surfIrr(V3 g, V3 n) const {
    float a;
    V3 d;
    const V3 A = cacheAt(g, a, d);
    return A * ((1.0f - a) * 0.25f + a * wmax(dot3(n, d), 0.0f));
  }
  __device__ V3 groundIrr(V3 p) const {
    const float u = (p.x - R.gc[0]) / R.gc[2], v = (p.z - R.gc[1]) / R.gc[2];
    if (u < 0.0f || v < 0.0f || u > 1.0f || v > 1.0f) return v3(0.0f, 0.0f, 0.0f);
    const float4 e = B.gE.sample(v3(u, v, 0.5f));
    return v3(e.x, e.y, e.z);
  }

  // Ray march through the medium (trace_lib.wgsl:93-178): emission with
  // MIS weights against next-event estimation, cached single scattering,
  // reservoir selection of one scattering point, and the first solid,
  // ground, sky or opaque hit.  At most 4097 steps.
  __device__ March march(V3 ro, V3 rd, bool wantScatter, float tau, float misPdf) {
    March r;
    r.L = v3(0.0f, 0.0f, 0.0f);
    r.Tr = v3(1.0f, 1.0f, 1.0f);
    r.W = 0.0f;
    r.selP = v3(0.0f, 0.0f, 0.0f);
    r.selThr = v3(0.0f, 0.0f, 0.0f);
    r.hit.t = 1e30f;
    r.hit.kind = 0u;
    r.hit.n = v3(0.0f, 0.0f, 0.0f);
    r.hit.Ts = 0.0f;
    r.hit.chr = 0.0f;
    r.hit.mat = 0u;
    const float dx = R.a[0];
    const V3 bmax = dimsF() * dx;
    if (R.b[0] > 0.5f && rd.y < -1e-6f && ro.y > 0.0f) {
      r.hit.t = -ro.y / rd.y;
      r.hit.kind = 2u;
      r.hit.n = v3(0.0f, 1.0f, 0.0f);
    }
    float bx, by;
    boxHit(ro, rd, bmax, bx, by);
    const float t1 = wmin(by, r.hit.t);
    if (bx >= t1) return r;
    const float ds = R.a[1] * dx;
    float t = bx + rnd() * ds;
    const V3 rdg = rd / dx;
    for (int guard = 0;; guard++) {
      if (t >= t1 || guard > 4096) break;
      const V3 p = ro + rd * t;
      const V3 g = p / dx;
      if (brickAt(g) < 1e-3f) {
        const float tex = brickExit(g, rdg);
        t += wmax(tex, 0.01f) * 1.0f + ds * rnd();
        continue;
      }
      if (solidOcc(g) > 0.5f) {
        float ta = t - ds, tb = t;
        for (int k = 0; k < 6; k++) {
          const float tm = 0.5f * (ta + tb);
          if (solidOcc((ro + rd * tm) / dx) > 0.5f) tb = tm;
          else ta = tm;
        }
        const V3 gh = (ro + rd * tb) / dx;
        const float e = 0.6f;
        const V3 n = -v3(solidOcc(gh + v3(e, 0.0f, 0.0f)) - solidOcc(gh - v3(e, 0.0f, 0.0f)),
                         solidOcc(gh + v3(0.0f, e, 0.0f)) - solidOcc(gh - v3(0.0f, e, 0.0f)),
                         solidOcc(gh + v3(0.0f, 0.0f, e)) - solidOcc(gh - v3(0.0f, 0.0f, e)));
        const float4 sv = B.sol.sample(gh / dimsF());
        r.hit.t = tb;
        r.hit.kind = 1u;
        r.hit.n = len3(n) > 1e-5f ? normalize3(n) : -rd;
        r.hit.Ts = sv.y / wmax(sv.x, 0.5f);
        r.hit.chr = wclamp(sv.z / wmax(sv.x, 0.5f), 0.0f, 1.0f);
        // the material slot; slots index the 8 albedo entries
        const float ms = nearbyintf(sv.w / wmax(sv.x, 0.5f));
        r.hit.mat = ms > 0.0f ? (uint32_t)fminf(ms, 7.0f) : 0u;
        break;
      }
      const float h = wmin(ds, t1 - t);
      const Med m = medium(g, tau);
      const V3 stl = vmax(m.st, v3(1e-6f, 1e-6f, 1e-6f));
      const V3 att = vexp(-stl * h);
      const V3 seg = (v3(1.0f, 1.0f, 1.0f) - att) / stl;
      float wm = 1.0f;
      if (misPdf > 0.0f) {
        const float tm = t + 0.5f * h;
        const float pp = misPdf / wmax(tm * tm, 1e-8f);
        const float pn = NEE_N * neePdf(blurSrc((ro + rd * tm) / dx, tau));
        wm = pp * pp / (pp * pp + pn * pn);
      }
      r.L = r.L + r.Tr * m.em * seg * wm;
      if (R.gc[3] > 0.5f) r.L = r.L + r.Tr * m.ss * seg * inscatter(g, rd);
      if (wantScatter) {
        const V3 wv = r.Tr * m.ss * seg;
        const float w = lum(wv);
        if (w > 0.0f) {
          r.W += w;
          if (rnd() * r.W < w) {
            r.selP = ro + rd * (t + rnd() * h);
            r.selThr = wv / w;
          }
        }
      }
      r.Tr = r.Tr * att;
      if (maxc(r.Tr) < 1e-3f) {
        r.Tr = v3(0.0f, 0.0f, 0.0f);
        r.hit.kind = 3u;
        break;
      }
      t += h;
    }
    return r;
  }

  // Transmittance along a shadow ray (trace_lib.wgsl:181-210), one-cell
  // steps, at most 2049 of them.
  __device__ V3 shadowTr(V3 ro, V3 rd, float tmax, float tau) {
    const float dx = R.a[0];
    float bx, by;
    boxHit(ro, rd, dimsF() * dx, bx, by);
    const float t1 = wmin(by, tmax);
    V3 tr = v3(1.0f, 1.0f, 1.0f);
    if (bx >= t1) return tr;
    const float ds = 1.0f * dx;
    float t = bx + rnd() * ds;
    const V3 rdg = rd / dx;
    for (int guard = 0;; guard++) {
      if (t >= t1 || guard > 2048) break;
      const V3 g = (ro + rd * t) / dx;
      if (brickAt(g) < 1e-3f) {
        const float tex = brickExit(g, rdg);
        t += wmax(tex, 0.01f) + ds * rnd();
        continue;
      }
      if (solidOcc(g) > 0.5f) return v3(0.0f, 0.0f, 0.0f);
      const float h = wmin(ds, t1 - t);
      tr = tr * vexp(-medium(g, tau).st * h);
      if (maxc(tr) < 1e-3f) return v3(0.0f, 0.0f, 0.0f);
      t += h;
    }
    return tr;
  }
  // the emitting cell that u selects (binary search of the CDF) and its
  // probability
  __device__ uint32_t pickCell(float u, float& pb) const {
    const uint32_t nbk = (uint32_t)(dimV(0) * dimV(1) * dimV(2));
    uint32_t lo = 0u, hi = nbk - 1u;
    while (lo < hi) {
      const uint32_t mid = (lo + hi) / 2u;
      if (__ldg(B.ecdf + mid) < u) lo = mid + 1u;
      else hi = mid;
    }
    pb = __ldg(B.ecdf + lo) - (lo > 0u ? __ldg(B.ecdf + (lo - 1u)) : 0.0f);
    return lo;
  }
  __device__ V3 cellOf(uint32_t lo) const {
    const int i = (int)lo, X = dimV(0), Y = dimV(1);
    return v3((float)(i % X), (float)((i / X) % Y), (float)(i / (X * Y)));
  }
  // one light sample for the caches (trace_lib.wgsl:225-252): its
  // contribution and direction
  __device__ NeeS neeSample(V3 x, float tau) {
    NeeS r;
    r.c = v3(0.0f, 0.0f, 0.0f);
    r.w = v3(0.0f, 1.0f, 0.0f);
    const uint32_t nbk = (uint32_t)(dimV(0) * dimV(1) * dimV(2));
    if (__ldg(B.ecdf + nbk) <= 0.0f) return r;
    const float u = rnd();
    float pb;
    const uint32_t lo = pickCell(u, pb);
    if (pb <= 0.0f) return r;
    const V3 cc = cellOf(lo);
    const float r1 = rnd(), r2 = rnd(), r3 = rnd();
    const V3 g = cc + v3(r1, r2, r3);
    const float dx = R.a[0];
    const V3 em = medium(cc + v3(0.5f, 0.5f, 0.5f), 0.0f).em;
    if (maxc(em) <= 0.0f) return r;
    const V3 d = g * dx - x;
    const float dist = len3(d);
    r.w = d / wmax(dist, 1e-6f);
    const float d2 = wmax(dist * dist, 4.0f * dx * dx);
    r.c = shadowTr(x, r.w, dist, tau) * em * (dx * dx * dx) / (pb * d2);
    return r;
  }
  // next-event estimation toward the fire with MIS (trace_lib.wgsl:256-291)
  __device__ V3 nee(V3 x, V3 wi, V3 n, bool surf, float tau) {
    const uint32_t nbk = (uint32_t)(dimV(0) * dimV(1) * dimV(2));
    const float total = __ldg(B.ecdf + nbk);
    if (total <= 0.0f) return v3(0.0f, 0.0f, 0.0f);
    const float u = rnd();
    float pb;
    const uint32_t lo = pickCell(u, pb);
    if (pb <= 0.0f) return v3(0.0f, 0.0f, 0.0f);
    const V3 cc = cellOf(lo);
    const float r1 = rnd(), r2 = rnd(), r3 = rnd();
    const V3 g0 = cc + v3(r1, r2, r3);
    const float dx = R.a[0];
    V3 g = g0;
    if (tau != 0.0f) {
      const float4 v = B.vel.sample(g0 / dimsF());
      g = g0 + v3(v.x, v.y, v.z) * tau / dx;
    }
    const V3 y = g * dx;
    const float vb = dx * dx * dx;
    const V3 em = medium(cc + v3(0.5f, 0.5f, 0.5f), 0.0f).em;
    if (maxc(em) <= 0.0f) return v3(0.0f, 0.0f, 0.0f);
    const V3 d = y - x;
    const float dist = len3(d);
    const V3 w = d / wmax(dist, 1e-6f);
    const float f = surf ? wmax(dot3(w, n), 0.0f) / PI : hgPdf(dot3(wi, w), R.c[2]);
    if (f <= 0.0f) return v3(0.0f, 0.0f, 0.0f);
    const V3 tr = shadowTr(x, w, dist, tau);
    const float d2 = wmax(dist * dist, 1e-8f);
    const float pn = pb / vb;
    const float pd = f / d2;
    const float wn = (NEE_N * pn) * (NEE_N * pn) / ((NEE_N * pn) * (NEE_N * pn) + pd * pd);
    return tr * em * f * wn / (pn * d2 * NEE_N);
  }
  __device__ V3 neeN(V3 x, V3 wi, V3 n, bool surf, float tau) {
    V3 s = v3(0.0f, 0.0f, 0.0f);
    for (int i = 0; i < 2; i++) s = s + nee(x, wi, n, surf, tau);
    return s;
  }
  // frame(n) * v: the columns tx, ty, n summed in that order
  __device__ static V3 frameMul(V3 n, V3 v) {
    const V3 up = fabsf(n.y) > 0.9f ? v3(1.0f, 0.0f, 0.0f) : v3(0.0f, 1.0f, 0.0f);
    const V3 tx = normalize3(cross3(up, n));
    const V3 ty = cross3(n, tx);
    return (tx * v.x + ty * v.y) + n * v.z;
  }
  __device__ V3 cosineDir(V3 n) {
    const float u1 = rnd(), u2 = rnd();
    const float r = sqrtf(u1);
    const float ph = 2.0f * PI * u2;
    return frameMul(n, v3(r * cosf(ph), r * sinf(ph), sqrtf(wmax(1.0f - u1, 0.0f))));
  }
  __device__ V3 hgDir(V3 wi, float g) {
    const float u1 = rnd(), u2 = rnd();
    float ct;
    if (fabsf(g) < 1e-3f) {
      ct = 1.0f - 2.0f * u1;
    } else {
      const float s = (1.0f - g * g) / (1.0f - g + 2.0f * g * u1);
      ct = (1.0f + g * g - s * s) / (2.0f * g);
    }
    const float st = sqrtf(wmax(1.0f - ct * ct, 0.0f));
    const float ph = 2.0f * PI * u2;
    return frameMul(wi, v3(st * cosf(ph), st * sinf(ph), ct));
  }
  __device__ V3 skyL(V3 d) const {
    const float h = wclamp(d.y, -1.0f, 1.0f);
    const float k = h > 0.0f ? 0.6f + 0.4f * (1.0f - h) : 0.15f;
    return R.a[3] * k * v3(0.55f, 0.75f, 1.25f);
  }

  // One pixel (render.wgsl:136-215): the sum of this dispatch's samples.
  __device__ V3 tracePixel(uint32_t gx, uint32_t gy) {
    const uint32_t pix = gy * R.res[0] + gx;
    V3 acc = v3(0.0f, 0.0f, 0.0f);
    const V3 fwd = v3(R.cam_fwd[0], R.cam_fwd[1], R.cam_fwd[2]);
    const V3 right = v3(R.cam_right[0], R.cam_right[1], R.cam_right[2]);
    const V3 upv = v3(R.cam_up[0], R.cam_up[1], R.cam_up[2]);
    for (uint32_t sI = 0u; sI < R.res[3]; sI++) {
      const uint32_t sn = R.res[2] + sI;
      rs = pcg(pix * 9781u + sn * 6271u + R.dims[3] * 26699u + 17u);
      const float j1 = rnd(), j2 = rnd();
      const float ux = ((float)gx + j1) / (float)R.res[0] * 2.0f - 1.0f;
      const float uy = ((float)gy + j2) / (float)R.res[1] * 2.0f - 1.0f;
      const float tau = (rnd() - 0.5f) * R.a[2];
      V3 dir = normalize3(fwd + ux * R.cam_pos[3] * R.cam_fwd[3] * right - uy * R.cam_pos[3] * upv);
      V3 ro = v3(R.cam_pos[0], R.cam_pos[1], R.cam_pos[2]);
      if (R.cam_right[3] > 0.0f) {  // thin lens
        const V3 fp = ro + dir * (R.cam_up[3] / dot3(dir, fwd));
        const float a = 2.0f * PI * rnd();
        const float rr = R.cam_right[3] * sqrtf(rnd());
        ro = ro + (right * cosf(a) + upv * sinf(a)) * rr;
        dir = normalize3(fp - ro);
      }
      V3 L = v3(0.0f, 0.0f, 0.0f);
      if (R.gc[3] > 0.5f) {  // light-cache mode: one march, cached lighting
        const March m = march(ro, dir, false, tau, 0.0f);
        L = m.L;
        const V3 hp = ro + dir * m.hit.t;
        if (m.hit.kind == 1u) {
          const float salb = mixf(R.alb[m.hit.mat], 0.035f, m.hit.chr);
          L = L + m.Tr * (lutAt(1024u, m.hit.Ts) * 0.9f +
                          salb / PI * surfIrr(hp / R.a[0] + m.hit.n * 1.5f, m.hit.n));
        } else if (m.hit.kind == 2u) {
          const V3 gi = groundIrr(hp);
          const float amb = PI * R.a[3] * 0.6f;
          L = L + m.Tr * R.b[1] / PI * (gi + v3(amb, amb, amb));
        } else if (m.hit.kind == 0u) {
          L = L + m.Tr * skyL(dir);
        }
      } else {  // path tracing with next-event estimation and roulette
        V3 thr = v3(1.0f, 1.0f, 1.0f);
        const uint32_t nb = (uint32_t)R.b[2];
        float misPdf = 0.0f;
        for (uint32_t bo = 0u; bo <= nb; bo++) {
          const March m = march(ro, dir, bo < nb, tau, misPdf);
          L = L + thr * m.L;
          V3 salb = v3(0.0f, 0.0f, 0.0f);
          if (m.hit.kind == 1u) {
            L = L + thr * m.Tr * lutAt(1024u, m.hit.Ts) * 0.9f;
            const float sa = mixf(R.alb[m.hit.mat], 0.035f, m.hit.chr);
            salb = v3(sa, sa, sa);
          } else if (m.hit.kind == 2u) {
            salb = v3(R.b[1], R.b[1], R.b[1]);
          } else if (m.hit.kind == 0u) {
            L = L + thr * m.Tr * skyL(dir);
          }
          if (bo == nb) break;
          const float surfW = lum(m.Tr * salb);
          const float tot = m.W + surfW;
          if (tot < 1e-6f) break;
          if (rnd() * tot < m.W) {
            thr = thr * (m.selThr * tot);
            ro = m.selP;
            L = L + thr * neeN(ro, dir, v3(0.0f, 0.0f, 0.0f), false, tau);
            const V3 nd = hgDir(dir, R.c[2]);
            misPdf = hgPdf(dot3(dir, nd), R.c[2]);
            dir = nd;
          } else {
            thr = thr * (m.Tr * salb * (tot / surfW));
            ro = ro + dir * m.hit.t + m.hit.n * (0.05f * R.a[0]);
            L = L + thr * neeN(ro, dir, m.hit.n, true, tau);
            dir = cosineDir(m.hit.n);
            misPdf = wmax(dot3(dir, m.hit.n), 1e-4f) / PI;
          }
          if (bo >= 1u) {
            const float pc = wclamp(maxc(thr) * 4.0f, 0.05f, 1.0f);
            if (rnd() > pc) break;
            thr = thr / pc;
          }
        }
      }
      const float ml = maxc(L);
      if (ml > 2e6f) L = L * (2e6f / ml);
      acc = acc + L;
    }
    return acc;
  }
};

__global__ void __launch_bounds__(64) k_trace(const __grid_constant__ PyroRenderParams R,
                                              const __grid_constant__ TraceBind B,
                                              float4* __restrict__ accum) {
  const uint32_t x = blockIdx.x * 8u + threadIdx.x, y = blockIdx.y * 8u + threadIdx.y;
  if (x >= R.res[0] || y >= R.res[1]) return;
  Tracer T{R, B, true, 0u};
  const V3 s = T.tracePixel(x, y);
  float4* a = accum + ((size_t)y * R.res[0] + x);
  float4 v = *a;
  v.x += s.x;
  v.y += s.y;
  v.z += s.z;
  v.w += (float)R.res[3];
  *a = v;
}

// lightvol (render.wgsl:217-251): cache cell (x, y, z) covers grid cells
// 2x .. 2x + 1; it is traced only when a brick within two cells of its
// centre holds anything.
__global__ void __launch_bounds__(64) k_lightvol(const __grid_constant__ PyroRenderParams R,
                                                 const __grid_constant__ TraceBind B, int lx,
                                                 int ly, int lz, int rays,
                                                 uint2* __restrict__ lvA,
                                                 uint2* __restrict__ lvB) {
  const int x = blockIdx.x * 4 + threadIdx.x, y = blockIdx.y * 4 + threadIdx.y;
  const int z = blockIdx.z * 4 + threadIdx.z;
  if (x >= lx || y >= ly || z >= lz) return;
  const size_t i = (size_t)x + (size_t)lx * ((size_t)y + (size_t)ly * z);
  const V3 g = v3(((float)x + 0.5f) * 2.0f, ((float)y + 0.5f) * 2.0f, ((float)z + 0.5f) * 2.0f);
  const int bd0 = ((int)R.dims[0] + 7) / 8, bd1 = ((int)R.dims[1] + 7) / 8;
  const int bd2 = ((int)R.dims[2] + 7) / 8;
  bool busy = false;
  for (int k = 0; k < 8; k++) {
    const V3 o = v3((float)(k & 1), (float)((k >> 1) & 1), (float)((k >> 2) & 1)) * 2.0f -
                 v3(1.0f, 1.0f, 1.0f);
    const V3 q = (g + o * 2.0f) / 8.0f;
    const int cx = min(max((int)floorf(q.x), 0), bd0 - 1);
    const int cy = min(max((int)floorf(q.y), 0), bd1 - 1);
    const int cz = min(max((int)floorf(q.z), 0), bd2 - 1);
    if (__ldg(B.bricks + (cx + bd0 * (cy + bd1 * cz))) >= 1e-3f) busy = true;
  }
  if (!busy) {
    lvA[i] = make_uint2(0u, 0u);
    lvB[i] = make_uint2(0u, 0u);
    return;
  }
  Tracer T{R, B, false, pcg((uint32_t)(x + lx * (y + ly * z)) * 7919u + R.dims[3] * 104729u + 3u)};
  const V3 xw = g * R.a[0];
  V3 F = v3(0.0f, 0.0f, 0.0f), D = v3(0.0f, 0.0f, 0.0f);
  float S = 0.0f;
  for (int s = 0; s < rays; s++) {
    const NeeS ns = T.neeSample(xw, 0.0f);
    F = F + ns.c;
    const float l = lum(ns.c);
    D = D + l * ns.w;
    S += l;
  }
  F = F / (float)rays;
  const V3 Dn = D / wmax(S, 1e-12f);
  lvA[i] = half4(F.x, F.y, F.z, 0.0f);
  lvB[i] = half4(Dn.x, Dn.y, Dn.z, 0.0f);
}

// lightground (render.wgsl:253-269): irradiance 2 mm above the ground at
// texel (x, y) of the gres x gres square gc.
__global__ void __launch_bounds__(64) k_lightground(const __grid_constant__ PyroRenderParams R,
                                                    const __grid_constant__ TraceBind B,
                                                    int gres, int rays,
                                                    uint2* __restrict__ gE) {
  const int x = blockIdx.x * 8 + threadIdx.x, y = blockIdx.y * 8 + threadIdx.y;
  if (x >= gres || y >= gres) return;
  Tracer T{R, B, false, pcg((uint32_t)(x + gres * y) * 7919u + R.dims[3] * 104729u + 5u)};
  const float u = ((float)x + 0.5f) / (float)gres, v = ((float)y + 0.5f) / (float)gres;
  const V3 xw = v3(R.gc[0] + u * R.gc[2], 0.002f, R.gc[1] + v * R.gc[2]);
  V3 E = v3(0.0f, 0.0f, 0.0f);
  for (int s = 0; s < rays; s++) {
    const NeeS ns = T.neeSample(xw, 0.0f);
    E = E + ns.c * wmax(ns.w.y, 0.0f);
  }
  E = E / (float)rays;
  gE[(size_t)x + (size_t)gres * y] = half4(E.x, E.y, E.z, 0.0f);
}

constexpr int BLUR_MAX_R = 16;
struct BlurW {
  float w[2 * BLUR_MAX_R + 1];  // exp(-k^2 / (0.5 r^2 + 0.5)), k = -r .. r
};

// blur (render.wgsl:271-304): one axis, clamp-to-edge, weights normalised
// by their sum.
__global__ void __launch_bounds__(256) k_blur(const uint2* __restrict__ src,
                                              uint2* __restrict__ dst, int nx, int ny, int nz,
                                              int axis, int r, const __grid_constant__ BlurW W) {
  const int x = blockIdx.x * 32 + threadIdx.x % 32, y = blockIdx.y * 8 + threadIdx.x / 32;
  const int z = blockIdx.z;
  if (x >= nx || y >= ny) return;
  const HVol s{src, nx, ny, nz};
  float4 acc = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  float ws = 0.0f;
  for (int k = -r; k <= r; k++) {
    const float w = W.w[k + r];
    const int cx = min(max(x + (axis == 0 ? k : 0), 0), nx - 1);
    const int cy = min(max(y + (axis == 1 ? k : 0), 0), ny - 1);
    const int cz = min(max(z + (axis == 2 ? k : 0), 0), nz - 1);
    const float4 t = s.load(cx, cy, cz);
    acc = make_float4(acc.x + w * t.x, acc.y + w * t.y, acc.z + w * t.z, acc.w + w * t.w);
    ws += w;
  }
  dst[(size_t)x + (size_t)nx * ((size_t)y + (size_t)ny * z)] =
      half4(acc.x / ws, acc.y / ws, acc.z / ws, acc.w / ws);
}

TraceBind bind(const PyroRenderParams& R, const void* vol, const void* sol, const void* vel,
               const float* bricks, const float* lut, const float* ecdf) {
  const int nx = (int)R.dims[0], ny = (int)R.dims[1], nz = (int)R.dims[2];
  TraceBind B{};
  B.vol = HVol{(const uint2*)vol, nx, ny, nz};
  B.sol = HVol{(const uint2*)sol, nx, ny, nz};
  B.vel = HVol{(const uint2*)vel, nx, ny, nz};
  B.bricks = bricks;
  B.lut = (const float4*)lut;
  B.ecdf = ecdf;
  return B;
}

}  // namespace

cudaError_t launch_render_trace(const PyroRenderParams& R, const void* vol, const void* sol,
                                const void* vel, const float* bricks, const float* lut,
                                const float* ecdf, const void* lvA, const void* lvB, int lx,
                                int ly, int lz, const void* gE, int gres, float* accum,
                                cudaStream_t st) {
  TraceBind B = bind(R, vol, sol, vel, bricks, lut, ecdf);
  B.lvA = HVol{(const uint2*)lvA, lx, ly, lz};
  B.lvB = HVol{(const uint2*)lvB, lx, ly, lz};
  B.gE = HVol{(const uint2*)gE, gres, gres, 1};
  const dim3 grid((R.res[0] + 7) / 8, (R.res[1] + 7) / 8, 1);
  k_trace<<<grid, dim3(8, 8, 1), 0, st>>>(R, B, (float4*)accum);
  return cudaGetLastError();
}

cudaError_t launch_render_lightvol(const PyroRenderParams& R, const void* vol, const void* sol,
                                   const void* vel, const float* bricks, const float* lut,
                                   const float* ecdf, int lx, int ly, int lz, int rays,
                                   void* lvA, void* lvB, cudaStream_t st) {
  const TraceBind B = bind(R, vol, sol, vel, bricks, lut, ecdf);
  const dim3 grid((lx + 3) / 4, (ly + 3) / 4, (lz + 3) / 4);
  k_lightvol<<<grid, dim3(4, 4, 4), 0, st>>>(R, B, lx, ly, lz, rays, (uint2*)lvA, (uint2*)lvB);
  return cudaGetLastError();
}

cudaError_t launch_render_lightground(const PyroRenderParams& R, const void* vol,
                                      const void* sol, const void* vel, const float* bricks,
                                      const float* lut, const float* ecdf, int gres, int rays,
                                      void* gE, cudaStream_t st) {
  const TraceBind B = bind(R, vol, sol, vel, bricks, lut, ecdf);
  const dim3 grid((gres + 7) / 8, (gres + 7) / 8, 1);
  k_lightground<<<grid, dim3(8, 8, 1), 0, st>>>(R, B, gres, rays, (uint2*)gE);
  return cudaGetLastError();
}

int render_blur_max_radius() { return BLUR_MAX_R; }

cudaError_t launch_render_blur(const void* src, void* dst, Dims3 d, int axis, int r,
                               cudaStream_t st) {
  BlurW W{};
  const float s2 = 0.5f * (float)(r * r) + 0.5f;
  for (int k = -r; k <= r; k++) W.w[k + r] = std::exp(-(float)(k * k) / s2);
  const dim3 grid((d.nx + 31) / 32, (d.ny + 7) / 8, d.nz);
  k_blur<<<grid, 256, 0, st>>>((const uint2*)src, (uint2*)dst, d.nx, d.ny, d.nz, axis, r, W);
  return cudaGetLastError();
}

}  // namespace pyro
