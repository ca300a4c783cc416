// trace_oracle.cpp — CPU oracle of pyro's volume path tracer and light caches.
//
// TEST INFRASTRUCTURE ONLY, like pyro_oracle.cpp: the checker for a CUDA
// renderer; the product never links, loads or calls it.
//
// It restates src/shaders/trace_lib.wgsl and the trace, lightvol,
// lightground and blur kernels of src/shaders/render.wgsl:100-304, one
// invocation at a time in dispatch order, in FP32 in the WGSL expression
// order (built with -ffp-contract=off).  Choices where WGSL leaves the
// result to the implementation, the same as the WGSL interpreter that makes
// the golden vectors (tests/golden/wgsl.py):
//   * textureSampleLevel with the renderer's sampler (linear filtering,
//     clamp-to-edge; src/render.rs:121-125) is exact FP32 trilinear
//     filtering: per axis p = u * n - 0.5, texels floor(p) and floor(p) + 1
//     clamped to the texture, weight p - floor(p), mixes along x, y, z;
//   * normalize(v) = v / length(v); dot products and matrix-vector products
//     are summed in component order;
//   * texture stores round to nearest even into binary16.
// The random numbers are the reference's PCG hash (trace_lib.wgsl:24-30),
// so both sides follow the same paths up to the rounding of exp, sin, cos
// and sqrt.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "half.h"

namespace {

using oracle_half::f16_to_f32;
using oracle_half::f32_to_f16;

struct V3 {
  float x, y, z;
};
inline V3 v3(float a, float b, float c) { return V3{a, b, c}; }
inline V3 operator+(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
inline V3 operator-(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
inline V3 operator*(V3 a, V3 b) { return v3(a.x * b.x, a.y * b.y, a.z * b.z); }
inline V3 operator/(V3 a, V3 b) { return v3(a.x / b.x, a.y / b.y, a.z / b.z); }
inline V3 operator*(V3 a, float s) { return v3(a.x * s, a.y * s, a.z * s); }
inline V3 operator*(float s, V3 a) { return v3(s * a.x, s * a.y, s * a.z); }
inline V3 operator/(V3 a, float s) { return v3(a.x / s, a.y / s, a.z / s); }
inline V3 operator-(V3 a) { return v3(-a.x, -a.y, -a.z); }
inline float dot3(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline float length3(V3 a) { return std::sqrt(a.x * a.x + a.y * a.y + a.z * a.z); }
inline V3 normalize3(V3 a) { return a / length3(a); }
inline V3 cross3(V3 a, V3 b) {
  return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
// WGSL min / max / clamp on f32, NaN-propagating like the interpreter's
inline float wmin(float a, float b) { return (a != a || b != b) ? NAN : (a < b ? a : b); }
inline float wmax(float a, float b) { return (a != a || b != b) ? NAN : (a > b ? a : b); }
inline float wclamp(float x, float lo, float hi) { return wmin(wmax(x, lo), hi); }
inline V3 vmax(V3 a, V3 b) { return v3(wmax(a.x, b.x), wmax(a.y, b.y), wmax(a.z, b.z)); }
inline V3 vmin(V3 a, V3 b) { return v3(wmin(a.x, b.x), wmin(a.y, b.y), wmin(a.z, b.z)); }
inline V3 vexp(V3 a) { return v3(std::exp(a.x), std::exp(a.y), std::exp(a.z)); }
inline float mixf(float a, float b, float t) { return a * (1.0f - t) + b * t; }
inline float lum(V3 c) { return dot3(c, v3(0.2126f, 0.7152f, 0.0722f)); }

struct F4 {
  float x, y, z, w;
};

// The uniform block RP (trace_lib.wgsl:1-14); u32 rows as uint32_t.
struct RP {
  uint32_t res[4], dims[4];
  float camPos[4], camFwd[4], camRight[4], camUp[4], a[4], b[4], soot[4], c[4];
  float alb[2][4];
  float gc[4];
};

// A 3D rgba16float texture as nz x ny x nx texels of 4 binary16 values.
struct Tex {
  int nx = 0, ny = 0, nz = 0;
  const uint16_t* h = nullptr;
  F4 load(int x, int y, int z) const {
    const uint16_t* q = h + 4 * ((size_t)x + (size_t)nx * ((size_t)y + (size_t)ny * z));
    return F4{f16_to_f32(q[0]), f16_to_f32(q[1]), f16_to_f32(q[2]), f16_to_f32(q[3])};
  }
  F4 sample(V3 uv) const {
    auto ax = [](float u, int n, int& i0, int& i1, float& w) {
      const float p = u * (float)n - 0.5f;
      const float f0 = std::floor(p);
      w = p - f0;
      const int k = (int)f0;
      i0 = std::min(std::max(k, 0), n - 1);
      i1 = std::min(std::max(k + 1, 0), n - 1);
    };
    int x0, x1, y0, y1, z0, z1;
    float fx, fy, fz;
    ax(uv.x, nx, x0, x1, fx);
    ax(uv.y, ny, y0, y1, fy);
    ax(uv.z, nz, z0, z1, fz);
    auto mix4 = [](F4 a, F4 b, float t) {
      return F4{mixf(a.x, b.x, t), mixf(a.y, b.y, t), mixf(a.z, b.z, t), mixf(a.w, b.w, t)};
    };
    const F4 c00 = mix4(load(x0, y0, z0), load(x1, y0, z0), fx);
    const F4 c10 = mix4(load(x0, y1, z0), load(x1, y1, z0), fx);
    const F4 c01 = mix4(load(x0, y0, z1), load(x1, y0, z1), fx);
    const F4 c11 = mix4(load(x0, y1, z1), load(x1, y1, z1), fx);
    return mix4(mix4(c00, c10, fy), mix4(c01, c11, fy), fz);
  }
  V3 dims() const { return v3((float)nx, (float)ny, (float)nz); }
};

const float PI = 3.14159265f;
const float NEE_N = 2.0f;

struct Med {
  V3 st, ss, em;
};
struct Hit {
  float t = 0.0f;
  uint32_t kind = 0u;
  V3 n{0.0f, 0.0f, 0.0f};
  float Ts = 0.0f, chr = 0.0f;
  uint32_t mat = 0u;
};
struct MR {
  V3 L{0.0f, 0.0f, 0.0f}, Tr{0.0f, 0.0f, 0.0f};
  float W = 0.0f;
  V3 selP{0.0f, 0.0f, 0.0f}, selThr{0.0f, 0.0f, 0.0f};
  Hit hit;
};
struct NS {
  V3 c, w;
};

// One invocation's view of the bindings; `rs` is its private RNG state.
struct Ctx {
  RP R;
  Tex volT, solT, velT, lvA, lvB, gE;
  const float* bricks = nullptr;
  const float* lut = nullptr;  // vec4 rows
  const float* ecdf = nullptr;
  bool cache_inscatter = false;  // the trace kernel's inscatter (else 0)
  uint32_t rs = 0u;

  static uint32_t pcg(uint32_t v) {
    const uint32_t s = v * 747796405u + 2891336453u;
    const uint32_t w = ((s >> ((s >> 28u) + 4u)) ^ s) * 277803737u;
    return (w >> 22u) ^ w;
  }
  float rnd() {
    rs = pcg(rs);
    return (float)(rs >> 8u) * (1.0f / 16777216.0f);
  }
  V3 dimsF() const { return v3((float)R.dims[0], (float)R.dims[1], (float)R.dims[2]); }
  int dimV(int k) const { return (int)R.dims[k]; }

  V3 lutAt(uint32_t off, float T) const {
    const float x = wclamp((T - 300.0f) / 3000.0f, 0.0f, 1.0f) * 1023.0f;
    const uint32_t i = (uint32_t)std::floor(x);
    const uint32_t j = std::min(i + 1u, 1023u);
    const float* a = lut + 4 * (off + i);
    const float* b = lut + 4 * (off + j);
    const float t = x - (float)i;
    return v3(mixf(a[0], b[0], t), mixf(a[1], b[1], t), mixf(a[2], b[2], t));
  }
  V3 blurSrc(V3 g, float tau) const {
    if (tau == 0.0f) return g;
    const F4 v = velT.sample(g / dimsF());
    return g - v3(v.x, v.y, v.z) * tau / R.a[0];
  }
  Med medium(V3 g, float tau) const {
    const V3 gp = blurSrc(g, tau);
    const F4 s = volT.sample(gp / dimsF());
    const float fv = wmax(s.x, 0.0f);
    const float aer = wmax(s.z, 0.0f);
    Med m;
    const V3 sootT = v3(R.soot[0], R.soot[1], R.soot[2]) * fv;
    const V3 aerT = v3(R.c[0] * aer, R.c[0] * aer, R.c[0] * aer);
    m.st = sootT + aerT;
    m.ss = sootT * R.soot[3] + aerT * R.c[1];
    const float ch = R.b[3] * wmax(s.w, 0.0f) * std::exp(-20.0f * fv);
    m.em = lutAt(0u, s.y) * fv * 1e-6f + ch * v3(0.12f, 0.28f, 1.0f);
    return m;
  }
  static void boxHit(V3 ro, V3 rd, V3 bmax, float& tn_out, float& tf_out) {
    const V3 inv = v3(1.0f / rd.x, 1.0f / rd.y, 1.0f / rd.z);
    const V3 t0 = (v3(0.0f, 0.0f, 0.0f) - ro) * inv;
    const V3 t1 = (bmax - ro) * inv;
    const V3 tn = vmin(t0, t1), tf = vmax(t0, t1);
    tn_out = wmax(wmax(tn.x, tn.y), wmax(tn.z, 0.0f));
    tf_out = wmin(wmin(tf.x, tf.y), tf.z);
  }
  float solidOcc(V3 g) const { return solT.sample(g / dimsF()).x; }
  float neePdf(V3 g) const {
    const int dx = dimV(0), dy = dimV(1), dz = dimV(2);
    const int cx = (int)std::floor(g.x), cy = (int)std::floor(g.y), cz = (int)std::floor(g.z);
    if (cx < 0 || cy < 0 || cz < 0 || cx >= dx || cy >= dy || cz >= dz) return 0.0f;
    const uint32_t i = (uint32_t)(cx + dx * (cy + dy * cz));
    const float pb = ecdf[i] - (i > 0u ? ecdf[std::max(i, 1u) - 1u] : 0.0f);
    return pb / (R.a[0] * R.a[0] * R.a[0]);
  }
  float brickAt(V3 g) const {
    const int bx = (dimV(0) + 7) / 8, by = (dimV(1) + 7) / 8, bz = (dimV(2) + 7) / 8;
    const int cx = std::min(std::max((int)std::floor(g.x / 8.0f), 0), bx - 1);
    const int cy = std::min(std::max((int)std::floor(g.y / 8.0f), 0), by - 1);
    const int cz = std::min(std::max((int)std::floor(g.z / 8.0f), 0), bz - 1);
    return bricks[cx + bx * (cy + by * cz)];
  }
  // the exit distance of the empty brick holding g, along rdg (grid units)
  float brickExit(V3 g, V3 rdg) const {
    const int bx = (dimV(0) + 7) / 8, by = (dimV(1) + 7) / 8, bz = (dimV(2) + 7) / 8;
    const int cx = std::min(std::max((int)std::floor(g.x / 8.0f), 0), bx - 1);
    const int cy = std::min(std::max((int)std::floor(g.y / 8.0f), 0), by - 1);
    const int cz = std::min(std::max((int)std::floor(g.z / 8.0f), 0), bz - 1);
    const V3 lo = v3((float)(cx * 8), (float)(cy * 8), (float)(cz * 8));
    const V3 hi = lo + v3(8.0f, 8.0f, 8.0f);
    const V3 sel = v3(rdg.x > 0.0f ? hi.x : lo.x, rdg.y > 0.0f ? hi.y : lo.y,
                      rdg.z > 0.0f ? hi.z : lo.z);
    const V3 te = (sel - g) / rdg;
    const float ex = std::fabs(rdg.x) > 1e-9f ? te.x : 1e30f;
    const float ey = std::fabs(rdg.y) > 1e-9f ? te.y : 1e30f;
    const float ez = std::fabs(rdg.z) > 1e-9f ? te.z : 1e30f;
    return wmin(wmin(ex, ey), ez);
  }
  static float hgPdf(float ct, float g) {
    const float d = 1.0f + g * g - 2.0f * g * ct;
    return (1.0f - g * g) / (4.0f * PI * d * std::sqrt(d));
  }
  // the trace kernel's single-scattering lookup (render.wgsl:108-116)
  V3 inscatter(V3 g, V3 rd) const {
    if (!cache_inscatter) return v3(0.0f, 0.0f, 0.0f);
    const V3 uv = g / (2.0f * lvA.dims());
    const F4 a4 = lvA.sample(uv), b4 = lvB.sample(uv);
    const V3 A = v3(a4.x, a4.y, a4.z), B = v3(b4.x, b4.y, b4.z);
    const float a = wclamp(length3(B), 0.0f, 1.0f);
    const V3 d = a > 1e-4f ? B / wmax(length3(B), 1e-6f) : v3(0.0f, 1.0f, 0.0f);
    return A * ((1.0f - a) / (4.0f * PI) + a * hgPdf(dot3(rd, d), R.c[2]));
  }
  V3 surfIrr(V3 g, V3 n) const {
    const V3 uv = g / (2.0f * lvA.dims());
    const F4 a4 = lvA.sample(uv), b4 = lvB.sample(uv);
    const V3 A = v3(a4.x, a4.y, a4.z), B = v3(b4.x, b4.y, b4.z);
    const float a = wclamp(length3(B), 0.0f, 1.0f);
    const V3 d = a > 1e-4f ? B / wmax(length3(B), 1e-6f) : v3(0.0f, 1.0f, 0.0f);
    return A * ((1.0f - a) * 0.25f + a * wmax(dot3(n, d), 0.0f));
  }
  V3 groundIrr(V3 p) const {
    const float u = (p.x - R.gc[0]) / R.gc[2], v = (p.z - R.gc[1]) / R.gc[2];
    if (u < 0.0f || v < 0.0f || u > 1.0f || v > 1.0f) return v3(0.0f, 0.0f, 0.0f);
    const F4 e = gE.sample(v3(u, v, 0.5f));
    return v3(e.x, e.y, e.z);
  }

  // trace_lib.wgsl:93-178
  MR march(V3 ro, V3 rd, bool wantScatter, float tau, float misPdf) {
    MR r;
    r.L = v3(0.0f, 0.0f, 0.0f);
    r.Tr = v3(1.0f, 1.0f, 1.0f);
    r.W = 0.0f;
    r.hit.kind = 0u;
    r.hit.t = 1e30f;
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
    int guard = 0;
    for (;;) {
      if (t >= t1 || guard > 4096) break;
      guard++;
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
        const F4 sv = solT.sample(gh / dimsF());
        r.hit.t = tb;
        r.hit.kind = 1u;
        r.hit.n = length3(n) > 1e-5f ? normalize3(n) : -rd;
        r.hit.Ts = sv.y / wmax(sv.x, 0.5f);
        r.hit.chr = wclamp(sv.z / wmax(sv.x, 0.5f), 0.0f, 1.0f);
        r.hit.mat = (uint32_t)std::nearbyint(sv.w / wmax(sv.x, 0.5f));
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
      if (wmax(r.Tr.x, wmax(r.Tr.y, r.Tr.z)) < 1e-3f) {
        r.Tr = v3(0.0f, 0.0f, 0.0f);
        r.hit.kind = 3u;
        break;
      }
      t += h;
    }
    return r;
  }

  // trace_lib.wgsl:181-210
  V3 shadowTr(V3 ro, V3 rd, float tmax, float tau) {
    const float dx = R.a[0];
    float bx, by;
    boxHit(ro, rd, dimsF() * dx, bx, by);
    const float t1 = wmin(by, tmax);
    V3 tr = v3(1.0f, 1.0f, 1.0f);
    if (bx >= t1) return tr;
    const float ds = 1.0f * dx;
    float t = bx + rnd() * ds;
    const V3 rdg = rd / dx;
    int guard = 0;
    for (;;) {
      if (t >= t1 || guard > 2048) break;
      guard++;
      const V3 g = (ro + rd * t) / dx;
      if (brickAt(g) < 1e-3f) {
        const float tex = brickExit(g, rdg);
        t += wmax(tex, 0.01f) + ds * rnd();
        continue;
      }
      if (solidOcc(g) > 0.5f) return v3(0.0f, 0.0f, 0.0f);
      const float h = wmin(ds, t1 - t);
      tr = tr * vexp(-medium(g, tau).st * h);
      if (wmax(tr.x, wmax(tr.y, tr.z)) < 1e-3f) return v3(0.0f, 0.0f, 0.0f);
      t += h;
    }
    return tr;
  }
  // the emission cell picked by u (binary search of the CDF) and its probability
  uint32_t pickCell(float u, float& pb) const {
    const uint32_t nbk = (uint32_t)(dimV(0) * dimV(1) * dimV(2));
    uint32_t lo = 0u, hi = nbk - 1u;
    for (;;) {
      if (lo >= hi) break;
      const uint32_t mid = (lo + hi) / 2u;
      if (ecdf[mid] < u) lo = mid + 1u;
      else hi = mid;
    }
    pb = ecdf[lo] - (lo > 0u ? ecdf[std::max(lo, 1u) - 1u] : 0.0f);
    return lo;
  }
  V3 cellOf(uint32_t lo) const {
    const int i = (int)lo, X = dimV(0), Y = dimV(1);
    return v3((float)(i % X), (float)((i / X) % Y), (float)(i / (X * Y)));
  }
  // trace_lib.wgsl:225-252
  NS neeSample(V3 x, float tau) {
    NS r;
    r.c = v3(0.0f, 0.0f, 0.0f);
    r.w = v3(0.0f, 1.0f, 0.0f);
    const uint32_t nbk = (uint32_t)(dimV(0) * dimV(1) * dimV(2));
    if (ecdf[nbk] <= 0.0f) return r;
    const float u = rnd();
    float pb;
    const uint32_t lo = pickCell(u, pb);
    if (pb <= 0.0f) return r;
    const V3 cc = cellOf(lo);
    const float r1 = rnd(), r2 = rnd(), r3 = rnd();
    const V3 g = cc + v3(r1, r2, r3);
    const float dx = R.a[0];
    const V3 em = medium(cc + v3(0.5f, 0.5f, 0.5f), 0.0f).em;
    if (wmax(em.x, wmax(em.y, em.z)) <= 0.0f) return r;
    const V3 d = g * dx - x;
    const float dist = length3(d);
    r.w = d / wmax(dist, 1e-6f);
    const float d2 = wmax(dist * dist, 4.0f * dx * dx);
    r.c = shadowTr(x, r.w, dist, tau) * em * (dx * dx * dx) / (pb * d2);
    return r;
  }
  // trace_lib.wgsl:256-291
  V3 nee(V3 x, V3 wi, V3 n, bool surf, float tau) {
    const uint32_t nbk = (uint32_t)(dimV(0) * dimV(1) * dimV(2));
    const float total = ecdf[nbk];
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
      const F4 v = velT.sample(g0 / dimsF());
      g = g0 + v3(v.x, v.y, v.z) * tau / dx;
    }
    const V3 y = g * dx;
    const float vb = dx * dx * dx;
    const V3 em = medium(cc + v3(0.5f, 0.5f, 0.5f), 0.0f).em;
    if (wmax(em.x, wmax(em.y, em.z)) <= 0.0f) return v3(0.0f, 0.0f, 0.0f);
    const V3 d = y - x;
    const float dist = length3(d);
    const V3 w = d / wmax(dist, 1e-6f);
    float f = 0.0f;
    if (surf) f = wmax(dot3(w, n), 0.0f) / PI;
    else f = hgPdf(dot3(wi, w), R.c[2]);
    if (f <= 0.0f) return v3(0.0f, 0.0f, 0.0f);
    const V3 tr = shadowTr(x, w, dist, tau);
    const float d2 = wmax(dist * dist, 1e-8f);
    const float pn = pb / vb;
    const float pd = f / d2;
    const float wn = (NEE_N * pn) * (NEE_N * pn) / ((NEE_N * pn) * (NEE_N * pn) + pd * pd);
    return tr * em * f * wn / (pn * d2 * NEE_N);
  }
  V3 neeN(V3 x, V3 wi, V3 n, bool surf, float tau) {
    V3 s = v3(0.0f, 0.0f, 0.0f);
    for (int i = 0; i < 2; i++) s = s + nee(x, wi, n, surf, tau);
    return s;
  }
  // frame(n) * v: columns tx, ty, n summed in that order
  static V3 frameMul(V3 n, V3 v) {
    const V3 up = std::fabs(n.y) > 0.9f ? v3(1.0f, 0.0f, 0.0f) : v3(0.0f, 1.0f, 0.0f);
    const V3 tx = normalize3(cross3(up, n));
    const V3 ty = cross3(n, tx);
    return (tx * v.x + ty * v.y) + n * v.z;
  }
  V3 cosineDir(V3 n) {
    const float u1 = rnd(), u2 = rnd();
    const float r = std::sqrt(u1);
    const float ph = 2.0f * PI * u2;
    return frameMul(n, v3(r * std::cos(ph), r * std::sin(ph), std::sqrt(wmax(1.0f - u1, 0.0f))));
  }
  V3 hgDir(V3 wi, float g) {
    const float u1 = rnd(), u2 = rnd();
    float ct;
    if (std::fabs(g) < 1e-3f) {
      ct = 1.0f - 2.0f * u1;
    } else {
      const float s = (1.0f - g * g) / (1.0f - g + 2.0f * g * u1);
      ct = (1.0f + g * g - s * s) / (2.0f * g);
    }
    const float st = std::sqrt(wmax(1.0f - ct * ct, 0.0f));
    const float ph = 2.0f * PI * u2;
    return frameMul(wi, v3(st * std::cos(ph), st * std::sin(ph), ct));
  }
  V3 skyL(V3 d) const {
    const float h = wclamp(d.y, -1.0f, 1.0f);
    const float k = h > 0.0f ? 0.6f + 0.4f * (1.0f - h) : 0.15f;
    return R.a[3] * k * v3(0.55f, 0.75f, 1.25f);
  }
  float albedoOf(uint32_t m) const { return R.alb[m / 4u][m % 4u]; }

  // render.wgsl:132-215, one pixel: the sum over this dispatch's samples
  F4 tracePixel(uint32_t gx, uint32_t gy) {
    const uint32_t pix = gy * R.res[0] + gx;
    V3 acc = v3(0.0f, 0.0f, 0.0f);
    for (uint32_t sI = 0u; sI < R.res[3]; sI++) {
      const uint32_t sn = R.res[2] + sI;
      rs = pcg(pix * 9781u + sn * 6271u + R.dims[3] * 26699u + 17u);
      const float j1 = rnd(), j2 = rnd();
      const float ux = ((float)gx + j1) / (float)R.res[0] * 2.0f - 1.0f;
      const float uy = ((float)gy + j2) / (float)R.res[1] * 2.0f - 1.0f;
      const float tau = (rnd() - 0.5f) * R.a[2];
      const V3 fwd = v3(R.camFwd[0], R.camFwd[1], R.camFwd[2]);
      const V3 right = v3(R.camRight[0], R.camRight[1], R.camRight[2]);
      const V3 upv = v3(R.camUp[0], R.camUp[1], R.camUp[2]);
      V3 dir = normalize3(fwd + ux * R.camPos[3] * R.camFwd[3] * right - uy * R.camPos[3] * upv);
      V3 ro = v3(R.camPos[0], R.camPos[1], R.camPos[2]);
      if (R.camRight[3] > 0.0f) {
        const V3 fp = ro + dir * (R.camUp[3] / dot3(dir, fwd));
        const float a = 2.0f * PI * rnd();
        const float rr = R.camRight[3] * std::sqrt(rnd());
        ro = ro + (right * std::cos(a) + upv * std::sin(a)) * rr;
        dir = normalize3(fp - ro);
      }
      V3 L = v3(0.0f, 0.0f, 0.0f);
      if (R.gc[3] > 0.5f) {
        const MR m = march(ro, dir, false, tau, 0.0f);
        L = m.L;
        const V3 hp = ro + dir * m.hit.t;
        if (m.hit.kind == 1u) {
          const float salb = mixf(albedoOf(m.hit.mat), 0.035f, m.hit.chr);
          L = L + m.Tr * (lutAt(1024u, m.hit.Ts) * 0.9f +
                          salb / PI * surfIrr(hp / R.a[0] + m.hit.n * 1.5f, m.hit.n));
        } else if (m.hit.kind == 2u) {
          const V3 gi = groundIrr(hp);
          const float amb = PI * R.a[3] * 0.6f;
          L = L + m.Tr * R.b[1] / PI * (gi + v3(amb, amb, amb));
        } else if (m.hit.kind == 0u) {
          L = L + m.Tr * skyL(dir);
        }
      } else {
        V3 thr = v3(1.0f, 1.0f, 1.0f);
        const uint32_t nb = (uint32_t)R.b[2];
        float misPdf = 0.0f;
        for (uint32_t bo = 0u; bo <= nb; bo++) {
          const MR m = march(ro, dir, bo < nb, tau, misPdf);
          L = L + thr * m.L;
          V3 salb = v3(0.0f, 0.0f, 0.0f);
          if (m.hit.kind == 1u) {
            L = L + thr * m.Tr * lutAt(1024u, m.hit.Ts) * 0.9f;
            const float sa = mixf(albedoOf(m.hit.mat), 0.035f, m.hit.chr);
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
            const float pc = wclamp(wmax(thr.x, wmax(thr.y, thr.z)) * 4.0f, 0.05f, 1.0f);
            if (rnd() > pc) break;
            thr = thr / pc;
          }
        }
      }
      const float ml = wmax(L.x, wmax(L.y, L.z));
      if (ml > 2e6f) L = L * (2e6f / ml);
      acc = acc + L;
    }
    return F4{acc.x, acc.y, acc.z, (float)R.res[3]};
  }
};

Tex tex_of(const uint16_t* h, int nx, int ny, int nz) {
  Tex t;
  t.nx = nx;
  t.ny = ny;
  t.nz = nz;
  t.h = h;
  return t;
}

void rp_from_rows(const double* rows, RP& R) {
  for (int k = 0; k < 4; k++) {
    R.res[k] = (uint32_t)rows[k];
    R.dims[k] = (uint32_t)rows[4 + k];
    R.camPos[k] = (float)rows[8 + k];
    R.camFwd[k] = (float)rows[12 + k];
    R.camRight[k] = (float)rows[16 + k];
    R.camUp[k] = (float)rows[20 + k];
    R.a[k] = (float)rows[24 + k];
    R.b[k] = (float)rows[28 + k];
    R.soot[k] = (float)rows[32 + k];
    R.c[k] = (float)rows[36 + k];
    R.alb[0][k] = (float)rows[40 + k];
    R.alb[1][k] = (float)rows[44 + k];
    R.gc[k] = (float)rows[48 + k];
  }
}

// rgba16float cache store.  WGSL leaves the conversion of values beyond the
// largest finite binary16 to the implementation; they are stored as 65504
// (saturated), the choice the CUDA tracer makes too.  Below that range the
// store is round to nearest even.
float sat16(float v) { return std::fmin(std::fmax(v, -65504.0f), 65504.0f); }
void store_h4(uint16_t* t, size_t i, float a, float b, float c, float d) {
  t[4 * i] = f32_to_f16(sat16(a));
  t[4 * i + 1] = f32_to_f16(sat16(b));
  t[4 * i + 2] = f32_to_f16(sat16(c));
  t[4 * i + 3] = f32_to_f16(sat16(d));
}

}  // namespace

extern "C" {

// The renderer's volumes and tables for one frame: rp = 13 rows of 4 (the
// uniform block, u32 rows as their values), vol / sol / vel packed
// volumes (nz, ny, nx, 4 binary16), bricks, the colour table (2048 float4)
// and the emission CDF (n + 1).  lv_n / gr_n: shadow rays per light-cache
// cell / ground texel (96 / 128 in the reference, render.wgsl:225,254).

// lightvol (render.wgsl:217-251): lvA, lvB of (lz, ly, lx, 4) binary16.
void or_render_lightvol(const double* rp, const uint16_t* vol, const uint16_t* sol,
                        const uint16_t* vel, const float* bricks, const float* lut,
                        const float* ecdf, int lx, int ly, int lz, int lv_n, uint16_t* lvA,
                        uint16_t* lvB) {
  Ctx C;
  rp_from_rows(rp, C.R);
  const int nx = (int)C.R.dims[0], ny = (int)C.R.dims[1], nz = (int)C.R.dims[2];
  C.volT = tex_of(vol, nx, ny, nz);
  C.solT = tex_of(sol, nx, ny, nz);
  C.velT = tex_of(vel, nx, ny, nz);
  C.bricks = bricks;
  C.lut = lut;
  C.ecdf = ecdf;
  const int bd[3] = {(nx + 7) / 8, (ny + 7) / 8, (nz + 7) / 8};
  // cells are independent (each seeds its own random numbers)
#pragma omp parallel for collapse(2) firstprivate(C) schedule(dynamic)
  for (int z = 0; z < lz; z++)
    for (int y = 0; y < ly; y++)
      for (int x = 0; x < lx; x++) {
        const size_t i = (size_t)x + (size_t)lx * ((size_t)y + (size_t)ly * z);
        const V3 g = v3(((float)x + 0.5f) * 2.0f, ((float)y + 0.5f) * 2.0f,
                        ((float)z + 0.5f) * 2.0f);
        bool busy = false;
        for (int k = 0; k < 8; k++) {
          const V3 o = v3((float)(k & 1), (float)((k >> 1) & 1), (float)((k >> 2) & 1)) * 2.0f -
                       v3(1.0f, 1.0f, 1.0f);
          const V3 q = (g + o * 2.0f) / 8.0f;
          const int bc[3] = {std::min(std::max((int)std::floor(q.x), 0), bd[0] - 1),
                             std::min(std::max((int)std::floor(q.y), 0), bd[1] - 1),
                             std::min(std::max((int)std::floor(q.z), 0), bd[2] - 1)};
          if (bricks[bc[0] + bd[0] * (bc[1] + bd[1] * bc[2])] >= 1e-3f) busy = true;
        }
        if (!busy) {
          store_h4(lvA, i, 0.0f, 0.0f, 0.0f, 0.0f);
          store_h4(lvB, i, 0.0f, 0.0f, 0.0f, 0.0f);
          continue;
        }
        C.rs = Ctx::pcg((uint32_t)(x + lx * (y + ly * z)) * 7919u + C.R.dims[3] * 104729u + 3u);
        const V3 xw = g * C.R.a[0];
        V3 F = v3(0.0f, 0.0f, 0.0f), D = v3(0.0f, 0.0f, 0.0f);
        float S = 0.0f;
        for (int s = 0; s < lv_n; s++) {
          const NS ns = C.neeSample(xw, 0.0f);
          F = F + ns.c;
          const float l = lum(ns.c);
          D = D + l * ns.w;
          S += l;
        }
        F = F / (float)lv_n;
        const V3 Dn = D / wmax(S, 1e-12f);
        store_h4(lvA, i, F.x, F.y, F.z, 0.0f);
        store_h4(lvB, i, Dn.x, Dn.y, Dn.z, 0.0f);
      }
}

// lightground (render.wgsl:253-269): gE of (1, gres, gres, 4) binary16.
void or_render_lightground(const double* rp, const uint16_t* vol, const uint16_t* sol,
                           const uint16_t* vel, const float* bricks, const float* lut,
                           const float* ecdf, int gres, int gr_n, uint16_t* gE) {
  Ctx C;
  rp_from_rows(rp, C.R);
  const int nx = (int)C.R.dims[0], ny = (int)C.R.dims[1], nz = (int)C.R.dims[2];
  C.volT = tex_of(vol, nx, ny, nz);
  C.solT = tex_of(sol, nx, ny, nz);
  C.velT = tex_of(vel, nx, ny, nz);
  C.bricks = bricks;
  C.lut = lut;
  C.ecdf = ecdf;
#pragma omp parallel for firstprivate(C) schedule(dynamic)
  for (int y = 0; y < gres; y++)
    for (int x = 0; x < gres; x++) {
      C.rs = Ctx::pcg((uint32_t)(x + gres * y) * 7919u + C.R.dims[3] * 104729u + 5u);
      const float u = ((float)x + 0.5f) / (float)gres, v = ((float)y + 0.5f) / (float)gres;
      const V3 xw = v3(C.R.gc[0] + u * C.R.gc[2], 0.002f, C.R.gc[1] + v * C.R.gc[2]);
      V3 E = v3(0.0f, 0.0f, 0.0f);
      for (int s = 0; s < gr_n; s++) {
        const NS ns = C.neeSample(xw, 0.0f);
        E = E + ns.c * wmax(ns.w.y, 0.0f);
      }
      E = E / (float)gr_n;
      store_h4(gE, (size_t)x + (size_t)gres * y, E.x, E.y, E.z, 0.0f);
    }
}

// blur (render.wgsl:271-304): one axis (0..2) of radius r, src -> dst, both
// (nz, ny, nx, 4) binary16.
void or_render_blur(const uint16_t* src, uint16_t* dst, int nx, int ny, int nz, int axis,
                    int r) {
  const Tex s = tex_of(src, nx, ny, nz);
  const float s2 = 0.5f * (float)(r * r) + 0.5f;
#pragma omp parallel for
  for (int z = 0; z < nz; z++)
    for (int y = 0; y < ny; y++)
      for (int x = 0; x < nx; x++) {
        F4 acc{0.0f, 0.0f, 0.0f, 0.0f};
        float ws = 0.0f;
        for (int k = -r; k <= r; k++) {
          const float w = std::exp(-(float)(k * k) / s2);
          const int cx = std::min(std::max(x + (axis == 0 ? k : 0), 0), nx - 1);
          const int cy = std::min(std::max(y + (axis == 1 ? k : 0), 0), ny - 1);
          const int cz = std::min(std::max(z + (axis == 2 ? k : 0), 0), nz - 1);
          const F4 t = s.load(cx, cy, cz);
          acc = F4{acc.x + w * t.x, acc.y + w * t.y, acc.z + w * t.z, acc.w + w * t.w};
          ws += w;
        }
        store_h4(dst, (size_t)x + (size_t)nx * ((size_t)y + (size_t)ny * z), acc.x / ws,
                 acc.y / ws, acc.z / ws, acc.w / ws);
      }
}

// trace (render.wgsl:132-215): accum (res.y * res.x float4) += this
// dispatch's samples; lvA / lvB (lz, ly, lx) and gE (1, gres, gres) are the
// blurred light caches (read in light-cache mode only).
void or_render_trace(const double* rp, const uint16_t* vol, const uint16_t* sol,
                     const uint16_t* vel, const float* bricks, const float* lut,
                     const float* ecdf, const uint16_t* lvA, const uint16_t* lvB, int lx, int ly,
                     int lz, const uint16_t* gE, int gres, float* accum) {
  Ctx C;
  rp_from_rows(rp, C.R);
  const int nx = (int)C.R.dims[0], ny = (int)C.R.dims[1], nz = (int)C.R.dims[2];
  C.volT = tex_of(vol, nx, ny, nz);
  C.solT = tex_of(sol, nx, ny, nz);
  C.velT = tex_of(vel, nx, ny, nz);
  C.lvA = tex_of(lvA, lx, ly, lz);
  C.lvB = tex_of(lvB, lx, ly, lz);
  C.gE = tex_of(gE, gres, gres, 1);
  C.bricks = bricks;
  C.lut = lut;
  C.ecdf = ecdf;
  C.cache_inscatter = true;
  // pixels are independent (each seeds its own random numbers)
#pragma omp parallel for firstprivate(C) schedule(dynamic)
  for (uint32_t y = 0; y < C.R.res[1]; y++)
    for (uint32_t x = 0; x < C.R.res[0]; x++) {
      const F4 v = C.tracePixel(x, y);
      float* a = accum + 4 * ((size_t)y * C.R.res[0] + x);
      a[0] += v.x;
      a[1] += v.y;
      a[2] += v.z;
      a[3] += v.w;
    }
}

}  // extern "C"
