// pyro_oracle.cpp — CPU oracle of pyro's fire-simulation step.
//
// TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA path of
// pyro_b200 and the timed CPU baseline; the product never links, loads or
// calls it.  Only tests/, __graft_entry__.smoke() and bench.py's CPU legs use
// it.
//
// It restates, kernel by kernel, the reference's WGSL simulation shaders
// (src/shaders/common.wgsl, vel.wgsl, tmpl_comp.wgsl, tmpl_scalar.wgsl,
// advect.wgsl, fluid.wgsl, combust.wgsl, mg.wgsl, stats.wgsl) and the host
// schedule of src/sim.rs (Sim::new level hierarchy :142-168, Sim::step
// dispatch order :394-414, V-cycle :451-491).  Arithmetic is FP32 in the
// reference's expression order with WGSL builtin semantics from the WGSL
// specification: mix(a,b,t) = a*(1-t) + b*t, smoothstep(e0,e1,x) = t*t*(3-2t)
// with t = clamp((x-e0)/(e1-e0), 0, 1), clamp(x,lo,hi) = min(max(x,lo),hi),
// select(f,t,c) = c ? t : f.  Build with -ffp-contract=off so that no
// multiply-add is fused.  The reference's statistics are float atomics in an
// unspecified order (stats.wgsl:1-36); here they are FP64 sums.
//
// Pinning: the kernels are checked against golden vectors produced by
// executing the reference's own WGSL source text with an interpreter
// (tests/golden/make_golden.py); the scene tests pin the voxelizer.
//
// Also here: an FP64 Jacobi-preconditioned CG solve of the same pressure
// system (src/shaders/mg.wgsl:2,25-35) used as the pressure-error oracle.

#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "half.h"
#include <algorithm>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/pyro_sim.h"

namespace {

struct F3 { float x, y, z; };
struct F4 { float x, y, z, w; };
struct I3 { int x, y, z; };

inline F3 f3(float x, float y, float z) { return F3{x, y, z}; }
inline F3 operator+(F3 a, F3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
inline F3 operator-(F3 a, F3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
inline F3 operator*(float s, F3 a) { return f3(s * a.x, s * a.y, s * a.z); }
inline F3 operator*(F3 a, float s) { return f3(a.x * s, a.y * s, a.z * s); }
inline F3 operator/(F3 a, float s) { return f3(a.x / s, a.y / s, a.z / s); }
inline F3 f3i(I3 c) { return f3((float)c.x, (float)c.y, (float)c.z); }
inline F3 f3s(float s) { return f3(s, s, s); }
inline F4 operator+(F4 a, F4 b) { return F4{a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w}; }
inline F4 operator-(F4 a, F4 b) { return F4{a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w}; }
inline F4 operator*(float s, F4 a) { return F4{s * a.x, s * a.y, s * a.z, s * a.w}; }
inline I3 operator+(I3 a, I3 b) { return I3{a.x + b.x, a.y + b.y, a.z + b.z}; }
inline I3 operator-(I3 a, I3 b) { return I3{a.x - b.x, a.y - b.y, a.z - b.z}; }
inline I3 operator*(I3 a, int s) { return I3{a.x * s, a.y * s, a.z * s}; }

// WGSL builtins (WGSL spec, section "Numeric built-in functions").  min/max
// return the non-NaN operand when one is NaN (IEEE minNum/maxNum, what the
// GPU's fminf/fmaxf do), so a NaN can never reach an index computation.
inline float wmin(float a, float b) { return std::fmin(a, b); }
inline float wmax(float a, float b) { return std::fmax(a, b); }
inline float clampf(float x, float lo, float hi) { return wmin(wmax(x, lo), hi); }
inline float mixf(float a, float b, float t) { return a * (1.0f - t) + b * t; }
inline F4 mix4(F4 a, F4 b, float t) {
  return F4{mixf(a.x, b.x, t), mixf(a.y, b.y, t), mixf(a.z, b.z, t), mixf(a.w, b.w, t)};
}
inline F4 min4(F4 a, F4 b) { return F4{wmin(a.x, b.x), wmin(a.y, b.y), wmin(a.z, b.z), wmin(a.w, b.w)}; }
inline F4 max4(F4 a, F4 b) { return F4{wmax(a.x, b.x), wmax(a.y, b.y), wmax(a.z, b.z), wmax(a.w, b.w)}; }
inline F4 clamp4(F4 x, F4 lo, F4 hi) { return min4(max4(x, lo), hi); }
inline float smoothstepf(float e0, float e1, float x) {
  float t = clampf((x - e0) / (e1 - e0), 0.0f, 1.0f);
  return t * t * (3.0f - 2.0f * t);
}
inline float length3(F3 v) { return std::sqrt(v.x * v.x + v.y * v.y + v.z * v.z); }
inline F3 cross3(F3 a, F3 b) {
  return f3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
inline float comp(F3 v, int k) { return k == 0 ? v.x : (k == 1 ? v.y : v.z); }

const float SIGMA = 5.670374e-8f;  // common.wgsl:31
const float RGAS = 8.314f;         // common.wgsl:32
const float RHO_SOOT = 1800.0f;    // common.wgsl:33
const I3 DIRS[6] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};

// ---------------------------------------------------------------------------
// Grid context: common.wgsl:38-89
struct Ctx {
  const PyroParams* P;
  int nx, ny, nz;
  explicit Ctx(const PyroParams* p) : P(p), nx((int)p->nx), ny((int)p->ny), nz((int)p->nz) {}
  I3 dims() const { return I3{nx, ny, nz}; }
  bool inb(I3 c) const { return c.x >= 0 && c.y >= 0 && c.z >= 0 && c.x < nx && c.y < ny && c.z < nz; }
  size_t sidx(I3 c) const { return (size_t)c.x + (size_t)nx * ((size_t)c.y + (size_t)ny * (size_t)c.z); }
  size_t vidx(I3 c) const {
    return (size_t)c.x + (size_t)(nx + 1) * ((size_t)c.y + (size_t)(ny + 1) * (size_t)c.z);
  }
  I3 clampC(I3 c) const {
    return I3{std::min(std::max(c.x, 0), nx - 1), std::min(std::max(c.y, 0), ny - 1),
              std::min(std::max(c.z, 0), nz - 1)};
  }
  static float pow4(float x) { float y = x * x; return y * y; }
  float rhoOf(float T) const { return P->rho0 * P->t0 / wmax(T, 200.0f); }
  float kapP(float T, float yo, float ys) const {
    float fv = rhoOf(T) * wmax(ys, 0.0f) / RHO_SOOT;
    return 1862.0f * fv * T + P->kap_gas * clampf(1.0f - yo / P->yo2, 0.0f, 1.0f);
  }
  static float cpOf(float T) { return clampf(1000.0f + 0.24f * (T - 300.0f), 1000.0f, 1450.0f); }
  F4 ambient0() const { return F4{P->t0, 0.0f, P->yo2, 0.0f}; }
  static F3 compOff(int k) {
    if (k == 0) return f3(0.0f, 0.5f, 0.5f);
    if (k == 1) return f3(0.5f, 0.0f, 0.5f);
    return f3(0.5f, 0.5f, 0.0f);
  }
  I3 compHi(int k) const {
    I3 d{nx - 1, ny - 1, nz - 1};
    if (k == 0) return I3{d.x + 1, d.y, d.z};
    if (k == 1) return I3{d.x, d.y + 1, d.z};
    return I3{d.x, d.y, d.z + 1};
  }
  bool compValid(int k, I3 c) const {
    I3 h = compHi(k);
    return c.x >= 0 && c.y >= 0 && c.z >= 0 && c.x <= h.x && c.y <= h.y && c.z <= h.z;
  }
  static I3 unitI(int k) {
    if (k == 0) return I3{1, 0, 0};
    if (k == 1) return I3{0, 1, 0};
    return I3{0, 0, 1};
  }
  float outside(F3 gc) const {
    F3 d = f3((float)nx, (float)ny, (float)nz);
    return wmax(wmax(-0.5f - gc.x, gc.x - (d.x - 0.5f)),
                wmax(wmax(-0.5f - gc.z, gc.z - (d.z - 0.5f)), gc.y - (d.y - 0.5f)));
  }
  float spongeSide(I3 c) const {
    float e = (float)std::min(std::min(c.x, nx - 1 - c.x), std::min(c.z, nz - 1 - c.z));
    return 1.0f - smoothstepf(0.0f, P->sponge, e);
  }
  float spongeTop(I3 c) const {
    float h = (float)ny;
    return smoothstepf(h - 1.5f * P->sponge, h - 1.0f, (float)c.y);
  }

  // tmpl_comp.wgsl:2-15 — trilinear sample of a staggered component.
  float triC(const float* X, F3 g0, I3 hi) const {
    F3 g = f3(clampf(g0.x, 0.0f, (float)hi.x), clampf(g0.y, 0.0f, (float)hi.y),
              clampf(g0.z, 0.0f, (float)hi.z));
    I3 b{std::min((int)std::floor(g.x), hi.x - 1), std::min((int)std::floor(g.y), hi.y - 1),
         std::min((int)std::floor(g.z), hi.z - 1)};
    F3 f = g - f3i(b);
    size_t sy = (size_t)(nx + 1), sz = (size_t)(nx + 1) * (size_t)(ny + 1);
    size_t i = vidx(b);
    float c00 = mixf(X[i], X[i + 1], f.x);
    float c10 = mixf(X[i + sy], X[i + sy + 1], f.x);
    float c01 = mixf(X[i + sz], X[i + sz + 1], f.x);
    float c11 = mixf(X[i + sy + sz], X[i + sy + sz + 1], f.x);
    return mixf(mixf(c00, c10, f.y), mixf(c01, c11, f.y), f.z);
  }
  // tmpl_comp.wgsl:16-25 — 8-corner min/max of the backtrace cell.
  void mmC(const float* X, F3 g0, I3 hi, float* lo, float* hiv) const {
    F3 g = f3(clampf(g0.x, 0.0f, (float)hi.x), clampf(g0.y, 0.0f, (float)hi.y),
              clampf(g0.z, 0.0f, (float)hi.z));
    I3 b{std::min((int)std::floor(g.x), hi.x - 1), std::min((int)std::floor(g.y), hi.y - 1),
         std::min((int)std::floor(g.z), hi.z - 1)};
    float rl = 1e30f, rh = -1e30f;
    for (int j = 0; j < 8; j++) {
      float v = X[vidx(b + I3{j & 1, (j >> 1) & 1, (j >> 2) & 1})];
      rl = wmin(rl, v);
      rh = wmax(rh, v);
    }
    *lo = rl;
    *hiv = rh;
  }
  // tmpl_scalar.wgsl:2-15 — trilinear sample of a cell-centred vec4 field.
  F4 triS(const F4* X, F3 gc0) const {
    F3 g = f3(clampf(gc0.x, 0.0f, (float)(nx - 1)), clampf(gc0.y, 0.0f, (float)(ny - 1)),
              clampf(gc0.z, 0.0f, (float)(nz - 1)));
    I3 b{std::min((int)std::floor(g.x), nx - 2), std::min((int)std::floor(g.y), ny - 2),
         std::min((int)std::floor(g.z), nz - 2)};
    F3 f = g - f3i(b);
    size_t sy = (size_t)nx, sz = (size_t)nx * (size_t)ny;
    size_t i = sidx(b);
    F4 c00 = mix4(X[i], X[i + 1], f.x);
    F4 c10 = mix4(X[i + sy], X[i + sy + 1], f.x);
    F4 c01 = mix4(X[i + sz], X[i + sz + 1], f.x);
    F4 c11 = mix4(X[i + sy + sz], X[i + sy + sz + 1], f.x);
    return mix4(mix4(c00, c10, f.y), mix4(c01, c11, f.y), f.z);
  }
  // tmpl_scalar.wgsl:16-19 — ambient value outside the open boundary.
  F4 advS(const F4* X, F3 gc, F4 amb) const {
    return mix4(triS(X, gc), amb, clampf(outside(gc), 0.0f, 1.0f));
  }
  // tmpl_scalar.wgsl:20-32
  void mmS(const F4* X, F3 gc0, F4* lo, F4* hi) const {
    F3 g = f3(clampf(gc0.x, 0.0f, (float)(nx - 1)), clampf(gc0.y, 0.0f, (float)(ny - 1)),
              clampf(gc0.z, 0.0f, (float)(nz - 1)));
    I3 b{std::min((int)std::floor(g.x), nx - 2), std::min((int)std::floor(g.y), ny - 2),
         std::min((int)std::floor(g.z), nz - 2)};
    F4 l{1e30f, 1e30f, 1e30f, 1e30f}, h{-1e30f, -1e30f, -1e30f, -1e30f};
    for (int j = 0; j < 8; j++) {
      F4 v = X[sidx(b + I3{j & 1, (j >> 1) & 1, (j >> 2) & 1})];
      l = min4(l, v);
      h = max4(h, v);
    }
    *lo = l;
    *hi = h;
  }
  // vel.wgsl:2-19 — velocity sample and RK2 traces.
  F3 velAt(const float* vu, const float* vv, const float* vw, F3 p) const {
    return f3(triC(vu, p - compOff(0), compHi(0)), triC(vv, p - compOff(1), compHi(1)),
              triC(vw, p - compOff(2), compHi(2)));
  }
  F3 traceBack(const float* vu, const float* vv, const float* vw, F3 x) const {
    float k = P->dt / P->dx;
    F3 u1 = velAt(vu, vv, vw, x);
    F3 u2 = velAt(vu, vv, vw, x - (0.5f * k) * u1);
    return x - k * u2;
  }
  F3 traceFwd(const float* vu, const float* vv, const float* vw, F3 x) const {
    float k = P->dt / P->dx;
    F3 u1 = velAt(vu, vv, vw, x);
    F3 u2 = velAt(vu, vv, vw, x + (0.5f * k) * u1);
    return x + k * u2;
  }
};

// Statistics accumulator (stats.wgsl): FP64 sums and maxima.
struct Stats {
  double v[PYRO_STATS_N];
  void clear() { std::memset(v, 0, sizeof(v)); }
};

#define OR_PARALLEL_Z _Pragma("omp parallel for schedule(static)")

// ---------------------------------------------------------------------------
// combust.wgsl:3-137 — solid surface energy balance, pyrolysis, burnout.
struct SolidK {
  const Ctx& C;
  const F4* solIn;
  const F4* s0;
  // out-of-range slots clamp to the last row (restricted array indexing)
  static uint32_t slotOf(F4 s) { return s.x <= 0.0f ? 0u : std::min((uint32_t)s.x, 7u); }
  uint32_t kindOf(F4 s) const { return (uint32_t)(C.P->mats[slotOf(s)][3] + 0.5f); }
  bool isSolidS(F4 s) const {
    if (kindOf(s) == 2u) return s.y > 0.5f;
    return s.y + s.z > C.P->burnout;
  }
  bool solidN(I3 c) const {
    if (!C.inb(c)) return false;
    return isSolidS(solIn[C.sidx(c)]);
  }
  float rayIrr(I3 c0, I3 d) const {
    static const int strides[10] = {1, 1, 1, 2, 2, 3, 4, 5, 7, 9};
    I3 p = c0;
    float tr = 1.0f, acc = 0.0f;
    float dl = length3(f3i(d)) * C.P->dx;
    for (int s = 0; s < 10; s++) {
      if (!C.inb(p)) break;
      size_t j = C.sidx(p);
      F4 so = solIn[j];
      if (isSolidS(so)) {
        acc += tr * Ctx::pow4(so.w);
        tr = 0.0f;
        break;
      }
      F4 g = s0[j];
      float T = g.x;
      float len = (float)strides[s] * dl;
      float e = 1.0f - std::exp(-C.kapP(T, g.z, g.w) * len);
      acc += tr * e * Ctx::pow4(T);
      tr *= 1.0f - e;
      p = p + d * strides[s];
    }
    acc += tr * Ctx::pow4(C.P->t0);
    return SIGMA * acc;
  }
  float faceIrr(I3 c0, int k) const {
    I3 d = DIRS[k];
    I3 t1{0, 1, 0}, t2{0, 0, 1};
    if (d.y != 0) t1 = I3{1, 0, 0};
    if (d.z != 0) t2 = I3{1, 0, 0};
    return 0.2f * (rayIrr(c0, d) + rayIrr(c0, d + t1) + rayIrr(c0, d - t1) + rayIrr(c0, d + t2) +
                   rayIrr(c0, d - t2));
  }
  // One cell; returns (pyro, mass, area) contributions.
  void cell(I3 c, F4* solOut, F4* pyr, uint32_t* flags, double* st) const {
    const PyroParams* P = C.P;
    size_t i = C.sidx(c);
    F4 s = solIn[i];
    F4 o = s;
    F4 po{0, 0, 0, 0};
    uint32_t fl = 0;
    float stPyro = 0, stMass = 0, stArea = 0;
    if (isSolidS(s)) {
      fl = 1;
      const float* m = P->mats[slotOf(s)];
      // m[0..3] = a, m[4..7] = b, m[8..11] = c
      uint32_t kind = kindOf(s);
      float fuel = s.y, chr = s.z, Ts = s.w;
      if (kind != 2u) {
        float nF = 0, Tg = 0, Yo = 0, qin = 0, qcond = 0;
        for (int k = 0; k < 6; k++) {
          I3 n = c + DIRS[k];
          if (n.y < 0) continue;
          if (solidN(n)) {
            qcond += m[7] / P->dx * (solIn[C.sidx(n)].w - Ts);
            continue;
          }
          nF += 1.0f;
          if (C.inb(n)) {
            F4 g = s0[C.sidx(n)];
            Tg += g.x;
            Yo += g.z;
            qin += faceIrr(n, k);
          } else {
            Tg += P->t0;
            Yo += P->yo2;
            qin += SIGMA * Ctx::pow4(P->t0);
          }
        }
        float layer = (kind == 1u) ? 0.001f : wmin(P->layer, P->dx);
        float cap = m[0] * m[6] * layer;
        if (nF > 0.0f) {
          Tg /= nF;
          Yo /= nF;
          qin /= nF;
          float qnet = m[5] * (qin - SIGMA * Ctx::pow4(Ts)) + P->h_conv * (Tg - Ts) + qcond / nF;
          if (P->ign_on > 0.5f) {
            float dI = length3((f3i(c) + f3s(0.5f)) * P->dx - f3(P->ign_x, P->ign_y, P->ign_z));
            qnet += P->ign_flux * clampf(1.0f - dI / (1.5f * P->ign_r), 0.0f, 1.0f);
          }
          float mv = 0, mc = 0;
          if (kind == 1u) {
            float Tb = m[2];
            mv = smoothstepf(Tb - 60.0f, Tb, Ts) * wmax(qnet, 0.0f) / m[1] * m[9];
            Ts = wmin(Ts + P->dt * wmax(qnet - mv * m[1], wmin(qnet, 0.0f)) / cap, Tb);
            fuel -= mv * nF / P->dx * P->dt;
          } else {
            if (fuel > 0.0f) {
              mv = smoothstepf(m[2] - 20.0f, m[2] + 30.0f, Ts) * wmax(qnet, 0.0f) / m[1] * m[9];
            }
            float chi = (kind == 0u) ? m[4] : 0.0f;
            float kin = P->char_a * std::exp(-P->char_e / (RGAS * Ts)) * chr * layer;
            float dif = P->h_mass * C.rhoOf(Tg) * Yo / 1.33f;
            mc = wmin(kin, dif);
            Ts += P->dt * (qnet - mv * m[1] + 0.5f * mc * P->dh_char) / cap;
            float virgin = wmin(mv / (1.0f - chi) * nF / P->dx * P->dt, fuel);
            fuel -= virgin;
            chr += virgin * chi - mc * nF / P->dx * P->dt;
          }
          stPyro = mv * nF * P->dx * P->dx;
          stArea = (mv > 1e-4f) ? nF * P->dx * P->dx : 0.0f;
          po = F4{mv, mc, nF, 0.0f};
        } else {
          Ts += P->dt * qcond / (m[0] * m[6] * P->dx);
        }
        Ts = clampf(Ts, 250.0f, 2000.0f);
        fuel = wmax(fuel, 0.0f);
        chr = wmax(chr, 0.0f);
        o = F4{s.x, fuel, chr, Ts};
        if (fuel + chr <= P->burnout) {
          o = F4{0.0f, 0.0f, 0.0f, P->t0};
          fl = 0;
          po = F4{0, 0, 0, 0};
        }
      }
      stMass = (o.y + o.z) * P->dx * P->dx * P->dx * ((kind == 2u) ? 0.0f : 1.0f);
    }
    solOut[i] = o;
    pyr[i] = po;
    flags[i] = fl;
    st[0] += stPyro;
    st[1] += stMass;
    st[2] += stArea;
  }
};

void k_solid(const Ctx& C, const F4* solIn, F4* solOut, F4* pyr, uint32_t* flags, const F4* s0,
             Stats* stats) {
  SolidK K{C, solIn, s0};
  double a = 0, b = 0, d = 0;
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : a, b, d)
  for (int z = 0; z < C.nz; z++)
    for (int y = 0; y < C.ny; y++)
      for (int x = 0; x < C.nx; x++) {
        double st[3] = {0, 0, 0};
        K.cell(I3{x, y, z}, solOut, pyr, flags, st);
        a += st[0];
        b += st[1];
        d += st[2];
      }
  if (stats) {
    stats->v[2] += a;
    stats->v[7] += b;
    stats->v[9] += d;
  }
}

// fluid.wgsl:3-29 — cell-centred vorticity and max speed.
void k_curl(const Ctx& C, const float* vu, const float* vv, const float* vw, F4* curl,
            Stats* stats) {
  auto uc = [&](I3 c0) {
    I3 c = C.clampC(c0);
    I3 X{1, 0, 0}, Y{0, 1, 0}, Z{0, 0, 1};
    return 0.5f * f3(vu[C.vidx(c)] + vu[C.vidx(c + X)], vv[C.vidx(c)] + vv[C.vidx(c + Y)],
                     vw[C.vidx(c)] + vw[C.vidx(c + Z)]);
  };
  double mx = 0;
#pragma omp parallel for schedule(static) reduction(max : mx)
  for (int z = 0; z < C.nz; z++)
    for (int y = 0; y < C.ny; y++)
      for (int x = 0; x < C.nx; x++) {
        I3 c{x, y, z};
        I3 X{1, 0, 0}, Y{0, 1, 0}, Z{0, 0, 1};
        F3 w = f3((uc(c + Y).z - uc(c - Y).z) - (uc(c + Z).y - uc(c - Z).y),
                  (uc(c + Z).x - uc(c - Z).x) - (uc(c + X).z - uc(c - X).z),
                  (uc(c + X).y - uc(c - X).y) - (uc(c + Y).x - uc(c - Y).x)) /
               (2.0f * C.P->dx);
        curl[C.sidx(c)] = F4{w.x, w.y, w.z, length3(w)};
        float spd = length3(uc(c));
        mx = std::max(mx, (double)wmax(spd, 0.0f));
      }
  if (stats) stats->v[5] = std::max(stats->v[5], mx);
}

// advect.wgsl:4-20 — semi-Lagrangian predictor of the staggered velocity.
void k_adv_vel1(const Ctx& C, const float* vu, const float* vv, const float* vw, float* hu,
                float* hv, float* hw) {
  float* H[3] = {hu, hv, hw};
  const float* V[3] = {vu, vv, vw};
#pragma omp parallel for schedule(static)
  for (int z = 0; z <= C.nz; z++)
    for (int y = 0; y <= C.ny; y++)
      for (int x = 0; x <= C.nx; x++) {
        I3 c{x, y, z};
        size_t i = C.vidx(c);
        for (int k = 0; k < 3; k++) {
          if (!C.compValid(k, c)) continue;
          F3 off = Ctx::compOff(k);
          H[k][i] = C.triC(V[k], C.traceBack(vu, vv, vw, f3i(c) + off) - off, C.compHi(k));
        }
      }
}

// advect.wgsl:22-70 — MacCormack corrector with the 8-corner limiter.
void k_adv_vel2(const Ctx& C, const float* vu, const float* vv, const float* vw, const float* hu,
                const float* hv, const float* hw, float* ou, float* ov, float* ow,
                const uint32_t* flags) {
  const float* V[3] = {vu, vv, vw};
  const float* H[3] = {hu, hv, hw};
  float* O[3] = {ou, ov, ow};
  auto solidAt = [&](I3 c) { return C.inb(c) && flags[C.sidx(c)] == 1u; };
#pragma omp parallel for schedule(static)
  for (int z = 0; z <= C.nz; z++)
    for (int y = 0; y <= C.ny; y++)
      for (int x = 0; x <= C.nx; x++) {
        I3 c{x, y, z};
        size_t i = C.vidx(c);
        for (int k = 0; k < 3; k++) {
          if (!C.compValid(k, c)) continue;
          bool blocked = (k == 1 && c.y == 0) || solidAt(c) || solidAt(c - Ctx::unitI(k));
          if (blocked) {
            O[k][i] = 0.0f;
            continue;
          }
          F3 off = Ctx::compOff(k);
          I3 hi = C.compHi(k);
          F3 xx = f3i(c) + off;
          F3 b = C.traceBack(vu, vv, vw, xx) - off;
          F3 f = C.traceFwd(vu, vv, vw, xx) - off;
          float lo, hv2;
          C.mmC(V[k], b, hi, &lo, &hv2);
          O[k][i] = clampf(H[k][i] + 0.5f * (V[k][i] - C.triC(H[k], f, hi)), lo, hv2);
        }
      }
}

// advect.wgsl:72-91 — scalar predictor.
void k_adv_s1(const Ctx& C, const float* vu, const float* vv, const float* vw, const F4* s0,
              const F4* s1, F4* h0, F4* h1) {
#pragma omp parallel for schedule(static)
  for (int z = 0; z < C.nz; z++)
    for (int y = 0; y < C.ny; y++)
      for (int x = 0; x < C.nx; x++) {
        I3 c{x, y, z};
        size_t i = C.sidx(c);
        F3 b = C.traceBack(vu, vv, vw, f3i(c) + f3s(0.5f)) - f3s(0.5f);
        h0[i] = C.advS(s0, b, C.ambient0());
        h1[i] = C.advS(s1, b, F4{0, 0, 0, 0});
      }
}

// advect.wgsl:93-125 — scalar corrector (first order when a trace leaves).
void k_adv_s2(const Ctx& C, const float* vu, const float* vv, const float* vw, const F4* s0,
              const F4* s1, const F4* h0, const F4* h1, F4* o0, F4* o1) {
#pragma omp parallel for schedule(static)
  for (int z = 0; z < C.nz; z++)
    for (int y = 0; y < C.ny; y++)
      for (int x = 0; x < C.nx; x++) {
        I3 c{x, y, z};
        size_t i = C.sidx(c);
        F3 xx = f3i(c) + f3s(0.5f);
        F3 b = C.traceBack(vu, vv, vw, xx) - f3s(0.5f);
        F3 f = C.traceFwd(vu, vv, vw, xx) - f3s(0.5f);
        F4 r0 = h0[i], r1 = h1[i];
        if (C.outside(b) <= 0.0f && C.outside(f) <= 0.0f) {
          F4 l0, u0, l1, u1;
          C.mmS(s0, b, &l0, &u0);
          C.mmS(s1, b, &l1, &u1);
          r0 = clamp4(r0 + 0.5f * (s0[i] - C.triS(h0, f)), l0, u0);
          r1 = clamp4(r1 + 0.5f * (s1[i] - C.triS(h1, f)), l1, u1);
        }
        o0[i] = r0;
        o1[i] = r1;
      }
}

// combust.wgsl:139-273 — combustion, soot, radiation, low-Mach source.
void k_react(const Ctx& C, const F4* s0in, const F4* s1in, F4* s0out, F4* s1out,
             const uint32_t* flags, const F4* sol, const F4* pyr, const F4* curl, Stats* stats) {
  const PyroParams* P = C.P;
  const float dV = P->dx * P->dx * P->dx;
  int nth = 1;
#ifdef _OPENMP
  nth = omp_get_max_threads();
#endif
  int nl = std::min(C.ny, PYRO_MAX_LAYERS);
  std::vector<double> layers((size_t)nth * nl, 0.0);
  double sH = 0, sR = 0, sS = 0, sF = 0, sM = 0, mT = 0;
#pragma omp parallel for schedule(static) reduction(+ : sH, sR, sS, sF, sM) reduction(max : mT)
  for (int z = 0; z < C.nz; z++) {
    int tid = 0;
#ifdef _OPENMP
    tid = omp_get_thread_num();
#endif
    double* lay = &layers[(size_t)tid * nl];
    for (int y = 0; y < C.ny; y++)
      for (int x = 0; x < C.nx; x++) {
        I3 c{x, y, z};
        size_t i = C.sidx(c);
        if (flags[i] == 1u) {
          s0out[i] = F4{sol[i].w, 0.0f, P->yo2, 0.0f};
          s1out[i] = F4{0, 0, 0, 0};
          continue;
        }
        F4 a = s0in[i];
        F4 b = s1in[i];
        float nut = (P->cs * P->dx) * (P->cs * P->dx) * curl[i].w;
        if (P->cs > 0.0f) {
          float kd = wmin(nut / 0.5f * P->dt / (P->dx * P->dx), 0.15f);
          F4 lapA{0, 0, 0, 0};
          float lapB = 0.0f;
          for (int k = 0; k < 6; k++) {
            I3 n = c + DIRS[k];
            if (C.inb(n)) {
              size_t j = C.sidx(n);
              if (flags[j] != 1u) {
                lapA = lapA + (s0in[j] - a);
                lapB += s1in[j].x - b.x;
              }
            } else if (n.y >= 0) {
              lapA = lapA + (C.ambient0() - a);
              lapB -= b.x;
            }
          }
          a = a + kd * lapA;
          b.x += kd * lapB;
        }
        float T = a.x;
        float yf = wmax(a.y, 0.0f);
        float yo = clampf(a.z, 0.0f, P->yo2);
        float ys = wmax(a.w, 0.0f);
        float ym = wmax(b.x, 0.0f);
        float S = 0.0f;
        for (int k = 0; k < 6; k++) {
          I3 n = c + DIRS[k];
          if (!C.inb(n)) continue;
          size_t j = C.sidx(n);
          if (flags[j] != 1u) continue;
          F4 pr = pyr[j];
          float Ts = sol[j].w;
          float rho = C.rhoOf(T);
          if (pr.x > 0.0f) {
            float dm = pr.x * P->dt / (rho * P->dx);
            float inv = 1.0f / (1.0f + dm);
            yf = (yf + dm) * inv;
            yo *= inv;
            ys *= inv;
            ym *= inv;
            T = (T + dm * Ts) * inv;
            S += pr.x / (rho * P->dx);
          }
          T += P->h_conv * (Ts - T) * P->dt / (rho * Ctx::cpOf(T) * P->dx);
          if (pr.y > 0.0f) {
            yo = wmax(yo - 1.33f * pr.y * P->dt / (rho * P->dx), 0.0f);
            T += 0.5f * P->dh_char * pr.y * P->dt / (rho * Ctx::cpOf(T) * P->dx);
          }
        }
        if (P->ign_on > 0.5f) {
          float dI = length3((f3i(c) + f3s(0.5f)) * P->dx - f3(P->ign_x, P->ign_y, P->ign_z));
          float w = clampf(1.0f - dI / P->ign_r, 0.0f, 1.0f);
          if (w > 0.0f) {
            T = wmax(T, mixf(P->t0, P->ign_temp, smoothstepf(0.0f, 0.5f, w)));
            yf += P->ign_fuel * w * P->dt;
          }
        }
        float rho = C.rhoOf(T);
        float tauU = 0.049f * P->dx * P->dx / (nut + 1e-6f);
        float tauG = std::sqrt(2.0f * P->dx / P->g);
        float tau = wmax(wmin(tauU, tauG), P->tau_min);
        float gate = smoothstepf(P->t_ign - 100.0f, P->t_ign + 100.0f, T);
        float lim = wmin(yf, yo / P->s_o2);
        float dY = lim * (1.0f - std::exp(-gate * P->dt / tau));
        yf -= dY;
        yo = wmax(yo - P->s_o2 * dY, 0.0f);
        T += dY * P->dhc / Ctx::cpOf(T + 0.5f * dY * P->dhc / Ctx::cpOf(T));
        float q = rho * dY * P->dhc / P->dt;
        float rich = smoothstepf(0.0f, 0.03f, yf);
        ys += P->soot_form * dY * (0.25f + 0.75f * rich);
        float oxg = smoothstepf(P->soot_ox_t, P->soot_ox_t + 300.0f, T) * (yo / P->yo2);
        ys *= std::exp(-P->soot_ox * oxg * P->dt);
        float cold = 1.0f - smoothstepf(450.0f, 650.0f, T);
        float cv = yf * wmin(P->smoke_conv * cold * P->dt, 1.0f);
        yf -= cv;
        ym += cv;
        rho = C.rhoOf(T);
        float kap = C.kapP(T, yo, ys);
        float tl = kap * P->rad_len;
        float esc = (tl > 1e-3f) ? (1.0f - std::exp(-tl)) / tl : 1.0f;
        float prad = 4.0f * kap * esc * SIGMA * (Ctx::pow4(T) - Ctx::pow4(P->t0));
        float dTr = wmin(prad * P->dt / (rho * Ctx::cpOf(T)), 0.5f * wmax(T - P->t0, 0.0f));
        T -= dTr;
        float prl = dTr * rho * Ctx::cpOf(T) / P->dt;
        S += (q - prl) / (rho * Ctx::cpOf(T) * T);
        float sp = wmax(C.spongeSide(c), C.spongeTop(c));
        float dec = 1.0f - std::exp(-P->dt * 4.0f * sp);
        T = mixf(T, P->t0, dec);
        yf *= 1.0f - dec;
        yo = mixf(yo, P->yo2, dec);
        ys *= 1.0f - dec;
        ym *= 1.0f - dec;
        T = clampf(T, 250.0f, 2600.0f);
        s0out[i] = F4{T, yf, yo, ys};
        s1out[i] = F4{ym, q, S, 0.0f};
        rho = C.rhoOf(T);
        float stH = q * dV;
        sH += stH;
        sR += prl * dV;
        sS += rho * ys * dV;
        sF += rho * yf * dV;
        sM += rho * ym * dV;
        mT = std::max(mT, (double)T);
        if (stH > 1.0f && y < nl) lay[y] += stH;
      }
  }
  if (stats) {
    stats->v[0] += sH;
    stats->v[1] += sR;
    stats->v[3] += sS;
    stats->v[6] += sF;
    stats->v[8] += sM;
    stats->v[4] = std::max(stats->v[4], mT);
    for (int t = 0; t < nth; t++)
      for (int y = 0; y < nl; y++) stats->v[16 + y] += layers[(size_t)t * nl + y];
  }
}

// fluid.wgsl:31-109 — buoyancy, vorticity confinement, wind, sponge, clamp.
void k_forces(const Ctx& C, float* vu, float* vv, float* vw, const F4* s0, const F4* s1,
              const F4* curl, const uint32_t* flags) {
  const PyroParams* P = C.P;
  float* V[3] = {vu, vv, vw};
  auto solidAt = [&](I3 c) { return C.inb(c) && flags[C.sidx(c)] == 1u; };
  auto cm = [&](I3 c) { return curl[C.sidx(C.clampC(c))].w; };
  auto confine = [&](I3 c) -> F3 {
    size_t i = C.sidx(c);
    float T = s0[i].x;
    float smoke = s0[i].w + s1[i].x;
    float gate = wmax(smoothstepf(P->vort_t, P->vort_t + 500.0f, T),
                      0.35f * smoothstepf(0.0f, 2e-4f, smoke));
    if (gate <= 0.0f) return f3(0, 0, 0);
    I3 X{1, 0, 0}, Y{0, 1, 0}, Z{0, 0, 1};
    F3 gr = f3(cm(c + X) - cm(c - X), cm(c + Y) - cm(c - Y), cm(c + Z) - cm(c - Z));
    float gl = length3(gr);
    if (gl < 1e-6f) return f3(0, 0, 0);
    F4 cw = curl[i];
    F3 f = (P->vort * P->dx) * cross3(gr / gl, f3(cw.x, cw.y, cw.z)) * gate;
    float fl = length3(f);
    if (fl > 60.0f) f = f * (60.0f / fl);
    return f;
  };
  auto windVel = [&](int k) { return k == 0 ? P->wind_x : (k == 2 ? P->wind_z : 0.0f); };
#pragma omp parallel for schedule(static)
  for (int z = 0; z <= C.nz; z++)
    for (int y = 0; y <= C.ny; y++)
      for (int x = 0; x <= C.nx; x++) {
        I3 c{x, y, z};
        size_t i = C.vidx(c);
        for (int k = 0; k < 3; k++) {
          if (!C.compValid(k, c)) continue;
          I3 a = c - Ctx::unitI(k);
          if ((k == 1 && c.y == 0) || solidAt(c) || solidAt(a)) continue;
          bool ia = C.inb(a), ib = C.inb(c);
          float f = 0.0f;
          if (k == 1) {
            float Ta = P->t0, Tb = P->t0, ma = 0.0f, mb = 0.0f;
            if (ia) { F4 s = s0[C.sidx(a)]; Ta = s.x; ma = s.w + s1[C.sidx(a)].x; }
            if (ib) { F4 s = s0[C.sidx(c)]; Tb = s.x; mb = s.w + s1[C.sidx(c)].x; }
            if (!ia) { Ta = Tb; ma = mb; }
            if (!ib) { Tb = Ta; mb = ma; }
            float Tf = 0.5f * (Ta + Tb);
            f += P->g * P->buoy * (Tf - P->t0) / Tf - P->g * P->smoke_w * 0.5f * (ma + mb);
          }
          F3 fc = f3(0, 0, 0);
          float n = 0.0f;
          if (ia) { fc = fc + confine(a); n += 1.0f; }
          if (ib) { fc = fc + confine(c); n += 1.0f; }
          if (n > 0.0f) f += comp(fc, k) / n;
          float u = V[k][i];
          u += f * P->dt;
          I3 cc = C.clampC(c);
          float ss = C.spongeSide(cc);
          if (k != 1) {
            float Tl = P->t0;
            if (ib) Tl = s0[C.sidx(c)].x;
            float hot = smoothstepf(350.0f, 900.0f, Tl);
            float kr = P->wind_relax * (1.0f - 0.85f * hot) + 8.0f * ss;
            u = mixf(u, windVel(k), 1.0f - std::exp(-kr * P->dt));
          } else {
            float st = C.spongeTop(cc);
            if (st > 0.0f) u = mixf(u, wmax(u, 0.0f), 1.0f - std::exp(-8.0f * st * P->dt));
          }
          u = clampf(u, -40.0f, 40.0f);
          V[k][i] = u;
        }
      }
}

// fluid.wgsl:111-128 — b = div u - S, 0 in solids.
void k_divergence(const Ctx& C, const float* vu, const float* vv, const float* vw, const F4* s1,
                  const uint32_t* flags, float* b) {
#pragma omp parallel for schedule(static)
  for (int z = 0; z < C.nz; z++)
    for (int y = 0; y < C.ny; y++)
      for (int x = 0; x < C.nx; x++) {
        I3 c{x, y, z};
        size_t i = C.sidx(c);
        if (flags[i] == 1u) { b[i] = 0.0f; continue; }
        I3 X{1, 0, 0}, Y{0, 1, 0}, Z{0, 0, 1};
        float d = (vu[C.vidx(c + X)] - vu[C.vidx(c)] + vv[C.vidx(c + Y)] - vv[C.vidx(c)] +
                   vw[C.vidx(c + Z)] - vw[C.vidx(c)]) /
                  C.P->dx;
        b[i] = d - s1[i].z;
      }
}

// fluid.wgsl:130-152 — u -= grad phi; blocked faces 0; phi = 0 outside.
void k_project(const Ctx& C, float* vu, float* vv, float* vw, const float* phi,
               const uint32_t* flags) {
  float* V[3] = {vu, vv, vw};
  auto solidAt = [&](I3 c) { return C.inb(c) && flags[C.sidx(c)] == 1u; };
  auto ph = [&](I3 c) { return C.inb(c) ? phi[C.sidx(c)] : 0.0f; };
#pragma omp parallel for schedule(static)
  for (int z = 0; z <= C.nz; z++)
    for (int y = 0; y <= C.ny; y++)
      for (int x = 0; x <= C.nx; x++) {
        I3 c{x, y, z};
        size_t i = C.vidx(c);
        for (int k = 0; k < 3; k++) {
          if (!C.compValid(k, c)) continue;
          I3 a = c - Ctx::unitI(k);
          float u = 0.0f;
          if (!((k == 1 && c.y == 0) || solidAt(c) || solidAt(a))) {
            u = V[k][i];
            u -= (ph(c) - ph(a)) / C.P->dx;
          }
          V[k][i] = u;
        }
      }
}

// ---------------------------------------------------------------------------
// mg.wgsl — multigrid level kernels.  bc_mode 0: Dirichlet sides and top,
// Neumann floor (the reference); 1: Dirichlet top only.
struct Lv { int nx, ny, nz; float h; };
inline bool inbL(I3 c, const Lv& d) {
  return c.x >= 0 && c.y >= 0 && c.z >= 0 && c.x < d.nx && c.y < d.ny && c.z < d.nz;
}
inline size_t idxL(I3 c, const Lv& d) {
  return (size_t)c.x + (size_t)d.nx * ((size_t)c.y + (size_t)d.ny * (size_t)c.z);
}
// Outside-domain neighbour: counts (Dirichlet) unless bc_mode 1 and it is a
// side neighbour.
inline bool dirichletOut(I3 n, const Lv& d, int bc_mode) {
  if (bc_mode == 0) return true;
  return n.y >= d.ny;
}

// mg.wgsl:5-36 (sum/cnt loop; one colour)
void mg_smooth(const Lv& d, const float* b, const uint32_t* f, float* p, int color, float omega,
               int bc_mode) {
#pragma omp parallel for schedule(static)
  for (int z = 0; z < d.nz; z++)
    for (int y = 0; y < d.ny; y++)
      for (int x = ((y + z + color) & 1); x < d.nx; x += 2) {
        I3 c{x, y, z};
        size_t i = idxL(c, d);
        if (f[i] == 1u) continue;
        float sum = 0.0f, cnt = 0.0f;
        for (int k = 0; k < 6; k++) {
          I3 n = c + DIRS[k];
          if (n.y < 0) continue;
          if (!inbL(n, d)) {
            if (dirichletOut(n, d, bc_mode)) cnt += 1.0f;
            continue;
          }
          size_t j = idxL(n, d);
          if (f[j] == 1u) continue;
          sum += p[j];
          cnt += 1.0f;
        }
        if (cnt < 0.5f) continue;
        p[i] = mixf(p[i], (sum - d.h * d.h * b[i]) / cnt, omega);
      }
}

// mg.wgsl:52-66 — fine residual of one cell.
inline float mg_resid_cell(const Lv& d, const float* p, const float* b, const uint32_t* f, I3 c,
                           int bc_mode) {
  size_t i = idxL(c, d);
  if (f[i] == 1u) return 0.0f;
  float pcen = p[i];
  float sum = 0.0f, cnt = 0.0f;
  for (int k = 0; k < 6; k++) {
    I3 n = c + DIRS[k];
    if (n.y < 0) continue;
    if (!inbL(n, d)) {
      if (dirichletOut(n, d, bc_mode)) cnt += 1.0f;
      continue;
    }
    size_t j = idxL(n, d);
    if (f[j] == 1u) continue;
    sum += p[j];
    cnt += 1.0f;
  }
  return b[i] - (sum - cnt * pcen) / (d.h * d.h);
}

// mg.wgsl:38-83
void mg_restrict(const Lv& df, const float* pf, const float* bf, const uint32_t* ff, const Lv& dc,
                 float* bc, float* pc, uint32_t* fc, int bc_mode) {
#pragma omp parallel for schedule(static)
  for (int z = 0; z < dc.nz; z++)
    for (int y = 0; y < dc.ny; y++)
      for (int x = 0; x < dc.nx; x++) {
        I3 c{x, y, z};
        float r = 0.0f, nfl = 0.0f;
        for (int k = 0; k < 8; k++) {
          I3 ch = c * 2 + I3{k & 1, (k >> 1) & 1, (k >> 2) & 1};
          if (!inbL(ch, df)) continue;
          if (ff[idxL(ch, df)] != 1u) {
            nfl += 1.0f;
            r += mg_resid_cell(df, pf, bf, ff, ch, bc_mode);
          }
        }
        size_t i = idxL(c, dc);
        bc[i] = (nfl > 0.0f) ? r / wmax(nfl, 1.0f) : 0.0f;
        pc[i] = 0.0f;
        fc[i] = (nfl > 0.0f) ? 0u : 1u;
      }
}

// mg.wgsl:85-120
void mg_prolong(const Lv& df, const float* pc, const uint32_t* ff, float* pf, const Lv& dc,
                const uint32_t* fc) {
#pragma omp parallel for schedule(static)
  for (int z = 0; z < df.nz; z++)
    for (int y = 0; y < df.ny; y++)
      for (int x = 0; x < df.nx; x++) {
        I3 c{x, y, z};
        size_t i = idxL(c, df);
        if (ff[i] == 1u) continue;
        F3 xx = (f3i(c) + f3s(0.5f)) * 0.5f - f3s(0.5f);
        I3 i0{(int)std::floor(xx.x), (int)std::floor(xx.y), (int)std::floor(xx.z)};
        F3 fr = xx - f3i(i0);
        float acc = 0.0f, ws = 0.0f;
        for (int k = 0; k < 8; k++) {
          I3 o{k & 1, (k >> 1) & 1, (k >> 2) & 1};
          I3 cc{std::min(std::max(i0.x + o.x, 0), dc.nx - 1),
                std::min(std::max(i0.y + o.y, 0), dc.ny - 1),
                std::min(std::max(i0.z + o.z, 0), dc.nz - 1)};
          size_t j = idxL(cc, dc);
          if (fc[j] == 1u) continue;
          float wx = o.x == 1 ? fr.x : 1.0f - fr.x;
          float wy = o.y == 1 ? fr.y : 1.0f - fr.y;
          float wz = o.z == 1 ? fr.z : 1.0f - fr.z;
          float w = wx * wy * wz;
          acc += w * pc[j];
          ws += w;
        }
        if (ws > 1e-4f) pf[i] += acc / ws;
      }
}

// mg.wgsl:122-158 — sums of r^2 and b^2 (FP64 here).
void mg_resid_sums(const Lv& d, const float* p, const float* b, const uint32_t* f, int bc_mode,
                   double* r2o, double* b2o) {
  double r2 = 0, b2 = 0;
#pragma omp parallel for schedule(static) reduction(+ : r2, b2)
  for (int z = 0; z < d.nz; z++)
    for (int y = 0; y < d.ny; y++)
      for (int x = 0; x < d.nx; x++) {
        I3 c{x, y, z};
        size_t i = idxL(c, d);
        if (f[i] == 1u) continue;
        float r = mg_resid_cell(d, p, b, f, c, bc_mode);
        r2 += (double)(r * r);
        b2 += (double)(b[i] * b[i]);
      }
  *r2o = r2;
  *b2o = b2;
}

// src/sim.rs:142-168 — level dimensions.
std::vector<Lv> build_levels(int nx, int ny, int nz, float h, int max_levels) {
  std::vector<Lv> v;
  Lv d{nx, ny, nz, h};
  for (int l = 0; l < max_levels; l++) {
    v.push_back(d);
    if (std::min(std::min(d.nx, d.ny), d.nz) < 16) break;
    d.nx = (d.nx + 1) / 2;
    d.ny = (d.ny + 1) / 2;
    d.nz = (d.nz + 1) / 2;
    d.h *= 2.0f;
  }
  return v;
}

struct Hier {
  std::vector<Lv> lv;
  std::vector<std::vector<float>> phi, b;
  std::vector<std::vector<uint32_t>> f;  // level 0 flags live outside
};

void hier_init(Hier& H, int nx, int ny, int nz, float h) {
  H.lv = build_levels(nx, ny, nz, h, 4);
  size_t L = H.lv.size();
  H.phi.resize(L);
  H.b.resize(L);
  H.f.resize(L);
  for (size_t l = 0; l < L; l++) {
    size_t n = (size_t)H.lv[l].nx * H.lv[l].ny * H.lv[l].nz;
    if (l > 0) {
      H.phi[l].assign(n, 0.0f);
      H.b[l].assign(n, 0.0f);
      H.f[l].assign(n, 0u);
    }
  }
}

// src/sim.rs:425-491 — smoother schedule and V-cycles on level-0 arrays.
void vcycles(Hier& H, float* phi0, const float* b0, const uint32_t* f0, int cycles, int bc_mode) {
  int nl = (int)H.lv.size();
  auto P = [&](int l) { return l == 0 ? phi0 : H.phi[l].data(); };
  auto B = [&](int l) { return l == 0 ? b0 : H.b[l].data(); };
  auto F = [&](int l) { return l == 0 ? f0 : H.f[l].data(); };
  auto smooth = [&](int l, int iters, bool coarse) {
    float om = coarse ? 1.6f : 1.0f;
    for (int it = 0; it < iters; it++)
      for (int c = 0; c < 2; c++) mg_smooth(H.lv[l], B(l), F(l), P(l), c, om, bc_mode);
  };
  for (int cy = 0; cy < cycles; cy++) {
    for (int l = 0; l < nl - 1; l++) {
      smooth(l, 2, false);
      mg_restrict(H.lv[l], P(l), B(l), F(l), H.lv[l + 1], H.b[l + 1].data(), H.phi[l + 1].data(),
                  H.f[l + 1].data(), bc_mode);
    }
    smooth(nl - 1, 80, true);
    for (int l = nl - 2; l >= 0; l--) {
      mg_prolong(H.lv[l], P(l + 1), F(l), P(l), H.lv[l + 1], F(l + 1));
      smooth(l, 2, false);
    }
  }
}

}  // namespace

// ===========================================================================
// C API of the oracle (ctypes from the tests and bench.py's CPU legs).
// ---------------------------------------------------------------------------
// Renderer input pack: src/shaders/render.wgsl:3-61 (dispatched by
// src/render.rs:263-292).  The reference stores into rgba16float textures;
// the texel conversion is IEEE 754 binary32 -> binary16 with round to
// nearest even (pinned against numpy's float16 conversion in the tests).

using oracle_half::f16_to_f32;
using oracle_half::f32_to_f16;
static void store_h4(uint16_t* t, size_t i, float a, float b, float c, float d) {
  t[4 * i] = f32_to_f16(a);
  t[4 * i + 1] = f32_to_f16(b);
  t[4 * i + 2] = f32_to_f16(c);
  t[4 * i + 3] = f32_to_f16(d);
}

// render.wgsl:17-35, one cell
static void render_pack(const Ctx& C, const F4* s0, const F4* s1, const F4* sol,
                        const uint32_t* flags, const float* vu, const float* vv, const float* vw,
                        uint16_t* volT, uint16_t* solT, uint16_t* velT) {
  for (int z = 0; z < C.nz; z++)
    for (int y = 0; y < C.ny; y++)
      for (int x = 0; x < C.nx; x++) {
        const I3 c{x, y, z};
        const size_t i = C.sidx(c);
        const F4 a = s0[i], b = s1[i];
        const float rho = C.rhoOf(a.x);
        const bool solid = flags[i] == 1u;
        if (solid) store_h4(volT, i, 0.0f, a.x, 0.0f, 0.0f);
        else store_h4(volT, i, rho * a.w / RHO_SOOT * 1e6f, a.x, rho * b.x * 1e3f, b.y * 1e-3f);
        const F4 so = sol[i];
        const float tot = so.y + so.z;
        const float oc = solid ? 1.0f : 0.0f;
        store_h4(solT, i, oc, so.w * oc, so.z / wmax(tot, 1e-6f) * oc, so.x * oc);
        const size_t f = C.vidx(c);
        const size_t sy = (size_t)C.nx + 1, sz = sy * ((size_t)C.ny + 1);
        store_h4(velT, i, 0.5f * (vu[f] + vu[f + 1]), 0.5f * (vv[f] + vv[f + sy]),
                 0.5f * (vw[f] + vw[f + sz]), 0.0f);
      }
}

// render.wgsl:38-61: per 8^3 brick, max over the brick and a one-cell shell
static void render_bricks(int nx, int ny, int nz, const uint16_t* volT, const uint16_t* solT,
                          float* bricks) {
  const int bx = (nx + 7) / 8, by = (ny + 7) / 8, bz = (nz + 7) / 8;
  for (int k = 0; k < bz; k++)
    for (int j = 0; j < by; j++)
      for (int i = 0; i < bx; i++) {
        float m = 0.0f;
        for (int z = -1; z < 9; z++)
          for (int y = -1; y < 9; y++)
            for (int x = -1; x < 9; x++) {
              const int cx = i * 8 + x, cy = j * 8 + y, cz = k * 8 + z;
              if (cx < 0 || cy < 0 || cz < 0 || cx >= nx || cy >= ny || cz >= nz) continue;
              const size_t c = (size_t)cx + (size_t)nx * ((size_t)cy + (size_t)ny * cz);
              const float vx = f16_to_f32(volT[4 * c]), vz = f16_to_f32(volT[4 * c + 2]);
              const float vw = f16_to_f32(volT[4 * c + 3]), sx = f16_to_f32(solT[4 * c]);
              m = wmax(m, wmax(wmax(vx * 10.0f, vz * 2.0f), wmax(vw * 0.1f, sx * 10.0f)));
            }
        bricks[i + bx * (j + by * k)] = m;
      }
}

// render.wgsl:63-98: emission power per cell with the six-axis escape
static void render_ecells(const Ctx& C, const uint16_t* volT, const F4* lut, const float* chemi,
                          float* ecell) {
  const float dx = C.P->dx;
  for (int z = 0; z < C.nz; z++)
    for (int y = 0; y < C.ny; y++)
      for (int x = 0; x < C.nx; x++) {
        const I3 c{x, y, z};
        const size_t i = C.sidx(c);
        const float vx = f16_to_f32(volT[4 * i]), vy = f16_to_f32(volT[4 * i + 1]);
        const float vw = f16_to_f32(volT[4 * i + 3]);
        // lutAt (render.wgsl:68-72)
        const float xt = clampf((vy - 300.0f) / 3000.0f, 0.0f, 1.0f) * 1023.0f;
        const uint32_t li = (uint32_t)std::floor(xt);
        const F4 l0 = lut[li], l1 = lut[std::min(li + 1u, 1023u)];
        const float fr = xt - (float)li;
        const float sx = wmax(vx, 0.0f);
        const float a = chemi[0] * wmax(vw, 0.0f) * std::exp(-20.0f * sx);
        const float er = mixf(l0.x, l1.x, fr) * sx * 1e-6f + a * 0.12f;
        const float eg = mixf(l0.y, l1.y, fr) * sx * 1e-6f + a * 0.28f;
        const float eb = mixf(l0.z, l1.z, fr) * sx * 1e-6f + a * 1.0f;
        float e = (er * 0.2126f + eg * 0.7152f + eb * 0.0722f) * dx * dx * dx;
        if (e > 0.0f) {
          float esc = 0.0f;
          for (int k = 0; k < 6; k++) {
            float od = 0.0f;
            I3 p = c;
            for (int s = 0; s < 48; s++) {
              p = I3{p.x + DIRS[k].x, p.y + DIRS[k].y, p.z + DIRS[k].z};
              if (!C.inb(p) || od > 7.0f) break;
              const size_t q = C.sidx(p);
              const float wx = f16_to_f32(volT[4 * q]), wz = f16_to_f32(volT[4 * q + 2]);
              od += (chemi[1] * wmax(wx, 0.0f) + chemi[2] * wmax(wz, 0.0f)) * dx;
            }
            esc += std::exp(-od);
          }
          e *= wmax(esc / 6.0f, 0.02f);
        }
        ecell[i] = e;
      }
}

// src/render.rs:316-333: FP64 running sum, c / total as f32, the total last
static void render_cdf(size_t n, const float* e, float* cdf) {
  std::vector<double> out(n);
  double acc = 0.0;
  for (size_t i = 0; i < n; i++) {
    acc += (double)wmax(e[i], 0.0f);
    out[i] = acc;
  }
  const double total = acc;
  for (size_t i = 0; i < n; i++) cdf[i] = total > 0.0 ? (float)(out[i] / total) : 0.0f;
  cdf[n] = (float)total;
}

extern "C" {

void or_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}
int or_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

static void put_stats(const Stats& s, double* out) {
  if (out)
    for (int i = 0; i < PYRO_STATS_N; i++) out[i] += s.v[i];
}

// Individual kernels; `stats` (double[PYRO_STATS_N]) accumulates when not
// NULL: sums add, maxima (slots 4, 5) take the max.
void or_solid(const PyroParams* P, const float* solIn, float* solOut, float* pyr, uint32_t* flags,
              const float* s0, double* stats) {
  Ctx C(P);
  Stats st;
  st.clear();
  k_solid(C, (const F4*)solIn, (F4*)solOut, (F4*)pyr, flags, (const F4*)s0, &st);
  put_stats(st, stats);
}
void or_curl(const PyroParams* P, const float* u, const float* v, const float* w, float* curl,
             double* stats) {
  Ctx C(P);
  Stats st;
  st.clear();
  k_curl(C, u, v, w, (F4*)curl, &st);
  if (stats) stats[5] = std::max(stats[5], st.v[5]);
}
void or_adv_vel1(const PyroParams* P, const float* u, const float* v, const float* w, float* hu,
                 float* hv, float* hw) {
  Ctx C(P);
  k_adv_vel1(C, u, v, w, hu, hv, hw);
}
void or_adv_vel2(const PyroParams* P, const float* u, const float* v, const float* w,
                 const float* hu, const float* hv, const float* hw, float* ou, float* ov, float* ow,
                 const uint32_t* flags) {
  Ctx C(P);
  k_adv_vel2(C, u, v, w, hu, hv, hw, ou, ov, ow, flags);
}
void or_adv_s1(const PyroParams* P, const float* u, const float* v, const float* w,
               const float* s0, const float* s1, float* h0, float* h1) {
  Ctx C(P);
  k_adv_s1(C, u, v, w, (const F4*)s0, (const F4*)s1, (F4*)h0, (F4*)h1);
}
void or_adv_s2(const PyroParams* P, const float* u, const float* v, const float* w,
               const float* s0, const float* s1, const float* h0, const float* h1, float* o0,
               float* o1) {
  Ctx C(P);
  k_adv_s2(C, u, v, w, (const F4*)s0, (const F4*)s1, (const F4*)h0, (const F4*)h1, (F4*)o0,
           (F4*)o1);
}
void or_react(const PyroParams* P, const float* s0in, const float* s1in, float* s0out,
              float* s1out, const uint32_t* flags, const float* sol, const float* pyr,
              const float* curl, double* stats) {
  Ctx C(P);
  Stats st;
  st.clear();
  k_react(C, (const F4*)s0in, (const F4*)s1in, (F4*)s0out, (F4*)s1out, flags, (const F4*)sol,
          (const F4*)pyr, (const F4*)curl, &st);
  if (stats) {
    for (int i = 0; i < PYRO_STATS_N; i++)
      if (i != 4) stats[i] += st.v[i];
    stats[4] = std::max(stats[4], st.v[4]);
  }
}
void or_forces(const PyroParams* P, float* u, float* v, float* w, const float* s0, const float* s1,
               const float* curl, const uint32_t* flags) {
  Ctx C(P);
  k_forces(C, u, v, w, (const F4*)s0, (const F4*)s1, (const F4*)curl, flags);
}
void or_divergence(const PyroParams* P, const float* u, const float* v, const float* w,
                   const float* s1, const uint32_t* flags, float* b) {
  Ctx C(P);
  k_divergence(C, u, v, w, (const F4*)s1, flags, b);
}
void or_project(const PyroParams* P, float* u, float* v, float* w, const float* phi,
                const uint32_t* flags) {
  Ctx C(P);
  k_project(C, u, v, w, phi, flags);
}
void or_render_pack(const PyroParams* P, const float* s0, const float* s1, const float* sol,
                    const uint32_t* flags, const float* u, const float* v, const float* w,
                    uint16_t* vol, uint16_t* solt, uint16_t* vel) {
  Ctx C(P);
  render_pack(C, (const F4*)s0, (const F4*)s1, (const F4*)sol, flags, u, v, w, vol, solt, vel);
}
void or_render_bricks(int nx, int ny, int nz, const uint16_t* vol, const uint16_t* solt,
                      float* bricks) {
  render_bricks(nx, ny, nz, vol, solt, bricks);
}
void or_render_ecells(const PyroParams* P, const uint16_t* vol, const float* lut,
                      const float* chemi, float* ecell) {
  Ctx C(P);
  render_ecells(C, vol, (const F4*)lut, chemi, ecell);
}
void or_render_cdf(size_t n, const float* ecell, float* cdf) { render_cdf(n, ecell, cdf); }
void or_f32_to_f16(const float* x, uint16_t* h, size_t n) {
  for (size_t i = 0; i < n; i++) h[i] = f32_to_f16(x[i]);
}
void or_f16_to_f32(const uint16_t* h, float* x, size_t n) {
  for (size_t i = 0; i < n; i++) x[i] = f16_to_f32(h[i]);
}
void or_mg_smooth(int nx, int ny, int nz, float h, const float* b, const uint32_t* f, float* p,
                  int color, float omega, int bc_mode) {
  mg_smooth(Lv{nx, ny, nz, h}, b, f, p, color, omega, bc_mode);
}
void or_mg_restrict(int fnx, int fny, int fnz, float fh, const float* pf, const float* bf,
                    const uint32_t* ff, int cnx, int cny, int cnz, float* bc, float* pc,
                    uint32_t* fc, int bc_mode) {
  mg_restrict(Lv{fnx, fny, fnz, fh}, pf, bf, ff, Lv{cnx, cny, cnz, 2 * fh}, bc, pc, fc, bc_mode);
}
void or_mg_prolong(int fnx, int fny, int fnz, const float* pc, const uint32_t* ff, float* pf,
                   int cnx, int cny, int cnz, const uint32_t* fc) {
  mg_prolong(Lv{fnx, fny, fnz, 1.0f}, pc, ff, pf, Lv{cnx, cny, cnz, 2.0f}, fc);
}
void or_mg_resid(int nx, int ny, int nz, float h, const float* p, const float* b,
                 const uint32_t* f, int bc_mode, double* r2, double* b2) {
  mg_resid_sums(Lv{nx, ny, nz, h}, p, b, f, bc_mode, r2, b2);
}
int or_mg_levels(int nx, int ny, int nz, int* dims_out /* 4*3 */) {
  std::vector<Lv> v = build_levels(nx, ny, nz, 1.0f, 4);
  for (size_t l = 0; l < v.size(); l++) {
    dims_out[3 * l] = v[l].nx;
    dims_out[3 * l + 1] = v[l].ny;
    dims_out[3 * l + 2] = v[l].nz;
  }
  return (int)v.size();
}
// Fixed V-cycles on caller arrays (src/sim.rs:451-491).
void or_vcycles(int nx, int ny, int nz, float h, float* phi, const float* b, const uint32_t* f,
                int cycles, int bc_mode) {
  Hier H;
  hier_init(H, nx, ny, nz, h);
  vcycles(H, phi, b, f, cycles, bc_mode);
}

// FP64 Jacobi-preconditioned CG on -A x = -b over fluid cells (A is the
// operator of mg.wgsl:25-35, negative semi-definite).  Returns iterations;
// *rel gets ||b - A x|| / ||b|| in FP64.
int or_poisson_f64(int nx, int ny, int nz, double h, const float* bf, const uint32_t* f,
                   double* x, double tol, int max_iters, int bc_mode, double* rel) {
  Lv d{nx, ny, nz, (float)h};
  size_t N = (size_t)nx * ny * nz;
  double ih2 = 1.0 / (h * h);
  std::vector<double> diag(N, 0.0), r(N), z(N), p(N), q(N);
  // diag of -A = cnt/h^2
#pragma omp parallel for schedule(static)
  for (int zz = 0; zz < nz; zz++)
    for (int y = 0; y < ny; y++)
      for (int xx = 0; xx < nx; xx++) {
        I3 c{xx, y, zz};
        size_t i = idxL(c, d);
        if (f[i] == 1u) continue;
        double cnt = 0;
        for (int k = 0; k < 6; k++) {
          I3 n = c + DIRS[k];
          if (n.y < 0) continue;
          if (!inbL(n, d)) {
            if (dirichletOut(n, d, bc_mode)) cnt += 1;
            continue;
          }
          if (f[idxL(n, d)] == 1u) continue;
          cnt += 1;
        }
        diag[i] = cnt * ih2;
      }
  auto applyNegA = [&](const std::vector<double>& v, std::vector<double>& out) {
#pragma omp parallel for schedule(static)
    for (int zz = 0; zz < nz; zz++)
      for (int y = 0; y < ny; y++)
        for (int xx = 0; xx < nx; xx++) {
          I3 c{xx, y, zz};
          size_t i = idxL(c, d);
          if (f[i] == 1u) { out[i] = 0; continue; }
          double sum = 0;
          for (int k = 0; k < 6; k++) {
            I3 n = c + DIRS[k];
            if (n.y < 0 || !inbL(n, d)) continue;
            size_t j = idxL(n, d);
            if (f[j] == 1u) continue;
            sum += v[j];
          }
          out[i] = diag[i] * v[i] - sum * ih2;
        }
  };
  auto dot = [&](const std::vector<double>& a, const std::vector<double>& b) {
    double s = 0;
#pragma omp parallel for schedule(static) reduction(+ : s)
    for (long i = 0; i < (long)N; i++) s += a[i] * b[i];
    return s;
  };
  std::vector<double> xv(N);
  for (size_t i = 0; i < N; i++) xv[i] = (f[i] == 1u) ? 0.0 : x[i];
  applyNegA(xv, q);
  double bn2 = 0;
  for (size_t i = 0; i < N; i++) {
    double bi = (f[i] == 1u) ? 0.0 : -(double)bf[i];
    r[i] = bi - q[i];
    bn2 += bi * bi;
  }
  double bn = std::sqrt(bn2);
  if (bn == 0) {
    for (size_t i = 0; i < N; i++) x[i] = 0;
    *rel = 0;
    return 0;
  }
  for (size_t i = 0; i < N; i++) z[i] = diag[i] > 0 ? r[i] / diag[i] : 0.0;
  p = z;
  double rz = dot(r, z);
  int it = 0;
  double rn = std::sqrt(dot(r, r));
  for (; it < max_iters && rn > tol * bn; it++) {
    applyNegA(p, q);
    double pq = dot(p, q);
    if (pq <= 0) break;
    double alpha = rz / pq;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)N; i++) {
      xv[i] += alpha * p[i];
      r[i] -= alpha * q[i];
      z[i] = diag[i] > 0 ? r[i] / diag[i] : 0.0;
    }
    double rz2 = dot(r, z);
    double beta = rz2 / rz;
    rz = rz2;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)N; i++) p[i] = z[i] + beta * p[i];
    rn = std::sqrt(dot(r, r));
  }
  // true residual
  applyNegA(xv, q);
  double tr2 = 0;
  for (size_t i = 0; i < N; i++) {
    double bi = (f[i] == 1u) ? 0.0 : -(double)bf[i];
    double e = bi - q[i];
    tr2 += e * e;
  }
  *rel = std::sqrt(tr2) / bn;
  for (size_t i = 0; i < N; i++) x[i] = xv[i];
  return it;
}

// Relative residual of a float solution in FP64 (the same operator).
double or_poisson_relres(int nx, int ny, int nz, double h, const float* phi, const float* bf,
                         const uint32_t* f, int bc_mode) {
  Lv d{nx, ny, nz, (float)h};
  double ih2 = 1.0 / (h * h);
  double r2 = 0, b2 = 0;
#pragma omp parallel for schedule(static) reduction(+ : r2, b2)
  for (int zz = 0; zz < nz; zz++)
    for (int y = 0; y < ny; y++)
      for (int xx = 0; xx < nx; xx++) {
        I3 c{xx, y, zz};
        size_t i = idxL(c, d);
        if (f[i] == 1u) continue;
        double sum = 0, cnt = 0;
        for (int k = 0; k < 6; k++) {
          I3 n = c + DIRS[k];
          if (n.y < 0) continue;
          if (!inbL(n, d)) {
            if (dirichletOut(n, d, bc_mode)) cnt += 1;
            continue;
          }
          size_t j = idxL(n, d);
          if (f[j] == 1u) continue;
          sum += phi[j];
          cnt += 1;
        }
        double r = (double)bf[i] - (sum - cnt * (double)phi[i]) * ih2;
        r2 += r * r;
        b2 += (double)bf[i] * (double)bf[i];
      }
  return b2 > 0 ? std::sqrt(r2 / b2) : 0.0;
}

// ---- whole-simulation oracle (Sim::new / Sim::step) ---------------------
struct OrSim {
  PyroParams p;
  int nx, ny, nz;
  size_t n, nv;
  std::vector<float> vel[2][3], hat[3];
  std::vector<F4> s0, s1, s0b, s1b, h0, h1, sol[2], pyr, curl;
  std::vector<uint32_t> flags;
  std::vector<float> phi0, b0;
  Hier H;
  Stats stats;
  std::vector<float> staging;
  int cur, sol_cur;
  uint32_t cycles;
};

OrSim* or_sim_create(const PyroParams* p, const float* sol_init, uint32_t cycles) {
  OrSim* S = new OrSim();
  S->p = *p;
  S->nx = (int)p->nx;
  S->ny = (int)p->ny;
  S->nz = (int)p->nz;
  S->n = (size_t)S->nx * S->ny * S->nz;
  S->nv = (size_t)(S->nx + 1) * (S->ny + 1) * (S->nz + 1);
  for (int a = 0; a < 2; a++)
    for (int k = 0; k < 3; k++) S->vel[a][k].assign(S->nv, 0.0f);
  for (int k = 0; k < 3; k++) S->hat[k].assign(S->nv, 0.0f);
  F4 z{0, 0, 0, 0};
  S->s0.assign(S->n, F4{p->t0, 0.0f, p->yo2, 0.0f});
  S->s1.assign(S->n, z);
  S->s0b.assign(S->n, z);
  S->s1b.assign(S->n, z);
  S->h0.assign(S->n, z);
  S->h1.assign(S->n, z);
  S->pyr.assign(S->n, z);
  S->curl.assign(S->n, z);
  for (int a = 0; a < 2; a++) {
    S->sol[a].resize(S->n);
    std::memcpy(S->sol[a].data(), sol_init, S->n * sizeof(F4));
  }
  S->flags.assign(S->n, 0u);
  S->phi0.assign(S->n, 0.0f);
  S->b0.assign(S->n, 0.0f);
  hier_init(S->H, S->nx, S->ny, S->nz, p->dx);
  S->stats.clear();
  S->staging.assign(PYRO_STATS_N, 0.0f);
  S->cur = 0;
  S->sol_cur = 0;
  S->cycles = cycles;
  return S;
}

// src/sim.rs:246-423
void or_sim_step(OrSim* S, float dt, float time, float ign_on, int want_stats) {
  S->p.dt = dt;
  S->p.time = time;
  S->p.ign_on = ign_on;
  Ctx C(&S->p);
  Stats& st = S->stats;
  if (want_stats) st.clear();
  std::vector<float>* va = S->vel[S->cur];
  std::vector<float>* vb = S->vel[1 - S->cur];
  std::vector<F4>& sa = S->sol[S->sol_cur];
  std::vector<F4>& sb = S->sol[1 - S->sol_cur];
  Stats* sp = want_stats ? &st : nullptr;
  k_solid(C, sa.data(), sb.data(), S->pyr.data(), S->flags.data(), S->s0.data(), sp);
  k_curl(C, va[0].data(), va[1].data(), va[2].data(), S->curl.data(), sp);
  k_adv_vel1(C, va[0].data(), va[1].data(), va[2].data(), S->hat[0].data(), S->hat[1].data(),
             S->hat[2].data());
  k_adv_vel2(C, va[0].data(), va[1].data(), va[2].data(), S->hat[0].data(), S->hat[1].data(),
             S->hat[2].data(), vb[0].data(), vb[1].data(), vb[2].data(), S->flags.data());
  k_adv_s1(C, va[0].data(), va[1].data(), va[2].data(), S->s0.data(), S->s1.data(), S->h0.data(),
           S->h1.data());
  k_adv_s2(C, va[0].data(), va[1].data(), va[2].data(), S->s0.data(), S->s1.data(), S->h0.data(),
           S->h1.data(), S->s0b.data(), S->s1b.data());
  k_react(C, S->s0b.data(), S->s1b.data(), S->s0.data(), S->s1.data(), S->flags.data(),
          sb.data(), S->pyr.data(), S->curl.data(), sp);
  k_forces(C, vb[0].data(), vb[1].data(), vb[2].data(), S->s0.data(), S->s1.data(),
           S->curl.data(), S->flags.data());
  k_divergence(C, vb[0].data(), vb[1].data(), vb[2].data(), S->s1.data(), S->flags.data(),
               S->b0.data());
  vcycles(S->H, S->phi0.data(), S->b0.data(), S->flags.data(), (int)S->cycles, 0);
  if (want_stats) {
    double r2, b2;
    mg_resid_sums(S->H.lv[0], S->phi0.data(), S->b0.data(), S->flags.data(), 0, &r2, &b2);
    st.v[10] += r2;
    st.v[11] += b2;
  }
  k_project(C, vb[0].data(), vb[1].data(), vb[2].data(), S->phi0.data(), S->flags.data());
  if (want_stats)
    for (int i = 0; i < PYRO_STATS_N; i++) S->staging[i] = (float)st.v[i];
  S->cur = 1 - S->cur;
  S->sol_cur = 1 - S->sol_cur;
  S->p.frame += 1;
}

void or_sim_read_stats(OrSim* S, float* out) {
  std::memcpy(out, S->staging.data(), PYRO_STATS_N * sizeof(float));
}

static void* or_field_ptr(OrSim* S, int field, size_t* bytes) {
  switch (field) {
    case PYRO_F_S0: *bytes = S->n * 16; return S->s0.data();
    case PYRO_F_S1: *bytes = S->n * 16; return S->s1.data();
    case PYRO_F_SOL: *bytes = S->n * 16; return S->sol[S->sol_cur].data();
    case PYRO_F_PYR: *bytes = S->n * 16; return S->pyr.data();
    case PYRO_F_FLAGS: *bytes = S->n * 4; return S->flags.data();
    case PYRO_F_CURL: *bytes = S->n * 16; return S->curl.data();
    case PYRO_F_U: *bytes = S->nv * 4; return S->vel[S->cur][0].data();
    case PYRO_F_V: *bytes = S->nv * 4; return S->vel[S->cur][1].data();
    case PYRO_F_W: *bytes = S->nv * 4; return S->vel[S->cur][2].data();
    case PYRO_F_PHI: *bytes = S->n * 4; return S->phi0.data();
    case PYRO_F_B: *bytes = S->n * 4; return S->b0.data();
    default: *bytes = 0; return nullptr;
  }
}

int or_sim_read_field(OrSim* S, int field, void* out, size_t bytes) {
  size_t nb = 0;
  void* p = or_field_ptr(S, field, &nb);
  if (!p || nb != bytes) return -1;
  std::memcpy(out, p, nb);
  return 0;
}
int or_sim_write_field(OrSim* S, int field, const void* in, size_t bytes) {
  size_t nb = 0;
  void* p = or_field_ptr(S, field, &nb);
  if (!p || nb != bytes) return -1;
  std::memcpy(p, in, nb);
  return 0;
}
void or_sim_destroy(OrSim* S) { delete S; }

// ---- scene voxelizer (src/scene.rs:621-667,695-728) ------------------------
static float or_hash(uint32_t v) {
  uint32_t x = v * 747796405u + 2891336453u;
  x = ((x >> ((x >> 28) + 4u)) ^ x) * 277803737u;
  x = (x >> 22) ^ x;
  return (float)x / (float)4294967295u;
}
float or_hash_f(uint32_t v) { return or_hash(v); }

static bool or_inside(const PyroShape& s, const float p[3], float dx) {
  switch (s.kind) {
    case PYRO_SHAPE_BOX: {
      float d0 = p[0] - s.c[0], d1 = p[1] - s.c[1], d2 = p[2] - s.c[2];
      float lx = s.cos_yaw * d0 + s.sin_yaw * d2;
      float lz = -s.sin_yaw * d0 + s.cos_yaw * d2;
      float h0 = wmax(s.e[0], 0.5f * dx), h1 = wmax(s.e[1], 0.5f * dx), h2 = wmax(s.e[2], 0.5f * dx);
      return std::fabs(lx) <= h0 && std::fabs(d1) <= h1 && std::fabs(lz) <= h2;
    }
    case PYRO_SHAPE_CYL: {
      float ba[3] = {s.e[0] - s.c[0], s.e[1] - s.c[1], s.e[2] - s.c[2]};
      float pa[3] = {p[0] - s.c[0], p[1] - s.c[1], p[2] - s.c[2]};
      float l2 = ba[0] * ba[0] + ba[1] * ba[1] + ba[2] * ba[2];
      float t = (pa[0] * ba[0] + pa[1] * ba[1] + pa[2] * ba[2]) / l2;
      if (!(t >= 0.0f && t <= 1.0f)) return false;
      float q[3] = {pa[0] - ba[0] * t, pa[1] - ba[1] * t, pa[2] - ba[2] * t};
      return std::sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2]) <= wmax(s.r, 0.5f * dx);
    }
    case PYRO_SHAPE_SPHERE: {
      float d[3] = {p[0] - s.c[0], p[1] - s.c[1], p[2] - s.c[2]};
      return std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]) <= s.r;
    }
    case PYRO_SHAPE_POOL: {
      float a = p[0] - s.c[0], b = p[2] - s.c[2];
      float dxz = std::sqrt(a * a + b * b);
      return dxz <= s.r && p[1] <= wmax(s.depth, dx * 0.99f);
    }
    default:
      return false;
  }
}

void or_voxelize(const PyroShape* shapes, uint32_t n_shapes, int nx, int ny, int nz, float dx,
                 float t0, uint32_t seed, const float* slot_density, const uint32_t* slot_kind,
                 float* sol_out) {
  F4* sol = (F4*)sol_out;
#pragma omp parallel for schedule(static)
  for (int k = 0; k < nz; k++)
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++) {
        size_t idx = (size_t)i + (size_t)nx * ((size_t)j + (size_t)ny * (size_t)k);
        F4 v{0.0f, 0.0f, 0.0f, t0};
        float p[3] = {((float)i + 0.5f) * dx, ((float)j + 0.5f) * dx, ((float)k + 0.5f) * dx};
        for (uint32_t s = 0; s < n_shapes; s++) {
          if (or_inside(shapes[s], p, dx)) {
            uint32_t slot = shapes[s].slot;
            float h = or_hash((uint32_t)idx ^ (seed * 0x9e3779b9u));
            float jit = 0.85f + 0.3f * h;
            float mass = slot_kind[slot] == 2u ? 1.0f : slot_density[slot] * jit;
            v = F4{(float)slot, mass, 0.0f, t0};
          }
        }
        sol[idx] = v;
      }
}

}  // extern "C"
