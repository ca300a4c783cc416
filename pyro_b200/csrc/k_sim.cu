// k_sim.cu — the fire-simulation kernels of one substep.
//
// One thread per cell (or per face position of the padded (nx+1)(ny+1)(nz+1)
// face grid), 32-wide in x so that every warp touches one contiguous row:
// coalesced float4 loads of the cell fields and float loads of the faces.
// Each kernel restates one reference WGSL entry point; the expression order
// follows the WGSL source so FP32 results match the CPU oracle up to the
// last-ulp differences of expf.
//
//   solid      src/shaders/combust.wgsl:3-137
//   curl       src/shaders/fluid.wgsl:3-29
//   adv_vel1   src/shaders/advect.wgsl:4-20
//   adv_vel2   src/shaders/advect.wgsl:22-70
//   adv_s1     src/shaders/advect.wgsl:72-91
//   adv_s2     src/shaders/advect.wgsl:93-125
//   react      src/shaders/combust.wgsl:139-273
//   forces     src/shaders/fluid.wgsl:31-109
//   divergence src/shaders/fluid.wgsl:111-128
//   project    src/shaders/fluid.wgsl:130-152
#include "common.cuh"
#include "kernels.h"

namespace pyro {

namespace {

constexpr int BX = 32, BY = 4, BZ = 2;

inline dim3 grid_for(int x, int y, int z) {
  return dim3((unsigned)((x + BX - 1) / BX), (unsigned)((y + BY - 1) / BY),
              (unsigned)((z + BZ - 1) / BZ));
}
__device__ __forceinline__ I3 thread_cell() {
  return I3{(int)(blockIdx.x * BX + threadIdx.x), (int)(blockIdx.y * BY + threadIdx.y),
            (int)(blockIdx.z * BZ + threadIdx.z)};
}

// ------------------------------------------------------------------- solid
struct SolidCtx {
  const PyroParams& P;
  Grid g;
  const float4* __restrict__ solIn;
  const float4* __restrict__ s0;

  // material slot of a solid state; out-of-range slots clamp to the last
  // row like the reference's restricted uniform-array indexing.
  __device__ __forceinline__ static uint32_t slotOf(float4 s) {
    return min(__float2uint_rz(s.x), 7u);
  }
  __device__ __forceinline__ uint32_t kindOf(float4 s) const {
    return (uint32_t)(P.mats[slotOf(s)][3] + 0.5f);
  }
  __device__ __forceinline__ bool isSolidS(float4 s) const {
    if (kindOf(s) == 2u) return s.y > 0.5f;
    return s.y + s.z > P.burnout;
  }
  __device__ __forceinline__ bool solidN(I3 c) const {
    if (!g.inb(c)) return false;
    return isSolidS(__ldg(solIn + g.sidx(c)));
  }
  // combust.wgsl:18-39: emission-absorption march along one ray.  The ten
  // sample positions (strides 1,1,1,2,2,3,4,5,7,9) do not depend on the
  // data, so the cells along the ray are loaded first, in two batches of
  // five, and the march then runs on registers with the reference's
  // arithmetic and early exits.
  __device__ float rayIrr(I3 c0, I3 d) const {
    constexpr int ST[10] = {1, 1, 1, 2, 2, 3, 4, 5, 7, 9};
    float tr = 1.0f, acc = 0.0f;
    const float dl = len3(tof3(d)) * P.dx;
    I3 p = c0;
    bool done = false;
#pragma unroll
    for (int h = 0; h < 2 && !done; h++) {
      float4 so[5], gg[5];
      bool in[5];
      I3 q = p;
#pragma unroll
      for (int s = 0; s < 5; s++) {
        in[s] = g.inb(q);
        const int j = in[s] ? g.sidx(q) : 0;
        so[s] = in[s] ? __ldg(solIn + j) : make_float4(0.f, 0.f, 0.f, 0.f);
        gg[s] = in[s] ? __ldg(s0 + j) : make_float4(0.f, 0.f, 0.f, 0.f);
        const int stv = ST[5 * h + s];
        q = I3{q.x + d.x * stv, q.y + d.y * stv, q.z + d.z * stv};
      }
#pragma unroll
      for (int s = 0; s < 5; s++) {
        if (!in[s]) {
          done = true;
          break;
        }
        if (isSolidS(so[s])) {
          acc += tr * pow4(so[s].w);
          tr = 0.0f;
          done = true;
          break;
        }
        const float T = gg[s].x;
        const float len = (float)ST[5 * h + s] * dl;
        const float e = 1.0f - expf(-kapP(P, T, gg[s].z, gg[s].w) * len);
        acc += tr * e * pow4(T);
        tr *= 1.0f - e;
      }
      p = q;
    }
    acc += tr * pow4(P.t0);
    return SIGMA * acc;
  }
  // combust.wgsl:41-48: normal + four 45-degree rays.
  __device__ float faceIrr(I3 c0, int k) const {
    I3 d = dir6(k);
    I3 t1{0, 1, 0}, t2{0, 0, 1};
    if (d.y != 0) t1 = I3{1, 0, 0};
    if (d.z != 0) t2 = I3{1, 0, 0};
    return 0.2f * (rayIrr(c0, d) + rayIrr(c0, d + t1) + rayIrr(c0, d - t1) + rayIrr(c0, d + t2) +
                   rayIrr(c0, d - t2));
  }
};

__global__ void __launch_bounds__(256) k_solid(const PyroParams* __restrict__ Pp, Grid g,
                                               const float4* __restrict__ solIn,
                                               float4* __restrict__ solOut,
                                               float4* __restrict__ pyr,
                                               uint32_t* __restrict__ flags,
                                               const float4* __restrict__ s0,
                                               float* __restrict__ stats) {
  __shared__ float sh[3 * 32];
  const PyroParams& P = *Pp;
  SolidCtx C{P, g, solIn, s0};
  I3 c = thread_cell();
  float stPyro = 0.0f, stMass = 0.0f, stArea = 0.0f;
  if (g.inb(c)) {
    int i = g.sidx(c);
    float4 s = __ldg(solIn + i);
    float4 o = s;
    float4 po = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    uint32_t fl = 0u;
    if (C.isSolidS(s)) {
      fl = 1u;
      const float* m = P.mats[SolidCtx::slotOf(s)];
      uint32_t kind = C.kindOf(s);
      float fuel = s.y, chr = s.z, Ts = s.w;
      if (kind != 2u) {
        float nF = 0.0f, Tg = 0.0f, Yo = 0.0f, qin = 0.0f, qcond = 0.0f;
        for (int k = 0; k < 6; k++) {
          I3 n = c + dir6(k);
          if (n.y < 0) continue;
          if (C.solidN(n)) {
            qcond += m[7] / P.dx * (__ldg(solIn + g.sidx(n)).w - Ts);
            continue;
          }
          nF += 1.0f;
          if (g.inb(n)) {
            float4 gg = __ldg(s0 + g.sidx(n));
            Tg += gg.x;
            Yo += gg.z;
            qin += C.faceIrr(n, k);
          } else {
            Tg += P.t0;
            Yo += P.yo2;
            qin += SIGMA * pow4(P.t0);
          }
        }
        float layer = (kind == 1u) ? 0.001f : fminf(P.layer, P.dx);
        float cap = m[0] * m[6] * layer;
        if (nF > 0.0f) {
          Tg /= nF;
          Yo /= nF;
          qin /= nF;
          float qnet = m[5] * (qin - SIGMA * pow4(Ts)) + P.h_conv * (Tg - Ts) + qcond / nF;
          if (P.ign_on > 0.5f) {
            F3 pc = (tof3(c) + F3{0.5f, 0.5f, 0.5f}) * P.dx;
            float dI = len3(pc - F3{P.ign_x, P.ign_y, P.ign_z});
            qnet += P.ign_flux * wclamp(1.0f - dI / (1.5f * P.ign_r), 0.0f, 1.0f);
          }
          float mv = 0.0f, mc = 0.0f;
          if (kind == 1u) {
            float Tb = m[2];
            mv = smoothstep(Tb - 60.0f, Tb, Ts) * fmaxf(qnet, 0.0f) / m[1] * m[9];
            Ts = fminf(Ts + P.dt * fmaxf(qnet - mv * m[1], fminf(qnet, 0.0f)) / cap, Tb);
            fuel -= mv * nF / P.dx * P.dt;
          } else {
            if (fuel > 0.0f)
              mv = smoothstep(m[2] - 20.0f, m[2] + 30.0f, Ts) * fmaxf(qnet, 0.0f) / m[1] * m[9];
            float chi = (kind == 0u) ? m[4] : 0.0f;
            float kin = P.char_a * expf(-P.char_e / (RGAS * Ts)) * chr * layer;
            float dif = P.h_mass * rhoOf(P, Tg) * Yo / 1.33f;
            mc = fminf(kin, dif);
            Ts += P.dt * (qnet - mv * m[1] + 0.5f * mc * P.dh_char) / cap;
            float virgin = fminf(mv / (1.0f - chi) * nF / P.dx * P.dt, fuel);
            fuel -= virgin;
            chr += virgin * chi - mc * nF / P.dx * P.dt;
          }
          stPyro = mv * nF * P.dx * P.dx;
          stArea = (mv > 1e-4f) ? nF * P.dx * P.dx : 0.0f;
          po = make_float4(mv, mc, nF, 0.0f);
        } else {
          Ts += P.dt * qcond / (m[0] * m[6] * P.dx);
        }
        Ts = wclamp(Ts, 250.0f, 2000.0f);
        fuel = fmaxf(fuel, 0.0f);
        chr = fmaxf(chr, 0.0f);
        o = make_float4(s.x, fuel, chr, Ts);
        if (fuel + chr <= P.burnout) {
          o = make_float4(0.0f, 0.0f, 0.0f, P.t0);
          fl = 0u;
          po = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        }
      }
      stMass = (o.y + o.z) * P.dx * P.dx * P.dx * ((kind == 2u) ? 0.0f : 1.0f);
    }
    solOut[i] = o;
    pyr[i] = po;
    flags[i] = fl;
  }
  if (stats) {
    float vals[3] = {stPyro, stMass, stArea};
    block_stats<3>(sh, vals, stats, {2, 7, 9}, 0u);
  }
}

// -------------------------------------------------------------------- curl
__device__ __forceinline__ F3 ucell(const Grid& g, const float* __restrict__ u,
                                    const float* __restrict__ v, const float* __restrict__ w,
                                    I3 c0) {
  I3 c = g.clampC(c0);
  int i = g.vidx(c);
  const int sy = g.nx + 1, sz = (g.nx + 1) * (g.ny + 1);
  return 0.5f * F3{__ldg(u + i) + __ldg(u + i + 1), __ldg(v + i) + __ldg(v + i + sy),
                   __ldg(w + i) + __ldg(w + i + sz)};
}

__global__ void __launch_bounds__(256) k_curl(const PyroParams* __restrict__ Pp, Grid g,
                                              const float* __restrict__ u,
                                              const float* __restrict__ v,
                                              const float* __restrict__ w,
                                              float4* __restrict__ curl,
                                              float* __restrict__ stats) {
  __shared__ float sh[32];
  I3 c = thread_cell();
  float spd = 0.0f;
  if (g.inb(c)) {
    const I3 X{1, 0, 0}, Y{0, 1, 0}, Z{0, 0, 1};
    F3 uxp = ucell(g, u, v, w, c + X), uxm = ucell(g, u, v, w, c - X);
    F3 uyp = ucell(g, u, v, w, c + Y), uym = ucell(g, u, v, w, c - Y);
    F3 uzp = ucell(g, u, v, w, c + Z), uzm = ucell(g, u, v, w, c - Z);
    F3 om = F3{(uyp.z - uym.z) - (uzp.y - uzm.y), (uzp.x - uzm.x) - (uxp.z - uxm.z),
               (uxp.y - uxm.y) - (uyp.x - uym.x)} /
            (2.0f * Pp->dx);
    curl[g.sidx(c)] = make_float4(om.x, om.y, om.z, len3(om));
    if (stats) spd = len3(ucell(g, u, v, w, c));
  }
  if (stats) block_max(sh, spd, stats + 5);
}

// ---------------------------------------------------------------- advection
__device__ __forceinline__ const float* pick3(int k, const float* a, const float* b,
                                              const float* c) {
  return k == 0 ? a : (k == 1 ? b : c);
}

// Predictor: h = v(backtrace(x)) per valid face component.  It also keeps
// the min / max of v over the 8 corners of that trilinear sample (the
// corrector's limiter, advect.wgsl:55-68, samples the same point), in
// lohi[0..2] / lohi[3..5] per component, so the corrector does not trace
// back again.
__global__ void __launch_bounds__(256) k_adv_vel1(const PyroParams* __restrict__ Pp, Grid g,
                                                  const float* __restrict__ u,
                                                  const float* __restrict__ v,
                                                  const float* __restrict__ w,
                                                  float* __restrict__ hu,
                                                  float* __restrict__ hv,
                                                  float* __restrict__ hw,
                                                  float* __restrict__ lohi) {
  I3 c = thread_cell();
  if (c.x > g.nx || c.y > g.ny || c.z > g.nz) return;
  const float kk = Pp->dt / Pp->dx;
  const size_t nv = (size_t)(g.nx + 1) * (g.ny + 1) * (g.nz + 1);
  Vel V{u, v, w};
  int i = g.vidx(c);
#pragma unroll
  for (int k = 0; k < 3; k++) {
    if (!g.compValid(k, c)) continue;
    F3 off = compOff(k);
    float lo, hi;
    float r = triC_mm_p(pick3(k, u, v, w), g, V.back_at<true>(g, kk, k, c, tof3(c) + off) - off,
                      g.compHi(k), lo, hi);
    if (k == 0) hu[i] = r; else if (k == 1) hv[i] = r; else hw[i] = r;
    lohi[k * nv + i] = lo;
    lohi[(3 + k) * nv + i] = hi;
  }
}

// Corrector: clamp(h + (v - h(fwdtrace(x))) / 2, min, max of v at the
// backtrace) (advect.wgsl:22-70); blocked faces 0.  The backtrace's
// min / max come from the predictor.
__global__ void __launch_bounds__(256) k_adv_vel2(const PyroParams* __restrict__ Pp, Grid g,
                                                  const float* __restrict__ u,
                                                  const float* __restrict__ v,
                                                  const float* __restrict__ w,
                                                  const float* __restrict__ hu,
                                                  const float* __restrict__ hv,
                                                  const float* __restrict__ hw,
                                                  const float* __restrict__ lohi,
                                                  float* __restrict__ ou,
                                                  float* __restrict__ ov,
                                                  float* __restrict__ ow,
                                                  const uint32_t* __restrict__ flags) {
  I3 c = thread_cell();
  if (c.x > g.nx || c.y > g.ny || c.z > g.nz) return;
  const float kk = Pp->dt / Pp->dx;
  const size_t nv = (size_t)(g.nx + 1) * (g.ny + 1) * (g.nz + 1);
  Vel V{u, v, w};
  int i = g.vidx(c);
  bool sc = g.inb(c) && __ldg(flags + g.sidx(c)) == 1u;
#pragma unroll
  for (int k = 0; k < 3; k++) {
    if (!g.compValid(k, c)) continue;
    I3 a = c - unitI(k);
    bool sa = g.inb(a) && __ldg(flags + g.sidx(a)) == 1u;
    float r;
    if ((k == 1 && c.y == 0) || sc || sa) {
      r = 0.0f;
    } else {
      F3 off = compOff(k);
      I3 hi = g.compHi(k);
      F3 x = tof3(c) + off;
      F3 f = V.fwd_at(g, kk, k, c, x) - off;
      const float* vk = pick3(k, u, v, w);
      const float* hk = pick3(k, hu, hv, hw);
      const float lo = __ldg(lohi + k * nv + i), hv2 = __ldg(lohi + (3 + k) * nv + i);
      r = wclamp(__ldg(hk + i) + 0.5f * (__ldg(vk + i) - triC_p(hk, g, f, hi)), lo, hv2);
    }
    if (k == 0) ou[i] = r; else if (k == 1) ov[i] = r; else ow[i] = r;
  }
}

__global__ void __launch_bounds__(256, 6) k_adv_s1(const PyroParams* __restrict__ Pp, Grid g,
                                                const float* __restrict__ u,
                                                const float* __restrict__ v,
                                                const float* __restrict__ w,
                                                const float4* __restrict__ s0,
                                                const float4* __restrict__ s1,
                                                float4* __restrict__ h0,
                                                float4* __restrict__ h1,
                                                float* __restrict__ bt) {
  I3 c = thread_cell();
  if (!g.inb(c)) return;
  const PyroParams& P = *Pp;
  const float kk = P.dt / P.dx;
  Vel V{u, v, w};
  const F3 half{0.5f, 0.5f, 0.5f};
  F3 b = V.back_at(g, kk, 3, c, tof3(c) + half) - half;
  float t = wclamp(g.outside(b), 0.0f, 1.0f);
  int i = g.sidx(c);
  // the backtrace, for the corrector's limiter (adv_s2)
  const size_t n = (size_t)g.nx * g.ny * g.nz;
  bt[i] = b.x;
  bt[n + i] = b.y;
  bt[2 * n + i] = b.z;
  h0[i] = wmix4(triS(s0, g, b), make_float4(P.t0, 0.0f, P.yo2, 0.0f), t);
  h1[i] = wmix4(triS(s1, g, b), make_float4(0.0f, 0.0f, 0.0f, 0.0f), t);
}

__global__ void __launch_bounds__(256, 4) k_adv_s2(const PyroParams* __restrict__ Pp, Grid g,
                                                const float* __restrict__ u,
                                                const float* __restrict__ v,
                                                const float* __restrict__ w,
                                                const float4* __restrict__ s0,
                                                const float4* __restrict__ s1,
                                                const float4* __restrict__ h0,
                                                const float4* __restrict__ h1,
                                                const float* __restrict__ bt,
                                                float4* __restrict__ o0,
                                                float4* __restrict__ o1) {
  I3 c = thread_cell();
  if (!g.inb(c)) return;
  const float kk = Pp->dt / Pp->dx;
  Vel V{u, v, w};
  const F3 half{0.5f, 0.5f, 0.5f};
  F3 x = tof3(c) + half;
  int i = g.sidx(c);
  // the backtrace from the predictor (the same expressions as both_at's)
  const size_t n = (size_t)g.nx * g.ny * g.nz;
  const F3 b{__ldg(bt + i), __ldg(bt + n + i), __ldg(bt + 2 * n + i)};
  const F3 f = V.fwd_at(g, kk, 3, c, x) - half;
  float4 r0 = __ldg(h0 + i), r1 = __ldg(h1 + i);
  if (g.outside(b) <= 0.0f && g.outside(f) <= 0.0f) {
    float4 l0, u0, l1, u1;
    mmS(s0, g, b, l0, u0);
    mmS(s1, g, b, l1, u1);
    r0 = min4(max4(r0 + 0.5f * (__ldg(s0 + i) - triS(h0, g, f)), l0), u0);
    r1 = min4(max4(r1 + 0.5f * (__ldg(s1 + i) - triS(h1, g, f)), l1), u1);
  }
  o0[i] = r0;
  o1[i] = r1;
}

// ------------------------------------------------------------------- react
__global__ void __launch_bounds__(256, 8) k_react(const PyroParams* __restrict__ Pp, Grid g,
                                               const float4* __restrict__ s0in,
                                               const float4* __restrict__ s1in,
                                               float4* __restrict__ s0out,
                                               float4* __restrict__ s1out,
                                               const uint32_t* __restrict__ flags,
                                               const float4* __restrict__ sol,
                                               const float4* __restrict__ pyr,
                                               const float4* __restrict__ curl,
                                               float* __restrict__ stats) {
  __shared__ float sh[6 * 32];
  const PyroParams& P = *Pp;
  I3 c = thread_cell();
  float stH = 0, stR = 0, stS = 0, stF = 0, stM = 0, stT = 0;
  const float dV = P.dx * P.dx * P.dx;
  bool active = g.inb(c);
  if (active) {
    int i = g.sidx(c);
    if (__ldg(flags + i) == 1u) {
      s0out[i] = make_float4(__ldg(sol + i).w, 0.0f, P.yo2, 0.0f);
      s1out[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    } else {
      float4 a = __ldg(s0in + i);
      float4 b = __ldg(s1in + i);
      // in-domain solid neighbours, bit k for direction k (+x -x +y -y +z -z)
      uint32_t smask = 0;
#pragma unroll
      for (int k = 0; k < 6; k++) {
        I3 n = c + dir6(k);
        if (g.inb(n) && __ldg(flags + g.sidx(n)) == 1u) smask |= 1u << k;
      }
      float nut = (P.cs * P.dx) * (P.cs * P.dx) * __ldg(curl + i).w;
      if (P.cs > 0.0f) {
        float kd = fminf(nut / 0.5f * P.dt / (P.dx * P.dx), 0.15f);
        float4 lapA = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        float lapB = 0.0f;
        const float4 amb = make_float4(P.t0, 0.0f, P.yo2, 0.0f);
#pragma unroll
        for (int k = 0; k < 6; k++) {
          I3 n = c + dir6(k);
          if (g.inb(n)) {
            int j = g.sidx(n);
            if (!((smask >> k) & 1u)) {
              lapA = lapA + (__ldg(s0in + j) - a);
              lapB += __ldg(s1in + j).x - b.x;
            }
          } else if (n.y >= 0) {
            lapA = lapA + (amb - a);
            lapB -= b.x;
          }
        }
        a = a + kd * lapA;
        b.x += kd * lapB;
      }
      float T = a.x;
      float yf = fmaxf(a.y, 0.0f);
      float yo = wclamp(a.z, 0.0f, P.yo2);
      float ys = fmaxf(a.w, 0.0f);
      float ym = fmaxf(b.x, 0.0f);
      float S = 0.0f;
      // solid neighbours in direction order (combust.wgsl:188-208)
#pragma unroll 1
      for (uint32_t sm = smask; sm; sm &= sm - 1u) {
        const int k = __ffs(sm) - 1;
        I3 n = c + dir6(k);
        int j = g.sidx(n);
        float4 pr = __ldg(pyr + j);
        float Ts = __ldg(sol + j).w;
        float rho = rhoOf(P, T);
        if (pr.x > 0.0f) {
          float dm = pr.x * P.dt / (rho * P.dx);
          float inv = 1.0f / (1.0f + dm);
          yf = (yf + dm) * inv;
          yo *= inv;
          ys *= inv;
          ym *= inv;
          T = (T + dm * Ts) * inv;
          S += pr.x / (rho * P.dx);
        }
        T += P.h_conv * (Ts - T) * P.dt / (rho * cpOf(T) * P.dx);
        if (pr.y > 0.0f) {
          yo = fmaxf(yo - 1.33f * pr.y * P.dt / (rho * P.dx), 0.0f);
          T += 0.5f * P.dh_char * pr.y * P.dt / (rho * cpOf(T) * P.dx);
        }
      }
      if (P.ign_on > 0.5f) {
        F3 pc = (tof3(c) + F3{0.5f, 0.5f, 0.5f}) * P.dx;
        float dI = len3(pc - F3{P.ign_x, P.ign_y, P.ign_z});
        float wgt = wclamp(1.0f - dI / P.ign_r, 0.0f, 1.0f);
        if (wgt > 0.0f) {
          T = fmaxf(T, wmix(P.t0, P.ign_temp, smoothstep(0.0f, 0.5f, wgt)));
          yf += P.ign_fuel * wgt * P.dt;
        }
      }
      // Exact shortcuts where a factor is exactly zero.  With gate = 0 the
      // factor 1 - exp(-0) is +0, so dY = lim * 0 (a signed zero); T then
      // changes by a zero (T > 0 stays), q = rho dY dhc / dt and the soot
      // term soot_form dY (...) are zeros of dY's sign (every other factor
      // is positive), so yf, yo, ys take exactly the values the full
      // expressions give, signs of zero included.
      float q;
      const float gate = smoothstep(P.t_ign - 100.0f, P.t_ign + 100.0f, T);
      if (gate == 0.0f) {
        const float dY = fminf(yf, yo / P.s_o2) * 0.0f;
        yf -= dY;
        yo = fmaxf(yo - P.s_o2 * dY, 0.0f);
        q = dY;
        ys += dY;
      } else {
        float rho = rhoOf(P, T);
        float tauU = 0.049f * P.dx * P.dx / (nut + 1e-6f);
        float tauG = sqrtf(2.0f * P.dx / P.g);
        float tau = fmaxf(fminf(tauU, tauG), P.tau_min);
        float lim = fminf(yf, yo / P.s_o2);
        float dY = lim * (1.0f - expf(-gate * P.dt / tau));
        yf -= dY;
        yo = fmaxf(yo - P.s_o2 * dY, 0.0f);
        T += dY * P.dhc / cpOf(T + 0.5f * dY * P.dhc / cpOf(T));
        q = rho * dY * P.dhc / P.dt;
        float rich = smoothstep(0.0f, 0.03f, yf);
        ys += P.soot_form * dY * (0.25f + 0.75f * rich);
      }
      // below the oxidation onset the factor is exp(-0) = 1
      const float oxs = smoothstep(P.soot_ox_t, P.soot_ox_t + 300.0f, T);
      if (oxs != 0.0f) {
        float oxg = oxs * (yo / P.yo2);
        ys *= expf(-P.soot_ox * oxg * P.dt);
      }
      float cold = 1.0f - smoothstep(450.0f, 650.0f, T);
      float cv = yf * fminf(P.smoke_conv * cold * P.dt, 1.0f);
      yf -= cv;
      ym += cv;
      float rho = rhoOf(P, T);
      float kap = kapP(P, T, yo, ys);
      float tl = kap * P.rad_len;
      float esc = (tl > 1e-3f) ? (1.0f - expf(-tl)) / tl : 1.0f;
      float prad = 4.0f * kap * esc * SIGMA * (pow4(T) - pow4(P.t0));
      float dTr = fminf(prad * P.dt / (rho * cpOf(T)), 0.5f * fmaxf(T - P.t0, 0.0f));
      T -= dTr;
      float prl = dTr * rho * cpOf(T) / P.dt;
      S += (q - prl) / (rho * cpOf(T) * T);
      float sp = fmaxf(spongeSide(P, g, c), spongeTop(P, g, c));
      if (sp != 0.0f) {
        float dec = 1.0f - expf(-P.dt * 4.0f * sp);
        T = wmix(T, P.t0, dec);
        yf *= 1.0f - dec;
        yo = wmix(yo, P.yo2, dec);
        ys *= 1.0f - dec;
        ym *= 1.0f - dec;
      } else {
        // outside the sponge layers dec = 1 - exp(-0) = +0: T (> 0), yf, ys
        // and ym keep their values; yo gains yo2 * 0 as the mix does
        yo = wmix(yo, P.yo2, 0.0f);
      }
      T = wclamp(T, 250.0f, 2600.0f);
      s0out[i] = make_float4(T, yf, yo, ys);
      s1out[i] = make_float4(ym, q, S, 0.0f);
      if (stats) {
        rho = rhoOf(P, T);
        stH = q * dV;
        stR = prl * dV;
        stS = rho * ys * dV;
        stF = rho * yf * dV;
        stM = rho * ym * dV;
        stT = T;
      }
    }
  }
  if (stats) {
    // per-layer HRR (combust.wgsl:263): cells with q*dV > 1 W.  A warp is
    // one x-row (blockDim.x == 32), so all its lanes share the layer.
    float lay = (active && stH > 1.0f) ? stH : 0.0f;
    lay = warp_sum(lay);
    if (threadIdx.x == 0 && lay != 0.0f && c.y < PYRO_MAX_LAYERS) atomicAdd(stats + 16 + c.y, lay);
    float vals[6] = {stH, stR, stS, stF, stM, stT};
    block_stats<6>(sh, vals, stats, {0, 1, 3, 6, 8, 4}, 1u << 5);
  }
}

// ------------------------------------------------------------------ forces
// Vorticity-confinement body force at each cell centre (fluid.wgsl:167-181),
// computed once per cell; forces adds the two cells' vectors per face
// exactly as the reference's fc += confine(a); fc += confine(c).
__global__ void __launch_bounds__(256) k_confine(const PyroParams* __restrict__ Pp, Grid g,
                                                 const float4* __restrict__ s0,
                                                 const float4* __restrict__ s1,
                                                 const float4* __restrict__ curl,
                                                 float4* __restrict__ conf) {
  I3 c = thread_cell();
  if (!g.inb(c)) return;
  const PyroParams& P = *Pp;
  int i = g.sidx(c);
  float4 a = __ldg(s0 + i);
  float T = a.x;
  float smoke = a.w + __ldg(s1 + i).x;
  float gate = fmaxf(smoothstep(P.vort_t, P.vort_t + 500.0f, T),
                     0.35f * smoothstep(0.0f, 2e-4f, smoke));
  F3 f{0.0f, 0.0f, 0.0f};
  if (gate > 0.0f) {
    auto cm = [&](I3 q) { return __ldg(curl + g.sidx(g.clampC(q))).w; };
    const I3 X{1, 0, 0}, Y{0, 1, 0}, Z{0, 0, 1};
    F3 gr{cm(c + X) - cm(c - X), cm(c + Y) - cm(c - Y), cm(c + Z) - cm(c - Z)};
    float gl = len3(gr);
    if (!(gl < 1e-6f)) {
      float4 cw = __ldg(curl + i);
      f = (P.vort * P.dx) * cross3(gr / gl, F3{cw.x, cw.y, cw.z}) * gate;
      float fl = len3(f);
      if (fl > 60.0f) f = f * (60.0f / fl);
    }
  }
  conf[i] = make_float4(f.x, f.y, f.z, 0.0f);
}

__device__ __forceinline__ float comp4(float4 v, int k) { return k == 0 ? v.x : (k == 1 ? v.y : v.z); }

__global__ void __launch_bounds__(256) k_forces(const PyroParams* __restrict__ Pp, Grid g,
                                                float* __restrict__ u, float* __restrict__ v,
                                                float* __restrict__ w,
                                                const float4* __restrict__ s0,
                                                const float4* __restrict__ s1,
                                                const float4* __restrict__ conf,
                                                const uint32_t* __restrict__ flags) {
  I3 c = thread_cell();
  if (c.x > g.nx || c.y > g.ny || c.z > g.nz) return;
  const PyroParams& P = *Pp;
  int i = g.vidx(c);
  bool ib = g.inb(c);
  int ic = ib ? g.sidx(c) : 0;
  bool sc = ib && __ldg(flags + ic) == 1u;
  float4 cc = ib ? __ldg(conf + ic) : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  float Tc = ib ? __ldg(s0 + ic).x : P.t0;
  I3 cl = g.clampC(c);
  float ss = spongeSide(P, g, cl);
#pragma unroll
  for (int k = 0; k < 3; k++) {
    if (!g.compValid(k, c)) continue;
    I3 a = c - unitI(k);
    bool ia = g.inb(a);
    int iaa = ia ? g.sidx(a) : 0;
    bool sa = ia && __ldg(flags + iaa) == 1u;
    if ((k == 1 && c.y == 0) || sc || sa) continue;
    float f = 0.0f;
    if (k == 1) {
      float Ta = P.t0, Tb = P.t0, ma = 0.0f, mb = 0.0f;
      if (ia) { float4 s = __ldg(s0 + iaa); Ta = s.x; ma = s.w + __ldg(s1 + iaa).x; }
      if (ib) { float4 s = __ldg(s0 + ic); Tb = s.x; mb = s.w + __ldg(s1 + ic).x; }
      if (!ia) { Ta = Tb; ma = mb; }
      if (!ib) { Tb = Ta; mb = ma; }
      float Tf = 0.5f * (Ta + Tb);
      f += P.g * P.buoy * (Tf - P.t0) / Tf - P.g * P.smoke_w * 0.5f * (ma + mb);
    }
    float fc = 0.0f, n = 0.0f;
    if (ia) { fc = fc + comp4(__ldg(conf + iaa), k); n += 1.0f; }
    if (ib) { fc = fc + comp4(cc, k); n += 1.0f; }
    // n is 1 or 2: the quotient equals the product with 1 or 1/2 exactly
    if (n > 0.0f) f += fc * (n == 2.0f ? 0.5f : 1.0f);
    float* vk = k == 0 ? u : (k == 1 ? v : w);
    float uu = vk[i];
    uu += f * P.dt;
    if (k != 1) {
      // without wind the relaxation rate is 8 ss; where that is 0 too, the
      // mix weight 1 - exp(-0) is +0 and the mix is uu * 1 + wv * 0
      float kr = 8.0f * ss;
      if (P.wind_relax != 0.0f) {
        float hot = smoothstep(350.0f, 900.0f, Tc);
        kr = P.wind_relax * (1.0f - 0.85f * hot) + 8.0f * ss;
      }
      float wv = k == 0 ? P.wind_x : P.wind_z;
      uu = kr != 0.0f ? wmix(uu, wv, 1.0f - expf(-kr * P.dt)) : uu + wv * 0.0f;
    } else {
      float st = spongeTop(P, g, cl);
      if (st > 0.0f) uu = wmix(uu, fmaxf(uu, 0.0f), 1.0f - expf(-8.0f * st * P.dt));
    }
    uu = wclamp(uu, -40.0f, 40.0f);
    vk[i] = uu;
  }
}

// -------------------------------------------------------------- divergence
__global__ void __launch_bounds__(256) k_divergence(const PyroParams* __restrict__ Pp, Grid g,
                                                    const float* __restrict__ u,
                                                    const float* __restrict__ v,
                                                    const float* __restrict__ w,
                                                    const float4* __restrict__ s1,
                                                    const uint32_t* __restrict__ flags,
                                                    float* __restrict__ b) {
  I3 c = thread_cell();
  if (!g.inb(c)) return;
  int i = g.sidx(c);
  int j = g.vidx(c);
  const int sy = g.nx + 1, sz = (g.nx + 1) * (g.ny + 1);
  // every load first, then the flag decides
  const float u0 = __ldg(u + j), u1 = __ldg(u + j + 1), v0 = __ldg(v + j), v1 = __ldg(v + j + sy);
  const float w0 = __ldg(w + j), w1 = __ldg(w + j + sz), src = __ldg(s1 + i).z;
  if (__ldg(flags + i) == 1u) { b[i] = 0.0f; return; }
  float d = (u1 - u0 + v1 - v0 + w1 - w0) / Pp->dx;
  b[i] = d - src;
}

// ----------------------------------------------------------------- project
__global__ void __launch_bounds__(256) k_project(const PyroParams* __restrict__ Pp, Grid g,
                                                 float* __restrict__ u, float* __restrict__ v,
                                                 float* __restrict__ w,
                                                 const float* __restrict__ phi,
                                                 const uint32_t* __restrict__ flags) {
  I3 c = thread_cell();
  if (c.x > g.nx || c.y > g.ny || c.z > g.nz) return;
  const float dx = Pp->dx;
  int i = g.vidx(c);
  // every load first: the cell's and its three lower neighbours' flag and
  // phi, and the three faces
  bool ib = g.inb(c);
  const int ic = ib ? g.sidx(c) : 0;
  const uint32_t fc = ib ? __ldg(flags + ic) : 0u;
  const float pc = ib ? __ldg(phi + ic) : 0.0f;
  bool ia[3], valid[3];
  uint32_t fa[3];
  float pa[3], vv[3];
#pragma unroll
  for (int k = 0; k < 3; k++) {
    const I3 a = c - unitI(k);
    ia[k] = g.inb(a);
    const int ja = ia[k] ? g.sidx(a) : 0;
    fa[k] = ia[k] ? __ldg(flags + ja) : 0u;
    pa[k] = ia[k] ? __ldg(phi + ja) : 0.0f;
    valid[k] = g.compValid(k, c);
    const float* vk = k == 0 ? u : (k == 1 ? v : w);
    vv[k] = valid[k] ? vk[i] : 0.0f;
  }
  const bool sc = ib && fc == 1u;
#pragma unroll
  for (int k = 0; k < 3; k++) {
    if (!valid[k]) continue;
    const bool sa = ia[k] && fa[k] == 1u;
    float* vk = k == 0 ? u : (k == 1 ? v : w);
    float uu = 0.0f;
    if (!((k == 1 && c.y == 0) || sc || sa)) {
      uu = vv[k];
      uu -= (pc - pa[k]) / dx;
    }
    vk[i] = uu;
  }
}

}  // namespace

// ----------------------------------------------------------------- launchers
#define PYRO_BLOCK dim3(BX, BY, BZ)

cudaError_t launch_solid(const PyroParams* P, Dims3 d, const float4* solIn, float4* solOut,
                         float4* pyr, uint32_t* flags, const float4* s0, float* stats,
                         cudaStream_t st) {
  Grid g{d.nx, d.ny, d.nz};
  k_solid<<<grid_for(d.nx, d.ny, d.nz), PYRO_BLOCK, 0, st>>>(P, g, solIn, solOut, pyr, flags, s0,
                                                           stats);
  return cudaGetLastError();
}
cudaError_t launch_curl(const PyroParams* P, Dims3 d, const float* u, const float* v,
                        const float* w, float4* curl, float* stats, cudaStream_t st) {
  Grid g{d.nx, d.ny, d.nz};
  k_curl<<<grid_for(d.nx, d.ny, d.nz), PYRO_BLOCK, 0, st>>>(P, g, u, v, w, curl, stats);
  return cudaGetLastError();
}
cudaError_t launch_adv_vel1(const PyroParams* P, Dims3 d, const float* u, const float* v,
                            const float* w, float* hu, float* hv, float* hw, float* lohi,
                            cudaStream_t st) {
  Grid g{d.nx, d.ny, d.nz};
  k_adv_vel1<<<grid_for(d.nx + 1, d.ny + 1, d.nz + 1), PYRO_BLOCK, 0, st>>>(P, g, u, v, w, hu, hv,
                                                                           hw, lohi);
  return cudaGetLastError();
}
cudaError_t launch_adv_vel2(const PyroParams* P, Dims3 d, const float* u, const float* v,
                            const float* w, const float* hu, const float* hv, const float* hw,
                            const float* lohi, float* ou, float* ov, float* ow,
                            const uint32_t* flags, cudaStream_t st) {
  Grid g{d.nx, d.ny, d.nz};
  k_adv_vel2<<<grid_for(d.nx + 1, d.ny + 1, d.nz + 1), PYRO_BLOCK, 0, st>>>(
      P, g, u, v, w, hu, hv, hw, lohi, ou, ov, ow, flags);
  return cudaGetLastError();
}
cudaError_t launch_adv_s1(const PyroParams* P, Dims3 d, const float* u, const float* v,
                          const float* w, const float4* s0, const float4* s1, float4* h0,
                          float4* h1, float* bt, cudaStream_t st) {
  Grid g{d.nx, d.ny, d.nz};
  k_adv_s1<<<grid_for(d.nx, d.ny, d.nz), PYRO_BLOCK, 0, st>>>(P, g, u, v, w, s0, s1, h0, h1, bt);
  return cudaGetLastError();
}
cudaError_t launch_adv_s2(const PyroParams* P, Dims3 d, const float* u, const float* v,
                          const float* w, const float4* s0, const float4* s1, const float4* h0,
                          const float4* h1, const float* bt, float4* o0, float4* o1,
                          cudaStream_t st) {
  Grid g{d.nx, d.ny, d.nz};
  k_adv_s2<<<grid_for(d.nx, d.ny, d.nz), PYRO_BLOCK, 0, st>>>(P, g, u, v, w, s0, s1, h0, h1, bt,
                                                            o0, o1);
  return cudaGetLastError();
}
cudaError_t launch_react(const PyroParams* P, Dims3 d, const float4* s0in, const float4* s1in,
                         float4* s0out, float4* s1out, const uint32_t* flags, const float4* sol,
                         const float4* pyr, const float4* curl, float* stats, cudaStream_t st) {
  Grid g{d.nx, d.ny, d.nz};
  k_react<<<grid_for(d.nx, d.ny, d.nz), PYRO_BLOCK, 0, st>>>(P, g, s0in, s1in, s0out, s1out, flags,
                                                           sol, pyr, curl, stats);
  return cudaGetLastError();
}
cudaError_t launch_forces(const PyroParams* P, Dims3 d, float* u, float* v, float* w,
                          const float4* s0, const float4* s1, const float4* curl,
                          float4* conf, const uint32_t* flags, cudaStream_t st) {
  Grid g{d.nx, d.ny, d.nz};
  k_confine<<<grid_for(d.nx, d.ny, d.nz), PYRO_BLOCK, 0, st>>>(P, g, s0, s1, curl, conf);
  k_forces<<<grid_for(d.nx + 1, d.ny + 1, d.nz + 1), PYRO_BLOCK, 0, st>>>(P, g, u, v, w, s0, s1,
                                                                         conf, flags);
  return cudaGetLastError();
}
cudaError_t launch_divergence(const PyroParams* P, Dims3 d, const float* u, const float* v,
                              const float* w, const float4* s1, const uint32_t* flags, float* b,
                              cudaStream_t st) {
  Grid g{d.nx, d.ny, d.nz};
  k_divergence<<<grid_for(d.nx, d.ny, d.nz), PYRO_BLOCK, 0, st>>>(P, g, u, v, w, s1, flags, b);
  return cudaGetLastError();
}
cudaError_t launch_project(const PyroParams* P, Dims3 d, float* u, float* v, float* w,
                           const float* phi, const uint32_t* flags, cudaStream_t st) {
  Grid g{d.nx, d.ny, d.nz};
  k_project<<<grid_for(d.nx + 1, d.ny + 1, d.nz + 1), PYRO_BLOCK, 0, st>>>(P, g, u, v, w, phi,
                                                                          flags);
  return cudaGetLastError();
}

}  // namespace pyro
