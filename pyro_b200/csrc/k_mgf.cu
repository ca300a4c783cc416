// k_mgf.cu — fused multigrid kernels (the V-cycle's fine and middle levels).
//
// The reference sweeps each level with one dispatch per colour
// (src/shaders/mg.wgsl:5-36), reading every neighbour's u32 solid flag, and
// restricts in a separate dispatch (mg.wgsl:38-83).  Here:
//
//  * k_mg_meta packs, once per substep and level, a byte per cell: bit k
//    (k = +x,-x,+y,-y,+z,-z) = neighbour k is inside the level and fluid,
//    bit 6 = the cell is solid.  The smoother's neighbour count is the
//    popcount plus the Dirichlet faces the cell touches.
//  * k_mg_pass4z / k_mg_pass2z update the cells of one colour in 4-cell
//    (rows of a multiple of 4) or 2-cell (other even rows) chunks, one to
//    four planes per thread, with the colour parity the same across each
//    warp (no per-lane selects); odd rows take k_mg_pass, one colour cell
//    per thread; k_mg_restrict_m / k_mg_prolong_m work one thread per
//    coarse cell.
//
// Per-cell arithmetic is the reference's, in its order, so results equal the
// per-pass kernels bit for bit.
#include <cuda_bf16.h>

#include "common.cuh"
#include "kernels.h"

namespace pyro {

namespace {

__device__ __forceinline__ float ldv(const float* p) { return *p; }
__device__ __forceinline__ float ldv(const __nv_bfloat16* p) { return __bfloat162float(*p); }
__device__ __forceinline__ void stv(float* p, float v) { *p = v; }
__device__ __forceinline__ void stv(__nv_bfloat16* p, float v) { *p = __float2bfloat16_rn(v); }

struct L {
  int nx, ny, nz;
  __device__ __forceinline__ bool inb(int x, int y, int z) const {
    return (unsigned)x < (unsigned)nx && (unsigned)y < (unsigned)ny && (unsigned)z < (unsigned)nz;
  }
  __device__ __forceinline__ int idx(int x, int y, int z) const { return x + nx * (y + ny * z); }
};

constexpr uint8_t META_SOLID = 0x40;

// Dirichlet faces a cell touches (they count in cnt with phi = 0).
__device__ __forceinline__ int dirichlet_faces(const L& d, int x, int y, int z, int bc_mode) {
  int n = (y == d.ny - 1);
  if (bc_mode == 0) n += (x == 0) + (x == d.nx - 1) + (z == 0) + (z == d.nz - 1);
  return n;
}

__global__ void __launch_bounds__(256) k_mg_meta(L d, const uint32_t* __restrict__ f,
                                                 uint8_t* __restrict__ meta) {
  pdl_trigger();
  pdl_wait();
  int x = blockIdx.x * 32 + threadIdx.x;
  int y = blockIdx.y * 4 + threadIdx.y;
  int z = blockIdx.z * 2 + threadIdx.z;
  if (!d.inb(x, y, z)) return;
  uint8_t m = (__ldg(f + d.idx(x, y, z)) == 1u) ? META_SOLID : 0;
#pragma unroll
  for (int k = 0; k < 6; k++) {
    int a = x + (k == 0) - (k == 1), b = y + (k == 2) - (k == 3), c = z + (k == 4) - (k == 5);
    if (d.inb(a, b, c) && __ldg(f + d.idx(a, b, c)) != 1u) m |= (uint8_t)(1u << k);
  }
  meta[d.idx(x, y, z)] = m;
}

// Coarse solid flag = every in-domain child solid (mg.wgsl:73-82, fc).
__global__ void __launch_bounds__(256) k_mg_flags_down(L df, const uint32_t* __restrict__ ff,
                                                       L dc, uint32_t* __restrict__ fc) {
  pdl_trigger();
  pdl_wait();
  int x = blockIdx.x * 32 + threadIdx.x;
  int y = blockIdx.y * 4 + threadIdx.y;
  int z = blockIdx.z * 2 + threadIdx.z;
  if (!dc.inb(x, y, z)) return;
  bool fluid = false;
#pragma unroll
  for (int k = 0; k < 8; k++) {
    int cx = 2 * x + (k & 1), cy = 2 * y + ((k >> 1) & 1), cz = 2 * z + ((k >> 2) & 1);
    if (df.inb(cx, cy, cz) && __ldg(ff + df.idx(cx, cy, cz)) != 1u) fluid = true;
  }
  fc[dc.idx(x, y, z)] = fluid ? 0u : 1u;
}

// Two cells x0, x0 + 1 of a row (x0 even).  V2: the row length is even, so
// both exist and the pair is aligned for one vector access; otherwise two
// scalar accesses, the second only when `two`.
__device__ __forceinline__ float2 ld2(const float* p) {
  return *reinterpret_cast<const float2*>(p);
}
__device__ __forceinline__ float2 ld2(const __nv_bfloat16* p) {
  return __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(p));
}
__device__ __forceinline__ void st2(float* p, float2 v) { *reinterpret_cast<float2*>(p) = v; }
__device__ __forceinline__ void st2(__nv_bfloat16* p, float2 v) {
  *reinterpret_cast<__nv_bfloat162*>(p) = __floats2bfloat162_rn(v.x, v.y);
}
template <bool V2, typename TS>
__device__ __forceinline__ float2 ldp(const TS* p, bool two) {
  if constexpr (V2) return ld2(p);
  return make_float2(ldv(p), two ? ldv(p + 1) : 0.0f);
}
template <bool V2, typename TS>
__device__ __forceinline__ void stp(TS* p, float2 v, bool two) {
  if constexpr (V2) {
    st2(p, v);
  } else {
    stv(p, v.x);
    if (two) stv(p + 1, v.y);
  }
}

// Fluid-weighted trilinear prolongation with the coarse solid bit from the
// coarse meta (mg.wgsl:85-120), in place on the fine level.  One thread per
// coarse cell (X, Y, Z) updates its 2x2x2 fine children.  Per axis, a fine
// cell 2X + s samples the coarse cells floor((2X + s + 0.5) / 2 - 0.5) + o,
// o = 0, 1, which is X - 1 + s + o (clamped to the level), with weight
// 1 - fr = 0.25, fr = 0.75 for s = 0 and 0.75, 0.25 for s = 1: every weight
// and weight product is exact, so with the corners visited in the
// reference's order (x fastest) the sums equal the per-fine-cell form bit
// for bit.  The 27 clamped coarse cells are loaded once.
template <typename TS, bool V2>
__global__ void __launch_bounds__(256) k_mg_prolong_m(L df, const TS* __restrict__ pc,
                                                      const uint8_t* __restrict__ mf,
                                                      TS* __restrict__ pf, L dc,
                                                      const uint8_t* __restrict__ mc) {
  pdl_trigger();
  pdl_wait();
  const int X = blockIdx.x * 32 + threadIdx.x;
  const int Y = blockIdx.y * 4 + threadIdx.y;
  const int Z = blockIdx.z * 2 + threadIdx.z;
  if (!dc.inb(X, Y, Z)) return;
  int cx[3], cy[3], cz[3];
#pragma unroll
  for (int q = 0; q < 3; q++) {
    cx[q] = min(max(X - 1 + q, 0), dc.nx - 1);
    cy[q] = min(max(Y - 1 + q, 0), dc.ny - 1) * dc.nx;
    cz[q] = min(max(Z - 1 + q, 0), dc.nz - 1) * (dc.nx * dc.ny);
  }
  float cv[27];
  uint32_t solid = 0;
#pragma unroll
  for (int q = 0; q < 27; q++) {
    const int j = cx[q % 3] + cy[(q / 3) % 3] + cz[q / 9];
    const float raw = ldv(pc + j);  // loaded regardless, so it need not wait for the mask
    const bool s = (__ldg(mc + j) & META_SOLID) != 0;
    solid |= (uint32_t)s << q;
    cv[q] = s ? 0.0f : raw;
  }
  const int fx = 2 * X;
  const bool two = fx + 1 < df.nx;
#pragma unroll
  for (int sz = 0; sz < 2; sz++) {
    const int fz = 2 * Z + sz;
    if (fz >= df.nz) break;
#pragma unroll
    for (int sy = 0; sy < 2; sy++) {
      const int fy = 2 * Y + sy;
      if (fy >= df.ny) break;
      const int i = df.idx(fx, fy, fz);
      const uint32_t m0 = __ldg(mf + i), m1 = two ? __ldg(mf + i + 1) : META_SOLID;
      if (m0 & m1 & META_SOLID) continue;
      float2 P = ldp<V2>(pf + i, two);
#pragma unroll
      for (int sx = 0; sx < 2; sx++) {
        if ((sx ? m1 : m0) & META_SOLID) continue;
        if (solid == 0u) {
          // no solid coarse neighbour: the eight weights are multiples of
          // 1/64 that sum to exactly 1, so acc / ws is acc itself
          float acc = 0.0f;
#pragma unroll
          for (int k = 0; k < 8; k++) {
            const int ox = k & 1, oy = (k >> 1) & 1, oz = (k >> 2) & 1;
            const int q = (sx + ox) + 3 * (sy + oy) + 9 * (sz + oz);
            const float w = (sx != ox ? 0.75f : 0.25f) * (sy != oy ? 0.75f : 0.25f) *
                            (sz != oz ? 0.75f : 0.25f);
            acc += w * cv[q];
          }
          if (sx) P.y = P.y + acc;
          else P.x = P.x + acc;
          continue;
        }
        float acc = 0.0f, ws = 0.0f;
#pragma unroll
        for (int k = 0; k < 8; k++) {
          const int ox = k & 1, oy = (k >> 1) & 1, oz = (k >> 2) & 1;
          const int q = (sx + ox) + 3 * (sy + oy) + 9 * (sz + oz);
          if ((solid >> q) & 1u) continue;
          const float w = (sx != ox ? 0.75f : 0.25f) * (sy != oy ? 0.75f : 0.25f) *
                          (sz != oz ? 0.75f : 0.25f);
          acc += w * cv[q];
          ws += w;
        }
        if (ws > 1e-4f) {
          if (sx) P.y = P.y + acc / ws;
          else P.x = P.x + acc / ws;
        }
      }
      stp<V2>(pf + i, P, two);
    }
  }
}

// Four cells of a row as one vector access (FP32 or BF16 storage).
__device__ __forceinline__ float4 ld4(const float* p) {
  return *reinterpret_cast<const float4*>(p);
}
__device__ __forceinline__ float4 ld4(const __nv_bfloat16* p) {
  uint2 u = *reinterpret_cast<const uint2*>(p);
  float2 a = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&u.x));
  float2 c = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&u.y));
  return make_float4(a.x, a.y, c.x, c.y);
}
__device__ __forceinline__ void st4(float* p, float4 v) { *reinterpret_cast<float4*>(p) = v; }
__device__ __forceinline__ void st4(__nv_bfloat16* p, float4 v) {
  uint2 u;
  *reinterpret_cast<__nv_bfloat162*>(&u.x) = __floats2bfloat162_rn(v.x, v.y);
  *reinterpret_cast<__nv_bfloat162*>(&u.y) = __floats2bfloat162_rn(v.z, v.w);
  *reinterpret_cast<uint2*>(p) = u;
}

// The two cells of the pass's colour in one 4-cell chunk x0..x0+3 of a row
// whose colour parity ODD = (y + z + colour) & 1 is known at compile time:
// cell a = x0 + ODD and cell b = x0 + ODD + 2, each with the reference's
// per-cell arithmetic (mg.wgsl:17-36) and neighbour order (+x, -x, +y, -y,
// +z, -z).  P0 is the chunk, left / right phi at x0 - 1 and x0 + 4, Yp ... Zm
// the neighbour rows' chunks, m4 the four mask bytes, da / db the Dirichlet
// faces of cells a and b.
template <bool ODD>
__device__ __forceinline__ bool chunk_colour(float4& P, const float4 P0, float left, float right,
                                             const float4 Yp, const float4 Ym, const float4 Zp,
                                             const float4 Zm, const float4 B, uint32_t m4, int da,
                                             int db, float h2, float omega) {
  const uint32_t ma = ODD ? (m4 >> 8) & 0xFFu : m4 & 0xFFu;
  const uint32_t mb = ODD ? (m4 >> 24) : (m4 >> 16) & 0xFFu;
  bool any = false;
  if (!(ma & META_SOLID)) {
    float sum = 0.0f;
    if (ma & 1u) sum += ODD ? P0.z : P0.y;
    if (ma & 2u) sum += ODD ? P0.x : left;
    if (ma & 4u) sum += ODD ? Yp.y : Yp.x;
    if (ma & 8u) sum += ODD ? Ym.y : Ym.x;
    if (ma & 16u) sum += ODD ? Zp.y : Zp.x;
    if (ma & 32u) sum += ODD ? Zm.y : Zm.x;
    const float cnt = (float)(__popc(ma & 63u) + da);
    if (cnt >= 0.5f) {
      const float v = wmix(ODD ? P0.y : P0.x, (sum - h2 * (ODD ? B.y : B.x)) / cnt, omega);
      if (ODD) P.y = v; else P.x = v;
      any = true;
    }
  }
  if (!(mb & META_SOLID)) {
    float sum = 0.0f;
    if (mb & 1u) sum += ODD ? right : P0.w;
    if (mb & 2u) sum += ODD ? P0.z : P0.y;
    if (mb & 4u) sum += ODD ? Yp.w : Yp.z;
    if (mb & 8u) sum += ODD ? Ym.w : Ym.z;
    if (mb & 16u) sum += ODD ? Zp.w : Zp.z;
    if (mb & 32u) sum += ODD ? Zm.w : Zm.z;
    const float cnt = (float)(__popc(mb & 63u) + db);
    if (cnt >= 0.5f) {
      const float v = wmix(ODD ? P0.w : P0.z, (sum - h2 * (ODD ? B.w : B.z)) / cnt, omega);
      if (ODD) P.w = v; else P.z = v;
      any = true;
    }
  }
  return any;
}

// One colour pass with the neighbour mask: thread (hx, y, z) updates the
// cell x = 2 hx + ((y + z + colour) & 1) (mg.wgsl:17-36) reading its own
// mask and b and the neighbours the mask marks.
template <typename TS>
__global__ void __launch_bounds__(256) k_mg_pass(L d, float h2, const TS* __restrict__ b,
                                                 const uint8_t* __restrict__ meta,
                                                 TS* __restrict__ p, int color, float omega,
                                                 int bc_mode) {
  pdl_trigger();
  pdl_wait();
  int y = blockIdx.y * 4 + threadIdx.y;
  int z = blockIdx.z * 2 + threadIdx.z;
  int x = (int)(blockIdx.x * 32 + threadIdx.x) * 2 + ((y + z + color) & 1);
  if (x >= d.nx || y >= d.ny || z >= d.nz) return;
  int i = d.idx(x, y, z);
  uint32_t m = __ldg(meta + i);
  if (m & META_SOLID) return;
  const int sy = d.nx, sz = d.nx * d.ny;
  float sum = 0.0f;
  if (m & 1u) sum += ldv(p + i + 1);
  if (m & 2u) sum += ldv(p + i - 1);
  if (m & 4u) sum += ldv(p + i + sy);
  if (m & 8u) sum += ldv(p + i - sy);
  if (m & 16u) sum += ldv(p + i + sz);
  if (m & 32u) sum += ldv(p + i - sz);
  float cnt = (float)(__popc(m & 63u) + dirichlet_faces(d, x, y, z, bc_mode));
  if (cnt < 0.5f) return;
  stv(p + i, wmix(ldv(p + i), (sum - h2 * ldv(b + i)) / cnt, omega));
}


// One colour pass over rows of a multiple of 4 cells with warp-uniform
// colour parity.  Block (8, 16): thread (tx, ty) takes the 4-cell chunk
// 8 blockIdx.x + tx of row y = 16 blockIdx.y + ry and ZT consecutive planes
// from z = ZT blockIdx.z, where warp w = ty / 4 holds rows
// ry = 8 (w / 2) + 2 (ty % 4) + w % 2: the four rows of a warp have one
// parity, so (y + z + colour) & 1 is the same in every lane and the update
// is compiled once per parity with its cells at fixed positions in the
// chunk (chunk_colour).  Per plane a thread loads b, the masks and the
// +-y rows; the -z row, the chunk and the +z row carry over from the
// previous plane (their cells of the other colour are not written in this
// pass), and phi at x0 - 1 and x0 + 4 comes from the neighbouring lanes of
// the same row.  Results equal the reference's pass bit for bit.
//
// Two more forms serve the first and the last pass on level 0 of the CG
// preconditioner's V-cycle:
//  * PASS_FIRST: phi is zero everywhere (the V-cycle's initial guess), so
//    no phi is read; the right-hand side comes in FP32 (b32) and, with BF16
//    storage, is written rounded to BF16 into b (the copy later passes
//    read) and used rounded; every cell of the chunk is written (the
//    colour's cells updated, the others 0).  This replaces clearing phi,
//    converting b and the pass itself.
//  * PASS_LAST_F32: the pass on BF16 storage whose chunk, every cell, is
//    written widened to FP32 into out (the V-cycle's result) instead of
//    back into p; the updated cells are rounded to BF16 first, as a store
//    to p and a conversion would do.
enum { PASS = 0, PASS_FIRST = 1, PASS_LAST_F32 = 2 };

template <typename TS>
__device__ __forceinline__ float4 round_to(float4 v) {
  if constexpr (sizeof(TS) == 2) {
    const float2 a = __bfloat1622float2(__floats2bfloat162_rn(v.x, v.y));
    const float2 c = __bfloat1622float2(__floats2bfloat162_rn(v.z, v.w));
    return make_float4(a.x, a.y, c.x, c.y);
  }
  return v;
}

template <typename TS, int ZT, int MODE>
__global__ void __launch_bounds__(128) k_mg_pass4z(L d, float h2, TS* __restrict__ b,
                                                   const uint8_t* __restrict__ meta,
                                                   TS* __restrict__ p, int color, float omega,
                                                   int bc_mode, const float* __restrict__ b32,
                                                   float* __restrict__ out) {
  pdl_trigger();
  pdl_wait();
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int w = ty >> 2;
  const int y = blockIdx.y * 16 + (w >> 1) * 8 + 2 * (ty & 3) + (w & 1);
  const int x0 = (blockIdx.x * 8 + tx) * 4;
  const bool act = x0 < d.nx && y < d.ny;
  const bool rd = act && MODE != PASS_FIRST;  // phi is read (not the zero guess)
  const int sy = d.nx, sz = d.nx * d.ny;
  const int zb = blockIdx.z * ZT;
  const bool open = bc_mode == 0;
  const float4 zero = make_float4(0.f, 0.f, 0.f, 0.f);
  // row start of plane zb; the window -z / chunk / +z
  int i0 = (zb * d.ny + y) * d.nx + x0;
  float4 Zm = (rd && zb > 0) ? ld4(p + i0 - sz) : zero;
  float4 P0 = rd ? ld4(p + i0) : zero;
  float4 Zp = (rd && zb + 1 < d.nz) ? ld4(p + i0 + sz) : zero;
  const int dy = (y == d.ny - 1);
  const int dxa = (open && x0 == 0), dxb = (open && x0 + 4 == d.nx);
#pragma unroll
  for (int k = 0; k < ZT; k++) {
    const int z = zb + k;
    if (z >= d.nz) break;  // the same in every thread of the block
    float4 B = zero;
    if (MODE == PASS_FIRST) {
      if (act) {
        B = round_to<TS>(ld4(b32 + i0));
        if constexpr (sizeof(TS) == 2) st4(b + i0, B);
      }
    } else {
      B = act ? ld4(b + i0) : zero;
    }
    const uint32_t m4 = act ? *reinterpret_cast<const uint32_t*>(meta + i0) : 0x40404040u;
    const float4 Yp = (rd && y + 1 < d.ny) ? ld4(p + i0 + sy) : zero;
    const float4 Ym = (rd && y > 0) ? ld4(p + i0 - sy) : zero;
    // the next plane's +z row, loaded ahead
    const float4 Zn = (rd && k + 1 < ZT && z + 2 < d.nz) ? ld4(p + i0 + 2 * sz) : zero;
    float left = __shfl_up_sync(0xffffffffu, P0.w, 1);
    float right = __shfl_down_sync(0xffffffffu, P0.x, 1);
    if (rd && tx == 0 && x0 > 0) left = ldv(p + i0 - 1);
    if (rd && tx == 7 && x0 + 4 < d.nx) right = ldv(p + i0 + 4);
    const int dyz = dy + (open ? (z == 0) + (z == d.nz - 1) : 0);
    float4 P = P0;
    const bool odd = ((y + z + color) & 1) != 0;  // the same in every lane of the warp
    bool any;
    if (odd)
      any = chunk_colour<true>(P, P0, left, right, Yp, Ym, Zp, Zm, B, m4, dyz, dyz + dxb, h2,
                               omega);
    else
      any = chunk_colour<false>(P, P0, left, right, Yp, Ym, Zp, Zm, B, m4, dyz + dxa, dyz, h2,
                                omega);
    if (MODE == PASS_LAST_F32) {
      if (act) *reinterpret_cast<float4*>(out + i0) = round_to<TS>(P);
    } else if (act && (any || MODE == PASS_FIRST)) {
      st4(p + i0, P);
    }
    Zm = P0;
    P0 = Zp;
    Zp = Zn;
    i0 += sz;
  }
}

// The same pass for rows whose length is not a multiple of 4 (a float4 row
// access would be misaligned there): 2-cell chunks, one cell of the pass's
// colour in each.  Block (16, 8): thread (tx, ty) takes the chunk
// 16 blockIdx.x + tx of row y = 8 blockIdx.y + ry, where warp w = ty / 2
// holds rows ry = 4 (w / 2) + 2 (ty % 2) + w % 2, two rows of one parity;
// the ZT-plane window, the modes and the arithmetic are those of
// k_mg_pass4z.  V2: the row length is even and a chunk is one aligned
// vector access; odd rows take scalar accesses, and a row's last chunk
// holds one cell (the second is treated as solid and never stored), which
// touches the +x face.
template <typename TS>
__device__ __forceinline__ float2 round_to2(float2 v) {
  if constexpr (sizeof(TS) == 2) return __bfloat1622float2(__floats2bfloat162_rn(v.x, v.y));
  return v;
}

// The cell of a 2-cell chunk with the pass's colour: position 1 when ODD,
// else 0 (left / right: phi at x0 - 1 and x0 + 2; dir: its Dirichlet
// faces).
template <bool ODD>
__device__ __forceinline__ bool pair_colour(float2& P, const float2 P0, float left, float right,
                                            const float2 Yp, const float2 Ym, const float2 Zp,
                                            const float2 Zm, const float2 B, uint32_t m2, int dir,
                                            float h2, float omega) {
  const uint32_t m = ODD ? (m2 >> 8) : (m2 & 0xFFu);
  if (m & META_SOLID) return false;
  float sum = 0.0f;
  if (m & 1u) sum += ODD ? right : P0.y;
  if (m & 2u) sum += ODD ? P0.x : left;
  if (m & 4u) sum += ODD ? Yp.y : Yp.x;
  if (m & 8u) sum += ODD ? Ym.y : Ym.x;
  if (m & 16u) sum += ODD ? Zp.y : Zp.x;
  if (m & 32u) sum += ODD ? Zm.y : Zm.x;
  const float cnt = (float)(__popc(m & 63u) + dir);
  if (cnt < 0.5f) return false;
  const float v = wmix(ODD ? P0.y : P0.x, (sum - h2 * (ODD ? B.y : B.x)) / cnt, omega);
  if (ODD) P.y = v; else P.x = v;
  return true;
}

template <typename TS, int ZT, int MODE, bool V2>
__global__ void __launch_bounds__(128) k_mg_pass2z(L d, float h2, TS* __restrict__ b,
                                                   const uint8_t* __restrict__ meta,
                                                   TS* __restrict__ p, int color, float omega,
                                                   int bc_mode, const float* __restrict__ b32,
                                                   float* __restrict__ out) {
  pdl_trigger();
  pdl_wait();
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int w = ty >> 1;
  const int y = blockIdx.y * 8 + (w >> 1) * 4 + 2 * (ty & 1) + (w & 1);
  const int x0 = (blockIdx.x * 16 + tx) * 2;
  const bool act = x0 < d.nx && y < d.ny;
  const bool two = V2 || x0 + 1 < d.nx;  // the chunk's second cell exists
  const bool rd = act && MODE != PASS_FIRST;  // phi is read (not the zero guess)
  const int sy = d.nx, sz = d.nx * d.ny;
  const int zb = blockIdx.z * ZT;
  const bool open = bc_mode == 0;
  const float2 zero = make_float2(0.f, 0.f);
  int i0 = (zb * d.ny + y) * d.nx + x0;
  float2 Zm = (rd && zb > 0) ? ldp<V2>(p + i0 - sz, two) : zero;
  float2 P0 = rd ? ldp<V2>(p + i0, two) : zero;
  float2 Zp = (rd && zb + 1 < d.nz) ? ldp<V2>(p + i0 + sz, two) : zero;
  const int dy = (y == d.ny - 1);
  // Dirichlet x faces of the chunk's cells (position 0 is a row's last cell
  // only in odd rows)
  const int dx0 = open ? (x0 == 0) + (x0 + 1 == d.nx) : 0, dx1 = (open && x0 + 2 == d.nx);
#pragma unroll
  for (int k = 0; k < ZT; k++) {
    const int z = zb + k;
    if (z >= d.nz) break;  // the same in every thread of the block
    const bool odd = ((y + z + color) & 1) != 0;  // the same in every lane of the warp
    float2 B = zero, Yp = zero, Ym = zero;
    uint32_t m2 = 0x4040u;
    if constexpr (V2) {
      if (MODE == PASS_FIRST) {
        if (act) {
          B = round_to2<TS>(ld2(b32 + i0));
          if constexpr (sizeof(TS) == 2) st2(b + i0, B);
        }
      } else if (act) {
        B = ld2(b + i0);
      }
      if (act) m2 = *reinterpret_cast<const uint16_t*>(meta + i0);
      if (rd && y + 1 < d.ny) Yp = ld2(p + i0 + sy);
      if (rd && y > 0) Ym = ld2(p + i0 - sy);
    } else {
      // scalar accesses: of b, the mask and the +-y rows only the element
      // of the pass's colour is used, so only it is loaded
      const int c = odd ? 1 : 0;
      const bool has = act && (c == 0 || two);  // the chunk holds that cell
      auto put = [&](float v) { return odd ? make_float2(0.f, v) : make_float2(v, 0.f); };
      if (MODE == PASS_FIRST) {
        if (act) {
          B = round_to2<TS>(ldp<false>(b32 + i0, two));
          if constexpr (sizeof(TS) == 2) stp<false>(b + i0, B, two);
        }
      } else if (has) {
        B = put(ldv(b + i0 + c));
      }
      if (has) {
        const uint32_t mc = meta[i0 + c];
        m2 = odd ? (mc << 8) | 0x40u : mc | 0x4000u;
      }
      if (rd && has && y + 1 < d.ny) Yp = put(ldv(p + i0 + c + sy));
      if (rd && has && y > 0) Ym = put(ldv(p + i0 + c - sy));
    }
    const float2 Zn = (rd && k + 1 < ZT && z + 2 < d.nz) ? ldp<V2>(p + i0 + 2 * sz, two) : zero;
    float left = __shfl_up_sync(0xffffffffu, P0.y, 1);
    float right = __shfl_down_sync(0xffffffffu, P0.x, 1);
    if (rd && tx == 0 && x0 > 0) left = ldv(p + i0 - 1);
    if (rd && tx == 15 && x0 + 2 < d.nx) right = ldv(p + i0 + 2);
    const int dyz = dy + (open ? (z == 0) + (z == d.nz - 1) : 0);
    float2 P = P0;
    const bool any = odd ? pair_colour<true>(P, P0, left, right, Yp, Ym, Zp, Zm, B, m2,
                                             dyz + dx1, h2, omega)
                         : pair_colour<false>(P, P0, left, right, Yp, Ym, Zp, Zm, B, m2,
                                              dyz + dx0, h2, omega);
    if (MODE == PASS_LAST_F32) {
      if (act) stp<V2>(out + i0, round_to2<TS>(P), two);
    } else if (act && (any || MODE == PASS_FIRST)) {
      stp<V2>(p + i0, P, two);
    }
    Zm = P0;
    P0 = Zp;
    Zp = Zn;
    i0 += sz;
  }
}

// Restriction with the neighbour mask (mg.wgsl:38-83): coarse rhs = mean of
// the fine residuals of the fluid children, coarse guess 0.
// One thread per coarse cell; the children are visited in the reference's
// order (x fastest) as two x-pairs per (y, z) row, whose own, b and +-y,
// +-z neighbour values are loaded as pairs and whose outer x neighbours as
// scalars.
template <typename TS, bool V2>
__global__ void __launch_bounds__(256, 6) k_mg_restrict_m(L df, float h2, const TS* __restrict__ pf,
                                                       const TS* __restrict__ bf,
                                                       const uint8_t* __restrict__ mf, L dc,
                                                       TS* __restrict__ bc, TS* __restrict__ pc,
                                                       int bc_mode) {
  pdl_trigger();
  pdl_wait();
  const int X = blockIdx.x * 32 + threadIdx.x;
  const int Y = blockIdx.y * 4 + threadIdx.y;
  const int Z = blockIdx.z * 2 + threadIdx.z;
  if (!dc.inb(X, Y, Z)) return;
  const int sy = df.nx, sz = df.nx * df.ny;
  const int fx = 2 * X;
  const bool two = fx + 1 < df.nx;
  const bool open = bc_mode == 0;
  float r = 0.0f, nfl = 0.0f;
#pragma unroll
  for (int s_z = 0; s_z < 2; s_z++) {
    const int fz = 2 * Z + s_z;
    if (fz >= df.nz) break;
#pragma unroll
    for (int s_y = 0; s_y < 2; s_y++) {
      const int fy = 2 * Y + s_y;
      if (fy >= df.ny) break;
      const int i = df.idx(fx, fy, fz);
      // the row's loads are issued together, none waiting for the masks
      const float2 zero = make_float2(0.0f, 0.0f);
      const float2 P = ldp<V2>(pf + i, two), B = ldp<V2>(bf + i, two);
      const float2 Yp = fy + 1 < df.ny ? ldp<V2>(pf + i + sy, two) : zero;
      const float2 Ym = fy > 0 ? ldp<V2>(pf + i - sy, two) : zero;
      const float2 Zp = fz + 1 < df.nz ? ldp<V2>(pf + i + sz, two) : zero;
      const float2 Zm = fz > 0 ? ldp<V2>(pf + i - sz, two) : zero;
      const float pl = fx > 0 ? ldv(pf + i - 1) : 0.0f;
      const float pr = fx + 2 < df.nx ? ldv(pf + i + 2) : 0.0f;
      const uint32_t m0 = __ldg(mf + i), m1 = two ? __ldg(mf + i + 1) : META_SOLID;
      if (m0 & m1 & META_SOLID) continue;
      const int dyz = (fy == df.ny - 1) + (open ? (fz == 0) + (fz == df.nz - 1) : 0);
      if (!(m0 & META_SOLID)) {
        nfl += 1.0f;
        float sum = 0.0f;
        if (m0 & 1u) sum += P.y;
        if (m0 & 2u) sum += pl;
        if (m0 & 4u) sum += Yp.x;
        if (m0 & 8u) sum += Ym.x;
        if (m0 & 16u) sum += Zp.x;
        if (m0 & 32u) sum += Zm.x;
        const int dx = open ? (fx == 0) + (fx == df.nx - 1) : 0;
        const float cnt = (float)(__popc(m0 & 63u) + dyz + dx);
        r += B.x - (sum - cnt * P.x) / h2;
      }
      if (!(m1 & META_SOLID)) {
        nfl += 1.0f;
        float sum = 0.0f;
        if (m1 & 1u) sum += pr;
        if (m1 & 2u) sum += P.x;
        if (m1 & 4u) sum += Yp.y;
        if (m1 & 8u) sum += Ym.y;
        if (m1 & 16u) sum += Zp.y;
        if (m1 & 32u) sum += Zm.y;
        const int dx = open ? (fx + 1 == df.nx - 1) : 0;
        const float cnt = (float)(__popc(m1 & 63u) + dyz + dx);
        r += B.y - (sum - cnt * P.y) / h2;
      }
    }
  }
  const int ci = dc.idx(X, Y, Z);
  // eight fluid children: dividing by 8 is the exact product with 1/8
  stv(bc + ci, nfl == 8.0f ? r * 0.125f : (nfl > 0.0f) ? r / fmaxf(nfl, 1.0f) : 0.0f);
  stv(pc + ci, 0.0f);
}

// ---- symmetric V-cycle pieces (MGPCG preconditioner) ----------------------
// The prolongation P of a fine cell c takes, per axis, the two coarse cells
// floor((c+0.5)/2-0.5) + {0,1} (clamped) with weights 1-fr, fr and
// renormalises by the fluid weight sum W_c (mg.wgsl:96-119).  The
// restriction used with it is R = P^T / 8, which makes the V-cycle with
// adjoint pre/post smoothing a symmetric preconditioner for CG.

// 1-D prolongation weight of coarse index J for fine index c.
__device__ __forceinline__ float pw1(int c, int J, int nc) {
  float g = ((float)c + 0.5f) * 0.5f - 0.5f;
  int i0 = (int)floorf(g);
  float fr = g - (float)i0;
  float w = 0.0f;
  if (min(max(i0, 0), nc - 1) == J) w += 1.0f - fr;
  if (min(max(i0 + 1, 0), nc - 1) == J) w += fr;
  return w;
}

// 64 W_c for each fluid fine cell c: W_c is the fluid weight sum of c's
// prolongation row, a sum of products of the per-axis weights 1/4 and 3/4
// (clamped taps counted per corner), so a multiple of 1/64 in [0, 1] and the
// byte is exact; 0 for solid cells.  Built once per flag field.
__global__ void __launch_bounds__(256) k_mg_wsum(L d, const uint8_t* __restrict__ m0, L dc,
                                                 const uint8_t* __restrict__ mc,
                                                 uint8_t* __restrict__ wq) {
  pdl_trigger();
  pdl_wait();
  int x = blockIdx.x * 32 + threadIdx.x;
  int y = blockIdx.y * 4 + threadIdx.y;
  int z = blockIdx.z * 2 + threadIdx.z;
  if (!d.inb(x, y, z)) return;
  int i = d.idx(x, y, z);
  float W = 0.0f;
  if (!(__ldg(m0 + i) & META_SOLID)) {
    float gx = ((float)x + 0.5f) * 0.5f - 0.5f, gy = ((float)y + 0.5f) * 0.5f - 0.5f,
          gz = ((float)z + 0.5f) * 0.5f - 0.5f;
    int ix = (int)floorf(gx), iy = (int)floorf(gy), iz = (int)floorf(gz);
    float fx = gx - (float)ix, fy = gy - (float)iy, fz = gz - (float)iz;
#pragma unroll
    for (int k = 0; k < 8; k++) {
      int ox = k & 1, oy = (k >> 1) & 1, oz = (k >> 2) & 1;
      int cx = min(max(ix + ox, 0), dc.nx - 1), cy = min(max(iy + oy, 0), dc.ny - 1),
          cz = min(max(iz + oz, 0), dc.nz - 1);
      if (__ldg(mc + dc.idx(cx, cy, cz)) & META_SOLID) continue;
      W += (ox ? fx : 1.0f - fx) * (oy ? fy : 1.0f - fy) * (oz ? fz : 1.0f - fz);
    }
  }
  wq[i] = (uint8_t)(int)(W * 64.0f);
}

// r~ = (b - A p) / W_c for fluid fine cells whose prolongation row is not
// empty (wq = 64 W_c from k_mg_wsum), else 0.
template <typename TS>
__global__ void __launch_bounds__(256) k_mg_resid_w(L d, float h2, const TS* __restrict__ p,
                                                    const TS* __restrict__ b,
                                                    const uint8_t* __restrict__ m0,
                                                    const uint8_t* __restrict__ wq, int bc_mode,
                                                    TS* __restrict__ rt) {
  pdl_trigger();
  pdl_wait();
  int x = blockIdx.x * 32 + threadIdx.x;
  int y = blockIdx.y * 4 + threadIdx.y;
  int z = blockIdx.z * 2 + threadIdx.z;
  if (!d.inb(x, y, z)) return;
  int i = d.idx(x, y, z);
  uint32_t m = __ldg(m0 + i);
  const uint32_t w = __ldg(wq + i);
  float out = 0.0f;
  if (!(m & META_SOLID) && w != 0u) {
    const int sy = d.nx, sz = d.nx * d.ny;
    float sum = 0.0f;
    if (m & 1u) sum += ldv(p + i + 1);
    if (m & 2u) sum += ldv(p + i - 1);
    if (m & 4u) sum += ldv(p + i + sy);
    if (m & 8u) sum += ldv(p + i - sy);
    if (m & 16u) sum += ldv(p + i + sz);
    if (m & 32u) sum += ldv(p + i - sz);
    float cnt = (float)(__popc(m & 63u) + dirichlet_faces(d, x, y, z, bc_mode));
    float r = ldv(b + i) - (sum - cnt * ldv(p + i)) / h2;
    out = r / ((float)w * 0.015625f);
  }
  stv(rt + i, out);
}

// Coarse rhs = (1/8) sum_c P[c,J] r~[c]; coarse guess 0.  A coarse cell
// with a neighbour on each side along every axis (1 <= X <= nc - 2) takes
// the fine cells 2X - 1 .. 2X + 2 with weights 1/4, 3/4, 3/4, 1/4 per axis
// and sums them axis by axis; the others evaluate the clamped weights.
template <typename TS>
__global__ void __launch_bounds__(256) k_mg_restrict_t(L df, const TS* __restrict__ rt,
                                                       const uint8_t* __restrict__ mf, L dc,
                                                       const uint8_t* __restrict__ mc,
                                                       TS* __restrict__ bc, TS* __restrict__ pc) {
  pdl_trigger();
  pdl_wait();
  int X = blockIdx.x * 32 + threadIdx.x;
  int Y = blockIdx.y * 4 + threadIdx.y;
  int Z = blockIdx.z * 2 + threadIdx.z;
  if (!dc.inb(X, Y, Z)) return;
  int J = dc.idx(X, Y, Z);
  float acc = 0.0f;
  if (!(__ldg(mc + J) & META_SOLID)) {
    const bool inner = X >= 1 && X <= dc.nx - 2 && Y >= 1 && Y <= dc.ny - 2 && Z >= 1 &&
                       Z <= dc.nz - 2;
    if (inner) {
      const TS* base = rt + df.idx(2 * X - 1, 2 * Y - 1, 2 * Z - 1);
      const int sy = df.nx, sz = df.nx * df.ny;
      float tz[4];
#pragma unroll
      for (int c = 0; c < 4; c++) {
        float ty[4];
#pragma unroll
        for (int bb = 0; bb < 4; bb++) {
          const TS* row = base + c * sz + bb * sy;
          ty[bb] = 0.25f * (ldv(row) + ldv(row + 3)) + 0.75f * (ldv(row + 1) + ldv(row + 2));
        }
        tz[c] = 0.25f * (ty[0] + ty[3]) + 0.75f * (ty[1] + ty[2]);
      }
      acc = 0.25f * (tz[0] + tz[3]) + 0.75f * (tz[1] + tz[2]);
    } else {
      float wx[4], wy[4], wz[4];
#pragma unroll
      for (int a = 0; a < 4; a++) {
        int cx = 2 * X - 1 + a, cy = 2 * Y - 1 + a, cz = 2 * Z - 1 + a;
        wx[a] = (cx >= 0 && cx < df.nx) ? pw1(cx, X, dc.nx) : 0.0f;
        wy[a] = (cy >= 0 && cy < df.ny) ? pw1(cy, Y, dc.ny) : 0.0f;
        wz[a] = (cz >= 0 && cz < df.nz) ? pw1(cz, Z, dc.nz) : 0.0f;
      }
#pragma unroll
      for (int c = 0; c < 4; c++) {
        if (wz[c] == 0.0f) continue;
#pragma unroll
        for (int bb = 0; bb < 4; bb++) {
          if (wy[bb] == 0.0f) continue;
#pragma unroll
          for (int a = 0; a < 4; a++) {
            if (wx[a] == 0.0f) continue;
            int i = df.idx(2 * X - 1 + a, 2 * Y - 1 + bb, 2 * Z - 1 + c);
            acc += wx[a] * wy[bb] * wz[c] * ldv(rt + i);
          }
        }
      }
    }
    acc *= 0.125f;
  }
  stv(bc + J, acc);
  stv(pc + J, 0.0f);
}

inline dim3 g3(Dims3 d) { return dim3((d.nx + 31) / 32, (d.ny + 3) / 4, (d.nz + 1) / 2); }

// Residual statistics of level 0 (mg.wgsl:122-158: the sums of r^2 and b^2
// over the fluid cells, stats slots 10 and 11) from the neighbour masks,
// for rows of a multiple of 4 cells.  Thread (tx, ty) of block (8, 16)
// takes the 4-cell chunk 8 blockIdx.x + tx of row 16 blockIdx.y + ty in
// plane blockIdx.z; phi at x0 - 1 and x0 + 4 comes from the neighbouring
// lanes of the row.  Per cell r = b - (sum of fluid neighbours - count phi)
// / h^2 with the neighbours in the reference's order, the same value as
// k_mg_resid; the thread's four cells and then the block are summed before
// one atomic per block and slot.
__global__ void __launch_bounds__(128) k_mg_resid_m(L d, float h2, const float* __restrict__ p,
                                                    const float* __restrict__ b,
                                                    const uint8_t* __restrict__ meta,
                                                    int bc_mode, float* __restrict__ stats) {
  __shared__ float sh[2 * 32];
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int x0 = (blockIdx.x * 8 + tx) * 4, y = blockIdx.y * 16 + ty, z = blockIdx.z;
  const bool act = x0 < d.nx && y < d.ny;
  const int sy = d.nx, sz = d.nx * d.ny;
  const int i0 = act ? (z * d.ny + y) * d.nx + x0 : 0;
  const float4 zero = make_float4(0.f, 0.f, 0.f, 0.f);
  const float4 P0 = act ? ld4(p + i0) : zero;
  float left = __shfl_up_sync(0xffffffffu, P0.w, 1);
  float right = __shfl_down_sync(0xffffffffu, P0.x, 1);
  float vals[2] = {0.0f, 0.0f};  // r^2, b^2
  if (act) {
    if (tx == 0 && x0 > 0) left = __ldg(p + i0 - 1);
    if (tx == 7 && x0 + 4 < d.nx) right = __ldg(p + i0 + 4);
    const float4 B = ld4(b + i0);
    const uint32_t m4 = *reinterpret_cast<const uint32_t*>(meta + i0);
    const float4 Yp = y + 1 < d.ny ? ld4(p + i0 + sy) : zero;
    const float4 Ym = y > 0 ? ld4(p + i0 - sy) : zero;
    const float4 Zp = z + 1 < d.nz ? ld4(p + i0 + sz) : zero;
    const float4 Zm = z > 0 ? ld4(p + i0 - sz) : zero;
    const float pc[6] = {left, P0.x, P0.y, P0.z, P0.w, right};
    const float yp[4] = {Yp.x, Yp.y, Yp.z, Yp.w}, ym[4] = {Ym.x, Ym.y, Ym.z, Ym.w};
    const float zp[4] = {Zp.x, Zp.y, Zp.z, Zp.w}, zm[4] = {Zm.x, Zm.y, Zm.z, Zm.w};
    const float bb[4] = {B.x, B.y, B.z, B.w};
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const uint32_t m = (m4 >> (8 * j)) & 0xFFu;
      if (m & META_SOLID) continue;
      float sum = 0.0f;
      if (m & 1u) sum += pc[j + 2];
      if (m & 2u) sum += pc[j];
      if (m & 4u) sum += yp[j];
      if (m & 8u) sum += ym[j];
      if (m & 16u) sum += zp[j];
      if (m & 32u) sum += zm[j];
      const float cnt = (float)(__popc(m & 63u) + dirichlet_faces(d, x0 + j, y, z, bc_mode));
      const float r = bb[j] - (sum - cnt * pc[j + 1]) / h2;
      vals[0] += r * r;
      vals[1] += bb[j] * bb[j];
    }
  }
  block_stats<2>(sh, vals, stats, {10, 11}, 0u);
}

}  // namespace

cudaError_t launch_mg_resid_m(Dims3 d, float h, const float* p, const float* b,
                              const uint8_t* meta, int bc_mode, float* stats, cudaStream_t st) {
  if (d.nx % 4 != 0) return cudaErrorNotSupported;
  k_mg_resid_m<<<dim3((unsigned)((d.nx / 4 + 7) / 8), (unsigned)((d.ny + 15) / 16),
                      (unsigned)d.nz),
                 dim3(8, 16), 0, st>>>(L{d.nx, d.ny, d.nz}, h * h, p, b, meta, bc_mode, stats);
  return cudaGetLastError();
}

// Planes per thread of k_mg_pass4z: 2; 4 on levels of at least
// PASS_ZT4_CELLS cells and 1 on levels below PASS_ZT1_CELLS (measured on
// the 2 cm pool: level-0 passes 0.677 ms per substep with 2 planes, 0.662
// with 4; the middle levels 0.516 ms with 2 planes, 0.495 with one plane
// on the 128 k-cell level 2 and 0.497 with one plane on level 1 as well,
// where the whole substep got slower).
constexpr int PASS_ZT = 2;
constexpr size_t PASS_ZT4_CELLS = 4u << 20;
constexpr size_t PASS_ZT1_CELLS = (size_t)1 << 18;

inline dim3 pass4z_grid(Dims3 d, int zt = PASS_ZT) {
  return dim3((unsigned)((d.nx / 4 + 7) / 8), (unsigned)((d.ny + 15) / 16),
              (unsigned)((d.nz + zt - 1) / zt));
}

// The chunked pass for a level: rows of a multiple of 4 cells take 4-cell
// chunks (k_mg_pass4z), other rows 2-cell chunks (k_mg_pass2z); zt planes
// per thread (1, 2 or 4).
template <typename TS, int MODE>
cudaError_t pass_chunked(Dims3 d, float h, TS* b, const uint8_t* meta, TS* p, int color,
                         float omega, int bc_mode, const float* b32, float* out, int zt,
                         cudaStream_t st) {
  const L l{d.nx, d.ny, d.nz};
  if (d.nx % 4 == 0) {
    const dim3 g = pass4z_grid(d, zt), blk(8, 16);
    if (zt == 4)
      return launch_pdl(k_mg_pass4z<TS, 4, MODE>, g, blk, 0, st, l, h * h, b, meta, p, color,
                        omega, bc_mode, b32, out);
    if (zt == 1)
      return launch_pdl(k_mg_pass4z<TS, 1, MODE>, g, blk, 0, st, l, h * h, b, meta, p, color,
                        omega, bc_mode, b32, out);
    return launch_pdl(k_mg_pass4z<TS, 2, MODE>, g, blk, 0, st, l, h * h, b, meta, p, color,
                      omega, bc_mode, b32, out);
  }
  const dim3 g((unsigned)(((d.nx + 1) / 2 + 15) / 16), (unsigned)((d.ny + 7) / 8),
               (unsigned)((d.nz + zt - 1) / zt)),
      blk(16, 8);
  if (d.nx % 2 == 0) {
    if (zt == 4)
      return launch_pdl(k_mg_pass2z<TS, 4, MODE, true>, g, blk, 0, st, l, h * h, b, meta, p,
                        color, omega, bc_mode, b32, out);
    if (zt == 1)
      return launch_pdl(k_mg_pass2z<TS, 1, MODE, true>, g, blk, 0, st, l, h * h, b, meta, p,
                        color, omega, bc_mode, b32, out);
    return launch_pdl(k_mg_pass2z<TS, 2, MODE, true>, g, blk, 0, st, l, h * h, b, meta, p, color,
                      omega, bc_mode, b32, out);
  }
  if (zt == 4)
    return launch_pdl(k_mg_pass2z<TS, 4, MODE, false>, g, blk, 0, st, l, h * h, b, meta, p,
                      color, omega, bc_mode, b32, out);
  if (zt == 1)
    return launch_pdl(k_mg_pass2z<TS, 1, MODE, false>, g, blk, 0, st, l, h * h, b, meta, p,
                      color, omega, bc_mode, b32, out);
  return launch_pdl(k_mg_pass2z<TS, 2, MODE, false>, g, blk, 0, st, l, h * h, b, meta, p, color,
                    omega, bc_mode, b32, out);
}

// Even rows take the chunked passes; odd rows one colour cell per thread
// (k_mg_pass), which measured faster there than 2-cell chunks of scalar
// accesses (150x365x150 with BF16 MGPCG, levels of 75 and 19 cells per
// row: 5.82 against 6.19 ms per substep).
template <typename TS>
cudaError_t pass_t(Dims3 d, float h, const TS* b, const uint8_t* meta, TS* p, int color,
                   float omega, int bc_mode, cudaStream_t st) {
  if (d.nx % 2 == 0) {
    const int zt = d.cells() >= PASS_ZT4_CELLS ? 4 : d.cells() < PASS_ZT1_CELLS ? 1 : PASS_ZT;
    return pass_chunked<TS, PASS>(d, h, const_cast<TS*>(b), meta, p, color, omega, bc_mode,
                                  nullptr, nullptr, zt, st);
  }
  dim3 grid(((d.nx + 1) / 2 + 31) / 32, (d.ny + 3) / 4, (d.nz + 1) / 2);
  return launch_pdl(k_mg_pass<TS>, grid, dim3(32, 4, 2), 0, st, L{d.nx, d.ny, d.nz}, h * h, b,
                    meta, p, color, omega, bc_mode);
}

cudaError_t launch_mg_pass_first(Dims3 d, float h, const float* r, void* bq,
                                 const uint8_t* meta, void* p, int color, float omega,
                                 int bc_mode, bool bf16, cudaStream_t st) {
  if (bf16) {
    using T = __nv_bfloat16;
    return pass_chunked<T, PASS_FIRST>(d, h, (T*)bq, meta, (T*)p, color, omega, bc_mode, r,
                                       nullptr, PASS_ZT, st);
  }
  return pass_chunked<float, PASS_FIRST>(d, h, const_cast<float*>(r), meta, (float*)p, color,
                                         omega, bc_mode, r, nullptr, PASS_ZT, st);
}

cudaError_t launch_mg_pass_last_f32(Dims3 d, float h, const void* b, const uint8_t* meta,
                                    void* p, float* out, int color, float omega, int bc_mode,
                                    cudaStream_t st) {
  using T = __nv_bfloat16;
  return pass_chunked<T, PASS_LAST_F32>(d, h, (T*)const_cast<void*>(b), meta, (T*)p, color,
                                        omega, bc_mode, nullptr, out, PASS_ZT, st);
}
template <typename TS>
cudaError_t restrict_t(Dims3 df, float h, const TS* pf, const TS* bf, const uint8_t* mf,
                       Dims3 dc, TS* bc, TS* pc, int bc_mode, cudaStream_t st) {
  auto kern = df.nx % 2 == 0 ? k_mg_restrict_m<TS, true> : k_mg_restrict_m<TS, false>;
  return launch_pdl(kern, g3(dc), dim3(32, 4, 2), 0, st, L{df.nx, df.ny, df.nz}, h * h, pf, bf,
                    mf, L{dc.nx, dc.ny, dc.nz}, bc, pc, bc_mode);
}

cudaError_t launch_mg_pass(Dims3 d, float h, const float* b, const uint8_t* meta, float* p,
                           int color, float omega, int bc_mode, cudaStream_t st) {
  return pass_t<float>(d, h, b, meta, p, color, omega, bc_mode, st);
}
cudaError_t launch_mg_pass_bf16(Dims3 d, float h, const void* b, const uint8_t* meta, void* p,
                                int color, float omega, int bc_mode, cudaStream_t st) {
  using T = __nv_bfloat16;
  return pass_t<T>(d, h, (const T*)b, meta, (T*)p, color, omega, bc_mode, st);
}
cudaError_t launch_mg_restrict_m(Dims3 df, float h, const float* pf, const float* bf,
                                 const uint8_t* mf, Dims3 dc, float* bc, float* pc, int bc_mode,
                                 cudaStream_t st) {
  return restrict_t<float>(df, h, pf, bf, mf, dc, bc, pc, bc_mode, st);
}
cudaError_t launch_mg_restrict_m_bf16(Dims3 df, float h, const void* pf, const void* bf,
                                      const uint8_t* mf, Dims3 dc, void* bc, void* pc,
                                      int bc_mode, cudaStream_t st) {
  using T = __nv_bfloat16;
  return restrict_t<T>(df, h, (const T*)pf, (const T*)bf, mf, dc, (T*)bc, (T*)pc, bc_mode, st);
}
template <typename TS>
cudaError_t restrict_sym_t(Dims3 df, float h, const TS* pf, const TS* bf, const uint8_t* mf,
                           const uint8_t* wq, TS* rt, Dims3 dc, const uint8_t* mc, TS* bc,
                           TS* pc, int bc_mode, cudaStream_t st) {
  cudaError_t e = launch_pdl(k_mg_resid_w<TS>, g3(df), dim3(32, 4, 2), 0, st,
                             L{df.nx, df.ny, df.nz}, h * h, pf, bf, mf, wq, bc_mode, rt);
  if (e != cudaSuccess) return e;
  return launch_pdl(k_mg_restrict_t<TS>, g3(dc), dim3(32, 4, 2), 0, st, L{df.nx, df.ny, df.nz},
                    (const TS*)rt, mf, L{dc.nx, dc.ny, dc.nz}, mc, bc, pc);
}

cudaError_t launch_mg_wsum(Dims3 df, const uint8_t* mf, Dims3 dc, const uint8_t* mc,
                           uint8_t* wq, cudaStream_t st) {
  return launch_pdl(k_mg_wsum, g3(df), dim3(32, 4, 2), 0, st, L{df.nx, df.ny, df.nz}, mf,
                    L{dc.nx, dc.ny, dc.nz}, mc, wq);
}
cudaError_t launch_mg_restrict_sym(Dims3 df, float h, const float* pf, const float* bf,
                                   const uint8_t* mf, const uint8_t* wq, float* rt, Dims3 dc,
                                   const uint8_t* mc, float* bc, float* pc, int bc_mode,
                                   cudaStream_t st) {
  return restrict_sym_t<float>(df, h, pf, bf, mf, wq, rt, dc, mc, bc, pc, bc_mode, st);
}
cudaError_t launch_mg_restrict_sym_bf16(Dims3 df, float h, const void* pf, const void* bf,
                                        const uint8_t* mf, const uint8_t* wq, void* rt,
                                        Dims3 dc, const uint8_t* mc, void* bc, void* pc,
                                        int bc_mode, cudaStream_t st) {
  using T = __nv_bfloat16;
  return restrict_sym_t<T>(df, h, (const T*)pf, (const T*)bf, mf, wq, (T*)rt, dc, mc, (T*)bc,
                           (T*)pc, bc_mode, st);
}

cudaError_t launch_mg_meta(Dims3 d, const uint32_t* f, uint8_t* meta, cudaStream_t st) {
  return launch_pdl(k_mg_meta, g3(d), dim3(32, 4, 2), 0, st, L{d.nx, d.ny, d.nz}, f, meta);
}

cudaError_t launch_mg_flags_down(Dims3 df, const uint32_t* ff, Dims3 dc, uint32_t* fc,
                                 cudaStream_t st) {
  return launch_pdl(k_mg_flags_down, g3(dc), dim3(32, 4, 2), 0, st, L{df.nx, df.ny, df.nz}, ff,
                    L{dc.nx, dc.ny, dc.nz}, fc);
}

template <typename TS>
cudaError_t prolong_t(Dims3 df, const TS* pc, const uint8_t* mf, TS* pf, Dims3 dc,
                      const uint8_t* mc, cudaStream_t st) {
  auto kern = df.nx % 2 == 0 ? k_mg_prolong_m<TS, true> : k_mg_prolong_m<TS, false>;
  return launch_pdl(kern, g3(dc), dim3(32, 4, 2), 0, st, L{df.nx, df.ny, df.nz}, pc, mf, pf,
                    L{dc.nx, dc.ny, dc.nz}, mc);
}

cudaError_t launch_mg_prolong_m(Dims3 df, const float* pc, const uint8_t* mf, float* pf,
                                Dims3 dc, const uint8_t* mc, cudaStream_t st) {
  return prolong_t<float>(df, pc, mf, pf, dc, mc, st);
}

cudaError_t launch_mg_prolong_m_bf16(Dims3 df, const void* pc, const uint8_t* mf, void* pf,
                                     Dims3 dc, const uint8_t* mc, cudaStream_t st) {
  using T = __nv_bfloat16;
  return prolong_t<T>(df, (const T*)pc, mf, (T*)pf, dc, mc, st);
}

}  // namespace pyro
