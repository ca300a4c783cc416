// k_conv.cu — 3x3x3 convolutions (padding 1, stride 1) as implicit GEMMs on
// the tcgen05 tensor cores, for the learned pressure warm start.
//
// One kernel, k_gemm<N, Load, Epi>, computes a 128 x N tile of
// D = A * B^T with BF16 operands staged in shared memory (two-stage
// pipeline, K in steps of 16) and the FP32 accumulator in TMEM:
//
//   forward          A[m = voxel][k = (tap, ci)] = x[voxel + tap][ci]
//                    B[n = co][k]                = W[co][tap][ci]
//   backward (data)  A[m = voxel][k = (tap, co)] = dy[voxel - tap][co]
//                    B[n = ci][k]                = W[co][tap][ci]
//   backward (weight) A[m = (tap, ci)][k = voxel] = x[voxel + tap][ci]
//                    B[n = co][k = voxel]        = dy[voxel][co]   (split over K)
//
// Activations are BF16 in planes of 8 channels, [C / 8][volume][z][y][x][8]
// (C a multiple of 8; [volume][z][y][x][C] otherwise); a tap
// outside its volume reads zero.  One thread issues the MMA, tcgen05.commit
// signals an mbarrier per stage, and every wait is bounded: a wait that runs
// out sets *err and the CTA still frees its TMEM.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <mutex>

#include "runtime.h"
#include "umma.cuh"

namespace pyro {

namespace {

using bf16 = __nv_bfloat16;
constexpr int GEMM_THREADS = 128;

struct Vol {
  int nx, ny, nz, nb;  // volume dims and count
  __device__ __forceinline__ int voxels() const { return nx * ny * nz * nb; }
};

// Voxel v shifted by tap (dx, dy, dz) within its volume, or -1.
__device__ __forceinline__ int shifted(const Vol& g, int v, int dx, int dy, int dz) {
  int x = v % g.nx;
  int r = v / g.nx;
  int y = r % g.ny;
  r /= g.ny;
  int z = r % g.nz;
  int b = r / g.nz;
  x += dx;
  y += dy;
  z += dz;
  if ((unsigned)x >= (unsigned)g.nx || (unsigned)y >= (unsigned)g.ny ||
      (unsigned)z >= (unsigned)g.nz)
    return -1;
  return ((b * g.nz + z) * g.ny + y) * g.nx + x;
}
// Activation layout: C a multiple of 8 -> C / 8 planes of [V][8 channels];
// otherwise [V][C].  Element offset of channel c of voxel v:
__device__ __forceinline__ size_t act_off(size_t v, int c, int C, size_t V) {
  return (C & 7) ? v * C + c : ((size_t)(c >> 3) * V + v) * 8 + (c & 7);
}

__device__ __forceinline__ void tap_offset(int t, int& dx, int& dy, int& dz) {
  dx = t % 3 - 1;
  dy = (t / 3) % 3 - 1;
  dz = t / 9 - 1;
}

__device__ __forceinline__ void st16(uint8_t* s, uint32_t off, uint4 v) {
  *reinterpret_cast<uint4*>(s + off) = v;
}
__device__ __forceinline__ void st_bf(uint8_t* s, uint32_t off, bf16 v) {
  *reinterpret_cast<bf16*>(s + off) = v;
}

template <int N, class Load, class Epi>
__global__ void __launch_bounds__(GEMM_THREADS) k_gemm(Load ld, Epi ep, int ksteps_total,
                                                       int ksteps_per_cta, int* err) {
  constexpr int NCOLS = N <= 32 ? 32 : (N <= 64 ? 64 : 128);
  __shared__ __align__(1024) uint8_t sA[2][128 * 32];
  __shared__ __align__(1024) uint8_t sB[2][N * 32];
  __shared__ __align__(8) uint64_t mbar[2];
  __shared__ uint32_t tslot;
  const int m0 = blockIdx.x * 128;
  const int k0 = blockIdx.y * ksteps_per_cta;
  const int k1 = min(k0 + ksteps_per_cta, ksteps_total);
  const int nks = max(k1 - k0, 0);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    umma::mbar_init(&mbar[0], 1);
    umma::mbar_init(&mbar[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    umma::tmem_alloc(&tslot, NCOLS);
    umma::tmem_relinquish();
  }
  umma::fence_before();
  __syncthreads();
  umma::fence_after();
  const uint32_t tbase = tslot;
  constexpr uint32_t IDESC = umma::idesc_bf16(128, N);
  bool ok = true;
  for (int i = 0; i < nks; i++) {
    const int s = i & 1;
    if (i >= 2 && !umma::mbar_wait_bounded(&mbar[s], ((i - 2) >> 1) & 1)) ok = false;
    ld(sA[s], sB[s], m0, k0 + i);
    umma::fence_proxy_async();
    __syncthreads();
    if (threadIdx.x == 0) {
      umma::fence_after();
      umma::mma_bf16(tbase, umma::smem_desc(sA[s], 128), umma::smem_desc(sB[s], N), IDESC,
                     i > 0 ? 1u : 0u);
      umma::mma_commit(&mbar[s]);
    }
  }
  if (nks > 0 && !umma::mbar_wait_bounded(&mbar[(nks - 1) & 1], ((nks - 1) >> 1) & 1))
    ok = false;
  umma::fence_after();
  const bool all_ok = __syncthreads_and(ok) != 0;
  if (all_ok && nks > 0) {
#pragma unroll
    for (int col = 0; col < N; col += 16) {
      float v[16];
      umma::tmem_ld16(tbase + ((uint32_t)(warp * 32) << 16) + (uint32_t)col, v);
      ep(m0 + warp * 32 + lane, col, v);
    }
  }
  if (!all_ok && threadIdx.x == 0) atomicExch(err, 1);
  umma::fence_before();
  __syncthreads();
  if (warp == 0) umma::tmem_dealloc(tbase, NCOLS);
}

// ---------------------------------------------------------------- loaders
// A = shifted activations (voxel rows, K = (tap, channel)); B = weight rows.
// `flip` negates the tap (backward data); `wt` selects the transposed
// weight gather for backward data: B[n = ci][k = (tap, co)] = W[co][tap][ci].
struct ConvLoad {
  const bf16* x;      // [V][C]
  const bf16* w;      // [Cw_out][27][Cw_in]
  Vol g;
  int C;              // channels of x (K = 27 C)
  int Nrows;          // rows of B that exist (co, or ci for backward data)
  int cw_in, cw_out;  // weight dims
  int flip, wt;
  __device__ void operator()(uint8_t* sA, uint8_t* sB, int m0, int ks) const {
    const int t0 = threadIdx.x;
    const int V = g.voxels();
    const int K = 27 * C;
    // A: row r = voxel m0 + r
    {
      int r = t0;
      int v = m0 + r;
      if ((C & 15) == 0) {
        int t = ks / (C >> 4), cc = ks % (C >> 4);
        int dx, dy, dz;
        tap_offset(t, dx, dy, dz);
        if (flip) { dx = -dx; dy = -dy; dz = -dz; }
        uint4 a0 = make_uint4(0, 0, 0, 0), a1 = a0;
        if (v < V) {
          int vs = shifted(g, v, dx, dy, dz);
          if (vs >= 0) {
            const uint4* p = reinterpret_cast<const uint4*>(x + act_off(vs, cc * 16, C, V));
            a0 = __ldg(p);
            a1 = __ldg(p + V);  // the next 8-channel plane
          }
        }
        st16(sA, umma::core_offset(r, 0, 128), a0);
        st16(sA, umma::core_offset(r, 8, 128), a1);
      } else {
        for (int e = 0; e < 16; e++) {
          int k = ks * 16 + e;
          bf16 val = __float2bfloat16(0.0f);
          if (v < V && k < K) {
            int t = k / C, ci = k % C;
            int dx, dy, dz;
            tap_offset(t, dx, dy, dz);
            if (flip) { dx = -dx; dy = -dy; dz = -dz; }
            int vs = shifted(g, v, dx, dy, dz);
            if (vs >= 0) val = x[act_off(vs, ci, C, V)];
          }
          st_bf(sA, umma::core_offset(r, e, 128), val);
        }
      }
    }
    // B: row n (co for forward, ci for backward data)
    if (t0 < Nrows_pad()) {
      int n = t0;
      for (int e = 0; e < 16; e++) {
        int k = ks * 16 + e;
        bf16 val = __float2bfloat16(0.0f);
        if (n < Nrows && k < K) {
          if (!wt) {
            val = w[(size_t)n * K + k];  // W[co][tap][ci], K index tap * C + ci
          } else {
            int t = k / C, co = k % C;   // K index tap * Cout + co
            val = w[((size_t)co * 27 + t) * cw_in + n];
          }
        }
        st_bf(sB, umma::core_offset(n, e, npad), val);
      }
    }
  }
  int npad;
  __device__ __forceinline__ int Nrows_pad() const { return npad; }
};

// Weight gradient: A[m = (tap, ci)][k = voxel] = x[voxel + tap][ci],
// B[n = co][k = voxel] = dy[voxel][co].
struct WgradLoad {
  const bf16* x;   // [V][Cin]
  const bf16* dy;  // [V][Cout]
  Vol g;
  int Cin, Cout, npad;
  __device__ void operator()(uint8_t* sA, uint8_t* sB, int m0, int ks) const {
    const int V = g.voxels();
    const int M = 27 * Cin;
    {
      int r = threadIdx.x;
      int m = m0 + r;
      int t = m / Cin, ci = m % Cin;
      int dx, dy_, dz;
      tap_offset(t < 27 ? t : 0, dx, dy_, dz);
      for (int e = 0; e < 16; e++) {
        int v = ks * 16 + e;
        bf16 val = __float2bfloat16(0.0f);
        if (m < M && v < V) {
          int vs = shifted(g, v, dx, dy_, dz);
          if (vs >= 0) val = x[act_off(vs, ci, Cin, V)];
        }
        st_bf(sA, umma::core_offset(r, e, 128), val);
      }
    }
    if ((int)threadIdx.x < npad) {
      int n = threadIdx.x;
      for (int e = 0; e < 16; e++) {
        int v = ks * 16 + e;
        bf16 val = __float2bfloat16(0.0f);
        if (n < Cout && v < V) val = dy[act_off(v, n, Cout, V)];
        st_bf(sB, umma::core_offset(n, e, npad), val);
      }
    }
  }
};

// -------------------------------------------------------------- epilogues
// Forward / backward data: row = voxel.  out_bf16 [V][Nout] with optional
// bias and ReLU, or out_f32 [V][Nout]; `mask` (BF16 activations of the layer
// input, [V][Nout]) zeroes the gradient where the input was <= 0 (ReLU).
struct ConvEpi {
  bf16* out_bf16;
  float* out_f32;
  const float* bias;
  const bf16* mask;
  int V, Nout, relu;
  __device__ void operator()(int m, int col, const float (&v)[16]) const {
    if (m < 0 || m >= V) return;
    if (out_bf16 && (Nout & 15) == 0) {
      // 16 channels of one row: 32 contiguous bytes, two 16-byte stores
      float a[16];
#pragma unroll
      for (int j = 0; j < 16; j += 4) {
        float4 bb = bias ? __ldg(reinterpret_cast<const float4*>(bias + col + j))
                         : make_float4(0.f, 0.f, 0.f, 0.f);
        a[j] = v[j] + bb.x;
        a[j + 1] = v[j + 1] + bb.y;
        a[j + 2] = v[j + 2] + bb.z;
        a[j + 3] = v[j + 3] + bb.w;
      }
      if (!bias) {
#pragma unroll
        for (int j = 0; j < 16; j++) a[j] = v[j];
      }
      if (relu) {
#pragma unroll
        for (int j = 0; j < 16; j++) a[j] = fmaxf(a[j], 0.0f);
      }
      if (mask) {
        const uint4* mp = reinterpret_cast<const uint4*>(mask + act_off(m, col, Nout, V));
        uint4 mk[2] = {__ldg(mp), __ldg(mp + V)};
        const bf16* mb = reinterpret_cast<const bf16*>(mk);
#pragma unroll
        for (int j = 0; j < 16; j++)
          if (!(__bfloat162float(mb[j]) > 0.0f)) a[j] = 0.0f;
      }
      uint4 o[2];
      __nv_bfloat162* ob = reinterpret_cast<__nv_bfloat162*>(o);
#pragma unroll
      for (int j = 0; j < 8; j++) ob[j] = __floats2bfloat162_rn(a[2 * j], a[2 * j + 1]);
      uint4* op = reinterpret_cast<uint4*>(out_bf16 + act_off(m, col, Nout, V));
      op[0] = o[0];
      op[V] = o[1];  // the next 8-channel plane
      return;
    }
#pragma unroll
    for (int j = 0; j < 16; j++) {
      int n = col + j;
      if (n >= Nout) break;
      float a = v[j];
      if (bias) a += bias[n];
      if (relu) a = fmaxf(a, 0.0f);
      if (mask && !(__bfloat162float(mask[act_off(m, n, Nout, V)]) > 0.0f)) a = 0.0f;
      if (out_f32) out_f32[(size_t)m * Nout + n] = a;
      else out_bf16[act_off(m, n, Nout, V)] = __float2bfloat16(a);
    }
  }
};

// Weight gradient: row m = (tap, ci), column n = co; FP32 atomics into
// dw[co][tap][ci] (split-K partial sums).
struct WgradEpi {
  float* dw;
  int M, Cout;
  __device__ void operator()(int m, int col, const float (&v)[16]) const {
    if (m >= M) return;
#pragma unroll
    for (int j = 0; j < 16; j++) {
      int n = col + j;
      if (n >= Cout) break;
      atomicAdd(dw + (size_t)n * M + m, v[j]);
    }
  }
};

template <int N, class Load, class Epi>
cudaError_t gemm_launch(dim3 grid, const Load& ld, const Epi& ep, int ksteps_total,
                        int ksteps_per_cta, int* err, cudaStream_t st) {
  k_gemm<N, Load, Epi><<<grid, GEMM_THREADS, 0, st>>>(ld, ep, ksteps_total, ksteps_per_cta, err);
  return cudaGetLastError();
}

template <class Load, class Epi>
cudaError_t gemm_dispatch(int npad, dim3 grid, const Load& ld, const Epi& ep, int kt, int kpc,
                          int* err, cudaStream_t st) {
  switch (npad) {
    case 16: return gemm_launch<16>(grid, ld, ep, kt, kpc, err, st);
    case 32: return gemm_launch<32>(grid, ld, ep, kt, kpc, err, st);
    case 48: return gemm_launch<48>(grid, ld, ep, kt, kpc, err, st);
    case 64: return gemm_launch<64>(grid, ld, ep, kt, kpc, err, st);
    case 96: return gemm_launch<96>(grid, ld, ep, kt, kpc, err, st);
    case 128: return gemm_launch<128>(grid, ld, ep, kt, kpc, err, st);
    default: return cudaErrorInvalidValue;
  }
}


// ------------------------------------------------------------ TMA path
// Convolution with TMA-staged operands, for input channel counts that are
// multiples of 16, computed transposed: D[co][voxel] = W[co][k] X[voxel][k]^T
// with the output channels as the MMA's M (128 rows; rows past the channel
// count are computed and never stored) and NT = 256 (or 128) voxels of a
// tile as its N.  A tcgen05.mma of K = 16 costs the same issue time for any
// N up to 256, so a wide voxel tile does the work of several narrow ones.
//
// A tile is BX x BY voxels of one z-plane (BX * BY = NT).  For every group
// of 16 input channels a tile needs, loaded by 4-D TMA boxes with zero fill
// outside the volume, three copies of the input patch shifted by
// dx = -1, 0, +1, each BX x (BY + 2) x 3 voxels (y and z with their halo) as
// two 8-channel chunks, and the weight slice w_tap[27][npad][16 channels].
// Voxel row r = x + BX y of tap (dx, dy, dz) then reads patch row
// r + BX (dy + 1) + BX (BY + 2) (dz + 1) of copy dx, so each of the 27 taps
// is one MMA whose B descriptor starts at that row: no gather, and every
// input element is fetched three times per tile instead of 27.  The A
// descriptor of tap t starts at weight row t * npad and reads 128 rows; the
// rows past npad belong to the next taps (or to a slack area) and only feed
// the D rows that are never stored.
//
// The kernel is persistent and warp-specialised.  CTA c takes tiles c,
// c + grid, c + 2 grid, ...; warp 0 streams the (tile, channel group)
// operand stages through a ring of S shared-memory stages, warp 1 issues
// the MMAs into one of two TMEM accumulators, and warps 2-5 drain the other
// accumulator (the epilogue; warp w reads TMEM lanes 32 (w % 4) ..,
// i.e. output channels 32 (w % 4) ..) while the next tile accumulates.  When
// the whole weight tensor fits beside two stages it is loaded once and
// stays resident.  Every wait is bounded; a wait that runs out stops the
// CTA's roles (shared abort flag), sets *err, lets the copies in flight land
// and frees the TMEM.
struct TmaGeom {
  int nx, ny, nz, nb;
  int BX, BY, tiles_x, tiles_y, ntiles;
  int groups, stages, resident_b, npad;
  uint32_t box_a, box_b, stage_a, stage_bytes, b_bytes, stage_off;
};

constexpr int CONV_THREADS = 192;
constexpr int CONV_MAX_STAGES = 8;
// Bytes the 128-row weight operand of the last tap reads past its rows:
// (128 - npad) rows of 16 bytes, rounded up to 1 KB.
__host__ __device__ __forceinline__ uint32_t conv_slack(int npad) {
  return ((uint32_t)(128 - npad) * 16u + 1023u) & ~1023u;
}
// epilogue transpose buffer: 32 voxels x (npad + 8) BF16 channels
__host__ __device__ __forceinline__ uint32_t conv_epi_bytes(int npad) {
  return 32u * (uint32_t)(npad + 8) * 2u;
}

// Named barrier 1 over the 128 epilogue threads; the _or form also returns
// whether any of them passed true.
__device__ __forceinline__ void epi_bar() { asm volatile("bar.sync 1, 128;" ::: "memory"); }
__device__ __forceinline__ bool epi_bar_or(bool p) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred pi, po;\n\t"
      "setp.ne.u32 pi, %1, 0;\n\t"
      "barrier.red.or.pred po, 1, 128, pi;\n\t"
      "selp.u32 %0, 1, 0, po;\n\t}"
      : "=r"(r)
      : "r"((uint32_t)p)
      : "memory");
  return r != 0;
}

__device__ __forceinline__ void mbar_arrive(uint64_t* mbar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(umma::smem_u32(mbar))
               : "memory");
}

template <int NT, int LOG2BX>
__global__ void __launch_bounds__(CONV_THREADS, 1)
    k_conv_tma(const __grid_constant__ CUtensorMap ta, const __grid_constant__ CUtensorMap tb,
               TmaGeom g, ConvEpi ep, int* err) {
  constexpr uint32_t IDESC = umma::idesc_bf16(128, NT);
  constexpr int BX = 1 << LOG2BX;
  extern __shared__ uint8_t dsm[];
  __shared__ __align__(8) uint64_t full[CONV_MAX_STAGES], empty[CONV_MAX_STAGES], accf[2],
      acce[2], bfull, done;
  __shared__ uint32_t tslot;
  __shared__ volatile int abort_flag;
  uint8_t* base = dsm + ((1024u - (umma::smem_u32(dsm) & 1023u)) & 1023u);
  uint8_t* sb_res = base;
  uint8_t* stages = base + g.stage_off;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int S = g.stages, G = g.groups;
  if (threadIdx.x == 0) {
    for (int s = 0; s < S; s++) {
      umma::mbar_init(&full[s], 1);
      umma::mbar_init(&empty[s], 1);
    }
    for (int a = 0; a < 2; a++) {
      umma::mbar_init(&accf[a], 1);
      umma::mbar_init(&acce[a], 4);
    }
    umma::mbar_init(&bfull, 1);
    umma::mbar_init(&done, 1);
    abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    umma::tmem_alloc(&tslot, 2 * NT);
    umma::tmem_relinquish();
  }
  umma::fence_before();
  __syncthreads();
  umma::fence_after();
  const uint32_t tbase = tslot;
  const int my_tiles =
      (int)blockIdx.x < g.ntiles ? (g.ntiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
  bool timed_out = false;
  if (warp == 0) {
    if (lane == 0) {
      // ---- producer
      if (g.resident_b && my_tiles > 0) {
        umma::mbar_expect_tx(&bfull, g.b_bytes);
        for (int grp = 0; grp < G; grp++)
          for (int j = 0; j < 2; j++)
            umma::tma_load_3d(sb_res + (size_t)(grp * 2 + j) * g.box_b, &tb, grp * 16 + j * 8, 0,
                              0, &bfull);
      }
      const int items = my_tiles * G;
      int issued = 0;
      for (int i = 0; i < items; i++) {
        if (abort_flag) break;
        const int s = i % S;
        if (i >= S && !umma::mbar_wait_bounded(&empty[s], ((i / S) - 1) & 1)) {
          timed_out = true;
          break;
        }
        const int jt = i / G, grp = i - jt * G;
        int t = (int)blockIdx.x + jt * (int)gridDim.x;
        const int tx = t % g.tiles_x;
        t /= g.tiles_x;
        const int ty = t % g.tiles_y;
        t /= g.tiles_y;
        const int z = t % g.nz, b = t / g.nz;
        uint8_t* sa = stages + (size_t)s * g.stage_bytes;
        umma::mbar_expect_tx(&full[s], g.stage_a + (g.resident_b ? 0u : 2u * g.box_b));
        for (int d = 0; d < 3; d++)
          for (int j = 0; j < 2; j++)
            umma::tma_load_4d(sa + (d * 2 + j) * g.box_a, &ta, (tx * g.BX + d - 1) * 8,
                              ty * g.BY - 1, z - 1, (grp * 2 + j) * g.nb + b, &full[s]);
        if (!g.resident_b)
          for (int j = 0; j < 2; j++)
            umma::tma_load_3d(sa + g.stage_a + j * g.box_b, &tb, grp * 16 + j * 8, 0, 0,
                              &full[s]);
        issued = i + 1;
      }
      if (timed_out) abort_flag = 1;
      // every issued copy lands before the CTA may exit
      for (int q = issued > S ? issued - S : 0; q < issued; q++)
        if (!umma::mbar_wait_bounded(&full[q % S], (q / S) & 1)) timed_out = true;
      if (g.resident_b && my_tiles > 0 && !umma::mbar_wait_bounded(&bfull, 0)) timed_out = true;
    }
  } else if (warp == 1) {
    if (lane == 0) {
      // ---- MMA issuer
      bool ok = true;
      if (g.resident_b && my_tiles > 0 && !umma::mbar_wait_bounded(&bfull, 0)) ok = false;
      const int items = my_tiles * G;
      const uint32_t wrow = (uint32_t)g.npad * 16u;  // bytes per tap of a weight half
      for (int i = 0; i < items && ok; i++) {
        if (abort_flag) break;
        const int s = i % S;
        const int jt = i / G, grp = i - jt * G;
        const int a = jt & 1;
        if (grp == 0 && jt >= 2 && !umma::mbar_wait_bounded(&acce[a], ((jt >> 1) - 1) & 1)) {
          ok = false;
          break;
        }
        if (!umma::mbar_wait_bounded(&full[s], (i / S) & 1)) {
          ok = false;
          break;
        }
        umma::fence_after();
        uint8_t* sa = stages + (size_t)s * g.stage_bytes;
        const uint8_t* sw = g.resident_b ? sb_res + (size_t)grp * 2 * g.box_b : sa + g.stage_a;
        const uint32_t dt = tbase + (uint32_t)(a * NT);
#pragma unroll 1
        for (int tap = 0; tap < 27; tap++) {
          const int dx = tap % 3, dy = (tap / 3) % 3, dz = tap / 9;
          const uint32_t row = (uint32_t)(dy * g.BX + dz * g.BX * (g.BY + 2));
          const uint64_t dw = umma::smem_desc_lbo(sw + tap * wrow, g.box_b);
          const uint64_t dv = umma::smem_desc_lbo(sa + dx * 2 * g.box_a + row * 16, g.box_a);
          umma::mma_bf16(dt, dw, dv, IDESC, (grp > 0 || tap > 0) ? 1u : 0u);
        }
        umma::mma_commit(&empty[s]);
        if (grp == G - 1) umma::mma_commit(&accf[a]);
      }
      if (!ok) {
        timed_out = true;
        abort_flag = 1;
      }
      // every MMA issued has finished before the TMEM is freed
      umma::mma_commit(&done);
      if (!umma::mbar_wait_bounded(&done, 0)) timed_out = true;
    }
    __syncwarp();
  } else {
    // ---- epilogue (warps 2-5, 128 threads).  Warp w reads TMEM lanes
    // 32 (w % 4) .. + 31, i.e. output channels co = 32 (w % 4) + lane, 32
    // voxel columns at a time.  BF16 outputs in 8-channel planes go through
    // a shared-memory transpose [voxel][channel] so that the global stores
    // are 16-byte rows of one plane; other outputs are stored per lane.
    const int q = warp & 3;
    const int et = threadIdx.x - 64;  // 0..127
    const int co = q * 32 + lane;
    const bool active = q * 32 < ep.Nout;
    const bool own = co < ep.Nout;
    const float bias = (ep.bias && own) ? ep.bias[co] : 0.0f;
    const bool planes = !ep.out_f32 && !(ep.Nout & 7);
    const int cs = g.npad + 8;  // channel stride of a transpose row (bf16)
    bf16* tr = reinterpret_cast<bf16*>(stages + (size_t)S * g.stage_bytes + conv_slack(g.npad));
    const int nch8 = ep.Nout >> 3;
    for (int jt = 0; jt < my_tiles; jt++) {
      const int a = jt & 1;
      const bool okw = __all_sync(0xffffffffu, umma::mbar_wait_bounded(&accf[a], (jt >> 1) & 1));
      if (!okw) timed_out = true;
      // the four epilogue warps leave the loop together
      if (epi_bar_or(!okw || abort_flag != 0)) {
        abort_flag = 1;
        break;
      }
      umma::fence_after();
      int t = (int)blockIdx.x + jt * (int)gridDim.x;
      const int tx = t % g.tiles_x;
      t /= g.tiles_x;
      const int ty = t % g.tiles_y;
      t /= g.tiles_y;
      const int z = t % g.nz, b = t / g.nz;
      const int x0 = tx * BX, y0 = ty * g.BY;
      const size_t row0 = (((size_t)b * g.nz + z) * g.ny + y0) * g.nx + x0;
#pragma unroll 1
      for (int c0 = 0; c0 < NT; c0 += 32) {
        float v[32];
        if (active)
          umma::tmem_ld32(tbase + (uint32_t)(a * NT + c0) + ((uint32_t)(q * 32) << 16), v);
        if (planes) {
          if (active && own) {
#pragma unroll
            for (int j = 0; j < 32; j++) {
              float val = v[j] + bias;
              if (ep.relu) val = fmaxf(val, 0.0f);
              tr[j * cs + co] = __float2bfloat16_rn(val);
            }
          }
          epi_bar();
          for (int it = et; it < 32 * nch8; it += 128) {
            const int p = it >> 5, j = it & 31;
            const int r = c0 + j;
            const int lx = r & (BX - 1), ly = r >> LOG2BX;
            if (x0 + lx < g.nx && y0 + ly < g.ny) {
              const size_t vox = row0 + (size_t)ly * g.nx + lx;
              uint4 u = *reinterpret_cast<const uint4*>(tr + j * cs + p * 8);
              if (ep.mask) {
                const uint4 m = __ldg(reinterpret_cast<const uint4*>(
                    ep.mask + ((size_t)p * ep.V + vox) * 8));
                const uint32_t* mw = reinterpret_cast<const uint32_t*>(&m);
                uint32_t* uw = reinterpret_cast<uint32_t*>(&u);
#pragma unroll
                for (int k = 0; k < 4; k++) {
                  // keep a BF16 half only where the mask half is > 0
                  const float lo = __uint_as_float(mw[k] << 16), hi = __uint_as_float(mw[k] & 0xFFFF0000u);
                  uw[k] &= (lo > 0.0f ? 0x0000FFFFu : 0u) | (hi > 0.0f ? 0xFFFF0000u : 0u);
                }
              }
              *reinterpret_cast<uint4*>(ep.out_bf16 + ((size_t)p * ep.V + vox) * 8) = u;
            }
          }
          epi_bar();
        } else if (active) {
#pragma unroll
          for (int j = 0; j < 32; j++) {
            const int r = c0 + j;
            const int lx = r & (BX - 1), ly = r >> LOG2BX;
            if (!own || x0 + lx >= g.nx || y0 + ly >= g.ny) continue;
            const size_t vox = row0 + (size_t)ly * g.nx + lx;
            float val = v[j] + bias;
            if (ep.relu) val = fmaxf(val, 0.0f);
            if (ep.mask && !(__bfloat162float(ep.mask[act_off(vox, co, ep.Nout, ep.V)]) > 0.0f))
              val = 0.0f;
            if (ep.out_f32) ep.out_f32[vox * ep.Nout + co] = val;
            else ep.out_bf16[act_off(vox, co, ep.Nout, ep.V)] = __float2bfloat16_rn(val);
          }
        }
      }
      umma::fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&acce[a]);
    }
  }
  if (timed_out) atomicExch(err, 1);
  umma::fence_before();
  __syncthreads();
  if (warp == 1) umma::tmem_dealloc(tbase, 2 * NT);
}

// --------------------------------------------------------- direct (CUDA cores)
// Layers too narrow for the tensor cores to pay: 2 -> 16 channels (the
// network's input layer, K = 54) and 16 -> 1 (its output layer, N = 1).
// A thread computes DV consecutive voxels of an x-row.  For every (dz, dy)
// input row it loads the DV + 2 voxels x0-1 .. x0+DV once (zero outside
// the volume), in chunks of CC input channels, and the three dx taps of
// all DV outputs read them from registers; every weight read from shared
// memory (FP32, [tap][ci][co]) feeds DV fused multiply-adds.  FP32
// accumulation.
template <int CIN, int COUT>
struct DirectShape {
  static constexpr int DV = 4;                  // voxels per thread
  static constexpr int CC = CIN == 2 ? 2 : 8;   // input channels per chunk
};

template <int CIN, int COUT>
__global__ void __launch_bounds__(256, 2) k_conv_direct(const bf16* __restrict__ x, Vol g,
                                                     const bf16* __restrict__ w,
                                                     const float* __restrict__ bias, int relu,
                                                     bf16* __restrict__ y_bf16,
                                                     float* __restrict__ y_f32) {
  static_assert(CIN == 2 || CIN % 8 == 0, "input rows are loaded as 4- or 16-byte chunks");
  constexpr int DV = DirectShape<CIN, COUT>::DV, CC = DirectShape<CIN, COUT>::CC;
  __shared__ __align__(16) float ws[27 * CIN * COUT];
  for (int i = threadIdx.x; i < 27 * CIN * COUT; i += blockDim.x) {
    const int co = i / (27 * CIN), t = (i / CIN) % 27, ci = i % CIN;  // w[co][t][ci]
    ws[(t * CIN + ci) * COUT + co] = __bfloat162float(w[i]);
  }
  __syncthreads();
  const long V = (long)g.nx * g.ny * g.nz * g.nb;
  const int cpr = (g.nx + DV - 1) / DV;  // chunks per x-row
  const long nchunks = (long)cpr * g.ny * g.nz * g.nb;
  const long c = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nchunks) return;
  const long row = c / cpr;  // (b, z, y) row index
  const int x0 = (int)(c - row * cpr) * DV;
  const int yy = (int)(row % g.ny);
  const int zz = (int)((row / g.ny) % g.nz);
  const long v0 = row * g.nx + x0;
  float acc[DV][COUT];
#pragma unroll
  for (int i = 0; i < DV; i++)
#pragma unroll
    for (int co = 0; co < COUT; co++) acc[i][co] = bias ? bias[co] : 0.0f;
  const long sy = g.nx, sz = (long)g.nx * g.ny;
#pragma unroll 1
  for (int dz = -1; dz <= 1; dz++) {
    if ((unsigned)(zz + dz) >= (unsigned)g.nz) continue;
#pragma unroll 1
    for (int dy = -1; dy <= 1; dy++) {
      if ((unsigned)(yy + dy) >= (unsigned)g.ny) continue;
      const long vr = v0 + sy * dy + sz * dz;  // voxel x0 of the input row
#pragma unroll
      for (int c0 = 0; c0 < CIN; c0 += CC) {
        float xin[DV + 2][CC];
#pragma unroll
        for (int i = 0; i < DV + 2; i++) {
          const int xs = x0 - 1 + i;
          const bool in = (unsigned)xs < (unsigned)g.nx;
          const long vs = vr - 1 + i;
          if constexpr (CIN == 2) {
            float2 f = make_float2(0.0f, 0.0f);
            if (in) f = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(x + vs * 2));
            xin[i][0] = f.x;
            xin[i][1] = f.y;
          } else {
            uint4 u = make_uint4(0, 0, 0, 0);
            if (in) u = __ldg(reinterpret_cast<const uint4*>(x + act_off(vs, c0, CIN, V)));
            const __nv_bfloat162* h = reinterpret_cast<const __nv_bfloat162*>(&u);
#pragma unroll
            for (int j = 0; j < 4; j++) {
              const float2 f = __bfloat1622float2(h[j]);
              xin[i][2 * j] = f.x;
              xin[i][2 * j + 1] = f.y;
            }
          }
        }
#pragma unroll
        for (int dx = 0; dx < 3; dx++) {
          const float* wt = ws + ((dx + 3 * (dy + 1) + 9 * (dz + 1)) * CIN + c0) * COUT;
#pragma unroll
          for (int ci = 0; ci < CC; ci++)
#pragma unroll
            for (int co = 0; co < COUT; co++) {
              const float wv = wt[ci * COUT + co];
#pragma unroll
              for (int i = 0; i < DV; i++)
                acc[i][co] = __fmaf_rn(xin[i + dx][ci], wv, acc[i][co]);
            }
        }
      }
    }
  }
#pragma unroll
  for (int i = 0; i < DV; i++) {
    if (x0 + i >= g.nx) break;
    const long v = v0 + i;
    if (relu) {
#pragma unroll
      for (int co = 0; co < COUT; co++) acc[i][co] = fmaxf(acc[i][co], 0.0f);
    }
    if (y_f32) {
#pragma unroll
      for (int co = 0; co < COUT; co++) y_f32[v * COUT + co] = acc[i][co];
    } else if constexpr (COUT % 8 == 0) {
#pragma unroll
      for (int c8 = 0; c8 < COUT; c8 += 8) {
        uint4 o;
        __nv_bfloat162* ob = reinterpret_cast<__nv_bfloat162*>(&o);
#pragma unroll
        for (int j = 0; j < 4; j++)
          ob[j] = __floats2bfloat162_rn(acc[i][c8 + 2 * j], acc[i][c8 + 2 * j + 1]);
        *reinterpret_cast<uint4*>(y_bf16 + act_off(v, c8, COUT, V)) = o;
      }
    } else {
#pragma unroll
      for (int co = 0; co < COUT; co++)
        y_bf16[act_off(v, co, COUT, V)] = __float2bfloat16_rn(acc[i][co]);
    }
  }
}

__global__ void k_wprep(const bf16* __restrict__ w, int Cout, int Cin, int backward,
                        bf16* __restrict__ out) {
  const int n = Cout * 27 * Cin;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int co = i / (27 * Cin), t = (i / Cin) % 27, ci = i % Cin;
    if (!backward)
      out[((size_t)t * Cout + co) * Cin + ci] = w[i];
    else
      out[((size_t)(26 - t) * Cin + ci) * Cout + co] = w[i];
  }
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}

// Tile width in x for a tile of nt voxels: a TMA box row is 8 BX elements,
// at most 256, so BX <= 32.
int pick_bx(int nx, int nt) {
  const int order256[3] = {16, 32, 8}, order128[3] = {16, 8, 32};
  const int* o = nt == 256 ? order256 : order128;
  for (int i = 0; i < 3; i++)
    if (nx % o[i] == 0) return o[i];
  return nx < 16 ? 8 : 16;
}

template <int NT, int LOG2BX>
cudaError_t tma_launch(const CUtensorMap& ta, const CUtensorMap& tb, const TmaGeom& g,
                       const ConvEpi& ep, int* err, cudaStream_t st) {
  const size_t smem = (size_t)g.stage_off + (size_t)g.stages * g.stage_bytes +
                      conv_slack(g.npad) + conv_epi_bytes(g.npad) + 1024;
  auto kern = k_conv_tma<NT, LOG2BX>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e != cudaSuccess) return e;
  int dev = 0, nsm = 148, occ = 1;
  if (cudaGetDevice(&dev) == cudaSuccess)
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, CONV_THREADS, smem) !=
          cudaSuccess ||
      occ < 1)
    occ = 1;
  // the TMEM of 2 NT columns per CTA bounds the CTAs per SM as well
  occ = std::min(occ, 512 / (2 * NT));
  const unsigned grid = (unsigned)std::min<long>((long)g.ntiles, (long)nsm * occ);
  kern<<<grid, CONV_THREADS, smem, st>>>(ta, tb, g, ep, err);
  return cudaGetLastError();
}

template <int NT>
cudaError_t tma_launch_bx(const CUtensorMap& ta, const CUtensorMap& tb, const TmaGeom& g,
                          const ConvEpi& ep, int* err, cudaStream_t st) {
  switch (g.BX) {
    case 8: return tma_launch<NT, 3>(ta, tb, g, ep, err, st);
    case 16: return tma_launch<NT, 4>(ta, tb, g, ep, err, st);
    case 32: return tma_launch<NT, 5>(ta, tb, g, ep, err, st);
    default: return cudaErrorInvalidValue;
  }
}

inline int pad16(int n) { return (n + 15) / 16 * 16; }

}  // namespace

// y = conv(x, W) (+ bias, ReLU), or its transpose for backward data.
cudaError_t conv3_forward(const bf16* x, int C, int nx, int ny, int nz, int nb, const bf16* w,
                          int Cout, const float* bias, int relu, bf16* y_bf16, float* y_f32,
                          int* err, cudaStream_t st) {
  Vol g{nx, ny, nz, nb};
  int V = nx * ny * nz * nb;
  int npad = pad16(Cout);
  int ksteps = (27 * C + 15) / 16;
  ConvLoad ld{x, w, g, C, Cout, C, Cout, 0, 0, npad};
  ConvEpi ep{y_bf16, y_f32, bias, nullptr, V, Cout, relu};
  dim3 grid((V + 127) / 128, 1, 1);
  return gemm_dispatch(npad, grid, ld, ep, ksteps, ksteps, err, st);
}

// dx = conv^T(dy, W), masked by (act > 0) when act is given.
cudaError_t conv3_backward_data(const bf16* dy, int Cout, int nx, int ny, int nz, int nb,
                                const bf16* w, int Cin, const bf16* act, bf16* dx_bf16,
                                float* dx_f32, int* err, cudaStream_t st) {
  Vol g{nx, ny, nz, nb};
  int V = nx * ny * nz * nb;
  int npad = pad16(Cin);
  int ksteps = (27 * Cout + 15) / 16;
  ConvLoad ld{dy, w, g, Cout, Cin, Cin, Cout, 1, 1, npad};
  ConvEpi ep{dx_bf16, dx_f32, nullptr, act, V, Cin, 0};
  dim3 grid((V + 127) / 128, 1, 1);
  return gemm_dispatch(npad, grid, ld, ep, ksteps, ksteps, err, st);
}

// dw[co][tap][ci] += sum_voxels dy[v][co] x[v + tap][ci]  (dw FP32, zeroed
// by the caller).
cudaError_t conv3_backward_weight(const bf16* x, int Cin, const bf16* dy, int Cout, int nx,
                                  int ny, int nz, int nb, float* dw, int* err, cudaStream_t st) {
  Vol g{nx, ny, nz, nb};
  int V = nx * ny * nz * nb;
  int M = 27 * Cin;
  int npad = pad16(Cout);
  int ksteps = (V + 15) / 16;
  int mt = (M + 127) / 128;
  // split K so that the grid covers the GPU a few times over
  int splits = std::max(1, std::min(ksteps, (148 * 8) / std::max(mt, 1)));
  int kpc = (ksteps + splits - 1) / splits;
  splits = (ksteps + kpc - 1) / kpc;
  WgradLoad ld{x, dy, g, Cin, Cout, npad};
  WgradEpi ep{dw, M, Cout};
  dim3 grid(mt, splits, 1);
  return gemm_dispatch(npad, grid, ld, ep, ksteps, kpc, err, st);
}


// Direct convolution for the shapes k_conv_direct covers (2 -> 16 and
// 16 -> 1 channels); cudaErrorInvalidValue for others.
bool conv3_direct_fits(int C, int Cout) { return (C == 2 && Cout == 16) || (C == 16 && Cout == 1); }

cudaError_t conv3_direct(const bf16* x, int C, int nx, int ny, int nz, int nb, const bf16* w,
                         int Cout, const float* bias, int relu, bf16* y_bf16, float* y_f32,
                         cudaStream_t st) {
  Vol g{nx, ny, nz, nb};
  auto blocks = [&](int dv) {
    return (unsigned)(((long)((nx + dv - 1) / dv) * ny * nz * nb + 255) / 256);
  };
  if (C == 2 && Cout == 16)
    k_conv_direct<2, 16><<<blocks(DirectShape<2, 16>::DV), 256, 0, st>>>(x, g, w, bias, relu,
                                                                         y_bf16, y_f32);
  else if (C == 16 && Cout == 1)
    k_conv_direct<16, 1><<<blocks(DirectShape<16, 1>::DV), 256, 0, st>>>(x, g, w, bias, relu,
                                                                         y_bf16, y_f32);
  else
    return cudaErrorInvalidValue;
  return cudaGetLastError();
}

// Weight layouts for conv3_tma: forward w_tap[t][co][ci] = w[co][t][ci];
// backward (data) w_tap[t][ci][co] = w[co][26 - t][ci] (flipped taps,
// transposed channels).
cudaError_t conv3_prep_weights(const bf16* w, int Cout, int Cin, int backward, bf16* w_tap,
                               cudaStream_t st) {
  const int n = Cout * 27 * Cin;
  k_wprep<<<std::min((n + 255) / 256, 1024), 256, 0, st>>>(w, Cout, Cin, backward, w_tap);
  return cudaGetLastError();
}

// y[v][n] = sum_{t, k} w_tap[t][n][k] x[v + tap(t)][k] (+ bias, ReLU, or
// zeroed where mask[v][n] <= 0); K (channels of x) a multiple of 16,
// N <= 128 output channels.  The input tensor must be 16-byte aligned.
cudaError_t conv3_tma(const bf16* x, int K, int nx, int ny, int nz, int nb, const bf16* w_tap,
                      int N, const float* bias, int relu, const bf16* mask, bf16* y_bf16,
                      float* y_f32, int* err, cudaStream_t st) {
  if (K % 16 != 0 || N < 1 || N > 128) return cudaErrorInvalidValue;
  PFN_cuTensorMapEncodeTiled_v12000 enc = encode_fn();
  if (!enc) return cudaErrorNotSupported;
  TmaGeom g{};
  g.nx = nx;
  g.ny = ny;
  g.nz = nz;
  g.nb = nb;
  g.groups = K / 16;
  g.npad = pad16(N);
  g.box_b = (uint32_t)(27 * g.npad * 16);
  g.b_bytes = (uint32_t)g.groups * 2u * g.box_b;
  // shared-memory plan: [resident weights][S stages][slack]; a voxel tile of
  // 256 when two stages fit, else 128
  const uint32_t budget =
      226u * 1024u - 1024u - conv_slack(g.npad) - ((conv_epi_bytes(g.npad) + 15u) & ~15u);
  int nt = 0;
  for (int cand : {256, 128}) {
    const int bx = pick_bx(nx, cand), by = cand / bx;
    const uint32_t box_a = (uint32_t)(bx * (by + 2) * 3 * 16);
    const uint32_t sa_al = (6 * box_a + 1023u) & ~1023u;
    const uint32_t b_al = (g.b_bytes + 1023u) & ~1023u;
    const bool res = b_al + 2 * sa_al <= budget;
    const uint32_t stage = res ? sa_al : ((6 * box_a + 2 * g.box_b + 1023u) & ~1023u);
    const uint32_t room = budget - (res ? b_al : 0u);
    const int stg = (int)std::min<uint32_t>(CONV_MAX_STAGES, room / stage);
    if (stg >= 2 || (cand == 128 && stg >= 1)) {
      nt = cand;
      g.BX = bx;
      g.BY = by;
      g.box_a = box_a;
      g.stage_a = 6 * box_a;
      g.resident_b = res ? 1 : 0;
      g.stage_off = res ? b_al : 0u;
      g.stage_bytes = stage;
      g.stages = stg;
      break;
    }
  }
  if (nt == 0) return cudaErrorInvalidValue;
  g.tiles_x = (nx + g.BX - 1) / g.BX;
  g.tiles_y = (ny + g.BY - 1) / g.BY;
  g.ntiles = g.tiles_x * g.tiles_y * nz * nb;
  CUtensorMap ta, tb;
  // input planes of 8 channels: dims (8 nx, ny, nz, nb K / 8), x and the
  // channel chunk innermost, so a box row is BX voxels x 16 bytes
  const cuuint64_t adim[4] = {(cuuint64_t)nx * 8, (cuuint64_t)ny, (cuuint64_t)nz,
                              (cuuint64_t)nb * (K / 8)};
  const cuuint64_t astr[3] = {(cuuint64_t)nx * 16, (cuuint64_t)nx * 16 * ny,
                              (cuuint64_t)nx * 16 * ny * nz};
  const cuuint32_t abox[4] = {(cuuint32_t)(8 * g.BX), (cuuint32_t)(g.BY + 2), 3, 1};
  const cuuint32_t es[5] = {1, 1, 1, 1, 1};
  if (enc(&ta, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<bf16*>(x), adim, astr, abox, es,
          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
          CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
    return cudaErrorInvalidValue;
  const cuuint64_t bdim[3] = {(cuuint64_t)K, (cuuint64_t)N, 27};
  const cuuint64_t bstr[2] = {(cuuint64_t)K * 2, (cuuint64_t)K * 2 * N};
  const cuuint32_t bbox[3] = {8, (cuuint32_t)g.npad, 27};
  if (enc(&tb, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, const_cast<bf16*>(w_tap), bdim, bstr, bbox,
          es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
          CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
    return cudaErrorInvalidValue;
  const int V = nx * ny * nz * nb;
  ConvEpi ep{y_bf16, y_f32, bias, mask, V, N, relu};
  return nt == 256 ? tma_launch_bx<256>(ta, tb, g, ep, err, st)
                   : tma_launch_bx<128>(ta, tb, g, ep, err, st);
}
}  // namespace pyro

// ------------------------------------------------------------------ C ABI
using namespace pyro;
using bf16 = __nv_bfloat16;

namespace {
int finish(cudaError_t e, DevBuf& err, cudaStream_t st, const char* what) {
  if (e != cudaSuccess) {
    set_error(std::string(what) + ": " + cudaGetErrorString(e));
    return PYRO_E_CUDA;
  }
  int h = 0;
  PYRO_CU(cudaMemcpyAsync(&h, err.p, 4, cudaMemcpyDeviceToHost, st));
  PYRO_CU(cudaStreamSynchronize(st));
  if (h) {
    set_error(std::string(what) + ": a tensor-core wait ran out");
    return PYRO_E_TIMEOUT;
  }
  return PYRO_OK;
}
bool conv_dims_ok(int nx, int ny, int nz, int nb) {
  return nx >= 1 && ny >= 1 && nz >= 1 && nb >= 1 && (int64_t)nx * ny * nz * nb < (1ll << 31);
}
bool chan_ok(int c) { return c >= 1 && c <= 128; }
}  // namespace

extern "C" {

int pyro_conv3_forward(const void* x, int C, int nx, int ny, int nz, int nb, const void* w,
                       int Cout, const float* bias, int relu, void* y, int y_f32, void* stream) {
  clear_error();
  PYRO_REQUIRE(x && w && y, "pyro_conv3_forward: null buffer");
  PYRO_REQUIRE(conv_dims_ok(nx, ny, nz, nb) && chan_ok(C) && chan_ok(Cout),
               "pyro_conv3_forward: invalid sizes");
  DevBuf err;
  int rc = err.alloc(4);
  if (rc != PYRO_OK) return rc;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  cudaError_t e;
  if (conv3_direct_fits(C, Cout)) {  // narrow layers on the CUDA cores
    e = conv3_direct((const bf16*)x, C, nx, ny, nz, nb, (const bf16*)w, Cout, bias, relu,
                     y_f32 ? nullptr : (bf16*)y, y_f32 ? (float*)y : nullptr, st);
    return finish(e, err, st, "pyro_conv3_forward");
  }
  if (C % 16 == 0) {  // TMA-staged kernel on tap-major weights
    DevBuf wt;
    if ((rc = wt.alloc((size_t)Cout * 27 * C * 2)) != PYRO_OK) return rc;
    e = conv3_prep_weights((const bf16*)w, Cout, C, 0, wt.as<bf16>(), st);
    if (e == cudaSuccess)
      e = conv3_tma((const bf16*)x, C, nx, ny, nz, nb, wt.as<bf16>(), Cout, bias, relu, nullptr,
                    y_f32 ? nullptr : (bf16*)y, y_f32 ? (float*)y : nullptr, err.as<int>(), st);
    return finish(e, err, st, "pyro_conv3_forward");
  }
  e = conv3_forward((const bf16*)x, C, nx, ny, nz, nb, (const bf16*)w, Cout, bias, relu,
                    y_f32 ? nullptr : (bf16*)y, y_f32 ? (float*)y : nullptr, err.as<int>(), st);
  return finish(e, err, st, "pyro_conv3_forward");
}

int pyro_conv3_backward_data(const void* dy, int Cout, int nx, int ny, int nz, int nb,
                             const void* w, int Cin, const void* act, void* dx, int dx_f32,
                             void* stream) {
  clear_error();
  PYRO_REQUIRE(dy && w && dx, "pyro_conv3_backward_data: null buffer");
  PYRO_REQUIRE(conv_dims_ok(nx, ny, nz, nb) && chan_ok(Cin) && chan_ok(Cout),
               "pyro_conv3_backward_data: invalid sizes");
  DevBuf err;
  int rc = err.alloc(4);
  if (rc != PYRO_OK) return rc;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  cudaError_t e;
  if (Cout % 16 == 0) {  // TMA-staged kernel on flipped, transposed weights
    DevBuf wt;
    if ((rc = wt.alloc((size_t)Cout * 27 * Cin * 2)) != PYRO_OK) return rc;
    e = conv3_prep_weights((const bf16*)w, Cout, Cin, 1, wt.as<bf16>(), st);
    if (e == cudaSuccess)
      e = conv3_tma((const bf16*)dy, Cout, nx, ny, nz, nb, wt.as<bf16>(), Cin, nullptr, 0,
                    (const bf16*)act, dx_f32 ? nullptr : (bf16*)dx, dx_f32 ? (float*)dx : nullptr,
                    err.as<int>(), st);
    return finish(e, err, st, "pyro_conv3_backward_data");
  }
  e = conv3_backward_data((const bf16*)dy, Cout, nx, ny, nz, nb, (const bf16*)w, Cin,
                          (const bf16*)act, dx_f32 ? nullptr : (bf16*)dx,
                          dx_f32 ? (float*)dx : nullptr, err.as<int>(), st);
  return finish(e, err, st, "pyro_conv3_backward_data");
}

int pyro_conv3_backward_weight(const void* x, int Cin, const void* dy, int Cout, int nx, int ny,
                               int nz, int nb, float* dw, void* stream) {
  clear_error();
  PYRO_REQUIRE(x && dy && dw, "pyro_conv3_backward_weight: null buffer");
  PYRO_REQUIRE(conv_dims_ok(nx, ny, nz, nb) && chan_ok(Cin) && chan_ok(Cout),
               "pyro_conv3_backward_weight: invalid sizes");
  DevBuf err;
  int rc = err.alloc(4);
  if (rc != PYRO_OK) return rc;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  cudaError_t e = conv3_backward_weight((const bf16*)x, Cin, (const bf16*)dy, Cout, nx, ny, nz,
                                        nb, dw, err.as<int>(), st);
  return finish(e, err, st, "pyro_conv3_backward_weight");
}

}  // extern "C"
