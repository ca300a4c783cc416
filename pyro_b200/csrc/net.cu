// net.cu — the learned pressure stage (network layout in net.h): the glue
// kernels around the tcgen05 convolutions (input normalisation, pooling,
// up-sampling with concatenation and their adjoints, bias gradients, loss,
// output scaling, Adam) and the C ABI.
//
// The network has no counterpart in the reference: it is the learned warm
// start that stands beside the multigrid pressure solve of
// src/sim.rs:451-491, which remains the fallback and the measure of its error.
#include <cuda_bf16.h>

#include <cmath>
#include <cstring>
#include <random>
#include <vector>

#include "net.h"

namespace pyro {

namespace {

using bf16 = __nv_bfloat16;
constexpr int NT = 256;
constexpr int MAX_VOLS = 64;
// device scalars: weighted pressure loss, gradient sum of squares, sum of
// squared normalised residuals and their cell count, then per volume
// (sum b^2, fluid cells)
enum { SC_LOSS = 0, SC_GSQ = 1, SC_RES = 2, SC_RCNT = 3, SC_VOL = 4 };

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
// Block of NT threads: sum v into *dst with one atomic.  Every thread calls.
__device__ __forceinline__ void block_add(double v, double* dst) {
  __shared__ double sh[NT / 32];
  v = warp_sum(v);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x < 32) {
    double s = threadIdx.x < NT / 32 ? sh[threadIdx.x] : 0.0;
    s = warp_sum(s);
    if (threadIdx.x == 0 && s != 0.0) atomicAdd(dst, s);
  }
}

// root mean square of b over the fluid cells of volume `vol` (0 if none)
__device__ __forceinline__ double vol_rms(const double* sc, int vol) {
  double s2 = sc[SC_VOL + 2 * vol], n = sc[SC_VOL + 2 * vol + 1];
  return (n > 0.0 && s2 > 0.0) ? sqrt(s2 / n) : 0.0;
}

struct Dv {  // volume dims on the device
  int nx, ny, nz, nb;
  // 32-bit arithmetic: a volume set holds fewer than 2^31 voxels (ensure())
  __device__ __forceinline__ void coords(size_t v, int& x, int& y, int& z, int& b) const {
    const uint32_t u = (uint32_t)v, r1 = u / (uint32_t)nx, r2 = r1 / (uint32_t)ny,
                   r3 = r2 / (uint32_t)nz;
    x = (int)(u - r1 * (uint32_t)nx);
    y = (int)(r1 - r2 * (uint32_t)ny);
    z = (int)(r2 - r3 * (uint32_t)nz);
    b = (int)r3;
  }
  __device__ __forceinline__ size_t idx(int x, int y, int z, int b) const {
    return (((size_t)b * nz + z) * ny + y) * nx + x;
  }
  __device__ __forceinline__ size_t voxels() const { return (size_t)nx * ny * nz * nb; }
};
inline Dv dv(NetVol v) { return Dv{v.nx, v.ny, v.nz, v.nb}; }

// Flat index i over (plane p, voxel v) of V voxels per plane, with 32-bit
// division when i fits.
__device__ __forceinline__ void plane_split(size_t i, size_t V, size_t& v, int& p) {
  if (i <= 0xFFFFFFFFull) {
    const uint32_t q = (uint32_t)i / (uint32_t)V;
    p = (int)q;
    v = (uint32_t)i - q * (uint32_t)V;
  } else {
    p = (int)(i / V);
    v = i - (size_t)p * V;
  }
}

// Activation layout: a tensor of C channels over V voxels with C a multiple
// of 8 is stored as C / 8 planes of [V][8 channels] (a plane is one 16-byte
// chunk per voxel, so a TMA box along x reads long contiguous rows); other
// channel counts (the 2-channel input, 1-channel gradients) as [V][C].
// Element offset of channel c of voxel v:
__device__ __forceinline__ size_t act_off(size_t v, int c, int C, size_t V) {
  return (C & 7) ? v * C + c : ((size_t)(c >> 3) * V + v) * 8 + (c & 7);
}

inline unsigned blocks_for(size_t n) {
  size_t b = (n + NT - 1) / NT;
  return (unsigned)std::min<size_t>(std::max<size_t>(b, 1), 148 * 32);
}

#define GRID_LOOP(i, n) \
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < (n); i += (size_t)gridDim.x * blockDim.x)

__global__ void __launch_bounds__(NT) k_stats(const float* __restrict__ b,
                                              const uint32_t* __restrict__ f, size_t cells,
                                              double* sc) {
  const int vol = blockIdx.y;
  const float* bv = b + (size_t)vol * cells;
  const uint32_t* fv = f + (size_t)vol * cells;
  double s2 = 0.0, n = 0.0;
  GRID_LOOP(i, cells) {
    if (fv[i] != 1u) {
      double x = bv[i];
      s2 += x * x;
      n += 1.0;
    }
  }
  block_add(s2, sc + SC_VOL + 2 * vol);
  block_add(n, sc + SC_VOL + 2 * vol + 1);
}

__global__ void __launch_bounds__(NT) k_input(const float* __restrict__ b,
                                              const uint32_t* __restrict__ f, size_t cells,
                                              int nb, const double* __restrict__ sc,
                                              __nv_bfloat162* __restrict__ in0) {
  GRID_LOOP(i, cells * nb) {
    int vol = (int)(i / cells);
    double s = vol_rms(sc, vol);
    bool solid = f[i] == 1u;
    float v = (!solid && s > 0.0) ? (float)((double)b[i] / s) : 0.0f;
    in0[i] = __floats2bfloat162_rn(v, solid ? 1.0f : 0.0f);
  }
}

// 8 channels as 4 x bf16x2 <-> float
__device__ __forceinline__ void unpack8(uint4 u, float (&f)[8]) {
  const __nv_bfloat162* h = reinterpret_cast<const __nv_bfloat162*>(&u);
#pragma unroll
  for (int j = 0; j < 4; j++) {
    float2 t = __bfloat1622float2(h[j]);
    f[2 * j] = t.x;
    f[2 * j + 1] = t.y;
  }
}
__device__ __forceinline__ uint4 pack8(const float (&f)[8]) {
  uint4 u;
  __nv_bfloat162* h = reinterpret_cast<__nv_bfloat162*>(&u);
#pragma unroll
  for (int j = 0; j < 4; j++) h[j] = __floats2bfloat162_rn(f[2 * j], f[2 * j + 1]);
  return u;
}

// coarse[cv][c] = mean of the children inside the fine volume
__global__ void __launch_bounds__(NT) k_pool(const bf16* __restrict__ in, int C, Dv fd,
                                             bf16* __restrict__ out) {
  Dv cd{(fd.nx + 1) / 2, (fd.ny + 1) / 2, (fd.nz + 1) / 2, fd.nb};
  const int ch = C / 8;
  GRID_LOOP(i, cd.voxels() * ch) {
    size_t cv;
    int c8;
    plane_split(i, cd.voxels(), cv, c8);
    int x, y, z, b;
    cd.coords(cv, x, y, z, b);
    float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    int cnt = 0;
    for (int dz = 0; dz < 2; dz++)
      for (int dy = 0; dy < 2; dy++)
        for (int dx = 0; dx < 2; dx++) {
          int fx = 2 * x + dx, fy = 2 * y + dy, fz = 2 * z + dz;
          if (fx >= fd.nx || fy >= fd.ny || fz >= fd.nz) continue;
          float t[8];
          unpack8(*reinterpret_cast<const uint4*>(in + act_off(fd.idx(fx, fy, fz, b), c8 * 8, C,
                                                               fd.voxels())),
                  t);
#pragma unroll
          for (int j = 0; j < 8; j++) acc[j] += t[j];
          cnt++;
        }
    float inv = 1.0f / (float)cnt;
#pragma unroll
    for (int j = 0; j < 8; j++) acc[j] *= inv;
    *reinterpret_cast<uint4*>(out + act_off(cv, c8 * 8, C, cd.voxels())) = pack8(acc);
  }
}

// out[fv] = [a[parent(fv)] (Ca channels), skip[fv] (Cb channels)]
__global__ void __launch_bounds__(NT) k_upcat(const bf16* __restrict__ a, int Ca,
                                              const bf16* __restrict__ skip, int Cb, Dv fd,
                                              bf16* __restrict__ out) {
  Dv cd{(fd.nx + 1) / 2, (fd.ny + 1) / 2, (fd.nz + 1) / 2, fd.nb};
  const int Ct = Ca + Cb, ch = (skip ? Ct : Ca) / 8;  // skip null: already in place
  GRID_LOOP(i, fd.voxels() * ch) {
    size_t fv;
    int c;
    plane_split(i, fd.voxels(), fv, c);
    c *= 8;
    uint4 u;
    if (c < Ca) {
      int x, y, z, b;
      fd.coords(fv, x, y, z, b);
      u = *reinterpret_cast<const uint4*>(
          a + act_off(cd.idx(x >> 1, y >> 1, z >> 1, b), c, Ca, cd.voxels()));
    } else {
      u = *reinterpret_cast<const uint4*>(skip + act_off(fv, c - Ca, Cb, fd.voxels()));
    }
    *reinterpret_cast<uint4*>(out + act_off(fv, c, Ct, fd.voxels())) = u;
  }
}

// adjoint of up2 on the first Ca channels of dc [fine][Ct]: sum of children
__global__ void __launch_bounds__(NT) k_upback(const bf16* __restrict__ dc, int Ct, int Ca,
                                               Dv fd, bf16* __restrict__ out) {
  Dv cd{(fd.nx + 1) / 2, (fd.ny + 1) / 2, (fd.nz + 1) / 2, fd.nb};
  const int ch = Ca / 8;
  GRID_LOOP(i, cd.voxels() * ch) {
    size_t cv;
    int c;
    plane_split(i, cd.voxels(), cv, c);
    c *= 8;
    int x, y, z, b;
    cd.coords(cv, x, y, z, b);
    float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int dz = 0; dz < 2; dz++)
      for (int dy = 0; dy < 2; dy++)
        for (int dx = 0; dx < 2; dx++) {
          int fx = 2 * x + dx, fy = 2 * y + dy, fz = 2 * z + dz;
          if (fx >= fd.nx || fy >= fd.ny || fz >= fd.nz) continue;
          float t[8];
          unpack8(*reinterpret_cast<const uint4*>(
                      dc + act_off(fd.idx(fx, fy, fz, b), c, Ct, fd.voxels())),
                  t);
#pragma unroll
          for (int j = 0; j < 8; j++) acc[j] += t[j];
        }
    *reinterpret_cast<uint4*>(out + act_off(cv, c, Ca, cd.voxels())) = pack8(acc);
  }
}

// dz[fv] = (dp[parent] / children(parent) + skip[fv]) * (act[fv] > 0):
// adjoint of the average pooling plus the skip connection's gradient,
// through the ReLU that produced act.
__global__ void __launch_bounds__(NT) k_poolback(const bf16* __restrict__ dp, int C,
                                                 const bf16* __restrict__ skip, int sstride,
                                                 int soff, const bf16* __restrict__ act, Dv fd,
                                                 bf16* __restrict__ dz) {
  Dv cd{(fd.nx + 1) / 2, (fd.ny + 1) / 2, (fd.nz + 1) / 2, fd.nb};
  const int ch = C / 8;
  GRID_LOOP(i, fd.voxels() * ch) {
    size_t fv;
    int c;
    plane_split(i, fd.voxels(), fv, c);
    c *= 8;
    int x, y, z, b;
    fd.coords(fv, x, y, z, b);
    int px = x >> 1, py = y >> 1, pz = z >> 1;
    int cnt = (2 * px + 1 < fd.nx ? 2 : 1) * (2 * py + 1 < fd.ny ? 2 : 1) *
              (2 * pz + 1 < fd.nz ? 2 : 1);
    float g[8], s[8], a[8];
    const size_t Vf = fd.voxels();
    unpack8(*reinterpret_cast<const uint4*>(dp + act_off(cd.idx(px, py, pz, b), c, C,
                                                         cd.voxels())),
            g);
    unpack8(*reinterpret_cast<const uint4*>(act + act_off(fv, c, C, Vf)), a);
    if (skip)
      unpack8(*reinterpret_cast<const uint4*>(skip + act_off(fv, soff + c, sstride, Vf)), s);
    float inv = 1.0f / (float)cnt;
#pragma unroll
    for (int j = 0; j < 8; j++) {
      float v = g[j] * inv + (skip ? s[j] : 0.0f);
      g[j] = a[j] > 0.0f ? v : 0.0f;
    }
    *reinterpret_cast<uint4*>(dz + act_off(fv, c, C, Vf)) = pack8(g);
  }
}

// db[c] += sum_v dz[v][c]   (C divides NT)
__global__ void __launch_bounds__(NT) k_bias_grad(const bf16* __restrict__ dz, size_t V, int C,
                                                  float* __restrict__ db) {
  __shared__ float sh[NT];
  const int c = threadIdx.x % C, lane = threadIdx.x / C, lanes = NT / C;
  float acc = 0.0f;
  for (size_t v = (size_t)blockIdx.x * lanes + lane; v < V; v += (size_t)gridDim.x * lanes)
    acc += __bfloat162float(dz[act_off(v, c, C, V)]);
  sh[threadIdx.x] = acc;
  __syncthreads();
  if ((int)threadIdx.x < C) {
    float s = 0.0f;
    for (int l = 0; l < lanes; l++) s += sh[l * C + threadIdx.x];
    atomicAdd(db + threadIdx.x, s);
  }
}

// phi = out * scale * s (fluid), 0 (solid); scale = out_scale * h^2
__global__ void __launch_bounds__(NT) k_output(const float* __restrict__ out,
                                               const uint32_t* __restrict__ f, size_t cells,
                                               int nb, const double* __restrict__ sc, double scale,
                                               float* __restrict__ phi) {
  GRID_LOOP(i, cells * nb) {
    int vol = (int)(i / cells);
    phi[i] = f[i] == 1u ? 0.0f : (float)((double)out[i] * scale * vol_rms(sc, vol));
  }
}

// Normalised residual of the prediction on the interior fluid cells of each
// volume (all six neighbours inside it): res = b / s - kappa (sum of fluid
// neighbours' out - count * out), the pressure operator of the solver in
// the network's units (kappa = out_scale); 0 elsewhere.  Accumulates
// sum res^2 and the cell count.
__global__ void __launch_bounds__(NT) k_res(const float* __restrict__ out,
                                            const float* __restrict__ b,
                                            const uint32_t* __restrict__ f, Dv d,
                                            double* __restrict__ sc, double kappa,
                                            float* __restrict__ res) {
  double r2 = 0.0, n = 0.0;
  GRID_LOOP(i, d.voxels()) {
    int x, y, z, v;
    d.coords(i, x, y, z, v);
    float r = 0.0f;
    if (f[i] != 1u && x > 0 && y > 0 && z > 0 && x < d.nx - 1 && y < d.ny - 1 && z < d.nz - 1) {
      const size_t st[3] = {1, (size_t)d.nx, (size_t)d.nx * d.ny};
      double sum = 0.0, cnt = 0.0;
#pragma unroll
      for (int k = 0; k < 6; k++) {
        size_t j = (k & 1) ? i - st[k >> 1] : i + st[k >> 1];
        if (f[j] == 1u) continue;
        sum += (double)out[j];
        cnt += 1.0;
      }
      double s = vol_rms(sc, v);
      float bh = s > 0.0 ? (float)((double)b[i] / s) : 0.0f;
      double rd = (double)bh - kappa * (sum - cnt * (double)out[i]);
      r = (float)rd;
      r2 += (double)r * (double)r;
      n += 1.0;
    }
    res[i] = r;
  }
  block_add(r2, sc + SC_RES);
  block_add(n, sc + SC_RCNT);
}

// Gradient of the loss with respect to out (BF16):
//   w_phi * mean over fluid cells of (out - phi_t / (scale s))^2
// + w_res * mean over the cells of k_res of res^2,
// scale = out_scale * h^2.  The first term's value is accumulated here;
// the second's comes from k_res.  The residual term's gradient is
// -2 kappa w_res / count * (L res) with L the same symmetric operator.
__global__ void __launch_bounds__(NT) k_loss(const float* __restrict__ out,
                                             const float* __restrict__ phi_t,
                                             const uint32_t* __restrict__ f, Dv d,
                                             double* __restrict__ sc, double scale, double w_phi,
                                             double w_res, double kappa,
                                             const float* __restrict__ res,
                                             bf16* __restrict__ g) {
  const size_t cells = (size_t)d.nx * d.ny * d.nz;
  double n = 0.0;
  for (int v = 0; v < d.nb; v++) n += sc[SC_VOL + 2 * v + 1];
  const double inv_n = n > 0.0 ? 1.0 / n : 0.0;
  const double rc = res ? sc[SC_RCNT] : 0.0;
  const double cres = rc > 0.0 ? -2.0 * kappa * w_res / rc : 0.0;
  double l = 0.0;
  GRID_LOOP(i, d.voxels()) {
    double gi = 0.0;
    if (f[i] != 1u) {
      int vol = (int)(i / cells);
      if (w_phi > 0.0) {
        double s = vol_rms(sc, vol) * scale;
        double t = s > 0.0 ? (double)phi_t[i] / s : 0.0;
        double dd = (double)out[i] - t;
        l += w_phi * dd * dd * inv_n;
        gi = 2.0 * w_phi * dd * inv_n;
      }
      if (cres != 0.0) {
        int x, y, z, v;
        d.coords(i, x, y, z, v);
        double sum = 0.0, cnt = 0.0;
        const int c[3] = {x, y, z}, lim[3] = {d.nx, d.ny, d.nz};
        const size_t st[3] = {1, (size_t)d.nx, (size_t)d.nx * d.ny};
#pragma unroll
        for (int k = 0; k < 6; k++) {
          int a = k >> 1;
          bool up = (k & 1) == 0;
          if (up ? c[a] + 1 >= lim[a] : c[a] == 0) continue;
          size_t j = up ? i + st[a] : i - st[a];
          if (f[j] == 1u) continue;
          sum += (double)res[j];
          cnt += 1.0;
        }
        gi += cres * (sum - cnt * (double)res[i]);
      }
    }
    g[i] = __float2bfloat16((float)gi);
  }
  block_add(l, sc + SC_LOSS);
}

__global__ void __launch_bounds__(NT) k_sumsq(const float* __restrict__ g, size_t n, double* dst) {
  double s = 0.0;
  GRID_LOOP(i, n) s += (double)g[i] * (double)g[i];
  block_add(s, dst);
}

// Adam with bias correction on the FP32 master copy; the gradient is scaled
// so that its global norm is at most `clip` (when clip > 0), and a step with
// a non-finite gradient is skipped.  The BF16
// weight copy is refreshed for the first n_w entries.
__global__ void __launch_bounds__(NT) k_adam(float* __restrict__ p, const float* __restrict__ g,
                                             float* __restrict__ m, float* __restrict__ v,
                                             size_t n, size_t n_w, bf16* __restrict__ wbf,
                                             float lr, float b1, float b2, float eps, float bc1,
                                             float bc2, float clip, const double* __restrict__ sc) {
  // a step whose gradient is not finite is skipped (state unchanged)
  const double norm = sqrt(sc[SC_GSQ]);
  if (!isfinite(norm)) return;
  float gs = 1.0f;
  if (clip > 0.0f && norm > (double)clip) gs = (float)((double)clip / norm);
  GRID_LOOP(i, n) {
    float gi = g[i] * gs;
    float mi = b1 * m[i] + (1.0f - b1) * gi;
    float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    float pi = p[i] - lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
    p[i] = pi;
    if (i < n_w) wbf[i] = __float2bfloat16(pi);
  }
}

__global__ void __launch_bounds__(NT) k_to_bf16(const float* __restrict__ p, size_t n,
                                                bf16* __restrict__ w) {
  GRID_LOOP(i, n) w[i] = __float2bfloat16(p[i]);
}

}  // namespace

}  // namespace pyro

using namespace pyro;
using bf16 = __nv_bfloat16;

int PyroNet::init() {
  size_t w = 0, b = 0;
  for (int l = 0; l < NET_LAYERS; l++) {
    w_off[l] = w;
    b_off[l] = b;
    w += (size_t)NET_SPEC[l].cout * 27 * NET_SPEC[l].cin;
    b += (size_t)NET_SPEC[l].cout;
  }
  w_off[NET_LAYERS] = w;
  b_off[NET_LAYERS] = b;
  n_w = w;
  n_params = w + b;
  int rc;
  if ((rc = master.alloc(n_params * 4)) || (rc = grad.alloc(n_params * 4)) ||
      (rc = adam_m.alloc(n_params * 4)) || (rc = adam_v.alloc(n_params * 4)) ||
      (rc = wbf.alloc(n_w * 2)) || (rc = wtf.alloc(n_w * 2)) || (rc = wtb.alloc(n_w * 2)) ||
      (rc = scal.alloc((SC_VOL + 2 * MAX_VOLS) * 8)) ||
      (rc = err.alloc(4)))
    return rc;
  if (cudaMallocHost(&host_scal, (SC_VOL + 2 * MAX_VOLS) * 8) != cudaSuccess) {
    set_error("net: pinned allocation failed");
    return PYRO_E_NOMEM;
  }
  if (cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking) != cudaSuccess) {
    set_error("net: cudaStreamCreate failed");
    return PYRO_E_CUDA;
  }
  return PYRO_OK;
}

PyroNet::~PyroNet() {
  if (stream) {
    cudaStreamSynchronize(stream);
    cudaStreamDestroy(stream);
  }
  if (host_scal) cudaFreeHost(host_scal);
}

int PyroNet::ensure(NetVol v, bool bwd) {
  PYRO_REQUIRE(v.nb >= 1 && v.nb <= MAX_VOLS, "net: 1 to 64 volumes per call");
  PYRO_REQUIRE(v.nx >= 1 && v.ny >= 1 && v.nz >= 1 && v.voxels() < (1ull << 31),
               "net: invalid volume dims");
  if (v == vol && (has_bwd || !bwd)) return PYRO_OK;
  const size_t V0 = v.voxels(), V1 = v.half().voxels(), V2 = v.half().half().voxels();
  struct A {
    DevBuf* b;
    size_t n;
  };
  std::vector<A> fw = {{&in0, V0 * 2},  {&e0a, V0 * 16}, {&p1, V1 * 16},
                       {&e1a, V1 * 32}, {&p2, V2 * 32}, {&e2a, V2 * 64},
                       {&e2, V2 * 64},  {&c1, V1 * 96},  {&d1, V1 * 32}, {&c0, V0 * 48},
                       {&d0, V0 * 16}};
  std::vector<A> bw = {{&g9, V0 * 1},   {&g8, V0 * 16}, {&gc0, V0 * 48}, {&g7, V1 * 32},
                       {&gc1, V1 * 96}, {&g6, V2 * 64}, {&g5, V2 * 64},  {&gp2, V2 * 32},
                       {&g4, V1 * 32},  {&g3, V1 * 32}, {&gp1, V1 * 16}, {&g2, V0 * 16},
                       {&g1, V0 * 16}};
  vol = NetVol{0, 0, 0, 0};
  has_bwd = false;
  int rc;
  for (auto& a : fw)
    if ((rc = a.b->alloc(a.n * 2))) return rc;
  if ((rc = out.alloc(V0 * 4))) return rc;
  if (bwd) {
    for (auto& a : bw)
      if ((rc = a.b->alloc(a.n * 2))) return rc;
    if ((rc = res.alloc(V0 * 4))) return rc;
  } else {
    for (auto& a : bw) a.b->release();
    res.release();
  }
  vol = v;
  has_bwd = bwd;
  return PYRO_OK;
}

#define NET_CU(call)                                                                  \
  do {                                                                                \
    cudaError_t e_ = (call);                                                          \
    if (e_ != cudaSuccess) {                                                          \
      set_error(std::string("net: ") + #call + ": " + cudaGetErrorString(e_));        \
      return PYRO_E_CUDA;                                                             \
    }                                                                                 \
  } while (0)

int PyroNet::forward(const float* b, const uint32_t* flags, NetVol v, cudaStream_t st) {
  const NetVol v1 = v.half(), v2 = v1.half();
  const size_t cells = (size_t)v.nx * v.ny * v.nz;
  double* S = scal.as<double>();
  int* E = err.as<int>();
  NET_CU(cudaMemsetAsync(scal.p, 0, scal.bytes, st));
  k_stats<<<dim3(std::min<unsigned>(blocks_for(cells), 148 * 4), v.nb), NT, 0, st>>>(b, flags,
                                                                                    cells, S);
  k_input<<<blocks_for(cells * v.nb), NT, 0, st>>>(b, flags, cells, v.nb, S,
                                                   in0.as<__nv_bfloat162>());
  NET_CU(cudaGetLastError());
  auto conv = [&](const bf16* x, int l, NetVol g, bf16* y, float* yf) -> cudaError_t {
    const NetLayer& L = NET_SPEC[l];
    if (conv3_direct_fits(L.cin, L.cout))
      return conv3_direct(x, L.cin, g.nx, g.ny, g.nz, g.nb, w(l), L.cout, bias(l), L.relu, y, yf,
                          st);
    if (L.cin % 16 == 0)
      return conv3_tma(x, L.cin, g.nx, g.ny, g.nz, g.nb, wf(l), L.cout, bias(l), L.relu, nullptr,
                       y, yf, E, st);
    return conv3_forward(x, L.cin, g.nx, g.ny, g.nz, g.nb, w(l), L.cout, bias(l), L.relu, y, yf,
                         E, st);
  };
  auto B = [](const DevBuf& d) { return d.as<bf16>(); };
  // the skip connections e0, e1 are written straight into their planes of
  // the concatenations c0, c1
  NET_CU(conv(B(in0), 0, v, B(e0a), nullptr));
  NET_CU(conv(B(e0a), 1, v, skip0(), nullptr));
  k_pool<<<blocks_for(v1.voxels() * 2), NT, 0, st>>>(skip0(), 16, dv(v), B(p1));
  NET_CU(conv(B(p1), 2, v1, B(e1a), nullptr));
  NET_CU(conv(B(e1a), 3, v1, skip1(), nullptr));
  k_pool<<<blocks_for(v2.voxels() * 4), NT, 0, st>>>(skip1(), 32, dv(v1), B(p2));
  NET_CU(conv(B(p2), 4, v2, B(e2a), nullptr));
  NET_CU(conv(B(e2a), 5, v2, B(e2), nullptr));
  k_upcat<<<blocks_for(v1.voxels() * 8), NT, 0, st>>>(B(e2), 64, nullptr, 32, dv(v1), B(c1));
  NET_CU(conv(B(c1), 6, v1, B(d1), nullptr));
  k_upcat<<<blocks_for(v.voxels() * 4), NT, 0, st>>>(B(d1), 32, nullptr, 16, dv(v), B(c0));
  NET_CU(conv(B(c0), 7, v, B(d0), nullptr));
  NET_CU(conv(B(d0), 8, v, nullptr, out.as<float>()));
  return PYRO_OK;
}

int PyroNet::output(const uint32_t* flags, float h, float* phi, NetVol v, cudaStream_t st) {
  const size_t cells = (size_t)v.nx * v.ny * v.nz;
  k_output<<<blocks_for(cells * v.nb), NT, 0, st>>>(out.as<float>(), flags, cells, v.nb,
                                                    scal.as<double>(),
                                                    (double)out_scale * h * h, phi);
  NET_CU(cudaGetLastError());
  return PYRO_OK;
}

int PyroNet::loss_backward(const float* b, const uint32_t* flags, const float* phi_t, float h,
                           NetVol v, cudaStream_t st) {
  int rc;
  if ((rc = forward(b, flags, v, st))) return rc;
  const NetVol v1 = v.half(), v2 = v1.half();
  const size_t cells = (size_t)v.nx * v.ny * v.nz;
  double* S = scal.as<double>();
  int* E = err.as<int>();
  float* G = grad.as<float>();
  NET_CU(cudaMemsetAsync(grad.p, 0, grad.bytes, st));
  if (w_res > 0.0f)
    k_res<<<blocks_for(cells * v.nb), NT, 0, st>>>(out.as<float>(), b, flags, dv(v), S,
                                                   (double)out_scale, res.as<float>());
  k_loss<<<blocks_for(cells * v.nb), NT, 0, st>>>(
      out.as<float>(), phi_t, flags, dv(v), S, (double)out_scale * h * h, (double)w_phi,
      (double)w_res, (double)out_scale, w_res > 0.0f ? res.as<float>() : nullptr, g9.as<bf16>());
  NET_CU(cudaGetLastError());
  auto wg = [&](const DevBuf& x, const DevBuf& dz, int l, NetVol g) -> cudaError_t {
    const NetLayer& L = NET_SPEC[l];
    cudaError_t e = conv3_backward_weight(x.as<bf16>(), L.cin, dz.as<bf16>(), L.cout, g.nx, g.ny,
                                          g.nz, g.nb, G + w_off[l], E, st);
    if (e != cudaSuccess) return e;
    k_bias_grad<<<std::min<unsigned>(blocks_for(g.voxels() * L.cout), 148 * 4), NT, 0, st>>>(
        dz.as<bf16>(), g.voxels(), L.cout, G + n_w + b_off[l]);
    return cudaGetLastError();
  };
  auto bd = [&](const DevBuf& dz, int l, NetVol g, const DevBuf* act, DevBuf& dx) -> cudaError_t {
    const NetLayer& L = NET_SPEC[l];
    if (L.cout % 16 == 0)
      return conv3_tma(dz.as<bf16>(), L.cout, g.nx, g.ny, g.nz, g.nb, wb(l), L.cin, nullptr, 0,
                       act ? act->as<bf16>() : nullptr, dx.as<bf16>(), nullptr, E, st);
    return conv3_backward_data(dz.as<bf16>(), L.cout, g.nx, g.ny, g.nz, g.nb, w(l), L.cin,
                               act ? act->as<bf16>() : nullptr, dx.as<bf16>(), nullptr, E, st);
  };
  NET_CU(wg(d0, g9, 8, v));
  NET_CU(bd(g9, 8, v, &d0, g8));
  NET_CU(wg(c0, g8, 7, v));
  NET_CU(bd(g8, 7, v, &c0, gc0));
  k_upback<<<blocks_for(v1.voxels() * 4), NT, 0, st>>>(gc0.as<bf16>(), 48, 32, dv(v),
                                                       g7.as<bf16>());
  NET_CU(wg(c1, g7, 6, v1));
  NET_CU(bd(g7, 6, v1, &c1, gc1));
  k_upback<<<blocks_for(v2.voxels() * 8), NT, 0, st>>>(gc1.as<bf16>(), 96, 64, dv(v1),
                                                       g6.as<bf16>());
  NET_CU(wg(e2a, g6, 5, v2));
  NET_CU(bd(g6, 5, v2, &e2a, g5));
  NET_CU(wg(p2, g5, 4, v2));
  NET_CU(bd(g5, 4, v2, nullptr, gp2));
  k_poolback<<<blocks_for(v1.voxels() * 4), NT, 0, st>>>(gp2.as<bf16>(), 32, gc1.as<bf16>(), 96,
                                                         64, skip1(), dv(v1),
                                                         g4.as<bf16>());
  NET_CU(wg(e1a, g4, 3, v1));
  NET_CU(bd(g4, 3, v1, &e1a, g3));
  NET_CU(wg(p1, g3, 2, v1));
  NET_CU(bd(g3, 2, v1, nullptr, gp1));
  k_poolback<<<blocks_for(v.voxels() * 2), NT, 0, st>>>(gp1.as<bf16>(), 16, gc0.as<bf16>(), 48,
                                                        32, skip0(), dv(v), g2.as<bf16>());
  NET_CU(wg(e0a, g2, 1, v));
  NET_CU(bd(g2, 1, v, &e0a, g1));
  NET_CU(wg(in0, g1, 0, v));
  NET_CU(cudaGetLastError());
  return PYRO_OK;
}

int PyroNet::adam(float lr, float clip, cudaStream_t st) {
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  adam_t++;
  float bc1 = (float)(1.0 - std::pow((double)b1, (double)adam_t));
  float bc2 = (float)(1.0 - std::pow((double)b2, (double)adam_t));
  double* S = scal.as<double>();
  NET_CU(cudaMemsetAsync(S + SC_GSQ, 0, 8, st));
  k_sumsq<<<blocks_for(n_params), NT, 0, st>>>(grad.as<float>(), n_params, S + SC_GSQ);
  k_adam<<<blocks_for(n_params), NT, 0, st>>>(master.as<float>(), grad.as<float>(),
                                              adam_m.as<float>(), adam_v.as<float>(), n_params,
                                              n_w, wbf.as<bf16>(), lr, b1, b2, eps, bc1, bc2,
                                              clip, S);
  NET_CU(cudaGetLastError());
  return refresh_taps(st);
}

int PyroNet::refresh_taps(cudaStream_t st) {
  for (int l = 0; l < NET_LAYERS; l++) {
    const NetLayer& L = NET_SPEC[l];
    NET_CU(conv3_prep_weights(w(l), L.cout, L.cin, 0, wtf.as<bf16>() + w_off[l], st));
    NET_CU(conv3_prep_weights(w(l), L.cout, L.cin, 1, wtb.as<bf16>() + w_off[l], st));
  }
  return PYRO_OK;
}

int PyroNet::read_loss(cudaStream_t st, double* loss) {
  int rc = check_err(st);
  if (rc) return rc;
  double h[4];
  NET_CU(cudaMemcpy(h, scal.p, sizeof(h), cudaMemcpyDeviceToHost));
  *loss = h[SC_LOSS] + (w_res > 0.0f && h[SC_RCNT] > 0.0 ? w_res * h[SC_RES] / h[SC_RCNT] : 0.0);
  return PYRO_OK;
}

int PyroNet::check_err(cudaStream_t st) {
  int h = 0;
  NET_CU(cudaMemcpyAsync(&h, err.p, 4, cudaMemcpyDeviceToHost, st));
  NET_CU(cudaStreamSynchronize(st));
  if (h) {
    cudaMemsetAsync(err.p, 0, 4, st);
    set_error("net: a tensor-core wait ran out");
    return PYRO_E_TIMEOUT;
  }
  return PYRO_OK;
}

// ------------------------------------------------------------------ C ABI
namespace {
cudaStream_t pick(PyroNet* n, void* s) { return s ? reinterpret_cast<cudaStream_t>(s) : n->stream; }
int check_vol(uint32_t nx, uint32_t ny, uint32_t nz, uint32_t nb) {
  PYRO_REQUIRE(nx >= 1 && ny >= 1 && nz >= 1 && nb >= 1 && nb <= (uint32_t)MAX_VOLS,
               "net: invalid volume dims");
  PYRO_REQUIRE((uint64_t)nx * ny * nz * nb < (1ull << 31), "net: volume too large");
  return PYRO_OK;
}
}  // namespace

extern "C" {

int pyro_net_create(uint64_t seed, PyroNet** out) {
  clear_error();
  PYRO_REQUIRE(out, "pyro_net_create: null argument");
  *out = nullptr;
  PyroNet* n = new PyroNet();
  int rc = n->init();
  if (rc) {
    delete n;
    return rc;
  }
  // He-normal weights (ReLU layers), zero biases; the last layer is scaled
  // down so the initial output is small.
  std::mt19937_64 rng(seed);
  std::vector<float> p(n->n_params, 0.0f);
  for (int l = 0; l < NET_LAYERS; l++) {
    const NetLayer& L = NET_SPEC[l];
    double sd = std::sqrt(2.0 / (27.0 * L.cin)) * (L.relu ? 1.0 : 0.1);
    std::normal_distribution<double> nd(0.0, sd);
    for (size_t i = n->w_off[l]; i < n->w_off[l + 1]; i++) p[i] = (float)nd(rng);
  }
  if (cudaMemcpyAsync(n->master.p, p.data(), n->n_params * 4, cudaMemcpyHostToDevice,
                      n->stream) != cudaSuccess) {
    delete n;
    set_error("pyro_net_create: upload failed");
    return PYRO_E_CUDA;
  }
  k_to_bf16<<<blocks_for(n->n_w), NT, 0, n->stream>>>(n->master.as<float>(), n->n_w,
                                                      n->wbf.as<bf16>());
  if (n->refresh_taps(n->stream) != PYRO_OK || cudaStreamSynchronize(n->stream) != cudaSuccess) {
    delete n;
    set_error("pyro_net_create: weight conversion failed");
    return PYRO_E_CUDA;
  }
  *out = n;
  return PYRO_OK;
}

int pyro_net_destroy(PyroNet* n) {
  clear_error();
  delete n;
  return PYRO_OK;
}

int pyro_net_param_count(const PyroNet* n, uint64_t* count) {
  clear_error();
  PYRO_REQUIRE(n && count, "pyro_net_param_count: null argument");
  *count = n->n_params;
  return PYRO_OK;
}

int pyro_net_get_params(PyroNet* n, float* host, uint64_t count, float* out_scale) {
  clear_error();
  PYRO_REQUIRE(n && host, "pyro_net_get_params: null argument");
  PYRO_REQUIRE(count == n->n_params, "pyro_net_get_params: wrong parameter count");
  PYRO_CU(cudaStreamSynchronize(n->stream));
  PYRO_CU(cudaMemcpy(host, n->master.p, count * 4, cudaMemcpyDeviceToHost));
  if (out_scale) *out_scale = n->out_scale;
  return PYRO_OK;
}

// Sets the FP32 master weights (and their BF16 copy) and the output scale;
// resets the optimiser state.
int pyro_net_set_params(PyroNet* n, const float* host, uint64_t count, float out_scale) {
  clear_error();
  PYRO_REQUIRE(n && host, "pyro_net_set_params: null argument");
  PYRO_REQUIRE(count == n->n_params, "pyro_net_set_params: wrong parameter count");
  PYRO_REQUIRE(std::isfinite(out_scale) && out_scale > 0.0f,
               "pyro_net_set_params: out_scale must be positive");
  PYRO_CU(cudaStreamSynchronize(n->stream));
  // on the network's stream, so the conversion below reads the new weights
  // (a pageable cudaMemcpy may still be in flight when it returns)
  PYRO_CU(cudaMemcpyAsync(n->master.p, host, count * 4, cudaMemcpyHostToDevice, n->stream));
  PYRO_CU(cudaMemsetAsync(n->adam_m.p, 0, n->adam_m.bytes, n->stream));
  PYRO_CU(cudaMemsetAsync(n->adam_v.p, 0, n->adam_v.bytes, n->stream));
  k_to_bf16<<<blocks_for(n->n_w), NT, 0, n->stream>>>(n->master.as<float>(), n->n_w,
                                                      n->wbf.as<bf16>());
  PYRO_CU(cudaGetLastError());
  int rc = n->refresh_taps(n->stream);
  if (rc) return rc;
  PYRO_CU(cudaStreamSynchronize(n->stream));
  n->out_scale = out_scale;
  n->adam_t = 0;
  return PYRO_OK;
}

int pyro_net_forward(PyroNet* n, const float* b, const uint32_t* flags, uint32_t nx,
                     uint32_t ny, uint32_t nz, uint32_t nb, float h, float* phi, void* stream) {
  clear_error();
  PYRO_REQUIRE(n && b && flags && phi, "pyro_net_forward: null argument");
  PYRO_REQUIRE(h > 0.0f, "pyro_net_forward: h must be positive");
  int rc = check_vol(nx, ny, nz, nb);
  if (rc) return rc;
  NetVol v{(int)nx, (int)ny, (int)nz, (int)nb};
  cudaStream_t st = pick(n, stream);
  if ((rc = n->ensure(v, false)) || (rc = n->forward(b, flags, v, st)) ||
      (rc = n->output(flags, h, phi, v, st)))
    return rc;
  return n->check_err(st);
}

int pyro_net_loss_grad(PyroNet* n, const float* b, const uint32_t* flags, const float* phi_t,
                       uint32_t nx, uint32_t ny, uint32_t nz, uint32_t nb, float h,
                       double* loss, float* grad_host, void* stream) {
  clear_error();
  PYRO_REQUIRE(n && b && flags && phi_t, "pyro_net_loss_grad: null argument");
  PYRO_REQUIRE(h > 0.0f, "pyro_net_loss_grad: h must be positive");
  int rc = check_vol(nx, ny, nz, nb);
  if (rc) return rc;
  NetVol v{(int)nx, (int)ny, (int)nz, (int)nb};
  cudaStream_t st = pick(n, stream);
  if ((rc = n->ensure(v, true)) || (rc = n->loss_backward(b, flags, phi_t, h, v, st))) return rc;
  double l = 0.0;
  if ((rc = n->read_loss(st, &l))) return rc;
  if (loss) *loss = l;
  if (grad_host) {
    PYRO_CU(cudaMemcpy(grad_host, n->grad.p, n->n_params * 4, cudaMemcpyDeviceToHost));
  }
  return PYRO_OK;
}

// One optimiser step on a batch: loss, gradients, Adam.  Asynchronous on
// the stream; pyro_net_last_loss waits for it and reads the loss.
int pyro_net_train_step(PyroNet* n, const float* b, const uint32_t* flags, const float* phi_t,
                        uint32_t nx, uint32_t ny, uint32_t nz, uint32_t nb, float h, float lr,
                        float clip, void* stream) {
  clear_error();
  PYRO_REQUIRE(n && b && flags && phi_t, "pyro_net_train_step: null argument");
  PYRO_REQUIRE(h > 0.0f && lr >= 0.0f, "pyro_net_train_step: invalid h or lr");
  int rc = check_vol(nx, ny, nz, nb);
  if (rc) return rc;
  NetVol v{(int)nx, (int)ny, (int)nz, (int)nb};
  cudaStream_t st = pick(n, stream);
  if ((rc = n->ensure(v, true)) || (rc = n->loss_backward(b, flags, phi_t, h, v, st)) ||
      (rc = n->adam(lr, clip, st)))
    return rc;
  return PYRO_OK;
}

int pyro_net_last_loss(PyroNet* n, double* loss, void* stream) {
  clear_error();
  PYRO_REQUIRE(n && loss, "pyro_net_last_loss: null argument");
  return n->read_loss(pick(n, stream), loss);
}

int pyro_net_set_loss(PyroNet* n, float w_phi, float w_res) {
  clear_error();
  PYRO_REQUIRE(n, "pyro_net_set_loss: null network");
  PYRO_REQUIRE(std::isfinite(w_phi) && std::isfinite(w_res) && w_phi >= 0.0f && w_res >= 0.0f &&
                   w_phi + w_res > 0.0f,
               "pyro_net_set_loss: weights must be >= 0 and not both 0");
  n->w_phi = w_phi;
  n->w_res = w_res;
  return PYRO_OK;
}

}  // extern "C"
