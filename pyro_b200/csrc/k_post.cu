// k_post.cu — frame development on the GPU: the reference's `post` module
// (src/post.rs:25-160), which runs on the CPU there, for the path tracer's
// accumulated image.
//
//   mean + keys   accum (r, g, b sums, samples) -> mean radiance per pixel
//                 (sums / max(samples, 1)) and each pixel's luminance
//                 (post.rs:31-33) as an order-preserving 32-bit key
//   select        the k-th smallest luminance by a 4-pass radix select
//                 (8 bits per pass, device-side bin choice) -- the exact
//                 value np.partition / the reference's sort picks
//   scale         linear = mean * 2^exposure
//   box_h, box_v  the glare's box filters with the reference's running sums
//                 (post.rs:109-160): one thread per row (column) and channel
//                 keeps the sum, so every sum is formed in the same order as
//                 on the CPU
//   final         glare mix, ACES fit, sRGB, dither and 8-bit quantisation
//                 (post.rs:47-88)
//
// FP32 in the reference's expression order (the library is built without
// fused multiply-add contraction): everything up to the sRGB curve is bit
// for bit the CPU restatement; powf in the sRGB curve may differ from the
// host's in the last place, which can move an 8-bit value by one.
#include <algorithm>
#include <cstring>

#include "common.cuh"
#include "kernels.h"

namespace pyro {

namespace {

// float -> unsigned key with the same order (negative values reversed)
__device__ __forceinline__ uint32_t fkey(float v) {
  const uint32_t u = __float_as_uint(v);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

__global__ void __launch_bounds__(256) k_post_mean(const float4* __restrict__ acc,
                                                   float* __restrict__ img,
                                                   uint32_t* __restrict__ keys, int n) {
  const int i = blockIdx.x * 256 + threadIdx.x;
  if (i >= n) return;
  const float4 a = acc[i];
  const float s = fmaxf(a.w, 1.0f);
  const float r = a.x / s, g = a.y / s, b = a.z / s;
  img[3 * i] = r;
  img[3 * i + 1] = g;
  img[3 * i + 2] = b;
  keys[i] = fkey(0.2126f * r + 0.7152f * g + 0.0722f * b);
}

// Radix-select state (POST_SEL_WORDS words): [0] prefix, [1] mask, [2] rank
// still to skip, [3] the selected key (after the last pass), [4..260) the
// histogram of the pass.
constexpr int SEL_HIST = 4;

__global__ void k_sel_init(uint32_t* __restrict__ sel, uint32_t rank) {
  for (int t = threadIdx.x; t < POST_SEL_WORDS; t += blockDim.x) sel[t] = t == 2 ? rank : 0u;
}

__global__ void __launch_bounds__(256) k_sel_hist(const uint32_t* __restrict__ keys, int n,
                                                  uint32_t* __restrict__ sel, int shift) {
  __shared__ uint32_t h[256];
  h[threadIdx.x] = 0;
  __syncthreads();
  const uint32_t prefix = sel[0], mask = sel[1];
  for (int i = blockIdx.x * 256 + threadIdx.x; i < n; i += gridDim.x * 256) {
    const uint32_t k = keys[i];
    if ((k & mask) == prefix) atomicAdd(&h[(k >> shift) & 255u], 1u);
  }
  __syncthreads();
  if (h[threadIdx.x]) atomicAdd(&sel[SEL_HIST + threadIdx.x], h[threadIdx.x]);
}

// One block of 256 threads: the bin holding the rank, by an inclusive scan
// of the 256 counts.
__global__ void __launch_bounds__(256) k_sel_pick(uint32_t* __restrict__ sel, int shift) {
  __shared__ uint32_t c[256];
  const int t = threadIdx.x;
  const uint32_t mine = sel[SEL_HIST + t];
  c[t] = mine;
  __syncthreads();
  for (int o = 1; o < 256; o <<= 1) {
    const uint32_t v = t >= o ? c[t - o] : 0u;
    __syncthreads();
    c[t] += v;
    __syncthreads();
  }
  const uint32_t rank = sel[2];
  const uint32_t below = c[t] - mine;  // keys of this prefix in lower bins
  __syncthreads();
  if (below <= rank && rank < c[t]) {
    sel[0] |= (uint32_t)t << shift;
    sel[1] |= 255u << shift;
    sel[2] = rank - below;
    if (shift == 0) sel[3] = sel[0];
  }
  sel[SEL_HIST + t] = 0u;
}

__global__ void __launch_bounds__(256) k_post_scale(const float* __restrict__ img, float gain,
                                                    float* __restrict__ lin, int n3) {
  const int i = blockIdx.x * 256 + threadIdx.x;
  if (i < n3) lin[i] = img[i] * gain;
}

// Box filter of radius r along x, clamp to edge (post.rs:109-133): thread
// (row, channel) runs the row's sum.
__global__ void __launch_bounds__(128) k_box_h(const float* __restrict__ b, float* __restrict__ out,
                                               int w, int h, int r) {
  const int t = blockIdx.x * 128 + threadIdx.x;
  if (t >= 3 * h) return;
  const int y = t / 3, c = t - 3 * y;
  const float* row = b + (size_t)y * w * 3 + c;
  float* o = out + (size_t)y * w * 3 + c;
  const float norm = 1.0f / (float)(2 * r + 1);
  float acc = 0.0f;
  const int m = min(r, w - 1);
  for (int i = 0; i <= m; i++) acc = acc + row[3 * i];
  acc = acc + row[0] * (float)r;
  for (int x = 0; x < w; x++) {
    o[3 * x] = acc * norm;
    acc = acc + (row[3 * min(x + r + 1, w - 1)] - row[3 * max(x - r, 0)]);
  }
}

// Along y (post.rs:135-160): thread (column, channel).
__global__ void __launch_bounds__(128) k_box_v(const float* __restrict__ b, float* __restrict__ out,
                                               int w, int h, int r) {
  const int t = blockIdx.x * 128 + threadIdx.x;
  if (t >= 3 * w) return;
  const size_t stride = (size_t)w * 3;
  const float* col = b + t;
  float* o = out + t;
  const float norm = 1.0f / (float)(2 * r + 1);
  float acc = 0.0f;
  const int m = min(r, h - 1);
  for (int i = 0; i <= m; i++) acc = acc + col[i * stride];
  acc = acc + col[0] * (float)r;
  for (int y = 0; y < h; y++) {
    o[y * stride] = acc * norm;
    acc = acc + (col[min(y + r + 1, h - 1) * stride] - col[max(y - r, 0) * stride]);
  }
}

// g = g + b * weight (the glare's sum over scales, post.rs:100-104)
__global__ void __launch_bounds__(256) k_post_axpy(const float* __restrict__ b, float wt,
                                                   float* __restrict__ g, int n3) {
  const int i = blockIdx.x * 256 + threadIdx.x;
  if (i < n3) g[i] = g[i] + b[i] * wt;
}

__device__ __forceinline__ float aces(float x) {
  x = x * 0.6f;
  const float num = x * (2.51f * x + 0.03f);
  const float den = x * (2.43f * x + 0.59f) + 0.14f;
  return fminf(fmaxf(num / den, 0.0f), 1.0f);
}
__device__ __forceinline__ float srgb(float x) {
  return x <= 0.0031308f ? 12.92f * x : 1.055f * powf(x, 1.0f / 2.4f) - 0.055f;
}
// PCG hash of the pixel index to [0, 1) with 24 bits (post.rs:83-88)
__device__ __forceinline__ float hash01(uint32_t v) {
  uint32_t x = v * 747796405u + 2891336453u;
  x = ((x >> ((x >> 28u) + 4u)) ^ x) * 277803737u;
  x = (x >> 22u) ^ x;
  return (float)(x >> 8u) / 16777216.0f;
}

__global__ void __launch_bounds__(256) k_post_final(const float* __restrict__ lin,
                                                    const float* __restrict__ gl, float glare,
                                                    uint8_t* __restrict__ out,
                                                    float* __restrict__ lin_out, int n) {
  const int p = blockIdx.x * 256 + threadIdx.x;
  if (p >= n) return;
  const float dith = (hash01((uint32_t)p) - 0.5f) / 255.0f;
#pragma unroll
  for (int c = 0; c < 3; c++) {
    float v = lin[3 * p + c];
    if (glare > 0.0f) v = v * (1.0f - glare) + gl[3 * p + c] * glare;
    if (lin_out) lin_out[3 * p + c] = v;
    const float s = srgb(aces(v)) + dith;
    out[3 * p + c] = (uint8_t)(fminf(fmaxf(s, 0.0f), 1.0f) * 255.0f + 0.5f);
  }
}

inline unsigned blocks(long n, int t) { return (unsigned)((n + t - 1) / t); }

}  // namespace

cudaError_t launch_post_select(const float* accum, int n, int k, float* img, uint32_t* keys,
                               uint32_t* sel, cudaStream_t st) {
  k_post_mean<<<blocks(n, 256), 256, 0, st>>>(reinterpret_cast<const float4*>(accum), img, keys,
                                               n);
  k_sel_init<<<1, 256, 0, st>>>(sel, (uint32_t)k);
  const unsigned hb = std::min(blocks(n, 256), 1184u);
  for (int shift = 24; shift >= 0; shift -= 8) {
    k_sel_hist<<<hb, 256, 0, st>>>(keys, n, sel, shift);
    k_sel_pick<<<1, 256, 0, st>>>(sel, shift);
  }
  return cudaGetLastError();
}

float post_key_value(uint32_t key) {
  const uint32_t u = (key & 0x80000000u) ? (key & 0x7FFFFFFFu) : ~key;
  float v;
  std::memcpy(&v, &u, 4);
  return v;
}

cudaError_t launch_post_develop(const float* img, int w, int h, float gain, float glare,
                                float* scratch, uint8_t* out, float* lin_out, cudaStream_t st) {
  const long n = (long)w * h, n3 = 3 * n;
  float* lin = scratch;
  float* t1 = scratch + n3;
  float* t2 = scratch + 2 * n3;
  float* gl = scratch + 3 * n3;
  k_post_scale<<<blocks(n3, 256), 256, 0, st>>>(img, gain, lin, (int)n3);
  if (glare > 0.0f) {
    cudaError_t e = cudaMemsetAsync(gl, 0, n3 * 4, st);
    if (e != cudaSuccess) return e;
    // (radius as a fraction of the width, weight), post.rs:93
    const float scales[3][2] = {{0.003f, 0.5f}, {0.012f, 0.3f}, {0.04f, 0.2f}};
    for (const auto& sw : scales) {
      const int rad = std::max((int)(sw[0] * (float)w), 1);
      const float* src = lin;
      for (int it = 0; it < 3; it++) {
        k_box_h<<<blocks(3L * h, 128), 128, 0, st>>>(src, t1, w, h, rad);
        k_box_v<<<blocks(3L * w, 128), 128, 0, st>>>(t1, t2, w, h, rad);
        src = t2;
      }
      k_post_axpy<<<blocks(n3, 256), 256, 0, st>>>(t2, sw[1], gl, (int)n3);
    }
  }
  k_post_final<<<blocks(n, 256), 256, 0, st>>>(lin, gl, glare, out, lin_out, (int)n);
  return cudaGetLastError();
}

}  // namespace pyro
