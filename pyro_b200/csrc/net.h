// net.h — the learned pressure stage: a 3-level 3D convolutional
// encoder-decoder (16/32/64 channels, 3x3x3 convolutions, BF16 weights and
// activations, FP32 accumulation in TMEM) that maps a right-hand side and the
// solid mask to a pressure estimate, with its training (MSE loss, backward
// pass, Adam on FP32 master weights).
//
//   in0 = [b / s, solid]                      level 0, 2 channels
//   e0a = relu(conv1(in0))   e0 = relu(conv2(e0a))          16
//   p1  = avgpool2(e0)       e1a = relu(conv3(p1)), e1 = relu(conv4(e1a))  32
//   p2  = avgpool2(e1)       e2a = relu(conv5(p2)), e2 = relu(conv6(e2a))  64
//   c1  = [up2(e2), e1]      d1  = relu(conv7(c1))          96 -> 32
//   c0  = [up2(d1), e0]      d0  = relu(conv8(c0))          48 -> 16
//   out = conv9(d0)                                         16 -> 1 (FP32)
//   phi = out * out_scale * s * h^2 on fluid cells, 0 in solids
//
// s is the root mean square of b over the fluid cells of each volume, so
// the map is linear in the scale of b, as the Poisson solution is.  Pooling
// halves with ceil (a coarse cell averages its children inside the volume);
// up2 copies a coarse cell to its children.  Activations of C channels are
// stored as C / 8 planes of [volume][z][y][x][8 channels] (C a multiple of
// 8), the 2-channel input as [volume][z][y][x][2].
#pragma once

#include <cuda_bf16.h>

#include "runtime.h"

namespace pyro {

cudaError_t conv3_forward(const __nv_bfloat16* x, int C, int nx, int ny, int nz, int nb,
                          const __nv_bfloat16* w, int Cout, const float* bias, int relu,
                          __nv_bfloat16* y_bf16, float* y_f32, int* err, cudaStream_t st);
cudaError_t conv3_backward_data(const __nv_bfloat16* dy, int Cout, int nx, int ny, int nz,
                                int nb, const __nv_bfloat16* w, int Cin,
                                const __nv_bfloat16* act, __nv_bfloat16* dx_bf16, float* dx_f32,
                                int* err, cudaStream_t st);
cudaError_t conv3_backward_weight(const __nv_bfloat16* x, int Cin, const __nv_bfloat16* dy,
                                  int Cout, int nx, int ny, int nz, int nb, float* dw, int* err,
                                  cudaStream_t st);

// Direct convolution on the CUDA cores for 2 -> 16 and 16 -> 1 channels.
bool conv3_direct_fits(int C, int Cout);
cudaError_t conv3_direct(const __nv_bfloat16* x, int C, int nx, int ny, int nz, int nb,
                         const __nv_bfloat16* w, int Cout, const float* bias, int relu,
                         __nv_bfloat16* y_bf16, float* y_f32, cudaStream_t st);

// TMA-staged convolution (input channels K a multiple of 16) on tap-major
// weights prepared by conv3_prep_weights.
cudaError_t conv3_prep_weights(const __nv_bfloat16* w, int Cout, int Cin, int backward,
                               __nv_bfloat16* w_tap, cudaStream_t st);
cudaError_t conv3_tma(const __nv_bfloat16* x, int K, int nx, int ny, int nz, int nb,
                      const __nv_bfloat16* w_tap, int N, const float* bias, int relu,
                      const __nv_bfloat16* mask, __nv_bfloat16* y_bf16, float* y_f32, int* err,
                      cudaStream_t st);

constexpr int NET_LAYERS = 9;
struct NetLayer {
  int cin, cout, level, relu;
};
// conv1 .. conv9 in order
constexpr NetLayer NET_SPEC[NET_LAYERS] = {{2, 16, 0, 1},  {16, 16, 0, 1}, {16, 32, 1, 1},
                                           {32, 32, 1, 1}, {32, 64, 2, 1}, {64, 64, 2, 1},
                                           {96, 32, 1, 1}, {48, 16, 0, 1}, {16, 1, 0, 0}};

struct NetVol {
  int nx, ny, nz, nb;
  size_t voxels() const { return (size_t)nx * ny * nz * nb; }
  NetVol half() const { return NetVol{(nx + 1) / 2, (ny + 1) / 2, (nz + 1) / 2, nb}; }
  bool operator==(const NetVol& o) const {
    return nx == o.nx && ny == o.ny && nz == o.nz && nb == o.nb;
  }
};

}  // namespace pyro

// Parameters: all weights first ([Cout][27][Cin] per layer, layers in
// order), then all biases; the BF16 weight copy mirrors the weight part.
struct PyroNet {
  size_t w_off[pyro::NET_LAYERS + 1] = {};  // into the weight part
  size_t b_off[pyro::NET_LAYERS + 1] = {};  // into the bias part (after weights)
  size_t n_w = 0, n_params = 0;
  float out_scale = 1.0f;
  float w_phi = 1.0f, w_res = 0.0f;  // loss weights (pyro_net_set_loss)
  pyro::DevBuf master, grad, adam_m, adam_v, wbf;  // FP32 x n_params; BF16 x n_w
  pyro::DevBuf wtf, wtb;  // tap-major BF16 weights for the forward / backward-data TMA path
  pyro::DevBuf scal;   // FP64 device scalars: [0] loss, [1] grad sum of squares, then 2 per volume
  pyro::DevBuf err;    // tensor-core wait error flag
  double* host_scal = nullptr;
  long adam_t = 0;
  // activation buffers for the current volume shape
  pyro::NetVol vol{0, 0, 0, 0};
  bool has_bwd = false;
  pyro::DevBuf in0, e0a, p1, e1a, p2, e2a, e2, c1, d1, c0, d0, out, res;
  // skip activations e0 (16 channels, level 0) and e1 (32, level 1): the
  // last 2 / 4 planes of the concatenations c0 / c1
  __nv_bfloat16* skip0() const { return c0.as<__nv_bfloat16>() + (size_t)4 * vol.voxels() * 8; }
  __nv_bfloat16* skip1() const {
    return c1.as<__nv_bfloat16>() + (size_t)8 * vol.half().voxels() * 8;
  }
  pyro::DevBuf g9, g8, gc0, g7, gc1, g6, g5, gp2, g4, g3, gp1, g2, g1;
  cudaStream_t stream = nullptr;

  int init();
  ~PyroNet();
  int ensure(pyro::NetVol v, bool bwd);
  const float* bias(int l) const { return master.as<float>() + n_w + b_off[l]; }
  const __nv_bfloat16* w(int l) const { return wbf.as<__nv_bfloat16>() + w_off[l]; }
  const __nv_bfloat16* wf(int l) const { return wtf.as<__nv_bfloat16>() + w_off[l]; }
  const __nv_bfloat16* wb(int l) const { return wtb.as<__nv_bfloat16>() + w_off[l]; }
  // rebuild wtf / wtb from the BF16 weights
  int refresh_taps(cudaStream_t st);
  // Forward pass; out holds the network output (FP32, per voxel).
  int forward(const float* b, const uint32_t* flags, pyro::NetVol v, cudaStream_t st);
  // Loss (weights w_phi, w_res; see pyro_net_set_loss) and the full
  // backward pass; gradients are accumulated into `grad` (zeroed here).
  int loss_backward(const float* b, const uint32_t* flags, const float* phi_t, float h,
                    pyro::NetVol v, cudaStream_t st);
  int adam(float lr, float clip, cudaStream_t st);
  // phi = out * out_scale * s * h^2 (fluid), 0 (solid)
  int output(const uint32_t* flags, float h, float* phi, pyro::NetVol v, cudaStream_t st);
  int check_err(cudaStream_t st);
  // loss of the last loss_backward from the device scalars (synchronises)
  int read_loss(cudaStream_t st, double* loss);
};
