// k_voxel.cu — scene voxelizer on the GPU (Scene::voxelize,
// src/scene.rs:621-667, shape tests :695-728).  One thread per cell tests
// every shape in order; the last shape containing the cell centre wins.  The
// reference runs this as a CPU triple loop over cells x shapes.
#include "common.cuh"
#include "kernels.h"

namespace pyro {

namespace {

// src/scene.rs:662-667 (the PCG hash of common.wgsl:54-58) as a float.
__device__ __forceinline__ float hash01(uint32_t v) {
  uint32_t x = v * 747796405u + 2891336453u;
  x = ((x >> ((x >> 28) + 4u)) ^ x) * 277803737u;
  x = (x >> 22) ^ x;
  return __uint2float_rn(x) / 4294967296.0f;
}

__device__ __forceinline__ bool inside(const PyroShape& s, float px, float py, float pz,
                                       float dx) {
  switch (s.kind) {
    case PYRO_SHAPE_BOX: {
      float d0 = px - s.c[0], d1 = py - s.c[1], d2 = pz - s.c[2];
      float lx = s.cos_yaw * d0 + s.sin_yaw * d2;
      float lz = -s.sin_yaw * d0 + s.cos_yaw * d2;
      float h0 = fmaxf(s.e[0], 0.5f * dx), h1 = fmaxf(s.e[1], 0.5f * dx),
            h2 = fmaxf(s.e[2], 0.5f * dx);
      return fabsf(lx) <= h0 && fabsf(d1) <= h1 && fabsf(lz) <= h2;
    }
    case PYRO_SHAPE_CYL: {
      float ba0 = s.e[0] - s.c[0], ba1 = s.e[1] - s.c[1], ba2 = s.e[2] - s.c[2];
      float pa0 = px - s.c[0], pa1 = py - s.c[1], pa2 = pz - s.c[2];
      float l2 = ba0 * ba0 + ba1 * ba1 + ba2 * ba2;
      float t = (pa0 * ba0 + pa1 * ba1 + pa2 * ba2) / l2;
      if (!(t >= 0.0f && t <= 1.0f)) return false;
      float q0 = pa0 - ba0 * t, q1 = pa1 - ba1 * t, q2 = pa2 - ba2 * t;
      return sqrtf(q0 * q0 + q1 * q1 + q2 * q2) <= fmaxf(s.r, 0.5f * dx);
    }
    case PYRO_SHAPE_SPHERE: {
      float d0 = px - s.c[0], d1 = py - s.c[1], d2 = pz - s.c[2];
      return sqrtf(d0 * d0 + d1 * d1 + d2 * d2) <= s.r;
    }
    case PYRO_SHAPE_POOL: {
      float a = px - s.c[0], b = pz - s.c[2];
      return sqrtf(a * a + b * b) <= s.r && py <= fmaxf(s.depth, dx * 0.99f);
    }
    default:
      return false;
  }
}

__global__ void __launch_bounds__(256) k_voxelize(const PyroShape* __restrict__ shapes,
                                                  uint32_t n, int nx, int ny, int nz, float dx,
                                                  float t0, uint32_t seed,
                                                  const float* __restrict__ dens,
                                                  const uint32_t* __restrict__ kind,
                                                  float4* __restrict__ sol) {
  int i = blockIdx.x * 32 + threadIdx.x;
  int j = blockIdx.y * 4 + threadIdx.y;
  int k = blockIdx.z * 2 + threadIdx.z;
  if (i >= nx || j >= ny || k >= nz) return;
  uint32_t idx = (uint32_t)i + (uint32_t)nx * ((uint32_t)j + (uint32_t)ny * (uint32_t)k);
  float px = ((float)i + 0.5f) * dx, py = ((float)j + 0.5f) * dx, pz = ((float)k + 0.5f) * dx;
  float4 v = make_float4(0.0f, 0.0f, 0.0f, t0);
  for (uint32_t s = 0; s < n; s++) {
    if (inside(shapes[s], px, py, pz, dx)) {
      uint32_t slot = min(shapes[s].slot, 7u);
      float h = hash01(idx ^ (seed * 0x9e3779b9u));
      float jit = 0.85f + 0.3f * h;
      float mass = kind[slot] == 2u ? 1.0f : dens[slot] * jit;
      v = make_float4((float)slot, mass, 0.0f, t0);
    }
  }
  sol[idx] = v;
}

}  // namespace

cudaError_t launch_voxelize(const PyroShape* shapes_dev, uint32_t n, Dims3 d, float dx, float t0,
                            uint32_t seed, const float* dens_dev, const uint32_t* kind_dev,
                            float4* sol, cudaStream_t st) {
  dim3 grid((d.nx + 31) / 32, (d.ny + 3) / 4, (d.nz + 1) / 2);
  k_voxelize<<<grid, dim3(32, 4, 2), 0, st>>>(shapes_dev, n, d.nx, d.ny, d.nz, dx, t0, seed,
                                             dens_dev, kind_dev, sol);
  return cudaGetLastError();
}

}  // namespace pyro
