// Device-side generation of the initial fields: particle shapes phi and the
// composition noise c0 (the inputs of core_shell.jl:27-37, plus the shape set of
// the historical 2-D program restated in physical coordinates).
//
// Coordinates follow core_shell.jl:29: x = (i - n/2) dx for column i (the
// contiguous index), y = (j - n/2) dx for row j; element (i, j) of a field sits
// at j*n + i.  Every profile is S(r, R) = (1 - tanh((r - R)/w)) / 2.
//
// Noise: SplitMix64 of (seed, element index) gives a uniform u in [0, 1) with 53
// bits, and c = mean + amplitude (2u - 1).  With a particle field the noise is
// applied where phi >= 0.5 and its mean over those points is removed
// (core_shell.jl:31-35); the reduction is a fixed-order two-level sum.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>

#include "esc.h"

extern void esc_set_thread_error(const char* msg);

namespace {

__device__ __forceinline__ double profile(double r, double R, double w) { return 0.5 * (1.0 - tanh((r - R) / w)); }

__global__ void k_particle(int shape, int n, double dx, double p0, double p1, double p2, double w, double* phi) {
  const size_t total = (size_t)n * n;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < total; k += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(k % n), j = (int)(k / n);
    const double x = (double)(i - n / 2) * dx, y = (double)(j - n / 2) * dx;
    const double r = sqrt(x * x + y * y);
    double v = 0.0;
    switch (shape) {
      case ESC_SHAPE_DISC:
        v = profile(r, p0, w);
        break;
      case ESC_SHAPE_BAND:  // between y = p0 and y = p1
        v = 0.5 * (tanh((y - p0) / w) - tanh((y - p1) / w));
        break;
      case ESC_SHAPE_ELLIPSE: {  // semi-axes p0 along x, p1 along y
        const double re = sqrt((x * p1 / p0) * (x * p1 / p0) + y * y);
        v = profile(re, p1, w);
        break;
      }
      case ESC_SHAPE_ANNULUS:  // radii p0 < p1
        v = profile(r, p1, w) - profile(r, p0, w);
        break;
      case ESC_SHAPE_SQUIRCLE: {  // (x^4 + y^4)^(1/4) = p0
        const double r4 = sqrt(sqrt(x * x * x * x + y * y * y * y));
        v = profile(r4, p0, w);
        break;
      }
      case ESC_SHAPE_ELLIPTIC_SHELL: {  // ellipse (p0 along x, p1 along y) with a circular hole of radius p2
        const double re = sqrt((x * p1 / p0) * (x * p1 / p0) + y * y);
        v = profile(re, p1, w) - profile(r, p2, w);
        break;
      }
      case ESC_SHAPE_ELLIPTIC_HOLE: {  // disc of radius p0 with an elliptical hole (p1 along x, p2 along y)
        const double re = sqrt((x * p2 / p1) * (x * p2 / p1) + y * y);
        v = profile(r, p0, w) - profile(re, p2, w);
        break;
      }
      default:
        break;
    }
    phi[k] = v;
  }
}

__device__ __forceinline__ double splitmix_uniform(uint64_t seed, uint64_t idx) {
  uint64_t z = seed + (idx + 1) * 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z ^= z >> 31;
  return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

constexpr int kBlocks = 256, kThreads = 256;

// per-block sum of the noise over the interior points and their count
__global__ void k_noise_partials(int n, const double* phi, double amp, uint64_t seed, double* part) {
  __shared__ double s_sum[kThreads];
  __shared__ double s_cnt[kThreads];
  const size_t total = (size_t)n * n;
  double sum = 0.0, cnt = 0.0;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < total; k += (size_t)gridDim.x * blockDim.x) {
    if (phi[k] >= 0.5) {
      sum += amp * (2.0 * splitmix_uniform(seed, k) - 1.0);
      cnt += 1.0;
    }
  }
  s_sum[threadIdx.x] = sum;
  s_cnt[threadIdx.x] = cnt;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) {
      s_sum[threadIdx.x] += s_sum[threadIdx.x + o];
      s_cnt[threadIdx.x] += s_cnt[threadIdx.x + o];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = s_sum[0];
    part[2 * blockIdx.x + 1] = s_cnt[0];
  }
}

// fixed-order fold of the block partials into the interior mean (part[2 * nparts])
__global__ void k_noise_fold(const double* part, int nparts, double* shift) {
  double sum = 0.0, cnt = 0.0;
  for (int b = 0; b < nparts; ++b) {
    sum += part[2 * b];
    cnt += part[2 * b + 1];
  }
  *shift = cnt > 0.0 ? sum / cnt : 0.0;
}

__global__ void k_noise_write(int n, const double* phi, double mean, double amp, uint64_t seed,
                              const double* shift_p, double* c) {
  const double shift = phi ? *shift_p : 0.0;
  const size_t total = (size_t)n * n;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < total; k += (size_t)gridDim.x * blockDim.x) {
    const double e = amp * (2.0 * splitmix_uniform(seed, k) - 1.0);
    if (!phi)
      c[k] = mean + e;
    else
      c[k] = phi[k] >= 0.5 ? mean + (e - shift) : mean;
  }
}

esc_status cuda_status(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return ESC_OK;
  static thread_local char buf[256];
  snprintf(buf, sizeof buf, "%s: %s", what, cudaGetErrorString(e));
  esc_set_thread_error(buf);
  return e == cudaErrorMemoryAllocation ? ESC_ENOMEM : ESC_ECUDA;
}

}  // namespace

extern "C" {

esc_status esc_particle_device(int shape, int n, double dx, const double* params, double width, double* phi,
                               void* stream) {
  if (n < 2 || !params || !phi || !(dx > 0.0) || !(width > 0.0) || shape < ESC_SHAPE_DISC ||
      shape > ESC_SHAPE_ELLIPTIC_HOLE) {
    esc_set_thread_error("esc_particle_device: bad argument");
    return ESC_EINVAL;
  }
  for (int q = 0; q < 4; ++q)
    if (!isfinite(params[q])) {
      esc_set_thread_error("esc_particle_device: non-finite shape parameter");
      return ESC_EINVAL;
    }
  if ((shape == ESC_SHAPE_ELLIPSE || shape == ESC_SHAPE_ELLIPTIC_SHELL) && !(params[0] > 0.0)) {
    esc_set_thread_error("esc_particle_device: the ellipse's x semi-axis must be positive");
    return ESC_EINVAL;
  }
  if (shape == ESC_SHAPE_ELLIPTIC_HOLE && !(params[1] > 0.0)) {
    esc_set_thread_error("esc_particle_device: the hole's x semi-axis must be positive");
    return ESC_EINVAL;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  k_particle<<<kBlocks * 4, kThreads, 0, st>>>(shape, n, dx, params[0], params[1], params[2], width, phi);
  esc_status s = cuda_status(cudaGetLastError(), "esc_particle_device launch");
  if (s != ESC_OK) return s;
  return cuda_status(cudaStreamSynchronize(st), "esc_particle_device");
}

esc_status esc_noise_device(int n, const double* phi, double mean, double amplitude, uint64_t seed, double* c,
                            void* stream) {
  if (n < 2 || !c || !isfinite(mean) || !isfinite(amplitude)) {
    esc_set_thread_error("esc_noise_device: bad argument");
    return ESC_EINVAL;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  double* part = nullptr;
  esc_status s = ESC_OK;
  if (phi) {
    s = cuda_status(cudaMallocAsync(&part, (2 * kBlocks + 1) * sizeof(double), st), "esc_noise_device scratch");
    if (s != ESC_OK) return s;
    k_noise_partials<<<kBlocks, kThreads, 0, st>>>(n, phi, amplitude, seed, part);
    k_noise_fold<<<1, 1, 0, st>>>(part, kBlocks, part + 2 * kBlocks);
  }
  k_noise_write<<<kBlocks * 4, kThreads, 0, st>>>(n, phi, mean, amplitude, seed, part ? part + 2 * kBlocks : nullptr,
                                                  c);
  s = cuda_status(cudaGetLastError(), "esc_noise_device launch");
  if (part) cudaFreeAsync(part, st);
  if (s != ESC_OK) return s;
  return cuda_status(cudaStreamSynchronize(st), "esc_noise_device");
}

}  // extern "C"
