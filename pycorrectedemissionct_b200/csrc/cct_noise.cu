// Synthetic-data noise on the device: the photon scaling, absolute-Gaussian background,
// Poisson counts and Gaussian read-out noise of corrct's testing.add_noise
// (corrct: src/corrct/testing.py:266-320), for sinograms that are already in HBM.
//
// Random numbers are counter based, so every element's draws depend only on (seed, element
// index, draw number) and not on the launch shape:
//   Philox-4x32-10 (J. K. Salmon, M. A. Moraes, R. O. Dror, D. E. Shaw, "Parallel random
//   numbers: as easy as 1, 2, 3", SC 2011), keyed by the 64-bit seed, counter =
//   (element index lo, hi, draw number, stream tag);
//   normal deviates by the Box-Muller transform;
//   Poisson counts by multiplication of uniforms (Knuth) for lambda < 10 and by the transformed
//   rejection method PTRS (W. Hormann, "The transformed rejection method for generating Poisson
//   random variables", Insurance: Mathematics and Economics 12, 1993) for lambda >= 10.
// The streams differ from numpy's generator, so results agree with the reference in
// distribution, not draw for draw.

#include <cstdint>

#include "cct_common.cuh"
#include "corrct_b200.h"

namespace cct {

constexpr int NOISE_THREADS = 256;
constexpr int NOISE_BLOCKS = 148 * 4;  // fixed grid: the background partial sums have a fixed order

constexpr uint32_t STREAM_BACKGROUND = 1, STREAM_POISSON = 2, STREAM_READOUT = 3;

struct U4 {
  uint32_t x, y, z, w;
};

// Philox-4x32 round constants as published (multipliers and Weyl key increments).
__device__ __forceinline__ U4 philox4x32_10(U4 c, uint32_t k0, uint32_t k1) {
  constexpr uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
  constexpr uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    const uint32_t hi0 = __umulhi(M0, c.x), lo0 = M0 * c.x;
    const uint32_t hi1 = __umulhi(M1, c.z), lo1 = M1 * c.z;
    c = U4{hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0};
    k0 += W0;
    k1 += W1;
  }
  return c;
}

// Two uniform doubles in (0, 1) with 53 random bits each.
struct Draws {
  uint32_t k0, k1;
  uint64_t elem;
  uint32_t tag;
  uint32_t n = 0;
  __device__ __forceinline__ void next2(double& a, double& b) {
    const U4 r = philox4x32_10(U4{(uint32_t)elem, (uint32_t)(elem >> 32), n++, tag}, k0, k1);
    const uint64_t ua = ((uint64_t)(r.x >> 5) << 26) | (r.y >> 6);
    const uint64_t ub = ((uint64_t)(r.z >> 5) << 26) | (r.w >> 6);
    a = ((double)ua + 0.5) * 0x1.0p-53;
    b = ((double)ub + 0.5) * 0x1.0p-53;
  }
  __device__ __forceinline__ double normal() {
    double u1, u2;
    next2(u1, u2);
    return sqrt(-2.0 * log(u1)) * cospi(2.0 * u2);
  }
};

// Poisson(lambda) for finite lambda >= 0; *capped = 1 when the (practically unreachable)
// iteration bound ended the draw, which then returns the nearest integer to lambda.
__device__ double poisson_draw(Draws& g, double lam, int* capped) {
  if (lam <= 0.0) return 0.0;
  if (lam < 10.0) {
    const double limit = exp(-lam);
    double prod = 1.0;
    for (int k = 0; k < 1024; k += 2) {
      double u1, u2;
      g.next2(u1, u2);
      prod *= u1;
      if (prod <= limit) return (double)k;
      prod *= u2;
      if (prod <= limit) return (double)(k + 1);
    }
    *capped = 1;
    return rint(lam);
  }
  const double slam = sqrt(lam), loglam = log(lam);
  const double b = 0.931 + 2.53 * slam;
  const double a = -0.059 + 0.02483 * b;
  const double inv_alpha = 1.1239 + 1.1328 / (b - 3.4);
  const double vr = 0.9277 - 3.6224 / (b - 2.0);
  for (int it = 0; it < 256; ++it) {
    double u, v;
    g.next2(u, v);
    u -= 0.5;
    const double us = 0.5 - fabs(u);
    const double k = floor((2.0 * a / us + b) * u + lam + 0.43);
    if (us >= 0.07 && v <= vr) return k;
    if (k < 0.0 || (us < 0.013 && v > us)) continue;
    if (log(v) + log(inv_alpha) - log(a / (us * us) + b) <= -lam + k * loglam - lgamma(k + 1.0)) return k;
  }
  *capped = 1;
  return rint(lam);
}

struct NoiseArgs {
  const float* clean;
  float* noisy;
  float* clean_scaled;
  int64_t count;
  float scale_f;   // (float)(num_photons * efficiency): the reference multiplies a float32 array by it
  double scale_d;  // num_photons * efficiency in double, for the float64 background term
  double bg_avg, bg_std, readout_std;
  uint32_t k0, k1;
  int add_poisson, has_background, has_readout;
  double* partials;
  int* flags;  // [0] invalid (negative or NaN) Poisson means, [1] capped draws
};

__global__ void __launch_bounds__(NOISE_THREADS) add_noise_kernel(NoiseArgs p) {
  __shared__ double red[NOISE_THREADS / 32];
  double bg_sum = 0.0;
  int invalid = 0, capped = 0;
  for (int64_t i = (int64_t)blockIdx.x * NOISE_THREADS + threadIdx.x; i < p.count;
       i += (int64_t)NOISE_BLOCKS * NOISE_THREADS) {
    const float c = p.clean[i] * p.scale_f;  // img_clean = photons * efficiency * img (float32)
    float v = c;
    if (p.has_background) {
      Draws g{p.k0, p.k1, (uint64_t)i, STREAM_BACKGROUND};
      const double e = p.bg_avg + p.bg_std * g.normal();
      v = (float)((double)v + p.scale_d * fabs(e));  // float32 += float64 array
    }
    bg_sum += (double)(v - c);  // background = mean(img_noise - img_clean), before the Poisson draw
    if (p.add_poisson) {
      if (!(v >= 0.f) || !((double)v < 9.2e18)) {  // numpy rejects negative, NaN and huge means
        invalid = 1;
        v = __int_as_float(0x7fc00000);  // NaN marks elements whose mean was invalid
      } else {
        Draws g{p.k0, p.k1, (uint64_t)i, STREAM_POISSON};
        v = (float)poisson_draw(g, (double)v, &capped);
      }
    }
    if (p.has_readout) {
      Draws g{p.k0, p.k1, (uint64_t)i, STREAM_READOUT};
      v = (float)((double)v + p.readout_std * g.normal());
    }
    p.noisy[i] = v;
    if (p.clean_scaled != nullptr) p.clean_scaled[i] = c;
  }
  bg_sum = warp_sum_double(bg_sum);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = bg_sum;
  if (invalid) atomicOr(&p.flags[0], 1);
  if (capped) atomicOr(&p.flags[1], 1);
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < NOISE_THREADS / 32; ++w) t += red[w];
    p.partials[blockIdx.x] = t;
  }
}

__global__ void noise_mean_kernel(const double* partials, int64_t count, double* background) {
  __shared__ double red[NOISE_THREADS / 32];
  double t = 0.0;
  for (int k = threadIdx.x; k < NOISE_BLOCKS; k += NOISE_THREADS) t += partials[k];
  t = warp_sum_double(t);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = t;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < NOISE_THREADS / 32; ++w) s += red[w];
    *background = s / (double)count;
  }
}

}  // namespace cct

extern "C" {

int cct_noise_partials_count(int64_t* count) {
  CCT_REQUIRE(count != nullptr, "count is required");
  *count = cct::NOISE_BLOCKS;
  return CCT_OK;
}

int cct_add_noise(const cct_noise_desc* desc, const float* clean, int64_t count, float* noisy, float* clean_scaled,
                  double* partials, double* background, int32_t* flags, void* stream) {
  CCT_REQUIRE(desc != nullptr, "noise descriptor is NULL");
  CCT_REQUIRE(clean != nullptr && noisy != nullptr && partials != nullptr && background != nullptr &&
                  flags != nullptr,
              "clean, noisy, partials, background and flags are required");
  CCT_REQUIRE(count >= 1, "count must be >= 1");
  CCT_REQUIRE(!desc->has_readout || desc->readout_std >= 0.0, "readout_std must be >= 0");
  CCT_REQUIRE(!desc->has_background || desc->background_std >= 0.0, "background_std must be >= 0");
  cct::NoiseArgs p;
  p.clean = clean;
  p.noisy = noisy;
  p.clean_scaled = clean_scaled;
  p.count = count;
  p.scale_d = desc->num_photons * desc->detection_efficiency;
  p.scale_f = (float)p.scale_d;
  p.bg_avg = desc->background_avg;
  p.bg_std = desc->background_std;
  p.readout_std = desc->readout_std;
  p.k0 = (uint32_t)desc->seed;
  p.k1 = (uint32_t)(desc->seed >> 32);
  p.add_poisson = desc->add_poisson;
  p.has_background = desc->has_background;
  p.has_readout = desc->has_readout;
  p.partials = partials;
  p.flags = flags;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  cct::add_noise_kernel<<<cct::NOISE_BLOCKS, cct::NOISE_THREADS, 0, s>>>(p);
  cct::noise_mean_kernel<<<1, cct::NOISE_THREADS, 0, s>>>(partials, count, background);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    cct_set_last_error(cudaGetErrorString(e));
    return CCT_ERR_CUDA;
  }
  return CCT_OK;
}

}  // extern "C"
