// Strong-strong beam-beam, soft-Gaussian 4D form: BeamBeam4D_SoftGaussian
// (simtrack.cpp:22846-22872) on the GPU.
//
// Two beams of macro-particles (AoS x[6n] in device memory) collide: each
// beam's transverse centroid and rms size (Cal_Mean_RMS, simtrack.cpp:
// 724-743: running sums of x, y, x^2, y^2 in particle order, mean = sum/N,
// rms = sqrt(sum2/N - mean^2)) define a Gaussian field that kicks every
// particle of the other beam through BB4D (6325-6377, the weak-strong map of
// the tracking kernels, bb4d in stb_physics.cuh).
//
// The moments are the reference's running sums in the reference's order:
// one CTA stages the particles in shared memory and one thread adds them one
// by one, so the sums round exactly as the reference's loop does (a tree
// reduction would round differently and the kicks would differ in the last
// bits).  That pass is a dependent chain of n additions; the kicks are one
// thread per particle.
#include <cuda_runtime.h>

#include <cstdint>

#include "stb_kernels.hpp"
#include "stb_physics.cuh"

namespace stb {
namespace {

// mean[0..1], rms[0..1] of x and y of n particles, AoS x[6 n].  The CTA
// stages kMomentChunk particles' x and y in shared memory; thread 0 adds them
// in particle order (the loads of the next chunk do not wait on its sums).
constexpr int kMomentBlock = 256, kMomentChunk = 2048;
__global__ void __launch_bounds__(kMomentBlock) soft_gaussian_moments_kernel(const double *x, long n, double *out4) {
  __shared__ double cx[kMomentChunk], cy[kMomentChunk];
  double sx = 0, sy = 0, sx2 = 0, sy2 = 0;
  for (long base = 0; base < n; base += kMomentChunk) {
    const int m = (int)(n - base < kMomentChunk ? n - base : kMomentChunk);
    for (int k = threadIdx.x; k < m; k += kMomentBlock) {
      cx[k] = x[6 * (base + k)];
      cy[k] = x[6 * (base + k) + 2];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll 8
      for (int j = 0; j < m; j++) {
        const double a = cx[j], b = cy[j];
        sx = sx + a;
        sy = sy + b;
        sx2 = sx2 + a * a;
        sy2 = sy2 + b * b;
      }
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const double N = (double)n;
    const double mx = sx / N, my = sy / N;
    out4[0] = mx;
    out4[1] = my;
    out4[2] = sqrt(sx2 / N - mx * mx);
    out4[3] = sqrt(sy2 / N - my * my);
  }
}

// Kick the n particles of one beam with the other beam's moments m4.
// c4 = 2 N_other rp / gamma (BB4D's constant prefix).
__global__ void soft_gaussian_kick_kernel(double *x, long n, const double *m4, double c4, double bbscale) {
  const double mx = m4[0], my = m4[1], sx = m4[2], sy = m4[3];
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    double *p = x + 6 * i;
    const double dx = p[0] - mx;
    const double dy = p[2] - my;
    double dpx, dpy;
    bb4d(dx, dy, c4, sx, sy, dpx, dpy);
    p[1] = p[1] + dpx * bbscale;
    p[3] = p[3] + dpy * bbscale;
  }
}

// Both beams' moments of the collision in flight (one collision at a time per
// device).
__device__ double g_soft_gaussian_moments[8];

}  // namespace

cudaError_t soft_gaussian_4d(double *x1, long n1, double *x2, long n2, double c4_1, double c4_2, double bbscale1,
                             double bbscale2, int num_sms, cudaStream_t s) {
  double *d_m8 = nullptr;
  cudaError_t e = cudaGetSymbolAddress((void **)&d_m8, g_soft_gaussian_moments);
  if (e != cudaSuccess) return e;
  soft_gaussian_moments_kernel<<<1, kMomentBlock, 0, s>>>(x1, n1, d_m8);
  soft_gaussian_moments_kernel<<<1, kMomentBlock, 0, s>>>(x2, n2, d_m8 + 4);
  const int block = 256;
  auto grid = [&](long n) {
    long g = (n + block - 1) / block;
    const long cap = (long)num_sms * 8;
    return (unsigned)(g < 1 ? 1 : g > cap ? cap : g);
  };
  if (n1 > 0) soft_gaussian_kick_kernel<<<grid(n1), block, 0, s>>>(x1, n1, d_m8 + 4, c4_1, bbscale1);
  if (n2 > 0) soft_gaussian_kick_kernel<<<grid(n2), block, 0, s>>>(x2, n2, d_m8, c4_2, bbscale2);
  return cudaGetLastError();
}

}  // namespace stb
