// Turn-by-turn diagnostics on the GPU: the peak-DFT tune finder
// (FineTuneFinder, simtrack.cpp:2288-2319 and 2321-2352) for many signals at
// once, and the early-turn feature vector of the loss-prediction surrogate.
//
// fine_tune_kernel: one CTA per signal.  The samples are staged in shared
// memory; each refinement level lays its tune grid out exactly as the
// reference's serial loop produces it (tune = lower, then repeated
// `tune + step` while below `upper`), evaluates the DFT power of every grid
// tune in parallel (one thread per tune, the sum over samples in the
// reference's order), and picks the first strict maximum, so the level
// sequence and the final tune follow the reference's search step by step.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>

#include "stb_tune.hpp"

namespace stb {
namespace {

constexpr int kTuneBlock = 128;
constexpr double kRefPi = 3.14159265358979323;  // PI, simtrack.cpp:23

template <bool kPx>
__global__ void __launch_bounds__(kTuneBlock) fine_tune_kernel(const __grid_constant__ FineTuneArgs a) {
  extern __shared__ __align__(16) double sm[];
  double *xs = sm;
  double *ps = sm + a.n;
  double *grid = sm + (kPx ? 2 : 1) * a.n;
  double *amp = grid + kMaxTuneGrid;
  __shared__ int m_s;
  __shared__ double peak_s;
  const int tid = threadIdx.x;
  const double c2pi = -2.0 * kRefPi;
  for (long sig = blockIdx.x; sig < a.nsig; sig += gridDim.x) {
    for (int i = tid; i < a.n; i += kTuneBlock) {
      xs[i] = a.x[(long)i * a.stride + sig];
      if (kPx) ps[i] = a.px[(long)i * a.stride + sig];
    }
    double lo = a.lo, hi = a.hi, step = 0.001, peak = lo;
    do {
      if (tid == 0) {
        int m = 0;
        double t = lo;
        do {
          grid[m++] = t;
          t = t + step;
        } while (t < hi && m < kMaxTuneGrid);
        m_s = m;
      }
      __syncthreads();
      const int m = m_s;
      for (int k = tid; k < m; k += kTuneBlock) {
        const double f = grid[k];
        double sr = 0.0, si = 0.0;
        for (int i = 0; i < a.n; i++) {
          double s, c;
          sincos(c2pi * (double)i * f, &s, &c);
          if (kPx) {
            sr = sr + xs[i] * c - ps[i] * s;
            si = si + xs[i] * s + ps[i] * c;
          } else {
            sr = sr + xs[i] * c;
            si = si + xs[i] * s;
          }
        }
        amp[k] = sr * sr + si * si;
      }
      __syncthreads();
      if (tid == 0) {
        double p = lo, pa = 0.0;
        for (int k = 0; k < m; k++)
          if (amp[k] > pa) {
            p = grid[k];
            pa = amp[k];
          }
        peak_s = p;
      }
      __syncthreads();
      peak = peak_s;
      lo = peak - step;
      hi = peak + step;
      step = step / 10.;
    } while (step > 1.0e-12);
    if (tid == 0) a.tune[sig] = peak;
    __syncthreads();
  }
}

// Normalised action (x_hat^2 + p_hat^2) / 2 with x_hat = x / sqrt(beta),
// p_hat = (alpha x + beta px) / sqrt(beta).
__device__ __forceinline__ double action(double x, double px, double beta, double alpha) {
  const double pn = alpha * x + beta * px;
  return 0.5 * (x * x + pn * pn) / beta;
}

__global__ void features_kernel(const __grid_constant__ FeatureArgs a) {
  const long N = a.ntot;
  for (long p = (long)blockIdx.x * blockDim.x + threadIdx.x; p < N; p += (long)gridDim.x * blockDim.x) {
    const double bx = a.twiss[0], ax = a.twiss[1], by = a.twiss[2], ay = a.twiss[3];
    const double ex = a.twiss[4], ey = a.twiss[5];  // geometric emittances: actions in units of emit
    const double jx0 = action(a.x0[p], a.x0[N + p], bx, ax);
    const double jy0 = action(a.x0[2 * N + p], a.x0[3 * N + p], by, ay);
    const double ampx = sqrt(2.0 * jx0 / ex), ampy = sqrt(2.0 * jy0 / ey);
    double jmax = 0.0, jmin = 1e300;
    for (int t = 0; t < a.nturn; t++) {
      const double *r = a.tbt + (size_t)t * 4 * N + p;
      const double j = action(r[0], r[N], bx, ax) / ex + action(r[2 * N], r[3 * N], by, ay) / ey;
      jmax = fmax(jmax, j);
      jmin = fmin(jmin, j);
    }
    const double j0 = jx0 / ex + jy0 / ey;
    const double qx1 = a.tunes[p], qy1 = a.tunes[N + p], qx2 = a.tunes[2 * N + p], qy2 = a.tunes[3 * N + p];
    float *o = a.out + p * kNumFeatures;
    o[0] = (float)ampx;
    o[1] = (float)ampy;
    o[2] = (float)(a.x0[5 * N + p] * 1e3);
    o[3] = (float)atan2(ampy, ampx);
    o[4] = (float)qx1;
    o[5] = (float)qy1;
    o[6] = (float)qx2;
    o[7] = (float)qy2;
    o[8] = (float)log10(fabs(qx1 - qx2) + 1e-10);
    o[9] = (float)log10(fabs(qy1 - qy2) + 1e-10);
    o[10] = (float)log10((jmax - jmin) / (j0 + 0.5) + 1e-8);
    o[11] = (float)sqrt(2.0 * jmax);
  }
}

}  // namespace

size_t fine_tune_smem_bytes(int n, bool with_px) {
  return (size_t)(with_px ? 2 : 1) * n * sizeof(double) + (size_t)2 * kMaxTuneGrid * sizeof(double);
}

cudaError_t launch_fine_tune(const FineTuneArgs &a, int num_sms, cudaStream_t st) {
  const bool px = a.px != nullptr;
  const size_t smem = fine_tune_smem_bytes(a.n, px);
  auto kern = px ? fine_tune_kernel<true> : fine_tune_kernel<false>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kTuneBlock, smem);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) return cudaErrorInvalidConfiguration;
  long grid = (long)num_sms * per_sm;
  if (grid > a.nsig) grid = a.nsig;
  kern<<<(unsigned)grid, kTuneBlock, smem, st>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_features(const FeatureArgs &a, cudaStream_t st) {
  long grid = (a.ntot + 255) / 256;
  if (grid > 65535) grid = 65535;
  features_kernel<<<(unsigned)grid, 256, 0, st>>>(a);
  return cudaGetLastError();
}

}  // namespace stb
