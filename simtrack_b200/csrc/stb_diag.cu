// Diagnostics: evaluation of the kernels' elementary functions on the GPU or
// on the host, for accuracy tests against the host C library.
#include <cuda_runtime.h>

#include <vector>

#include "stb_crmath.cuh"
#include "stb_kernels.hpp"
#include "stb_physics.cuh"
#include "stb_rng.cuh"

namespace stb {

namespace {

__host__ __device__ inline double eval_fn(int fn, const double *in, long i) {
  switch (fn) {
    case 0: return cr_asin(in[i]);
    case 1: return cr_exp(in[i]);
    case 2: return cr_sin(in[i]);
    case 3: return cr_cos(in[i]);
    case 4: return cr_pown(in[2 * i], (int)in[2 * i + 1]);
#ifdef __CUDA_ARCH__
    case 5: return qdiv(in[2 * i], in[2 * i + 1], 1.0 / in[2 * i + 1]);
#else
    case 5: return in[2 * i] / in[2 * i + 1];
#endif
    case 10: return asin(in[i]);
    case 11: return exp(in[i]);
    case 12: return sin(in[i]);
    case 13: return cos(in[i]);
    case 14: return pow(in[2 * i], in[2 * i + 1]);
    case 15: return in[2 * i] / in[2 * i + 1];
    default: return 0.0;
  }
}

__global__ void math_eval_kernel(int fn, const double *in, double *out, long n) {
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    out[i] = eval_fn(fn, in, i);
}

// FP64 FMA throughput probe: 8 independent FMA chains per thread, `iters`
// rounds, result folded into one store so nothing is dead code.
__global__ void dfma_peak_kernel(double *out, int iters, double a, double b) {
  double v0 = threadIdx.x * 1e-9, v1 = v0 + 1e-3, v2 = v0 + 2e-3, v3 = v0 + 3e-3;
  double v4 = v0 + 4e-3, v5 = v0 + 5e-3, v6 = v0 + 6e-3, v7 = v0 + 7e-3;
  for (int i = 0; i < iters; i++) {
    v0 = fma(v0, a, b); v1 = fma(v1, a, b); v2 = fma(v2, a, b); v3 = fma(v3, a, b);
    v4 = fma(v4, a, b); v5 = fma(v5, a, b); v6 = fma(v6, a, b); v7 = fma(v7, a, b);
  }
  const double s = ((v0 + v1) + (v2 + v3)) + ((v4 + v5) + (v6 + v7));
  if (s == 12345.678) out[blockIdx.x] = s;
}

// splitmix64: the i-th draw of a seeded stream, the same on host and device.
__host__ __device__ inline uint64_t mix64(uint64_t z) {
  z += 0x9e3779b97f4a7c15ull;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}
__host__ __device__ inline double unif(uint64_t seed, uint64_t i, int k) {
  return (double)(mix64(seed ^ (i * 8 + (uint64_t)k) * 0x2545f4914f6cdd1dull) >> 11) * (1.0 / 9007199254740992.0);
}

// Random drift arguments (a proton beam at gamma 106.6: pt up to 2e-3, slopes
// up to 7e-3 with a logarithmic spread down to 7e-7 and every 64th sample up
// to 0.05, lengths 0.01-6 m) and the number of drift quotients
// (drift_quotients) that differ from the IEEE results: pz, 1/pz, betaz,
// L/betaz.
__host__ __device__ inline void drift_check_one(uint64_t seed, uint64_t i, unsigned long long *bad) {
  const double beta = 0.99995598, gamma = 106.58, sg = sqrt(gamma * gamma - 1.);
  const double pt = (2 * unif(seed, i, 0) - 1) * 2e-3 * pow(10.0, -3 * unif(seed, i, 1));
  const double smax = (i % 64 == 63) ? 0.05 : kSeedSlope2;
  const double px = (2 * unif(seed, i, 2) - 1) * smax * pow(10.0, -4 * unif(seed, i, 3));
  const double py = (2 * unif(seed, i, 4) - 1) * smax * pow(10.0, -4 * unif(seed, i, 5));
  const double L = 0.01 + 6 * unif(seed, i, 6);
  const double delta1 = sqrt(1.0 + 2 * pt / beta + pt * pt) - 1.0;
  const double gamma1 = gamma + sg * pt;
  const double beta1 = sqrt(1.0 - 1.0 / gamma1 / gamma1);
  const double opd = 1.0 + delta1, opd2 = opd * opd, iopd = 1.0 / opd, ibeta1 = 1.0 / beta1;
  double pz, ipz, betaz, lb;
  drift_quotients(opd, opd2, beta1, iopd, mul_rn(opd, ibeta1), px, py, L, pz, ipz, betaz, lb);
  const double rpz = sqrt(opd2 - px * px - py * py);
  const double ripz = 1.0 / rpz;
  const double rbetaz = mul_rn(rpz, beta1) / opd;
  const double rlb = L / rbetaz;
  if (pz != rpz) bad[0]++;
  if (ipz != ripz) bad[1]++;
  if (betaz != rbetaz) bad[2]++;
  if (lb != rlb) bad[3]++;
}

__global__ void drift_check_kernel(uint64_t seed, long n, unsigned long long *bad) {
  unsigned long long loc[4] = {0, 0, 0, 0};
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    drift_check_one(seed, (uint64_t)i, loc);
  for (int k = 0; k < 4; k++)
    if (loc[k]) atomicAdd(bad + k, loc[k]);
}

// Random sin/cos arguments: log-uniform magnitudes in [2^-40, 800]; uniform
// in [-pi, pi] (spin rotation angles); uniform in [-pi/256, pi/256] (the
// table's first interval); and multiples k pi/128 (|k| <= 32000) offset by a
// log-uniform amount in [2^-40, 2^-6] (small reduced arguments).  Counts:
// sin and cos of the fast path that differ from the double-double series,
// arguments the fast path leaves to the series among the first three
// classes, and among the last.
__host__ __device__ inline void sincos_check_one(uint64_t seed, uint64_t i, unsigned long long *cnt) {
  const double u = unif(seed, i, 0), sgn = unif(seed, i, 1) < 0.5 ? -1.0 : 1.0;
  double x;
  int cls;
  if (u < 0.4) {
    x = sgn * exp2(-40.0 + (40.0 + 9.64) * unif(seed, i, 2));
    cls = 0;
  } else if (u < 0.7) {
    x = sgn * 3.141592653589793 * unif(seed, i, 2);
    cls = 0;
  } else if (u < 0.8) {
    x = sgn * 0.01227184630308513 * unif(seed, i, 2);
    cls = 0;
  } else {
    const double k = floor(32001.0 * unif(seed, i, 2));
    x = sgn * (k * 0.02454369260617026 + exp2(-40.0 + 34.0 * unif(seed, i, 3)) * (unif(seed, i, 4) - 0.5));
    cls = 1;
  }
  if (!(fabs(x) < 800.0)) x = 799.0 * sgn;
  double fs, fc, ss, sc;
  cr_sincos_series(x, ss, sc);
  if (sincos_fast(x, fs, fc)) {
    if (fs != ss) cnt[0]++;
    if (fc != sc) cnt[1]++;
  } else {
    cnt[2 + cls]++;
  }
}

__global__ void sincos_check_kernel(uint64_t seed, long n, unsigned long long *cnt) {
  unsigned long long loc[4] = {0, 0, 0, 0};
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    sincos_check_one(seed, (uint64_t)i, loc);
  for (int k = 0; k < 4; k++)
    if (loc[k]) atomicAdd(cnt + k, loc[k]);
}

template <class One>
cudaError_t run_check(long n, unsigned long long seed, int device, unsigned long long *cnt4, One one,
                      void (*kern)(uint64_t, long, unsigned long long *)) {
  for (int k = 0; k < 4; k++) cnt4[k] = 0;
  if (device < 0) {
    for (long i = 0; i < n; i++) one(seed, (uint64_t)i, cnt4);
    return cudaSuccess;
  }
  unsigned long long *d = nullptr;
  cudaError_t e = cudaMalloc(&d, 4 * sizeof(unsigned long long));
  if (e != cudaSuccess) return e;
  cudaMemset(d, 0, 4 * sizeof(unsigned long long));
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  kern<<<sms * 8, 256>>>(seed, n, d);
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpy(cnt4, d, 4 * sizeof(unsigned long long), cudaMemcpyDeviceToHost);
  cudaFree(d);
  return e;
}

__global__ void rad_normals_kernel(uint64_t seed, uint64_t id, uint64_t k0, long n, double *out) {
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    out[i] = rad_gaussian(seed, id, k0 + (uint64_t)i);
}

}  // namespace

// Deviates k0 .. k0+n-1 of particle `id`'s quantum-excitation stream, on
// `device` (out in device memory) or on the host (device < 0).
cudaError_t rad_normals(unsigned long long seed, unsigned long long id, unsigned long long k0, long n, double *out,
                        int device) {
  if (device < 0) {
    for (long i = 0; i < n; i++) out[i] = rad_gaussian(seed, id, k0 + (uint64_t)i);
    return cudaSuccess;
  }
  if (n <= 0) return cudaSuccess;
  long grid = (n + 255) / 256;
  if (grid > 4096) grid = 4096;
  rad_normals_kernel<<<(unsigned)grid, 256>>>(seed, id, k0, n, out);
  return cudaGetLastError();
}

void philox_block(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
  const Philox4 r = philox4x32_10(Philox4{{ctr[0], ctr[1], ctr[2], ctr[3]}}, key[0], key[1]);
  for (int i = 0; i < 4; i++) out[i] = r.v[i];
}

// Fast sin/cos path against the double-double series over n random
// arguments, on `device` (or the host for device < 0); counts as in
// sincos_check_one.
cudaError_t sincos_fast_check(long n, unsigned long long seed, int device, unsigned long long *cnt4) {
  return run_check(n, seed, device, cnt4, [](uint64_t s, uint64_t i, unsigned long long *c) { sincos_check_one(s, i, c); },
                   sincos_check_kernel);
}

// Mismatch counts of the drift quotients against IEEE sqrt and division over
// n random drift arguments, on `device` (or the host for device < 0).
cudaError_t drift_quotient_check(long n, unsigned long long seed, int device, unsigned long long *bad4) {
  return run_check(n, seed, device, bad4, [](uint64_t s, uint64_t i, unsigned long long *c) { drift_check_one(s, i, c); },
                   drift_check_kernel);
}

// Measured FP64 FMA peak of `device` in TFLOP/s (2 flops per FMA).
cudaError_t fp64_peak_probe(int device, double *tflops) {
  int sms = 0;
  cudaError_t e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  if (e != cudaSuccess) return e;
  double *d = nullptr;
  const int blocks = sms * 8, threads = 256, iters = 1 << 15;
  e = cudaMalloc(&d, sizeof(double) * blocks);
  if (e != cudaSuccess) return e;
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  dfma_peak_kernel<<<blocks, threads>>>(d, 1024, 0.999999, 1e-7);  // warm-up
  float best = 1e30f;
  for (int r = 0; r < 3; r++) {
    cudaEventRecord(a);
    dfma_peak_kernel<<<blocks, threads>>>(d, iters, 0.999999, 1e-7);
    cudaEventRecord(b);
    cudaEventSynchronize(b);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    if (ms < best) best = ms;
  }
  e = cudaGetLastError();
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaFree(d);
  *tflops = 2.0 * 8.0 * (double)iters * blocks * threads / (best * 1e-3) / 1e12;
  return e;
}

int math_input_arity(int fn) { return (fn == 4 || fn == 5 || fn == 14 || fn == 15) ? 2 : 1; }

bool math_fn_valid(int fn) { return (fn >= 0 && fn <= 5) || (fn >= 10 && fn <= 15); }

cudaError_t math_eval_device(int fn, const double *d_in, double *d_out, long n, cudaStream_t s) {
  const int block = 256;
  long grid = (n + block - 1) / block;
  if (grid > 65535) grid = 65535;
  if (grid < 1) grid = 1;
  math_eval_kernel<<<(unsigned)grid, block, 0, s>>>(fn, d_in, d_out, n);
  return cudaGetLastError();
}

void math_eval_host(int fn, const double *in, double *out, long n) {
  for (long i = 0; i < n; i++) out[i] = eval_fn(fn, in, i);
}

}  // namespace stb
