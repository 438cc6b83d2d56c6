// Turn-by-turn diagnostics: tune finder and surrogate feature kernels.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace stb {

constexpr int kMaxTuneGrid = 1024;  // tunes per refinement level (coarse level: <= 1002)
constexpr int kMaxTuneSamples = 4096;
constexpr int kNumFeatures = 12;

struct FineTuneArgs {
  const double *x;   // sample i of signal j at x[i * stride + j]
  const double *px;  // optional conjugate signal (same layout), NULL for the x-only form
  int n;
  long nsig;
  long stride;
  double lo, hi;
  double *tune;      // [nsig]
};

struct FeatureArgs {
  const double *tbt;    // [nturn][4][ntot]: x, px, y, py after each turn
  const double *x0;     // [6][ntot] initial coordinates
  const double *tunes;  // [4][ntot]: Qx (turns 0..n-1), Qy, Qx (second window), Qy
  long ntot;
  int nturn;
  double twiss[6];      // beta_x, alpha_x, beta_y, alpha_y, emit_x, emit_y at the record point
  float *out;           // [ntot][kNumFeatures]
};

size_t fine_tune_smem_bytes(int n, bool with_px);
cudaError_t launch_fine_tune(const FineTuneArgs &a, int num_sms, cudaStream_t st);
cudaError_t launch_features(const FeatureArgs &a, cudaStream_t st);

}  // namespace stb
