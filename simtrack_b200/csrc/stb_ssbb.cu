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
// a CTA per beam stages the particles in shared memory and one thread per
// sum adds them one by one, so the sums round exactly as the reference's
// loop does (a tree reduction would round differently and the kicks would
// differ in the last bits).  Each sum is a dependent chain of n additions;
// the kicks are one thread per particle.
#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "stb_kernels.hpp"
#include "stb_physics.cuh"

namespace stb {
namespace {

// mean[0..1], rms[0..1] of x and y of n particles, AoS x[6 n]; CTA b
// (0 or 1) takes beam b of the pair and writes out8[4b .. 4b+3].  The four
// running sums are independent chains: lane 0 of warps 0-3 each keeps one
// (sum x, sum y, sum x^2, sum y^2), adding the staged particles in order,
// while warps 4-7 stage the next kMomentChunk particles' x and y in the other
// shared-memory buffer.  Each chain is a dependent sequence of n additions,
// which no parallel split would round the same way.
constexpr int kMomentBlock = 256, kMomentChunk = 1024;
__global__ void __launch_bounds__(kMomentBlock) moments_pair_kernel(const double *xa, long na, const double *xb,
                                                                    long nb, double *out8) {
  __shared__ double cx[2][kMomentChunk], cy[2][kMomentChunk];
  __shared__ double sums[4];
  const double *x = blockIdx.x == 0 ? xa : xb;
  const long n = blockIdx.x == 0 ? na : nb;
  double *out4 = out8 + 4 * blockIdx.x;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  auto stage = [&](long base, int buf, int t0, int nt) {
    const int m = (int)(n - base < kMomentChunk ? n - base : kMomentChunk);
    for (int k = t0; k < m; k += nt) {
      cx[buf][k] = x[6 * (base + k)];
      cy[buf][k] = x[6 * (base + k) + 2];
    }
  };
  if (n > 0) stage(0, 0, threadIdx.x, kMomentBlock);
  __syncthreads();
  double acc = 0;
  for (long base = 0, c = 0; base < n; base += kMomentChunk, c++) {
    const int buf = (int)(c & 1);
    if (warp >= 4) {
      if (base + kMomentChunk < n) stage(base + kMomentChunk, buf ^ 1, threadIdx.x - 128, kMomentBlock - 128);
    } else if (lane == 0) {
      const int m = (int)(n - base < kMomentChunk ? n - base : kMomentChunk);
      const double *v = (warp & 1) ? cy[buf] : cx[buf];
      if (warp < 2) {
#pragma unroll 8
        for (int j = 0; j < m; j++) acc = acc + v[j];
      } else {
#pragma unroll 8
        for (int j = 0; j < m; j++) acc = acc + v[j] * v[j];
      }
    }
    __syncthreads();
  }
  if (warp < 4 && lane == 0) sums[warp] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    const double N = (double)n;
    const double mx = sums[0] / N, my = sums[1] / N;
    out4[0] = mx;
    out4[1] = my;
    out4[2] = sqrt(sums[2] / N - mx * mx);
    out4[3] = sqrt(sums[3] / N - my * my);
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

// Rank of particle i when the bunch is ordered by z, largest first (the
// order of BeamBeam6D_SoftGaussian's exchange sort, simtrack.cpp:22897-22916,
// for distinct z; equal z keep their input order): order[rank] = i.
constexpr int kRankBlock = 256;
__global__ void __launch_bounds__(kRankBlock) z_rank_kernel(const double *x, long n, int32_t *order) {
  __shared__ double zt[kRankBlock];
  const long i = (long)blockIdx.x * kRankBlock + threadIdx.x;
  const double zi = i < n ? x[6 * i + 4] : 0.0;
  long rank = 0;
  for (long t0 = 0; t0 < n; t0 += kRankBlock) {
    const long j = t0 + threadIdx.x;
    zt[threadIdx.x] = j < n ? x[6 * j + 4] : 0.0;
    __syncthreads();
    const int m = (int)(n - t0 < kRankBlock ? n - t0 : kRankBlock);
    for (int k = 0; k < m; k++) {
      const double zj = zt[k];
      rank += (zj > zi || (zj == zi && t0 + k < i)) ? 1 : 0;
    }
    __syncthreads();
  }
  if (i < n) order[rank] = (int32_t)i;
}

__global__ void gather_particles_kernel(const double *src, const int32_t *order, long n, double *dst) {
  for (long r = (long)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (long)gridDim.x * blockDim.x) {
    const long i = order[r];
    for (int k = 0; k < 6; k++) dst[6 * r + k] = src[6 * i + k];
  }
}

// Mean z of each slice of m consecutive particles (the reference's running
// sum, 22986-23004): one thread per slice.
__global__ void slice_mean_z_kernel(const double *x, int nslice, long m, double *z) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nslice) return;
  double t = 0;
  for (long j = (long)s * m; j < (long)(s + 1) * m; j++) t = t + x[6 * j + 4];
  z[s] = t / (double)m;
}

// Members of each z slice [zb[s+1], zb[s]) in particle order (one thread per
// slice, the reference's running sum of their z, 23172-23191): idx[s * cap
// + r] for r < cap, count[s] (beyond cap only counted).
__global__ void zb_slice_members_kernel(const double *x, long n, const double *zb, int nslice, long cap,
                                        int32_t *idx, long *count, double *zsum) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nslice) return;
  const double hi = zb[s], lo = zb[s + 1];
  double t = 0;
  long c = 0;
  for (long j = 0; j < n; j++) {
    const double z = x[6 * j + 4];
    if (z < hi && z >= lo) {
      t = t + z;
      if (c < cap) idx[(long)s * cap + c] = (int32_t)j;
      c++;
    }
  }
  count[s] = c;
  zsum[s] = t;
}

__global__ void gather_members_kernel(const double *x, const int32_t *idx, long m, double *xc) {
  for (long r = (long)blockIdx.x * blockDim.x + threadIdx.x; r < m; r += (long)gridDim.x * blockDim.x)
    for (int k = 0; k < 6; k++) xc[6 * r + k] = x[6 * (long)idx[r] + k];
}

__global__ void scatter_members_kernel(double *x, const int32_t *idx, long m, const double *xc) {
  for (long r = (long)blockIdx.x * blockDim.x + threadIdx.x; r < m; r += (long)gridDim.x * blockDim.x)
    for (int k = 0; k < 6; k++) x[6 * (long)idx[r] + k] = xc[6 * r + k];
}

// x += sign * px * S, y += sign * py * S over n particles (the drift to and
// from the slices' collision point, 23059-23066, 23096-23103).
__global__ void slice_drift_kernel(double *x, long n, double S, bool forward) {
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    double *p = x + 6 * i;
    if (forward) {
      p[0] = p[0] + p[1] * S;
      p[2] = p[2] + p[3] * S;
    } else {
      p[0] = p[0] - p[1] * S;
      p[2] = p[2] - p[3] * S;
    }
  }
}

// Lorentz_Transfer (simtrack.cpp:6790-6815): the boost of one particle to
// the head-on frame of a collision with half crossing angle theta; sn, cs,
// tn = sin, cos, tan(theta) as the reference forms them on the host.
__global__ void lorentz_boost_kernel(double *x, long n, double sn, double cs, double tn) {
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    double *q = x + 6 * i;
    const double x0 = q[0], px0 = q[1], y0 = q[2], py0 = q[3], z0 = q[4], pz0 = q[5];
    const double ps0 = sqrt((1 + pz0) * (1 + pz0) - px0 * px0 - py0 * py0);
    const double h0 = (1 + pz0) - ps0;
    const double px_s = (px0 - tn * h0) / cs;
    const double py_s = py0 / cs;
    const double pz_s = pz0 - tn * px0 + tn * tn * h0;
    const double ps_s = sqrt((1 + pz_s) * (1 + pz_s) - px_s * px_s - py_s * py_s);
    const double h_s = (1 + pz_s) - ps_s;
    q[0] = tn * z0 + (1 + (px_s / ps_s) * sn) * x0;
    q[1] = px_s;
    q[2] = y0 + sn * (py_s / ps_s) * x0;
    q[3] = py_s;
    q[4] = z0 / cs + (-h_s / ps_s) * sn * x0;
    q[5] = pz_s;
  }
}

}  // namespace

cudaError_t sort_bunch_by_z(double *x, long n, double *scratch, int32_t *order, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  z_rank_kernel<<<(unsigned)((n + kRankBlock - 1) / kRankBlock), kRankBlock, 0, s>>>(x, n, order);
  gather_particles_kernel<<<(unsigned)((n + 255) / 256 < 4096 ? (n + 255) / 256 : 4096), 256, 0, s>>>(x, order, n,
                                                                                                    scratch);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  return cudaMemcpyAsync(x, scratch, sizeof(double) * 6 * (size_t)n, cudaMemcpyDeviceToDevice, s);
}

cudaError_t slice_mean_z(const double *x, int nslice, long m, double *z, cudaStream_t s) {
  slice_mean_z_kernel<<<(nslice + 63) / 64, 64, 0, s>>>(x, nslice, m, z);
  return cudaGetLastError();
}

cudaError_t slice_pair_collision(double *x1, long m1, double *x2, long m2, double S, double c4_1, double c4_2,
                                 double bbscale1, double bbscale2, int num_sms, cudaStream_t s) {
  const unsigned g1 = (unsigned)((m1 + 255) / 256 < num_sms * 8 ? (m1 + 255) / 256 : num_sms * 8);
  const unsigned g2 = (unsigned)((m2 + 255) / 256 < num_sms * 8 ? (m2 + 255) / 256 : num_sms * 8);
  slice_drift_kernel<<<g1 < 1 ? 1 : g1, 256, 0, s>>>(x1, m1, S, true);
  slice_drift_kernel<<<g2 < 1 ? 1 : g2, 256, 0, s>>>(x2, m2, -S, true);
  cudaError_t e = soft_gaussian_4d(x1, m1, x2, m2, c4_1, c4_2, bbscale1, bbscale2, num_sms, s);
  if (e != cudaSuccess) return e;
  slice_drift_kernel<<<g1 < 1 ? 1 : g1, 256, 0, s>>>(x1, m1, S, false);
  slice_drift_kernel<<<g2 < 1 ? 1 : g2, 256, 0, s>>>(x2, m2, -S, false);
  return cudaGetLastError();
}

cudaError_t beam_pair_mean_rms(const double *x1, long n1, const double *x2, long n2, double *out8, cudaStream_t s) {
  moments_pair_kernel<<<2, kMomentBlock, 0, s>>>(x1, n1, x2, n2, out8);
  return cudaGetLastError();
}

cudaError_t soft_gaussian_4d(double *x1, long n1, double *x2, long n2, double c4_1, double c4_2, double bbscale1,
                             double bbscale2, int num_sms, cudaStream_t s) {
  double *d_m8 = nullptr;
  cudaError_t e = cudaGetSymbolAddress((void **)&d_m8, g_soft_gaussian_moments);
  if (e != cudaSuccess) return e;
  moments_pair_kernel<<<2, kMomentBlock, 0, s>>>(x1, n1, x2, n2, d_m8);
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

// BeamBeam6D_SoftGaussian (simtrack.cpp:22874-23132) on device AoS bunches:
// both bunches ordered by z (largest first) in place; each cut into Nslice
// slices of Mp/Nslice consecutive particles (the remainder is not
// collided); slice pairs (i, j) taken in increasing order of
// -(Z1[i] + Z2[j])/2 by the reference's own exchange sort; for each pair
// both slices drift to the collision point (S = (Z1[i] - Z2[j])/2), kick
// each other as soft Gaussians (strength N/Nslice) and drift back.  The
// reference also writes its slice centroids to ./bunch1_Z.dat and
// ./bunch2_Z.dat on every call; nothing is written here.
namespace {
// The sliced 6D collision of BeamBeam6D_SoftGaussian (simtrack.cpp:
// 22874-23132) and BeamBeam6D_PIC (23380-23615), which differ only in the
// collision of a slice pair: both bunches sorted by z (largest first), cut
// into Nslice slices of Mp/Nslice consecutive particles, the slice pairs put
// in the reference's collision order, and `collide(slice1, m1, slice2, m2,
// S)` called for each pair in that order.
template <class Collide>
cudaError_t sliced_6d(long Mp1, double *x1, long Mp2, double *x2, int Nslice1, int Nslice2, cudaStream_t s,
                      Collide collide) {
  const long nmax = Mp1 > Mp2 ? Mp1 : Mp2;
  double *scratch = nullptr;
  cudaError_t e = cudaMalloc(&scratch, sizeof(double) * (6 * (size_t)nmax + (size_t)Nslice1 + (size_t)Nslice2) +
                                           sizeof(int32_t) * (size_t)nmax);
  if (e != cudaSuccess) return e;
  double *dz = scratch + 6 * nmax;
  int32_t *order = reinterpret_cast<int32_t *>(dz + Nslice1 + Nslice2);
  const long m1 = Mp1 / Nslice1, m2 = Mp2 / Nslice2;
  std::vector<double> Z1(Nslice1), Z2(Nslice2);
  if ((e = sort_bunch_by_z(x1, Mp1, scratch, order, s)) == cudaSuccess &&
      (e = sort_bunch_by_z(x2, Mp2, scratch, order, s)) == cudaSuccess &&
      (e = slice_mean_z(x1, Nslice1, m1, dz, s)) == cudaSuccess &&
      (e = slice_mean_z(x2, Nslice2, m2, dz + Nslice1, s)) == cudaSuccess &&
      (e = cudaMemcpyAsync(Z1.data(), dz, sizeof(double) * Nslice1, cudaMemcpyDeviceToHost, s)) == cudaSuccess &&
      (e = cudaMemcpyAsync(Z2.data(), dz + Nslice1, sizeof(double) * Nslice2, cudaMemcpyDeviceToHost, s)) ==
          cudaSuccess &&
      (e = cudaStreamSynchronize(s)) == cudaSuccess) {
    // collision order, simtrack.cpp:23022-23042 (the same exchange sort)
    const int np = Nslice1 * Nslice2;
    std::vector<int> I1(np), I2(np);
    std::vector<double> S(np), Z10(np);
    for (int i = 0; i < Nslice1; i++)
      for (int j = 0; j < Nslice2; j++) {
        I1[i * Nslice2 + j] = i;
        I2[i * Nslice2 + j] = j;
        S[i * Nslice2 + j] = (Z1[i] - Z2[j]) / 2.;
        Z10[i * Nslice2 + j] = -(Z1[i] + Z2[j]) / 2.;
      }
    for (int i = 0; i < np; i++)
      for (int j = i + 1; j < np; j++)
        if (Z10[j] < Z10[i]) {
          std::swap(Z10[i], Z10[j]);
          std::swap(S[i], S[j]);
          std::swap(I1[i], I1[j]);
          std::swap(I2[i], I2[j]);
        }
    for (int i = 0; i < np && e == cudaSuccess; i++)
      e = collide(x1 + 6 * (long)I1[i] * m1, m1, x2 + 6 * (long)I2[i] * m2, m2, S[i]);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  }
  cudaFree(scratch);
  return e;
}
}  // namespace

cudaError_t soft_gaussian_6d(double Np1, long Mp1, double *x1, double Np2, long Mp2, double *x2, double gamma1,
                             double gamma2, double bbscale1, double bbscale2, int Nslice1, int Nslice2, int num_sms,
                             cudaStream_t s) {
  const double rp = 1.53469826769e-18;  // BB4D, simtrack.cpp:6328
  const double N2s = Np2 / Nslice2, N1s = Np1 / Nslice1;
  const double c4_1 = 2 * N2s * rp / gamma1, c4_2 = 2 * N1s * rp / gamma2;
  return sliced_6d(Mp1, x1, Mp2, x2, Nslice1, Nslice2, s, [&](double *a, long m1, double *b, long m2, double S) {
    return slice_pair_collision(a, m1, b, m2, S, c4_1, c4_2, bbscale1, bbscale2, num_sms, s);
  });
}

// BeamBeam6D_PIC (simtrack.cpp:23380-23615): each slice pair drifts to its
// collision point, collides as BeamBeam4D_PIC with N/Nslice, drifts back.
// The reference also writes every bunch and slice to ./bunch*.dat files on
// each call; this build writes nothing.
cudaError_t pic_6d(double Np1, long Mp1, double *x1, double Np2, long Mp2, double *x2, double gamma1, double gamma2,
                   double bbscale1, double bbscale2, int Nslice1, int Nslice2, int num_sms, cudaStream_t s) {
  return sliced_6d(Mp1, x1, Mp2, x2, Nslice1, Nslice2, s, [&](double *a, long m1, double *b, long m2, double S) {
    const unsigned g1 = (unsigned)((m1 + 255) / 256 < num_sms * 8 ? (m1 + 255) / 256 : num_sms * 8);
    const unsigned g2 = (unsigned)((m2 + 255) / 256 < num_sms * 8 ? (m2 + 255) / 256 : num_sms * 8);
    slice_drift_kernel<<<g1 < 1 ? 1 : g1, 256, 0, s>>>(a, m1, S, true);
    slice_drift_kernel<<<g2 < 1 ? 1 : g2, 256, 0, s>>>(b, m2, -S, true);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess)
      e = pic_4d(Np1 / Nslice1, m1, a, Np2 / Nslice2, m2, b, gamma1, gamma2, bbscale1, bbscale2, num_sms, s);
    if (e != cudaSuccess) return e;
    slice_drift_kernel<<<g1 < 1 ? 1 : g1, 256, 0, s>>>(a, m1, S, false);
    slice_drift_kernel<<<g2 < 1 ? 1 : g2, 256, 0, s>>>(b, m2, -S, false);
    return cudaGetLastError();
  });
}

// Lumi_Cal_PIC_6D (simtrack.cpp:23703-23944): the sliced driver above; for
// each slice pair in collision order, drifted to its collision point, the
// luminosity of Lumi_Cal_PIC_4D with N/Nslice is added to the running sum,
// then the pair collides as soft Gaussians (BB4D with N/Nslice and the
// other slice's moments) and drifts back.  The reference also writes the
// collision order to ./collide_order.dat; this build writes nothing.
cudaError_t lumi_pic_6d(double Np1, long Mp1, double *x1, double Np2, long Mp2, double *x2, double gamma1,
                        double gamma2, double bbscale1, double bbscale2, int Nslice1, int Nslice2, int Ncoll,
                        double freq, int num_sms, cudaStream_t s, double *lumi_out) {
  const double rp = 1.53469826769e-18;  // BB4D, simtrack.cpp:6328
  const double N2s = Np2 / Nslice2, N1s = Np1 / Nslice1;
  const double c4_1 = 2 * N2s * rp / gamma1, c4_2 = 2 * N1s * rp / gamma2;
  double lumi = 0;
  const cudaError_t e =
      sliced_6d(Mp1, x1, Mp2, x2, Nslice1, Nslice2, s, [&](double *a, long m1, double *b, long m2, double S) {
        const unsigned g1 = (unsigned)((m1 + 255) / 256 < num_sms * 8 ? (m1 + 255) / 256 : num_sms * 8);
        const unsigned g2 = (unsigned)((m2 + 255) / 256 < num_sms * 8 ? (m2 + 255) / 256 : num_sms * 8);
        slice_drift_kernel<<<g1 < 1 ? 1 : g1, 256, 0, s>>>(a, m1, S, true);
        slice_drift_kernel<<<g2 < 1 ? 1 : g2, 256, 0, s>>>(b, m2, -S, true);
        cudaError_t r = cudaGetLastError();
        double l = 0;
        if (r == cudaSuccess) r = lumi_pic_4d(N1s, m1, N2s, m2, a, b, Ncoll, freq, num_sms, s, &l);
        if (r != cudaSuccess) return r;
        lumi = lumi + l;
        if ((r = soft_gaussian_4d(a, m1, b, m2, c4_1, c4_2, bbscale1, bbscale2, num_sms, s)) != cudaSuccess) return r;
        slice_drift_kernel<<<g1 < 1 ? 1 : g1, 256, 0, s>>>(a, m1, S, false);
        slice_drift_kernel<<<g2 < 1 ? 1 : g2, 256, 0, s>>>(b, m2, -S, false);
        return cudaGetLastError();
      });
  if (e == cudaSuccess) *lumi_out = lumi;
  return e;
}

// Lumi_Cal_PIC_6D_Angle (simtrack.cpp:23946-24224): every particle of
// both bunches boosted to the head-on frame (Lorentz_Transfer; the bunches
// stay boosted, as in the reference), then Lumi_Cal_PIC_6D.  The reference's
// bunch, slice and collision-order files are not written.
cudaError_t lumi_pic_6d_angle(double Np1, long Mp1, double *x1, double Np2, long Mp2, double *x2, double theta,
                              double gamma1, double gamma2, double bbscale1, double bbscale2, int Nslice1,
                              int Nslice2, int Ncoll, double freq, int num_sms, cudaStream_t s, double *lumi_out) {
  // sin(theta), cos(theta) (correctly rounded) and their quotient, as
  // Lorentz_Transfer forms them (its second cos(theta) is the same value)
  const double sn = cr_sin(theta), cs = cr_cos(theta), tn = sn / cs;
  const unsigned cap = (unsigned)num_sms * 8;
  for (int b = 0; b < 2; b++) {
    const long n = b == 0 ? Mp1 : Mp2;
    const unsigned g = (unsigned)((n + 255) / 256 < cap ? (n + 255) / 256 : cap);
    if (n > 0) lorentz_boost_kernel<<<g < 1 ? 1 : g, 256, 0, s>>>(b == 0 ? x1 : x2, n, sn, cs, tn);
  }
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  return lumi_pic_6d(Np1, Mp1, x1, Np2, Mp2, x2, gamma1, gamma2, bbscale1, bbscale2, Nslice1, Nslice2, Ncoll, freq,
                     num_sms, s, lumi_out);
}

// BeamBeam6D_SoftGaussian with slice boundaries (simtrack.cpp:23134-23283):
// slice s of a bunch holds its particles with zb[s+1] <= z < zb[s], in
// place (no reordering); slice centroids from the running sums of z over
// the members; the slice pairs in the same collision order as above; each
// pair's members are gathered in particle order, drift, collide as the 4D
// soft-Gaussian form with N scaled by the slice's share of the bunch
// (Np Mp_coll / Mp), drift back and are scattered to their places.  The
// reference copies each slice into a buffer of 2 Mp/Nslice particles and
// initialises its per-slice counters for Nslice1 entries of both bunches, so
// it is defined only for Nslice1 == Nslice2 and slices of at most that
// size, and a slice of fewer than two particles has no rms size: all are
// checked before any particle moves.  Returns cudaErrorInvalidValue when a
// slice is too full or too thin.
namespace {
template <class Collide>
cudaError_t sliced_6d_zb(double Np1, long Mp1, double *x1, double Np2, long Mp2, double *x2, int nslice,
                         const double *zb1, const double *zb2, int num_sms, cudaStream_t s, Collide collide) {
  const long cap1 = 2 * Mp1 / nslice, cap2 = 2 * Mp2 / nslice;
  const size_t nidx = (size_t)nslice * (size_t)(cap1 + cap2);
  const size_t bytes = sizeof(double) * (6 * (size_t)(cap1 + cap2) + 2 * (size_t)(nslice + 1) + 2 * (size_t)nslice) +
                       sizeof(long) * 2 * (size_t)nslice + sizeof(int32_t) * nidx;
  unsigned char *buf = nullptr;
  cudaError_t e = cudaMalloc(&buf, bytes);
  if (e != cudaSuccess) return e;
  double *xc1 = reinterpret_cast<double *>(buf), *xc2 = xc1 + 6 * cap1;
  double *dzb1 = xc2 + 6 * cap2, *dzb2 = dzb1 + (nslice + 1);
  double *zs = dzb2 + (nslice + 1);
  long *cnt = reinterpret_cast<long *>(zs + 2 * nslice);
  int32_t *idx1 = reinterpret_cast<int32_t *>(cnt + 2 * nslice), *idx2 = idx1 + (size_t)nslice * cap1;
  std::vector<long> c(2 * nslice);
  std::vector<double> z(2 * nslice);
  if ((e = cudaMemcpyAsync(dzb1, zb1, sizeof(double) * (nslice + 1), cudaMemcpyHostToDevice, s)) == cudaSuccess &&
      (e = cudaMemcpyAsync(dzb2, zb2, sizeof(double) * (nslice + 1), cudaMemcpyHostToDevice, s)) == cudaSuccess) {
    zb_slice_members_kernel<<<(nslice + 63) / 64, 64, 0, s>>>(x1, Mp1, dzb1, nslice, cap1, idx1, cnt, zs);
    zb_slice_members_kernel<<<(nslice + 63) / 64, 64, 0, s>>>(x2, Mp2, dzb2, nslice, cap2, idx2, cnt + nslice,
                                                              zs + nslice);
    if ((e = cudaGetLastError()) == cudaSuccess &&
        (e = cudaMemcpyAsync(c.data(), cnt, sizeof(long) * 2 * nslice, cudaMemcpyDeviceToHost, s)) == cudaSuccess &&
        (e = cudaMemcpyAsync(z.data(), zs, sizeof(double) * 2 * nslice, cudaMemcpyDeviceToHost, s)) ==
            cudaSuccess &&
        (e = cudaStreamSynchronize(s)) == cudaSuccess) {
      for (int i = 0; i < nslice; i++)
        if (c[i] > cap1 || c[nslice + i] > cap2 || c[i] < 2 || c[nslice + i] < 2) e = cudaErrorInvalidValue;
    }
  }
  if (e == cudaSuccess) {
    const int np = nslice * nslice;
    std::vector<int> I1(np), I2(np);
    std::vector<double> S(np), Z10(np), Z1(nslice), Z2(nslice);
    for (int i = 0; i < nslice; i++) {
      Z1[i] = z[i] / (double)(int)c[i];
      Z2[i] = z[nslice + i] / (double)(int)c[nslice + i];
    }
    for (int i = 0; i < nslice; i++)
      for (int j = 0; j < nslice; j++) {
        I1[i * nslice + j] = i;
        I2[i * nslice + j] = j;
        S[i * nslice + j] = (Z1[i] - Z2[j]) / 2.;
        Z10[i * nslice + j] = -(Z1[i] + Z2[j]) / 2.;
      }
    for (int i = 0; i < np; i++)
      for (int j = i + 1; j < np; j++)
        if (Z10[j] < Z10[i]) {
          std::swap(Z10[i], Z10[j]);
          std::swap(S[i], S[j]);
          std::swap(I1[i], I1[j]);
          std::swap(I2[i], I2[j]);
        }
    const unsigned cap = (unsigned)num_sms * 8;
    for (int i = 0; i < np && e == cudaSuccess; i++) {
      const long m1 = c[I1[i]], m2 = c[nslice + I2[i]];
      const int32_t *j1 = idx1 + (size_t)I1[i] * cap1, *j2 = idx2 + (size_t)I2[i] * cap2;
      // the pair collides with Np1*Mp1_coll/Mp1 and Np2*Mp2_coll/Mp2 (23245, 24400)
      const double N1c = Np1 * (int)m1 / (int)Mp1, N2c = Np2 * (int)m2 / (int)Mp2;
      const unsigned g1 = (unsigned)((m1 + 255) / 256 < cap ? (m1 + 255) / 256 : cap);
      const unsigned g2 = (unsigned)((m2 + 255) / 256 < cap ? (m2 + 255) / 256 : cap);
      if (m1 > 0) gather_members_kernel<<<g1, 256, 0, s>>>(x1, j1, m1, xc1);
      if (m2 > 0) gather_members_kernel<<<g2, 256, 0, s>>>(x2, j2, m2, xc2);
      e = collide(xc1, m1, xc2, m2, S[i], N1c, N2c, Z1[I1[i]], Z2[I2[i]]);
      if (m1 > 0) scatter_members_kernel<<<g1, 256, 0, s>>>(x1, j1, m1, xc1);
      if (m2 > 0) scatter_members_kernel<<<g2, 256, 0, s>>>(x2, j2, m2, xc2);
      if (e == cudaSuccess) e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  }
  cudaFree(buf);
  return e;
}

}  // namespace

cudaError_t soft_gaussian_6d_zb(double Np1, long Mp1, double *x1, double Np2, long Mp2, double *x2, double gamma1,
                                double gamma2, double bbscale1, double bbscale2, int nslice, const double *zb1,
                                const double *zb2, int num_sms, cudaStream_t s) {
  const double rp = 1.53469826769e-18;  // BB4D, simtrack.cpp:6328
  return sliced_6d_zb(Np1, Mp1, x1, Np2, Mp2, x2, nslice, zb1, zb2, num_sms, s,
                      [&](double *a, long m1, double *b, long m2, double S, double N1c, double N2c, double, double) {
                        const double c4_1 = 2 * N2c * rp / gamma1, c4_2 = 2 * N1c * rp / gamma2;
                        return slice_pair_collision(a, m1, b, m2, S, c4_1, c4_2, bbscale1, bbscale2, num_sms, s);
                      });
}

// BeamBeam6D_PIC_NonOffset (simtrack.cpp:24282-24432): the slice-boundary
// driver above with each slice pair colliding as BeamBeam4D_PIC_NonOffset on
// the caller's grid and Green spectrum (device arrays).
cudaError_t pic_6d_nonoffset(double Np1, long Mp1, double *x1, double Np2, long Mp2, double *x2, double gamma1,
                             double gamma2, double bbscale1, double bbscale2, int nslice, const double *zb1,
                             const double *zb2, int nx, double hx, double hy, const double *grn_re,
                             const double *grn_im, int num_sms, cudaStream_t s) {
  return sliced_6d_zb(Np1, Mp1, x1, Np2, Mp2, x2, nslice, zb1, zb2, num_sms, s,
                      [&](double *a, long m1, double *b, long m2, double S, double N1c, double N2c, double, double) {
                        const unsigned g1 = (unsigned)((m1 + 255) / 256 < num_sms * 8 ? (m1 + 255) / 256 : num_sms * 8);
                        const unsigned g2 = (unsigned)((m2 + 255) / 256 < num_sms * 8 ? (m2 + 255) / 256 : num_sms * 8);
                        slice_drift_kernel<<<g1 < 1 ? 1 : g1, 256, 0, s>>>(a, m1, S, true);
                        slice_drift_kernel<<<g2 < 1 ? 1 : g2, 256, 0, s>>>(b, m2, -S, true);
                        cudaError_t r = cudaGetLastError();
                        if (r == cudaSuccess)
                          r = pic_4d_nonoffset(N1c, m1, a, N2c, m2, b, gamma1, gamma2, bbscale1, bbscale2, nx, hx, hy,
                                               grn_re, grn_im, num_sms, s);
                        if (r != cudaSuccess) return r;
                        slice_drift_kernel<<<g1 < 1 ? 1 : g1, 256, 0, s>>>(a, m1, S, false);
                        slice_drift_kernel<<<g2 < 1 ? 1 : g2, 256, 0, s>>>(b, m2, -S, false);
                        return cudaGetLastError();
                      });
}

// BeamBeam6D_PIC_Interpolation (simtrack.cpp:24434-24700): the
// slice-boundary driver above; in each slice pair, each slice in turn
// deposits its charge drifted to the front and the back of the other slice
// (two potentials on the caller's grid and Green spectrum), and the other
// slice's particles, each drifted to its own collision point, take the field
// of the potential interpolated between the two, with N/Mp of the whole
// depositing bunch.
cudaError_t pic_6d_interpolation(double Np1, long Mp1, double *x1, double Np2, long Mp2, double *x2, double gamma1,
                                 double gamma2, double bbscale1, double bbscale2, int nslice, const double *zb1,
                                 const double *zb2, int nx, double hx, double hy, const double *grn_re,
                                 const double *grn_im, int num_sms, cudaStream_t s) {
  const double q1 = Np1 / (int)Mp1, q2 = Np2 / (int)Mp2;
  return sliced_6d_zb(Np1, Mp1, x1, Np2, Mp2, x2, nslice, zb1, zb2, num_sms, s,
                      [&](double *a, long m1, double *b, long m2, double, double, double, double z1c, double z2c) {
                        return pic_interpolation_pair(a, m1, b, m2, z1c, z2c, q1, q2, gamma1, gamma2, bbscale1,
                                                      bbscale2, nx, hx, hy, grn_re, grn_im, num_sms, s);
                      });
}

}  // namespace stb
