// Strong-strong beam-beam by particle-in-cell, 4D: BeamBeam4D_PIC
// (simtrack.cpp:23286-23378) on the GPU.
//
// Each beam's charge is deposited on a 64 x 64 grid (triangular-shaped
// cloud, Cal_Grid_Weight 2747-2791, Charge2Grid 2793-2806), the potential
// is the convolution of the charge with the integrated Green function of the
// 2D Poisson equation on the doubled 128 x 128 grid (Cal_Effective_Green_
// Function 2881-2921, Cal_Potential_Convolution 2955-2989, both through the
// reference's radix-2 FFT2D, 2583-2695), the field its 3 x 3-stencil
// gradient (Cal_Electric_Field 2998-3019), interpolated back to the other
// beam's particles with the same weights (Interpolate_Electric_Field
// 3021-3045), which take the kick.
//
// Every result equals the reference's bit for bit, so each step keeps the
// reference's operations and their order:
//   * deposition: the reference adds each particle's nine weights to the grid
//     in particle order.  Here every particle emits its nine (cell, weight)
//     items, a stable radix sort on the cell brings each cell's items
//     together in particle order, and one thread per cell adds them from
//     zero, so each cell's sum is the reference's chain of additions;
//   * FFT: the reference's in-place radix-2 transform (bit reversal, then
//     log2 n butterfly stages whose twiddles follow a recurrence).  The
//     twiddles do not depend on the data: the host runs the recurrence once
//     and the butterflies of a stage, independent of each other, run one per
//     thread with the reference's expressions;
//   * the Green function takes atan and log per cell: it is tabulated on the
//     host with the C library the reference calls (both directions' tables
//     at once, rows split across host threads), then transformed on the GPU.
#include <cuda_runtime.h>

#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <thread>
#include <vector>

#include "stb_kernels.hpp"

namespace stb {
namespace {

// Grids are square, nx x nx cells with nx a power of two (the reference
// indexes both axes with Nx as the row length, and its FFT2D takes powers of
// two); the doubled grid of the convolution is 2nx x 2nx.  BeamBeam4D_PIC and
// Lumi_Cal_PIC_4D use nx = 64 (Nx = Ny = 64 in the reference).
constexpr int kPicNx = 64;
constexpr int kMinLog2N2 = 4, kMaxLog2N2 = 10;  // nx from 8 to 512
constexpr int kNsigma = 15;                     // grid width in rms sizes
constexpr double kEps0 = 8.854187817e-12;

// Radix-sort key bits for the cell keys 0 .. ncell (ncell: outside the cut).
int key_bits(int ncell) {
  int b = 1;
  while ((1u << b) <= (unsigned)ncell) b++;
  return b;
}

// Cal_Grid_Weight (simtrack.cpp:2747-2791): the three mesh lines nearest the
// point and their weights along one axis.
__device__ __forceinline__ void grid_weight_1d(double d, double h, int m[3], double w[3]) {
  const double f = d / h;
  const int i = (int)f;
  double r;
  if ((f - i) <= 0.5) {
    m[0] = i;
    m[1] = i + 1;
    m[2] = i - 1;
    r = f - i;
  } else {
    m[0] = i + 1;
    m[1] = i;
    m[2] = i + 2;
    r = (i + 1) - f;
  }
  const double r2 = r * r;
  w[0] = 0.75 - r2;
  w[1] = 0.5 * (0.25 + r + r2);
  w[2] = 0.5 * (0.25 - r + r2);
}

__device__ __forceinline__ bool mesh_ok(const int m[3], int n) {
  return m[0] >= 0 && m[0] < n && m[1] >= 0 && m[1] < n && m[2] >= 0 && m[2] < n;
}

struct GridFrame {
  double mx, my;  // centre of the cut (the beam's mean, or 0)
  double x0, y0;  // grid origin
  double hx, hy;
  int nx;         // cells per side
};

// The cut of Charge2Grid's and the kick's callers: |x - mx| < (Nx/2 - 3) hx.
__device__ __forceinline__ bool in_cut(double xp, double yp, const GridFrame &g) {
  return fabs(xp - g.mx) < (g.nx / 2 - 3) * g.hx && fabs(yp - g.my) < (g.nx / 2 - 3) * g.hy;
}

// Nine (cell, weight) items per particle of the depositing beam, in the
// reference's (i, j) order; with `cut`, a particle outside the cut emits
// the key nx * nx (after every cell).
__global__ void deposit_items_kernel(const double *x, long n, GridFrame g, bool cut, uint32_t *keys, double *vals,
                                     int *err) {
  for (long p = (long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long)gridDim.x * blockDim.x) {
    const double xp = x[6 * p], yp = x[6 * p + 2];
    uint32_t *k = keys + 9 * p;
    double *v = vals + 9 * p;
    int xm[3], ym[3];
    double xw[3], yw[3];
    bool ok = !cut || in_cut(xp, yp, g);
    if (ok && !cut && !(isfinite(xp) && isfinite(yp))) {  // no cut to exclude it: no cell either
      atomicExch(err, 1);
      ok = false;
    }
    if (ok) {
      grid_weight_1d(xp - g.x0, g.hx, xm, xw);
      grid_weight_1d(yp - g.y0, g.hy, ym, yw);
      if (!mesh_ok(xm, g.nx) || !mesh_ok(ym, g.nx)) {
        atomicExch(err, 1);
        ok = false;
      }
    }
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) {
        k[3 * i + j] = ok ? (uint32_t)(xm[i] * g.nx + ym[j]) : (uint32_t)(g.nx * g.nx);
        v[3 * i + j] = ok ? xw[i] * yw[j] : 0.0;
      }
  }
}

// First and one-past-last item of every cell in the sorted keys.
__global__ void cell_bounds_kernel(const uint32_t *keys, long m, int ncell, int *start, int *end) {
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (long)gridDim.x * blockDim.x) {
    const uint32_t k = keys[i];
    if (k >= (uint32_t)ncell) continue;
    if (i == 0 || keys[i - 1] != k) start[k] = (int)i;
    if (i == m - 1 || keys[i + 1] != k) end[k] = (int)(i + 1);
  }
}

// src[c] = 0 + w_1 + w_2 + ... over the cell's items in particle order,
// written straight into the zero-padded real part of the doubled grid
// (Cal_Potential_Convolution's src_c_r); the rest of both parts is zero.
__global__ void cell_sum_pad_kernel(const double *vals, const int *start, const int *end, double *re, double *im,
                                    int nx) {
  const int n2 = 2 * nx;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n2 * n2) return;
  const int i = t / n2, j = t % n2;
  double s = 0.;
  if (i < nx && j < nx) {
    const int c = i * nx + j;
    for (int q = start[c]; q < end[c]; q++) s = s + vals[q];
  }
  re[t] = s;
  im[t] = 0.;
}

// One FFT1D (simtrack.cpp:2583-2647) per block over n = 2^LOG2N points: line b
// holds the elements base + t * es, base = b * ls.  tw holds the butterfly
// twiddles (u1, u2) of every stage, stage l's l1 = 2^l values from offset
// l1 - 1, as the reference's recurrence produces them for this direction.
// dir == 1 divides by n, as the reference's forward transform does.
template <int LOG2N>
__global__ void __launch_bounds__((1 << LOG2N) / 2) fft_lines_kernel(double *re, double *im, int ls, int es,
                                                                    const double2 *tw, int dir) {
  constexpr int N = 1 << LOG2N;
  __shared__ double sr[N], si[N];
  const int base = blockIdx.x * ls;
  for (int t = threadIdx.x; t < N; t += blockDim.x) {
    const int r = (int)(__brev((unsigned)t) >> (32 - LOG2N));
    sr[r] = re[base + t * es];
    si[r] = im[base + t * es];
  }
  const int b = threadIdx.x;
  for (int l = 0; l < LOG2N; l++) {
    __syncthreads();
    const int l1 = 1 << l;
    const int j = b & (l1 - 1);
    const int i = ((b >> l) << (l + 1)) + j, i1 = i + l1;
    const double2 u = tw[l1 - 1 + j];
    const double t1 = u.x * sr[i1] - u.y * si[i1];
    const double t2 = u.x * si[i1] + u.y * sr[i1];
    sr[i1] = sr[i] - t1;
    si[i1] = si[i] - t2;
    sr[i] += t1;
    si[i] += t2;
  }
  __syncthreads();
  for (int t = threadIdx.x; t < N; t += blockDim.x) {
    double a = sr[t], c = si[t];
    if (dir == 1) {
      a /= (double)N;
      c /= (double)N;
    }
    re[base + t * es] = a;
    im[base + t * es] = c;
  }
}

// FFT2D (simtrack.cpp:2649-2695) of an n x n array, n = 2^log2n: the
// columns x[i*n + j] over i, then the rows.
template <int LOG2N>
void fft2d_n(double *re, double *im, const double2 *tw, int dir, cudaStream_t s) {
  constexpr int N = 1 << LOG2N;
  fft_lines_kernel<LOG2N><<<N, N / 2, 0, s>>>(re, im, 1, N, tw, dir);
  fft_lines_kernel<LOG2N><<<N, N / 2, 0, s>>>(re, im, N, 1, tw, dir);
}
void fft2d(double *re, double *im, const double2 *tw, int dir, int log2n, cudaStream_t s) {
  switch (log2n) {
    case 4: return fft2d_n<4>(re, im, tw, dir, s);
    case 5: return fft2d_n<5>(re, im, tw, dir, s);
    case 6: return fft2d_n<6>(re, im, tw, dir, s);
    case 7: return fft2d_n<7>(re, im, tw, dir, s);
    case 8: return fft2d_n<8>(re, im, tw, dir, s);
    case 9: return fft2d_n<9>(re, im, tw, dir, s);
    default: return fft2d_n<10>(re, im, tw, dir, s);
  }
}

// The spectrum product of Cal_Potential_Convolution, in place into (re, im).
__global__ void spectrum_product_kernel(double *re, double *im, const double *gr, const double *gi, int total) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= total) return;
  const double a = re[t], b = im[t], c = gr[t], d = gi[t];
  re[t] = a * c - b * d;
  im[t] = a * d + b * c;
}

// phi from the inverse transform, then Cal_Electric_Field's stencil
// (zero on the grid's border).  One thread per cell; phi is re-derived by
// each neighbour with the same expression, so every value is the reference's.
__device__ __forceinline__ double phi_at(const double *re, int i, int j, int nx) {
  return re[i * 2 * nx + j] * 2 * nx * 2 * nx / 2 / 3.14159265 / kEps0;
}

// Interpolate_Electric_Field_1Potential (3047-3094) differences the same
// potential values with the same stencil around the particle, so this field
// serves both interpolations bit for bit.
__global__ void field_kernel(const double *re, double hx, double hy, double *Ex, double *Ey, int nx) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nx * nx) return;
  const int i = t / nx, j = t % nx;
  double ex = 0., ey = 0.;
  if (i >= 1 && i < nx - 1 && j >= 1 && j < nx - 1) {
    ex = -((phi_at(re, i + 1, j + 1, nx) - phi_at(re, i - 1, j + 1, nx)) +
           4 * (phi_at(re, i + 1, j, nx) - phi_at(re, i - 1, j, nx)) +
           (phi_at(re, i + 1, j - 1, nx) - phi_at(re, i - 1, j - 1, nx))) /
         12. / hx;
    ey = -((phi_at(re, i + 1, j + 1, nx) - phi_at(re, i + 1, j - 1, nx)) +
           4 * (phi_at(re, i, j + 1, nx) - phi_at(re, i, j - 1, nx)) +
           (phi_at(re, i - 1, j + 1, nx) - phi_at(re, i - 1, j - 1, nx))) /
         12. / hy;
  }
  Ex[t] = ex;
  Ey[t] = ey;
}

// The kicked beam: particles inside the cut (around their own mean) take
// the field interpolated at (x - xoffset, y - yoffset) on the other beam's
// grid; px += ex e bbscale / (gamma m_p c^2 / e) (Np_other / Mp_other).
__global__ void pic_kick_kernel(double *x, long n, GridFrame g, double xoffset, double yoffset, const double *Ex,
                                const double *Ey, double bbscale, double gamma, double np_per_mp, int *err) {
  for (long p = (long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long)gridDim.x * blockDim.x) {
    double *q = x + 6 * p;
    const double xp = q[0], yp = q[2];
    if (!in_cut(xp, yp, g)) continue;
    const double xs = xp - xoffset, ys = yp - yoffset;
    int xm[3], ym[3];
    double xw[3], yw[3];
    grid_weight_1d(xs - g.x0, g.hx, xm, xw);
    grid_weight_1d(ys - g.y0, g.hy, ym, yw);
    if (!mesh_ok(xm, g.nx) || !mesh_ok(ym, g.nx)) {
      atomicExch(err, 1);
      continue;
    }
    double ex = 0., ey = 0.;
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) {
        ex = ex + Ex[xm[i] * g.nx + ym[j]] * xw[i] * yw[j];
        ey = ey + Ey[xm[i] * g.nx + ym[j]] * xw[i] * yw[j];
      }
    q[1] = q[1] + ex * 1.60217662e-19 * bbscale / (gamma * 938.27201e6) * np_per_mp;
    q[3] = q[3] + ey * 1.60217662e-19 * bbscale / (gamma * 938.27201e6) * np_per_mp;
  }
}

// The potential of Cal_Potential_Convolution, phi[i*nx + j], from the
// inverse transform.
__global__ void potential_kernel(const double *re, double *phi, int nx) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nx * nx) return;
  phi[t] = phi_at(re, t / nx, t % nx, nx);
}

// x -= px S (plus = false) or x += px S, and the same for y.
__global__ void drift_xy_kernel(double *x, long n, double S, bool plus) {
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    double *q = x + 6 * i;
    if (plus) {
      q[0] = q[0] + q[1] * S;
      q[2] = q[2] + q[3] * S;
    } else {
      q[0] = q[0] - q[1] * S;
      q[2] = q[2] - q[3] * S;
    }
  }
}

// The z range of a slice, from -100 and 100 as the reference starts
// (exact in any order): out2 = zfront (largest), zback (smallest).
__global__ void __launch_bounds__(1024) zrange_kernel(const double *x, long n, double *out2) {
  __shared__ double red[2][32];
  double zf = -100, zb = 100;
  for (long i = threadIdx.x; i < n; i += 1024) {
    const double z = x[6 * i + 4];
    if (z > zf) zf = z;
    if (z < zb) zb = z;
  }
  for (int o = 16; o > 0; o >>= 1) {
    const double a = __shfl_down_sync(0xffffffffu, zf, o), c = __shfl_down_sync(0xffffffffu, zb, o);
    if (a > zf) zf = a;
    if (c < zb) zb = c;
  }
  if ((threadIdx.x & 31) == 0) {
    red[0][threadIdx.x >> 5] = zf;
    red[1][threadIdx.x >> 5] = zb;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    zf = red[0][0];
    zb = red[1][0];
    for (int w = 1; w < 32; w++) {
      if (red[0][w] > zf) zf = red[0][w];
      if (red[1][w] < zb) zb = red[1][w];
    }
    out2[0] = zf;
    out2[1] = zb;
  }
}

// The kicked slice of BeamBeam6D_PIC_Interpolation (simtrack.cpp:24600-24615
// and its mirror): each particle drifts by sp = (z - zc) / 2, takes the
// field of Interpolate_Electric_Field_2Potential (3096-3152: a 5 x 5 patch of
// the potential interpolated in s between phi1 at sfront and phi2 at sback,
// differenced with the field stencil at the 3 x 3 mesh lines, weighted) if
// inside the cut around the origin, and drifts back with the kicked momenta.
__global__ void interp2_kick_kernel(double *x, long n, double zc, GridFrame g, double sfront, double sback,
                                    const double *phi1, const double *phi2, double bbscale, double gamma,
                                    double np_per_mp, int *err) {
  for (long p = (long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long)gridDim.x * blockDim.x) {
    double *q = x + 6 * p;
    const double sp = (q[4] - zc) / 2;
    q[0] = q[0] + q[1] * sp;
    q[2] = q[2] + q[3] * sp;
    const double xp = q[0], yp = q[2];
    if (in_cut(xp, yp, g)) {
      int xm[3], ym[3];
      double xw[3], yw[3];
      grid_weight_1d(xp - g.x0, g.hx, xm, xw);
      grid_weight_1d(yp - g.y0, g.hy, ym, yw);
      int i0 = 10000, j0 = 10000;
      for (int k = 0; k < 3; k++) {
        if (xm[k] < i0) i0 = xm[k];
        if (ym[k] < j0) j0 = ym[k];
      }
      if (i0 < 1 || j0 < 1 || i0 + 3 >= g.nx || j0 + 3 >= g.nx) {
        atomicExch(err, 1);
      } else {
        double ph[25];
        for (int a = 0; a < 5; a++)
          for (int b = 0; b < 5; b++) {
            const int c = g.nx * (i0 - 1 + a) + (j0 - 1 + b);
            if (sfront == sback) {
              ph[5 * a + b] = phi1[c];
            } else {
              const double pf = phi1[c], pb = phi2[c];
              ph[5 * a + b] = pb + (pf - pb) * (sp - sback) / (sfront - sback);
            }
          }
        double ex = 0., ey = 0.;
        for (int i = 0; i < 3; i++)
          for (int j = 0; j < 3; j++) {
            const int a = xm[i] - i0 + 1, b = ym[j] - j0 + 1;
            const double fx = -((ph[(a + 1) * 5 + b + 1] - ph[(a - 1) * 5 + b + 1]) +
                                4 * (ph[(a + 1) * 5 + b] - ph[(a - 1) * 5 + b]) +
                                (ph[(a + 1) * 5 + b - 1] - ph[(a - 1) * 5 + b - 1])) /
                              12. / g.hx;
            const double fy = -((ph[(a + 1) * 5 + b + 1] - ph[(a + 1) * 5 + b - 1]) +
                                4 * (ph[a * 5 + b + 1] - ph[a * 5 + b - 1]) +
                                (ph[(a - 1) * 5 + b + 1] - ph[(a - 1) * 5 + b - 1])) /
                              12. / g.hy;
            ex = ex + fx * xw[i] * yw[j];
            ey = ey + fy * xw[i] * yw[j];
          }
        q[1] = q[1] + ex * 1.60217662e-19 * bbscale / (gamma * 938.27201e6) * np_per_mp;
        q[3] = q[3] + ey * 1.60217662e-19 * bbscale / (gamma * 938.27201e6) * np_per_mp;
      }
    }
    q[0] = q[0] - q[1] * sp;
    q[2] = q[2] - q[3] * sp;
  }
}

// src[c] = 0 + w_1 + w_2 + ... for the 64 x 64 grid alone (Charge2Grid's
// array).
__global__ void cell_sum_kernel(const double *vals, const int *start, const int *end, double *src, int ncell) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncell) return;
  double s = 0.;
  for (int q = start[c]; q < end[c]; q++) s = s + vals[q];
  src[c] = s;
}

// Lumi_Cal_PIC_4D's grid extent (simtrack.cpp:23639-23652): min and max of
// x and y over both beams, starting from 1000 and -1000 as the reference
// does.  Exact in any order; one CTA, out4 = xmin, xmax, ymin, ymax.
constexpr int kExtentBlock = 1024;
__global__ void __launch_bounds__(kExtentBlock) extent_kernel(const double *x1, long n1, const double *x2, long n2,
                                                              double *out4) {
  __shared__ double red[4][kExtentBlock / 32];
  double v[4] = {1000., -1000., 1000., -1000.};
  for (int b = 0; b < 2; b++) {
    const double *x = b == 0 ? x1 : x2;
    const long n = b == 0 ? n1 : n2;
    for (long i = threadIdx.x; i < n; i += kExtentBlock) {
      const double a = x[6 * i], c = x[6 * i + 2];
      if (a < v[0]) v[0] = a;
      if (a > v[1]) v[1] = a;
      if (c < v[2]) v[2] = c;
      if (c > v[3]) v[3] = c;
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    const double a0 = __shfl_down_sync(0xffffffffu, v[0], o), a1 = __shfl_down_sync(0xffffffffu, v[1], o);
    const double a2 = __shfl_down_sync(0xffffffffu, v[2], o), a3 = __shfl_down_sync(0xffffffffu, v[3], o);
    if (a0 < v[0]) v[0] = a0;
    if (a1 > v[1]) v[1] = a1;
    if (a2 < v[2]) v[2] = a2;
    if (a3 > v[3]) v[3] = a3;
  }
  const int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0)
    for (int k = 0; k < 4; k++) red[k][w] = v[k];
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = 0; k < 4; k++) v[k] = red[k][0];
    for (int q = 1; q < kExtentBlock / 32; q++) {
      if (red[0][q] < v[0]) v[0] = red[0][q];
      if (red[1][q] > v[1]) v[1] = red[1][q];
      if (red[2][q] < v[2]) v[2] = red[2][q];
      if (red[3][q] > v[3]) v[3] = red[3][q];
    }
    for (int k = 0; k < 4; k++) out4[k] = v[k];
  }
}

// The overlap sum of Lumi_Cal_PIC_4D (23680-23683), in cell order.
__global__ void overlap_sum_kernel(const double *src1, const double *src2, double *out, int ncell) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double l = 0;
  for (int i = 0; i < ncell; i++) l = l + src1[i] * src2[i];
  *out = l;
}

// The butterfly twiddles of FFT1D for n = 2^m in direction dir, from the
// reference's recurrence (u advanced by (c1, c2) within a stage; c1, c2
// halved in angle between stages).
std::vector<double2> fft_twiddles(int m, int dir) {
  std::vector<double2> tw;
  double c1 = -1.0, c2 = 0.0;
  long l2 = 1;
  for (int l = 0; l < m; l++) {
    const long l1 = l2;
    l2 <<= 1;
    double u1 = 1.0, u2 = 0.0;
    for (long j = 0; j < l1; j++) {
      tw.push_back(make_double2(u1, u2));
      const double z = u1 * c1 - u2 * c2;
      u2 = u1 * c2 + u2 * c1;
      u1 = z;
    }
    c2 = std::sqrt((1.0 - c1) / 2.0);
    if (dir == 1) c2 = -c2;
    c1 = std::sqrt((1.0 + c1) / 2.0);
  }
  return tw;
}

// int_green and calc_egreen (simtrack.cpp:2808-2879): the Green function
// of the 2D Poisson equation integrated over the cell [x1, x2] x [y1, y2].
double int_green(double x, double y) {
  if (0 == x || 0 == y) return 0;
  const double x2 = x * x, y2 = y * y;
  return -3 * x * y + x2 * std::atan(y / x) + y2 * std::atan(x / y) + x * y * std::log(x2 + y2);
}

double calc_egreen(double x1, double x2, double y1, double y2, double hx, double hy) {
  if (x1 * x2 * y1 * y2 != 0.) {
    int s11 = 1, s12 = 1, s21 = 1, s22 = 1;
    if (x1 > 0) {
      s11 *= -1;
      s12 *= -1;
    } else if (x1 < 0 && x2 < 0) {
      s21 *= -1;
      s22 *= -1;
    }
    if (y1 > 0) {
      s11 *= -1;
      s21 *= -1;
    } else if (y1 < 0 && y2 < 0) {
      s12 *= -1;
      s22 *= -1;
    }
    x1 = std::fabs(x1);
    x2 = std::fabs(x2);
    y1 = std::fabs(y1);
    y2 = std::fabs(y2);
    const double v11 = int_green(x1, y1), v12 = int_green(x1, y2);
    const double v21 = int_green(x2, y1), v22 = int_green(x2, y2);
    const double r = s11 * v11 + s12 * v12 + s21 * v21 + s22 * v22;
    return -1.0 * r / hx / hy / 2;
  }
  double r = 0.;
  for (int i = 0; i < 20; i++)
    for (int j = 0; j < 20; j++) {
      const double tx = x1 + (i - 1) * hx / 20 + hx / 40;
      const double ty = y1 + (j - 1) * hy / 20 + hy / 40;
      if (tx != 0. && ty != 0.) r = r - 0.5 * std::log(tx * tx + ty * ty);
    }
  return r / 400.;
}

// Cal_Effective_Green_Function's tables before their transform (2881-2918)
// for nd directions: g[d][i * 2nx + j] over the four quadrants of the
// doubled grid, offsets (xoff[d], yoff[d]); the rows are split across host
// threads.
void green_tables(int nd, const double *xoff, const double *yoff, double hx, double hy, int nx, double *const *g) {
  const int n2 = 2 * nx;
  auto rows = [&](int r0, int r1) {
    for (int r = r0; r < r1; r++) {
      const int d = r / n2, i = r % n2;
      for (int j = 0; j < n2; j++) {
        double x1, y1;
        if (i <= nx - 1) x1 = xoff[d] + i * hx - 0.5 * hx;
        else x1 = xoff[d] - (2 * nx - i) * hx - 0.5 * hx;
        if (j <= nx - 1) y1 = yoff[d] + j * hy - 0.5 * hy;
        else y1 = yoff[d] - (2 * nx - j) * hy - 0.5 * hy;
        g[d][i * n2 + j] = calc_egreen(x1, x1 + hx, y1, y1 + hy, hx, hy);
      }
    }
  };
  const int nrows = nd * n2;
  const int nt = (int)std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
  std::vector<std::thread> th;
  const int per = (nrows + nt - 1) / nt;
  for (int t = 0; t < nt; t++) {
    const int a = t * per, b = std::min(nrows, a + per);
    if (a < b) th.emplace_back(rows, a, b);
  }
  for (auto &t : th) t.join();
}

int log2_of(int n) {
  int l = 0;
  while ((1 << l) < n) l++;
  return l;
}

// Device scratch of one collision on an nx x nx grid with at most nmax
// particles per beam: two Green spectra, the work grid, the field, the
// moments, the twiddles of both directions, the (cell, weight) items, the
// cell bounds, the error flag and the radix sort's scratch.
struct PicScratch {
  unsigned char *buf = nullptr;
  int nx = 0, n2 = 0, log2n2 = 0, ncell = 0, kbits = 0;
  size_t grid2 = 0, sort_bytes = 0;
  long nitem = 0;
  double *g_re[2] = {nullptr, nullptr}, *g_im[2] = {nullptr, nullptr};
  double *wr = nullptr, *wi = nullptr, *Ex = nullptr, *Ey = nullptr, *m8 = nullptr;
  double2 *tw_fwd = nullptr, *tw_inv = nullptr;
  double *vals_in = nullptr, *vals_out = nullptr;
  uint32_t *keys_in = nullptr, *keys_out = nullptr;
  int *cstart = nullptr, *cend = nullptr, *err = nullptr;
  void *sort_tmp = nullptr;
  std::vector<double2> twf, twi;

  ~PicScratch() {
    if (buf) cudaFree(buf);
  }
  cudaError_t init(int nx_, long nmax, cudaStream_t s) {
    nx = nx_;
    n2 = 2 * nx;
    log2n2 = log2_of(n2);
    ncell = nx * nx;
    kbits = key_bits(ncell);
    grid2 = (size_t)n2 * n2;
    nitem = 9 * nmax;
    cudaError_t e = cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, (const uint32_t *)nullptr,
                                                    (uint32_t *)nullptr, (const double *)nullptr, (double *)nullptr,
                                                    (int)nitem, 0, kbits, s);
    if (e != cudaSuccess) return e;
    const int ntw = n2 - 1;
    const size_t nd = 6 * grid2 + 2 * (size_t)ncell + 8 + 4 * (size_t)ntw + 2 * (size_t)nitem;
    const size_t bytes = sizeof(double) * nd + sizeof(uint32_t) * 2 * (size_t)nitem +
                         sizeof(int) * (2 * (size_t)ncell + 2) + sort_bytes + 256;
    if ((e = cudaMalloc(&buf, bytes)) != cudaSuccess) return e;
    g_re[0] = reinterpret_cast<double *>(buf);
    g_im[0] = g_re[0] + grid2;
    g_re[1] = g_im[0] + grid2;
    g_im[1] = g_re[1] + grid2;
    wr = g_im[1] + grid2;
    wi = wr + grid2;
    Ex = wi + grid2;
    Ey = Ex + ncell;
    m8 = Ey + ncell;
    tw_fwd = reinterpret_cast<double2 *>(m8 + 8);
    tw_inv = tw_fwd + ntw;
    vals_in = reinterpret_cast<double *>(tw_inv + ntw);
    vals_out = vals_in + nitem;
    keys_in = reinterpret_cast<uint32_t *>(vals_out + nitem);
    keys_out = keys_in + nitem;
    cstart = reinterpret_cast<int *>(keys_out + nitem);
    cend = cstart + ncell;
    err = cend + ncell;
    sort_tmp = reinterpret_cast<void *>(((uintptr_t)(err + 2) + 255) & ~(uintptr_t)255);
    twf = fft_twiddles(log2n2, 1);
    twi = fft_twiddles(log2n2, -1);
    if ((e = cudaMemcpyAsync(tw_fwd, twf.data(), sizeof(double2) * ntw, cudaMemcpyHostToDevice, s)) != cudaSuccess)
      return e;
    if ((e = cudaMemcpyAsync(tw_inv, twi.data(), sizeof(double2) * ntw, cudaMemcpyHostToDevice, s)) != cudaSuccess)
      return e;
    return cudaMemsetAsync(err, 0, sizeof(int), s);
  }
};

unsigned grid_of(long n, int num_sms) {
  const long g = (n + 255) / 256, cap = (long)num_sms * 8;
  return (unsigned)(g < 1 ? 1 : g > cap ? cap : g);
}

// Charge2Grid over the n particles of x (with or without the cut), the
// per-cell ordered sums into `src` (nx x nx), or, when `pad`, into the real
// part of the zero-padded doubled grid (wr, wi).
cudaError_t deposit(PicScratch &S, const double *x, long n, const GridFrame &g, bool cut, bool pad, double *src,
                    int num_sms, cudaStream_t s) {
  deposit_items_kernel<<<grid_of(n, num_sms), 256, 0, s>>>(x, n, g, cut, S.keys_in, S.vals_in, S.err);
  cudaError_t e = cub::DeviceRadixSort::SortPairs(S.sort_tmp, S.sort_bytes, S.keys_in, S.keys_out, S.vals_in,
                                                  S.vals_out, (int)(9 * n), 0, S.kbits, s);
  if (e != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(S.cstart, 0, sizeof(int) * 2 * (size_t)S.ncell, s)) != cudaSuccess) return e;
  cell_bounds_kernel<<<grid_of(9 * n, num_sms), 256, 0, s>>>(S.keys_out, 9 * n, S.ncell, S.cstart, S.cend);
  if (pad)
    cell_sum_pad_kernel<<<(int)((S.grid2 + 127) / 128), 128, 0, s>>>(S.vals_out, S.cstart, S.cend, S.wr, S.wi,
                                                                      S.nx);
  else
    cell_sum_kernel<<<(S.ncell + 127) / 128, 128, 0, s>>>(S.vals_out, S.cstart, S.cend, src, S.ncell);
  return cudaGetLastError();
}

// Cal_Potential_Convolution and Cal_Electric_Field on the deposited charge
// (wr, wi) with the Green spectrum (gre, gim): Ex, Ey.
cudaError_t potential_field(PicScratch &S, const double *gre, const double *gim, double hx, double hy,
                            cudaStream_t s) {
  fft2d(S.wr, S.wi, S.tw_fwd, 1, S.log2n2, s);
  spectrum_product_kernel<<<(int)((S.grid2 + 255) / 256), 256, 0, s>>>(S.wr, S.wi, gre, gim, (int)S.grid2);
  fft2d(S.wr, S.wi, S.tw_inv, -1, S.log2n2, s);
  field_kernel<<<(S.ncell + 127) / 128, 128, 0, s>>>(S.wr, hx, hy, S.Ex, S.Ey, S.nx);
  return cudaGetLastError();
}

// Cal_Potential_Convolution alone: the potential of the deposited charge
// (wr, wi) with the Green spectrum (gre, gim) into phi (nx x nx).
cudaError_t potential(PicScratch &S, const double *gre, const double *gim, double *phi, cudaStream_t s) {
  fft2d(S.wr, S.wi, S.tw_fwd, 1, S.log2n2, s);
  spectrum_product_kernel<<<(int)((S.grid2 + 255) / 256), 256, 0, s>>>(S.wr, S.wi, gre, gim, (int)S.grid2);
  fft2d(S.wr, S.wi, S.tw_inv, -1, S.log2n2, s);
  potential_kernel<<<(S.ncell + 127) / 128, 128, 0, s>>>(S.wr, phi, S.nx);
  return cudaGetLastError();
}

cudaError_t finish(PicScratch &S, cudaError_t e, cudaStream_t s) {
  int h_err = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&h_err, S.err, sizeof(int), cudaMemcpyDeviceToHost, s);
  const cudaError_t e2 = cudaStreamSynchronize(s);
  if (e == cudaSuccess) e = e2;
  if (e == cudaSuccess && h_err) e = cudaErrorInvalidValue;
  return e;
}

}  // namespace

bool pic_grid_valid(int nx, int ny) {
  if (nx != ny || nx < 1 || (nx & (nx - 1)) != 0) return false;
  const int l = log2_of(2 * nx);
  return l >= kMinLog2N2 && l <= kMaxLog2N2;
}

cudaError_t pic_4d(double Np1, long Mp1, double *x1, double Np2, long Mp2, double *x2, double gamma1, double gamma2,
                   double bbscale1, double bbscale2, int num_sms, cudaStream_t s) {
  PicScratch S;
  cudaError_t e = S.init(kPicNx, std::max(Mp1, Mp2), s);
  std::vector<double> h_m8(8), h_green(2 * S.grid2);
  do {
    if (e != cudaSuccess) break;
    if ((e = beam_pair_mean_rms(x1, Mp1, x2, Mp2, S.m8, s)) != cudaSuccess) break;
    if ((e = cudaMemcpyAsync(h_m8.data(), S.m8, sizeof(double) * 8, cudaMemcpyDeviceToHost, s)) != cudaSuccess) break;
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) break;
    const double mean1[2] = {h_m8[0], h_m8[1]}, rms1[2] = {h_m8[2], h_m8[3]};
    const double mean2[2] = {h_m8[4], h_m8[5]}, rms2[2] = {h_m8[6], h_m8[7]};
    const double rmsx = rms1[0] > rms2[0] ? rms2[0] : rms1[0];
    const double rmsy = rms1[1] > rms2[1] ? rms2[1] : rms1[1];
    const double hx = kNsigma * rmsx / kPicNx, hy = kNsigma * rmsy / kPicNx;
    // direction 0: beam 1 deposits, beam 2 is kicked; direction 1 the reverse
    const double xoff[2] = {mean2[0] - mean1[0], mean1[0] - mean2[0]};
    const double yoff[2] = {mean2[1] - mean1[1], mean1[1] - mean2[1]};
    double *const hg[2] = {h_green.data(), h_green.data() + S.grid2};
    green_tables(2, xoff, yoff, hx, hy, kPicNx, hg);
    for (int d = 0; d < 2 && e == cudaSuccess; d++) {
      if ((e = cudaMemcpyAsync(S.g_re[d], hg[d], sizeof(double) * S.grid2, cudaMemcpyHostToDevice, s)) !=
              cudaSuccess ||
          (e = cudaMemsetAsync(S.g_im[d], 0, sizeof(double) * S.grid2, s)) != cudaSuccess)
        break;
      fft2d(S.g_re[d], S.g_im[d], S.tw_fwd, 1, S.log2n2, s);
    }
    for (int d = 0; d < 2 && e == cudaSuccess; d++) {
      const double *ms = d == 0 ? mean1 : mean2, *mt = d == 0 ? mean2 : mean1;
      const long ns = d == 0 ? Mp1 : Mp2, nt = d == 0 ? Mp2 : Mp1;
      const GridFrame gs{ms[0], ms[1], ms[0] - kPicNx * hx / 2, ms[1] - kPicNx * hy / 2, hx, hy, kPicNx};
      if ((e = deposit(S, d == 0 ? x1 : x2, ns, gs, true, true, nullptr, num_sms, s)) != cudaSuccess) break;
      if ((e = potential_field(S, S.g_re[d], S.g_im[d], hx, hy, s)) != cudaSuccess) break;
      GridFrame gt = gs;
      gt.mx = mt[0];
      gt.my = mt[1];
      pic_kick_kernel<<<grid_of(nt, num_sms), 256, 0, s>>>(d == 0 ? x2 : x1, nt, gt, xoff[d], yoff[d], S.Ex, S.Ey,
                                                            d == 0 ? bbscale2 : bbscale1, d == 0 ? gamma2 : gamma1,
                                                            (d == 0 ? Np1 : Np2) / (double)(int)ns, S.err);
      e = cudaGetLastError();
    }
  } while (false);
  return finish(S, e, s);
}

cudaError_t pic_4d_nonoffset(double Np1, long Mp1, double *x1, double Np2, long Mp2, double *x2, double gamma1,
                             double gamma2, double bbscale1, double bbscale2, int nx, double hx, double hy,
                             const double *grn_re, const double *grn_im, int num_sms, cudaStream_t s) {
  PicScratch S;
  cudaError_t e = S.init(nx, std::max(Mp1, Mp2), s);
  // the grid is centred on the origin: x0 = -Nx hx / 2, no offset, the cut around 0
  const GridFrame g{0., 0., -nx * hx / 2, -nx * hy / 2, hx, hy, nx};
  for (int d = 0; d < 2 && e == cudaSuccess; d++) {
    const long ns = d == 0 ? Mp1 : Mp2, nt = d == 0 ? Mp2 : Mp1;
    if ((e = deposit(S, d == 0 ? x1 : x2, ns, g, true, true, nullptr, num_sms, s)) != cudaSuccess) break;
    if ((e = potential_field(S, grn_re, grn_im, hx, hy, s)) != cudaSuccess) break;
    pic_kick_kernel<<<grid_of(nt, num_sms), 256, 0, s>>>(d == 0 ? x2 : x1, nt, g, 0., 0., S.Ex, S.Ey,
                                                          d == 0 ? bbscale2 : bbscale1, d == 0 ? gamma2 : gamma1,
                                                          (d == 0 ? Np1 : Np2) / (double)(int)ns, S.err);
    e = cudaGetLastError();
  }
  return finish(S, e, s);
}

cudaError_t pic_interpolation_pair(double *x1, long m1, double *x2, long m2, double z1c, double z2c,
                                   double np1_per_mp1, double np2_per_mp2, double gamma1, double gamma2,
                                   double bbscale1, double bbscale2, int nx, double hx, double hy,
                                   const double *grn_re, const double *grn_im, int num_sms, cudaStream_t s) {
  PicScratch S;
  cudaError_t e = S.init(nx, std::max(m1, m2), s);
  const GridFrame g{0., 0., -nx * hx / 2, -nx * hy / 2, hx, hy, nx};
  double zr[2] = {0, 0};
  // direction 0: slice 1 deposits at the front and back of slice 2, slice 2
  // is kicked; direction 1 the reverse, with slice 2's kicked momenta
  for (int d = 0; d < 2 && e == cudaSuccess; d++) {
    double *xs = d == 0 ? x1 : x2, *xt = d == 0 ? x2 : x1;
    const long ms = d == 0 ? m1 : m2, mt = d == 0 ? m2 : m1;
    const double zc = d == 0 ? z1c : z2c;
    zrange_kernel<<<1, 1024, 0, s>>>(xt, mt, S.m8);
    if ((e = cudaMemcpyAsync(zr, S.m8, sizeof(zr), cudaMemcpyDeviceToHost, s)) != cudaSuccess) break;
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) break;
    const double sfront = (zr[0] - zc) / 2, sback = (zr[1] - zc) / 2;
    const double sd[2] = {sfront, sback};
    double *phi[2] = {S.Ex, S.Ey};
    for (int k = 0; k < 2 && e == cudaSuccess; k++) {
      drift_xy_kernel<<<grid_of(ms, num_sms), 256, 0, s>>>(xs, ms, sd[k], false);
      if ((e = deposit(S, xs, ms, g, true, true, nullptr, num_sms, s)) != cudaSuccess) break;
      if ((e = potential(S, grn_re, grn_im, phi[k], s)) != cudaSuccess) break;
      drift_xy_kernel<<<grid_of(ms, num_sms), 256, 0, s>>>(xs, ms, sd[k], true);
      e = cudaGetLastError();
    }
    if (e != cudaSuccess) break;
    interp2_kick_kernel<<<grid_of(mt, num_sms), 256, 0, s>>>(xt, mt, zc, g, sfront, sback, S.Ex, S.Ey,
                                                              d == 0 ? bbscale2 : bbscale1, d == 0 ? gamma2 : gamma1,
                                                              d == 0 ? np1_per_mp1 : np2_per_mp2, S.err);
    e = cudaGetLastError();
  }
  return finish(S, e, s);
}

cudaError_t pic_green_function(double xoffset, double yoffset, int nx, double hx, double hy, double *grn_re,
                               double *grn_im, cudaStream_t s) {
  PicScratch S;
  cudaError_t e = S.init(nx, 1, s);
  std::vector<double> h(S.grid2);
  do {
    if (e != cudaSuccess) break;
    double *const hg[1] = {h.data()};
    green_tables(1, &xoffset, &yoffset, hx, hy, nx, hg);
    if ((e = cudaMemcpyAsync(S.g_re[0], h.data(), sizeof(double) * S.grid2, cudaMemcpyHostToDevice, s)) !=
            cudaSuccess ||
        (e = cudaMemsetAsync(S.g_im[0], 0, sizeof(double) * S.grid2, s)) != cudaSuccess)
      break;
    fft2d(S.g_re[0], S.g_im[0], S.tw_fwd, 1, S.log2n2, s);
    if ((e = cudaMemcpyAsync(grn_re, S.g_re[0], sizeof(double) * S.grid2, cudaMemcpyDeviceToHost, s)) !=
            cudaSuccess ||
        (e = cudaMemcpyAsync(grn_im, S.g_im[0], sizeof(double) * S.grid2, cudaMemcpyDeviceToHost, s)) != cudaSuccess)
      break;
  } while (false);
  return finish(S, e, s);
}

cudaError_t lumi_pic_4d(double Np1, long Mp1, double Np2, long Mp2, const double *x1, const double *x2, int Ncoll,
                        double freq, int num_sms, cudaStream_t s, double *lumi_out) {
  PicScratch S;
  cudaError_t e = S.init(kPicNx, std::max(Mp1, Mp2), s);
  double h_ext[4] = {0, 0, 0, 0}, h_ov = 0;
  bool degenerate = false;
  double hx = 0, hy = 0;
  do {
    if (e != cudaSuccess) break;
    extent_kernel<<<1, kExtentBlock, 0, s>>>(x1, Mp1, x2, Mp2, S.m8);
    if ((e = cudaMemcpyAsync(h_ext, S.m8, sizeof(h_ext), cudaMemcpyDeviceToHost, s)) != cudaSuccess) break;
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) break;
    const double xmin = h_ext[0], xmax = h_ext[1], ymin = h_ext[2], ymax = h_ext[3];
    // the reference's grid: 64 cells over the extent, widened by 4 of them on each side
    hx = (xmax - xmin) / kPicNx;
    hy = (ymax - ymin) / kPicNx;
    const double x0 = xmin - 4 * hx, y0 = ymin - 4 * hy;
    hx = (xmax - xmin + 8 * hx) / kPicNx;
    hy = (ymax - ymin + 8 * hy) / kPicNx;
    if (!(hx > 0) || !(hy > 0) || !std::isfinite(hx) || !std::isfinite(hy)) {
      degenerate = true;
      break;
    }
    const GridFrame g{0., 0., x0, y0, hx, hy, kPicNx};
    if ((e = deposit(S, x1, Mp1, g, false, false, S.wr, num_sms, s)) != cudaSuccess) break;
    if ((e = deposit(S, x2, Mp2, g, false, false, S.wi, num_sms, s)) != cudaSuccess) break;
    overlap_sum_kernel<<<1, 32, 0, s>>>(S.wr, S.wi, S.m8 + 4, S.ncell);
    if ((e = cudaMemcpyAsync(&h_ov, S.m8 + 4, sizeof(double), cudaMemcpyDeviceToHost, s)) != cudaSuccess) break;
  } while (false);
  e = finish(S, e, s);
  if (e == cudaSuccess && degenerate) e = cudaErrorInvalidValue;
  if (e == cudaSuccess) *lumi_out = Ncoll * h_ov * (Np1 / (int)Mp1) * (Np2 / (int)Mp2) * freq / hx / hy / 10000;
  return e;
}

}  // namespace stb
