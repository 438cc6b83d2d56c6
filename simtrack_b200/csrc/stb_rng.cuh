// Counter-based normal deviates for quantum excitation (radiate1,
// simtrack.cpp:4236-4288).
//
// The reference draws them from GSL's default generator (gsl_ran_gaussian on
// gsl_r2, seeded 1324 in Init_GSL_Seeds, simtrack.cpp:317-329): one
// sequential stream for the whole process.  A GPU thread per particle needs
// a stream per particle instead, reproducible whatever the launch shape: the
// k-th draw of particle `id` is a pure function of (seed, id, k).
//
// Generator: Philox4x32-10 (J. K. Salmon, M. A. Moraes, R. O. Dror,
// D. E. Shaw, "Parallel random numbers: as easy as 1, 2, 3", SC'11): ten
// rounds of two 32x32->64-bit multiplies with the key bumped by the Weyl
// constants between rounds; counter = (k lo, k hi, id lo, id hi), key =
// (seed lo, seed hi).  Two 53-bit uniforms u1, u2 in (0, 1] from the four
// output words, then Box-Muller: g = sqrt(-2 ln u1) cos(2 pi u2).  Every
// step is IEEE basic arithmetic, the correctly rounded cos of stb_crmath.cuh
// and det_log below (a fixed sequence of basic operations), so host and
// device builds return the same bits.
#pragma once
#include <cstdint>

#include "stb_crmath.cuh"

namespace stb {

struct Philox4 {
  uint32_t v[4];
};

__host__ __device__ __forceinline__ Philox4 philox4x32_10(Philox4 c, uint32_t k0, uint32_t k1) {
#pragma unroll
  for (int r = 0; r < 10; r++) {
    if (r > 0) {
      k0 += 0x9E3779B9u;
      k1 += 0xBB67AE85u;
    }
    const uint64_t p0 = (uint64_t)0xD2511F53u * c.v[0];
    const uint64_t p1 = (uint64_t)0xCD9E8D57u * c.v[2];
    const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    c = Philox4{{hi1 ^ c.v[1] ^ k0, lo1, hi0 ^ c.v[3] ^ k1, lo0}};
  }
  return c;
}

// ln x for 0 < x <= 1 (normal x), about 1 ulp: x = m 2^e with m in
// [sqrt(1/2), sqrt(2)), ln m = 2 atanh(s), s = (m - 1)/(m + 1), |s| < 0.1716,
// from its series through s^23 (truncation below 2^-60 relative).
__host__ __device__ __forceinline__ double det_log(double x) {
  const uint64_t u = dbl_bits(x);
  int e = (int)((u >> 52) & 0x7ff) - 1023;
  double m = bits_dbl((u & 0xfffffffffffffull) | 0x3ff0000000000000ull);  // [1, 2)
  if (m > 1.4142135623730951) {
    m = m * 0.5;
    e = e + 1;
  }
  const double s = (m - 1.0) / (m + 1.0);
  const double t = s * s;
  double q = 1.0 / 23.0;
  q = q * t + 1.0 / 21.0;
  q = q * t + 1.0 / 19.0;
  q = q * t + 1.0 / 17.0;
  q = q * t + 1.0 / 15.0;
  q = q * t + 1.0 / 13.0;
  q = q * t + 1.0 / 11.0;
  q = q * t + 1.0 / 9.0;
  q = q * t + 1.0 / 7.0;
  q = q * t + 1.0 / 5.0;
  q = q * t + 1.0 / 3.0;
  const double lnm = 2.0 * s + 2.0 * s * (t * q);
  const double ln2_hi = 0.6931471805599453094, ln2_lo = 2.319046813846299558e-17;
  return (double)e * ln2_hi + ((double)e * ln2_lo + lnm);
}

// The k-th standard normal deviate of particle `id` under `seed`.
__host__ __device__ __forceinline__ double rad_gaussian(uint64_t seed, uint64_t id, uint64_t k) {
  const Philox4 r = philox4x32_10(Philox4{{(uint32_t)k, (uint32_t)(k >> 32), (uint32_t)id, (uint32_t)(id >> 32)}},
                                  (uint32_t)seed, (uint32_t)(seed >> 32));
  const uint64_t a = ((uint64_t)r.v[0] << 32) | r.v[1], b = ((uint64_t)r.v[2] << 32) | r.v[3];
  const double u1 = (double)((a >> 11) + 1) * 0x1p-53;  // (0, 1]
  const double u2 = (double)((b >> 11) + 1) * 0x1p-53;
  return sqrt(-2.0 * det_log(u1)) * cr_cos(6.283185307179586 * u2);
}

// The photon-emission draws of radiate2 (simtrack.cpp:4290-4372), which the
// reference takes from GSL (gsl_ran_poisson on gsl_r1, gsl_rng_uniform on
// gsl_r2): for radiating slice k of particle id, draw j = 0 is the uniform
// behind the photon count and draws j = 1, 2, ... the photons' uniforms.  The
// counter's second word has its top bit set, so these never coincide with
// the normal deviates above (whose second word is k's high half, below 2^31).
__host__ __device__ __forceinline__ double rad_uniform(uint64_t seed, uint64_t id, uint64_t k, uint32_t j) {
  const Philox4 r = philox4x32_10(Philox4{{(uint32_t)k, 0x80000000u | j, (uint32_t)id, (uint32_t)(id >> 32)}},
                                  (uint32_t)seed, (uint32_t)(seed >> 32));
  const uint64_t a = ((uint64_t)r.v[0] << 32) | r.v[1];
  return (double)((a >> 11) + 1) * 0x1p-53;  // (0, 1]
}

// Photon count with mean mu: inversion of the Poisson distribution
// (D. E. Knuth, TAOCP vol. 2, 3.4.1), the smallest n with u <= F(n),
// F summed term by term from exp(-mu); at most 1000.
__host__ __device__ __forceinline__ int rad_poisson(double u, double mu) {
  double term = cr_exp(-mu), cdf = term;
  int n = 0;
  while (u > cdf && n < 1000) {
    n = n + 1;
    term = term * mu / (double)n;
    cdf = cdf + term;
  }
  return n;
}

}  // namespace stb
