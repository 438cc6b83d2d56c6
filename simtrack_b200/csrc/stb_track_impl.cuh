// Device code of the element-by-element tracking kernels, shared by the
// single-lattice tracker (stb_track.cu), the batched scan (stb_scan.cu) and
// the spin tracker (stb_spin.cu).  Everything here has internal linkage.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "stb_kernels.hpp"
#include "stb_physics.cuh"
#include "stb_photon_spectrum.cuh"
#include "stb_rng.cuh"

namespace stb {
namespace {

constexpr double kPI = 3.14159265358979323;
constexpr double kC = 2.99792458e8;

// Bulk copy of `bytes` (multiple of 16, both addresses 16-byte aligned) from
// global to shared memory, completing on `bar`.
__device__ __forceinline__ void bulk_g2s(void *smem_dst, const void *gsrc, uint32_t bytes, uint64_t *bar) {
  const uint32_t d = (uint32_t)__cvta_generic_to_shared(smem_dst);
  const uint32_t b = (uint32_t)__cvta_generic_to_shared(bar);
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(d),
               "l"(gsrc), "r"(bytes), "r"(b)
               : "memory");
}

// Stage an element table (headers then pool) into shared memory with bulk
// copies completing on `bar`.  `phase` is the barrier phase this staging
// completes (0 for the first use of a freshly initialised barrier, then
// alternating).  Returns false if the bounded wait ran out (the caller then
// records STB_ETIMEOUT and returns).  Must be called by all threads of the CTA.
__device__ bool stage_table_ptr(const ElemHeader *ghdr, int nelem, const double *gpool, int npool_padded,
                                unsigned char *smem, uint64_t *bar, uint32_t phase, bool init) {
  const uint32_t hbytes = (uint32_t)nelem * (uint32_t)sizeof(ElemHeader);
  const uint32_t pbytes = (uint32_t)npool_padded * 8u;
  const uint32_t total = hbytes + pbytes;
  const uint32_t b = (uint32_t)__cvta_generic_to_shared(bar);
  if (init && threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(b) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    // Order earlier generic-proxy accesses of the buffer before the async copies.
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(b), "r"(total) : "memory");
    constexpr uint32_t kChunk = 32768;
    for (uint32_t off = 0; off < hbytes; off += kChunk) {
      const uint32_t n = (hbytes - off) < kChunk ? (hbytes - off) : kChunk;
      bulk_g2s(smem + off, (const unsigned char *)ghdr + off, n, bar);
    }
    for (uint32_t off = 0; off < pbytes; off += kChunk) {
      const uint32_t n = (pbytes - off) < kChunk ? (pbytes - off) : kChunk;
      bulk_g2s(smem + hbytes + off, (const unsigned char *)gpool + off, n, bar);
    }
  }
  // Bounded wait on the barrier phase; the CTA agrees on the outcome.
  uint32_t done = 0;
  for (int iter = 0; iter < (1 << 22); iter++) {
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(b), "r"(phase & 1u)
        : "memory");
    if (done) break;
  }
  return __syncthreads_and((int)done) != 0;
}

__device__ bool stage_table(const TrackArgs &a, unsigned char *smem, uint64_t *bar) {
  return stage_table_ptr(a.hdr, a.nelem, a.pool, a.npool_padded, smem, bar, 0, true);
}

// Segmented staging.  One thread issues the bulk copies of segment `sg`
// (its headers, then its pool slice) into `buf`, completing on `bar`.  Every
// copy starts on a 16-byte boundary and is a multiple of 16 bytes (headers
// are 32 bytes, pool_lo and pool_n are even).
__device__ __forceinline__ void issue_segment(const TrackArgs &a, const SegDesc &sg, unsigned char *buf,
                                              uint64_t *bar) {
  const uint32_t hbytes = (uint32_t)sg.ne * (uint32_t)sizeof(ElemHeader);
  const uint32_t pbytes = (uint32_t)sg.pool_n * 8u;
  const uint32_t b = (uint32_t)__cvta_generic_to_shared(bar);
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(b), "r"(hbytes + pbytes) : "memory");
  constexpr uint32_t kChunk = 32768;
  const unsigned char *gh = (const unsigned char *)(a.hdr + sg.e0);
  const unsigned char *gp = (const unsigned char *)(a.pool + sg.pool_lo);
  for (uint32_t off = 0; off < hbytes; off += kChunk)
    bulk_g2s(buf + off, gh + off, (hbytes - off) < kChunk ? (hbytes - off) : kChunk, bar);
  for (uint32_t off = 0; off < pbytes; off += kChunk)
    bulk_g2s(buf + hbytes + off, gp + off, (pbytes - off) < kChunk ? (pbytes - off) : kChunk, bar);
}

// Bounded wait of the calling thread for phase `phase` of `bar`.
__device__ __forceinline__ bool wait_phase(uint64_t *bar, uint32_t phase) {
  const uint32_t b = (uint32_t)__cvta_generic_to_shared(bar);
  uint32_t done = 0;
  for (int iter = 0; iter < (1 << 22) && !done; iter++) {
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(b), "r"(phase & 1u)
        : "memory");
  }
  return done != 0;
}

// Track()'s loss test (simtrack.cpp:20802): |x| > APx, |y| > APy or NaN;
// !(|x| <= APx) is true for NaN as well.  r2 is the circular aperture radius
// squared, +inf when there is none.
//
// loss_mode (uniform per launch, chosen on the host) drops the terms that
// cannot change the outcome: kLossCircle when the circle lies strictly inside
// every element's rectangle in rounded arithmetic (r2 < RN(APx^2), RN(APy^2):
// a point outside a rectangle is then outside the circle, and a NaN fails
// x^2 + y^2 <= r2), kLossRect when there is no circle (r2 = +inf, whose test
// never fires).
constexpr int kLossFull = 0, kLossCircle = 1, kLossRect = 2;
__device__ __forceinline__ bool is_lost(const Particle &p, double apx, double apy, double r2, int mode = kLossFull) {
  if (mode == kLossCircle) return !(p.x * p.x + p.y * p.y <= r2);
  if (mode == kLossRect) return !(fabs(p.x) <= apx) || !(fabs(p.y) <= apy);
  return !(fabs(p.x) <= apx) || !(fabs(p.y) <= apy) || p.x * p.x + p.y * p.y > r2;
}

__device__ __forceinline__ bool needs_loss_check(const ElemHeader &h) { return (h.flags & EF_NO_LOSS_CHECK) == 0; }

// The element maps are inlined into the kernels, the rare ones included: a
// call anywhere in a kernel makes the compiler keep an ABI stack frame and
// spill the live particle state around it, which costs the hot loop more
// (about 6 % of a RHIC-like turn, measured) than the larger instruction
// footprint of inlined rare maps.

__device__ __forceinline__ void op_gsbend(const ElemHeader &h, const double *P, Particle &p, const PtCache &c) {
  if (h.flags & EF_EDGE1) {
    p.px = p.px + P[0] * p.x;
    p.py = p.py - P[0] * p.y;
  }
  gbend_exact(p, c, P + 2);
  if (h.flags & EF_EDGE2) {
    p.px = p.px + P[1] * p.x;
    p.py = p.py - P[1] * p.y;
  }
}

template <int kOrder>
__device__ __forceinline__ void op_thick_sext_oct(const ElemHeader &h, const double *P, Particle &p, const PtCache &c) {
  const double d1 = P[0], d1b = P[1], d2 = P[2], d2b = P[3];
  const double a1 = P[4], s1 = P[5], a2 = P[6], s2 = P[7];
  DriftStep last = drift(p, c, d1, d1b);  // slice 0's opening drift
#pragma unroll 1
  for (int s = 0; s < h.nint; s++) {
    if (s > 0) drift_again(p, last);  // the same increments as the drift before it
    if (kOrder == 2) sext_kick(p, a1, s1); else oct_kick(p, a1, s1);
    drift(p, c, d2, d2b);
    if (kOrder == 2) sext_kick(p, a2, s2); else oct_kick(p, a2, s2);
    drift(p, c, d2, d2b);
    if (kOrder == 2) sext_kick(p, a1, s1); else oct_kick(p, a1, s1);
    last = drift(p, c, d1, d1b);
  }
}

__device__ __forceinline__ void op_mult_thick(const ElemHeader &h, const double *P, Particle &p, const PtCache &c) {
  const volatile double *V = P;
  const int no = h.aux;
  const double *K1 = P + 4;
  const double *K2 = K1 + 2 + 3 * no;
  DriftStep last = drift(p, c, V[0], V[1]);  // slice 0's opening drift
#pragma unroll 1
  for (int s = 0; s < h.nint; s++) {
    if (s > 0) drift_again(p, last);  // the same increments as the drift before it
    mult_kick(p, no, K1);
    drift(p, c, V[2], V[3]);
    mult_kick(p, no, K2);
    drift(p, c, V[2], V[3]);
    mult_kick(p, no, K1);
    last = drift(p, c, V[0], V[1]);
  }
}

__device__ __forceinline__ void op_bendmult(const ElemHeader &h, const double *P, Particle &p, const PtCache &c) {
  const int no = h.aux;
  const double *B1 = P + 2, *B2 = P + 8;
  const double *K1 = P + 14;
  const double *K2 = K1 + 2 + 3 * no;
  p.px = p.px + P[0] * p.x;
  p.py = p.py - P[0] * p.y;
#pragma unroll 1
  for (int s = 0; s < h.nint; s++) {
    bend_exact(p, c, B1);
    mult_kick(p, no, K1);
    bend_exact(p, c, B2);
    mult_kick(p, no, K2);
    bend_exact(p, c, B2);
    mult_kick(p, no, K1);
    bend_exact(p, c, B1);
  }
  p.px = p.px + P[1] * p.x;
  p.py = p.py - P[1] * p.y;
}

// Which particles a thread carries, for the normal-deviate streams of the
// radiating bends: particle k of the thread has id id0 + k * id_stride (its
// index in the caller's arrays); `turn` is the global turn.  Kernels that
// never see a radiating table pass the default.
struct RadKey {
  long id0 = 0, id_stride = 0;
  long turn = 0;
};

// SBEND_Pass, exact radiating branch (simtrack.cpp:4740-4748): Nint slices
// of sbend_exact_pass over Lint and Angle/Nint, each followed by radiate1
// with the field {0, Angle/Nint, 0}.  P = [tan(E1)h, tan(E2)h, slice bend
// (6), Lint, href, Angle/Nint, E3, Cf, first slice index within the turn].
__device__ __forceinline__ void op_sbend_rad(const ElemHeader &h, const double *P, Particle &p, PtCache &c,
                                             const RefConsts &R, long id, long turn) {
  if (h.flags & EF_EDGE1) {
    p.px = p.px + P[0] * p.x;
    p.py = p.py - P[0] * p.y;
  }
  const double Lint = P[8], href = P[9], an = P[10], E3 = P[11], Cf = P[12];
  const uint64_t k0 = (uint64_t)turn * (uint64_t)R.rad_slices + (uint64_t)P[13];
#pragma unroll 1
  for (int s = 0; s < h.nint; s++) {
    bend_exact(p, c, P + 2);
    const double g = rad_gaussian(R.rad_seed, (uint64_t)id, k0 + (uint64_t)s);
    radiate_step(p, c, R, Lint, href, 0., an, 0., E3, true, Cf, g);
  }
  if (h.flags & EF_EDGE2) {
    p.px = p.px + P[1] * p.x;
    p.py = p.py - P[1] * p.y;
  }
}

// GSBEND_Pass, exact radiating branch (simtrack.cpp:4866-4873): Nint slices
// of general_sbend_exact_pass over (Lint, Angle/Nint, K0L/Nint), each
// followed by radiate2 with the field {0, K0L/Nint, 0}.  P = [tan(E1)hreal,
// tan(E2)hreal, slice bend (9, as OP_GSBEND), href, K0L/Nint, facg, first
// slice index within the turn].
__device__ __forceinline__ void op_gsbend_rad(const ElemHeader &h, const double *P, Particle &p, PtCache &c,
                                              const RefConsts &R, long id, long turn) {
  if (h.flags & EF_EDGE1) {
    p.px = p.px + P[0] * p.x;
    p.py = p.py - P[0] * p.y;
  }
  const double Lint = P[2], href = P[11], kn = P[12], facg = P[13];
  const uint64_t k0 = (uint64_t)turn * (uint64_t)R.rad_slices + (uint64_t)P[14];
#pragma unroll 1
  for (int s = 0; s < h.nint; s++) {
    gbend_exact(p, c, P + 2);
    const uint64_t k = k0 + (uint64_t)s;
    radiate2_step(p, c, R, Lint, href, kn, facg, kPhotonU, kPhotonE, kPhotonTable,
                  [&](uint32_t j) { return rad_uniform(R.rad_seed, (uint64_t)id, k, j); });
  }
  if (h.flags & EF_EDGE2) {
    p.px = p.px + P[1] * p.x;
    p.py = p.py - P[1] * p.y;
  }
}

// GMULT_Pass / SBENDMULT_Pass, exact radiating branch (simtrack.cpp:
// 5312-5338, 5437-5463): each slice as in op_bendmult, then radiate() with
// the field of the element's own strengths at the slice's midpoint
// (cal_Bfield, 4169-4196).  P as OP_BENDMULT, then [block(KNL), Angle, Nint,
// Lint, href, E3].
__device__ __forceinline__ void op_bendmult_rad(const ElemHeader &h, const double *P, Particle &p, PtCache &c,
                                                const RefConsts &R) {
  const int no = h.aux, bs = 2 + 3 * no;
  const double *B1 = P + 2, *B2 = P + 8;
  const double *K1 = P + 14, *K2 = K1 + bs, *KR = K2 + bs;
  const double Angle = KR[bs], nd = KR[bs + 1], Lint = KR[bs + 2], href = KR[bs + 3], E3 = KR[bs + 4];
  p.px = p.px + P[0] * p.x;
  p.py = p.py - P[0] * p.y;
#pragma unroll 1
  for (int s = 0; s < h.nint; s++) {
    const Particle x1 = p;
    bend_exact(p, c, B1);
    mult_kick(p, no, K1);
    bend_exact(p, c, B2);
    mult_kick(p, no, K2);
    bend_exact(p, c, B2);
    mult_kick(p, no, K1);
    bend_exact(p, c, B1);
    double By, Bx;
    bfield_sum((p.x + x1.x) / 2., (p.y + x1.y) / 2., no, KR, By, Bx);
    radiate_step(p, c, R, Lint, href, Bx / nd, (Angle + By) / nd, 0., E3, false, 0., 0.);
  }
  p.px = p.px + P[1] * p.x;
  p.py = p.py - P[1] * p.y;
}

__device__ __forceinline__ void op_misc(const ElemHeader &h, const double *P, Particle &p, PtCache &c,
                                     const RefConsts &R) {
  switch (h.op) {
    case OP_OCT_KICK:
      oct_kick(p, P[0], P[1]);
      break;
    case OP_MULT_KICK:
      mult_kick(p, h.aux, P);
      break;
    case OP_KICK:
      drift(p, c, P[0], P[1]);
      p.px = p.px + P[2];
      p.py = p.py + P[3];
      drift(p, c, P[0], P[1]);
      break;
    case OP_RFCAV: {
      // RFCAV_Pass, simtrack.cpp:6008-6010
      drift(p, c, P[0], P[1]);
      const double absvq = P[2], kf = P[3], phase0 = P[4];
      p.pt = p.pt + absvq * cr_sin(kf * p.z / kC + kPI - phase0) / R.beta / R.energy;
      pt_refresh(R, p.pt, c);
      drift(p, c, P[0], P[1]);
      break;
    }
    case OP_CRABRF: {
      // CRABRF_Pass, simtrack.cpp:6020-6023
      drift(p, c, P[0], P[1]);
      const double vq = P[2], kf = P[3], phase0 = P[4], kk = P[5];
      const double arg = kf * p.z / kC + phase0;
      p.px = p.px - vq * cr_sin(arg) / R.beta / R.energy;
      p.pt = p.pt - vq * cr_cos(arg) * p.x * kk / R.beta / R.energy;
      pt_refresh(R, p.pt, c);
      drift(p, c, P[0], P[1]);
      break;
    }
    case OP_CCMULT:
      drift(p, c, P[0], P[1]);
      ccmult_kick(p, P + 2);
      pt_refresh(R, p.pt, c);
      drift(p, c, P[0], P[1]);
      break;
    case OP_LBT:
      lbt(p, P);
      pt_refresh(R, p.pt, c);
      break;
    case OP_ILBT:
      ilbt(p, P);
      pt_refresh(R, p.pt, c);
      break;
    case OP_BB6D:
      bb6d(p, P, h.nint);
      pt_refresh(R, p.pt, c);
      break;
    case OP_BB4D: {
      double Dpx, Dpy;
      bb4d(p.x, p.y, P[0], P[1], P[2], Dpx, Dpy);
      p.px = p.px + Dpx * P[3];
      p.py = p.py + Dpy * P[3];
      break;
    }
    case OP_PATCH:
      patch_map(p, c, P, h.aux != 0);
      break;
    case OP_SOLEN:
      solen_map(p, c, R, P, h.nint, [](double, double, double, double, double, double) {});
      break;
    default:  // OP_IDENTITY
      break;
  }
}

// Runs one element on the kPPT particles of this thread; the caller checks
// loss.  For the hot element types the per-particle maps are issued back to
// back, so their independent FP64 dependency chains interleave in the
// instruction stream (latency hiding without more resident warps).
// kRad: compile the radiating maps (GP.radiate tables); only the tracking
// kernel instantiation that such tables launch carries them, so the code of
// every other kernel stays as small as without radiation.
template <int kPPT, bool kLoopSlices = false, bool kRad = false>
__device__ __forceinline__ void apply_element(const ElemHeader &h, const double *P, Particle (&p)[kPPT],
                                              PtCache (&c)[kPPT], const RefConsts &R, const RadKey &rk = RadKey{}) {
  const double *M = P;
  const bool mis = (h.flags & (EF_MISALIGN_OFFSET | EF_MISALIGN_ROLL)) != 0;
  if (mis) {
#pragma unroll
    for (int k = 0; k < kPPT; k++) gtol1(p[k], M, h.flags);
    P += kMisalignParams;
  }
  switch (h.op) {
    case OP_DRIFT: {
      const double L = P[0], Lb = P[1];
#pragma unroll
      for (int k = 0; k < kPPT; k++) drift(p[k], c[k], L, Lb);
      break;
    }
    case OP_SBEND:
#pragma unroll
      for (int k = 0; k < kPPT; k++) {
        if (h.flags & EF_EDGE1) {
          p[k].px = p[k].px + P[0] * p[k].x;
          p[k].py = p[k].py - P[0] * p[k].y;
        }
        bend_exact(p[k], c[k], P + 2);
        if (h.flags & EF_EDGE2) {
          p[k].px = p[k].px + P[1] * p[k].x;
          p[k].py = p[k].py - P[1] * p[k].y;
        }
      }
      break;
    case OP_QUAD_THICK: {
      // Wide CTAs (few registers) re-read the slice constants from the table at
      // each use (volatile view) instead of holding eight register pairs; the
      // latency variants (up to 255 registers) keep them in registers.
      const double *V = P;
      const volatile double *VV = P;
      if (h.flags & EF_FRINGE)
        for (int k = 0; k < kPPT; k++) quad_fringe(p[k], P[8], true);
      // Slice s is d1 k1 d2 k2 d2 k1 d1.  The closing d1 of slice s and the
      // opening d1 of slice s+1 meet with no kick between them, so the second
      // adds the first one's increments again (drift_again), bit for bit what
      // recomputing them gives.
      DriftStep d1[kPPT];
#pragma unroll
      for (int k = 0; k < kPPT; k++) d1[k] = drift(p[k], c[k], V[0], V[1]);
      if (kLoopSlices) {
        // one copy of the drift code: smaller instruction footprint, better
        // for many resident warps; the unrolled form has the shorter latency
#pragma unroll 1
        for (int s = 0; s < h.nint; s++) {
#pragma unroll 1
          for (int q = 0; q < 3; q++) {
            const int kofs = (q == 1) ? 6 : 4;
            const int dofs = (q == 2) ? 0 : 2;
#pragma unroll
            for (int k = 0; k < kPPT; k++) quad_kick(p[k], VV[kofs], VV[kofs + 1]);
#pragma unroll
            for (int k = 0; k < kPPT; k++) d1[k] = drift(p[k], c[k], VV[dofs], VV[dofs + 1]);
          }
          if (s + 1 < h.nint) {
#pragma unroll
            for (int k = 0; k < kPPT; k++) drift_again(p[k], d1[k]);
          }
        }
      } else {
#pragma unroll 1
        for (int s = 0; s < h.nint; s++) {
#pragma unroll
          for (int k = 0; k < kPPT; k++) quad_kick(p[k], V[4], V[5]);
#pragma unroll
          for (int k = 0; k < kPPT; k++) drift(p[k], c[k], V[2], V[3]);
#pragma unroll
          for (int k = 0; k < kPPT; k++) quad_kick(p[k], V[6], V[7]);
#pragma unroll
          for (int k = 0; k < kPPT; k++) drift(p[k], c[k], V[2], V[3]);
#pragma unroll
          for (int k = 0; k < kPPT; k++) quad_kick(p[k], V[4], V[5]);
#pragma unroll
          for (int k = 0; k < kPPT; k++) d1[k] = drift(p[k], c[k], V[0], V[1]);
          if (s + 1 < h.nint) {
#pragma unroll
            for (int k = 0; k < kPPT; k++) drift_again(p[k], d1[k]);
          }
        }
      }
      if (h.flags & EF_FRINGE)
        for (int k = 0; k < kPPT; k++) quad_fringe(p[k], P[8], false);
      break;
    }
    case OP_QUAD_KICK:
#pragma unroll
      for (int k = 0; k < kPPT; k++) quad_kick(p[k], P[0], P[1]);
      break;
    case OP_SEXT_KICK:
#pragma unroll
      for (int k = 0; k < kPPT; k++) sext_kick(p[k], P[0], P[1]);
      break;
    case OP_GSBEND:
      for (int k = 0; k < kPPT; k++) op_gsbend(h, P, p[k], c[k]);
      break;
    case OP_SEXT_THICK:
      for (int k = 0; k < kPPT; k++) op_thick_sext_oct<2>(h, P, p[k], c[k]);
      break;
    case OP_OCT_THICK:
      for (int k = 0; k < kPPT; k++) op_thick_sext_oct<3>(h, P, p[k], c[k]);
      break;
    case OP_MULT_THICK:
      for (int k = 0; k < kPPT; k++) op_mult_thick(h, P, p[k], c[k]);
      break;
    case OP_BENDMULT:
      for (int k = 0; k < kPPT; k++) op_bendmult(h, P, p[k], c[k]);
      break;
    case OP_SBEND_RAD:
      if (kRad)
        for (int k = 0; k < kPPT; k++) op_sbend_rad(h, P, p[k], c[k], R, rk.id0 + (long)k * rk.id_stride, rk.turn);
      break;
    case OP_BENDMULT_RAD:
      if (kRad)
        for (int k = 0; k < kPPT; k++) op_bendmult_rad(h, P, p[k], c[k], R);
      break;
    case OP_GSBEND_RAD:
      if (kRad)
        for (int k = 0; k < kPPT; k++) op_gsbend_rad(h, P, p[k], c[k], R, rk.id0 + (long)k * rk.id_stride, rk.turn);
      break;
    default:
      for (int k = 0; k < kPPT; k++) op_misc(h, P, p[k], c[k], R);
      break;
  }
  if (mis) {
#pragma unroll
    for (int k = 0; k < kPPT; k++) ltog1(p[k], M, h.flags);
  }
}

__device__ __forceinline__ void store_particle(const TrackArgs &a, long i, const Particle &p) {
  a.x[i] = p.x;
  a.px[i] = p.px;
  a.y[i] = p.y;
  a.py[i] = p.py;
  a.z[i] = p.z;
  a.pt[i] = p.pt;
}

// Loads particle base + k*kBlock (k < kPPT) into registers, applying
// Track()'s entry check at turn 0; returns how many are alive.
template <int kBlock, int kPPT>
__device__ __forceinline__ int load_particles(const TrackArgs &a, long base, Particle (&p)[kPPT],
                                              PtCache (&c)[kPPT], bool (&alive)[kPPT]) {
  int nalive = 0;
#pragma unroll
  for (int k = 0; k < kPPT; k++) {
    const long i = base + (long)k * kBlock;
    alive[k] = i < a.n && a.lost_turn[i] < 0;
    p[k] = Particle{0., 0., 0., 0., 0., 0.};
    if (alive[k]) {
      p[k] = Particle{a.x[i], a.px[i], a.y[i], a.py[i], a.z[i], a.pt[i]};
      // Track()'s entry quick check, simtrack.cpp:20795-20796
      if (a.turn0 == 0 && (fabs(p[k].x) > 0.1 || fabs(p[k].y) > 0.1)) {
        a.lost_turn[i] = 0;
        a.lost_elem[i] = 0;
        alive[k] = false;
        p[k] = Particle{0., 0., 0., 0., 0., 0.};
      }
    }
    pt_refresh(a.ref, p[k].pt, c[k]);
    nalive += alive[k] ? 1 : 0;
  }
  return nalive;
}

// Loss bookkeeping after global element e of turn t (see track_kernel).
template <int kBlock, int kPPT, bool kDump>
__device__ __forceinline__ void after_element(const TrackArgs &a, const ElemHeader &h, long base, int t, int e,
                                              Particle (&p)[kPPT], PtCache (&c)[kPPT], bool (&alive)[kPPT],
                                              int &nalive) {
#pragma unroll
  for (int k = 0; k < kPPT; k++) {
    if (!alive[k]) continue;
    const long i = base + (long)k * kBlock;
    if (kDump) {
      double *d = a.dump + (((size_t)i * a.nturn + t) * a.nelem + e) * 6;
      d[0] = p[k].x; d[1] = p[k].px; d[2] = p[k].y; d[3] = p[k].py; d[4] = p[k].z; d[5] = p[k].pt;
    }
    if (needs_loss_check(h) && is_lost(p[k], h.apx, h.apy, a.r2, a.loss_mode)) {
      store_particle(a, i, p[k]);
      a.lost_turn[i] = a.turn0 + t;
      a.lost_elem[i] = e;
      alive[k] = false;
      nalive--;
      p[k] = Particle{0., 0., 0., 0., 0., 0.};
      pt_refresh(a.ref, 0.0, c[k]);
    }
  }
}

// The segmented form of track_kernel (kSeg).  Step s of this CTA's sequence
// tracks segment s % nseg from buffer s & 1; buffer b's mbarrier completes
// once per staging, so its parity alternates with every use.
template <int kBlock, int kPPT, bool kDump, bool kRad>
__device__ void track_segmented(const TrackArgs &a, unsigned char *smem, uint64_t *sbar) {
  const long chunk = (long)kBlock * kPPT;
  const long stride = (long)gridDim.x * chunk;
  const long first = (long)blockIdx.x * chunk;
  const long my_chunks = first < a.n ? (a.n - first + stride - 1) / stride : 0;
  const int nseg = a.nseg;
  const long total = my_chunks * (long)a.nturn * nseg;
  if (total == 0) return;
  unsigned char *buf[2] = {smem, smem + a.seg_bytes};
  if (threadIdx.x == 0) {
    for (int b = 0; b < 2; b++) {
      const uint32_t ba = (uint32_t)__cvta_generic_to_shared(&sbar[b]);
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(ba) : "memory");
    }
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    issue_segment(a, a.segs[0], buf[0], &sbar[0]);
    if (total > 1) issue_segment(a, a.segs[1 % nseg], buf[1], &sbar[1]);
  }
  uint32_t phase[2] = {0u, 0u};
  long step = 0;
  const RefConsts &R = a.ref;
  for (long base = first + threadIdx.x; step < total; base += stride) {
    Particle p[kPPT];
    PtCache c[kPPT];
    bool alive[kPPT];
    int nalive = load_particles<kBlock, kPPT>(a, base, p, c, alive);
    for (int t = 0; t < a.nturn; t++) {
      for (int k = 0; k < nseg; k++, step++) {
        const int b = (int)(step & 1);
        const bool ok = wait_phase(&sbar[b], phase[b]);
        phase[b] ^= 1u;
        if (!__syncthreads_and((int)ok)) {
          // give the copies in flight a bounded time to land before the CTA exits
          if (threadIdx.x == 0) {
            atomicExch(a.status, STB_ETIMEOUT);
            wait_phase(&sbar[b ^ 1], phase[b ^ 1]);
          }
          __syncthreads();
          return;
        }
        const SegDesc sg = a.segs[k];
        const ElemHeader *hs = reinterpret_cast<const ElemHeader *>(buf[b]);
        const double *ps = reinterpret_cast<const double *>(buf[b] + (size_t)sg.ne * sizeof(ElemHeader));
        if (nalive > 0) {
          for (int j = 0; j < sg.ne; j++) {
            const ElemHeader h = hs[j];
            apply_element<kPPT, (kBlock >= 512), kRad>(h, ps + (h.poff - sg.pool_lo), p, c, R,
                                                 RadKey{base, kBlock, (long)a.turn0 + t});
            after_element<kBlock, kPPT, kDump>(a, h, base, t, sg.e0 + j, p, c, alive, nalive);
            if (nalive == 0) break;
          }
        }
        __syncthreads();  // every thread is done with buffer b
        if (threadIdx.x == 0 && step + 2 < total) issue_segment(a, a.segs[(step + 2) % nseg], buf[b], &sbar[b]);
      }
    }
#pragma unroll
    for (int k = 0; k < kPPT; k++)
      if (alive[k]) store_particle(a, base + (long)k * kBlock, p[k]);
  }
}

// kPPT particles per thread: particle base + k*kBlock for k < kPPT, so every
// load and store of a warp stays coalesced.  A particle that is lost has its
// coordinates and loss record stored at once; its slot is then reset to the
// reference orbit so the remaining particles of the thread keep running on
// benign operands.
//
// kSeg (with kSmem): the table is staged segment by segment into two
// shared-memory buffers, the next segment's bulk copy running while the
// current one is tracked.  The whole CTA walks the same sequence of
// (particle chunk, turn, segment) steps in lockstep: a barrier after every
// segment frees its buffer for the copy two steps ahead.  Threads whose
// particles are lost (or that have none) keep taking part in the barriers.
template <bool kSmem, int kBlock, int kMinBlocks, int kPPT, bool kDump, bool kPF = false, bool kSeg = false,
          bool kRad = false>
__global__ void __launch_bounds__(kBlock, kMinBlocks) track_kernel(const __grid_constant__ TrackArgs a) {
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ __align__(8) uint64_t bar;
  __shared__ __align__(8) uint64_t sbar[2];
  const ElemHeader *hdr = a.hdr;
  const double *pool = a.pool;
  if (kSeg) {
    track_segmented<kBlock, kPPT, kDump, kRad>(a, smem, sbar);
    return;
  }
  if (kSmem) {
    if (!stage_table(a, smem, &bar)) {
      if (threadIdx.x == 0) atomicExch(a.status, STB_ETIMEOUT);
      return;
    }
    hdr = reinterpret_cast<const ElemHeader *>(smem);
    pool = reinterpret_cast<const double *>(smem + (size_t)a.nelem * sizeof(ElemHeader));
  }
  const RefConsts &R = a.ref;
  const long chunk = (long)kBlock * kPPT;
  const long stride = (long)gridDim.x * chunk;
  for (long base = (long)blockIdx.x * chunk + threadIdx.x; base < a.n; base += stride) {
    Particle p[kPPT];
    PtCache c[kPPT];
    bool alive[kPPT];
    int nalive = 0;
#pragma unroll
    for (int k = 0; k < kPPT; k++) {
      const long i = base + (long)k * kBlock;
      alive[k] = i < a.n && a.lost_turn[i] < 0;
      p[k] = Particle{0., 0., 0., 0., 0., 0.};
      if (alive[k]) {
        p[k].x = a.x[i];
        p[k].px = a.px[i];
        p[k].y = a.y[i];
        p[k].py = a.py[i];
        p[k].z = a.z[i];
        p[k].pt = a.pt[i];
        // Track()'s entry quick check, simtrack.cpp:20795-20796
        if (a.turn0 == 0 && (fabs(p[k].x) > 0.1 || fabs(p[k].y) > 0.1)) {
          a.lost_turn[i] = 0;
          a.lost_elem[i] = 0;
          alive[k] = false;
          p[k] = Particle{0., 0., 0., 0., 0., 0.};
        }
      }
      pt_refresh(R, p[k].pt, c[k]);
      nalive += alive[k] ? 1 : 0;
    }
    for (int t = 0; t < a.nturn && nalive > 0; t++) {
      ElemHeader hnext;
      if (kPF) hnext = hdr[0];
      for (int e = 0; e < a.nelem; e++) {
        ElemHeader h;
        if (kPF) {
          // the next header's shared-memory load overlaps this element's maps
          h = hnext;
          if (e + 1 < a.nelem) hnext = hdr[e + 1];
        } else {
          h = hdr[e];
        }
        apply_element<kPPT, (kBlock >= 512), kRad>(h, pool + h.poff, p, c, R,
                                                   RadKey{base, kBlock, (long)a.turn0 + t});
#pragma unroll
        for (int k = 0; k < kPPT; k++) {
          if (!alive[k]) continue;
          const long i = base + (long)k * kBlock;
          if (kDump) {
            double *d = a.dump + (((size_t)i * a.nturn + t) * a.nelem + e) * 6;
            d[0] = p[k].x; d[1] = p[k].px; d[2] = p[k].y; d[3] = p[k].py; d[4] = p[k].z; d[5] = p[k].pt;
          }
          if (needs_loss_check(h) && is_lost(p[k], h.apx, h.apy, a.r2, a.loss_mode)) {
            store_particle(a, i, p[k]);
            a.lost_turn[i] = a.turn0 + t;
            a.lost_elem[i] = e;
            alive[k] = false;
            nalive--;
            p[k] = Particle{0., 0., 0., 0., 0., 0.};
            pt_refresh(R, 0.0, c[k]);
          }
        }
        // a thread whose particles are all lost finishes the turn on benign
        // operands and stops at the turn boundary (no per-element test)
      }
    }
#pragma unroll
    for (int k = 0; k < kPPT; k++)
      if (alive[k]) store_particle(a, base + (long)k * kBlock, p[k]);
  }
}

}  // namespace
}  // namespace stb
