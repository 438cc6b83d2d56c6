// Spin tracking: Track_Spin (simtrack.cpp:21766-21789) on the GPU.
//
// One thread carries one particle: the six orbit coordinates and the spin
// unit vector (x[6..8] of the reference's x[9]).  Elements whose
// Element::sPass equals their Pass run the orbit maps of the plain tracker
// (apply_element); the OP_S_* forms interleave the orbit slices with the
// Thomas-BMT rotation spin() (simtrack.cpp:4574-4630): after every slice
// the spin turns about the field integrated over the slice, evaluated at the
// slice's midpoint coordinates, with the direction of motion and energy
// taken at the slice's start, exactly as the reference orders it.
//
// Parameter layouts of the spin opcodes (after the optional misalignment
// block [dx, dy, cos(dpsi), sin(dpsi)]), as stb_flatten.cpp writes them:
//   OP_S_SBEND          [tan(E1)h, tan(E2)h, sub-bend(6), Angle/Nint, Angle/L (, E3 with EF_RADIATE)]
//   OP_S_MPOLE_THICK    [d1, d1/b, d2, d2/b, k1 kick pair, k2 kick pair, KL, KSL, Nint]   aux = order
//   OP_S_MPOLE_KICK     [KL, KSL, Nint]                                                 aux = order
//   OP_S_MULT_THICK     [d1, d1/b, d2, d2/b, block(k1), block(k2), block(KNL), Nint]     aux = Norder
//   OP_S_MULT_KICK      [block(KNL)]                                                    aux = Norder
//   OP_S_BENDMULT       [tan(E1)h, tan(E2)h, bend(d1), bend(d2), block(k1), block(k2), block(KNL),
//                        Angle/Nint, Angle/L, Angle, Nint (, Lint, E3 with EF_RADIATE)]  aux = Norder
//   OP_S_BENDMULT_KICK  [block(KNL), Angle]                                             aux = Norder
//   OP_S_KICK           [L/2, L/2/b, HKICK, VKICK]
//   OP_S_SOLEN          [q*Bz/2, L, Nint, L/Nint, L/beta/c, m0, p0, Bz*(L/Nint)/brho]  (Bz = KS*brho/L)
// where a block is [KNL0, KNSL0, (KNLi, KNSLi, 1/i!) i = 1..Norder].
#include <cuda_runtime.h>

#include <cstdint>

#include "stb_track_impl.cuh"

namespace stb {
namespace {

struct Spin {
  double x, y, z;
};

// spin(), simtrack.cpp:4574-4630.  x0: coordinates at the start of the step
// (direction of motion, pt, horizontal offset); c: the pt cache of x0;
// angle, href: the reference orbit's bend angle and curvature over the step;
// B: the integrated field over (B rho)_0.  Rotates s in place.
__device__ __forceinline__ void spin_rotate(const Particle &x0, const PtCache &c, const RefConsts &R, double angle,
                                            double href, double B0, double B1, double B2, Spin &s) {
  if (!(B0 * B0 + B1 * B1 + B2 * B2 != 0.)) return;
  const double gamma1 = R.gamma + R.sqrt_g2m1 * x0.pt;
  const double Gr = R.G * gamma1;
  // Quotients by a shared divisor use its reciprocal and the one-FMA
  // correction (qdiv); the square roots and their reciprocals come from
  // seeds close to them (1/(1+delta) for the longitudinal momentum, 1 for
  // the norm of (px/pz, py/pz, 1)), IEEE sqrt and division for steep slopes.
  double temp, itemp;
  if (!seeded_sqrt_recip(c.opd2 - x0.px * x0.px - x0.py * x0.py, c.iopd, x0.px, x0.py, temp, itemp)) {
    temp = sqrt(c.opd2 - x0.px * x0.px - x0.py * x0.py);
    itemp = 1.0 / temp;
  }
  double u0 = qdiv(x0.px, temp, itemp), u1 = qdiv(x0.py, temp, itemp), u2 = 1.0;
  double itemp2;
  if (!seeded_sqrt_recip(u0 * u0 + u1 * u1 + u2 * u2, 1.0, u0, u1, temp, itemp2)) {
    temp = sqrt(u0 * u0 + u1 * u1 + u2 * u2);
    itemp2 = 1.0 / temp;
  }
  u0 = qdiv(u0, temp, itemp2);
  u1 = qdiv(u1, temp, itemp2);
  u2 = qdiv(u2, temp, itemp2);
  temp = (1 + href * x0.x) * temp;
  const double udotB = u0 * B0 + u1 * B1 + u2 * B2;
  const double g1 = 1 + Gr, g2 = R.G * (1 - gamma1);
  double F0 = g1 * B0 + g2 * (udotB * u0);
  double F1 = g1 * B1 + g2 * (udotB * u1);
  double F2 = g1 * B2 + g2 * (udotB * u2);
  F0 = qdiv(F0 * temp, c.opd, c.iopd);
  F1 = qdiv(F1 * temp, c.opd, c.iopd);
  F2 = qdiv(F2 * temp, c.opd, c.iopd);
  F1 = F1 - angle;
  const double Fabs = sqrt(F0 * F0 + F1 * F1 + F2 * F2);
  const double iFabs = 1.0 / Fabs;
  const double a0 = qdiv(F0, Fabs, iFabs), a1 = qdiv(F1, Fabs, iFabs), a2 = qdiv(F2, Fabs, iFabs);
  const double theta = -Fabs;
  double st, ct;
  cr_sincos(theta, st, ct);
  const double r0 = a0 * a0 * (1 - ct) + ct;
  const double r1 = a0 * a1 * (1 - ct) - a2 * st;
  const double r2 = a0 * a2 * (1 - ct) + a1 * st;
  const double r3 = a0 * a1 * (1 - ct) + a2 * st;
  const double r4 = a1 * a1 * (1 - ct) + ct;
  const double r5 = a1 * a2 * (1 - ct) - a0 * st;
  const double r6 = a0 * a2 * (1 - ct) - a1 * st;
  const double r7 = a1 * a2 * (1 - ct) + a0 * st;
  const double r8 = a2 * a2 * (1 - ct) + ct;
  double n0 = 0.;
  n0 = n0 + r0 * s.x;
  n0 = n0 + r1 * s.y;
  n0 = n0 + r2 * s.z;
  double n1 = 0.;
  n1 = n1 + r3 * s.x;
  n1 = n1 + r4 * s.y;
  n1 = n1 + r5 * s.z;
  double n2 = 0.;
  n2 = n2 + r6 * s.x;
  n2 = n2 + r7 * s.y;
  n2 = n2 + r8 * s.z;
  s.x = n0;
  s.y = n1;
  s.z = n2;
}

// The field sum of cal_Bfield / mult_kick_pass (simtrack.cpp:4169-4196):
// By + i Bx of the multipole block K at (x, y).
__device__ __forceinline__ void mult_field(double x, double y, int norder, const double *K, double &By, double &Bx) {
  double Xn = 1., Yn = 0.;
  By = K[0];
  Bx = K[1];
  double fac = 1.;
#pragma unroll 1
  for (int i = 1; i <= norder; i++) {
    const double Xn0 = Xn, Yn0 = Yn;
    Xn = Xn0 * x - Yn0 * y;
    Yn = Xn0 * y + Yn0 * x;
    fac = fac * (double)i;
    const double kn = K[3 * i - 1], ks = K[3 * i], ifac = K[3 * i + 1];
    if (kn != 0. || ks != 0.) {
      By = By + qdiv(kn * Xn - ks * Yn, fac, ifac);
      Bx = Bx + qdiv(kn * Yn + ks * Xn, fac, ifac);
    }
  }
}

__device__ __forceinline__ void mpole_kick(Particle &p, int order, double kl, double ksl) {
  if (order == 1) quad_kick(p, kl, ksl);
  else if (order == 2) sext_kick(p, kl, ksl);
  else oct_kick(p, kl, ksl);
}

// Field of a thin or sliced quadrupole / sextupole / octupole from the
// midpoint coordinates (QUAD_sPass 7563-7567 / 7580-7584, SEXT_sPass
// 7609-7612 / 7635-7638, OCT_sPass 7663-7666 / 7689-7692).
__device__ __forceinline__ void mpole_field(int order, bool thick, double x1, double y1, double kl, double ksl,
                                            double nd, double &B0, double &B1) {
  if (order == 1) {
    const double preal = x1, pimag = y1;
    B0 = ksl * preal + kl * pimag;
    B1 = kl * preal - ksl * pimag;
    if (thick) {
      B0 = B0 / nd;
      B1 = B1 / nd;
    }
  } else if (order == 2) {
    const double preal = x1 * x1 - y1 * y1;
    const double pimag = 2. * x1 * y1;
    B0 = (ksl * preal + kl * pimag) / 2.;
    B1 = (kl * preal - ksl * pimag) / 2.;
    if (thick) {
      B0 = B0 / nd;
      B1 = B1 / nd;
    }
  } else {
    const double preal = x1 * x1 * x1 - 3 * x1 * y1 * y1;
    const double pimag = 3 * x1 * x1 * y1 - y1 * y1 * y1;
    B0 = (ksl * preal + kl * pimag) / 6 / nd;  // the reference divides by Nint in both branches
    B1 = (kl * preal - ksl * pimag) / 6 / nd;
  }
}

// One spin-opcode element (after the misalignment entrance transform).
// kRad: compile radiate() after the slice rotations of the bends (tables
// flattened with GP.radiate run the one kernel instantiation that has it).
template <bool kRad>
__device__ __forceinline__ void spin_element(const ElemHeader &h, const double *P, Particle &p, Spin &s, PtCache &c,
                                             const RefConsts &R) {
  switch (h.op) {
    case OP_S_SBEND: {
      p.px = p.px + P[0] * p.x;
      p.py = p.py - P[0] * p.y;
      const double an = P[8], href = P[9];
#pragma unroll 1
      for (int i = 0; i < h.nint; i++) {
        const Particle x0 = p;
        bend_exact(p, c, P + 2);
        spin_rotate(x0, c, R, an, href, 0., an, 0., s);
        if (kRad && (h.flags & EF_RADIATE)) radiate_step(p, c, R, P[2], href, 0., an, 0., P[10], false, 0., 0.);
      }
      p.px = p.px + P[1] * p.x;
      p.py = p.py - P[1] * p.y;
      break;
    }
    case OP_S_MPOLE_THICK: {
      const int order = h.aux;
      const double kl = P[8], ksl = P[9], nd = P[10];
#pragma unroll 1
      for (int i = 0; i < h.nint; i++) {
        const Particle x0 = p;
        drift(p, c, P[0], P[1]);
        mpole_kick(p, order, P[4], P[5]);
        drift(p, c, P[2], P[3]);
        mpole_kick(p, order, P[6], P[7]);
        drift(p, c, P[2], P[3]);
        mpole_kick(p, order, P[4], P[5]);
        drift(p, c, P[0], P[1]);
        const double x1 = (p.x + x0.x) / 2., y1 = (p.y + x0.y) / 2.;
        double B0, B1;
        mpole_field(order, true, x1, y1, kl, ksl, nd, B0, B1);
        spin_rotate(x0, c, R, 0., 0., B0, B1, 0., s);
      }
      break;
    }
    case OP_S_MPOLE_KICK: {
      const Particle x0 = p;
      mpole_kick(p, h.aux, P[0], P[1]);
      const double x1 = (p.x + x0.x) / 2., y1 = (p.y + x0.y) / 2.;
      double B0, B1;
      mpole_field(h.aux, false, x1, y1, P[0], P[1], P[2], B0, B1);
      spin_rotate(x0, c, R, 0., 0., B0, B1, 0., s);
      break;
    }
    case OP_S_MULT_KICK: {
      double By, Bx;
      mult_field(p.x, p.y, h.aux, P, By, Bx);
      spin_rotate(p, c, R, 0., 0., Bx / 1.0, (0. + By) / 1.0, 0., s);
      mult_kick(p, h.aux, P);
      break;
    }
    case OP_S_MULT_THICK: {
      const int no = h.aux, bs = 2 + 3 * no;
      const double *K1 = P + 4, *K2 = K1 + bs, *KR = K2 + bs;
      const double nd = KR[bs];
#pragma unroll 1
      for (int i = 0; i < h.nint; i++) {
        const Particle x0 = p;
        drift(p, c, P[0], P[1]);
        mult_kick(p, no, K1);
        drift(p, c, P[2], P[3]);
        mult_kick(p, no, K2);
        drift(p, c, P[2], P[3]);
        mult_kick(p, no, K1);
        drift(p, c, P[0], P[1]);
        const double x1 = (p.x + x0.x) / 2., y1 = (p.y + x0.y) / 2.;
        double By, Bx;
        mult_field(x1, y1, no, KR, By, Bx);
        spin_rotate(x0, c, R, 0., 0., Bx / nd, (0. + By) / nd, 0., s);
      }
      break;
    }
    case OP_S_BENDMULT: {
      const int no = h.aux, bs = 2 + 3 * no;
      const double *B1 = P + 2, *B2 = P + 8;
      const double *K1 = P + 14, *K2 = K1 + bs, *KR = K2 + bs;
      const double an = KR[bs], href = KR[bs + 1], Angle = KR[bs + 2], nd = KR[bs + 3];
      p.px = p.px + P[0] * p.x;
      p.py = p.py - P[0] * p.y;
#pragma unroll 1
      for (int i = 0; i < h.nint; i++) {
        const Particle x0 = p;
        bend_exact(p, c, B1);
        mult_kick(p, no, K1);
        bend_exact(p, c, B2);
        mult_kick(p, no, K2);
        bend_exact(p, c, B2);
        mult_kick(p, no, K1);
        bend_exact(p, c, B1);
        const double x1 = (p.x + x0.x) / 2., y1 = (p.y + x0.y) / 2.;
        double By, Bx;
        mult_field(x1, y1, no, KR, By, Bx);
        const double B0 = Bx / nd, B1 = (Angle + By) / nd;
        spin_rotate(x0, c, R, an, href, B0, B1, 0., s);
        if (kRad && (h.flags & EF_RADIATE))
          radiate_step(p, c, R, KR[bs + 4], href, B0, B1, 0., KR[bs + 5], false, 0., 0.);
      }
      p.px = p.px + P[1] * p.x;
      p.py = p.py - P[1] * p.y;
      break;
    }
    case OP_S_BENDMULT_KICK: {
      const int no = h.aux;
      const double Angle = P[2 + 3 * no];
      const Particle x0 = p;
      mult_kick(p, no, P);
      const double x1 = (p.x + x0.x) / 2., y1 = (p.y + x0.y) / 2.;
      double By, Bx;
      mult_field(x1, y1, no, P, By, Bx);
      spin_rotate(x0, c, R, Angle, 0., Bx / 1.0, (Angle + By) / 1.0, 0., s);
      break;
    }
    case OP_S_KICK: {
      drift(p, c, P[0], P[1]);
      spin_rotate(p, c, R, 0., 0., P[3], -P[2], 0., s);
      p.px = p.px + P[2];
      p.py = p.py + P[3];
      drift(p, c, P[0], P[1]);
      break;
    }
    case OP_S_SOLEN: {
      // SOLEN_sPass, simtrack.cpp:8118-8183: before every slice the spin turns
      // about the longitudinal field integrated over the slice, with the
      // slice's entry state (momenta converted back to px, py).
      const double m0 = P[5], p0 = P[6], B2 = P[7];
      const double z = p.z, pt = p.pt;
      solen_map(p, c, R, P, h.nint, [&](double t0, double t1, double t2, double t3, double gamma1, double vz) {
        const Particle xs{t0, gamma1 * m0 * t1 * vz / p0, t2, gamma1 * m0 * t3 * vz / p0, z, pt};
        spin_rotate(xs, c, R, 0., 0., 0., 0., B2, s);
      });
      break;
    }
    default:
      break;
  }
}

template <bool kSmem, int kBlock, int kMinBlocks, bool kDump, bool kRad = false>
__global__ void __launch_bounds__(kBlock, kMinBlocks) spin_track_kernel(const __grid_constant__ SpinArgs sa) {
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ __align__(8) uint64_t bar;
  const TrackArgs &a = sa.t;
  const ElemHeader *hdr = a.hdr;
  const double *pool = a.pool;
  if (kSmem) {
    if (!stage_table(a, smem, &bar)) {
      if (threadIdx.x == 0) atomicExch(a.status, STB_ETIMEOUT);
      return;
    }
    hdr = reinterpret_cast<const ElemHeader *>(smem);
    pool = reinterpret_cast<const double *>(smem + (size_t)a.nelem * sizeof(ElemHeader));
  }
  const RefConsts &R = a.ref;
  for (long i = (long)blockIdx.x * kBlock + threadIdx.x; i < a.n; i += (long)gridDim.x * kBlock) {
    if (a.lost_turn[i] >= 0) continue;
    Particle p[1];
    PtCache c[1];
    p[0] = Particle{a.x[i], a.px[i], a.y[i], a.py[i], a.z[i], a.pt[i]};
    Spin s{sa.sx[i], sa.sy[i], sa.sz[i]};
    // Track_Spin()'s entry quick check, simtrack.cpp:21770-21772
    if (a.turn0 == 0 && (fabs(p[0].x) > 0.1 || fabs(p[0].y) > 0.1)) {
      a.lost_turn[i] = 0;
      a.lost_elem[i] = 0;
      continue;
    }
    pt_refresh(R, p[0].pt, c[0]);
    int lt = -1, le = 0;
    for (int t = 0; t < a.nturn && lt < 0; t++) {
      for (int e = 0; e < a.nelem; e++) {
        const ElemHeader h = hdr[e];
        const double *P = pool + h.poff;
        if (h.op >= OP_S_FIRST && h.op <= OP_S_LAST) {
          const double *M = P;
          const bool mis = (h.flags & (EF_MISALIGN_OFFSET | EF_MISALIGN_ROLL)) != 0;
          if (mis) {
            gtol1(p[0], M, h.flags);
            P += kMisalignParams;
          }
          spin_element<kRad>(h, P, p[0], s, c[0], R);
          if (mis) ltog1(p[0], M, h.flags);
        } else {
          apply_element<1>(h, P, p, c, R);
        }
        if (kDump) {
          double *d = sa.dump + (((size_t)i * a.nturn + t) * a.nelem + e) * 9;
          d[0] = p[0].x; d[1] = p[0].px; d[2] = p[0].y; d[3] = p[0].py; d[4] = p[0].z; d[5] = p[0].pt;
          d[6] = s.x; d[7] = s.y; d[8] = s.z;
        }
        if (needs_loss_check(h) && is_lost(p[0], h.apx, h.apy, a.r2, a.loss_mode)) {
          lt = a.turn0 + t;
          le = e;
          break;
        }
      }
    }
    a.x[i] = p[0].x;
    a.px[i] = p[0].px;
    a.y[i] = p[0].y;
    a.py[i] = p[0].py;
    a.z[i] = p[0].z;
    a.pt[i] = p[0].pt;
    sa.sx[i] = s.x;
    sa.sy[i] = s.y;
    sa.sz[i] = s.z;
    if (lt >= 0) {
      a.lost_turn[i] = lt;
      a.lost_elem[i] = le;
    }
  }
}

template <bool kSmem, int kBlock, int kMinBlocks, bool kDump, bool kRad = false>
cudaError_t launch_spin_variant(const SpinArgs &a, int num_sms, size_t smem, cudaStream_t stream) {
  auto kern = spin_track_kernel<kSmem, kBlock, kMinBlocks, kDump, kRad>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kBlock, smem);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) return cudaErrorInvalidConfiguration;
  long need = (a.t.n + kBlock - 1) / kBlock;
  long grid = (long)num_sms * per_sm;
  if (grid > need) grid = need;
  if (grid < 1) grid = 1;
  kern<<<(unsigned)grid, kBlock, smem, stream>>>(a);
  return cudaGetLastError();
}

}  // namespace

// Launch variants of the spin kernel the autotuner chooses from: the element
// table staged in shared memory (one CTA per SM) or read through L1; CTA
// size and minimum resident CTAs (registers per thread = 65536 / (block *
// min_blocks)).  Small CTAs spread a few thousand particles per seed over
// every SM when several seeds run side by side on their own streams.
const SpinVariant kSpinVariants[kNumSpinVariants] = {
    {true, 512, 1, "smem_b512_r128"}, {true, 1024, 1, "smem_b1024_r64"}, {true, 768, 1, "smem_b768_r85"},
    {false, 256, 2, "l1_b256_r128"},  {false, 256, 3, "l1_b256_r80"},    {false, 256, 4, "l1_b256_r64"},
    {false, 128, 4, "l1_b128_r128"},  {false, 64, 8, "l1_b64_r128"},     {false, 64, 12, "l1_b64_r85"},
    {false, 64, 4, "l1_b64_r255"},    {false, 128, 2, "l1_b128_r255"},   {true, 256, 1, "smem_b256_r255"},
};

cudaError_t launch_spin(const SpinArgs &a, int num_sms, int variant, cudaStream_t stream) {
  if (a.t.n <= 0 || a.t.nturn <= 0) return cudaSuccess;
  if (a.dump) return launch_spin_variant<false, 128, 1, true, true>(a, num_sms, 0, stream);
  // tables flattened with GP.radiate: the instantiation with radiate() (the
  // shape of l1_b128_r255), whatever the variant
  if (a.radiate) return launch_spin_variant<false, 128, 2, false, true>(a, num_sms, 0, stream);
  const size_t sm = track_smem_bytes(a.t.nelem, a.t.npool_padded);
  switch (variant) {
    case 0: return launch_spin_variant<true, 512, 1, false>(a, num_sms, sm, stream);
    case 1: return launch_spin_variant<true, 1024, 1, false>(a, num_sms, sm, stream);
    case 2: return launch_spin_variant<true, 768, 1, false>(a, num_sms, sm, stream);
    case 3: return launch_spin_variant<false, 256, 2, false>(a, num_sms, 0, stream);
    case 4: return launch_spin_variant<false, 256, 3, false>(a, num_sms, 0, stream);
    case 5: return launch_spin_variant<false, 256, 4, false>(a, num_sms, 0, stream);
    case 6: return launch_spin_variant<false, 128, 4, false>(a, num_sms, 0, stream);
    case 7: return launch_spin_variant<false, 64, 8, false>(a, num_sms, 0, stream);
    case 8: return launch_spin_variant<false, 64, 12, false>(a, num_sms, 0, stream);
    case 9: return launch_spin_variant<false, 64, 4, false>(a, num_sms, 0, stream);
    case 10: return launch_spin_variant<false, 128, 2, false>(a, num_sms, 0, stream);
    case 11: return launch_spin_variant<true, 256, 1, false>(a, num_sms, sm, stream);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace stb
