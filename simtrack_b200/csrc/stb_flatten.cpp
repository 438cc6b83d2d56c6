// Flattener: polymorphic Line -> ElemHeader[] + FP64 parameter pool.
//
// Every constant the reference recomputes inside a Pass call is computed here
// once, with the reference's own expression and operand order, so the value
// the kernel reads is bit-identical to the value the reference uses.  The
// header of each case cites the reference routine whose constants it builds.
#include "stb_flatten.hpp"

#include <cmath>
#include <cstring>
#include <string>

#include "stb_status.hpp"

namespace stb {

namespace {

const double kPI = 3.14159265358979323;  // simtrack.cpp:23
const double kRp4D = 1.53469826769e-18;  // BB4D classical proton radius, simtrack.cpp:6328
const double kRp6D = 1.534698e-18;       // BB6D value, simtrack.cpp:6586

struct Builder {
  HostTable t;
  Yoshida y = yoshida();

  int push(double v) {
    t.pool.push_back(v);
    return (int)t.pool.size() - 1;
  }
  int here() const { return (int)t.pool.size(); }

  // [L, L/GP.beta] for one DRIFT_Pass(x, L) call.
  void drift_params(double L) {
    push(L);
    push(L / GP.beta);
  }
  // sbend_exact_pass(x, L, Angle, cosA, sinA) constants (simtrack.cpp:3833-3858):
  // [L, L/GP.beta, href, 1.0/href, cosA, sinA]
  void bend_params(double L, double Angle, double cosA, double sinA) {
    double href = Angle / L;
    push(L);
    push(L / GP.beta);
    push(href);
    push(1.0 / href);
    push(cosA);
    push(sinA);
  }
  // Kick coefficient block for mult_kick_pass:
  // [KNL[0], KNSL[0], (KNL[i], KNSL[i], RN(1/i!)) i=1..Norder]
  void mult_block(int norder, const double *knl, const double *knsl) {
    push(knl[0]);
    push(knsl[0]);
    double fac = 1.0;
    for (int i = 1; i <= norder; i++) {
      fac *= i;
      push(knl[i]);
      push(knsl[i]);
      push(1.0 / fac);
    }
  }
};

// Operation counts used for the roofline (see HostTable::flops_per_turn).
const double kFlDrift = 16;
const double kFlQuadKick = 8;
const double kFlSextKick = 15;
const double kFlOctKick = 22;
const double kFlBend = 52;  // sbend_exact_pass with pt-only terms hoisted, 2 asin counted as 1 each
const double kFlEdge = 4;
const double kFlPtRefresh = 12;  // delta1, gamma1, beta1, 1+delta1, (1+delta1)^2

double mult_kick_flops(int norder, const double *kn, const double *ks) {
  double f = 2;
  for (int i = 1; i <= norder; i++) {
    f += 6;
    if (kn[i] != 0. || ks[i] != 0.) f += 10;
  }
  return f;
}

}  // namespace

Yoshida yoshida() {
  Yoshida c;
  c.d1 = 1.e0 / (2.e0 * (2.e0 - std::pow(2.e0, 1.0 / 3.0)));
  c.d2 = 0.5e0 - c.d1;
  c.k1 = 2.e0 * c.d1;
  c.k2 = 1.e0 - 2e0 * c.k1;
  return c;
}

double inverse_normal_cdf(double p) {
  // Wichura, AS241 (PPND16): rational approximations in three regions.
  static const double a[8] = {3.387132872796366608, 133.14166789178437745, 1971.5909503065514427,
                              13731.693765509461125, 45921.953931549871457, 67265.770927008700853,
                              33430.575583588128105, 2509.0809287301226727};
  static const double b[8] = {1.0, 42.313330701600911252, 687.1870074920579083, 5394.1960214247511077,
                              21213.794301586595867, 39307.89580009271061, 28729.085735721942674,
                              5226.495278852545925};
  static const double c[8] = {1.42343711074968357734, 4.6303378461565452959, 5.7694972214606914055,
                              3.64784832476320460504, 1.27045825245236838258, 0.24178072517745061177,
                              0.0227238449892691845833, 7.7454501427834140764e-4};
  static const double d[8] = {1.0, 2.05319162663775882187, 1.6763848301838038494, 0.68976733498510000455,
                              0.14810397642748007459, 0.0151986665636164571966, 5.475938084995344946e-4,
                              1.05075007164441684324e-9};
  static const double e[8] = {6.6579046435011037772, 5.4637849111641143699, 1.7848265399172913358,
                              0.29656057182850489123, 0.026532189526576123093, 0.0012426609473880784386,
                              2.71155556874348757815e-5, 2.01033439929228813265e-7};
  static const double f[8] = {1.0, 0.59983220655588793769, 0.13692988092273580531,
                              0.0148753612908506148525, 7.868691311456132591e-4, 1.8463183175100546818e-5,
                              1.4215117583164458887e-7, 2.04426310338993978564e-15};
  if (p == 1.0) return INFINITY;
  if (p == 0.0) return -INFINITY;
  const double q = p - 0.5;
  const double *num, *den;
  double r;
  const bool central = std::fabs(q) <= 0.425;
  if (central) {
    r = 0.180625 - q * q;
    num = a;
    den = b;
  } else {
    r = std::sqrt(-std::log(p < 0.5 ? p : 1.0 - p));
    if (r <= 5.0) {
      r = r - 1.6;
      num = c;
      den = d;
    } else {
      r = r - 5.0;
      num = e;
      den = f;
    }
  }
  double u = num[7], v = den[7];
  for (int i = 7; i > 0; i--) u = r * u + num[i - 1];
  for (int i = 7; i > 0; i--) v = r * v + den[i - 1];
  if (central) return q * (u / v);
  return p < 0.5 ? -(u / v) : (u / v);
}

namespace {

// Spin-tracking flop estimate of one spin() call (simtrack.cpp:4574-4630):
// direction vector, field terms, rotation matrix and product, cos + sin.
const double kFlSpin = 110;

// One solenoid slice with its entry and exit conversions (SOLEN_Pass).
const double kFlSolen = 76;
// radiate(): pz, the direction cosines, the cross product, the pt update,
// delta2 and the momentum rescaling, plus the pt-cache refresh it forces;
// radiate1() adds the fluctuation term and its normal deviate (ln and cos
// counted 1 each).
const double kFlRadiate = 50 + kFlPtRefresh;
const double kFlQuantum = 25;

// Parameters of SOLEN_Pass / SOLEN_sPass for KS != 0 (simtrack.cpp:5804-5857,
// 8118-8183): Bz is KS*brho in Pass and KS*brho/L in sPass.  The solenoid's
// slice count is fixed at 1 by its constructor (simtrack.cpp:9645-9660).
void solen_params(Builder &B, const Element &E, double Bz, bool spin) {
  const double L = E.L, Nint = 1.0, Lint = L / Nint;
  B.push(GP.q * Bz / 2.0);
  B.push(L);
  B.push(Nint);
  B.push(Lint);
  B.push(L / GP.beta / 2.99792458e8);
  B.push(GP.m0);
  B.push(GP.p);
  if (spin) B.push(Bz * Lint / GP.brho);
}

// Element::sPass forms that differ from Pass (simtrack.cpp:8436-11213).
// Returns false when the element's sPass is its Pass (the caller then emits
// the orbit form).  Parameter layouts are documented in stb_spin.cuh.
bool spin_form(Builder &B, const Element &E, ElemHeader &h, double &fl) {
  const std::string &T = E.TYPE;
  const Yoshida &Y = B.y;
  auto as_drift = [&](double L) {
    h.op = OP_DRIFT;
    B.drift_params(L);
    fl += kFlDrift;
  };
  if (T == "GSBEND" || T == "GMULT")
    throw Error(STB_EUNSUPPORTED, "element " + E.NAME + ": spin tracking of " + T + " is not implemented");
  if (T == "CRABRF") {
    as_drift(E.L);  // CRABRF::sPass 10808-10812: a drift inside GtoL/LtoG
    return true;
  }
  if (T == "SBEND") {
    // SBEND_sPass 7486-7536: Nint exact sub-bends, spin() after each
    const double L = E.L, Angle = E.GetP("ANGLE"), E1 = E.GetP("E1"), E2 = E.GetP("E2");
    const int Nint = (int)E.GetP("Nint");
    if (Angle == 0.) {
      as_drift(L);
      return true;
    }
    if (Nint <= 0) throw Error(STB_EINVAL, "element " + E.NAME + ": Nint must be positive");
    const double href = Angle / L, Lint = L / Nint, an = Angle / Nint;
    h.op = OP_S_SBEND;
    h.nint = Nint;
    B.push(std::tan(E1) * href);
    B.push(std::tan(E2) * href);
    B.bend_params(Lint, an, std::cos(an), std::sin(an));
    B.push(an);
    B.push(href);
    fl += 2 * kFlEdge + Nint * (kFlBend + kFlSpin);
    if (GP.radiate) {  // radiate() after each slice's rotation, 7529
      h.flags |= EF_RADIATE | EF_CHANGES_PT;
      B.push(std::pow(GP.energy / 1000., 3));
      fl += Nint * kFlRadiate;
      B.t.pt_refreshes += Nint;
    }
    return true;
  }
  if (T == "QUAD" || T == "SKEWQ" || T == "SEXT" || T == "OCT") {
    // QUAD_sPass 7538-7590 (SKEWQ::sPass 8766: K1L = 0), SEXT_sPass 7592-7644, OCT_sPass 7646-7698
    const int order = (T == "SEXT") ? 2 : (T == "OCT") ? 3 : 1;
    double kl, ksl;
    if (T == "QUAD") { kl = E.GetP("K1L"); ksl = E.GetP("K1SL"); }
    else if (T == "SKEWQ") { kl = 0.; ksl = E.GetP("K1SL"); }
    else if (T == "SEXT") { kl = E.GetP("K2L"); ksl = E.GetP("K2SL"); }
    else { kl = E.GetP("K3L"); ksl = E.GetP("K3SL"); }
    const int Nint = (int)E.GetP("Nint");
    const double L = E.L;
    const double kick_fl = order == 1 ? kFlQuadKick : order == 2 ? kFlSextKick : kFlOctKick;
    h.aux = order;
    if (kl == 0. && ksl == 0.) {
      as_drift(L);
    } else if (L == 0.) {
      h.op = OP_S_MPOLE_KICK;
      B.push(kl);
      B.push(ksl);
      B.push((double)Nint);
      fl += kick_fl + 10 + kFlSpin;
    } else {
      if (Nint <= 0) throw Error(STB_EINVAL, "element " + E.NAME + ": Nint must be positive");
      h.op = OP_S_MPOLE_THICK;
      h.nint = Nint;
      const double Lint = L / Nint;
      B.drift_params(Y.d1 * Lint);
      B.drift_params(Y.d2 * Lint);
      B.push(Y.k1 * kl / Nint);
      B.push(Y.k1 * ksl / Nint);
      B.push(Y.k2 * kl / Nint);
      B.push(Y.k2 * ksl / Nint);
      B.push(kl);
      B.push(ksl);
      B.push((double)Nint);
      fl += Nint * (4 * kFlDrift + 3 * kick_fl + 12 + kFlSpin);
    }
    return true;
  }
  if (T == "MULT") {
    // MULT_sPass 7700-7740
    const int Nint = (int)E.GetP("Nint"), Norder = (int)E.GetP("Norder");
    if (Norder < 0 || Norder > kMaxOrder) throw Error(STB_EINVAL, "element " + E.NAME + ": Norder out of range");
    const double *knl = E.KNL(), *knsl = E.KNSL();
    h.aux = Norder;
    if (E.L == 0.) {
      h.op = OP_S_MULT_KICK;
      B.mult_block(Norder, knl, knsl);
      fl += 2 * mult_kick_flops(Norder, knl, knsl) + 3 + kFlSpin;
    } else {
      if (Nint <= 0) throw Error(STB_EINVAL, "element " + E.NAME + ": Nint must be positive");
      h.op = OP_S_MULT_THICK;
      h.nint = Nint;
      const double Lint = E.L / Nint;
      double k1[11], s1[11], k2[11], s2[11];
      for (int i = 0; i < 11; i++) {
        k1[i] = Y.k1 * knl[i] / Nint;
        s1[i] = Y.k1 * knsl[i] / Nint;
        k2[i] = Y.k2 * knl[i] / Nint;
        s2[i] = Y.k2 * knsl[i] / Nint;
      }
      B.drift_params(Y.d1 * Lint);
      B.drift_params(Y.d2 * Lint);
      B.mult_block(Norder, k1, s1);
      B.mult_block(Norder, k2, s2);
      B.mult_block(Norder, knl, knsl);
      B.push((double)Nint);
      fl += Nint * (4 * kFlDrift + 2 * mult_kick_flops(Norder, k1, s1) + mult_kick_flops(Norder, k2, s2) +
                    mult_kick_flops(Norder, knl, knsl) + 7 + kFlSpin);
    }
    return true;
  }
  if (T == "SBENDMULT") {
    // SBENDMULT_sPass 7836-7928, exact (non-H_expand) branch
    const int Nint = (int)E.GetP("Nint"), Norder = (int)E.GetP("Norder");
    if (Norder < 0 || Norder > kMaxOrder) throw Error(STB_EINVAL, "element " + E.NAME + ": Norder out of range");
    const double *knl = E.KNL(), *knsl = E.KNSL();
    const double Angle = E.GetP("ANGLE");
    h.aux = Norder;
    if (E.L == 0.) {
      h.op = OP_S_BENDMULT_KICK;
      B.mult_block(Norder, knl, knsl);
      B.push(Angle);
      fl += 2 * mult_kick_flops(Norder, knl, knsl) + 5 + kFlSpin;
    } else {
      if (Nint <= 0) throw Error(STB_EINVAL, "element " + E.NAME + ": Nint must be positive");
      const double L = E.L, E1 = E.GetP("E1"), E2 = E.GetP("E2");
      const double href = Angle / L, Lint = L / Nint;
      h.op = OP_S_BENDMULT;
      h.nint = Nint;
      B.push(std::tan(E1) * href);
      B.push(std::tan(E2) * href);
      double k1[11], s1[11], k2[11], s2[11];
      for (int i = 0; i < 11; i++) {
        k1[i] = Y.k1 * knl[i] / Nint;
        s1[i] = Y.k1 * knsl[i] / Nint;
        k2[i] = Y.k2 * knl[i] / Nint;
        s2[i] = Y.k2 * knsl[i] / Nint;
      }
      B.bend_params(Y.d1 * Lint, Y.d1 * Angle / Nint, std::cos(Y.d1 * Angle / Nint), std::sin(Y.d1 * Angle / Nint));
      B.bend_params(Y.d2 * Lint, Y.d2 * Angle / Nint, std::cos(Y.d2 * Angle / Nint), std::sin(Y.d2 * Angle / Nint));
      B.mult_block(Norder, k1, s1);
      B.mult_block(Norder, k2, s2);
      B.mult_block(Norder, knl, knsl);
      B.push(Angle / Nint);
      B.push(href);
      B.push(Angle);
      B.push((double)Nint);
      fl += 2 * kFlEdge + Nint * (4 * kFlBend + 2 * mult_kick_flops(Norder, k1, s1) +
                                  mult_kick_flops(Norder, k2, s2) + mult_kick_flops(Norder, knl, knsl) + 8 +
                                  kFlSpin);
      if (GP.radiate) {  // radiate() after each slice's rotation, 7918
        h.flags |= EF_RADIATE | EF_CHANGES_PT;
        B.push(Lint);
        B.push(std::pow(GP.energy / 1000., 3));
        fl += Nint * kFlRadiate;
        B.t.pt_refreshes += Nint;
      }
    }
    return true;
  }
  if (T == "SOLEN") {
    // SOLEN_sPass 8118-8183; KS == 0 is DRIFT_Pass, the orbit form
    const double KS = E.GetP("KS");
    if (KS == 0) return false;
    h.op = OP_S_SOLEN;
    h.nint = 1;
    solen_params(B, E, KS * GP.brho / E.L, true);
    fl += kFlSolen + kFlSpin;
    return true;
  }
  if (T == "KICKER" || T == "HKICKER" || T == "VKICKER") {
    // KICK_sPass 8193-8208
    double hk = 0., vk = 0.;
    if (T != "VKICKER") hk = E.GetP("HKICK");
    if (T != "HKICKER") vk = E.GetP("VKICK");
    h.op = OP_S_KICK;
    B.drift_params(E.L / 2.0);
    B.push(hk);
    B.push(vk);
    fl += 2 * kFlDrift + 2 + kFlSpin;
    return true;
  }
  return false;
}

unsigned long long g_radiation_seed = 1324;

HostTable flatten_impl(const Line &line, bool spin, bool skip_rfcav) {
  if (GP.H_expand) throw Error(STB_EUNSUPPORTED, "GP.H_expand == true is not implemented on the GPU path");
  Builder B;
  HostTable &t = B.t;
  t.ref.gamma = GP.gamma;
  t.ref.beta = GP.beta;
  t.ref.energy = GP.energy;
  t.ref.brho = GP.brho;
  t.ref.sqrt_g2m1 = std::sqrt(GP.gamma * GP.gamma - 1.);
  t.ref.G = GP.G;
  t.ref.ibeta = 1.0 / GP.beta;
  t.ref.ienergy = 1.0 / GP.energy;
  t.ref.rad_seed = radiation_seed();
  t.ref.rad_slices = 0;
  t.radiate = GP.radiate;
  // radiate()/radiate1() constants: pow(GP.energy/1000., 3) (simtrack.cpp:4224)
  // and Cf (simtrack.cpp:26), with the reference's expressions
  const double rad_E3 = std::pow(GP.energy / 1000., 3);
  const double rad_Cf = (55. / 24. / std::sqrt(3.)) * 2.8179403e-15 * 1.054572e-34 / 9.1093822e-31;
  t.flops_per_turn = kFlPtRefresh;  // turn-start evaluation of the pt cache
  t.spin = spin;
  const Yoshida &Y = B.y;

  for (size_t idx = 0; idx < line.Cell.size(); idx++) {
    const Element &E = *line.Cell[idx];
    const std::string &T = E.TYPE;
    ElemHeader h{};
    h.apx = E.APx;
    h.apy = E.APy;
    double fl = 0;
    if (skip_rfcav && T == "RFCAV") {
      // Cal_SRLoss_Particle (simtrack.cpp:20768-20781) passes every element
      // but the cavities: no map, no misalignment.
      h.op = OP_IDENTITY;
      h.poff = B.here();
      t.hdr.push_back(h);
      continue;
    }

    // GtoL dispatch (simtrack.cpp:3701-3741).  DRIFT and MARKER never call it,
    // nor do LBT::sPass and ILBT::sPass (11004, 11053) in spin tracking.
    const bool straight_drift = (T == "DRIFT" || T == "MARKER" || T == "BPM" || T == "HBPM" || T == "VBPM");
    // PATCH::Pass/sPass (12323-12333) apply the patch alone: its DX, DY, DS
    // are the patch's own offsets, not a misalignment.
    const bool no_gtol = straight_drift || T == "PATCH" || (spin && (T == "LBT" || T == "ILBT"));
    if (!no_gtol) {
      double s = std::fabs(E.DX) + std::fabs(E.DY) + std::fabs(E.DS) + std::fabs(E.DTHETA) +
                 std::fabs(E.DPHI) + std::fabs(E.DPSI);
      if (!(s < 1.0e-9)) {
        if (!(std::fabs(E.DTHETA) + std::fabs(E.DPHI) < 1.0e-9))
          throw Error(STB_EUNSUPPORTED, "element " + E.NAME + ": pitch/yaw misalignment (GtoL2) is not implemented");
        // GtoL1/LtoG1 thresholds, simtrack.cpp:3450, 3453
        if (std::fabs(E.DX) + std::fabs(E.DY) > 1.0e-10) h.flags |= EF_MISALIGN_OFFSET;
        if (std::fabs(E.DPSI) > 1.0e-10) h.flags |= EF_MISALIGN_ROLL;
      }
    }
    h.poff = B.here();
    if (h.flags & (EF_MISALIGN_OFFSET | EF_MISALIGN_ROLL)) {
      B.push(E.DX);
      B.push(E.DY);
      B.push(std::cos(E.DPSI));
      B.push(std::sin(E.DPSI));
      if (h.flags & EF_MISALIGN_OFFSET) fl += 4;
      if (h.flags & EF_MISALIGN_ROLL) fl += 24;
    }

    auto as_drift = [&](double L) {
      h.op = OP_DRIFT;
      B.drift_params(L);
      fl += kFlDrift;
    };

    if (straight_drift) {
      as_drift(E.L);  // DRIFT::Pass 8426, MARKER::Pass 10617, BPM/HBPM/VBPM::Pass 10497-10579
    } else if (spin && spin_form(B, E, h, fl)) {
      // Element::sPass form emitted by spin_form
    } else if (T == "PATCH") {
      // PATCH_Pass, simtrack.cpp:6248-6256 (also PATCH::sPass)
      const double th = E.GetP("THETA");
      h.op = OP_PATCH;
      B.push(E.GetP("DX"));
      B.push(E.GetP("DY"));
      B.push(E.GetP("DS"));
      fl += 3;
      if (!(std::fabs(th) < 1.0e-9)) {  // YROTAT_Pass returns early below 1e-9 (6195)
        h.aux = 1;
        B.push(std::cos(th));
        B.push(std::sin(th));
        B.push(std::tan(th));
        fl += 22;
      }
    } else if (T == "SOLEN") {
      // SOLEN::Pass, simtrack.cpp:9688-9692; KS == 0 is DRIFT_Pass (5811-5814)
      const double KS = E.GetP("KS");
      if (KS == 0) {
        as_drift(E.L);
      } else {
        h.op = OP_SOLEN;
        h.nint = 1;
        solen_params(B, E, KS * GP.brho, false);
        fl += kFlSolen;
      }
    } else if (T == "SBEND") {
      // SBEND_Pass, simtrack.cpp:4693-4752
      const double L = E.L, Angle = E.GetP("ANGLE"), E1 = E.GetP("E1"), E2 = E.GetP("E2");
      if (Angle == 0.) {
        as_drift(L);
      } else if (GP.radiate) {
        // radiating exact branch, simtrack.cpp:4740-4748
        const int Nint = (int)E.GetP("Nint");
        if (Nint <= 0) throw Error(STB_EINVAL, "element " + E.NAME + ": Nint must be positive");
        const double href = Angle / L, Lint = L / Nint, an = Angle / Nint;
        h.op = OP_SBEND_RAD;
        h.nint = Nint;
        h.flags |= EF_CHANGES_PT;
        B.push(std::tan(E1) * href);
        B.push(std::tan(E2) * href);
        B.bend_params(Lint, an, std::cos(an), std::sin(an));
        B.push(Lint);
        B.push(href);
        B.push(an);
        B.push(rad_E3);
        B.push(rad_Cf);
        B.push((double)t.ref.rad_slices);
        t.ref.rad_slices += Nint;
        if (E1 != 0.) { h.flags |= EF_EDGE1; fl += kFlEdge; }
        if (E2 != 0.) { h.flags |= EF_EDGE2; fl += kFlEdge; }
        fl += Nint * (kFlBend + kFlRadiate + kFlQuantum);
        t.pt_refreshes += Nint;
      } else {
        const double href = Angle / L;
        h.op = OP_SBEND;
        B.push(std::tan(E1) * href);
        B.push(std::tan(E2) * href);
        B.bend_params(L, Angle, std::cos(Angle), std::sin(Angle));
        if (E1 != 0.) { h.flags |= EF_EDGE1; fl += kFlEdge; }
        if (E2 != 0.) { h.flags |= EF_EDGE2; fl += kFlEdge; }
        fl += kFlBend;
      }
    } else if (T == "GSBEND") {
      // GSBEND_Pass, simtrack.cpp:4818-4880; general_sbend_exact_pass 3974-4010
      const double L = E.L, Angle = E.GetP("ANGLE"), K0L = E.GetP("K0L");
      const double E1 = E.GetP("E1"), E2 = E.GetP("E2");
      if (Angle == 0.) {
        as_drift(L);
      } else if (GP.radiate) {
        // radiating exact branch, simtrack.cpp:4866-4873: Nint slices of
        // general_sbend_exact_pass(Lint, Angle/Nint, K0L/Nint), radiate2 after each
        const int Nint = (int)E.GetP("Nint");
        if (Nint <= 0) throw Error(STB_EINVAL, "element " + E.NAME + ": Nint must be positive");
        const double href = Angle / L, hreal = K0L / L, Lint = L / Nint;
        const double an = Angle / Nint, kn = K0L / Nint;
        const double rhoc = Lint / an, b0 = kn / Lint;
        h.op = OP_GSBEND_RAD;
        h.nint = Nint;
        h.flags |= EF_CHANGES_PT;
        B.push(std::tan(E1) * hreal);
        B.push(std::tan(E2) * hreal);
        B.push(Lint);
        B.push(Lint / GP.beta);
        B.push(rhoc);
        B.push(b0);
        B.push(b0 * rhoc);
        B.push(std::cos(an));
        B.push(std::sin(an));
        B.push(1.0 / rhoc);
        B.push(1.0 / b0);
        B.push(href);
        B.push(kn);
        // facg of radiate2, simtrack.cpp:4316
        B.push(12. * std::sqrt(3.) / (std::pow(2., 1.0 / 3.0) * 5.0 * 2.6789385347077475));
        B.push((double)t.ref.rad_slices);
        t.ref.rad_slices += Nint;
        if (E1 != 0.) { h.flags |= EF_EDGE1; fl += kFlEdge; }
        if (E2 != 0.) { h.flags |= EF_EDGE2; fl += kFlEdge; }
        fl += Nint * (kFlBend + 4 + kFlRadiate + kFlQuantum);
        t.pt_refreshes += Nint;
      } else {
        const double hreal = K0L / L;
        const double rhoc = L / Angle, b0 = K0L / L;
        h.op = OP_GSBEND;
        B.push(std::tan(E1) * hreal);
        B.push(std::tan(E2) * hreal);
        B.push(L);
        B.push(L / GP.beta);
        B.push(rhoc);
        B.push(b0);
        B.push(b0 * rhoc);
        B.push(std::cos(Angle));
        B.push(std::sin(Angle));
        B.push(1.0 / rhoc);
        B.push(1.0 / b0);
        if (E1 != 0.) { h.flags |= EF_EDGE1; fl += kFlEdge; }
        if (E2 != 0.) { h.flags |= EF_EDGE2; fl += kFlEdge; }
        fl += kFlBend + 4;
      }
    } else if (T == "QUAD" || T == "SKEWQ" || T == "SEXT" || T == "OCT") {
      // QUAD_Pass 4882-4959, SEXT_Pass 5004-5034, OCT_Pass 5077-5105; SKEWQ::Pass 8754 uses QUAD_Pass(0, K1SL)
      int order = (T == "SEXT") ? 2 : (T == "OCT") ? 3 : 1;
      double kl, ksl;
      if (T == "QUAD") { kl = E.GetP("K1L"); ksl = E.GetP("K1SL"); }
      else if (T == "SKEWQ") { kl = 0.; ksl = E.GetP("K1SL"); }
      else if (T == "SEXT") { kl = E.GetP("K2L"); ksl = E.GetP("K2SL"); }
      else { kl = E.GetP("K3L"); ksl = E.GetP("K3SL"); }
      const int Nint = (int)E.GetP("Nint");
      const double L = E.L;
      const double kick_fl = order == 1 ? kFlQuadKick : order == 2 ? kFlSextKick : kFlOctKick;
      if (kl == 0. && ksl == 0.) {
        as_drift(L);
      } else if (L == 0.) {
        h.op = order == 1 ? OP_QUAD_KICK : order == 2 ? OP_SEXT_KICK : OP_OCT_KICK;
        B.push(kl);
        B.push(ksl);
        fl += kick_fl;
      } else {
        if (Nint <= 0) throw Error(STB_EINVAL, "element " + E.NAME + ": Nint must be positive");
        h.op = order == 1 ? OP_QUAD_THICK : order == 2 ? OP_SEXT_THICK : OP_OCT_THICK;
        h.nint = Nint;
        const double Lint = L / Nint;
        B.drift_params(Y.d1 * Lint);
        B.drift_params(Y.d2 * Lint);
        B.push(Y.k1 * kl / Nint);
        B.push(Y.k1 * ksl / Nint);
        B.push(Y.k2 * kl / Nint);
        B.push(Y.k2 * ksl / Nint);
        fl += Nint * (4 * kFlDrift + 3 * kick_fl);
        if (order == 1 && GP.quad_fringe) {
          h.flags |= EF_FRINGE;
          B.push(kl / L);
          fl += 2 * 60;
        }
      }
    } else if (T == "MULT") {
      // MULT_Pass, simtrack.cpp:5152-5182
      const int Nint = (int)E.GetP("Nint"), Norder = (int)E.GetP("Norder");
      if (Norder < 0 || Norder > kMaxOrder) throw Error(STB_EINVAL, "element " + E.NAME + ": Norder out of range");
      const double *knl = E.KNL(), *knsl = E.KNSL();
      h.aux = Norder;
      if (E.L == 0.) {
        h.op = OP_MULT_KICK;
        B.mult_block(Norder, knl, knsl);
        fl += mult_kick_flops(Norder, knl, knsl);
      } else {
        if (Nint <= 0) throw Error(STB_EINVAL, "element " + E.NAME + ": Nint must be positive");
        h.op = OP_MULT_THICK;
        h.nint = Nint;
        const double Lint = E.L / Nint;
        double k1[11], s1[11], k2[11], s2[11];
        for (int i = 0; i < 11; i++) {
          k1[i] = Y.k1 * knl[i] / Nint;
          s1[i] = Y.k1 * knsl[i] / Nint;
          k2[i] = Y.k2 * knl[i] / Nint;
          s2[i] = Y.k2 * knsl[i] / Nint;
        }
        B.drift_params(Y.d1 * Lint);
        B.drift_params(Y.d2 * Lint);
        B.mult_block(Norder, k1, s1);
        B.mult_block(Norder, k2, s2);
        fl += Nint * (4 * kFlDrift + 2 * mult_kick_flops(Norder, k1, s1) + mult_kick_flops(Norder, k2, s2));
      }
    } else if (T == "GMULT" || T == "SBENDMULT") {
      // GMULT_Pass 5223-5346 / SBENDMULT_Pass 5348-5470, exact non-radiating branch
      const int Nint = (int)E.GetP("Nint"), Norder = (int)E.GetP("Norder");
      if (Norder < 0 || Norder > kMaxOrder) throw Error(STB_EINVAL, "element " + E.NAME + ": Norder out of range");
      const double *knl = E.KNL(), *knsl = E.KNSL();
      h.aux = Norder;
      if (E.L == 0.) {
        h.op = OP_MULT_KICK;
        B.mult_block(Norder, knl, knsl);
        fl += mult_kick_flops(Norder, knl, knsl);
      } else {
        if (Nint <= 0) throw Error(STB_EINVAL, "element " + E.NAME + ": Nint must be positive");
        const double L = E.L, Angle = E.GetP("ANGLE"), E1 = E.GetP("E1"), E2 = E.GetP("E2");
        const double href = Angle / L, Lint = L / Nint;
        h.op = OP_BENDMULT;
        h.nint = Nint;
        B.push(std::tan(E1) * href);
        B.push(std::tan(E2) * href);
        h.flags |= EF_EDGE1 | EF_EDGE2;  // the reference applies both edges unconditionally here
        double k1[11], s1[11], k2[11], s2[11];
        for (int i = 0; i < 11; i++) {
          k1[i] = Y.k1 * knl[i] / Nint;
          s1[i] = Y.k1 * knsl[i] / Nint;
          k2[i] = Y.k2 * knl[i] / Nint;
          s2[i] = Y.k2 * knsl[i] / Nint;
        }
        const double a1 = Y.d1 * Angle / Nint, a2 = Y.d2 * Angle / Nint;
        B.bend_params(Y.d1 * Lint, a1, std::cos(Y.d1 * Angle / Nint), std::sin(Y.d1 * Angle / Nint));
        B.bend_params(Y.d2 * Lint, a2, std::cos(Y.d2 * Angle / Nint), std::sin(Y.d2 * Angle / Nint));
        B.mult_block(Norder, k1, s1);
        B.mult_block(Norder, k2, s2);
        fl += 2 * kFlEdge + Nint * (4 * kFlBend + 2 * mult_kick_flops(Norder, k1, s1) + mult_kick_flops(Norder, k2, s2));
        if (GP.radiate) {
          // radiating exact branch, GMULT_Pass 5312-5338 / SBENDMULT_Pass 5437-5463
          h.op = OP_BENDMULT_RAD;
          h.flags |= EF_CHANGES_PT;
          B.mult_block(Norder, knl, knsl);
          B.push(Angle);
          B.push((double)Nint);
          B.push(Lint);
          B.push(href);
          B.push(rad_E3);
          fl += Nint * (mult_kick_flops(Norder, knl, knsl) + 11 + kFlRadiate);
          t.pt_refreshes += Nint;
        }
      }
    } else if (T == "KICKER" || T == "HKICKER" || T == "VKICKER") {
      // KICK_Pass, simtrack.cpp:5887-5893
      double hk = 0., vk = 0.;
      if (T != "VKICKER") hk = E.GetP("HKICK");
      if (T != "HKICKER") vk = E.GetP("VKICK");
      h.op = OP_KICK;
      B.drift_params(E.L / 2.0);
      B.push(hk);
      B.push(vk);
      fl += 2 * kFlDrift + 2;
    } else if (T == "RFCAV") {
      // RFCAV_Pass, simtrack.cpp:6002-6012
      const double VRF = E.GetP("VRF"), FRF = E.GetP("FRF"), PHASE0 = E.GetP("PHASE0");
      if (VRF == 0.) {
        as_drift(E.L);
      } else {
        h.op = OP_RFCAV;
        h.flags |= EF_CHANGES_PT;
        B.drift_params(E.L / 2.);
        B.push(std::abs(VRF * GP.Q));
        B.push(-2.0 * kPI * FRF);
        B.push(PHASE0);
        fl += 2 * kFlDrift + 9 + kFlPtRefresh;
        t.pt_refreshes++;
      }
    } else if (T == "CRABRF") {
      // CRABRF_Pass, simtrack.cpp:6014-6025
      const double VRF = E.GetP("VRF"), FRF = E.GetP("FRF"), PHASE0 = E.GetP("PHASE0");
      if (VRF == 0.) {
        as_drift(E.L);
      } else {
        h.op = OP_CRABRF;
        h.flags |= EF_CHANGES_PT;
        B.drift_params(E.L / 2.);
        B.push(VRF * GP.Q);
        B.push(2.0 * kPI * FRF);
        B.push(PHASE0);
        B.push(2.0 * kPI * FRF / 2.99792458e8);
        fl += 2 * kFlDrift + 18 + kFlPtRefresh;
        t.pt_refreshes++;
      }
    } else if (T == "CCMULT") {
      // CCMULT_Pass, simtrack.cpp:6027-6067 (element B1..A4 feed arguments B2..A5)
      const double VRF = E.GetP("VRF"), FRF = E.GetP("FRF"), PHASE0 = E.GetP("PHASE0");
      if (VRF == 0.) {
        as_drift(E.L);
      } else {
        h.op = OP_CCMULT;
        h.flags |= EF_CHANGES_PT;
        B.drift_params(E.L / 2.);
        const double c = 2.99792458e8;
        B.push(2.0 * kPI * FRF);
        B.push(PHASE0);
        B.push(2 * kPI * FRF / c / GP.brho);
        B.push(GP.brho);
        static const char *names[8] = {"B1", "A1", "B2", "A2", "B3", "A3", "B4", "A4"};
        for (int i = 0; i < 8; i++) B.push(E.GetP(names[i]));
        fl += 2 * kFlDrift + 150 + kFlPtRefresh;
        t.pt_refreshes++;
      }
    } else if (T == "LBT" || T == "ILBT") {
      // LBT_Pass 6069-6093 / ILBT_Pass 6095-6123
      const double theta = E.GetP("THETA");
      const double st = std::sin(theta), ct = std::cos(theta);
      h.op = (T == "LBT") ? OP_LBT : OP_ILBT;
      h.flags |= EF_CHANGES_PT;
      B.push(st);
      B.push(ct);
      B.push(st / ct);
      fl += 45 + kFlPtRefresh;
      t.pt_refreshes++;
    } else if (T == "BEAMBEAM") {
      // BEAMBEAM::Pass 11191 -> BEAMBEAM_Pass 7343-7356
      const int treatment = (int)E.GetP("TREATMENT");
      const double NP = E.GetP("NP"), BBSCALE = E.GetP("BBSCALE"), SIGMAL = E.GetP("SIGMAL");
      const int N = (int)E.GetP("NSLICE");
      const double EMITX = E.GetP("EMITX"), BETAX = E.GetP("BETAX"), ALFAX = E.GetP("ALFAX");
      const double EMITY = E.GetP("EMITY"), BETAY = E.GetP("BETAY"), ALFAY = E.GetP("ALFAY");
      if (NP == 0.) {
        h.op = OP_IDENTITY;
      } else if (treatment == 6) {
        // BB6D, simtrack.cpp:6579-6678
        if (N < 1 || N > kMaxSlices) throw Error(STB_EINVAL, "element " + E.NAME + ": NSLICE out of range");
        h.op = OP_BB6D;
        h.nint = N;
        h.flags |= EF_CHANGES_PT;
        const double gamma = GP.gamma;
        const double Np_slice = 1.0 * NP / N;
        B.push(BBSCALE);
        B.push(EMITX);
        B.push(EMITY);
        B.push(BETAX);
        B.push(ALFAX);
        B.push(BETAY);
        B.push(ALFAY);
        B.push((1.0 + ALFAX * ALFAX) / BETAX);        // gx_star
        B.push((1.0 + ALFAY * ALFAY) / BETAY);        // gy_star
        B.push(2.0 * EMITX);                          // leading factor of dsigmax2ds
        B.push(2.0 * EMITY);
        B.push(2. * Np_slice * kRp6D / gamma);        // temp3
        B.push(2 * Np_slice * kRp4D / gamma);         // BB4D 2*N*rp/gamma
        // Slice centroids (simtrack.cpp:6593-6620), including the truncated
        // 3.14159265 of the general formula.
        double zs[kMaxSlices];
        if (N == 11) {
          static const double tab[11] = {1.7996765362153655, 1.1049618149811977, 0.75072324235797372,
                                         0.47407703558819131, 0.23041113693387344, 0., -0.23041113693387344,
                                         -0.47407703558819131, -0.75072324235797372, -1.1049618149811977,
                                         -1.7996765362153655};
          for (int i = 0; i < 11; i++) zs[i] = tab[i] * SIGMAL;
        } else {
          double yv[kMaxSlices];
          for (int i = 0; i < N - 1; i++) yv[i] = inverse_normal_cdf((i + 1) * 1.0 / N);
          if (N == 1) {
            zs[0] = 0.;  // the reference reads y[0] of an empty array here; a centred slice is used
          } else {
            zs[0] = N * (std::exp(-yv[0] * yv[0] / 2)) / std::sqrt(2.0 * 3.14159265);
            zs[N - 1] = N * (0 - std::exp(-yv[0] * yv[0] / 2)) / std::sqrt(2.0 * 3.14159265);
            for (int i = 1; i < N - 1; i++)
              zs[i] = N * (std::exp(-yv[i] * yv[i] / 2) - std::exp(-yv[i - 1] * yv[i - 1] / 2)) /
                      std::sqrt(2.0 * 3.14159265);
          }
          for (int i = 0; i < N; i++) zs[i] = zs[i] * SIGMAL;
        }
        for (int i = 0; i < N; i++) B.push(zs[i]);
        const bool round = std::fabs(EMITX * BETAX - EMITY * BETAY) == 0. && ALFAX == ALFAY;
        fl += N * (round ? 75 : 75 + 2 * 300) + kFlPtRefresh;
        t.pt_refreshes++;
      } else {
        // treatment 4: BB4D with fixed sigmas, simtrack.cpp:7350-7352
        h.op = OP_BB4D;
        const double sx = std::sqrt(EMITX * BETAX), sy = std::sqrt(EMITY * BETAY);
        const double c4 = 2 * NP * kRp4D / GP.gamma;
        B.push(c4);
        B.push(sx);
        B.push(sy);
        B.push(BBSCALE);
        fl += 30;
      }
    } else {
      throw Error(STB_EUNSUPPORTED, "element type " + T + " (" + E.NAME + ") is not implemented on the GPU path");
    }
    if (h.flags & EF_CHANGES_PT) {
      // refresh count already added with the element
    }
    t.flops_per_turn += fl;
    t.hdr.push_back(h);
  }
  // Elements after which the loss test cannot newly fail: thin kicks (x, y
  // unchanged) without misalignment whose aperture is no tighter than the
  // previous element's.  The test after the previous element passed, so it
  // passes again with the same x, y; the kernels skip it.
  for (size_t i = 1; i < t.hdr.size(); i++) {
    ElemHeader &h = t.hdr[i];
    const ElemHeader &q = t.hdr[i - 1];
    const bool kick = h.op == OP_QUAD_KICK || h.op == OP_SEXT_KICK || h.op == OP_OCT_KICK || h.op == OP_MULT_KICK ||
                      h.op == OP_BB4D || h.op == OP_IDENTITY;
    const bool mis = (h.flags & (EF_MISALIGN_OFFSET | EF_MISALIGN_ROLL)) != 0;
    if (kick && !mis && h.apx >= q.apx && h.apy >= q.apy) h.flags |= EF_NO_LOSS_CHECK;
  }
  return t;
}

}  // namespace

unsigned long long radiation_seed() { return g_radiation_seed; }
void set_radiation_seed(unsigned long long seed) { g_radiation_seed = seed; }

HostTable flatten(const Line &line, bool skip_rfcav) { return flatten_impl(line, false, skip_rfcav); }
HostTable flatten_spin(const Line &line) { return flatten_impl(line, true, false); }

}  // namespace stb
