// Line -> device element table (host side).
#pragma once
#include <vector>

#include "simtrack_b200.hpp"
#include "stb_table.hpp"

namespace stb {

struct HostTable {
  std::vector<ElemHeader> hdr;
  std::vector<double> pool;
  RefConsts ref{};
  // Algorithmic FP64 operations per particle per turn (add/sub/mul/div/sqrt
  // count 1, each transcendental counts 1), for the element sequence as the
  // kernel executes it (pt-only invariants evaluated once per refresh).
  double flops_per_turn = 0.;
  // Number of per-turn refreshes of the pt-only cache (elements that change pt).
  int pt_refreshes = 0;
  // Flattened for spin tracking (Element::sPass semantics).
  bool spin = false;
  // Flattened with GP.radiate: radiating bends (OP_SBEND_RAD, OP_BENDMULT_RAD),
  // tracked by the plain Track() entry points only.
  bool radiate = false;
};

// Seed of the quantum-excitation normal deviates (stb_rng.cuh), read at
// flatten time; the default is the seed the reference gives its GSL stream
// (Init_GSL_Seeds, simtrack.cpp:328).
unsigned long long radiation_seed();
void set_radiation_seed(unsigned long long seed);

// Flatten `line` against the current reference-particle state GP.
// Throws stb::Error(STB_EUNSUPPORTED) for element types or settings that
// the GPU kernel does not implement (H_expand, pitch/yaw, GSBEND's photon
// Monte Carlo under GP.radiate).
// skip_rfcav: every RFCAV becomes a no-op (Cal_SRLoss_Particle's pass).
HostTable flatten(const Line &line, bool skip_rfcav = false);
// Flatten for Track_Spin (simtrack.cpp:21766-21789): the orbit maps of
// Element::sPass plus the Thomas-BMT rotation of spin() after every slice.
// GSBEND and GMULT are not available in this form (STB_EUNSUPPORTED).
HostTable flatten_spin(const Line &line);

// Yoshida coefficients Fdrift1/Fdrift2/Fkick1/Fkick2 (simtrack.cpp:29-32),
// computed with the same expressions as the reference.
struct Yoshida {
  double d1, d2, k1, k2;
};
Yoshida yoshida();

// Inverse standard-normal CDF (Wichura's AS241), used for the strong-bunch
// slice centroids that the reference obtains from GSL (simtrack.cpp:6614).
double inverse_normal_cdf(double p);

}  // namespace stb
