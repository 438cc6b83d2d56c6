// Device element table: the flattened, read-only form of a Line that the
// tracking kernel walks.  Shared by the host flattener and the CUDA kernel.
//
// A Line of polymorphic Element objects (simtrack.h:373-1100) becomes
//   * one 32-byte ElemHeader per element (opcode, slice count, offset of its
//     parameters in the parameter pool, aperture), and
//   * one FP64 parameter pool holding every per-element constant, already in
//     the exact form the reference computes at run time (for instance
//     Fdrift1*Lint, Fkick1*K1L/Nint, tan(E1)*href, L/GP.beta), so that the
//     kernel performs only the particle-dependent operations and rounds them
//     exactly as the reference does.
#pragma once
#include <cstdint>

namespace stb {

enum Op : int32_t {
  OP_DRIFT = 0,      // DRIFT_Pass                    simtrack.cpp:3743-3766
  OP_SBEND = 1,      // SBEND_Pass exact branch       simtrack.cpp:4693-4752
  OP_GSBEND = 2,     // GSBEND_Pass exact branch      simtrack.cpp:4818-4880
  OP_QUAD_THICK = 3, // QUAD_Pass Yoshida slices      simtrack.cpp:4882-4959
  OP_SEXT_THICK = 4, // SEXT_Pass                     simtrack.cpp:5004-5034
  OP_OCT_THICK = 5,  // OCT_Pass                      simtrack.cpp:5077-5105
  OP_MULT_THICK = 6, // MULT_Pass                     simtrack.cpp:5152-5182
  OP_QUAD_KICK = 7,  // quad_kick_pass (L == 0)       simtrack.cpp:4046-4058
  OP_SEXT_KICK = 8,  // sext_kick_pass                simtrack.cpp:4060-4071
  OP_OCT_KICK = 9,   // oct_kick_pass                 simtrack.cpp:4073-4084
  OP_MULT_KICK = 10, // mult_kick_pass                simtrack.cpp:4086-4111
  OP_BENDMULT = 11,  // GMULT/SBENDMULT exact branch  simtrack.cpp:5288-5311, 5413-5436
  OP_KICK = 12,      // KICK_Pass                     simtrack.cpp:5887-5893
  OP_RFCAV = 13,     // RFCAV_Pass                    simtrack.cpp:6002-6012
  OP_CRABRF = 14,    // CRABRF_Pass                   simtrack.cpp:6014-6025
  OP_CCMULT = 15,    // CCMULT_Pass                   simtrack.cpp:6027-6067
  OP_LBT = 16,       // LBT_Pass                      simtrack.cpp:6069-6093
  OP_ILBT = 17,      // ILBT_Pass                     simtrack.cpp:6095-6123
  OP_BB6D = 18,      // BB6D                          simtrack.cpp:6579-6678
  OP_BB4D = 19,      // BEAMBEAM_Pass treatment 4     simtrack.cpp:7348-7353
  OP_IDENTITY = 20,  // element whose Pass is a no-op (BEAMBEAM with NP == 0)
  OP_PATCH = 21,     // PATCH_Pass: TRANS_Pass + YROTAT_Pass simtrack.cpp:6140-6151, 6192-6217, 6248-6256
  OP_SOLEN = 22,     // SOLEN_Pass, KS != 0           simtrack.cpp:5804-5857
  // Spin-tracking forms (Element::sPass), used only in tables flattened for
  // spin; every other element's sPass equals its Pass (or a drift).
  OP_S_SBEND = 23,          // SBEND_sPass exact branch          simtrack.cpp:7486-7536
  OP_S_MPOLE_THICK = 24,    // QUAD/SEXT/OCT_sPass slices (aux = order) 7538-7698
  OP_S_MPOLE_KICK = 25,     // their L == 0 branches
  OP_S_MULT_THICK = 26,     // MULT_sPass                        7700-7740
  OP_S_MULT_KICK = 27,      // MULT_sPass L == 0
  OP_S_BENDMULT = 28,       // SBENDMULT_sPass exact branch      7836-7928
  OP_S_BENDMULT_KICK = 29,  // SBENDMULT_sPass L == 0
  OP_S_KICK = 30,           // KICK_sPass                        8193-8208
  OP_S_SOLEN = 31,          // SOLEN_sPass, KS != 0              8118-8183
  // Radiating forms (GP.radiate == true), orbit tables only.
  OP_SBEND_RAD = 32,     // SBEND_Pass exact radiating branch: Nint slices + radiate1   4740-4748
  OP_BENDMULT_RAD = 33,  // GMULT/SBENDMULT exact radiating branch: + radiate           5312-5338, 5437-5463
  OP_GSBEND_RAD = 34,    // GSBEND_Pass exact radiating branch: Nint slices + radiate2    4866-4873
  OP_COUNT = 35
};
constexpr int16_t OP_S_FIRST = OP_S_SBEND;
constexpr int16_t OP_S_LAST = OP_S_SOLEN;

// Header flag bits (ElemHeader::flags).
enum : int16_t {
  EF_MISALIGN_OFFSET = 1,  // GtoL1/LtoG1 offset part   simtrack.cpp:3450-3452, 3478-3480
  EF_MISALIGN_ROLL = 2,    // GtoL1/LtoG1 roll part     simtrack.cpp:3453-3460, 3470-3477
  EF_EDGE1 = 4,            // entrance edge focusing present
  EF_EDGE2 = 8,            // exit edge focusing present
  EF_FRINGE = 16,          // GP.quad_fringe hard-edge maps around a thick quad
  EF_CHANGES_PT = 32,      // element modifies pt: the pt-only cache is refreshed after it
  // The loss test after this element cannot fail when it passed after the
  // previous one: a kick that leaves x and y untouched, no misalignment, an
  // aperture no tighter than the previous element's.
  EF_NO_LOSS_CHECK = 64,
  // GP.radiate in a spin table: radiate() after each slice's spin rotation
  // (SBEND_sPass 7519-7529, SBENDMULT_sPass 7887-7918); the element's
  // parameters end with [Lint, E3] (OP_S_BENDMULT) or [E3] (OP_S_SBEND).
  EF_RADIATE = 128,
};

struct ElemHeader {
  int16_t op;     // Op
  int16_t flags;  // EF_* bits
  int32_t nint;   // Yoshida slices (thick) / slices (BB6D)
  int32_t poff;   // offset (in doubles) of this element's parameters in the pool
  int32_t aux;    // Norder for the multipole family
  double apx, apy;  // rectangular aperture (Element::APx/APy, default 1 m)
};
static_assert(sizeof(ElemHeader) == 32, "ElemHeader must stay 32 bytes");

// A lattice segment for tables too large for shared memory: elements
// [e0, e0 + ne) whose headers and pool slice [pool_lo, pool_lo + pool_n)
// (pool_lo and pool_n even, so both bulk copies start and end on 16-byte
// boundaries) fit one staging buffer.
struct SegDesc {
  int32_t e0, ne;
  int32_t pool_lo, pool_n;
};

// Reference-particle constants snapshotted from the global state at flatten time.
struct RefConsts {
  double gamma, beta, energy, brho;
  double sqrt_g2m1;  // sqrt(GP.gamma*GP.gamma-1.)
  double G;          // spin G
  double ibeta;      // RN(1/GP.beta)
  double ienergy;    // RN(1/GP.energy)
  // Quantum excitation (OP_SBEND_RAD): the normal-deviate stream's seed and
  // the number of radiating bend slices per turn (the k-th draw of a
  // particle is its (turn * rad_slices + slice index in the turn)-th).
  uint64_t rad_seed;
  int64_t rad_slices;
};

// Misalignment parameters sit in front of the element parameters when an
// EF_MISALIGN_* flag is set: [dx, dy, cos(dpsi), sin(dpsi)].
constexpr int kMisalignParams = 4;

// Largest multipole order the reference stores (KNL[11]).
constexpr int kMaxOrder = 10;
// Largest strong-bunch slice count accepted by the BB6D opcode.
constexpr int kMaxSlices = 64;

}  // namespace stb
