// simtrack_b200 C++ host API: the beamline construction and tracking
// interface of SimTrack (simtrack.h), with tracking executed on a B200 GPU.
//
// A driver written against the reference builds a Line with `new QUAD(...)`,
// `SetP("Nint", 4)`, `Line::Append(...)` and calls `Track(...)`.  The same
// driver compiles against this header after `using namespace stb;`.  The
// classes here hold element parameters only; every Pass runs inside the
// CUDA tracking kernel after the Line is flattened into a device table.
//
// Deviations from the reference, all deliberate:
//   * errors throw stb::Error (derived from std::runtime_error) instead of
//     printing and calling exit() (e.g. SetP on an unknown name,
//     simtrack.cpp:8653-8685);
//   * there is no CPU Pass: an element type without a GPU implementation is
//     rejected when the Line is flattened.
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

namespace stb {

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

// Reference-particle state, GlobalVariables (simtrack.h:28-68).  Only the
// fields the tracking path reads are kept.
struct GlobalVariables {
  int A = 1, Q = 1, turn = 0;
  double m0 = 1.6726216e-27, m = 1.6726216e-27, q = 1.6021765e-19;
  double energy0 = 938.27201, energy = 99456.8, p = 1., cp = 1.;
  double gamma = 106., beta = 0.999955, brho = 331.738;
  double G = 1.7928474, Gr = 191.079706193;
  bool H_expand = false, radiate = false, quad_fringe = false;
  double U0rad = 0.;  // reference particle's radiation loss per turn, MeV (Cal_SRLoss_U0rad)
};
extern GlobalVariables GP;

// Cal_SRLoss_U0rad / Cal_SRLoss_U0rad_Track (simtrack.cpp:20691-20766): the
// reference particle's synchrotron-radiation loss per turn in MeV, into
// GP.U0rad (0 unless GP.radiate); the track form takes every bend's path on
// the orbit stored in the element before it (Cal_Orbit_Num fills X).
class Line;
double Cal_SRLoss_U0rad(Line &line, bool track_form = false);
// Cal_SRLoss_Particle (simtrack.cpp:20768-20781): x[6] passed once through
// every element but the RF cavities on the GPU (radiating bends radiate, with
// the particle-0 deviate stream), loss = (pt - pt0) GP.beta GP.energy (MeV,
// negative for a loss).  A particle that Track()'s loss tests would stop is
// rejected (stb::Error, STB_EINVAL) with x unchanged.
void Cal_SRLoss_Particle(Line &line, double x[], double &loss, int device = 0);
// Cal_gsbend_l_angle (simtrack.cpp:4006-4044).
void Cal_gsbend_l_angle(double x[6], double L, double Angle, double K0L, double &actual_l, double &actual_angle);

// Set_RefPartEnergy (simtrack.cpp:87-108) and Set_Spin_G (simtrack.cpp:110-115).
void Set_RefPartEnergy(double gamma, double E0, double Q, double A);
void Set_Spin_G(double g);

// Default integration slice lengths (simtrack.cpp:45-47).
extern double BLslice, QLslice, GLslice;

// Abstract element (simtrack.h:373-396).  Named parameters are reached through
// SetP/GetP exactly as in the reference; geometry and aperture are public
// fields.
class Element {
 public:
  explicit Element(std::string name);
  virtual ~Element() = default;
  void SetP(const char *name, double value);
  double GetP(const char *name) const;

  std::string NAME, TYPE, GROUP;
  double S = 0., L = 0.;
  double DX = 0., DY = 0., DS = 0.;
  double DTHETA = 0., DPHI = 0., DPSI = 0.;
  double APx = 1., APy = 1.;
  double X[6] = {0., 0., 0., 0., 0., 0.};  // closed orbit at the element's exit (simtrack.h:389), see Cal_Orbit_Num

  // Parameter access for the flattener (names as accepted by SetP).
  double P(const char *name) const { return GetP(name); }
  const double *KNL() const { return knl_; }
  const double *KNSL() const { return knsl_; }

 protected:
  void add_param(const char *name, double *slot, bool integer = false);
  void add_multipoles();
  virtual void on_setp(const char *name) { (void)name; }
  double knl_[11] = {0};
  double knsl_[11] = {0};

 private:
  struct Param {
    const char *name;
    double *slot;
    bool integer;
  };
  std::vector<Param> params_;
};

class DRIFT : public Element { public: DRIFT(std::string name, double l); };
class MARKER : public Element { public: MARKER(std::string name, double l); };
// Beam position monitors (simtrack.cpp:10470-10600): drifts for tracking.
class BPM : public Element { public: BPM(std::string name, double l); };
class HBPM : public Element { public: HBPM(std::string name, double l); };
class VBPM : public Element { public: VBPM(std::string name, double l); };
class SBEND : public Element {
 public:
  SBEND(std::string name, double l, double angle, double e1, double e2);
 private:
  double ANGLE, E1, E2, Nint;
};
class GSBEND : public Element {
 public:
  GSBEND(std::string name, double l, double angle, double k0l, double e1, double e2);
 private:
  double ANGLE, K0L, E1, E2, Nint;
};
class QUAD : public Element {
 public:
  QUAD(std::string name, double l, double k1l, double k1sl);
 private:
  double K1L, K1SL, Nint;
};
class SKEWQ : public Element {
 public:
  SKEWQ(std::string name, double l, double k1sl);
 private:
  double K1SL, Nint;
};
class SEXT : public Element {
 public:
  SEXT(std::string name, double l, double k2l, double k2sl);
 private:
  double K2L, K2SL, Nint;
};
class OCT : public Element {
 public:
  OCT(std::string name, double l, double k3l, double k3sl);
 private:
  double K3L, K3SL, Nint;
};
class MULT : public Element {
 public:
  MULT(std::string name, double l, const double knl[11], const double knsl[11]);
 private:
  double Nint, Norder;
};
class GMULT : public Element {
 public:
  GMULT(std::string name, double l, double angle, double e1, double e2, const double knl[11],
        const double knsl[11]);
 private:
  double ANGLE, E1, E2, Nint, Norder;
};
class SBENDMULT : public Element {
 public:
  SBENDMULT(std::string name, double l, double angle, double e1, double e2, const double knl[11],
            const double knsl[11]);
 private:
  double ANGLE, E1, E2, Nint, Norder;
};
class KICKER : public Element {
 public:
  KICKER(std::string name, double l, double hkick, double vkick);
 private:
  double HKICK, VKICK;
};
class HKICKER : public Element {
 public:
  HKICKER(std::string name, double l, double hkick);
 private:
  double HKICK;
};
class VKICKER : public Element {
 public:
  VKICKER(std::string name, double l, double vkick);
 private:
  double VKICK;
};
// Solenoid (simtrack.h:576-587): KS = Bs / (B rho) as in MAD-X; one slice.
class SOLEN : public Element {
 public:
  SOLEN(std::string name, double l, double ks);
 private:
  double KS;
};
// Coordinate patch (simtrack.h:1048-1059): a translation by (DX, DY, DS)
// followed by a rotation THETA about the y axis.  These are the patch's own
// parameters (SetP/GetP "DX", "DY", "DS", "THETA"), not the Element
// misalignment fields, which a patch ignores; L = DS at construction.
class PATCH : public Element {
 public:
  PATCH(std::string name, double dx, double dy, double ds, double theta);
 private:
  double PDX, PDY, PDS, THETA;
};
class RFCAV : public Element {
 public:
  RFCAV(std::string name, double l, double vrf, double frf, double phase0);
 private:
  double VRF, FRF, PHASE0;
};
class CRABRF : public Element {
 public:
  CRABRF(std::string name, double l, double vrf, double frf, double phase0);
 private:
  double VRF, FRF, PHASE0;
};
class CCMULT : public Element {
 public:
  CCMULT(std::string name, double l, double vrf, double frf, double phase0, double b1, double a1,
         double b2, double a2, double b3, double a3, double b4, double a4);
 private:
  double VRF, FRF, PHASE0, B1, A1, B2, A2, B3, A3, B4, A4;
};
class LBT : public Element {
 public:
  LBT(std::string name, double theta);
 private:
  double THETA;
};
class ILBT : public Element {
 public:
  ILBT(std::string name, double theta);
 private:
  double THETA;
};
class BEAMBEAM : public Element {
 public:
  BEAMBEAM(std::string name, int treatment, double np, double bbscale, double sigmal, int nslice,
           double emitx, double betax, double alfax, double emity, double betay, double alfay);
 protected:
  void on_setp(const char *name) override;
 private:
  double TREATMENT, NP, BBSCALE, SIGMAL, NSLICE, EMITX, BETAX, ALFAX, EMITY, BETAY, ALFAY;
};

// Line container (simtrack.h:1067-1100).  Owns its elements, like the
// reference: Delete/Replace/Empty and the destructor delete them.
class Line {
 public:
  Line() = default;
  ~Line();
  Line(const Line &) = delete;
  Line &operator=(const Line &) = delete;

  void Update();
  void Append(Element *x);
  void Delete(int i);
  void Insert(int i, Element *temp);
  void Replace(int i, Element *temp);
  void Rewind(int i);
  void Invert();
  void Empty();

  std::vector<Element *> Cell;
  double Length = 0.;
  long Ncell = 0;
  double frev0 = 0.;
  double Tune1 = 0., Tune2 = 0.;  // set by Cal_Tunes_Track (simtrack.h:1085)
  double Chromx1 = 0., Chromy1 = 0., Chromx2 = 0., Chromy2 = 0.;  // set by Cal_Chrom_Track
};

// Options that have no counterpart in Track()'s signature.
struct TrackOptions {
  double aperture_radius = 0.;  // circular aperture checked after every element; <= 0 disables
  int device = 0;
};

// Track() drop-in (simtrack.cpp:20791-20814): one particle, x[6] updated in
// place; stable/lost_turn/lost_post as in the reference.  Runs on the GPU.
void Track(Line &line, double x[], int nturn, int &stable, int &lost_turn, int &lost_post);

// Batched Track over n particles in AoS x[n*6] (the per-particle loop of the
// DA drivers, simtrack.cpp:21389-21441, moved onto the GPU in one launch).
void Track_Batch(Line &line, double *x, long n, int nturn, int *stable, int *lost_turn,
                 int *lost_post, const TrackOptions &opt = TrackOptions());

// Track_DA (simtrack.cpp:21389-21441): twin-particle bisection of the stable
// amplitude at 10 phase angles between 0 and 50 sigma, written to `filename`
// as the reference writes it ("angle sigma" per line; NULL: no file).  All
// midpoints the bisections can visit are tracked in one GPU launch and the
// bisections replayed on the outcomes, which reproduces the reference's file.
// angles_out / sigma_out (optional) receive the 10 results.
void Track_DA(Line &line, int nturn, double deltap0, double sigmax0, double sigmay0, const char *filename,
              double *angles_out = nullptr, double *sigma_out = nullptr, int device = 0);

// The other bisection drivers, same method and output format:
//   Track_DA1 (simtrack.cpp:21443-21495): twin particles, 5 angles 15..75 deg, 0-50 sigma;
//   Track_DA2 (21497-21533): single particles, 10 angles (90/11)(i+1) deg, 0-50 sigma;
//   Track_DA3 (21535-21572): Cal_Orbit_Num(line, 0) first, single particles, 5 angles 15..75 deg, 0-30 sigma;
//   Track_DA_Radial (21682-21734): twin particles through Track_Radial, 10 angles, 0-15 sigma.
void Track_DA1(Line &line, int nturn, double deltap0, double sigmax0, double sigmay0, const char *filename,
               double *angles_out = nullptr, double *sigma_out = nullptr, int device = 0);
void Track_DA2(Line &line, int nturn, double deltap0, double sigmax0, double sigmay0, const char *filename,
               double *angles_out = nullptr, double *sigma_out = nullptr, int device = 0);
void Track_DA3(Line &line, int nturn, double deltap0, double sigmax0, double sigmay0, const char *filename,
               double *angles_out = nullptr, double *sigma_out = nullptr, int device = 0);
void Track_DA_Radial(Line &line, int nturn, double deltap0, double sigmax0, double sigmay0, const char *filename,
                     double *angles_out = nullptr, double *sigma_out = nullptr, int device = 0);

// Track_DA_Uniform (simtrack.cpp:21574-21603) / Track_DA_Radial_Uniform
// (21736-21764): amplitudes 1, 1.2, ..., 30.8 sigma at one angle [rad]
// through Track / Track_Radial, one "angle sigma stable" line per amplitude
// up to and including the first loss (where the reference ends the process;
// here the function returns).  Returns the number of lines; sigma_out /
// stable_out (optional, 150 entries) receive their values.
long Track_DA_Uniform(Line &line, int nturn, double deltap0, double angle, double sigmax0, double sigmay0,
                      const char *filename, double *sigma_out = nullptr, double *stable_out = nullptr,
                      int device = 0);
long Track_DA_Radial_Uniform(Line &line, int nturn, double deltap0, double angle, double sigmax0, double sigmay0,
                             const char *filename, double *sigma_out = nullptr, double *stable_out = nullptr,
                             int device = 0);

// Cal_Tunes_Track (simtrack.cpp:20971-21025): tunes of a tracked particle by
// FineTuneFinder over its Track_tbt record in [tune_low, tune_high).  The
// first form tracks x (x[0], x[2] below 1e-9 are raised by 1e-9, in place)
// for Nturn turns and leaves tune1/tune2 unchanged if it is lost; the second
// tracks the closed orbit at deltap0 for 1,024 turns and stores the tunes in
// line.Tune1 / line.Tune2 (0 if the particle is lost).
void Cal_Tunes_Track(Line &line, double x[], int Nturn, double &tune1, double &tune2, int device = 0);
void Cal_Tunes_Track(Line &line, double deltap0, int device = 0);

// Cal_Chrom_Track (simtrack.cpp:21027-21051): first and second order
// chromaticities from the tracked tunes at deltap = +3e-4, -3e-4 and 0
// (Cal_Tunes_Track(line, deltap) each), stored in line.Chromx1 ... Chromy2.
void Cal_Chrom_Track(Line &line, int device = 0);

// Cal_Orbit_Num (simtrack.cpp:14947-15030): 4D closed orbit at momentum
// offset deltap by Newton iteration on the one-turn map (RF voltages off,
// one-sided finite differences with step 1e-9, the reference's own matrix
// inversion), one-turn tracks on the GPU; fills every element's X[] with the
// orbit after it.  Throws Error(STB_EABORTED) where the reference exits.
void Cal_Orbit_Num(Line &line, double deltap, int device = 0);

// Read_MADX_Lattice (simtrack.cpp:13591-13791): appends the elements of a
// MAD-X TFS twiss table (columns NAME KEYWORD S L ANGLE E1 E2 TILT K0L K0SL
// ... K10L K10SL KS) to `line`, mapping keywords to element types as the
// reference does.  Throws Error(STB_EUNSUPPORTED) for an electron lens (not
// implemented on the GPU path) and Error(STB_EINVAL) for an unreadable file.
void Read_MADX_Lattice(Line &line, const char *filename);

// Read_BMAD_Lattice (simtrack.cpp:14054-14244): appends the elements of a
// Bmad table (one header line, then rows NAME KEY S L ANGLE ANGLE1 E1 E2 TILT
// X_OFFSET Z_OFFSET X_PITCH K0L K0SL ... K10L K10SL KS HKICK VKICK) to
// `line`, mapping keys to element types as the reference does.  Rows whose
// S column is not a number (column-name and unit lines) are skipped.  Throws
// Error(STB_EUNSUPPORTED) for an electron lens and Error(STB_EINVAL) for an
// unreadable file or a beam-beam element of non-zero length.
void Read_BMAD_Lattice(Line &line, const char *filename);

// Track_tbt() drop-in (simtrack.cpp:20841-20860): Track() that also records
// x[6] at the start of every turn, x_tbt[turn*6 + k], up to and including the
// turn of the loss.  Track_tbt_Batch: n particles (AoS x[n*6], stable[] as
// Track()'s input flags), x_tbt[(i*nturn + turn)*6 + k].
void Track_tbt(Line &line, double x[], int nturn, double x_tbt[], int &stable, int &lost_turn, int &lost_post);
void Track_tbt_Batch(Line &line, double *x, long n, int nturn, double *x_tbt, int *stable, int *lost_turn,
                     int *lost_post, int device = 0);
// Track_tbt() with a BPM index (simtrack.cpp:20884-20905): records x[6] after
// element bpm_index in every turn that reaches it (x_tbt[turn*6 + k]).  The
// batch form runs the tracking kernel's per-element probe, so n x Ncell x
// 48 B must stay under 4 GB.
void Track_tbt(Line &line, double x[], int nturn, double x_tbt[], int &bpm_index, int &stable, int &lost_turn,
               int &lost_post);
void Track_tbt_bpm_Batch(Line &line, double *x, long n, int nturn, double *x_tbt, int bpm_index, int *stable,
                         int *lost_turn, int *lost_post, int device = 0);
// Track_tbt_spin() (simtrack.cpp:20863-20882): the same with spin tracking,
// x[9] and x_tbt[turn*9 + k]; the batch form takes x9[n*9], x_tbt9[(i*nturn + turn)*9 + k].
void Track_tbt_spin(Line &line, double x[], int nturn, double x_tbt[], int &stable, int &lost_turn,
                    int &lost_post);
void Track_tbt_spin_Batch(Line &line, double *x9, long n, int nturn, double *x_tbt9, int *stable, int *lost_turn,
                          int *lost_post, int device = 0);
// Track_tbt_spin() with a BPM index (simtrack.cpp:20907-20927): x[9] recorded
// after element bpm_index; n x Ncell x 72 B must stay under 4 GB.
void Track_tbt_spin(Line &line, double x[], int nturn, double x_tbt[], int &bpm_index, int &stable, int &lost_turn,
                    int &lost_post);
void Track_tbt_spin_bpm_Batch(Line &line, double *x9, long n, int nturn, double *x_tbt9, int bpm_index, int *stable,
                              int *lost_turn, int *lost_post, int device = 0);

// FineTuneFinder's search window used by Track_tbt_FMA (simtrack.cpp:27).
extern double tune_low, tune_high;

// Track_tbt_FMA (simtrack.cpp:21179-21241): frequency map of a 0-6 sigma
// quarter-disc grid (step 0.1 sigma) around the closed orbit at deltap0,
// 2,048 turns, tunes of turns 0-1023 and 1023-2046 by FineTuneFinder in
// [tune_low, tune_high); writes the reference's FMA-output.dat rows (to
// `filename`) and returns their number.
long Track_tbt_FMA(Line &line, double deltap0, double sigmax0, double sigmay0,
                   const char *filename = "./FMA-output.dat", int device = 0);

// Track_tbt_Lyapunov (simtrack.cpp:21243-21306): for a 0-6 sigma quarter-disc
// grid (step 0.05 sigma), the growth of the distance between a particle and
// a twin 1e-6 away over 2,048 turns, averaged over the last 25 turns; writes
// the reference's Lmap-output.dat rows (to `filename`) and returns their number.
long Track_tbt_Lyapunov(Line &line, double deltap0, double sigmax0, double sigmay0,
                        const char *filename = "./Lmap-output.dat", int device = 0);

// Cal_dz0_OnMomentumPart (simtrack.cpp:20929-20940): x0[6] (in/out) passes
// every element with z and pt reset to zero before each; dz0[j] (Ncell
// entries) = its z after element j.  Track_wrt_OnMomentumPart (20942-20967):
// Track() with dz0[j] subtracted from z after every element j (Track_Radial
// with a caller-supplied path).  The batch form takes AoS x[n*6].
void Cal_dz0_OnMomentumPart(Line &line, double x0[], double dz0[]);
void Cal_dz0_OnMomentumPart_dev(Line &line, double x0[], double dz0[], int device);
void Track_wrt_OnMomentumPart(Line &line, double x[], double dz0[], int nturn, int &stable, int &lost_turn,
                              int &lost_post);
void Track_wrt_OnMomentumPart_Batch(Line &line, double *x, long n, const double *dz0, int nturn, int *stable,
                                    int *lost_turn, int *lost_post, int device = 0);

// Track_Radial() drop-in (simtrack.cpp:21641-21680): Track() with z taken
// relative to the on-momentum reference particle after every element.
void Track_Radial(Line &line, double x[], int nturn, int &stable, int &lost_turn, int &lost_post);

// Track_Spin() drop-in (simtrack.cpp:21766-21789): x[9] = orbit + spin.
void Track_Spin(Line &line, double x[], int nturn, int &stable, int &lost_turn, int &lost_post);

}  // namespace stb
