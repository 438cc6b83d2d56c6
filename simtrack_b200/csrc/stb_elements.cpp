// Element classes and the Line container of the C++ host API.
// Constructor arguments, default slice counts, parameter names accepted by
// SetP/GetP and the Line editing semantics follow simtrack.h:373-1100 and
// simtrack.cpp:8357-12431; see each constructor for its reference line.
#include "simtrack_b200.hpp"
#include "stb_status.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>

namespace stb {

GlobalVariables GP;
double BLslice = 0.25;  // simtrack.cpp:45
double QLslice = 0.05;  // simtrack.cpp:46
double GLslice = 0.05;  // simtrack.cpp:47

// Set_RefPartEnergy, simtrack.cpp:87-108: same expressions, same order.
void Set_RefPartEnergy(double gamma, double E0, double Q, double A) {
  GP.Q = (int)Q;
  GP.A = (int)A;
  GP.m0 = E0 * 1.0e6 * 1.6021765e-19 / 299792458. / 299792458.;
  GP.m = gamma * GP.m0;
  GP.q = Q * 1.6021765e-19;
  GP.gamma = gamma;
  GP.beta = std::sqrt(1.0 - 1.0 / gamma / gamma);
  GP.energy0 = E0;
  GP.energy = gamma * GP.energy0;
  GP.cp = GP.energy * GP.beta;
  GP.p = GP.energy * GP.beta * 1.0e6 * 1.6021765e-19 / 299792458.;
  GP.brho = 3.33564095198 * GP.beta * (GP.energy / 1000) / GP.Q;
}

// Set_Spin_G, simtrack.cpp:110-115
void Set_Spin_G(double g) {
  GP.G = g;
  GP.Gr = g * GP.gamma;
}

Element::Element(std::string name) : NAME(std::move(name)) {}

void Element::add_param(const char *name, double *slot, bool integer) {
  params_.push_back(Param{name, slot, integer});
}

void Element::add_multipoles() {
  static const char *kn[11] = {"K0L", "K1L", "K2L", "K3L", "K4L", "K5L",
                               "K6L", "K7L", "K8L", "K9L", "K10L"};
  static const char *ks[11] = {"K0SL", "K1SL", "K2SL", "K3SL", "K4SL", "K5SL",
                               "K6SL", "K7SL", "K8SL", "K9SL", "K10SL"};
  for (int i = 0; i < 11; i++) add_param(kn[i], &knl_[i]);
  for (int i = 0; i < 11; i++) add_param(ks[i], &knsl_[i]);
}

void Element::SetP(const char *name, double value) {
  for (auto &p : params_) {
    if (std::strcmp(p.name, name) == 0) {
      // Integer parameters are truncated like the reference's int(value).
      *p.slot = p.integer ? (double)(int)value : value;
      on_setp(name);
      return;
    }
  }
  throw Error(STB_EINVAL, TYPE + " does not have a parameter of " + std::string(name));
}

double Element::GetP(const char *name) const {
  for (auto &p : params_)
    if (std::strcmp(p.name, name) == 0) return *p.slot;
  throw Error(STB_EINVAL, TYPE + " does not have a parameter of " + std::string(name));
}

static void require(bool ok, const std::string &msg) {
  if (!ok) throw Error(STB_EINVAL, msg);
}

// Norder from the highest non-zero coefficient, MULT ctor simtrack.cpp:8943-8950
static double highest_order(const double *knl, const double *knsl) {
  for (int i = 0; i < 10; i++)
    if (knl[10 - i] != 0. || knsl[10 - i] != 0.) return 10 - i;
  return 1;
}

// DRIFT, simtrack.cpp:8399-8412 (no settable parameters)
DRIFT::DRIFT(std::string name, double l) : Element(std::move(name)) {
  require(l >= 0, "Error: check signs of L and S of DRFIT " + NAME);
  TYPE = "DRIFT";
  L = l;
}

// MARKER, simtrack.cpp:10590-10603
MARKER::MARKER(std::string name, double l) : Element(std::move(name)) {
  require(l >= 0, "Error: MARKER length should be non-negative.");
  TYPE = "MARKER";
  L = l;
}

// BPM / HBPM / VBPM, simtrack.cpp:10470-10600 (Pass = DRIFT_Pass)
BPM::BPM(std::string name, double l) : Element(std::move(name)) {
  require(l >= 0, "Error: BPM length should be non-negative.");
  TYPE = "BPM";
  L = l;
}
HBPM::HBPM(std::string name, double l) : Element(std::move(name)) {
  require(l >= 0, "Error: HBPM length should be non-negative.");
  TYPE = "HBPM";
  L = l;
}
VBPM::VBPM(std::string name, double l) : Element(std::move(name)) {
  require(l >= 0, "Error: VBPM length should be non-negative.");
  TYPE = "VBPM";
  L = l;
}

// SBEND, simtrack.cpp:8441-8458
SBEND::SBEND(std::string name, double l, double angle, double e1, double e2)
    : Element(std::move(name)), ANGLE(angle), E1(e1), E2(e2) {
  require(l > 0, "Error: SBEND length should be positive. ");
  TYPE = "SBEND";
  L = l;
  Nint = int(L / BLslice) + 1;
  add_param("ANGLE", &ANGLE);
  add_param("E1", &E1);
  add_param("E2", &E2);
  add_param("Nint", &Nint, true);
}

// GSBEND, simtrack.cpp:8529-8547
GSBEND::GSBEND(std::string name, double l, double angle, double k0l, double e1, double e2)
    : Element(std::move(name)), ANGLE(angle), K0L(k0l), E1(e1), E2(e2) {
  require(l > 0, "Error: GSBEND length should be positive. ");
  TYPE = "GSBEND";
  L = l;
  Nint = int(L / BLslice) + 1;
  add_param("ANGLE", &ANGLE);
  add_param("K0L", &K0L);
  add_param("E1", &E1);
  add_param("E2", &E2);
  add_param("Nint", &Nint, true);
}

// QUAD, simtrack.cpp:8626-8643
QUAD::QUAD(std::string name, double l, double k1l, double k1sl)
    : Element(std::move(name)), K1L(k1l), K1SL(k1sl) {
  require(l >= 0, "Error: QUAD length should be non-negative.");
  TYPE = "QUAD";
  L = l;
  Nint = int(L / QLslice) + 1;
  add_param("K1L", &K1L);
  add_param("K1SL", &K1SL);
  add_param("Nint", &Nint, true);
}

// SKEWQ, simtrack.cpp:8706-8720
SKEWQ::SKEWQ(std::string name, double l, double k1sl) : Element(std::move(name)), K1SL(k1sl) {
  require(l >= 0, "Error: SKEWQ length should be non-negative.");
  TYPE = "SKEWQ";
  L = l;
  Nint = int(L / QLslice) + 1;
  add_param("K1SL", &K1SL);
  add_param("Nint", &Nint, true);
}

// SEXT, simtrack.cpp:8773-8790
SEXT::SEXT(std::string name, double l, double k2l, double k2sl)
    : Element(std::move(name)), K2L(k2l), K2SL(k2sl) {
  require(l >= 0, "Error: SEXT length should be non-negative.");
  TYPE = "SEXT";
  L = l;
  Nint = int(L / QLslice) + 1;
  add_param("K2L", &K2L);
  add_param("K2SL", &K2SL);
  add_param("Nint", &Nint, true);
}

// OCT, simtrack.cpp:8853-8870
OCT::OCT(std::string name, double l, double k3l, double k3sl)
    : Element(std::move(name)), K3L(k3l), K3SL(k3sl) {
  require(l >= 0, "Error: OCT length should be non-negative.");
  TYPE = "OCT";
  L = l;
  Nint = int(L / QLslice) + 1;
  add_param("K3L", &K3L);
  add_param("K3SL", &K3SL);
  add_param("Nint", &Nint, true);
}

// MULT, simtrack.cpp:8933-8957.  As in the reference, SetP on a coefficient
// does not recompute Norder; SetP("Norder") sets it explicitly.
MULT::MULT(std::string name, double l, const double knl[11], const double knsl[11])
    : Element(std::move(name)) {
  require(l >= 0, "Error: MULT length should be non-negative.");
  TYPE = "MULT";
  L = l;
  for (int i = 0; i < 11; i++) {
    knl_[i] = knl[i];
    knsl_[i] = knsl[i];
  }
  Nint = int(L / QLslice) + 1;
  Norder = highest_order(knl_, knsl_);
  add_multipoles();
  add_param("Nint", &Nint, true);
  add_param("Norder", &Norder, true);
}

// GMULT, simtrack.cpp:9046-9069
GMULT::GMULT(std::string name, double l, double angle, double e1, double e2, const double knl[11],
             const double knsl[11])
    : Element(std::move(name)), ANGLE(angle), E1(e1), E2(e2) {
  require(l >= 0, "Error: GMULT length should be non-negative.");
  TYPE = "GMULT";
  L = l;
  Nint = int(L / BLslice) + 1;
  for (int i = 0; i < 11; i++) {
    knl_[i] = knl[i];
    knsl_[i] = knsl[i];
  }
  Norder = highest_order(knl_, knsl_);
  add_param("ANGLE", &ANGLE);
  add_param("E1", &E1);
  add_param("E2", &E2);
  add_param("Nint", &Nint, true);
  add_multipoles();
  add_param("Norder", &Norder, true);
}

// SBENDMULT, simtrack.cpp:9192-9215
SBENDMULT::SBENDMULT(std::string name, double l, double angle, double e1, double e2,
                     const double knl[11], const double knsl[11])
    : Element(std::move(name)), ANGLE(angle), E1(e1), E2(e2) {
  require(l >= 0, "Error: SBENDMULT length should be non-negative.");
  TYPE = "SBENDMULT";
  L = l;
  Nint = int(L / BLslice) + 1;
  for (int i = 0; i < 11; i++) {
    knl_[i] = knl[i];
    knsl_[i] = knsl[i];
  }
  Norder = highest_order(knl_, knsl_);
  add_param("ANGLE", &ANGLE);
  add_param("E1", &E1);
  add_param("E2", &E2);
  add_param("Nint", &Nint, true);
  add_multipoles();
  add_param("Norder", &Norder, true);
}

// KICKER / HKICKER / VKICKER, simtrack.cpp:9912-10100
// SOLEN, simtrack.cpp:9645-9686 (Nint fixed at 1; only KS is settable)
SOLEN::SOLEN(std::string name, double l, double ks) : Element(std::move(name)), KS(ks) {
  require(l > 0, "Solenoid: L must be positive. ");
  TYPE = "SOLEN";
  L = l;
  add_param("KS", &KS);
}

// PATCH, simtrack.cpp:12262-12321
PATCH::PATCH(std::string name, double dx, double dy, double ds, double theta)
    : Element(std::move(name)), PDX(dx), PDY(dy), PDS(ds), THETA(theta) {
  TYPE = "PATCH";
  L = ds;
  add_param("DX", &PDX);
  add_param("DY", &PDY);
  add_param("DS", &PDS);
  add_param("THETA", &THETA);
}

KICKER::KICKER(std::string name, double l, double hkick, double vkick)
    : Element(std::move(name)), HKICK(hkick), VKICK(vkick) {
  require(l >= 0, "Error: KICKER length should be non-negative.");
  TYPE = "KICKER";
  L = l;
  add_param("HKICK", &HKICK);
  add_param("VKICK", &VKICK);
}
HKICKER::HKICKER(std::string name, double l, double hkick) : Element(std::move(name)), HKICK(hkick) {
  require(l >= 0, "Error: HKICKER length should be non-negative.");
  TYPE = "HKICKER";
  L = l;
  add_param("HKICK", &HKICK);
}
VKICKER::VKICKER(std::string name, double l, double vkick) : Element(std::move(name)), VKICK(vkick) {
  require(l >= 0, "Error: VKICKER length should be non-negative.");
  TYPE = "VKICKER";
  L = l;
  add_param("VKICK", &VKICK);
}

// RFCAV, simtrack.cpp:10630-10645
RFCAV::RFCAV(std::string name, double l, double vrf, double frf, double phase0)
    : Element(std::move(name)), VRF(vrf), FRF(frf), PHASE0(phase0) {
  require(l >= 0, "Error: RFCAV length must be non-negative.");
  TYPE = "RFCAV";
  L = l;
  add_param("VRF", &VRF);
  add_param("FRF", &FRF);
  add_param("PHASE0", &PHASE0);
}

// CRABRF, simtrack.cpp:10719-10734
CRABRF::CRABRF(std::string name, double l, double vrf, double frf, double phase0)
    : Element(std::move(name)), VRF(vrf), FRF(frf), PHASE0(phase0) {
  require(l >= 0, "Error: CRABRF length must be non-negative.");
  TYPE = "CRABRF";
  L = l;
  add_param("VRF", &VRF);
  add_param("FRF", &FRF);
  add_param("PHASE0", &PHASE0);
}

// CCMULT, simtrack.cpp:10815-10840
CCMULT::CCMULT(std::string name, double l, double vrf, double frf, double phase0, double b1,
               double a1, double b2, double a2, double b3, double a3, double b4, double a4)
    : Element(std::move(name)), VRF(vrf), FRF(frf), PHASE0(phase0), B1(b1), A1(a1), B2(b2),
      A2(a2), B3(b3), A3(a3), B4(b4), A4(a4) {
  require(l >= 0, "Error: CCMULT length must be non-negative.");
  TYPE = "CCMULT";
  L = l;
  add_param("VRF", &VRF);
  add_param("FRF", &FRF);
  add_param("PHASE0", &PHASE0);
  add_param("B1", &B1);
  add_param("A1", &A1);
  add_param("B2", &B2);
  add_param("A2", &A2);
  add_param("B3", &B3);
  add_param("A3", &A3);
  add_param("B4", &B4);
  add_param("A4", &A4);
}

// LBT / ILBT, simtrack.cpp:10960-10967, 11009-11016 (L = 0)
LBT::LBT(std::string name, double theta) : Element(std::move(name)), THETA(theta) {
  TYPE = "LBT";
  L = 0.;
  add_param("THETA", &THETA);
}
ILBT::ILBT(std::string name, double theta) : Element(std::move(name)), THETA(theta) {
  TYPE = "ILBT";
  L = 0.;
  add_param("THETA", &THETA);
}

// BEAMBEAM, simtrack.cpp:11058-11076 (L = 0); TREATMENT must be 4 or 6 (11081-11088)
BEAMBEAM::BEAMBEAM(std::string name, int treatment, double np, double bbscale, double sigmal,
                   int nslice, double emitx, double betax, double alfax, double emity,
                   double betay, double alfay)
    : Element(std::move(name)), TREATMENT(treatment), NP(np), BBSCALE(bbscale), SIGMAL(sigmal),
      NSLICE(nslice), EMITX(emitx), BETAX(betax), ALFAX(alfax), EMITY(emity), BETAY(betay),
      ALFAY(alfay) {
  TYPE = "BEAMBEAM";
  L = 0.;
  add_param("TREATMENT", &TREATMENT, true);
  add_param("NP", &NP);
  add_param("BBSCALE", &BBSCALE);
  add_param("SIGMAL", &SIGMAL);
  add_param("NSLICE", &NSLICE, true);
  add_param("EMITX", &EMITX);
  add_param("EMITY", &EMITY);
  add_param("BETAX", &BETAX);
  add_param("ALFAX", &ALFAX);
  add_param("BETAY", &BETAY);
  add_param("ALFAY", &ALFAY);
}

void BEAMBEAM::on_setp(const char *name) {
  if (std::strcmp(name, "TREATMENT") == 0 && TREATMENT != 4 && TREATMENT != 6) {
    TREATMENT = 6;
    throw Error(STB_EINVAL, "Error: beambeam treatment only can be 4 or 6");
  }
}

// Line, simtrack.cpp:12341-12431
Line::~Line() { Empty(); }

void Line::Update() {
  double sp = 0.;
  for (size_t i = 0; i < Cell.size(); i++) {
    sp = Cell[i]->L + sp;
    Cell[i]->S = sp;
  }
  Ncell = (long)Cell.size();
  Length = sp;
  frev0 = (299792458. * GP.beta) / Length;
}

void Line::Append(Element *x) {
  Cell.push_back(x);
  Update();
}

void Line::Delete(int i) {
  if (i < 0 || i >= (int)Cell.size()) return;
  delete Cell[i];
  Cell.erase(Cell.begin() + i);
  Update();
}

void Line::Insert(int i, Element *temp) {
  if (i < 0 || i >= (int)Cell.size()) return;
  Cell.insert(Cell.begin() + i, temp);
  Update();
}

void Line::Replace(int i, Element *temp) {
  if (i < 0 || i >= (int)Cell.size()) return;
  delete Cell[i];
  Cell[i] = temp;
  Update();
}

void Line::Rewind(int i) {
  if (i < 0 || i >= (int)Cell.size()) return;
  std::rotate(Cell.begin(), Cell.begin() + i, Cell.end());
  Update();
}

void Line::Invert() { std::reverse(Cell.begin(), Cell.end()); }

void Line::Empty() {
  for (auto *p : Cell) delete p;
  Cell.clear();
  Ncell = 0;
}

}  // namespace stb
