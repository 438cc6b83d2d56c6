// Lattice file readers: MAD-X TFS twiss tables -> Line
// (Read_MADX_Lattice, simtrack.cpp:13591-13791).
//
// The reader locates the column header (the line holding "KEYWORD" among the
// first 100 lines), skips it and the format line after it, and reads every
// further row as NAME KEYWORD S L ANGLE E1 E2 TILT, the 22 normal/skew
// integrated strengths K0L K0SL ... K10L K10SL, and KS.  Names and keywords
// lose their quotes.  Keyword -> element, as the reference maps them:
//   DRIFT -> DRIFT;  SBEND -> GSBEND if K0L != 0 and K2L == 0, SBEND if K1L
//   and K2L are 0, GMULT otherwise (all with DPSI = TILT);  RBEND -> SBEND
//   with E1 = E2 = ANGLE/2 if K1L and K2L are 0, else GMULT;  QUADRUPOLE,
//   SEXTUPOLE, OCTUPOLE -> QUAD, SEXT, OCT with their (K, KS) pair and
//   DPSI = TILT;  HKICKER, VKICKER, TKICKER -> zero-kick correctors;
//   MULTIPOLE -> MULT(L, KNL, KNSL) with DPSI = TILT;  VMONITOR -> VBPM,
//   MONITOR -> BPM;  MARKER -> MARKER;  SOLENOID -> a drift when KS or L is
//   zero;  RFCAVITY -> RFCAV with zero voltage;  BEAMBEAM -> a BEAMBEAM with
//   zero intensity;  anything else -> DRIFT.
#include <fstream>
#include <sstream>
#include <string>

#include "simtrack_b200.hpp"
#include "stb_status.hpp"

namespace stb {

namespace {

std::string unquote(const std::string &s) { return s.size() >= 2 ? s.substr(1, s.size() - 2) : std::string(); }

}  // namespace

void Read_MADX_Lattice(Line &line, const char *filename) {
  if (!filename) throw Error(STB_EINVAL, "NULL file name");
  std::ifstream f(filename);
  if (!f) throw Error(STB_EINVAL, std::string("error in opening the file: ") + filename);
  std::string row;
  int header = -1;
  for (int i = 0; i < 100 && std::getline(f, row); i++)
    if (row.find("KEYWORD") != std::string::npos) {
      header = i;
      break;
    }
  // As the reference, a file without the header within 100 lines is read
  // from line 102 on.
  const int nskip = (header < 0 ? 100 : header) + 2;
  f.clear();
  f.seekg(0);
  for (int i = 0; i < nskip && std::getline(f, row); i++) {
  }
  while (std::getline(f, row)) {
    std::istringstream ss(row);
    std::string qname, qtype;
    double s = 0, l = 0, angle = 0, e1 = 0, e2 = 0, tilt = 0, ks = 0;
    double knl[11] = {0}, knsl[11] = {0};
    ss >> qname >> qtype >> s >> l >> angle >> e1 >> e2 >> tilt;
    for (int k = 0; k < 11; k++) ss >> knl[k] >> knsl[k];
    ss >> ks;
    if (qname.empty()) continue;
    const std::string name = unquote(qname), type = unquote(qtype);
    Element *e = nullptr;
    if (type == "DRIFT") {
      e = new DRIFT(name, l);
    } else if (type == "SBEND") {
      if (knl[0] != 0. && knl[2] == 0.)
        e = new GSBEND(name, l, angle, knl[0], e1, e2);
      else if (knl[1] == 0. && knl[2] == 0.)
        e = new SBEND(name, l, angle, e1, e2);
      else
        e = new GMULT(name, l, angle, e1, e2, knl, knsl);
      e->DPSI = tilt;
    } else if (type == "RBEND") {
      if (knl[1] == 0. && knl[2] == 0.)
        e = new SBEND(name, l, angle, angle / 2, angle / 2);
      else
        e = new GMULT(name, l, angle, e1, e2, knl, knsl);
    } else if (type == "QUADRUPOLE") {
      e = new QUAD(name, l, knl[1], knsl[1]);
      e->DPSI = tilt;
    } else if (type == "SEXTUPOLE") {
      e = new SEXT(name, l, knl[2], knsl[2]);
      e->DPSI = tilt;
    } else if (type == "OCTUPOLE") {
      e = new OCT(name, l, knl[3], knsl[3]);
      e->DPSI = tilt;
    } else if (type == "HKICKER") {
      e = new HKICKER(name, l, 0.0);
    } else if (type == "VKICKER") {
      e = new VKICKER(name, l, 0.0);
    } else if (type == "TKICKER") {
      e = new KICKER(name, l, 0.0, 0.0);
    } else if (type == "MULTIPOLE") {
      e = new MULT(name, l, knl, knsl);
      e->DPSI = tilt;
    } else if (type == "VMONITOR") {
      e = new VBPM(name, l);
    } else if (type == "MONITOR") {
      e = new BPM(name, l);
    } else if (type == "MARKER") {
      e = new MARKER(name, l);
    } else if (type == "SOLENOID") {
      if (ks != 0.0 && l != 0.)
        throw Error(STB_EUNSUPPORTED, "solenoid " + name + " with KS != 0 is not implemented on the GPU path");
      e = new DRIFT(name, l);
    } else if (type == "RFCAVITY") {
      e = new RFCAV(name, l, 0.0, 0.0, 0.);
    } else if (type == "BEAMBEAM") {
      if (l != 0.) throw Error(STB_EINVAL, "Beam-Beam element should have zero length!");
      e = new BEAMBEAM(name, 6, 0., 1, 0.4545, 11, 2.5e-06, 2.5e-06, 0.53, 0.0, 0.53, 0.0);
    } else if (type == "ELENS") {
      throw Error(STB_EUNSUPPORTED, "electron lens " + name + " is not implemented on the GPU path");
    } else {
      e = new DRIFT(name, l);
    }
    line.Cell.push_back(e);
  }
  line.Update();
}

}  // namespace stb
