// Lattice file readers: MAD-X TFS twiss tables and Bmad tables -> Line
// (Read_MADX_Lattice, simtrack.cpp:13591-13791; Read_BMAD_Lattice,
// simtrack.cpp:14054-14244).
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
//   MONITOR -> BPM;  MARKER -> MARKER;  SOLENOID -> SOLEN, or a drift when
//   KS or L is zero;  RFCAVITY -> RFCAV with zero voltage;  BEAMBEAM -> a
//   BEAMBEAM with zero intensity;  anything else -> DRIFT.
//
// Bmad tables (Read_BMAD_Lattice, simtrack.cpp:14054-14244): see below.
#include <cmath>
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
        e = new SOLEN(name, l, ks);
      else
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

// Bmad table reader.  After one header line every row is read as NAME KEY S
// L ANGLE ANGLE1 E1 E2 TILT X_OFFSET Z_OFFSET X_PITCH, the 22 normal/skew
// integrated strengths K0L K0SL ... K10L K10SL, then KS HKICK VKICK.  As in
// the reference the numeric fields keep their values from the previous row
// when a row ends early (the first missing field reads as 0).  Key ->
// element, case-sensitive as the reference compares them:
//   Drift -> DRIFT;  Sbend -> MULT(L, KNL, KNSL) if |ANGLE| < 1e-9, GSBEND
//   if |ANGLE - K0L| > 1e-6, else (K0L := 0) SBEND if K1L and K2L are 0,
//   SBENDMULT otherwise;  RBEND -> SBEND with E1 = E2 = ANGLE/2 if K1L and K2L
//   are 0, else SBENDMULT with those edges;  Quadrupole, Sextupole, OCTUPOLE
//   -> QUAD, SEXT, OCT with their (K, KS) pair;  HKICKER, VKICKER, Kicker ->
//   correctors with HKICK / VKICK;  Multipole -> MULT if K0L == 0, else a
//   1 um SBEND "<name>_tb" of angle K0L;  HMONITOR, VMONITOR, Monitor -> HBPM,
//   VBPM, BPM;  MARKER -> MARKER;  Solenoid -> SOLEN(L, KS), a drift when L
//   is 0;  RFcavity -> RFCAV with zero voltage;  BEAMBEAM -> a BEAMBEAM with
//   zero intensity;  Patch -> PATCH(X_OFFSET, 0, Z_OFFSET, -X_PITCH);
//   anything else (Beginning_Ele, Marker, Instrument, Pipe, ...) -> DRIFT.
// The reference turns rows whose S column is not a number (the table's
// column-name and unit lines) into drifts of an undefined length; they are
// skipped here.
void Read_BMAD_Lattice(Line &line, const char *filename) {
  if (!filename) throw Error(STB_EINVAL, "NULL file name");
  std::ifstream f(filename);
  if (!f) throw Error(STB_EINVAL, std::string("error in opening the file: ") + filename);
  std::string row;
  std::getline(f, row);
  // fields persist from row to row, as the reference's locals do
  constexpr int kNum = 35;  // S .. VKICK
  double v[kNum] = {0};
  while (std::getline(f, row)) {
    std::istringstream ss(row);
    std::string name, type;
    if (!(ss >> name >> type)) continue;
    int got = 0;
    for (; got < kNum; got++) {
      double d;
      if (!(ss >> d)) {
        v[got] = 0.;
        break;
      }
      v[got] = d;
    }
    if (got == 0) continue;  // S is not a number: a column-name or unit line
    double l = v[1];
    const double angle = v[2], e1 = v[4], e2 = v[5], xoff = v[7], zoff = v[8], xpitch = v[9];
    double knl[11], knsl[11];
    for (int k = 0; k < 11; k++) {
      knl[k] = v[10 + 2 * k];
      knsl[k] = v[11 + 2 * k];
    }
    const double ks = v[32], hkick = v[33], vkick = v[34];
    Element *e = nullptr;
    if (type == "Drift") {
      e = new DRIFT(name, l);
    } else if (type == "Sbend") {
      if (std::fabs(angle) < 1.0e-9) {
        e = new MULT(name, l, knl, knsl);
      } else if (std::fabs(angle - knl[0]) > 1.0e-6) {
        e = new GSBEND(name, l, angle, knl[0], e1, e2);
      } else {
        knl[0] = 0.;
        v[10] = 0.;
        if (knl[2] == 0. && knl[1] == 0.)
          e = new SBEND(name, l, angle, e1, e2);
        else
          e = new SBENDMULT(name, l, angle, e1, e2, knl, knsl);
      }
    } else if (type == "RBEND") {
      if (knl[1] == 0. && knl[2] == 0.)
        e = new SBEND(name, l, angle, angle / 2., angle / 2.);
      else
        e = new SBENDMULT(name, l, angle, angle / 2., angle / 2., knl, knsl);
    } else if (type == "Quadrupole") {
      e = new QUAD(name, l, knl[1], knsl[1]);
    } else if (type == "Sextupole") {
      e = new SEXT(name, l, knl[2], knsl[2]);
    } else if (type == "OCTUPOLE") {
      e = new OCT(name, l, knl[3], knsl[3]);
    } else if (type == "HKICKER") {
      e = new HKICKER(name, l, hkick);
    } else if (type == "VKICKER") {
      e = new VKICKER(name, l, vkick);
    } else if (type == "Kicker") {
      e = new KICKER(name, l, hkick, vkick);
    } else if (type == "Multipole") {
      if (knl[0] == 0) {
        e = new MULT(name, l, knl, knsl);
      } else {
        const double a = knl[0];
        knl[0] = 0;
        v[10] = 0.;
        l = 1.0e-6;
        v[1] = l;
        e = new SBEND(name + "_tb", l, a, 0, 0);
      }
    } else if (type == "HMONITOR") {
      e = new HBPM(name, l);
    } else if (type == "VMONITOR") {
      e = new VBPM(name, l);
    } else if (type == "Monitor") {
      e = new BPM(name, l);
    } else if (type == "MARKER") {
      e = new MARKER(name, l);
    } else if (type == "Solenoid") {
      if (l != 0.)
        e = new SOLEN(name, l, ks);
      else
        e = new DRIFT(name, l);
    } else if (type == "RFcavity") {
      e = new RFCAV(name, l, 0.0, 0.0, 0.);
    } else if (type == "BEAMBEAM") {
      if (l != 0.) throw Error(STB_EINVAL, "Beam-Beam element should have zero length!");
      e = new BEAMBEAM(name, 6, 0., 1, 0.4545, 11, 2.5e-06, 2.5e-06, 0.53, 0.0, 0.53, 0.0);
    } else if (type == "ELENS") {
      throw Error(STB_EUNSUPPORTED, "electron lens " + name + " is not implemented on the GPU path");
    } else if (type == "Patch") {
      e = new PATCH(name, xoff, 0.0, zoff, -xpitch);
    } else {
      e = new DRIFT(name, l);
    }
    line.Cell.push_back(e);
  }
  line.Update();
}

}  // namespace stb
