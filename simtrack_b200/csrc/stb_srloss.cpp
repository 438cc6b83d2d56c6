// Synchrotron-radiation energy loss per turn of the reference particle
// (host side): Cal_SRLoss_U0rad and Cal_SRLoss_U0rad_Track
// (simtrack.cpp:20691-20766), and the general bend's path length and angle
// on an orbit, Cal_gsbend_l_angle (simtrack.cpp:4006-4044).  Every
// expression keeps the reference's operations and their order; the
// transcendentals are the host C library's, as in the reference.
#include <cmath>
#include <string>

#include "simtrack_b200.hpp"
#include "stb_status.hpp"

namespace stb {

namespace {
const double kCrRad = 8.84627632682e-5;     // Cr, simtrack.cpp:25
const double kPIRad = 3.14159265358979323;  // PI, simtrack.cpp:23
}  // namespace

// x: the orbit entering the GSBEND (updated to its exit, as the reference
// does); L, Angle: the frame's; K0L: the real field's.
void Cal_gsbend_l_angle(double x[6], double L, double Angle, double K0L, double &actual_l, double &actual_angle) {
  const double rhoc = L / Angle;
  const double b0 = K0L / L;
  const double cosAngle = std::cos(Angle), sinAngle = std::sin(Angle);
  double x0[6];
  for (int i = 0; i < 6; i++) x0[i] = x[i];
  const double delta = std::sqrt(1.0 + 2 * x[5] / GP.beta + x[5] * x[5]) - 1.0;
  const double gamma = GP.gamma + std::sqrt(GP.gamma * GP.gamma - 1) * x[5];
  const double beta = std::sqrt(1.0 - 1.0 / gamma / gamma);
  const double pz0 = std::sqrt((1. + delta) * (1. + delta) - x0[1] * x0[1] - x0[3] * x0[3]);
  x[1] = x0[1] * cosAngle + (pz0 - b0 * rhoc - b0 * x0[0]) * sinAngle;
  const double pz1 = std::sqrt((1. + delta) * (1. + delta) - x[1] * x[1] - x[3] * x[3]);
  const double derivative = -x0[1] * sinAngle / rhoc + (pz0 - b0 * rhoc - b0 * x0[0]) * cosAngle / rhoc;
  x[0] = pz1 / b0 - derivative * rhoc / b0 - rhoc;
  double temp = std::sqrt((1. + delta) * (1. + delta) - x0[3] * x0[3]);
  const double arcsin1 = std::asin(x0[1] / temp), arcsin2 = std::asin(x[1] / temp);
  x[2] = x0[2] + x0[3] * L / b0 / rhoc + x0[3] * (arcsin1 - arcsin2) / b0;
  temp = (1 + delta) * L / b0 / rhoc + (1 + delta) * (arcsin1 - arcsin2) / b0;
  x[4] = x[4] - (temp / beta - L / GP.beta);
  actual_l = temp;
  actual_angle = K0L * actual_l / L;
}

namespace {

// One bend's share, Cr (E/GeV)^4 href angle / (2 pi).
double bend_loss(double href1, double angle1) {
  return kCrRad * std::pow((GP.energy / 1000.), 4.0) * href1 * (angle1 / 2. / kPIRad);
}

// A bend whose path is taken on the orbit of the element before it; the
// reference reads Cell[i-1] even for i = 0, which is rejected here.
void path_on_orbit(const Line &line, size_t i, double L, double Angle, double K0L, double &l, double &angle) {
  if (i == 0)
    throw Error(STB_EINVAL, "the first element of the line is a bend: the reference would read the orbit "
                            "before element 0");
  double x0[6];
  for (int j = 0; j < 6; j++) x0[j] = line.Cell[i - 1]->X[j];
  Cal_gsbend_l_angle(x0, L, Angle, K0L, l, angle);
}

}  // namespace

// Cal_SRLoss_U0rad (analytic; GSBEND's path on the orbit) and, with
// track_form, Cal_SRLoss_U0rad_Track (the sector bends' path on the orbit
// too).  Sets GP.U0rad (MeV; 0 without GP.radiate) and returns it.
double Cal_SRLoss_U0rad(Line &line, bool track_form) {
  if (!GP.radiate) {
    GP.U0rad = 0.0;
    return GP.U0rad;
  }
  double sum = 0;
  for (size_t i = 0; i < line.Cell.size(); i++) {
    const Element &E = *line.Cell[i];
    if (E.TYPE == "SBEND") {
      const double L = E.L, Angle = E.GetP("ANGLE");
      if (track_form) {
        double l, angle;
        path_on_orbit(line, i, L, Angle, Angle, l, angle);
        sum += bend_loss(angle / l, angle);
      } else {
        sum += bend_loss(Angle / L, Angle);
      }
    } else if (E.TYPE == "GSBEND") {
      double l, angle;
      path_on_orbit(line, i, E.L, E.GetP("ANGLE"), E.GetP("K0L"), l, angle);
      sum += bend_loss(angle / l, angle);
    }
  }
  GP.U0rad = sum * 1000.;
  return GP.U0rad;
}

}  // namespace stb
