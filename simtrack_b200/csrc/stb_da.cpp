// The reference's dynamic-aperture drivers on the GPU, with their output
// files: Track_DA (simtrack.cpp:21389-21441), Track_DA1 (21443-21495),
// Track_DA2 (21497-21533), Track_DA3 (21535-21572), Track_DA_Radial
// (21682-21734), Track_DA_Uniform (21574-21603), Track_DA_Radial_Uniform
// (21736-21764); and Cal_Tunes_Track (20971-21025), Cal_Chrom_Track
// (21027-21051).
//
// The bisection drivers halve the stable amplitude interval [0, sigma_max] of
// each phase angle until it is no longer than 0.1 sigma; every step tracks
// the midpoint (and, in the twin forms, a second particle 0.05 sigma further
// out) with Track() or Track_Radial() and keeps the upper half if all of them
// survive.  A bisection can only visit the midpoints of its binary tree (511
// nodes for sigma_max = 50), so all of them, twins included, are tracked in
// one batched launch and the bisection is then replayed on the outcomes.
// Track() is deterministic and particles are independent, so the replay
// visits the same midpoints, sees the same outcomes and writes the same file
// as the reference.  The uniform drivers sweep 150 amplitudes 1, 1.2, ...
// sigma, all tracked at once; the reference writes one line per amplitude and
// ends the process at the first loss, here the function stops writing there
// and returns.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <memory>
#include <string>
#include <vector>

#include "simtrack_b200.h"
#include "simtrack_b200.hpp"
#include "stb_runtime.hpp"

namespace stb {

namespace {

constexpr double kPi = 3.14159265358979323;  // PI, simtrack.cpp:23

struct Node {
  double sigma;
  int lo, hi;  // child nodes (index into the same vector) after an unstable / stable outcome, -1: leaf
};

// The bisection tree of one angle: node 0 is the first midpoint; every node
// carries the interval the reference would hold when it reaches it.
void build_tree(std::vector<Node> &t, double s, double e) {
  struct Item {
    double s, e;
    int parent;
    bool stable_side;
  };
  std::vector<Item> todo{{s, e, -1, false}};
  while (!todo.empty()) {
    Item it = todo.back();
    todo.pop_back();
    const double sigma = (it.s + it.e) / 2.0;
    const int idx = (int)t.size();
    t.push_back(Node{sigma, -1, -1});
    if (it.parent >= 0) (it.stable_side ? t[it.parent].hi : t[it.parent].lo) = idx;
    // outcome unstable: e = sigma; stable: s = sigma; continue while |e - s| > 0.1
    if (std::fabs(sigma - it.s) > 0.1) todo.push_back({it.s, sigma, idx, false});
    if (std::fabs(it.e - sigma) > 0.1) todo.push_back({sigma, it.e, idx, true});
  }
}

// n particles AoS x[n*6] through Track() or Track_Radial() for nturn turns.
void track_all(Line &line, std::vector<double> &x, int nturn, bool radial, std::vector<int> &stable, int device) {
  const long n = (long)(x.size() / 6);
  stable.assign((size_t)n, 1);
  std::vector<int> lt((size_t)n), lp((size_t)n);
  if (!radial) {
    Track_Batch(line, x.data(), n, nturn, stable.data(), lt.data(), lp.data(), TrackOptions{0.0, device});
    return;
  }
  stb_table *raw = nullptr;
  int rc = stb_table_create(reinterpret_cast<const stb_line *>(&line), device, &raw);
  if (rc != STB_OK) throw Error(rc, stb_last_error());
  std::unique_ptr<stb_table, int (*)(stb_table *)> t(raw, stb_table_free);
  rc = stb_track_radial_host(t.get(), x.data(), n, nturn, 0.0, stable.data(), lt.data(), lp.data());
  if (rc != STB_OK) throw Error(rc, stb_last_error());
}

// Angle i of a driver: (90/11)(i+1) degrees (Track_DA, Track_DA2,
// Track_DA_Radial) or 15(i+1) degrees (Track_DA1, Track_DA3), with the
// reference's expressions for the label and the angle in radians.
struct Angles {
  bool fifteen;
  double label(int i) const { return fifteen ? 15. * (i + 1) : (90 / 11.) * (i + 1); }
  double rad(int i) const { return fifteen ? 15 * (i + 1) * kPi / 180 : (90 / 11.) * (i + 1) * kPi / 180; }
};

struct Bisection {
  int nang;
  Angles angles;
  double sigma_max;
  bool twin;
  bool radial;
};

void bisection_da(Line &line, int nturn, double deltap0, double sigmax0, double sigmay0, const char *filename,
                  const Bisection &B, double *angles_out, double *sigma_out, int device) {
  if (nturn < 0) throw Error(STB_EINVAL, "negative turn count");
  std::vector<Node> tree;
  build_tree(tree, 0., B.sigma_max);
  const int nn = (int)tree.size();
  const int per_node = B.twin ? 2 : 1;
  std::vector<double> x((size_t)B.nang * nn * per_node * 6, 0.0);
  for (int i = 0; i < B.nang; i++) {
    const double angle = B.angles.rad(i);
    for (int k = 0; k < nn; k++)
      for (int twin = 0; twin < per_node; twin++) {
        const double sg = twin == 0 ? tree[k].sigma : tree[k].sigma + 0.05;
        double *p = &x[(((size_t)i * nn + k) * per_node + twin) * 6];
        p[0] = sg * std::cos(angle) * sigmax0;
        p[2] = sg * std::sin(angle) * sigmay0;
        p[5] = deltap0;
      }
  }
  std::vector<int> stable;
  track_all(line, x, nturn, B.radial, stable, device);
  FILE *f = filename ? std::fopen(filename, "w") : nullptr;
  if (filename && !f) throw Error(STB_EINVAL, std::string("cannot open ") + filename);
  for (int i = 0; i < B.nang; i++) {
    // replay: the reference's do { ... } while (|e - s| > 0.1) walks the tree
    int k = 0;
    double sigma = tree[0].sigma;
    while (k >= 0) {
      sigma = tree[k].sigma;
      const size_t b = ((size_t)i * nn + k) * per_node;
      bool st = stable[b] == 1;
      if (B.twin) st = stable[b] * stable[b + 1] == 1;
      k = st ? tree[k].hi : tree[k].lo;
    }
    if (angles_out) angles_out[i] = B.angles.label(i);
    if (sigma_out) sigma_out[i] = sigma;
    if (f) std::fprintf(f, "%f %f \n", B.angles.label(i), sigma);
  }
  if (f) std::fclose(f);
}

long uniform_da(Line &line, int nturn, double deltap0, double angle, double sigmax0, double sigmay0,
                const char *filename, bool radial, double *sigma_out, double *stable_out, int device) {
  if (nturn < 0) throw Error(STB_EINVAL, "negative turn count");
  constexpr int kN = 150;
  std::vector<double> x((size_t)kN * 6, 0.0), sig(kN);
  for (int i = 0; i < kN; i++) {
    sig[i] = 1. + i * 0.2;
    x[6 * i + 0] = sig[i] * std::cos(angle) * sigmax0;
    x[6 * i + 2] = sig[i] * std::sin(angle) * sigmay0;
    x[6 * i + 5] = deltap0;
  }
  std::vector<int> stable;
  track_all(line, x, nturn, radial, stable, device);
  FILE *f = filename ? std::fopen(filename, "w") : nullptr;
  if (filename && !f) throw Error(STB_EINVAL, std::string("cannot open ") + filename);
  long rows = 0;
  for (int i = 0; i < kN; i++) {
    if (f) std::fprintf(f, "%f %f %f \n", angle, sig[i], 1.0 * stable[i]);
    if (sigma_out) sigma_out[rows] = sig[i];
    if (stable_out) stable_out[rows] = 1.0 * stable[i];
    rows++;
    if (stable[i] == 0) break;  // where the reference calls exit(0)
  }
  if (f) std::fclose(f);
  return rows;
}

// FineTuneFinder over the x and y records of one particle's Track_tbt.
bool tbt_tunes(Line &line, double *x, int nturn, int nfft, double &tune1, double &tune2, int device) {
  if (nturn < 0 || nfft > nturn) throw Error(STB_EINVAL, "bad turn count");
  std::vector<double> tbt((size_t)nturn * 6);
  int stable = 1, lt = 0, lp = 0;
  Track_tbt_Batch(line, x, 1, nturn, tbt.data(), &stable, &lt, &lp, device);
  if (stable != 1) return false;
  // signals x and y interleaved: sample k of signal j at [2k + j]
  std::vector<double> xy((size_t)nfft * 2);
  for (int k = 0; k < nfft; k++) {
    xy[2 * (size_t)k] = tbt[(size_t)k * 6 + 0];
    xy[2 * (size_t)k + 1] = tbt[(size_t)k * 6 + 2];
  }
  DeviceGuard g(device);
  double *d = nullptr;
  cuda_check(cudaMalloc(&d, sizeof(double) * (xy.size() + 2)), "cudaMalloc(tune signals)");
  std::unique_ptr<double, cudaError_t (*)(void *)> hold(d, cudaFree);
  cuda_check(cudaMemcpy(d, xy.data(), sizeof(double) * xy.size(), cudaMemcpyHostToDevice), "upload tune signals");
  const int rc = stb_fine_tune(d, nullptr, nfft, 2, 2, tune_low, tune_high, d + xy.size(), device, nullptr);
  if (rc != STB_OK) throw Error(rc, stb_last_error());
  double t[2];
  cuda_check(cudaMemcpy(t, d + xy.size(), sizeof(t), cudaMemcpyDeviceToHost), "download tunes");
  tune1 = t[0];
  tune2 = t[1];
  return true;
}

}  // namespace

void Track_DA(Line &line, int nturn, double deltap0, double sigmax0, double sigmay0, const char *filename,
              double *angles_out, double *sigma_out, int device) {
  bisection_da(line, nturn, deltap0, sigmax0, sigmay0, filename, Bisection{10, Angles{false}, 50.0, true, false},
               angles_out, sigma_out, device);
}

void Track_DA1(Line &line, int nturn, double deltap0, double sigmax0, double sigmay0, const char *filename,
               double *angles_out, double *sigma_out, int device) {
  bisection_da(line, nturn, deltap0, sigmax0, sigmay0, filename, Bisection{5, Angles{true}, 50.0, true, false},
               angles_out, sigma_out, device);
}

void Track_DA2(Line &line, int nturn, double deltap0, double sigmax0, double sigmay0, const char *filename,
               double *angles_out, double *sigma_out, int device) {
  bisection_da(line, nturn, deltap0, sigmax0, sigmay0, filename, Bisection{10, Angles{false}, 50.0, false, false},
               angles_out, sigma_out, device);
}

void Track_DA3(Line &line, int nturn, double deltap0, double sigmax0, double sigmay0, const char *filename,
               double *angles_out, double *sigma_out, int device) {
  Cal_Orbit_Num(line, 0, device);  // as the reference (the orbit only fills the elements' X)
  bisection_da(line, nturn, deltap0, sigmax0, sigmay0, filename, Bisection{5, Angles{true}, 30.0, false, false},
               angles_out, sigma_out, device);
}

void Track_DA_Radial(Line &line, int nturn, double deltap0, double sigmax0, double sigmay0, const char *filename,
                     double *angles_out, double *sigma_out, int device) {
  bisection_da(line, nturn, deltap0, sigmax0, sigmay0, filename, Bisection{10, Angles{false}, 15.0, true, true},
               angles_out, sigma_out, device);
}

long Track_DA_Uniform(Line &line, int nturn, double deltap0, double angle, double sigmax0, double sigmay0,
                      const char *filename, double *sigma_out, double *stable_out, int device) {
  return uniform_da(line, nturn, deltap0, angle, sigmax0, sigmay0, filename, false, sigma_out, stable_out, device);
}

long Track_DA_Radial_Uniform(Line &line, int nturn, double deltap0, double angle, double sigmax0, double sigmay0,
                             const char *filename, double *sigma_out, double *stable_out, int device) {
  return uniform_da(line, nturn, deltap0, angle, sigmax0, sigmay0, filename, true, sigma_out, stable_out, device);
}

void Cal_Tunes_Track(Line &line, double x[], int Nturn, double &tune1, double &tune2, int device) {
  if (x[0] < 1.0e-9) x[0] = x[0] + 1.0e-9;
  if (x[2] < 1.0e-9) x[2] = x[2] + 1.0e-9;
  tbt_tunes(line, x, Nturn, Nturn, tune1, tune2, device);
}

void Cal_Tunes_Track(Line &line, double deltap0, int device) {
  const int Nturn = 1024;
  Cal_Orbit_Num(line, deltap0, device);
  const double *X = line.Cell[line.Ncell - 1]->X;
  double x[6] = {X[0], X[1], X[2], X[3], 0., deltap0};
  if (x[0] < 1.0e-9) x[0] = x[0] + 1.0e-9;
  if (x[2] < 1.0e-9) x[2] = x[2] + 1.0e-9;
  double t1 = 0., t2 = 0.;  // the reference leaves them undefined for an unstable particle
  tbt_tunes(line, x, Nturn, 1024, t1, t2, device);
  line.Tune1 = t1;
  line.Tune2 = t2;
}

void Cal_Chrom_Track(Line &line, int device) {
  Cal_Tunes_Track(line, 0.0003, device);
  const double qxp = line.Tune1, qyp = line.Tune2;
  Cal_Tunes_Track(line, -0.0003, device);
  const double qxm = line.Tune1, qym = line.Tune2;
  Cal_Tunes_Track(line, 0.00, device);
  const double qx0 = line.Tune1, qy0 = line.Tune2;
  line.Chromx1 = (qxp - qxm) / 2. / 0.0003;
  line.Chromy1 = (qyp - qym) / 2. / 0.0003;
  line.Chromx2 = (qxp + qxm - 2 * qx0) / 2. / 0.0003 / 0.0003;
  line.Chromy2 = (qyp + qym - 2 * qy0) / 2. / 0.0003 / 0.0003;
}

}  // namespace stb
