// Turn-by-turn tracking and its diagnostics on the GPU: Track_tbt
// (simtrack.cpp:20841-20860; with a BPM index 20884-20905), Track_tbt_spin
// (20863-20882; with a BPM index 20907-20927), Track_tbt_FMA
// (21179-21241) and Track_tbt_Lyapunov (21243-21306).
//
// A batch of particles is tracked one turn per launch; before every turn the
// coordinates of all particles are copied (device to device) into a record
// rec[(t*ncoord + k)*n + i] (k in x, px, y, py, z, pt order): what Track_tbt
// stores in x_tbt at the start of each turn.  The frequency-map tunes come from the GPU
// FineTuneFinder (stb_fine_tune) over two 1,024-turn windows of the record;
// the Lyapunov indicator needs only the last 25 turns of it.  The BPM form
// records after a given element instead: each one-turn launch runs the
// tracking kernel's per-element probe variant and the element's slice of
// the probe is copied into the record.  The output
// files are written with the reference's stream formatting, including the
// scientific/18-digit state its stream keeps after the first row.
#include <cuda_runtime.h>

#include <cmath>
#include <fstream>
#include <iomanip>
#include <memory>
#include <string>
#include <vector>

#include "simtrack_b200.h"
#include "simtrack_b200.hpp"
#include "stb_runtime.hpp"

namespace stb {

double tune_low = 0.660, tune_high = 0.70;  // simtrack.cpp:27

namespace {

void check(int rc) {
  if (rc != STB_OK) throw Error(rc, stb_last_error());
}

struct DevMem {
  void *p = nullptr;
  explicit DevMem(size_t bytes) { cuda_check(cudaMalloc(&p, bytes ? bytes : 16), "cudaMalloc(turn-by-turn)"); }
  ~DevMem() { cudaFree(p); }
  DevMem(const DevMem &) = delete;
  DevMem &operator=(const DevMem &) = delete;
  template <class T>
  T *as() const { return static_cast<T *>(p); }
};

using TablePtr = std::unique_ptr<stb_table, int (*)(stb_table *)>;

TablePtr make_table(const Line &line, int device) {
  stb_table *raw = nullptr;
  check(stb_table_create(reinterpret_cast<const stb_line *>(&line), device, &raw));
  return TablePtr(raw, stb_table_free);
}

// Particles of one batch on the device, SoA, with Track()'s loss state:
// nc = 6 orbit coordinates, or 9 with the spin vector (Track_Spin's x[9]).
struct DeviceBatch {
  long n;
  int nc;
  DevMem coords, loss;
  DeviceBatch(const double *xa, const int *stable, long n_, int nc_ = 6)
      : n(n_), nc(nc_), coords(sizeof(double) * nc_ * (size_t)n_), loss(sizeof(int32_t) * 2 * (size_t)n_) {
    std::vector<double> soa((size_t)n * nc);
    std::vector<int32_t> l((size_t)n * 2, 0);
    for (long i = 0; i < n; i++) {
      for (int k = 0; k < nc; k++) soa[(size_t)k * n + i] = xa[(size_t)nc * i + k];
      // Track()'s entry check: stable == 0, |x| > 0.1 or |y| > 0.1 -> lost at turn 0, post 0
      l[i] = entry_rejected(xa + (size_t)nc * i, stable[i]) ? 0 : -1;
    }
    cuda_check(cudaMemcpy(coords.p, soa.data(), sizeof(double) * soa.size(), cudaMemcpyHostToDevice),
               "upload coordinates");
    cuda_check(cudaMemcpy(loss.p, l.data(), sizeof(int32_t) * l.size(), cudaMemcpyHostToDevice), "upload loss state");
  }
  double *c(int k) const { return coords.as<double>() + (size_t)k * n; }
  int32_t *lost_turn() const { return loss.as<int32_t>(); }
  int32_t *lost_elem() const { return loss.as<int32_t>() + n; }

  // Final coordinates (AoS) and Track()'s outputs.
  void download(double *xa, int *stable, int *lost_turn_out, int *lost_post) const {
    std::vector<double> soa((size_t)n * nc);
    std::vector<int32_t> l((size_t)n * 2);
    cuda_check(cudaMemcpy(soa.data(), coords.p, sizeof(double) * soa.size(), cudaMemcpyDeviceToHost),
               "download coordinates");
    cuda_check(cudaMemcpy(l.data(), loss.p, sizeof(int32_t) * l.size(), cudaMemcpyDeviceToHost), "download loss");
    for (long i = 0; i < n; i++) {
      if (xa)
        for (int k = 0; k < nc; k++) xa[(size_t)nc * i + k] = soa[(size_t)k * n + i];
      const bool alive = l[i] < 0;
      stable[i] = alive ? 1 : 0;
      lost_turn_out[i] = alive ? 0 : l[i];
      lost_post[i] = alive ? 0 : l[n + i];
    }
  }
};

// nturn one-turn launches (spin tracking for a 9-coordinate batch).  rec
// (device, [nturn - rec_from][ncoord][n]) gets the first ncoord coordinates
// (x, px, y, py, z, pt, sx, sy, sz order) at the start of every turn from
// rec_from on.
void track_recorded(stb_table *t, const DeviceBatch &b, int nturn, int ncoord, double *rec, int rec_from = 0) {
  const long n = b.n;
  const size_t bytes = sizeof(double) * (size_t)n;
  for (int turn = 0; turn < nturn; turn++) {
    if (turn >= rec_from)
      for (int k = 0; k < ncoord; k++)
        cuda_check(cudaMemcpyAsync(rec + ((size_t)(turn - rec_from) * ncoord + k) * n, b.c(k), bytes,
                                   cudaMemcpyDeviceToDevice, 0),
                   "record turn");
    if (b.nc == 9)
      check(stb_track_spin_device(t, b.c(0), b.c(1), b.c(2), b.c(3), b.c(4), b.c(5), b.c(6), b.c(7), b.c(8), n, turn,
                                  1, 0.0, b.lost_turn(), b.lost_elem(), nullptr));
    else
      check(stb_track_device(t, b.c(0), b.c(1), b.c(2), b.c(3), b.c(4), b.c(5), n, turn, 1, 0.0, b.lost_turn(),
                             b.lost_elem(), nullptr));
  }
  cuda_check(cudaDeviceSynchronize(), "turn-by-turn tracking");
}

// Track_tbt / Track_tbt_spin for n particles of nc coordinates (AoS x).
void tbt_batch(Line &line, double *x, long n, int nc, int nturn, double *x_tbt, int *stable, int *lost_turn,
               int *lost_post, int device) {
  if (n < 0 || nturn < 0) throw Error(STB_EINVAL, "negative particle count or turn count");
  if (n == 0) return;
  if (!x || !stable || !lost_turn || !lost_post) throw Error(STB_EINVAL, "NULL host buffer");
  // the entry check returns before anything is recorded
  std::vector<char> rejected((size_t)n);
  for (long i = 0; i < n; i++)
    rejected[i] = std::fabs(x[(size_t)nc * i]) > 0.1 || std::fabs(x[(size_t)nc * i + 2]) > 0.1 || stable[i] == 0;
  DeviceGuard g(device);
  stb_table *raw = nullptr;
  if (nc == 9)
    check(stb_table_create_spin(reinterpret_cast<const stb_line *>(&line), device, &raw));
  else
    check(stb_table_create(reinterpret_cast<const stb_line *>(&line), device, &raw));
  TablePtr t(raw, stb_table_free);
  DeviceBatch b(x, stable, n, nc);
  DevMem rec(sizeof(double) * nc * (size_t)n * (size_t)nturn);
  track_recorded(t.get(), b, nturn, nc, rec.as<double>());
  b.download(x, stable, lost_turn, lost_post);
  if (!x_tbt) return;
  std::vector<double> r((size_t)nc * n * nturn);
  cuda_check(cudaMemcpy(r.data(), rec.p, sizeof(double) * r.size(), cudaMemcpyDeviceToHost), "download record");
  // x_tbt[(i*nturn + turn)*nc + k] for the turns recorded: every turn up to
  // and including the one in which the particle is lost
  for (long i = 0; i < n; i++) {
    const int last = rejected[i] ? 0 : stable[i] ? nturn : lost_turn[i] + 1;
    for (int turn = 0; turn < last; turn++)
      for (int k = 0; k < nc; k++)
        x_tbt[((size_t)i * nturn + turn) * nc + k] = r[((size_t)turn * nc + k) * n + i];
  }
}

// The reference's grid of amplitudes inside a quarter circle of 6 sigma.
struct GridPoint {
  int i, j;
};
std::vector<GridPoint> quarter_disc(int nsigma, double sigma_step) {
  std::vector<GridPoint> g;
  for (int i = 0; i < nsigma; i++)
    for (int j = 0; j < nsigma; j++)
      if (std::sqrt(1.0 * i * i + 1.0 * j * j) <= (6. / sigma_step)) g.push_back({i, j});
  return g;
}

}  // namespace

void Track_tbt_Batch(Line &line, double *x, long n, int nturn, double *x_tbt, int *stable, int *lost_turn,
                     int *lost_post, int device) {
  tbt_batch(line, x, n, 6, nturn, x_tbt, stable, lost_turn, lost_post, device);
}

void Track_tbt_spin_Batch(Line &line, double *x9, long n, int nturn, double *x_tbt9, int *stable, int *lost_turn,
                          int *lost_post, int device) {
  tbt_batch(line, x9, n, 9, nturn, x_tbt9, stable, lost_turn, lost_post, device);
}

void Track_tbt_spin(Line &line, double x[], int nturn, double x_tbt[], int &stable, int &lost_turn, int &lost_post) {
  Track_tbt_spin_Batch(line, x, 1, nturn, x_tbt, &stable, &lost_turn, &lost_post, 0);
}

namespace {

// Track_tbt / Track_tbt_spin with a BPM index for n particles of nc = 6 or 9
// coordinates: one-turn launches of the probe variant, whose record of the
// element is copied out after each turn.
void tbt_bpm_batch(Line &line, double *x, long n, int nc, int nturn, double *x_tbt, int bpm_index, int *stable,
                   int *lost_turn, int *lost_post, int device) {
  if (n < 0 || nturn < 0) throw Error(STB_EINVAL, "negative particle count or turn count");
  if (n == 0) return;
  if (!x || !stable || !lost_turn || !lost_post) throw Error(STB_EINVAL, "NULL host buffer");
  const long nelem = line.Ncell;
  if (nelem < 1) throw Error(STB_EINVAL, "line has no elements");
  // the per-element record of one turn must fit a modest device buffer
  const double dump_bytes = 8.0 * nc * (double)n * (double)nelem;
  if (dump_bytes > 4.0e9)
    throw Error(STB_EINVAL, "particles x elements too large for the element record (over 4 GB per turn)");
  std::vector<char> rejected((size_t)n);
  for (long i = 0; i < n; i++)
    rejected[i] = std::fabs(x[(size_t)nc * i]) > 0.1 || std::fabs(x[(size_t)nc * i + 2]) > 0.1 || stable[i] == 0;
  const bool in_line = bpm_index >= 0 && bpm_index < nelem;
  DeviceGuard g(device);
  stb_table *raw = nullptr;
  if (nc == 9)
    check(stb_table_create_spin(reinterpret_cast<const stb_line *>(&line), device, &raw));
  else
    check(stb_table_create(reinterpret_cast<const stb_line *>(&line), device, &raw));
  TablePtr t(raw, stb_table_free);
  DeviceBatch b(x, stable, n, nc);
  DevMem dump((size_t)dump_bytes);
  DevMem rec(sizeof(double) * nc * (size_t)n * (size_t)nturn);  // [turn][i][nc]
  double *c[9];
  for (int k = 0; k < nc; k++) c[k] = b.c(k);
  const size_t row = (size_t)nc * sizeof(double);
  for (int turn = 0; turn < nturn; turn++) {
    if (nc == 9)
      spin_device_dump(t.get(), c, n, turn, 1, b.lost_turn(), b.lost_elem(), dump.as<double>());
    else
      track_device_dump(t.get(), c, n, turn, 1, b.lost_turn(), b.lost_elem(), dump.as<double>());
    if (in_line)
      cuda_check(cudaMemcpy2DAsync(rec.as<double>() + (size_t)turn * n * nc, row,
                                   dump.as<double>() + (size_t)bpm_index * nc, (size_t)nelem * row, row, (size_t)n,
                                   cudaMemcpyDeviceToDevice, 0),
                 "record element");
  }
  cuda_check(cudaDeviceSynchronize(), "turn-by-turn tracking");
  int st = 0;
  cuda_check(cudaMemcpy(&st, t->d_status, sizeof(int), cudaMemcpyDeviceToHost), "read status");
  if (st != 0) throw Error(st, "tracking kernel reported status " + std::to_string(st));
  b.download(x, stable, lost_turn, lost_post);
  if (!x_tbt || !in_line) return;
  std::vector<double> r((size_t)nc * n * nturn);
  cuda_check(cudaMemcpy(r.data(), rec.p, sizeof(double) * r.size(), cudaMemcpyDeviceToHost), "download record");
  // a turn is recorded when the particle passed the element in it: every turn
  // before its loss, and the turn of the loss if it came at or after the element
  for (long i = 0; i < n; i++) {
    if (rejected[i]) continue;
    int last = nturn;
    if (!stable[i]) last = lost_post[i] >= bpm_index ? lost_turn[i] + 1 : lost_turn[i];
    for (int turn = 0; turn < last; turn++)
      for (int k = 0; k < nc; k++)
        x_tbt[((size_t)i * nturn + turn) * nc + k] = r[((size_t)turn * n + i) * nc + k];
  }
}

}  // namespace

void Track_tbt_bpm_Batch(Line &line, double *x, long n, int nturn, double *x_tbt, int bpm_index, int *stable,
                         int *lost_turn, int *lost_post, int device) {
  tbt_bpm_batch(line, x, n, 6, nturn, x_tbt, bpm_index, stable, lost_turn, lost_post, device);
}

void Track_tbt_spin_bpm_Batch(Line &line, double *x9, long n, int nturn, double *x_tbt9, int bpm_index, int *stable,
                              int *lost_turn, int *lost_post, int device) {
  tbt_bpm_batch(line, x9, n, 9, nturn, x_tbt9, bpm_index, stable, lost_turn, lost_post, device);
}

void Track_tbt_spin(Line &line, double x[], int nturn, double x_tbt[], int &bpm_index, int &stable, int &lost_turn,
                    int &lost_post) {
  Track_tbt_spin_bpm_Batch(line, x, 1, nturn, x_tbt, bpm_index, &stable, &lost_turn, &lost_post, 0);
}

void Track_tbt(Line &line, double x[], int nturn, double x_tbt[], int &bpm_index, int &stable, int &lost_turn,
               int &lost_post) {
  Track_tbt_bpm_Batch(line, x, 1, nturn, x_tbt, bpm_index, &stable, &lost_turn, &lost_post, 0);
}

void Track_tbt(Line &line, double x[], int nturn, double x_tbt[], int &stable, int &lost_turn, int &lost_post) {
  Track_tbt_Batch(line, x, 1, nturn, x_tbt, &stable, &lost_turn, &lost_post, 0);
}

long Track_tbt_FMA(Line &line, double deltap0, double sigmax0, double sigmay0, const char *filename, int device) {
  const int Nturn = 2048, Nfft = 1024;
  const double sigma_step = 0.1;
  const int sigma0 = 0, sigma1 = 6, nsigma = int((sigma1 - sigma0) * 1.0 / sigma_step) + 1;
  if (!filename) throw Error(STB_EINVAL, "NULL file name");
  {
    std::ofstream f(filename);  // the reference empties the file first
    if (!f) throw Error(STB_EINVAL, std::string("cannot open ") + filename);
  }
  Cal_Orbit_Num(line, deltap0, device);
  const double *X = line.Cell[line.Ncell - 1]->X;
  const std::vector<GridPoint> grid = quarter_disc(nsigma, sigma_step);
  const long n = (long)grid.size();
  std::vector<double> x((size_t)n * 6);
  std::vector<int> stable((size_t)n, 1), lt((size_t)n), lp((size_t)n);
  for (long p = 0; p < n; p++) {
    double *q = &x[6 * p];
    q[0] = grid[p].i * sigma_step * sigmax0 + 0.;
    q[1] = 0.;
    q[2] = grid[p].j * sigma_step * sigmay0;
    q[3] = 0.;
    q[4] = 0.;
    q[5] = deltap0;
    q[0] = q[0] + X[0];
    q[1] = q[1] + X[1];
    q[2] = q[2] + X[2];
    q[3] = q[3] + X[3];
    if (q[0] < 1.0e-09) q[0] = q[0] + 1.0e-09;
    if (q[2] < 1.0e-09) q[2] = q[2] + 1.0e-09;
  }
  DeviceGuard g(device);
  TablePtr t = make_table(line, device);
  DeviceBatch b(x.data(), stable.data(), n);
  const int nc = 3;  // x, px, y
  DevMem rec(sizeof(double) * nc * (size_t)n * (size_t)Nturn);
  track_recorded(t.get(), b, Nturn, nc, rec.as<double>());
  b.download(nullptr, stable.data(), lt.data(), lp.data());
  // tunes of x and y over turns [0, 1024) and [1023, 2047), FineTuneFinder's x-only form
  DevMem dt(sizeof(double) * 4 * (size_t)n);
  const double *r = rec.as<double>();
  const struct {
    int coord, first;
  } win[4] = {{0, 0}, {2, 0}, {0, Nfft - 1}, {2, Nfft - 1}};
  for (int w = 0; w < 4; w++)
    check(stb_fine_tune(r + ((size_t)win[w].first * nc + win[w].coord) * n, nullptr, Nfft, n, (long)nc * n, tune_low,
                        tune_high, dt.as<double>() + (size_t)w * n, device, nullptr));
  cuda_check(cudaDeviceSynchronize(), "tune finder");
  std::vector<double> tunes((size_t)4 * n);
  cuda_check(cudaMemcpy(tunes.data(), dt.p, sizeof(double) * tunes.size(), cudaMemcpyDeviceToHost), "download tunes");
  std::ofstream f(filename, std::ios::out | std::ios::app);
  long rows = 0;
  for (long p = 0; p < n; p++) {
    if (stable[p] != 1) continue;
    const double tunex1 = tunes[p], tuney1 = tunes[n + p], tunex2 = tunes[2 * n + p], tuney2 = tunes[3 * n + p];
    f << grid[p].i * sigma_step << " " << grid[p].j * sigma_step << " " << std::setw(25) << std::setprecision(18)
      << std::scientific << tunex1 << " " << std::setw(25) << std::setprecision(18) << std::scientific << tunex2 << " "
      << std::setw(25) << std::setprecision(18) << std::scientific << tuney1 << " " << std::setw(25)
      << std::setprecision(18) << std::scientific << tuney2 << "  " << std::setw(25) << std::setprecision(18)
      << std::scientific << tunex1 - tunex2 << " " << std::setw(25) << std::setprecision(18) << std::scientific
      << tuney1 - tuney2 << std::endl;
    rows++;
  }
  if (!f) throw Error(STB_EINVAL, std::string("cannot write ") + filename);
  return rows;
}

long Track_tbt_Lyapunov(Line &line, double deltap0, double sigmax0, double sigmay0, const char *filename, int device) {
  const int Nturn = 2048, Navg = 25;
  const double sigma_step = 0.05;
  const int sigma0 = 0, sigma1 = 6, nsigma = int((sigma1 - sigma0) * 1.0 / sigma_step);
  const double distance0 = 1.0e-06;
  if (!filename) throw Error(STB_EINVAL, "NULL file name");
  {
    std::ofstream f(filename);
    if (!f) throw Error(STB_EINVAL, std::string("cannot open ") + filename);
  }
  const std::vector<GridPoint> grid = quarter_disc(nsigma, sigma_step);
  const long m = (long)grid.size(), n = 2 * m;  // particle pairs: [0, m) and [m, 2m)
  std::vector<double> x((size_t)n * 6, 0.0);
  std::vector<int> stable((size_t)n, 1), lt((size_t)n), lp((size_t)n);
  for (long p = 0; p < m; p++) {
    double *x1 = &x[6 * p], *x2 = &x[6 * (m + p)];
    x1[0] = grid[p].i * sigma_step * sigmax0;
    x1[2] = grid[p].j * sigma_step * sigmay0;
    x1[5] = deltap0;
    if (x1[0] == 0.) x1[0] = x1[0] + 1.0e-09;
    if (x1[2] == 0.) x1[2] = x1[2] + 1.0e-09;
    x2[0] = x1[0] + 0.707e-06;
    x2[2] = x1[2] + 0.707e-06;
    x2[5] = deltap0;
  }
  DeviceGuard g(device);
  TablePtr t = make_table(line, device);
  DeviceBatch b(x.data(), stable.data(), n);
  const int nc = 4;  // x, px, y, py of the last Navg turns
  DevMem rec(sizeof(double) * nc * (size_t)n * Navg);
  track_recorded(t.get(), b, Nturn, nc, rec.as<double>(), Nturn - Navg);
  b.download(nullptr, stable.data(), lt.data(), lp.data());
  std::vector<double> r((size_t)nc * n * Navg);
  cuda_check(cudaMemcpy(r.data(), rec.p, sizeof(double) * r.size(), cudaMemcpyDeviceToHost), "download record");
  auto at = [&](int turn, int k, long i) { return r[((size_t)(turn - (Nturn - Navg)) * nc + k) * n + i]; };
  std::ofstream f(filename, std::ios::out | std::ios::app);
  long rows = 0;
  for (long p = 0; p < m; p++) {
    if (stable[p] * stable[m + p] != 1) continue;
    // Lay[k] = log(distance[k] / distance0) / (k + 1), averaged over the last 25 turns
    double sum = 0.0;
    for (int k = 0; k < Navg; k++) {
      const int turn = Nturn - 1 - k;
      const double d0 = at(turn, 0, p) - at(turn, 0, m + p), d1 = at(turn, 1, p) - at(turn, 1, m + p);
      const double d2 = at(turn, 2, p) - at(turn, 2, m + p), d3 = at(turn, 3, p) - at(turn, 3, m + p);
      const double distance = std::sqrt(d0 * d0 + d1 * d1 + d2 * d2 + d3 * d3);
      sum = sum + std::log(distance / distance0) / (turn + 1);
    }
    const double LayAvg = sum / 25;
    f << grid[p].i * sigma_step << "  " << grid[p].j * sigma_step << std::setw(25) << std::setprecision(18)
      << std::scientific << LayAvg << std::endl;
    rows++;
  }
  if (!f) throw Error(STB_EINVAL, std::string("cannot write ") + filename);
  return rows;
}

}  // namespace stb
