// Reference oracle harness.  TEST INFRASTRUCTURE ONLY.
//
// Compiled together with the unmodified SimTrack source (simtrack.cpp) into
// oracle/_ref/libsimtrack_ref.so by oracle/Makefile.  It exposes a C ABI that
// pytest loads through ctypes to build a Line with the reference's own element
// constructors (simtrack.h:399-1059) and to run the reference's own tracking
// entry points:
//   ref_track       -> Track()       simtrack.cpp:20791-20814 (called as is)
//   ref_track_spin  -> Track_Spin()  simtrack.cpp:21766-21789 (called as is)
//   ref_track_radial -> Track_Radial()  simtrack.cpp:21641-21680 (called as is)
//   ref_track_spin_dump -> the Track_Spin() loop recording x[9] after every
//                      element.
//   ref_track_circ  -> the Track() loop with one extra loss predicate, a
//                      circular aperture x^2+y^2 > R^2, evaluated after the
//                      reference's own rectangular/NaN check.
//   ref_track_dump  -> the Track() loop that also records all six
//                      coordinates after every element (the per-element
//                      parity probe).
//   ref_set_radiation -> GP.radiate, with the deviates radiate1 draws from
//                      GSL supplied by the stream below.
// Nothing in the product links or loads this file.
#include "simtrack.h"

#include <cstdio>
#include <cstring>
#include <vector>
#include <cmath>
#include <cstdint>

extern GlobalVariables GP;
extern double tune_low, tune_high;

namespace {

void copy11(const double *src, double *dst) {
  for (int i = 0; i < 11; i++) dst[i] = src[i];
}

Element *make_element(const char *type, const char *name, const double *p, int np) {
  std::string nm(name ? name : "");
  std::string t(type);
  auto need = [&](int k) { return np >= k; };
  if (t == "DRIFT" && need(1)) return new DRIFT(nm, p[0]);
  if (t == "MARKER" && need(1)) return new MARKER(nm, p[0]);
  if (t == "BPM" && need(1)) return new BPM(nm, p[0]);
  if (t == "HBPM" && need(1)) return new HBPM(nm, p[0]);
  if (t == "VBPM" && need(1)) return new VBPM(nm, p[0]);
  if (t == "SBEND" && need(4)) return new SBEND(nm, p[0], p[1], p[2], p[3]);
  if (t == "GSBEND" && need(5)) return new GSBEND(nm, p[0], p[1], p[2], p[3], p[4]);
  if (t == "QUAD" && need(3)) return new QUAD(nm, p[0], p[1], p[2]);
  if (t == "SKEWQ" && need(2)) return new SKEWQ(nm, p[0], p[1]);
  if (t == "SEXT" && need(3)) return new SEXT(nm, p[0], p[1], p[2]);
  if (t == "OCT" && need(3)) return new OCT(nm, p[0], p[1], p[2]);
  if (t == "MULT" && need(23)) {
    double knl[11], knsl[11];
    copy11(p + 1, knl);
    copy11(p + 12, knsl);
    return new MULT(nm, p[0], knl, knsl);
  }
  if ((t == "GMULT" || t == "SBENDMULT") && need(26)) {
    double knl[11], knsl[11];
    copy11(p + 4, knl);
    copy11(p + 15, knsl);
    if (t == "GMULT") return new GMULT(nm, p[0], p[1], p[2], p[3], knl, knsl);
    return new SBENDMULT(nm, p[0], p[1], p[2], p[3], knl, knsl);
  }
  if (t == "KICKER" && need(3)) return new KICKER(nm, p[0], p[1], p[2]);
  if (t == "HKICKER" && need(2)) return new HKICKER(nm, p[0], p[1]);
  if (t == "VKICKER" && need(2)) return new VKICKER(nm, p[0], p[1]);
  if (t == "SOLEN" && need(2)) return new SOLEN(nm, p[0], p[1]);
  if (t == "PATCH" && need(4)) return new PATCH(nm, p[0], p[1], p[2], p[3]);
  if (t == "RFCAV" && need(4)) return new RFCAV(nm, p[0], p[1], p[2], p[3]);
  if (t == "CRABRF" && need(4)) return new CRABRF(nm, p[0], p[1], p[2], p[3]);
  if (t == "CCMULT" && need(12))
    return new CCMULT(nm, p[0], p[1], p[2], p[3], p[4], p[5], p[6], p[7], p[8], p[9], p[10], p[11]);
  if (t == "LBT" && need(1)) return new LBT(nm, p[0]);
  if (t == "ILBT" && need(1)) return new ILBT(nm, p[0]);
  if (t == "BEAMBEAM" && need(11))
    return new BEAMBEAM(nm, int(p[0]), p[1], p[2], p[3], int(p[4]), p[5], p[6], p[7], p[8], p[9], p[10]);
  return nullptr;
}

inline bool circ_lost(const double *x, double r2) {
  return r2 > 0.0 && x[0] * x[0] + x[2] * x[2] > r2;
}

// Normal deviates for the reference's radiate1 (gsl_ran_gaussian, reached
// through the GSL shim).  GSL is absent, so the stream is the tracker's
// definition, restated here independently: the k-th deviate of particle id
// under seed is Philox4x32-10 (Salmon et al., SC'11; counter (k, id), key
// seed) -> two 53-bit uniforms in (0, 1] -> Box-Muller with a natural log
// made of basic operations (ln m = 2 atanh((m-1)/(m+1)), series through the
// 23rd power) and the library cos (correctly rounded in libsimtrack_ref_cr).
// k counts the particle's calls from the start of its tracking.
unsigned long long g_rng_seed = 1324;
long g_rng_base = 0, g_rng_id = 0;
unsigned long long g_rng_k = 0;

void rng_particle(long id) {
  g_rng_id = id;
  g_rng_k = 0;
}

void philox10(uint32_t ctr[4], uint32_t key0, uint32_t key1) {
  for (int round = 0; round < 10; round++) {
    if (round) {
      key0 += 0x9E3779B9u;
      key1 += 0xBB67AE85u;
    }
    const uint64_t m0 = (uint64_t)ctr[0] * 0xD2511F53u;
    const uint64_t m1 = (uint64_t)ctr[2] * 0xCD9E8D57u;
    const uint32_t n0 = (uint32_t)(m1 >> 32) ^ ctr[1] ^ key0;
    const uint32_t n2 = (uint32_t)(m0 >> 32) ^ ctr[3] ^ key1;
    ctr[0] = n0;
    ctr[1] = (uint32_t)m1;
    ctr[2] = n2;
    ctr[3] = (uint32_t)m0;
  }
}

double series_log(double x) {
  uint64_t bits;
  std::memcpy(&bits, &x, 8);
  int ex = (int)((bits >> 52) & 0x7ff) - 1023;
  bits = (bits & 0x000fffffffffffffull) | 0x3ff0000000000000ull;
  double m;
  std::memcpy(&m, &bits, 8);
  if (m > 1.4142135623730951) {
    m = m * 0.5;
    ex = ex + 1;
  }
  const double s = (m - 1.0) / (m + 1.0);
  const double s2 = s * s;
  double acc = 1.0 / 23.0;
  for (int odd = 21; odd >= 3; odd -= 2) acc = acc * s2 + 1.0 / (double)odd;
  const double lnm = 2.0 * s + 2.0 * s * (s2 * acc);
  return (double)ex * 0.6931471805599453094 + ((double)ex * 2.319046813846299558e-17 + lnm);
}

double stream_gaussian(unsigned long long seed, unsigned long long id, unsigned long long k) {
  uint32_t c[4] = {(uint32_t)k, (uint32_t)(k >> 32), (uint32_t)id, (uint32_t)(id >> 32)};
  philox10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
  const uint64_t w1 = ((uint64_t)c[0] << 32) | c[1], w2 = ((uint64_t)c[2] << 32) | c[3];
  const double u1 = (double)((w1 >> 11) + 1) * (1.0 / 9007199254740992.0);
  const double u2 = (double)((w2 >> 11) + 1) * (1.0 / 9007199254740992.0);
  return std::sqrt(-2.0 * series_log(u1)) * std::cos(6.283185307179586 * u2);
}

// radiate2's photon draws: for the particle's k-th radiating slice, draw 0
// gives the photon count (Poisson by inversion from exp(-mu), at most 1000)
// and draws 1, 2, ... the photons' uniforms; Philox counter (k, 2^31 | j,
// id), key seed.
unsigned long long g_photon_k = 0;
uint32_t g_photon_j = 0;

double stream_uniform(unsigned long long seed, unsigned long long id, unsigned long long k, uint32_t j) {
  uint32_t c[4] = {(uint32_t)k, 0x80000000u | j, (uint32_t)id, (uint32_t)(id >> 32)};
  philox10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
  const uint64_t w = ((uint64_t)c[0] << 32) | c[1];
  return (double)((w >> 11) + 1) * (1.0 / 9007199254740992.0);
}

}  // namespace

extern "C" double ref_rng_gaussian(void) { return stream_gaussian(g_rng_seed, (unsigned long long)g_rng_id, g_rng_k++); }

extern "C" unsigned int ref_rng_poisson(double mu) {
  g_photon_k = g_rng_k++;
  g_photon_j = 0;
  const double u = stream_uniform(g_rng_seed, (unsigned long long)g_rng_id, g_photon_k, 0);
  double term = std::exp(-mu), cdf = term;
  unsigned int count = 0;
  while (u > cdf && count < 1000) {
    count = count + 1;
    term = term * mu / (double)count;
    cdf = cdf + term;
  }
  return count;
}

extern "C" double ref_rng_uniform(void) {
  return stream_uniform(g_rng_seed, (unsigned long long)g_rng_id, g_photon_k, ++g_photon_j);
}

extern "C" {

void ref_set_ref_energy(double gamma, double E0, double Q, double A) {
  Set_RefPartEnergy(gamma, E0, Q, A);
}

void ref_set_spin_g(double g) { Set_Spin_G(g); }

void ref_set_flags(int h_expand, int quad_fringe) {
  GP.H_expand = h_expand != 0;
  GP.quad_fringe = quad_fringe != 0;
  GP.radiate = false;
}

// GP.radiate and the seed of the deviate stream (ref_set_flags clears
// GP.radiate).  Particle i of a ref_track / ref_track_circ call, and the one
// particle of ref_track_dump, draws as stream id base + i.
void ref_set_radiation(int radiate, unsigned long long seed) {
  GP.radiate = radiate != 0;
  g_rng_seed = seed;
}
void ref_rng_id_base(long base) { g_rng_base = base; }

// Cal_SRLoss_U0rad / Cal_SRLoss_U0rad_Track, called as is; returns GP.U0rad.
double ref_cal_srloss(void *line, int track_form) {
  if (track_form) Cal_SRLoss_U0rad_Track(*static_cast<Line *>(line));
  else Cal_SRLoss_U0rad(*static_cast<Line *>(line));
  return GP.U0rad;
}
// The reference's Cal_SRLoss_Particle (simtrack.cpp:20768), the pass drawing
// from particle g_rng_base's stream; x6 updated in place.
double ref_cal_srloss_particle(void *line, double *x6) {
  double loss = 0;
  rng_particle(g_rng_base);
  Cal_SRLoss_Particle(*static_cast<Line *>(line), x6, loss);
  return loss;
}
// Deviate k of stream `id` under `seed` (the stream's own check).
double ref_rng_stream(unsigned long long seed, unsigned long long id, unsigned long long k) {
  return stream_gaussian(seed, id, k);
}

// gamma, beta, energy, brho, Q, energy0, G
void ref_get_gp(double *out) {
  out[0] = GP.gamma;
  out[1] = GP.beta;
  out[2] = GP.energy;
  out[3] = GP.brho;
  out[4] = GP.Q;
  out[5] = GP.energy0;
  out[6] = GP.G;
}

void *ref_line_new(void) { return new Line(); }
void ref_line_free(void *line) { delete static_cast<Line *>(line); }
long ref_line_ncell(void *line) { return static_cast<Line *>(line)->Ncell; }
double ref_line_length(void *line) { return static_cast<Line *>(line)->Length; }

int ref_line_append(void *line, const char *type, const char *name, const double *p, int np) {
  Element *e = make_element(type, name, p, np);
  if (!e) return -1;
  static_cast<Line *>(line)->Append(e);
  return 0;
}

void ref_line_setp(void *line, long idx, const char *pname, double v) {
  static_cast<Line *>(line)->Cell[idx]->SetP(pname, v);
}

double ref_line_getp(void *line, long idx, const char *pname) {
  return static_cast<Line *>(line)->Cell[idx]->GetP(pname);
}

void ref_line_set_misalign(void *line, long idx, double dx, double dy, double ds, double dtheta,
                           double dphi, double dpsi) {
  Element *e = static_cast<Line *>(line)->Cell[idx];
  e->DX = dx; e->DY = dy; e->DS = ds;
  e->DTHETA = dtheta; e->DPHI = dphi; e->DPSI = dpsi;
}

void ref_line_set_aperture(void *line, long idx, double apx, double apy) {
  Element *e = static_cast<Line *>(line)->Cell[idx];
  e->APx = apx;
  e->APy = apy;
}

void ref_pass(void *line, long idx, double *x) { static_cast<Line *>(line)->Cell[idx]->Pass(x); }

// Read_MADX_Lattice (simtrack.cpp:13591) into a new Line.  The reference
// exits the process on a missing file: callers check the path first.
void *ref_line_read_madx(const char *path) {
  Line *l = new Line();
  Read_MADX_Lattice(*l, path);
  return l;
}

// Track_tbt (simtrack.cpp:20841), the overload without a BPM index.
void ref_track_tbt(void *line, double *x, int nturn, double *x_tbt, int *stable, int *lost_turn, int *lost_post) {
  Track_tbt(*static_cast<Line *>(line), x, nturn, x_tbt, *stable, *lost_turn, *lost_post);
}

// Cal_dz0_OnMomentumPart / Track_wrt_OnMomentumPart (simtrack.cpp:20929, 20942).
void ref_cal_dz0(void *line, double *x0, double *dz0) {
  Cal_dz0_OnMomentumPart(*static_cast<Line *>(line), x0, dz0);
}
void ref_track_wrt_onmom(void *line, double *x, long n, double *dz0, int nturn, int *stable, int *lost_turn,
                         int *lost_post) {
  Line &l = *static_cast<Line *>(line);
  for (long i = 0; i < n; i++) {
    int st = 1, lt = 0, lp = 0;
    Track_wrt_OnMomentumPart(l, x + 6 * i, dz0, nturn, st, lt, lp);
    stable[i] = st;
    lost_turn[i] = lt;
    lost_post[i] = lp;
  }
}

// Track_tbt with a BPM index (simtrack.cpp:20884).
void ref_track_tbt_bpm(void *line, double *x, int nturn, double *x_tbt, int bpm_index, int *stable, int *lost_turn,
                       int *lost_post) {
  Track_tbt(*static_cast<Line *>(line), x, nturn, x_tbt, bpm_index, *stable, *lost_turn, *lost_post);
}

// Track_tbt_spin with a BPM index (simtrack.cpp:20907).
void ref_track_tbt_spin_bpm(void *line, double *x9, int nturn, double *x_tbt9, int bpm_index, int *stable,
                            int *lost_turn, int *lost_post) {
  Track_tbt_spin(*static_cast<Line *>(line), x9, nturn, x_tbt9, bpm_index, *stable, *lost_turn, *lost_post);
}

// Track_tbt_spin (simtrack.cpp:20863), the overload without a BPM index.
void ref_track_tbt_spin(void *line, double *x9, int nturn, double *x_tbt9, int *stable, int *lost_turn,
                        int *lost_post) {
  Track_tbt_spin(*static_cast<Line *>(line), x9, nturn, x_tbt9, *stable, *lost_turn, *lost_post);
}

// Track_tbt_FMA / Track_tbt_Lyapunov (simtrack.cpp:21179, 21243): write
// ./FMA-output.dat / ./Lmap-output.dat in the current directory.
void ref_track_tbt_fma(void *line, double deltap0, double sigmax0, double sigmay0, double lo, double hi) {
  tune_low = lo;
  tune_high = hi;
  Track_tbt_FMA(*static_cast<Line *>(line), deltap0, sigmax0, sigmay0);
}
void ref_track_tbt_lyapunov(void *line, double deltap0, double sigmax0, double sigmay0) {
  Track_tbt_Lyapunov(*static_cast<Line *>(line), deltap0, sigmax0, sigmay0);
}

// Read_BMAD_Lattice (simtrack.cpp:14054) into a new Line.  The reference
// turns a row whose S column is not a number into a drift of an
// uninitialised length, so callers pass a table without such rows.
void *ref_line_read_bmad(const char *path) {
  Line *l = new Line();
  Read_BMAD_Lattice(*l, path);
  return l;
}

// TYPE, NAME and the public geometry fields of element idx.
void ref_line_elem(void *line, long idx, char *type, char *name, int cap, double *geom10) {
  Element *e = static_cast<Line *>(line)->Cell[idx];
  std::snprintf(type, (size_t)cap, "%s", e->TYPE.c_str());
  std::snprintf(name, (size_t)cap, "%s", e->NAME.c_str());
  const double v[10] = {e->L, e->S, e->DX, e->DY, e->DS, e->DTHETA, e->DPHI, e->DPSI, e->APx, e->APy};
  for (int k = 0; k < 10; k++) geom10[k] = v[k];
}

// n particles, AoS x[n*6], through the reference Track(); stable[] is read as
// the caller's input flag (Track's own convention) and overwritten.
void ref_track(void *line, double *x, long n, int nturn, int *stable, int *lost_turn, int *lost_post) {
  Line &l = *static_cast<Line *>(line);
  for (long i = 0; i < n; i++) {
    int st = stable[i], lt = 0, lp = 0;
    rng_particle(g_rng_base + i);
    Track(l, x + 6 * i, nturn, st, lt, lp);
    stable[i] = st; lost_turn[i] = lt; lost_post[i] = lp;
  }
}

// The reference's Cal_Orbit_Num (simtrack.cpp:14947) and the orbit it stores
// in every element's X[] (orbit6[j*6 + k]).
void ref_cal_orbit(void *line, double deltap, double *orbit6) {
  Line &l = *static_cast<Line *>(line);
  Cal_Orbit_Num(l, deltap);
  for (long j = 0; j < l.Ncell; j++)
    for (int k = 0; k < 6; k++) orbit6[j * 6 + k] = l.Cell[j]->X[k];
}

// The reference's Track_DA (simtrack.cpp:21389-21441), writing `filename`.
void ref_track_da(void *line, int nturn, double deltap0, double sigmax0, double sigmay0, const char *filename) {
  Track_DA(*static_cast<Line *>(line), nturn, deltap0, sigmax0, sigmay0, filename);
}

// The reference's other bisection drivers: 1 Track_DA1, 2 Track_DA2,
// 3 Track_DA3, 4 Track_DA_Radial (simtrack.cpp:21443, 21497, 21535, 21682).
// The uniform sweeps are not wrapped: they end the process at the first loss.
void ref_track_da_driver(void *line, int which, int nturn, double deltap0, double sigmax0, double sigmay0,
                         const char *filename) {
  Line &l = *static_cast<Line *>(line);
  if (which == 1) Track_DA1(l, nturn, deltap0, sigmax0, sigmay0, filename);
  if (which == 2) Track_DA2(l, nturn, deltap0, sigmax0, sigmay0, filename);
  if (which == 3) Track_DA3(l, nturn, deltap0, sigmax0, sigmay0, filename);
  if (which == 4) Track_DA_Radial(l, nturn, deltap0, sigmax0, sigmay0, filename);
}

// n particles through the reference Track_Radial() (simtrack.cpp:21641-21680).
void ref_track_radial(void *line, double *x, long n, int nturn, int *stable, int *lost_turn, int *lost_post) {
  Line &l = *static_cast<Line *>(line);
  for (long i = 0; i < n; i++) {
    int st = stable[i], lt = 0, lp = 0;
    Track_Radial(l, x + 6 * i, nturn, st, lt, lp);
    stable[i] = st; lost_turn[i] = lt; lost_post[i] = lp;
  }
}

void ref_track_spin(void *line, double *x9, long n, int nturn, int *stable, int *lost_turn,
                    int *lost_post) {
  Line &l = *static_cast<Line *>(line);
  for (long i = 0; i < n; i++) {
    int st = stable[i], lt = 0, lp = 0;
    Track_Spin(l, x9 + 9 * i, nturn, st, lt, lp);
    stable[i] = st; lost_turn[i] = lt; lost_post[i] = lp;
  }
}

// One particle through the Track_Spin() loop (simtrack.cpp:21766-21789) with
// dump[(turn*ncell + j)*9 + k] = x[k] after element j of turn (the
// per-element probe of the spin path; entries after a loss are untouched).
void ref_track_spin_dump(void *line, double *x9, int nturn, double *dump, int *stable, int *lost_turn,
                         int *lost_post) {
  Line &l = *static_cast<Line *>(line);
  *stable = 1; *lost_turn = 0; *lost_post = 0;
  if (std::abs(x9[0]) > 0.1 || std::abs(x9[2]) > 0.1) { *stable = 0; return; }
  for (GP.turn = 0; GP.turn < nturn; GP.turn++) {
    for (long j = 0; j < l.Ncell; j++) {
      l.Cell[j]->sPass(x9);
      std::memcpy(dump + ((long)GP.turn * l.Ncell + j) * 9, x9, 9 * sizeof(double));
      if (std::abs(x9[0]) > l.Cell[j]->APx || std::abs(x9[2]) > l.Cell[j]->APy || std::isnan(x9[0]) ||
          std::isnan(x9[2])) {
        *stable = 0; *lost_turn = GP.turn; *lost_post = (int)j;
        return;
      }
    }
  }
}

// Track() loop plus a circular aperture of radius R (R <= 0 disables it).
void ref_track_circ(void *line, double *x, long n, int nturn, double radius, int *stable,
                    int *lost_turn, int *lost_post) {
  Line &l = *static_cast<Line *>(line);
  const double r2 = radius > 0.0 ? radius * radius : 0.0;
  for (long i = 0; i < n; i++) {
    double *xi = x + 6 * i;
    stable[i] = 1; lost_turn[i] = 0; lost_post[i] = 0;
    rng_particle(g_rng_base + i);
    if (std::abs(xi[0]) > 0.1 || std::abs(xi[2]) > 0.1) { stable[i] = 0; continue; }
    bool lost = false;
    for (GP.turn = 0; GP.turn < nturn && !lost; GP.turn++) {
      for (long j = 0; j < l.Ncell; j++) {
        l.Cell[j]->Pass(xi);
        if (std::abs(xi[0]) > l.Cell[j]->APx || std::abs(xi[2]) > l.Cell[j]->APy ||
            std::isnan(xi[0]) || std::isnan(xi[2]) || circ_lost(xi, r2)) {
          stable[i] = 0; lost_turn[i] = GP.turn; lost_post[i] = (int)j; lost = true;
          break;
        }
      }
    }
  }
}

// One particle; dump[(turn*ncell + j)*6 + k] = x[k] after element j of turn.
// Entries after a loss are left untouched.
void ref_track_dump(void *line, double *x, int nturn, double radius, double *dump, int *stable,
                    int *lost_turn, int *lost_post) {
  Line &l = *static_cast<Line *>(line);
  const double r2 = radius > 0.0 ? radius * radius : 0.0;
  *stable = 1; *lost_turn = 0; *lost_post = 0;
  rng_particle(g_rng_base);
  if (std::abs(x[0]) > 0.1 || std::abs(x[2]) > 0.1) { *stable = 0; return; }
  for (GP.turn = 0; GP.turn < nturn; GP.turn++) {
    for (long j = 0; j < l.Ncell; j++) {
      l.Cell[j]->Pass(x);
      std::memcpy(dump + ((long)GP.turn * l.Ncell + j) * 6, x, 6 * sizeof(double));
      if (std::abs(x[0]) > l.Cell[j]->APx || std::abs(x[2]) > l.Cell[j]->APy || std::isnan(x[0]) ||
          std::isnan(x[2]) || circ_lost(x, r2)) {
        *stable = 0; *lost_turn = GP.turn; *lost_post = (int)j;
        return;
      }
    }
  }
}

double ref_pinv(double p) { return gsl_cdf_ugaussian_Pinv(p); }

// The reference's sliced 6D soft-Gaussian collision, called as is (it also
// writes ./bunch1_Z.dat and ./bunch2_Z.dat in the working directory).
void ref_bb6d_soft_gaussian(double Np1, int Mp1, double *x1, double Np2, int Mp2, double *x2, double gamma1,
                            double gamma2, double bbscale1, double bbscale2, int ns1, int ns2) {
  BeamBeam6D_SoftGaussian(Np1, Mp1, x1, Np2, Mp2, x2, gamma1, gamma2, bbscale1, bbscale2, ns1, ns2);
}

// Its overload with slice boundaries zb1, zb2, called as is.
void ref_bb6d_soft_gaussian_zb(double Np1, int Mp1, double *x1, double Np2, int Mp2, double *x2, double gamma1,
                               double gamma2, double bbscale1, double bbscale2, int ns1, int ns2, double *zb1,
                               double *zb2) {
  BeamBeam6D_SoftGaussian(Np1, Mp1, x1, Np2, Mp2, x2, gamma1, gamma2, bbscale1, bbscale2, ns1, ns2, zb1, zb2);
}

// The reference's strong-strong soft-Gaussian collision, called as is.
void ref_bb4d_soft_gaussian(double Np1, int n1, double *x1, double Np2, int n2, double *x2, double gamma1,
                            double gamma2, double bbscale1, double bbscale2) {
  BeamBeam4D_SoftGaussian(Np1, n1, x1, Np2, n2, x2, gamma1, gamma2, bbscale1, bbscale2);
}

// BeamBeam4D_PIC (simtrack.cpp:23286).
void ref_bb4d_pic(double Np1, int n1, double *x1, double Np2, int n2, double *x2, double gamma1, double gamma2,
                  double bbscale1, double bbscale2) {
  BeamBeam4D_PIC(Np1, n1, x1, Np2, n2, x2, gamma1, gamma2, bbscale1, bbscale2);
}

// Cal_Effective_Green_Function (simtrack.cpp:2881) and
// BeamBeam4D_PIC_NonOffset (simtrack.cpp:24226).
void ref_green_function(double xoffset, double yoffset, int nx, int ny, double hx, double hy, double *gr, double *gi) {
  Cal_Effective_Green_Function(xoffset, yoffset, nx, ny, hx, hy, gr, gi);
}
void ref_bb4d_pic_nonoffset(double Np1, int n1, double *x1, double Np2, int n2, double *x2, double gamma1,
                            double gamma2, double bbscale1, double bbscale2, int nx, int ny, double hx, double hy,
                            double *gr, double *gi) {
  BeamBeam4D_PIC_NonOffset(Np1, n1, x1, Np2, n2, x2, gamma1, gamma2, bbscale1, bbscale2, nx, ny, hx, hy, gr, gi);
}

// BeamBeam6D_PIC (simtrack.cpp:23380); it writes bunch and slice files
// into the working directory.
void ref_bb6d_pic(double Np1, int n1, double *x1, double Np2, int n2, double *x2, double gamma1, double gamma2,
                  double bbscale1, double bbscale2, int ns1, int ns2) {
  BeamBeam6D_PIC(Np1, n1, x1, Np2, n2, x2, gamma1, gamma2, bbscale1, bbscale2, ns1, ns2);
}

// BeamBeam6D_PIC_NonOffset (simtrack.cpp:24282).
void ref_bb6d_pic_nonoffset(double Np1, int n1, double *x1, double Np2, int n2, double *x2, double gamma1,
                            double gamma2, double bbscale1, double bbscale2, int ns1, int ns2, double *zb1,
                            double *zb2, int nx, int ny, double hx, double hy, double *gr, double *gi) {
  BeamBeam6D_PIC_NonOffset(Np1, n1, x1, Np2, n2, x2, gamma1, gamma2, bbscale1, bbscale2, ns1, ns2, zb1, zb2, nx, ny,
                           hx, hy, gr, gi);
}

// Lumi_Cal_PIC_6D_Angle (simtrack.cpp:23946); it writes bunch, slice and
// collision-order files into the working directory.
double ref_lumi_pic_6d_angle(double Np1, int n1, double Np2, int n2, double theta, int ns1, int ns2, double *x1,
                             double *x2, double gamma1, double gamma2, double bbscale1, double bbscale2, int ncoll,
                             double freq) {
  return Lumi_Cal_PIC_6D_Angle(Np1, n1, Np2, n2, theta, ns1, ns2, x1, x2, gamma1, gamma2, bbscale1, bbscale2, ncoll,
                               freq);
}

// BeamBeam6D_PIC_Interpolation (simtrack.cpp:24434).
void ref_bb6d_pic_interpolation(double Np1, int n1, double *x1, double Np2, int n2, double *x2, double gamma1,
                                double gamma2, double bbscale1, double bbscale2, int ns1, int ns2, double *zb1,
                                double *zb2, int nx, int ny, double hx, double hy, double *gr, double *gi) {
  BeamBeam6D_PIC_Interpolation(Np1, n1, x1, Np2, n2, x2, gamma1, gamma2, bbscale1, bbscale2, ns1, ns2, zb1, zb2, nx,
                               ny, hx, hy, gr, gi);
}

// Lumi_Cal_PIC_6D (simtrack.cpp:23703); it writes ./collide_order.dat.
double ref_lumi_pic_6d(double Np1, int n1, double Np2, int n2, int ns1, int ns2, double *x1, double *x2,
                       double gamma1, double gamma2, double bbscale1, double bbscale2, int ncoll, double freq) {
  return Lumi_Cal_PIC_6D(Np1, n1, Np2, n2, ns1, ns2, x1, x2, gamma1, gamma2, bbscale1, bbscale2, ncoll, freq);
}

// Lumi_Cal_PIC_4D (simtrack.cpp:23617).
double ref_lumi_pic_4d(double Np1, int n1, double Np2, int n2, double *x1, double *x2, int ncoll, double freq) {
  return Lumi_Cal_PIC_4D(Np1, n1, Np2, n2, x1, x2, ncoll, freq);
}

// FineTuneFinder, both overloads (simtrack.cpp:2288, 2321).
double ref_fine_tune(int n, const double *x, const double *px, double lo, double hi) {
  std::vector<double> a(x, x + n);
  double tune = 0.0;
  if (px) {
    std::vector<double> b(px, px + n);
    FineTuneFinder(n, a.data(), b.data(), lo, hi, tune);
  } else {
    FineTuneFinder(n, a.data(), lo, hi, tune);
  }
  return tune;
}

}  // extern "C"
