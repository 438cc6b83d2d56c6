// Cal_Orbit_Num (simtrack.cpp:14947-15030) with its one-turn maps on the GPU.
//
// Newton iteration for the 4D closed orbit at a fixed momentum offset: each
// iteration tracks the current guess and its four one-sided finite-difference
// neighbours (step 1e-9) through one turn in one batched launch, forms the
// Jacobian minus the identity (the reference subtracts 1.0000001 from the
// diagonal), inverts it with the same full-pivoting Gauss-Jordan elimination
// as the reference's mat_inv (simtrack.cpp:1440-1496) and corrects the
// guess; every host-side operation is done in the reference's order so the
// orbit agrees with the reference's bit for bit.  RF, crab and RF-multipole
// voltages are switched off during the search, as in the reference, and the
// final orbit is recorded after every element from one probed turn.
#include <cmath>
#include <memory>
#include <string>
#include <vector>

#include "simtrack_b200.h"
#include "simtrack_b200.hpp"

namespace stb {

namespace {

// Full-pivoting Gauss-Jordan inversion in place, n x n row-major; returns
// false for a singular matrix (|largest pivot| + 1 == 1).  The pivot search,
// row/column swaps, elimination order and the final unswapping follow
// mat_inv, simtrack.cpp:1440-1496, so that the rounding is the same.
bool invert_gauss_jordan(double *a, int n) {
  std::vector<int> is(n), js(n);
  for (int k = 0; k < n; k++) {
    double d = 0.0;
    for (int i = k; i < n; i++)
      for (int j = k; j < n; j++) {
        const double p = std::fabs(a[i * n + j]);
        if (p > d) {
          d = p;
          is[k] = i;
          js[k] = j;
        }
      }
    if (d + 1.0 == 1.0) return false;
    if (is[k] != k)
      for (int j = 0; j < n; j++) std::swap(a[k * n + j], a[is[k] * n + j]);
    if (js[k] != k)
      for (int i = 0; i < n; i++) std::swap(a[i * n + k], a[i * n + js[k]]);
    const int l = k * n + k;
    a[l] = 1.0 / a[l];
    for (int j = 0; j < n; j++)
      if (j != k) a[k * n + j] = a[k * n + j] * a[l];
    for (int i = 0; i < n; i++)
      if (i != k)
        for (int j = 0; j < n; j++)
          if (j != k) a[i * n + j] = a[i * n + j] - a[i * n + k] * a[k * n + j];
    for (int i = 0; i < n; i++)
      if (i != k) a[i * n + k] = -a[i * n + k] * a[l];
  }
  for (int k = n - 1; k >= 0; k--) {
    if (js[k] != k)
      for (int j = 0; j < n; j++) std::swap(a[k * n + j], a[js[k] * n + j]);
    if (is[k] != k)
      for (int i = 0; i < n; i++) std::swap(a[i * n + k], a[i * n + is[k]]);
  }
  return true;
}

bool is_rf(const Element *e) { return e->TYPE == "RFCAV" || e->TYPE == "CRABRF" || e->TYPE == "CCMULT"; }

// One turn of n particles (AoS x[n*6]) through a table of `line`.
void one_turn(stb_table *t, double *x, int n) {
  std::vector<int> st(n, 1), lt(n), lp(n);
  int rc = stb_track_host(t, x, n, 1, 0.0, st.data(), lt.data(), lp.data());
  if (rc != STB_OK) throw Error(rc, stb_last_error());
}

}  // namespace

void Cal_Orbit_Num(Line &line, double deltap, int device) {
  const double d = 1.0e-09, codeps = 1e-12;
  const int max_iter = 20;
  // RF voltages off for the search (simtrack.cpp:14958-14965), restored at the end
  std::vector<double> voltage;
  for (Element *e : line.Cell)
    if (is_rf(e)) {
      voltage.push_back(e->GetP("VRF"));
      e->SetP("VRF", 0.0);
    }
  auto restore = [&] {
    size_t j = 0;
    for (Element *e : line.Cell)
      if (is_rf(e)) e->SetP("VRF", voltage[j++]);
  };
  try {
    stb_table *raw = nullptr;
    int rc = stb_table_create(reinterpret_cast<const stb_line *>(&line), device, &raw);
    if (rc != STB_OK) throw Error(rc, stb_last_error());
    std::unique_ptr<stb_table, int (*)(stb_table *)> t(raw, stb_table_free);
    double x0[6] = {0., 0., 0., 0., 0., 0.};
    double chi = 0.;
    int iter = 0;
    do {
      iter++;
      x0[4] = 0;
      x0[5] = deltap;
      // x01 = M(x0) and the four neighbours x0 + d e_k, one launch
      double xs[5 * 6];
      for (int m = 0; m < 5; m++)
        for (int j = 0; j < 6; j++) xs[m * 6 + j] = x0[j];
      for (int k = 0; k < 4; k++) xs[(k + 1) * 6 + k] = xs[(k + 1) * 6 + k] + d;
      one_turn(t.get(), xs, 5);
      const double *x01 = xs;
      double mat[4][4], dx[4];
      for (int k = 0; k < 4; k++)
        for (int j = 0; j < 4; j++) mat[j][k] = (xs[(k + 1) * 6 + j] - x01[j]) / d;
      for (int i = 0; i < 4; i++) dx[i] = x0[i] - x01[i];
      chi = 0;
      for (int i = 0; i < 4; i++) chi += dx[i] * dx[i];
      chi = std::sqrt(chi / 4.);
      if (chi > codeps) {
        for (int i = 0; i < 4; i++) mat[i][i] = mat[i][i] - 1.0000001;
        if (!invert_gauss_jordan(&mat[0][0], 4))
          throw Error(STB_EABORTED, "Failed in closed orbit searching (singular matrix).");
        for (int i = 0; i < 4; i++)
          for (int j = 0; j < 4; j++) x0[i] += mat[i][j] * dx[j];
      }
    } while (chi > codeps && iter < max_iter);
    if (iter == max_iter - 1) throw Error(STB_EABORTED, "Failed to find COD.");
    // the orbit after every element, from one probed turn
    x0[4] = 0.000;
    x0[5] = deltap;
    const long ne = (long)line.Cell.size();
    std::vector<double> dump((size_t)ne * 6, NAN);
    int st = 1, lt = 0, lp = 0;
    rc = stb_track_probe(t.get(), x0, 1, 1, 0.0, dump.data(), &st, &lt, &lp);
    if (rc != STB_OK) throw Error(rc, stb_last_error());
    for (long j = 0; j < ne; j++)
      for (int i = 0; i < 6; i++) line.Cell[(size_t)j]->X[i] = dump[(size_t)j * 6 + i];
  } catch (...) {
    restore();
    throw;
  }
  restore();
}

}  // namespace stb
