// Track_DA (simtrack.cpp:21389-21441) on the GPU with the reference's output.
//
// The reference bisects the stable amplitude of each of 10 phase angles
// between 0 and 50 sigma: every step tracks a twin pair (sigma, sigma + 0.05)
// with Track() and keeps the upper half if both survive; it stops when the
// interval is no longer than 0.1 sigma and writes "angle sigma" per angle.
// Each bisection can only visit the midpoints of its binary tree (511 nodes
// down to the 0.1 sigma resolution), so all of them, twins included, are
// tracked here in one batched launch; the bisection is then replayed on the
// results.  Track() is deterministic and every particle is independent, so
// the replay visits the same midpoints, sees the same outcomes and writes the
// same file as the reference.
#include <cmath>
#include <cstdio>
#include <string>
#include <vector>

#include "simtrack_b200.h"
#include "simtrack_b200.hpp"

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

}  // namespace

void Track_DA(Line &line, int nturn, double deltap0, double sigmax0, double sigmay0, const char *filename,
              double *angles_out, double *sigma_out, int device) {
  const double sigma_max = 50.0;
  std::vector<Node> tree;
  build_tree(tree, 0., sigma_max);
  const int nn = (int)tree.size();
  const int nang = 10;
  // twin particles of every node of every angle, AoS x[6] as Track() takes them
  std::vector<double> x((size_t)nang * nn * 2 * 6, 0.0);
  std::vector<double> angle(nang);
  for (int i = 0; i < nang; i++) {
    angle[i] = (90 / 11.) * (i + 1) * kPi / 180;
    for (int k = 0; k < nn; k++)
      for (int twin = 0; twin < 2; twin++) {
        const double sg = twin == 0 ? tree[k].sigma : tree[k].sigma + 0.05;
        double *p = &x[(((size_t)i * nn + k) * 2 + twin) * 6];
        p[0] = sg * std::cos(angle[i]) * sigmax0;
        p[2] = sg * std::sin(angle[i]) * sigmay0;
        p[5] = deltap0;
      }
  }
  const long n = (long)nang * nn * 2;
  std::vector<int> stable((size_t)n, 1), lost_turn((size_t)n), lost_post((size_t)n);
  Track_Batch(line, x.data(), n, nturn, stable.data(), lost_turn.data(), lost_post.data(),
              TrackOptions{0.0, device});
  FILE *f = filename ? std::fopen(filename, "w") : nullptr;
  if (filename && !f) throw Error(STB_EINVAL, std::string("cannot open ") + filename);
  for (int i = 0; i < nang; i++) {
    // replay: the reference's do { ... } while (|e - s| > 0.1) walks the tree
    int k = 0;
    double sigma = tree[0].sigma;
    while (k >= 0) {
      sigma = tree[k].sigma;
      const size_t b = ((size_t)i * nn + k) * 2;
      const bool st = stable[b] * stable[b + 1] == 1;
      k = st ? tree[k].hi : tree[k].lo;
    }
    if (angles_out) angles_out[i] = (90 / 11.) * (i + 1);
    if (sigma_out) sigma_out[i] = sigma;
    if (f) std::fprintf(f, "%f %f \n", (90 / 11.) * (i + 1), sigma);
  }
  if (f) std::fclose(f);
}

}  // namespace stb
