// Host forest builder and flattener (include/octlb_forest.h): a brick of
// octrees with recursive refinement and 2:1 face balance, flattened into the
// lists p4est's FacePairList provides to the solver.
#include <algorithm>
#include <array>
#include <cstdint>
#include <map>
#include <tuple>
#include <vector>

#include "../../include/octlb_forest.h"

namespace {

constexpr int kMaxL = 20;  // finest representable level inside a tree

struct Leaf {
  int tx, ty, tz;     // tree
  int level;
  int64_t i, j, k;    // coordinates at `level` inside the tree
};

// Global integer coordinates (units of 2^-kMaxL of a tree).
inline std::array<int64_t, 3> gmin(const Leaf& q) {
  const int sh = kMaxL - q.level;
  return {(static_cast<int64_t>(q.tx) << kMaxL) + (q.i << sh), (static_cast<int64_t>(q.ty) << kMaxL) + (q.j << sh),
          (static_cast<int64_t>(q.tz) << kMaxL) + (q.k << sh)};
}

using Key = std::tuple<int, int64_t, int64_t, int64_t>;  // level, global min corner

uint64_t morton(int64_t x, int64_t y, int64_t z) {
  uint64_t m = 0;
  for (int b = 0; b < 21; ++b) {
    m |= ((static_cast<uint64_t>(x) >> b) & 1ull) << (3 * b);
    m |= ((static_cast<uint64_t>(y) >> b) & 1ull) << (3 * b + 1);
    m |= ((static_cast<uint64_t>(z) >> b) & 1ull) << (3 * b + 2);
  }
  return m;
}

}  // namespace

struct octlb_forest {
  int b[3];
  int per[3];
  double dom[6];
  std::vector<Leaf> leaves;
  std::map<Key, int> index;  // valid after reindex()
  bool built = false;
  std::vector<int> sl, cf, tb;
  std::vector<double> cfb;

  int64_t extent(int a) const { return static_cast<int64_t>(b[a]) << kMaxL; }

  void reindex() {
    index.clear();
    for (size_t n = 0; n < leaves.size(); ++n) {
      const auto g = gmin(leaves[n]);
      index[Key(leaves[n].level, g[0], g[1], g[2])] = static_cast<int>(n);
    }
  }
  // Leaf covering the finest-level point p (global coords), or -1 outside.
  int cover(std::array<int64_t, 3> p) const {
    for (int a = 0; a < 3; ++a) {
      if (p[a] < 0 || p[a] >= extent(a)) {
        if (!per[a]) return -1;
        p[a] = ((p[a] % extent(a)) + extent(a)) % extent(a);
      }
    }
    for (int l = kMaxL; l >= 0; --l) {
      const int64_t m = ~((static_cast<int64_t>(1) << (kMaxL - l)) - 1);
      auto it = index.find(Key(l, p[0] & m, p[1] & m, p[2] & m));
      if (it != index.end()) return it->second;
    }
    return -1;
  }
  std::array<double, 6> bounds(const Leaf& q) const {
    const auto g = gmin(q);
    const int64_t len = static_cast<int64_t>(1) << (kMaxL - q.level);
    std::array<double, 6> r{};
    for (int a = 0; a < 3; ++a) {
      const double s = (dom[3 + a] - dom[a]) / static_cast<double>(extent(a));
      r[a] = dom[a] + static_cast<double>(g[a]) * s;
      r[3 + a] = dom[a] + static_cast<double>(g[a] + len) * s;
    }
    return r;
  }
  void refine_leaf(size_t n, std::vector<Leaf>& out) const {
    const Leaf& q = leaves[n];
    for (int c = 0; c < 8; ++c)
      out.push_back({q.tx, q.ty, q.tz, q.level + 1, 2 * q.i + (c & 1), 2 * q.j + ((c >> 1) & 1),
                     2 * q.k + ((c >> 2) & 1)});
  }
  template <class Pred>
  bool refine_if(Pred pred) {
    std::vector<Leaf> out;
    bool changed = false;
    for (size_t n = 0; n < leaves.size(); ++n) {
      if (pred(leaves[n])) { refine_leaf(n, out); changed = true; }
      else out.push_back(leaves[n]);
    }
    leaves.swap(out);
    built = false;
    return changed;
  }
};

extern "C" {

octlb_forest* octlb_forest_new(int bx, int by, int bz, int px, int py, int pz, const double domain[6]) {
  if (bx < 1 || by < 1 || bz < 1 || !domain) return nullptr;
  auto* f = new octlb_forest;
  f->b[0] = bx; f->b[1] = by; f->b[2] = bz;
  f->per[0] = px != 0; f->per[1] = py != 0; f->per[2] = pz != 0;
  for (int a = 0; a < 6; ++a) f->dom[a] = domain[a];
  for (int z = 0; z < bz; ++z)
    for (int y = 0; y < by; ++y)
      for (int x = 0; x < bx; ++x) f->leaves.push_back({x, y, z, 0, 0, 0, 0});
  return f;
}

void octlb_forest_free(octlb_forest* f) { delete f; }

int octlb_forest_refine_uniform(octlb_forest* f, int level) {
  if (!f || level < 0 || level > kMaxL) return -1;
  while (f->refine_if([&](const Leaf& q) { return q.level < level; })) {}
  return 0;
}

int octlb_forest_refine_box(octlb_forest* f, const double box[6], int level) {
  if (!f || !box || level < 0 || level > kMaxL) return -1;
  while (f->refine_if([&](const Leaf& q) {
    if (q.level >= level) return false;
    const auto bd = f->bounds(q);
    for (int a = 0; a < 3; ++a)
      if (!(bd[a] < box[3 + a] && bd[3 + a] > box[a])) return false;
    return true;
  })) {}
  return 0;
}

int octlb_forest_balance(octlb_forest* f) {
  if (!f) return -1;
  for (;;) {
    f->reindex();
    std::vector<char> mark(f->leaves.size(), 0);
    bool any = false;
    for (const Leaf& q : f->leaves) {
      const auto g = gmin(q);
      const int64_t len = static_cast<int64_t>(1) << (kMaxL - q.level);
      for (int d = 0; d < 6; ++d) {
        const int a = d / 2;
        std::array<int64_t, 3> p = g;
        p[a] += (d & 1) ? len : -1;
        const int c = f->cover(p);
        if (c >= 0 && f->leaves[c].level < q.level - 1 && !mark[c]) { mark[c] = 1; any = true; }
      }
    }
    if (!any) break;
    std::vector<Leaf> out;
    for (size_t n = 0; n < f->leaves.size(); ++n) {
      if (mark[n]) f->refine_leaf(n, out);
      else out.push_back(f->leaves[n]);
    }
    f->leaves.swap(out);
  }
  f->built = false;
  return 0;
}

int octlb_forest_build(octlb_forest* f) {
  if (!f) return -1;
  std::stable_sort(f->leaves.begin(), f->leaves.end(), [&](const Leaf& a, const Leaf& b) {
    const int ta = a.tx + f->b[0] * (a.ty + f->b[1] * a.tz), tb = b.tx + f->b[0] * (b.ty + f->b[1] * b.tz);
    if (ta != tb) return ta < tb;
    const int sa = kMaxL - a.level, sb = kMaxL - b.level;
    const uint64_t ma = morton(a.i << sa, a.j << sa, a.k << sa), mb = morton(b.i << sb, b.j << sb, b.k << sb);
    if (ma != mb) return ma < mb;
    return a.level < b.level;
  });
  f->reindex();
  f->sl.clear(); f->cf.clear(); f->tb.clear(); f->cfb.clear();
  std::vector<std::pair<int, std::vector<int>>> cf_rows;       // (coarse level, row)
  std::vector<std::vector<double>> cf_bounds;
  for (size_t n = 0; n < f->leaves.size(); ++n) {
    const Leaf& q = f->leaves[n];
    const auto g = gmin(q);
    const int64_t len = static_cast<int64_t>(1) << (kMaxL - q.level);
    for (int d = 0; d < 6; ++d) {
      const int a = d / 2, t0 = (a + 1) % 3, t1 = (a + 2) % 3;
      std::array<int64_t, 3> p = g;
      p[a] += (d & 1) ? len : -1;
      const int c = f->cover(p);
      if (c < 0) {  // outer face
        f->tb.push_back(static_cast<int>(n));
        f->tb.push_back(d);
        continue;
      }
      const Leaf& r = f->leaves[c];
      if (r.level == q.level) {
        f->sl.push_back(static_cast<int>(n)); f->sl.push_back(d); f->sl.push_back(c);
      } else if (r.level == q.level + 1) {
        // Hanging face seen from the coarse side: the four fine leaves.
        std::vector<int> fine;
        const int64_t h = len / 2;
        for (int s1 = 0; s1 < 2; ++s1)
          for (int s0 = 0; s0 < 2; ++s0) {
            std::array<int64_t, 3> pp = p;
            pp[std::min(t0, t1)] += s0 * h;
            pp[std::max(t0, t1)] += s1 * h;
            fine.push_back(f->cover(pp));
          }
        std::sort(fine.begin(), fine.end());
        std::vector<int> row = {static_cast<int>(n), fine[0], fine[1], fine[2], fine[3], d, q.level, q.level + 1};
        std::vector<double> bd;
        const auto cb = f->bounds(q);
        bd.insert(bd.end(), cb.begin(), cb.end());
        for (int s = 0; s < 4; ++s) {
          const auto fb = f->bounds(f->leaves[fine[s]]);
          bd.insert(bd.end(), fb.begin(), fb.end());
        }
        cf_rows.push_back({q.level, row});
        cf_bounds.push_back(bd);
      }
      // r.level == q.level - 1: listed from the coarse side.
    }
  }
  std::vector<size_t> order(cf_rows.size());
  for (size_t k = 0; k < order.size(); ++k) order[k] = k;
  std::stable_sort(order.begin(), order.end(), [&](size_t x, size_t y) { return cf_rows[x].first < cf_rows[y].first; });
  for (size_t k : order) {
    f->cf.insert(f->cf.end(), cf_rows[k].second.begin(), cf_rows[k].second.end());
    f->cfb.insert(f->cfb.end(), cf_bounds[k].begin(), cf_bounds[k].end());
  }
  f->built = true;
  return static_cast<int>(f->leaves.size());
}

int octlb_forest_num_leaves(const octlb_forest* f) { return f ? static_cast<int>(f->leaves.size()) : -1; }

int octlb_forest_leaves(const octlb_forest* f, int* levels, double* bounds) {
  if (!f || !f->built) return -1;
  for (size_t n = 0; n < f->leaves.size(); ++n) {
    if (levels) levels[n] = f->leaves[n].level;
    if (bounds) {
      const auto b = f->bounds(f->leaves[n]);
      for (int a = 0; a < 6; ++a) bounds[6 * n + a] = b[a];
    }
  }
  return static_cast<int>(f->leaves.size());
}
int octlb_forest_num_same_level(const octlb_forest* f) { return f && f->built ? static_cast<int>(f->sl.size() / 3) : -1; }
int octlb_forest_same_level(const octlb_forest* f, int* out) {
  if (!f || !f->built) return -1;
  std::copy(f->sl.begin(), f->sl.end(), out);
  return static_cast<int>(f->sl.size() / 3);
}
int octlb_forest_num_coarse_fine(const octlb_forest* f) { return f && f->built ? static_cast<int>(f->cf.size() / 8) : -1; }
int octlb_forest_coarse_fine(const octlb_forest* f, int* out, double* bounds) {
  if (!f || !f->built) return -1;
  std::copy(f->cf.begin(), f->cf.end(), out);
  if (bounds) std::copy(f->cfb.begin(), f->cfb.end(), bounds);
  return static_cast<int>(f->cf.size() / 8);
}
int octlb_forest_num_tree_boundary(const octlb_forest* f) { return f && f->built ? static_cast<int>(f->tb.size() / 2) : -1; }
int octlb_forest_tree_boundary(const octlb_forest* f, int* out) {
  if (!f || !f->built) return -1;
  std::copy(f->tb.begin(), f->tb.end(), out);
  return static_cast<int>(f->tb.size() / 2);
}

}  // extern "C"
