// Synthetic block-AMR forests and right-hand sides (see forest.hpp).
#include "forest.hpp"

#include <algorithm>
#include <cmath>
#include <random>
#include <unordered_map>
#include <unordered_set>

namespace cup2d {

namespace {

inline uint64_t key3(int l, int64_t i, int64_t j) {
  return ((uint64_t)l << 58) | ((uint64_t)i << 29) | (uint64_t)j;
}

inline uint64_t spread_bits(uint64_t v) {
  v &= 0xffffffffull;
  v = (v | (v << 16)) & 0x0000ffff0000ffffull;
  v = (v | (v << 8)) & 0x00ff00ff00ff00ffull;
  v = (v | (v << 4)) & 0x0f0f0f0f0f0f0f0full;
  v = (v | (v << 2)) & 0x3333333333333333ull;
  v = (v | (v << 1)) & 0x5555555555555555ull;
  return v;
}

struct LeafSet {
  int L;  // levels
  std::vector<std::unordered_set<uint64_t>> lv;
  explicit LeafSet(int levels) : L(levels), lv(levels) {}
  static uint64_t k(int64_t i, int64_t j) { return ((uint64_t)i << 32) | (uint64_t)j; }
  bool has(int l, int64_t i, int64_t j) const { return lv[l].count(k(i, j)) != 0; }
  void add(int l, int64_t i, int64_t j) { lv[l].insert(k(i, j)); }
  void del(int l, int64_t i, int64_t j) { lv[l].erase(k(i, j)); }
};

bool rect_meets_band(double x0, double y0, double x1, double y1, const Disk& d,
                     double band) {
  const double dx = std::max({x0 - d.cx, 0.0, d.cx - x1});
  const double dy = std::max({y0 - d.cy, 0.0, d.cy - y1});
  const double dmin = std::sqrt(dx * dx + dy * dy);
  const double fx = std::max(std::fabs(x0 - d.cx), std::fabs(x1 - d.cx));
  const double fy = std::max(std::fabs(y0 - d.cy), std::fabs(y1 - d.cy));
  const double dmax = std::sqrt(fx * fx + fy * fy);
  return dmin <= d.r + band && dmax >= d.r - band;
}

// Finds the level of the leaf covering position (l,i,j), searching coarser
// levels; -1 if the position is covered by finer leaves (or nothing).
int covering_level(const LeafSet& s, int l, int64_t i, int64_t j) {
  for (int q = l; q >= 0; --q) {
    const int sh = l - q;
    if (s.has(q, i >> sh, j >> sh)) return q;
  }
  return -1;
}

void balance(LeafSet& s, const ForestSpec& sp) {
  bool changed = true;
  while (changed) {
    changed = false;
    for (int l = sp.level_max - 1; l >= 2; --l) {
      std::vector<uint64_t> cur(s.lv[l].begin(), s.lv[l].end());
      const int64_t nx = (int64_t)sp.bpdx << l, ny = (int64_t)sp.bpdy << l;
      for (uint64_t kk : cur) {
        const int64_t i = (int64_t)(kk >> 32), j = (int64_t)(kk & 0xffffffffu);
        for (int dj = -1; dj <= 1; ++dj)
          for (int di = -1; di <= 1; ++di) {
            if (!di && !dj) continue;
            int64_t ni = i + di, nj = j + dj;
            if (ni < 0 || ni >= nx) {
              if (!sp.periodic_x) continue;
              ni = (ni + nx) % nx;
            }
            if (nj < 0 || nj >= ny) {
              if (!sp.periodic_y) continue;
              nj = (nj + ny) % ny;
            }
            const int q = covering_level(s, l, ni, nj);
            if (q >= 0 && q < l - 1) {
              // split the coarse leaf (q, ni>>(l-q), nj>>(l-q)) once
              const int sh = l - q;
              const int64_t ci = ni >> sh, cj = nj >> sh;
              s.del(q, ci, cj);
              for (int c = 0; c < 4; ++c) s.add(q + 1, 2 * ci + (c & 1), 2 * cj + (c >> 1));
              changed = true;
            }
          }
      }
    }
  }
}

Forest to_forest(const LeafSet& s, const ForestSpec& sp) {
  struct Item { uint64_t key; int l; int32_t i, j; };
  std::vector<Item> items;
  const int top = sp.level_max - 1;
  for (int l = 0; l < sp.level_max; ++l)
    for (uint64_t kk : s.lv[l]) {
      const int32_t i = (int32_t)(kk >> 32), j = (int32_t)(kk & 0xffffffffu);
      const uint64_t fi = (uint64_t)i << (top - l), fj = (uint64_t)j << (top - l);
      items.push_back({spread_bits(fi) | (spread_bits(fj) << 1), l, i, j});
    }
  std::sort(items.begin(), items.end(),
            [](const Item& a, const Item& b) { return a.key < b.key; });
  Forest f;
  f.spec = sp;
  f.level.reserve(items.size());
  for (auto& it : items) {
    f.level.push_back(it.l);
    f.bx.push_back(it.i);
    f.by.push_back(it.j);
  }
  return f;
}

}  // namespace

double cell_h(const ForestSpec& s, int level) {
  return s.extent / ((double)std::max(s.bpdx, s.bpdy) * 8.0 * (double)(1ll << level));
}

Forest build_disk_forest(const ForestSpec& sp, const std::vector<Disk>& disks,
                         double band) {
  LeafSet s(sp.level_max);
  // depth-first refinement from the roots
  struct Node { int l; int64_t i, j; };
  std::vector<Node> stack;
  for (int j = 0; j < sp.bpdy; ++j)
    for (int i = 0; i < sp.bpdx; ++i) stack.push_back({0, i, j});
  while (!stack.empty()) {
    Node n = stack.back();
    stack.pop_back();
    bool refine = false;
    if (n.l < sp.level_max - 1) {
      const double bs = 8.0 * cell_h(sp, n.l);
      const double x0 = n.i * bs, y0 = n.j * bs;
      for (const Disk& d : disks)
        if (rect_meets_band(x0, y0, x0 + bs, y0 + bs, d, band)) { refine = true; break; }
    }
    if (refine) {
      for (int c = 0; c < 4; ++c)
        stack.push_back({n.l + 1, 2 * n.i + (c & 1), 2 * n.j + (c >> 1)});
    } else {
      s.add(n.l, n.i, n.j);
    }
  }
  balance(s, sp);
  return to_forest(s, sp);
}

Forest build_uniform_forest(const ForestSpec& sp, int level) {
  LeafSet s(sp.level_max);
  const int64_t nx = (int64_t)sp.bpdx << level, ny = (int64_t)sp.bpdy << level;
  for (int64_t j = 0; j < ny; ++j)
    for (int64_t i = 0; i < nx; ++i) s.add(level, i, j);
  return to_forest(s, sp);
}

int validate_forest(const Forest& f) {
  const ForestSpec& sp = f.spec;
  if (sp.level_max < 1 || sp.level_max > 20 || sp.bpdx < 1 || sp.bpdy < 1) return 3;
  LeafSet s(sp.level_max);
  const int top = sp.level_max - 1;
  long double area = 0;
  for (int64_t b = 0; b < f.size(); ++b) {
    const int l = f.level[b];
    if (l < 0 || l > top) return 3;
    const int64_t nx = (int64_t)sp.bpdx << l, ny = (int64_t)sp.bpdy << l;
    if (f.bx[b] < 0 || f.bx[b] >= nx || f.by[b] < 0 || f.by[b] >= ny) return 3;
    if (s.has(l, f.bx[b], f.by[b])) return 1;
    s.add(l, f.bx[b], f.by[b]);
    area += std::ldexp(1.0L, -2 * l);
  }
  if (area != (long double)sp.bpdx * sp.bpdy) return 1;
  // overlap between levels: an ancestor of a leaf must not be a leaf
  for (int64_t b = 0; b < f.size(); ++b)
    for (int q = f.level[b] - 1; q >= 0; --q) {
      const int sh = f.level[b] - q;
      if (s.has(q, f.bx[b] >> sh, f.by[b] >> sh)) return 1;
    }
  // 2:1 across faces and corners
  for (int64_t b = 0; b < f.size(); ++b) {
    const int l = f.level[b];
    const int64_t nx = (int64_t)sp.bpdx << l, ny = (int64_t)sp.bpdy << l;
    for (int dj = -1; dj <= 1; ++dj)
      for (int di = -1; di <= 1; ++di) {
        if (!di && !dj) continue;
        int64_t ni = f.bx[b] + di, nj = f.by[b] + dj;
        if (ni < 0 || ni >= nx) {
          if (!sp.periodic_x) continue;
          ni = (ni + nx) % nx;
        }
        if (nj < 0 || nj >= ny) {
          if (!sp.periodic_y) continue;
          nj = (nj + ny) % ny;
        }
        // A neighbour covered by finer leaves is checked from the finer
        // leaves' side, where this block is the coarser one.
        const int q = covering_level(s, l, ni, nj);
        if (q >= 0 && q < l - 1) return 2;
      }
  }
  return 0;
}

// ---------------------------------------------------------------- RHS --------

int fourier_num_modes(int kmax) {
  int n = 0;
  for (int ky = -kmax; ky <= kmax; ++ky)
    for (int kx = 0; kx <= kmax; ++kx) {
      if (kx == 0 && ky <= 0) continue;
      if (kx * kx + ky * ky > kmax * kmax) continue;
      ++n;
    }
  return n;
}

namespace {
struct Mode { int kx, ky; double amp; };
std::vector<Mode> modes_of(int kmax) {
  std::vector<Mode> m;
  for (int ky = -kmax; ky <= kmax; ++ky)
    for (int kx = 0; kx <= kmax; ++kx) {
      if (kx == 0 && ky <= 0) continue;
      const int k2 = kx * kx + ky * ky;
      if (k2 > kmax * kmax) continue;
      m.push_back({kx, ky, 1.0 / (double)k2});  // |k|^-2
    }
  return m;
}
}  // namespace

void fourier_init_coefs(uint64_t seed, int kmax, double* coef) {
  std::mt19937_64 rng(seed);
  std::normal_distribution<double> nd(0.0, 1.0);
  const int nm = fourier_num_modes(kmax);
  for (int q = 0; q < 4 * nm; ++q) coef[q] = nd(rng);
}

void fourier_advance_coefs(uint64_t seed, int kmax, double rho, int64_t step,
                           double* coef) {
  std::mt19937_64 rng(seed ^ (0x9e3779b97f4a7c15ull * (uint64_t)(step + 1)));
  std::normal_distribution<double> nd(0.0, 1.0);
  const int nm = fourier_num_modes(kmax);
  const double s = std::sqrt(std::max(0.0, 1.0 - rho * rho));
  for (int q = 0; q < 4 * nm; ++q) coef[q] = rho * coef[q] + s * nd(rng);
}

void fourier_rhs_from_coefs(const Forest& f, int kmax, const double* coef,
                            double* b) {
  const ForestSpec& sp = f.spec;
  const std::vector<Mode> modes = modes_of(kmax);
  const int nm = (int)modes.size();
  const double h0 = cell_h(sp, 0);
  const double Lx = sp.bpdx * 8.0 * h0, Ly = sp.bpdy * 8.0 * h0;
  const double wx = 2.0 * M_PI / Lx, wy = 2.0 * M_PI / Ly;
  const int64_t nb = f.size();
  // velocity components at one point
  auto vel = [&](double x, double y, int comp) {
    double cx[32], sx[32], cy[64], sy[64];
    for (int k = 0; k <= kmax; ++k) {
      cx[k] = std::cos(wx * k * x);
      sx[k] = std::sin(wx * k * x);
    }
    for (int k = -kmax; k <= kmax; ++k) {
      cy[k + kmax] = std::cos(wy * k * y);
      sy[k + kmax] = std::sin(wy * k * y);
    }
    double acc = 0.0;
    for (int q = 0; q < nm; ++q) {
      const Mode& m = modes[q];
      const double c = cx[m.kx] * cy[m.ky + kmax] - sx[m.kx] * sy[m.ky + kmax];
      const double s = sx[m.kx] * cy[m.ky + kmax] + cx[m.kx] * sy[m.ky + kmax];
      const double a = coef[4 * q + 2 * comp], bb = coef[4 * q + 2 * comp + 1];
      acc += m.amp * (a * c + bb * s);
    }
    return acc;
  };
#pragma omp parallel for schedule(static)
  for (int64_t blk = 0; blk < nb; ++blk) {
    const int l = f.level[blk];
    const double h = cell_h(sp, l);
    for (int iy = 0; iy < 8; ++iy)
      for (int ix = 0; ix < 8; ++ix) {
        const double x = (f.bx[blk] * 8 + ix + 0.5) * h;
        const double y = (f.by[blk] * 8 + iy + 0.5) * h;
        const double du = vel(x + h, y, 0) - vel(x - h, y, 0);
        const double dv = vel(x, y + h, 1) - vel(x, y - h, 1);
        b[blk * 64 + iy * 8 + ix] = 0.5 * h * (du + dv);
      }
  }
  // zero entry-sum (compensated sum so the projection is exact to rounding)
  long double s = 0;
  const int64_t n = nb * 64;
  for (int64_t i = 0; i < n; ++i) s += b[i];
  const double mean = (double)(s / (long double)n);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) b[i] -= mean;
}

void fourier_rhs(const Forest& f, uint64_t seed, int kmax, double* b) {
  std::vector<double> coef(4 * fourier_num_modes(kmax));
  fourier_init_coefs(seed, kmax, coef.data());
  fourier_rhs_from_coefs(f, kmax, coef.data(), b);
}

}  // namespace cup2d
