// ORACLE — test infrastructure only.  CPU FP64 restatement of the three field
// kernels of CUP2D's pressure projection around the Poisson solve, written
// the way the reference runs them: a lab (the block plus one ghost layer) per
// block, the kernel's per-cell formula over the 64 cells, the face values the
// kernel stores for coarse/fine faces, then a flux-correction pass.
// Nothing in the product library links, loads or calls this file.
//
// Reference kernels (source/Operators/PressureSingle.cpp):
//   updatePressureRHS  :324-397   TMP = facDiv ((u_E - u_W) + (v_N - v_S))
//                                       + (-facDiv CHI) ((ud_E - ud_W) + (vd_N - vd_S)),
//                                 facDiv = 0.5 h / dt; stored faces :357-396
//   updatePressureRHS1 :399-456   TMP -= ((p_W + p_E) + (p_S + p_N)) - 4 p;
//                                 stored faces lab(nb) - lab(self) :433-455
//   pressureCorrection :123-210   tmpV = pFac (P_E - P_W, P_N - P_S), pFac = -0.5 dt h;
//                                 stored faces :152-185; V += tmpV (1/h)/h :191-210
//   operator()         :826-849   RHS, POLD = PRES, PRES = 0, RHS1.
//
// Cubism, the AMR library that supplies the labs and the flux correction, is
// an un-vendored submodule of CUP2D; its parts are restated from their use:
//   * domain edges: BlockLabDirichlet (source/Definitions.h:71-196) flips the
//     sign of the normal velocity component in the ghost (wall and free-space
//     alike); BlockLabNeumann (:200-228) copies the edge cell into the ghost;
//   * a ghost from a coarser block: the quadratic interpolation ExpAMRSolver
//     applies to the same cells (ExpAMRSolver.cpp:100-128, D1/D2 of
//     ExpAMRSolver.h:268-300), evaluated on values;
//   * a ghost from finer blocks: the mean of the four fine cells it covers;
//   * flux correction: each coarse cell on a coarse/fine face adds its own
//     stored face value and the two fine cells' stored face values.
// Parity of cells next to a coarse/fine face is therefore unpinned (the
// reference's own Cubism could not be run); cells away from such faces follow
// PressureSingle.cpp's formulas exactly.
#include <array>
#include <cstdint>
#include <stdexcept>
#include <unordered_map>
#include <vector>

extern "C" {
typedef struct oracle_forest {
  int32_t bpdx, bpdy, level_max, periodic_x, periodic_y;
  double extent;
  int64_t nblocks;
  const int32_t* level;
  const int32_t* bx;
  const int32_t* by;
} oracle_forest;
}

namespace {

constexpr int BS = 8;
constexpr double k23 = 2. / 3., k15 = 1. / 5., k815 = 8. / 15.;

struct Forest {
  const oracle_forest& f;
  std::vector<std::unordered_map<uint64_t, int64_t>> lv;
  double h0;
  explicit Forest(const oracle_forest& ff) : f(ff), lv(ff.level_max) {
    for (int64_t b = 0; b < f.nblocks; ++b) lv[f.level[b]][key(f.bx[b], f.by[b])] = b;
    h0 = f.extent / ((double)(f.bpdx > f.bpdy ? f.bpdx : f.bpdy) * BS);
  }
  static uint64_t key(int64_t i, int64_t j) { return ((uint64_t)i << 32) | (uint64_t)(uint32_t)j; }
  int64_t find(int l, int64_t i, int64_t j) const {
    if (l < 0 || l >= f.level_max) return -1;
    auto it = lv[l].find(key(i, j));
    return it == lv[l].end() ? -1 : it->second;
  }
  double h(int64_t b) const { return h0 / (double)(1ll << f.level[b]); }
  // same-level position across face (0 W, 1 E, 2 S, 3 N); false at a wall
  bool across(int64_t b, int face, int64_t& ni, int64_t& nj) const {
    const int l = f.level[b];
    const int64_t nx = (int64_t)f.bpdx << l, ny = (int64_t)f.bpdy << l;
    ni = f.bx[b] + (face == 0 ? -1 : face == 1 ? 1 : 0);
    nj = f.by[b] + (face == 2 ? -1 : face == 3 ? 1 : 0);
    if (ni < 0 || ni >= nx) {
      if (!f.periodic_x) return false;
      ni = (ni + nx) % nx;
    }
    if (nj < 0 || nj >= ny) {
      if (!f.periodic_y) return false;
      nj = (nj + ny) % ny;
    }
    return true;
  }
};

inline int64_t at(int64_t b, int ix, int iy) { return b * 64 + iy * BS + ix; }

// A field: `nc` doubles per cell (1 scalar, 2 velocity).
struct Field {
  const double* p;
  int nc;
  double v(int64_t b, int ix, int iy, int c) const { return p[at(b, ix, iy) * nc + c]; }
};

// Kind of face neighbour.
enum { SAME, WALL, COARSE, FINE };
struct Nei {
  int kind;
  int64_t blk;       // SAME / COARSE: that block
  int64_t fine[2];   // FINE: the child blocks touching cells 0-3 and 4-7 of the face
};

Nei neighbour(const Forest& F, int64_t b, int face) {
  Nei n{WALL, -1, {-1, -1}};
  int64_t ni, nj;
  if (!F.across(b, face, ni, nj)) return n;
  const int l = F.f.level[b];
  if ((n.blk = F.find(l, ni, nj)) >= 0) { n.kind = SAME; return n; }
  if ((n.blk = F.find(l - 1, ni / 2, nj / 2)) >= 0) { n.kind = COARSE; return n; }
  for (int half = 0; half < 2; ++half) {
    int64_t ci, cj;
    switch (face) {
      case 0: ci = 2 * ni + 1; cj = 2 * nj + half; break;
      case 1: ci = 2 * ni;     cj = 2 * nj + half; break;
      case 2: ci = 2 * ni + half; cj = 2 * nj + 1; break;
      default: ci = 2 * ni + half; cj = 2 * nj; break;
    }
    n.fine[half] = F.find(l + 1, ci, cj);
    if (n.fine[half] < 0) throw std::runtime_error("hole in the forest");
  }
  n.kind = FINE;
  return n;
}

// Cell (ix, iy) of block nb seen across `face`, `depth` cells in.
void mirror(int face, int ix, int iy, int depth, int& jx, int& jy) {
  jx = ix;
  jy = iy;
  switch (face) {
    case 0: jx = BS - 1 - depth; break;
    case 1: jx = depth; break;
    case 2: jy = BS - 1 - depth; break;
    default: jy = depth; break;
  }
}

// ExpAMRSolver::interpolate on values: ghost of the fine cell `close` (next
// inward fine cell `far`) from coarse cell (xc, yc) of block bc, Taylor sign sT.
double interp(const Field& w, int c, int64_t bc, int xc, int yc, double vclose, double vfar, double sT, bool xface) {
  const int t = xface ? yc : xc;  // position along the face
  auto cv = [&](int d) { return xface ? w.v(bc, xc, yc + d, c) : w.v(bc, xc + d, yc, c); };
  double v0, v1, a0, a1, a2, b0, b1, b2;
  const double v2 = cv(0);
  if (t == BS - 1 || t == BS / 2 - 1) {
    v0 = cv(-2); v1 = cv(-1);
    a0 = 1. / 8.; a1 = -1. / 2.; a2 = 3. / 8.;
    b0 = 1. / 32.; b1 = -1. / 16.; b2 = 1. / 32.;
  } else if (t == 0 || t == BS / 2) {
    v0 = cv(2); v1 = cv(1);
    a0 = -1. / 8.; a1 = 1. / 2.; a2 = -3. / 8.;
    b0 = 1. / 32.; b1 = -1. / 16.; b2 = 1. / 32.;
  } else {
    v0 = cv(-1); v1 = cv(1);
    a0 = -1. / 8.; a1 = 1. / 8.; a2 = 0.;
    b0 = 1. / 32.; b1 = 1. / 32.; b2 = -1. / 16.;
  }
  const double d1 = (a0 * v0 + a1 * v1) + a2 * v2;
  const double d2 = (b0 * v0 + b1 * v1) + b2 * v2;
  const double tay = (v2 + sT * d1) + d2;
  return (k23 * vclose - k15 * vfar) + k815 * tay;
}

// The lab of block b for field w: lab[(iy+1)*10 + ix+1][c], ghosts on the four
// faces (corners unused).  `vector`: the BlockLabDirichlet edge rule, else
// BlockLabNeumann's.
struct Lab {
  std::vector<double> d;
  int nc;
  double& operator()(int ix, int iy, int c) { return d[((iy + 1) * (BS + 2) + ix + 1) * nc + c]; }
};

void fill_lab(const Forest& F, const Field& w, bool vector, int64_t b, const Nei nb[4], Lab& L) {
  L.nc = w.nc;
  L.d.assign((BS + 2) * (BS + 2) * w.nc, 0.0);
  for (int iy = 0; iy < BS; ++iy)
    for (int ix = 0; ix < BS; ++ix)
      for (int c = 0; c < w.nc; ++c) L(ix, iy, c) = w.v(b, ix, iy, c);
  const int64_t bi = F.f.bx[b], bj = F.f.by[b];
  for (int face = 0; face < 4; ++face) {
    const bool xface = face < 2;
    for (int k = 0; k < BS; ++k) {
      const int ix = xface ? (face == 0 ? 0 : BS - 1) : k;   // edge cell
      const int iy = xface ? k : (face == 2 ? 0 : BS - 1);
      const int gx = ix + (face == 0 ? -1 : face == 1 ? 1 : 0);
      const int gy = iy + (face == 2 ? -1 : face == 3 ? 1 : 0);
      for (int c = 0; c < w.nc; ++c) {
        double g;
        const Nei& n = nb[face];
        if (n.kind == SAME) {
          int jx, jy;
          mirror(face, ix, iy, 0, jx, jy);
          g = w.v(n.blk, jx, jy, c);
        } else if (n.kind == WALL) {
          const bool normal = vector && (c == (xface ? 0 : 1));
          g = normal ? -w.v(b, ix, iy, c) : w.v(b, ix, iy, c);
        } else if (n.kind == COARSE) {
          const int xc = face == 0 ? BS - 1 : face == 1 ? 0 : (bi % 2 == 0 ? ix / 2 : ix / 2 + BS / 2);
          const int yc = face == 2 ? BS - 1 : face == 3 ? 0 : (bj % 2 == 0 ? iy / 2 : iy / 2 + BS / 2);
          const int fx = ix + (face == 0 ? 1 : face == 1 ? -1 : 0);  // inward cell
          const int fy = iy + (face == 2 ? 1 : face == 3 ? -1 : 0);
          const double sT = xface ? (iy % 2 == 0 ? -1. : 1.) : (ix % 2 == 0 ? -1. : 1.);
          g = interp(w, c, n.blk, xc, yc, w.v(b, ix, iy, c), w.v(b, fx, fy, c), sT, xface);
        } else {
          const int64_t fb = n.fine[xface ? (iy >= BS / 2) : (ix >= BS / 2)];
          const int f0 = (k % (BS / 2)) * 2;
          double s[2][2];  // [depth][along]
          for (int dpt = 0; dpt < 2; ++dpt)
            for (int q = 0; q < 2; ++q) {
              int jx, jy;
              mirror(face, xface ? 0 : f0 + q, xface ? f0 + q : 0, dpt, jx, jy);
              s[dpt][q] = w.v(fb, jx, jy, c);
            }
          g = 0.25 * ((s[0][0] + s[0][1]) + (s[1][0] + s[1][1]));
        }
        L(gx, gy, c) = g;
      }
    }
  }
}

// Face values a kernel stores on the faces of block b whose neighbour is at
// another level: faces[face][k][c] for cell k along the face.
using Faces = std::vector<double>;  // [4][BS][nc]

struct Stored {
  std::vector<Faces> f;  // per block
  int nc;
  double& operator()(int64_t b, int face, int k, int c) { return f[b][(face * BS + k) * nc + c]; }
};

// The fine cells of block nb that face cell k of a coarse face `face`, with
// their position along their own (opposite) face.
void fine_cells(int face, int k, int q, int& kk) {
  (void)face;
  kk = (k % (BS / 2)) * 2 + q;
}

// Flux correction: coarse cell += coarse face + (fine face 0 + fine face 1).
void correct(const Forest& F, const std::vector<std::array<Nei, 4>>& nbs, Stored& S,
             double* out, int nc) {
  for (int64_t b = 0; b < F.f.nblocks; ++b)
    for (int face = 0; face < 4; ++face) {
      const Nei& n = nbs[b][face];
      if (n.kind != FINE) continue;
      const int opp = face ^ 1;
      const bool xface = face < 2;
      for (int k = 0; k < BS; ++k) {
        const int ix = xface ? (face == 0 ? 0 : BS - 1) : k;
        const int iy = xface ? k : (face == 2 ? 0 : BS - 1);
        const int64_t fb = n.fine[k >= BS / 2];
        for (int c = 0; c < nc; ++c) {
          int k0, k1;
          fine_cells(face, k, 0, k0);
          fine_cells(face, k, 1, k1);
          const double add = S(b, face, k, c) + (S(fb, opp, k0, c) + S(fb, opp, k1, c));
          out[at(b, ix, iy) * nc + c] = out[at(b, ix, iy) * nc + c] + add;
        }
      }
    }
}

}  // namespace

extern "C" {

// PressureSingle.cpp:826-849 before the solve.  vel/udef: 2 doubles per cell,
// chi: 1; tmp out.  With pres set: pold = pres and tmp -= L(pres) (pres itself
// is not changed here; the reference then zeroes it).  vel may be NULL: tmp is
// then only reduced by L(pres).
int oracle_pressure_rhs(const oracle_forest* fp, double dt, const double* vel, const double* udef,
                        const double* chi, const double* pres, double* tmp, double* pold) {
  try {
    const Forest F(*fp);
    const int64_t nb = fp->nblocks;
    std::vector<std::array<Nei, 4>> nbs(nb);
    for (int64_t b = 0; b < nb; ++b)
      for (int face = 0; face < 4; ++face) nbs[b][face] = neighbour(F, b, face);
    if (vel) {  // updatePressureRHS + flux correction
      const Field V{vel, 2}, U{udef, 2};
      Stored S{std::vector<Faces>(nb, Faces(4 * BS * 1, 0.0)), 1};
      for (int64_t b = 0; b < nb; ++b) {
        Lab vl, ul;
        fill_lab(F, V, true, b, nbs[b].data(), vl);
        fill_lab(F, U, true, b, nbs[b].data(), ul);
        const double h = F.h(b);
        const double facDiv = 0.5 * h / dt;
        for (int iy = 0; iy < BS; ++iy)
          for (int ix = 0; ix < BS; ++ix) {
            const double CHI = chi[at(b, ix, iy)];
            double t = facDiv * ((vl(ix + 1, iy, 0) - vl(ix - 1, iy, 0)) + (vl(ix, iy + 1, 1) - vl(ix, iy - 1, 1)));
            t += -facDiv * CHI * ((ul(ix + 1, iy, 0) - ul(ix - 1, iy, 0)) + (ul(ix, iy + 1, 1) - ul(ix, iy - 1, 1)));
            tmp[at(b, ix, iy)] = t;
          }
        for (int face = 0; face < 4; ++face) {
          if (nbs[b][face].kind != COARSE && nbs[b][face].kind != FINE) continue;
          for (int k = 0; k < BS; ++k) {
            const bool xface = face < 2;
            const int ix = xface ? (face == 0 ? 0 : BS - 1) : k;
            const int iy = xface ? k : (face == 2 ? 0 : BS - 1);
            const int gx = ix + (face == 0 ? -1 : face == 1 ? 1 : 0);
            const int gy = iy + (face == 2 ? -1 : face == 3 ? 1 : 0);
            const int c = xface ? 0 : 1;
            const double CHI = chi[at(b, ix, iy)];
            double s;
            if (face == 0 || face == 2) {
              s = facDiv * (vl(gx, gy, c) + vl(ix, iy, c));
              s += -(facDiv * CHI) * (ul(gx, gy, c) + ul(ix, iy, c));
            } else {
              s = -facDiv * (vl(gx, gy, c) + vl(ix, iy, c));
              s -= -(facDiv * CHI) * (ul(gx, gy, c) + ul(ix, iy, c));
            }
            S(b, face, k, 0) = s;
          }
        }
      }
      correct(F, nbs, S, tmp, 1);
    }
    if (pres) {  // POLD = PRES; updatePressureRHS1 + flux correction
      const Field P{pres, 1};
      for (int64_t i = 0; i < nb * 64; ++i) pold[i] = pres[i];
      Stored S{std::vector<Faces>(nb, Faces(4 * BS * 1, 0.0)), 1};
      for (int64_t b = 0; b < nb; ++b) {
        Lab L;
        fill_lab(F, P, false, b, nbs[b].data(), L);
        for (int iy = 0; iy < BS; ++iy)
          for (int ix = 0; ix < BS; ++ix)
            tmp[at(b, ix, iy)] -= ((L(ix - 1, iy, 0) + L(ix + 1, iy, 0)) + (L(ix, iy - 1, 0) + L(ix, iy + 1, 0))) -
                                  4.0 * L(ix, iy, 0);
        for (int face = 0; face < 4; ++face) {
          if (nbs[b][face].kind != COARSE && nbs[b][face].kind != FINE) continue;
          for (int k = 0; k < BS; ++k) {
            const bool xface = face < 2;
            const int ix = xface ? (face == 0 ? 0 : BS - 1) : k;
            const int iy = xface ? k : (face == 2 ? 0 : BS - 1);
            const int gx = ix + (face == 0 ? -1 : face == 1 ? 1 : 0);
            const int gy = iy + (face == 2 ? -1 : face == 3 ? 1 : 0);
            S(b, face, k, 0) = L(gx, gy, 0) - L(ix, iy, 0);
          }
        }
      }
      correct(F, nbs, S, tmp, 1);
    }
    return 0;
  } catch (const std::exception&) {
    return -1;
  }
}

// PressureSingle::pressureCorrection (:191-210): vel += tmpV / h^2.
int oracle_pressure_correction(const oracle_forest* fp, double dt, const double* pres, double* vel) {
  try {
    const Forest F(*fp);
    const int64_t nb = fp->nblocks;
    std::vector<std::array<Nei, 4>> nbs(nb);
    for (int64_t b = 0; b < nb; ++b)
      for (int face = 0; face < 4; ++face) nbs[b][face] = neighbour(F, b, face);
    const Field P{pres, 1};
    std::vector<double> tmpV(nb * 64 * 2, 0.0);
    Stored S{std::vector<Faces>(nb, Faces(4 * BS * 2, 0.0)), 2};
    for (int64_t b = 0; b < nb; ++b) {
      Lab L;
      fill_lab(F, P, false, b, nbs[b].data(), L);
      const double h = F.h(b), pFac = -0.5 * dt * h;
      for (int iy = 0; iy < BS; ++iy)
        for (int ix = 0; ix < BS; ++ix) {
          tmpV[at(b, ix, iy) * 2 + 0] = pFac * (L(ix + 1, iy, 0) - L(ix - 1, iy, 0));
          tmpV[at(b, ix, iy) * 2 + 1] = pFac * (L(ix, iy + 1, 0) - L(ix, iy - 1, 0));
        }
      for (int face = 0; face < 4; ++face) {
        if (nbs[b][face].kind != COARSE && nbs[b][face].kind != FINE) continue;
        for (int k = 0; k < BS; ++k) {
          const bool xface = face < 2;
          const int ix = xface ? (face == 0 ? 0 : BS - 1) : k;
          const int iy = xface ? k : (face == 2 ? 0 : BS - 1);
          const int gx = ix + (face == 0 ? -1 : face == 1 ? 1 : 0);
          const int gy = iy + (face == 2 ? -1 : face == 3 ? 1 : 0);
          const int c = xface ? 0 : 1;
          S(b, face, k, 0) = 0.0;  // clear()
          S(b, face, k, 1) = 0.0;
          S(b, face, k, c) = (face == 0 || face == 2 ? pFac : -pFac) * (L(gx, gy, 0) + L(ix, iy, 0));
        }
      }
    }
    correct(F, nbs, S, tmpV.data(), 2);
    for (int64_t b = 0; b < nb; ++b) {
      const double ih2 = 1.0 / F.h(b) / F.h(b);
      for (int i = 0; i < 64; ++i) {
        vel[(b * 64 + i) * 2 + 0] += tmpV[(b * 64 + i) * 2 + 0] * ih2;
        vel[(b * 64 + i) * 2 + 1] += tmpV[(b * 64 + i) * 2 + 1] * ih2;
      }
    }
    return 0;
  } catch (const std::exception&) {
    return -1;
  }
}

}  // extern "C"
