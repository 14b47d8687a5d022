// ORACLE — test infrastructure only.  CPU FP64 restatement of CUP2D's GPU
// Poisson path, used as the reference of the parity tests and as the timed CPU baseline.
// Nothing in the product library links, loads or calls this file.
//
// What it restates (paths relative to the CUP2D source tree):
//   * P^-1 construction: ExpAMRSolver::getA_local + constructor,
//     source/Poisson/ExpAMRSolver.cpp:11-99 (Cholesky-Crout of the 64x64
//     block Laplacian K, Gauss-Jordan inverse of L, P^-1 = -(L^T)^-1 L^-1).
//   * Matrix assembly: ExpAMRSolver::getMat / makeFlux / interpolate,
//     ExpAMRSolver.cpp:100-313, with the index maps and Taylor stencils of
//     ExpAMRSolver.h:69-300 (CellIndexer, X/Y{min,max}Indexer, D1, D2).
//   * Row accumulation: SpRowInfo::mapColVal (LocalSpMatDnVec.h:25-38):
//     duplicate columns summed in call order, columns emitted in ascending
//     order (std::map); interior rows pushed as 5 COO entries
//     (ExpAMRSolver.cpp:270-277).
//   * Solver: BiCGSTABSolver::main, source/Poisson/BiCGSTAB.cu:412-620 —
//     right-preconditioned BiCGSTAB, eps = 1e-21, restart on
//     rho^2 < 1e-16 |r|^2 |rhat|^2, best iterate x_opt by L-inf residual,
//     stop at |r|_inf <= abs or |r|_inf/|r0|_inf <= rel, 1000-iteration cap;
//     with bMeanConstraint, the SpMV's mean row replaced by sum h^2 x
//     (BiCGSTAB.cu:393-410).
//   * Mean removal: ExpAMRSolver::solve, ExpAMRSolver.cpp:383-415.
//
// Cubism (the AMR grid library of CUP2D) is an un-vendored submodule, so its
// neighbour queries are restated from their use in getMat: a face neighbour
// at the same level Exists, or the parent-level block covering it is a leaf
// (CheckCoarser), or it is refined (CheckFiner).  Block order is the caller's;
// blockOffset(info) = blockID * 64 on one rank.
//
// Parity pinning: the reference ships no golden vectors or tests for this
// path, so its own code is built and run instead (oracle/ref: ExpAMRSolver.cpp,
// LocalSpMatDnVec.cpp and BiCGSTAB.cu compiled unchanged against a Cubism
// stand-in and a one-rank MPI stand-in).  P^-1 and the assembled system are
// bit-identical to the reference's (tests/golden/ref_assembly.json holds
// SHA-256 digests of its COO bytes on 13 meshes; tests/test_ref_pin.py also
// compares random forests live); the solver stage matches the reference's
// cuBLAS/cuSPARSE solve run on a B200 (tests/golden/ref_solve_*.npz) to rel.
// L2 1e-6 at rel. residual 1e-8, and stops at the same 1000-iteration cap.
// Analytic known-answer tests (row and column sums, uniform-mesh 5-point
// matrix, quadratic exactness, P^-1 K = -I) remain in tests/test_oracle_kat.py.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <map>
#include <stdexcept>
#include <unordered_map>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

extern "C" {

typedef struct oracle_forest {
  int32_t bpdx, bpdy, level_max, periodic_x, periodic_y;
  double extent;
  int64_t nblocks;
  const int32_t* level;
  const int32_t* bx;
  const int32_t* by;
} oracle_forest;

typedef struct oracle_stats {
  int32_t iterations;   // completed BiCGSTAB iterations (p-update..r-update)
  int32_t restarts;
  int32_t converged;
  int32_t hit_max_iter;
  double err_init;      // |b - A x0|_inf
  double err_opt;       // best |r|_inf
  double norm_ax0;      // |A x0|_inf
} oracle_stats;
}

namespace {

constexpr int BSX = 8, BSY = 8, BLEN = 64;

// ------------------------------------------------------------------ P^-1 ---

double getA_local(int I1, int I2) {  // ExpAMRSolver.cpp:11-23
  const int j1 = I1 / BSX, i1 = I1 % BSX, j2 = I2 / BSX, i2 = I2 % BSX;
  if (i1 == i2 && j1 == j2) return 4.0;
  if (std::abs(i1 - i2) + std::abs(j1 - j2) == 1) return -1.0;
  return 0.0;
}

void build_pinv(double* P) {  // ExpAMRSolver.cpp:37-95
  std::vector<std::vector<double>> L(BLEN), Li(BLEN);
  for (int i = 0; i < BLEN; i++) {
    L[i].assign(i + 1, 0.0);
    Li[i].assign(i + 1, 0.0);
    for (int j = 0; j <= i; j++) Li[i][j] = (i == j) ? 1. : 0.;
  }
  for (int i = 0; i < BLEN; i++) {  // Cholesky-Crout
    double s1 = 0;
    for (int k = 0; k <= i - 1; k++) s1 += L[i][k] * L[i][k];
    L[i][i] = std::sqrt(getA_local(i, i) - s1);
    for (int j = i + 1; j < BLEN; j++) {
      double s2 = 0;
      for (int k = 0; k <= i - 1; k++) s2 += L[i][k] * L[j][k];
      L[j][i] = (getA_local(j, i) - s2) / L[i][i];
    }
  }
  for (int br = 0; br < BLEN; br++) {  // Gauss-Jordan on [L | I]
    const double bsf = 1. / L[br][br];
    for (int c = 0; c <= br; c++) Li[br][c] *= bsf;
    for (int wr = br + 1; wr < BLEN; wr++) {
      const double wsf = L[wr][br];
      for (int c = 0; c <= br; c++) Li[wr][c] -= (wsf * Li[br][c]);
    }
  }
  for (int i = 0; i < BLEN; i++)
    for (int j = 0; j < BLEN; j++) {
      double aux = 0.;
      for (int k = 0; k < BLEN; k++)
        aux += (i <= k && j <= k) ? Li[k][i] * Li[k][j] : 0.;
      P[i * BLEN + j] = -aux;
    }
}

// -------------------------------------------------------------- forest -----

struct BInfo {
  int level;
  int64_t i, j;
  int64_t id;
};

struct Tree {
  const oracle_forest& f;
  std::vector<std::unordered_map<uint64_t, int64_t>> lv;
  explicit Tree(const oracle_forest& ff) : f(ff), lv(ff.level_max) {
    for (int64_t b = 0; b < f.nblocks; ++b)
      lv[f.level[b]][key(f.bx[b], f.by[b])] = b;
  }
  static uint64_t key(int64_t i, int64_t j) { return ((uint64_t)i << 32) | (uint64_t)(uint32_t)j; }
  int64_t find(int l, int64_t i, int64_t j) const {
    if (l < 0 || l >= f.level_max) return -1;
    auto it = lv[l].find(key(i, j));
    return it == lv[l].end() ? -1 : it->second;
  }
  int64_t nx(int l) const { return (int64_t)f.bpdx << l; }
  int64_t ny(int l) const { return (int64_t)f.bpdy << l; }
};

// --------------------------------------------------------- row builder -----

struct Row {  // SpRowInfo (single rank): std::map col -> accumulated value
  std::map<int64_t, double> cv;
  void map(int64_t c, double v) { cv[c] += v; }
};

inline int64_t This(int64_t blk, int ix, int iy) { return blk * BLEN + (int64_t)(iy * BSX + ix); }
inline int64_t Xmin(int64_t blk, int ix, int iy, int off = 0) { (void)ix; return blk * BLEN + (iy * BSX + off); }
inline int64_t Xmax(int64_t blk, int ix, int iy, int off = 0) { (void)ix; return blk * BLEN + (iy * BSX + (BSX - 1 - off)); }
inline int64_t Ymin(int64_t blk, int ix, int iy, int off = 0) { (void)iy; return blk * BLEN + (off * BSX + ix); }
inline int64_t Ymax(int64_t blk, int ix, int iy, int off = 0) { (void)iy; return blk * BLEN + ((BSY - 1 - off) * BSX + ix); }
inline int ix_f(int ix) { return (ix % (BSX / 2)) * 2; }
inline int iy_f(int iy) { return (iy % (BSY / 2)) * 2; }

// Face indexers (ExpAMRSolver.h:150-258); face 0 Xm, 1 Xp, 2 Ym, 3 Yp.
struct Indexer {
  int face;
  bool xbase() const { return face < 2; }
  double taylorSign(int ix, int iy) const {
    return xbase() ? (iy % 2 == 0 ? -1. : 1.) : (ix % 2 == 0 ? -1. : 1.);
  }
  bool isBD(int ix, int iy) const {
    return xbase() ? (iy == BSY - 1 || iy == BSY / 2 - 1) : (ix == BSX - 1 || ix == BSX / 2 - 1);
  }
  bool isFD(int ix, int iy) const {
    return xbase() ? (iy == 0 || iy == BSY / 2) : (ix == 0 || ix == BSX / 2);
  }
  int64_t Nei(int64_t blk, int ix, int iy, int dist) const {
    return xbase() ? This(blk, ix, iy + dist) : This(blk, ix + dist, iy);
  }
  int64_t neiUnif(int64_t nblk, int ix, int iy) const {
    switch (face) {
      case 0: return Xmax(nblk, ix, iy);
      case 1: return Xmin(nblk, ix, iy);
      case 2: return Ymax(nblk, ix, iy);
      default: return Ymin(nblk, ix, iy);
    }
  }
  int64_t neiInward(int64_t blk, int ix, int iy) const {
    switch (face) {
      case 0: return This(blk, ix + 1, iy);
      case 1: return This(blk, ix - 1, iy);
      case 2: return This(blk, ix, iy + 1);
      default: return This(blk, ix, iy - 1);
    }
  }
  // index[] of the fine block decides which half of the coarse block
  int ix_c(int64_t fine_bx, int ix) const {
    if (face == 0) return BSX - 1;
    if (face == 1) return 0;
    return fine_bx % 2 == 0 ? ix / 2 : ix / 2 + BSX / 2;
  }
  int iy_c(int64_t fine_by, int iy) const {
    if (face == 2) return BSY - 1;
    if (face == 3) return 0;
    return fine_by % 2 == 0 ? iy / 2 : iy / 2 + BSY / 2;
  }
  int64_t neiFine1(int64_t nblk, int ix, int iy, int off) const {
    switch (face) {
      case 0: return Xmax(nblk, ix_f(ix), iy_f(iy), off);
      case 1: return Xmin(nblk, ix_f(ix), iy_f(iy), off);
      case 2: return Ymax(nblk, ix_f(ix), iy_f(iy), off);
      default: return Ymin(nblk, ix_f(ix), iy_f(iy), off);
    }
  }
  int64_t neiFine2(int64_t nblk, int ix, int iy, int off) const {
    switch (face) {
      case 0: return Xmax(nblk, ix_f(ix), iy_f(iy) + 1, off);
      case 1: return Xmin(nblk, ix_f(ix), iy_f(iy) + 1, off);
      case 2: return Ymax(nblk, ix_f(ix) + 1, iy_f(iy), off);
      default: return Ymin(nblk, ix_f(ix) + 1, iy_f(iy), off);
    }
  }
  // Zchild[a][b][0] = child (2*ni + a, 2*nj + b) of the same-level
  // neighbour position (ni, nj)
  void zchild(int64_t ni, int64_t nj, int ix, int iy, int64_t& ci, int64_t& cj) const {
    switch (face) {
      case 0: ci = 2 * ni + 1; cj = 2 * nj + (iy >= BSY / 2); break;
      case 1: ci = 2 * ni + 0; cj = 2 * nj + (iy >= BSY / 2); break;
      case 2: ci = 2 * ni + (ix >= BSX / 2); cj = 2 * nj + 1; break;
      default: ci = 2 * ni + (ix >= BSX / 2); cj = 2 * nj + 0; break;
    }
  }
};

struct Assembler {
  const oracle_forest& f;
  Tree tree;
  explicit Assembler(const oracle_forest& ff) : f(ff), tree(ff) {}

  // D1, D2 (ExpAMRSolver.h:268-300)
  void D1(int64_t blk, const Indexer& ind, int ix, int iy, int64_t c[3], double w[3]) const {
    if (ind.isBD(ix, iy)) {
      c[0] = ind.Nei(blk, ix, iy, -2); w[0] = 1. / 8.;
      c[1] = ind.Nei(blk, ix, iy, -1); w[1] = -1. / 2.;
      c[2] = This(blk, ix, iy);        w[2] = 3. / 8.;
    } else if (ind.isFD(ix, iy)) {
      c[0] = ind.Nei(blk, ix, iy, 2);  w[0] = -1. / 8.;
      c[1] = ind.Nei(blk, ix, iy, 1);  w[1] = 1. / 2.;
      c[2] = This(blk, ix, iy);        w[2] = -3. / 8.;
    } else {
      c[0] = ind.Nei(blk, ix, iy, -1); w[0] = -1. / 8.;
      c[1] = ind.Nei(blk, ix, iy, 1);  w[1] = 1. / 8.;
      c[2] = This(blk, ix, iy);        w[2] = 0.;
    }
  }
  void D2(int64_t blk, const Indexer& ind, int ix, int iy, int64_t c[3], double w[3]) const {
    if (ind.isBD(ix, iy)) {
      c[0] = ind.Nei(blk, ix, iy, -2); w[0] = 1. / 32.;
      c[1] = ind.Nei(blk, ix, iy, -1); w[1] = -1. / 16.;
      c[2] = This(blk, ix, iy);        w[2] = 1. / 32.;
    } else if (ind.isFD(ix, iy)) {
      c[0] = ind.Nei(blk, ix, iy, 2);  w[0] = 1. / 32.;
      c[1] = ind.Nei(blk, ix, iy, 1);  w[1] = -1. / 16.;
      c[2] = This(blk, ix, iy);        w[2] = 1. / 32.;
    } else {
      c[0] = ind.Nei(blk, ix, iy, -1); w[0] = 1. / 32.;
      c[1] = ind.Nei(blk, ix, iy, 1);  w[1] = 1. / 32.;
      c[2] = This(blk, ix, iy);        w[2] = -1. / 16.;
    }
  }

  // ExpAMRSolver::interpolate, ExpAMRSolver.cpp:100-128
  void interpolate(int64_t blk_c, int ix_c, int iy_c, int64_t fine_close,
                   int64_t fine_far, double signInt, double signTaylor,
                   const Indexer& ind, Row& row) const {
    row.map(fine_close, signInt * 2. / 3.);
    row.map(fine_far, -signInt * 1. / 5.);
    const double tf = signInt * 8. / 15.;
    row.map(This(blk_c, ix_c, iy_c), tf);
    int64_t c[3];
    double w[3];
    D1(blk_c, ind, ix_c, iy_c, c, w);
    for (int i = 0; i < 3; i++) row.map(c[i], signTaylor * tf * w[i]);
    D2(blk_c, ind, ix_c, iy_c, c, w);
    for (int i = 0; i < 3; i++) row.map(c[i], tf * w[i]);
  }

  // neighbour position across `face` at the same level (periodic wrap)
  void nei_pos(const BInfo& b, int face, int64_t& ni, int64_t& nj) const {
    ni = b.i + (face == 0 ? -1 : face == 1 ? 1 : 0);
    nj = b.j + (face == 2 ? -1 : face == 3 ? 1 : 0);
    const int64_t nx = tree.nx(b.level), ny = tree.ny(b.level);
    ni = (ni % nx + nx) % nx;
    nj = (nj % ny + ny) % ny;
  }

  // ExpAMRSolver::makeFlux, ExpAMRSolver.cpp:131-178
  void makeFlux(const BInfo& b, int ix, int iy, int face, const Indexer& ind, Row& row) const {
    const int64_t sfc = This(b.id, ix, iy);
    int64_t ni, nj;
    nei_pos(b, face, ni, nj);
    const int64_t same = tree.find(b.level, ni, nj);
    if (same >= 0) {  // Exists()
      row.map(ind.neiUnif(same, ix, iy), 1.);
      row.map(sfc, -1.);
      return;
    }
    const int64_t coarse = tree.find(b.level - 1, ni / 2, nj / 2);
    if (coarse >= 0) {  // CheckCoarser(): Zparent of the neighbour position
      const int ixc = ind.ix_c(b.i, ix);
      const int iyc = ind.iy_c(b.j, iy);
      const int64_t inward = ind.neiInward(b.id, ix, iy);
      const double st = ind.taylorSign(ix, iy);
      interpolate(coarse, ixc, iyc, sfc, inward, 1., st, ind, row);
      row.map(sfc, -1.);
      return;
    }
    int64_t ci, cj;
    ind.zchild(ni, nj, ix, iy, ci, cj);
    const int64_t fine = tree.find(b.level + 1, ci, cj);
    if (fine >= 0) {  // CheckFiner()
      int64_t close = ind.neiFine1(fine, ix, iy, 0), far = ind.neiFine1(fine, ix, iy, 1);
      row.map(close, 1.);
      interpolate(b.id, ix, iy, close, far, -1., -1., ind, row);
      close = ind.neiFine2(fine, ix, iy, 0);
      far = ind.neiFine2(fine, ix, iy, 1);
      row.map(close, 1.);
      interpolate(b.id, ix, iy, close, far, -1., 1., ind, row);
      return;
    }
    throw std::runtime_error("Neighbour doesn't exist, isn't coarser, nor finer...");
  }

  // ExpAMRSolver::getMat, ExpAMRSolver.cpp:180-313 (CSR output)
  void getMat(std::vector<int64_t>& rp, std::vector<int32_t>& col, std::vector<double>& val) const {
    const int64_t nb = f.nblocks;
    rp.assign(nb * BLEN + 1, 0);
    col.clear();
    val.clear();
    col.reserve(6 * nb * BLEN);
    val.reserve(6 * nb * BLEN);
    const Indexer idx[4] = {{0}, {1}, {2}, {3}};
    for (int64_t blk = 0; blk < nb; ++blk) {
      const BInfo b{f.level[blk], f.bx[blk], f.by[blk], blk};
      const int64_t MAXX = tree.nx(b.level) - 1, MAXY = tree.ny(b.level) - 1;
      const bool isBoundary[4] = {b.i == 0, b.i == MAXX, b.j == 0, b.j == MAXY};
      const bool isPeriodic[2] = {f.periodic_x != 0, f.periodic_y != 0};
      for (int iy = 0; iy < BSY; iy++)
        for (int ix = 0; ix < BSX; ix++) {
          const int64_t sfc = This(blk, ix, iy);
          if ((ix > 0 && ix < BSX - 1) && (iy > 0 && iy < BSY - 1)) {
            const int64_t cs[5] = {This(blk, ix, iy - 1), This(blk, ix - 1, iy), sfc,
                                   This(blk, ix + 1, iy), This(blk, ix, iy + 1)};
            const double vs[5] = {1, 1, -4, 1, 1};
            for (int q = 0; q < 5; ++q) {
              col.push_back((int32_t)cs[q]);
              val.push_back(vs[q]);
            }
          } else {
            const bool validNei[4] = {ix > 0, ix < BSX - 1, iy > 0, iy < BSY - 1};
            const int64_t idxNei[4] = {This(blk, ix - 1, iy), This(blk, ix + 1, iy),
                                       This(blk, ix, iy - 1), This(blk, ix, iy + 1)};
            Row row;
            for (int j = 0; j < 4; j++) {
              if (validNei[j]) {
                row.map(idxNei[j], 1);
                row.map(sfc, -1);
              } else if (!isBoundary[j] || (isBoundary[j] && isPeriodic[j / 2])) {
                makeFlux(b, ix, iy, j, idx[j], row);
              }
            }
            for (const auto& kv : row.cv) {
              col.push_back((int32_t)kv.first);
              val.push_back(kv.second);
            }
          }
          rp[sfc + 1] = (int64_t)col.size();
        }
    }
  }
};

struct Csr {
  int64_t n = 0;
  std::vector<int64_t> rp;
  std::vector<int32_t> col;
  std::vector<double> val;
};

void spmv(const Csr& A, const double* x, double* y) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < A.n; ++i) {
    double s = 0.0;
    for (int64_t k = A.rp[i]; k < A.rp[i + 1]; ++k) s += A.val[k] * x[A.col[k]];
    y[i] = s;
  }
}

double dot(int64_t n, const double* a, const double* b) {
  double s = 0.0;
#pragma omp parallel for reduction(+ : s) schedule(static)
  for (int64_t i = 0; i < n; ++i) s += a[i] * b[i];
  return s;
}

double amax(int64_t n, const double* a) {
  double m = 0.0;
#pragma omp parallel for reduction(max : m) schedule(static)
  for (int64_t i = 0; i < n; ++i) m = std::max(m, std::fabs(a[i]));
  return m;
}

// z = P^-1 p per block (cublasDgemm(T,N,64,Nb,64) with row-major P_inv,
// BiCGSTAB.cu:520,545): z[b*64+i] = sum_j P[i*64+j] p[b*64+j]
void precond(int64_t nb, const double* P, const double* p, double* z) {
#pragma omp parallel for schedule(static)
  for (int64_t b = 0; b < nb; ++b)
    for (int i = 0; i < BLEN; ++i) {
      double s = 0.0;
      for (int j = 0; j < BLEN; ++j) s += P[i * BLEN + j] * p[b * BLEN + j];
      z[b * BLEN + i] = s;
    }
}

// bMeanConstraint (BiCGSTAB.cu:393-410): after the SpMV, row mean_row of the
// result holds sum_i h_i^2 op_i over the operand (blockDscal then a sum).
struct MeanRow {
  int64_t row = -1;
  const double* h_block = nullptr;
};

void spmv_mean(const Csr& A, const MeanRow& mr, const double* x, double* y) {
  spmv(A, x, y);
  if (mr.row < 0) return;
  double s = 0.0;
  for (int64_t i = 0; i < A.n; ++i) s += (mr.h_block[i / BLEN] * mr.h_block[i / BLEN]) * x[i];
  y[mr.row] = s;
}

// BiCGSTABSolver::main, BiCGSTAB.cu:412-620 (single rank); with mr.row >= 0
// the bMeanConstraint SpMV (b already holds 0 in that row, as getVec leaves it)
void bicgstab(const Csr& A, const double* P, const double* b, double* x,
              double max_error, double max_rel_error, int max_restarts,
              int max_iter, oracle_stats* st, const MeanRow& mr = MeanRow{}) {
  const int64_t m = A.n, nb = m / BLEN;
  std::vector<double> r(b, b + m), rhat(m), p(m, 0.0), nu(m, 0.0), t(m), z(m), xopt(m);
  double alpha = 1., beta = 1., omega = 1., eps = 1e-21, rho_prev = 1., rho_curr = 1.;
  (void)beta;
  double error = 1e50, error_init = 1e50, error_opt = 1e50;
  bool bConverged = false;
  int restarts = 0;

  spmv_mean(A, mr, x, nu.data());                          // nu = A x0
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < m; ++i) r[i] = b[i] - nu[i];     // r = b - A x0
  const double nax0 = amax(m, nu.data());
  error = amax(m, r.data());
  error_init = error;
  error_opt = error;
  std::copy(x, x + m, xopt.begin());
  rhat = r;
  std::fill(nu.begin(), nu.end(), 0.0);
  std::fill(p.begin(), p.end(), 0.0);

  int k = 0;
  bool hit_cap = true;
  for (k = 0; k < max_iter; k++) {
    rho_curr = dot(m, rhat.data(), r.data());
    const double n1 = dot(m, r.data(), r.data());
    const double n2 = dot(m, rhat.data(), rhat.data());
    const bool serious_breakdown = rho_curr * rho_curr < 1e-16 * n1 * n2;
    beta = (rho_curr / (rho_prev + eps)) * (alpha / (omega + eps));
    if (serious_breakdown && max_restarts > 0) {
      restarts++;
      if (restarts >= max_restarts) { hit_cap = false; break; }
      rhat = r;
      rho_curr = dot(m, rhat.data(), rhat.data());
      std::fill(nu.begin(), nu.end(), 0.0);
      std::fill(p.begin(), p.end(), 0.0);
      rho_prev = 1.;
      alpha = 1.;
      omega = 1.;
      beta = (rho_curr / (rho_prev + eps)) * (alpha / (omega + eps));
    }
    // p = r + beta (p - omega nu)
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < m; ++i) p[i] = r[i] + beta * (p[i] - omega * nu[i]);
    precond(nb, P, p.data(), z.data());
    spmv_mean(A, mr, z.data(), nu.data());
    const double rn = dot(m, rhat.data(), nu.data());
    alpha = rho_curr / (rn + eps);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < m; ++i) {
      x[i] += alpha * z[i];
      r[i] -= alpha * nu[i];  // s
    }
    precond(nb, P, r.data(), z.data());
    spmv_mean(A, mr, z.data(), t.data());
    const double ts = dot(m, t.data(), r.data());
    const double tt = dot(m, t.data(), t.data());
    omega = ts / (tt + eps);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < m; ++i) {
      x[i] += omega * z[i];
      r[i] -= omega * t[i];
    }
    error = amax(m, r.data());
    if (error < error_opt) {
      error_opt = error;
      std::copy(x, x + m, xopt.begin());
      if ((error <= max_error) || (error / error_init <= max_rel_error)) {
        bConverged = true;
        hit_cap = false;
        ++k;  // this iteration completed
        break;
      }
    }
    rho_prev = rho_curr;
  }
  std::copy(xopt.begin(), xopt.end(), x);
  if (st) {
    st->iterations = k;
    st->restarts = restarts;
    st->converged = bConverged ? 1 : 0;
    st->hit_max_iter = hit_cap ? 1 : 0;
    st->err_init = error_init;
    st->err_opt = error_opt;
    st->norm_ax0 = nax0;
  }
}

}  // namespace

// ------------------------------------------------------------- C ABI -------
extern "C" {

struct oracle_matrix {
  Csr A;
};

int oracle_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

void oracle_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

void oracle_pinv(double* P) { build_pinv(P); }

// Returns nullptr (and writes a message to stderr) on a malformed forest.
oracle_matrix* oracle_assemble(const oracle_forest* f) {
  try {
    auto* M = new oracle_matrix();
    Assembler as(*f);
    as.getMat(M->A.rp, M->A.col, M->A.val);
    M->A.n = f->nblocks * BLEN;
    return M;
  } catch (const std::exception& e) {
    std::fprintf(stderr, "oracle_assemble: %s\n", e.what());
    return nullptr;
  }
}

int64_t oracle_matrix_n(const oracle_matrix* M) { return M->A.n; }
int64_t oracle_matrix_nnz(const oracle_matrix* M) { return (int64_t)M->A.val.size(); }

void oracle_matrix_copy(const oracle_matrix* M, int64_t* rp, int32_t* col, double* val) {
  std::memcpy(rp, M->A.rp.data(), sizeof(int64_t) * M->A.rp.size());
  std::memcpy(col, M->A.col.data(), sizeof(int32_t) * M->A.col.size());
  std::memcpy(val, M->A.val.data(), sizeof(double) * M->A.val.size());
}

void oracle_matrix_free(oracle_matrix* M) { delete M; }

void oracle_spmv(const oracle_matrix* M, const double* x, double* y) { spmv(M->A, x, y); }

void oracle_precond(int64_t nblocks, const double* P, const double* p, double* z) {
  precond(nblocks, P, p, z);
}

// Solve A x = b from the initial guess in x (overwritten with x_opt).
int oracle_bicgstab(const oracle_matrix* M, const double* P, const double* b, double* x,
                    double max_error, double max_rel_error, int max_restarts,
                    int max_iter, oracle_stats* st) {
  bicgstab(M->A, P, b, x, max_error, max_rel_error, max_restarts, max_iter, st);
  return 0;
}

// The same with bMeanConstraint: row mean_row is sum(h^2 x) (h per block).
int oracle_bicgstab_mean(const oracle_matrix* M, const double* P, const double* b, double* x,
                         double max_error, double max_rel_error, int max_restarts, int max_iter,
                         int64_t mean_row, const double* h_block, oracle_stats* st) {
  MeanRow mr;
  mr.row = mean_row;
  mr.h_block = h_block;
  bicgstab(M->A, P, b, x, max_error, max_rel_error, max_restarts, max_iter, st, mr);
  return 0;
}

// ExpAMRSolver.cpp:383-415: x -= sum(h^2 x) / sum(h^2), h per block
void oracle_subtract_mean(int64_t nblocks, const double* h_block, double* x) {
  double avg = 0, avg1 = 0;
#pragma omp parallel for reduction(+ : avg, avg1) schedule(static)
  for (int64_t i = 0; i < nblocks; ++i) {
    const double vv = h_block[i] * h_block[i];
    for (int c = 0; c < BLEN; ++c) {
      avg += x[i * BLEN + c] * vv;
      avg1 += vv;
    }
  }
  avg = avg / avg1;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < nblocks * BLEN; ++i) x[i] += -avg;
}

}  // extern "C"
