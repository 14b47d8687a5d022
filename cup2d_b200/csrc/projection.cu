// The pressure projection around the Poisson solve, on the device.
//
// CUP2D's PressureSingle (source/Operators/PressureSingle.cpp) runs three
// field kernels on Cubism block labs (the block plus one ghost layer), each
// followed by Cubism's flux correction on coarse/fine faces:
//   updatePressureRHS  (:324-397)  TMP = facDiv ((u_E - u_W) + (v_N - v_S))
//                                       + (-facDiv CHI) ((ud_E - ud_W) + (vd_N - vd_S)),
//                                  facDiv = 0.5 h / dt
//   updatePressureRHS1 (:399-456)  TMP -= ((p_W + p_E) + (p_S + p_N)) - 4 p
//   pressureCorrection (:123-210)  tmpV = pFac (P_E - P_W, P_N - P_S),
//                                  pFac = -0.5 dt h; V += tmpV (1/h)/h
// Here one thread owns one cell and evaluates its formula in the same order,
// reading its ghosts straight from the neighbouring blocks:
//   * same-level neighbour: the touching cell;
//   * non-periodic domain edge: velocities flip the sign of the normal
//     component (BlockLabDirichlet, source/Definitions.h:71-196, wall and
//     free-space alike), scalars copy the edge cell (BlockLabNeumann,
//     :200-228);
//   * coarser neighbour: the quadratic interpolation ExpAMRSolver uses for
//     the same cells when it assembles the operator (ExpAMRSolver.cpp:100-128
//     with D1/D2 of ExpAMRSolver.h:268-300), evaluated on values:
//     2/3 close - 1/5 far + 8/15 ((c + sT D1) + D2);
//   * finer neighbours: the mean of the four fine cells the ghost covers.
// The flux correction is folded into the coarse cell's own thread: after its
// formula it adds its own face value (the kernel's storedFace expression with
// that ghost) plus the two fine cells' face values (the same expression from
// the fine side, with their interpolated ghosts).  Cubism, which owns the labs
// and the correction, is an un-vendored submodule of CUP2D; the rules above
// are its role restated from CUP2D's use of it.
//
// The file is compiled without FMA contraction so that every expression
// rounds like the plain IEEE evaluation of the CPU restatement.
//
// Memory: streaming, one pass; per cell the RHS reads vel, udef (16 B each),
// chi, pres (8 B each) and writes tmp, pold (8 B each); the correction reads
// pres (8 B) and updates vel (16 B + 16 B).  Neighbour reads hit L1/L2.
#include <cuda_runtime.h>

#include "kernels.hpp"

namespace cup2d {

namespace {

constexpr int kProjThreads = 256;  // 4 blocks of 64 cells per CTA
constexpr double kI23 = 2. / 3., kI15 = 1. / 5., kI815 = 8. / 15.;

enum : int { kSame = 0, kEdge = 1, kCoarser = 2, kFiner = 3 };

__device__ __forceinline__ int64_t cidx(int64_t blk, int ix, int iy) { return blk * kBLEN + iy * kBS + ix; }

// Cell of block nb across face f (0 W, 1 E, 2 S, 3 N), `d` cells deep, at the
// along-face position of (ix, iy).
__device__ __forceinline__ int64_t mirror(int f, int64_t nb, int ix, int iy, int d) {
  switch (f) {
    case 0: return cidx(nb, kBS - 1 - d, iy);
    case 1: return cidx(nb, d, iy);
    case 2: return cidx(nb, ix, kBS - 1 - d);
    default: return cidx(nb, ix, d);
  }
}

struct Side {
  int kind;
  int64_t blk;      // same-level or coarser block
  int64_t fine[2];  // finer blocks touching cells 0-3 / 4-7 of the face
};

struct Geo {
  ForestView F;
  const int32_t* __restrict__ nbr;

  __device__ int32_t leaf(int l, int64_t i, int64_t j) const {
    if (l < 0 || l >= F.L) return -1;
    return F.table[F.off[l] + j * ((int64_t)F.bpdx << l) + i];
  }

  __device__ Side side(int64_t b, int f) const {
    Side s{kEdge, -1, {-1, -1}};
    const int32_t code = nbr[4 * b + f];
    if (code >= 0) {
      s.kind = kSame;
      s.blk = code;
      return s;
    }
    if (code != kExplicit) return s;  // domain edge
    const int l = F.level[b];
    const int64_t nx = (int64_t)F.bpdx << l, ny = (int64_t)F.bpdy << l;
    const int64_t ni = ((int64_t)F.bx[b] + (f == 0 ? -1 : f == 1 ? 1 : 0) + nx) % nx;
    const int64_t nj = ((int64_t)F.by[b] + (f == 2 ? -1 : f == 3 ? 1 : 0) + ny) % ny;
    const int32_t c = leaf(l - 1, ni >> 1, nj >> 1);
    if (c >= 0) {
      s.kind = kCoarser;
      s.blk = c;
      return s;
    }
    for (int h = 0; h < 2; ++h) {
      int64_t ci, cj;
      switch (f) {
        case 0: ci = 2 * ni + 1; cj = 2 * nj + h; break;
        case 1: ci = 2 * ni; cj = 2 * nj + h; break;
        case 2: ci = 2 * ni + h; cj = 2 * nj + 1; break;
        default: ci = 2 * ni + h; cj = 2 * nj; break;
      }
      s.fine[h] = leaf(l + 1, ci, cj);
    }
    // assembly rejected forests with holes; keep every index valid anyway
    s.kind = (s.fine[0] >= 0 && s.fine[1] >= 0) ? kFiner : kEdge;
    return s;
  }
};

// A field with `nc` doubles per cell.
struct Fld {
  const double* __restrict__ p;
  int nc;
  __device__ __forceinline__ double v(int64_t cell, int c) const { return p[cell * nc + c]; }
};

// Ghost of a fine cell (value vclose, next inward cell vfar) from coarse cell
// (xc, yc) of block bc: ExpAMRSolver::interpolate on values.
__device__ double interp_ghost(const Fld& w, int c, int64_t bc, int xc, int yc, double vclose, double vfar, double sT,
                               bool xface) {
  const int t = xface ? yc : xc;
  auto cv = [&](int d) { return xface ? w.v(cidx(bc, xc, yc + d), c) : w.v(cidx(bc, xc + d, yc), c); };
  double v0, v1, a0, a1, a2, b0, b1, b2;
  const double v2 = cv(0);
  if (t == kBS - 1 || t == kBS / 2 - 1) {
    v0 = cv(-2); v1 = cv(-1);
    a0 = 1. / 8.; a1 = -1. / 2.; a2 = 3. / 8.;
    b0 = 1. / 32.; b1 = -1. / 16.; b2 = 1. / 32.;
  } else if (t == 0 || t == kBS / 2) {
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
  return (kI23 * vclose - kI15 * vfar) + kI815 * tay;
}

// One cell and its four faces.
struct CellCtx {
  const Geo& G;
  int64_t b, cell;
  int ix, iy, l;
  Side s[4];  // valid for the faces on the block edge
  __device__ bool on_edge(int f) const {
    return f == 0 ? ix == 0 : f == 1 ? ix == kBS - 1 : f == 2 ? iy == 0 : iy == kBS - 1;
  }
  __device__ int64_t inblock(int f) const {
    return cidx(b, ix + (f == 0 ? -1 : f == 1 ? 1 : 0), iy + (f == 2 ? -1 : f == 3 ? 1 : 0));
  }
  // fine block and the along-face position of the fine cells facing this cell
  __device__ void fine_cells(int f, int64_t& fb, int& k0) const {
    const bool xface = f < 2;
    fb = s[f].fine[xface ? (iy >= kBS / 2) : (ix >= kBS / 2)];
    k0 = ((xface ? iy : ix) % (kBS / 2)) * 2;
  }
  // fine cell q of face f (depth d), as a global cell index
  __device__ int64_t fine_cell(int f, int64_t fb, int k0, int q, int d) const {
    return f < 2 ? mirror(f, fb, 0, k0 + q, d) : mirror(f, fb, k0 + q, 0, d);
  }

  // Lab value of component c of field w across face f.
  __device__ double nb(const Fld& w, int c, int f, bool vector) const {
    if (!on_edge(f)) return w.v(inblock(f), c);
    const bool xface = f < 2;
    switch (s[f].kind) {
      case kSame:
        return w.v(mirror(f, s[f].blk, ix, iy, 0), c);
      case kEdge: {
        const double own = w.v(cell, c);
        return (vector && c == (xface ? 0 : 1)) ? -own : own;
      }
      case kCoarser: {
        const int64_t bx = G.F.bx[b], by = G.F.by[b];
        const int xc = f == 0 ? kBS - 1 : f == 1 ? 0 : (bx % 2 == 0 ? ix / 2 : ix / 2 + kBS / 2);
        const int yc = f == 2 ? kBS - 1 : f == 3 ? 0 : (by % 2 == 0 ? iy / 2 : iy / 2 + kBS / 2);
        const double sT = xface ? (iy % 2 == 0 ? -1. : 1.) : (ix % 2 == 0 ? -1. : 1.);
        const int64_t inward = cidx(b, ix + (f == 0 ? 1 : f == 1 ? -1 : 0), iy + (f == 2 ? 1 : f == 3 ? -1 : 0));
        return interp_ghost(w, c, s[f].blk, xc, yc, w.v(cell, c), w.v(inward, c), sT, xface);
      }
      default: {
        int64_t fb;
        int k0;
        fine_cells(f, fb, k0);
        const double s00 = w.v(fine_cell(f, fb, k0, 0, 0), c), s01 = w.v(fine_cell(f, fb, k0, 1, 0), c);
        const double s10 = w.v(fine_cell(f, fb, k0, 0, 1), c), s11 = w.v(fine_cell(f, fb, k0, 1, 1), c);
        return 0.25 * ((s00 + s01) + (s10 + s11));
      }
    }
  }

  // Ghost of fine cell q of finer face f (seen from the fine block), the
  // interpolation centred on this coarse cell.
  __device__ double fine_ghost(const Fld& w, int c, int f, int64_t fb, int k0, int q) const {
    return interp_ghost(w, c, b, ix, iy, w.v(fine_cell(f, fb, k0, q, 0), c), w.v(fine_cell(f, fb, k0, q, 1), c),
                        q == 0 ? -1. : 1., f < 2);
  }
};

__device__ __forceinline__ double cell_h(const ForestView& F, int l) { return F.h0 / (double)(1ll << l); }

// updatePressureRHS stored face value (PressureSingle.cpp:357-396) of face f
// of a cell: ghost (g, gd), own (w, wd), facDiv and CHI of that cell.
__device__ __forceinline__ double div_face(int f, double facDiv, double chi, double g, double w, double gd, double wd) {
  double s;
  if ((f & 1) == 0) {
    s = facDiv * (g + w);
    s += -(facDiv * chi) * (gd + wd);
  } else {
    s = -facDiv * (g + w);
    s -= -(facDiv * chi) * (gd + wd);
  }
  return s;
}

__global__ void __launch_bounds__(kProjThreads) k_pressure_rhs(Geo G, double dt, ProjFields P) {
  const int64_t cell = (int64_t)blockIdx.x * kProjThreads + threadIdx.x;
  if (cell >= G.F.nb * kBLEN) return;
  const int64_t b = cell >> 6;
  const int ci = (int)(cell & 63);
  CellCtx C{G, b, cell, ci & 7, ci >> 3, G.F.level[b], {}};
  for (int f = 0; f < 4; ++f)
    if (C.on_edge(f)) C.s[f] = G.side(b, f);
  const double h = cell_h(G.F, C.l);
  double t;
  if (P.vel) {
    const Fld V{P.vel, 2}, U{P.udef, 2};
    const double facDiv = 0.5 * h / dt;
    const double CHI = P.chi[cell];
    t = facDiv * ((C.nb(V, 0, 1, true) - C.nb(V, 0, 0, true)) + (C.nb(V, 1, 3, true) - C.nb(V, 1, 2, true)));
    t += -facDiv * CHI * ((C.nb(U, 0, 1, true) - C.nb(U, 0, 0, true)) + (C.nb(U, 1, 3, true) - C.nb(U, 1, 2, true)));
    for (int f = 0; f < 4; ++f) {
      if (!C.on_edge(f) || C.s[f].kind != kFiner) continue;
      const int c = f < 2 ? 0 : 1;
      const double own = div_face(f, facDiv, CHI, C.nb(V, c, f, true), V.v(cell, c), C.nb(U, c, f, true), U.v(cell, c));
      int64_t fb;
      int k0;
      C.fine_cells(f, fb, k0);
      const int lf = G.F.level[fb];
      const double facDivF = 0.5 * cell_h(G.F, lf) / dt;
      double fs[2];
      for (int q = 0; q < 2; ++q) {
        const int64_t fc = C.fine_cell(f, fb, k0, q, 0);
        fs[q] = div_face(f ^ 1, facDivF, P.chi[fc], C.fine_ghost(V, c, f, fb, k0, q), V.v(fc, c),
                         C.fine_ghost(U, c, f, fb, k0, q), U.v(fc, c));
      }
      t = t + (own + (fs[0] + fs[1]));
    }
  } else {
    t = P.tmp[cell];
  }
  if (P.pres) {
    const Fld Q{P.pres, 1};
    const double p0 = Q.v(cell, 0);
    t -= ((C.nb(Q, 0, 0, false) + C.nb(Q, 0, 1, false)) + (C.nb(Q, 0, 2, false) + C.nb(Q, 0, 3, false))) - 4.0 * p0;
    for (int f = 0; f < 4; ++f) {
      if (!C.on_edge(f) || C.s[f].kind != kFiner) continue;
      const double own = C.nb(Q, 0, f, false) - p0;
      int64_t fb;
      int k0;
      C.fine_cells(f, fb, k0);
      double fs[2];
      for (int q = 0; q < 2; ++q) fs[q] = C.fine_ghost(Q, 0, f, fb, k0, q) - Q.v(C.fine_cell(f, fb, k0, q, 0), 0);
      t = t + (own + (fs[0] + fs[1]));
    }
    P.pold[cell] = p0;
  }
  P.tmp[cell] = t;
}

// pressureCorrectionKernel stored face value (PressureSingle.cpp:152-185).
__device__ __forceinline__ double grad_face(int f, double pFac, double g, double w) {
  return ((f & 1) == 0 ? pFac : -pFac) * (g + w);
}

__global__ void __launch_bounds__(kProjThreads) k_pressure_correction(Geo G, double dt, const double* __restrict__ pres,
                                                                     double* __restrict__ vel) {
  const int64_t cell = (int64_t)blockIdx.x * kProjThreads + threadIdx.x;
  if (cell >= G.F.nb * kBLEN) return;
  const int64_t b = cell >> 6;
  const int ci = (int)(cell & 63);
  CellCtx C{G, b, cell, ci & 7, ci >> 3, G.F.level[b], {}};
  for (int f = 0; f < 4; ++f)
    if (C.on_edge(f)) C.s[f] = G.side(b, f);
  const Fld Q{pres, 1};
  const double h = cell_h(G.F, C.l);
  const double pFac = -0.5 * dt * h;
  const double p0 = Q.v(cell, 0);
  double tv[2];
  tv[0] = pFac * (C.nb(Q, 0, 1, false) - C.nb(Q, 0, 0, false));
  tv[1] = pFac * (C.nb(Q, 0, 3, false) - C.nb(Q, 0, 2, false));
  for (int f = 0; f < 4; ++f) {
    if (!C.on_edge(f) || C.s[f].kind != kFiner) continue;
    const double own = grad_face(f, pFac, C.nb(Q, 0, f, false), p0);
    int64_t fb;
    int k0;
    C.fine_cells(f, fb, k0);
    const double pFacF = -0.5 * dt * cell_h(G.F, G.F.level[fb]);
    double fs[2];
    for (int q = 0; q < 2; ++q)
      fs[q] = grad_face(f ^ 1, pFacF, C.fine_ghost(Q, 0, f, fb, k0, q), Q.v(C.fine_cell(f, fb, k0, q, 0), 0));
    tv[f < 2 ? 0 : 1] = tv[f < 2 ? 0 : 1] + (own + (fs[0] + fs[1]));
  }
  const double ih2 = 1.0 / h / h;
  vel[2 * cell] += tv[0] * ih2;
  vel[2 * cell + 1] += tv[1] * ih2;
}

}  // namespace

cudaError_t launch_pressure_rhs(const ForestView& F, const int32_t* nbr, double dt, const ProjFields& f,
                                cudaStream_t s) {
  const int64_t n = F.nb * kBLEN;
  if (n <= 0) return cudaSuccess;
  k_pressure_rhs<<<(unsigned)((n + kProjThreads - 1) / kProjThreads), kProjThreads, 0, s>>>(Geo{F, nbr}, dt, f);
  return cudaGetLastError();
}

cudaError_t launch_pressure_correction(const ForestView& F, const int32_t* nbr, double dt, const double* pres,
                                       double* vel, cudaStream_t s) {
  const int64_t n = F.nb * kBLEN;
  if (n <= 0) return cudaSuccess;
  k_pressure_correction<<<(unsigned)((n + kProjThreads - 1) / kProjThreads), kProjThreads, 0, s>>>(Geo{F, nbr}, dt,
                                                                                                  pres, vel);
  return cudaGetLastError();
}

}  // namespace cup2d
