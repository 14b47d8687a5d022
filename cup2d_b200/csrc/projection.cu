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

#include <algorithm>
#include <atomic>

#include "kernels.hpp"
#include "spmv.cuh"

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

  // The side of face f of block b from the face's neighbour table entry
  // (nbr[4 b + f], loaded ahead by the caller).
  __device__ Side side_from_code(int64_t b, int f, int32_t code) const {
    Side s{kEdge, -1, {-1, -1}};
    if (code >= 0) {
      s.kind = kSame;
      s.blk = code;
      return s;
    }
    if (code != kExplicit) return s;  // domain edge
    const int l = F.level[b];
    const int64_t nx = (int64_t)F.bpdx << l, ny = (int64_t)F.bpdy << l;
    int64_t ni = (int64_t)F.bx[b] + (f == 0 ? -1 : f == 1 ? 1 : 0);
    int64_t nj = (int64_t)F.by[b] + (f == 2 ? -1 : f == 3 ? 1 : 0);
    ni = ni < 0 ? ni + nx : ni >= nx ? ni - nx : ni;  // periodic wrap (one step at most)
    nj = nj < 0 ? nj + ny : nj >= ny ? nj - ny : nj;
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
__device__ __noinline__ double interp_ghost(const Fld& w, int c, int64_t bc, int xc, int yc, double vclose, double vfar, double sT,
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

// The ghost cell of one edge cell of block b across face f: one thread of the
// block's lab fill (thread g of the block: face g / 8, cell g % 8 along it).
struct Ghost {
  const Geo& G;
  int64_t b, cell;
  int ix, iy, f;
  Side s;

  // gi: the ghost's index in the block (face gi / 8); sd: the face's side,
  // looked up by the caller ahead of its other loads
  __device__ Ghost(const Geo& g, int64_t blk, int gi, const Side& sd) : G(g), b(blk), f(gi >> 3), s(sd) {
    const int k = gi & 7;
    ix = f == 0 ? 0 : f == 1 ? kBS - 1 : k;
    iy = f == 2 ? 0 : f == 3 ? kBS - 1 : k;
    cell = cidx(b, ix, iy);
  }
  __device__ bool xface() const { return f < 2; }
  // fine block and the along-face position of the fine cells facing this cell
  __device__ void fine_cells(int64_t& fb, int& k0) const {
    fb = s.fine[xface() ? (iy >= kBS / 2) : (ix >= kBS / 2)];
    k0 = ((xface() ? iy : ix) % (kBS / 2)) * 2;
  }
  // fine cell q (depth d), as a global cell index
  __device__ int64_t fine_cell(int64_t fb, int k0, int q, int d) const {
    return xface() ? mirror(f, fb, 0, k0 + q, d) : mirror(f, fb, k0 + q, 0, d);
  }
  // The lab value of component c of field w in the ghost cell.
  __device__ double value(const Fld& w, int c, bool vector) const {
    switch (s.kind) {
      case kSame:
        return w.v(mirror(f, s.blk, ix, iy, 0), c);
      case kEdge: {
        const double own = w.v(cell, c);
        return (vector && c == (xface() ? 0 : 1)) ? -own : own;
      }
      case kCoarser: {
        const int64_t bx = G.F.bx[b], by = G.F.by[b];
        const int xc = f == 0 ? kBS - 1 : f == 1 ? 0 : (bx % 2 == 0 ? ix / 2 : ix / 2 + kBS / 2);
        const int yc = f == 2 ? kBS - 1 : f == 3 ? 0 : (by % 2 == 0 ? iy / 2 : iy / 2 + kBS / 2);
        const double sT = xface() ? (iy % 2 == 0 ? -1. : 1.) : (ix % 2 == 0 ? -1. : 1.);
        const int64_t inward = cidx(b, ix + (f == 0 ? 1 : f == 1 ? -1 : 0), iy + (f == 2 ? 1 : f == 3 ? -1 : 0));
        return interp_ghost(w, c, s.blk, xc, yc, w.v(cell, c), w.v(inward, c), sT, xface());
      }
      default: {
        int64_t fb;
        int k0;
        fine_cells(fb, k0);
        const double s00 = w.v(fine_cell(fb, k0, 0, 0), c), s01 = w.v(fine_cell(fb, k0, 1, 0), c);
        const double s10 = w.v(fine_cell(fb, k0, 0, 1), c), s11 = w.v(fine_cell(fb, k0, 1, 1), c);
        return 0.25 * ((s00 + s01) + (s10 + s11));
      }
    }
  }
  // Ghost of fine cell q of a finer face (seen from the fine block), the
  // interpolation centred on this coarse cell.
  __device__ double fine_ghost(const Fld& w, int c, int64_t fb, int k0, int q) const {
    return interp_ghost(w, c, b, ix, iy, w.v(fine_cell(fb, k0, q, 0), c), w.v(fine_cell(fb, k0, q, 1), c),
                        q == 0 ? -1. : 1., xface());
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

// pressureCorrectionKernel stored face value (PressureSingle.cpp:152-185).
__device__ __forceinline__ double grad_face(int f, double pFac, double g, double w) {
  return ((f & 1) == 0 ? pFac : -pFac) * (g + w);
}

// Labs in shared memory: kLabBlocks blocks per CTA, 64 threads each.  Every
// thread stages its cell; 32 threads of each block then fill the ghost
// layer (the face neighbours, the edge rules, the coarse/fine rules) and, on
// faces with finer neighbours, the flux-correction terms; then every thread
// evaluates its cell from shared memory.  The stencil threads stay simple,
// the irregular work is confined to the ghost threads.
constexpr int kLabBlocks = kProjThreads / kBLEN;
constexpr int kLab = kBS + 2;
enum : int { kLabU = 0, kLabV = 1, kLabUd = 2, kLabVd = 3, kLabP = 4, kLabs = 5 };

struct ProjSmem {
  double lab[kLabs][kLabBlocks][kLab][kLab];
  double corr[2][kLabBlocks][4][kBS];  // finer faces: [0] divergence / gradient, [1] Laplacian
  int kind[kLabBlocks][4];
};

__device__ __forceinline__ double& labv(ProjSmem& S, int q, int lb, int ix, int iy) {
  return S.lab[q][lb][iy + 1][ix + 1];
}

// What one thread loads for its cell of a group of kLabBlocks blocks, one
// group ahead of the group it computes: the staged values and, for ghost
// threads, the face's neighbour table entry.  CTAs are persistent: each
// walks groups blockIdx.x, + gridDim.x, ..., so the loads of the next group
// are in flight while the ghost work and the stencil of the current one run.
struct Prefetch {
  double2 u, ud;
  double chi, p;
  int32_t code;
};

// The RHS kernel's labs, double-buffered: the next group's cells are copied
// in with cp.async (16-byte (u, v) pairs straight into shared memory, no
// registers held) while the current group is computed.
struct RhsSmem {
  double2 uv[2][kLabBlocks][kLab][kLab];  // (u, v); a face's ghost fills the normal component only
  double2 ud[2][kLabBlocks][kLab][kLab];  // (ud, vd)
  double p[2][kLabBlocks][kLab][kLab];
  double chi[2][kLabBlocks][kBLEN];
  double corr[2][kLabBlocks][4][kBS];     // finer faces: [0] divergence, [1] Laplacian
  int kind[kLabBlocks][4];
};

__global__ void __launch_bounds__(kProjThreads, 4) k_pressure_rhs(const __grid_constant__ Geo G, double dt,
                                                                    const __grid_constant__ ProjFields P) {
  __shared__ __align__(16) RhsSmem S;
  const int lb = threadIdx.x >> 6, c = threadIdx.x & 63, ix = c & 7, iy = c >> 3;
  const bool vel = P.vel != nullptr, pres = P.pres != nullptr;
  // ghost work: threads 0-31 of a block the velocity ghosts, 32-63 the
  // pressure ghosts (ghost index c % 32)
  const int gi = c & 31;
  const bool gvel = c < 32 && vel, gpres = c >= 32 && pres, gthr = gvel || gpres;
  const int64_t ngroups = (G.F.nb + kLabBlocks - 1) / kLabBlocks;
  // copies of group grp's cells into buffer q, and the face's table entry
  auto issue = [&](int64_t grp, int q, int32_t& code) {
    const int64_t b = grp * kLabBlocks + lb;
    if (b >= G.F.nb) return;
    const int64_t cell = b * kBLEN + c;
    if (vel) {
      cp_async_n<16>(&S.uv[q][lb][iy + 1][ix + 1], P.vel + 2 * cell, 16);
      cp_async_n<16>(&S.ud[q][lb][iy + 1][ix + 1], P.udef + 2 * cell, 16);
      cp_async_n<8>(&S.chi[q][lb][c], P.chi + cell, 8);
    }
    if (pres) cp_async_n<8>(&S.p[q][lb][iy + 1][ix + 1], P.pres + cell, 8);
    if (gthr) code = __ldg(G.nbr + 4 * b + (gi >> 3));
  };
  int32_t code = 0, code_next = 0;
  int64_t grp = blockIdx.x;
  if (grp < ngroups) issue(grp, 0, code);
  cp_async_commit_group();
  for (int it = 0; grp < ngroups; grp += gridDim.x, ++it) {
    const int q = it & 1;
    cp_async_wait_n<0>();  // this group's cells have landed (every thread's, after the barrier)
    __syncthreads();
    if (grp + gridDim.x < ngroups) issue(grp + gridDim.x, q ^ 1, code_next);
    cp_async_commit_group();
    const int64_t b = grp * kLabBlocks + lb;
    const bool valid = b < G.F.nb;
    const int64_t cell = b * kBLEN + c;
    // ghost layer and flux-correction terms
    if (valid && gthr) {
      const Ghost gh(G, b, gi, G.side_from_code(b, gi >> 3, code));
      const int k = gi & 7, f = gh.f;
      if (k == 0 && (c < 32 || !vel)) S.kind[lb][f] = gh.s.kind;
      const int gx = gh.ix + (f == 0 ? -1 : f == 1 ? 1 : 0), gy = gh.iy + (f == 2 ? -1 : f == 3 ? 1 : 0);
      const double h = cell_h(G.F, G.F.level[b]);
      if (gvel) {
        const Fld V{P.vel, 2}, U{P.udef, 2};
        const int cmp = gh.xface() ? 0 : 1;  // the normal component: the only one the divergence reads
        const double g = gh.value(V, cmp, true), gd = gh.value(U, cmp, true);
        if (cmp == 0) {
          S.uv[q][lb][gy + 1][gx + 1].x = g;
          S.ud[q][lb][gy + 1][gx + 1].x = gd;
        } else {
          S.uv[q][lb][gy + 1][gx + 1].y = g;
          S.ud[q][lb][gy + 1][gx + 1].y = gd;
        }
        if (gh.s.kind == kFiner) {
          const double facDiv = 0.5 * h / dt;
          const double own =
              div_face(f, facDiv, __ldg(P.chi + gh.cell), g, V.v(gh.cell, cmp), gd, U.v(gh.cell, cmp));
          int64_t fb;
          int k0;
          gh.fine_cells(fb, k0);
          const double facDivF = 0.5 * cell_h(G.F, G.F.level[fb]) / dt;
          double fs[2];
          for (int r = 0; r < 2; ++r) {
            const int64_t fc = gh.fine_cell(fb, k0, r, 0);
            fs[r] = div_face(f ^ 1, facDivF, __ldg(P.chi + fc), gh.fine_ghost(V, cmp, fb, k0, r), V.v(fc, cmp),
                             gh.fine_ghost(U, cmp, fb, k0, r), U.v(fc, cmp));
          }
          S.corr[0][lb][f][k] = own + (fs[0] + fs[1]);
        }
      }
      if (gpres) {
        const Fld Q{P.pres, 1};
        const double g = gh.value(Q, 0, false);
        S.p[q][lb][gy + 1][gx + 1] = g;
        if (gh.s.kind == kFiner) {
          const double own = g - Q.v(gh.cell, 0);
          int64_t fb;
          int k0;
          gh.fine_cells(fb, k0);
          double fs[2];
          for (int r = 0; r < 2; ++r) fs[r] = gh.fine_ghost(Q, 0, fb, k0, r) - Q.v(gh.fine_cell(fb, k0, r, 0), 0);
          S.corr[1][lb][f][k] = own + (fs[0] + fs[1]);
        }
      }
    }
    __syncthreads();
    if (valid) {
      const bool edge[4] = {ix == 0, ix == kBS - 1, iy == 0, iy == kBS - 1};
      const int along[4] = {iy, iy, ix, ix};
      const int X = ix + 1, Y = iy + 1;
      double t;
      if (vel) {
        const double h = cell_h(G.F, G.F.level[b]);
        const double facDiv = 0.5 * h / dt;
        const double chi = S.chi[q][lb][c];
        t = facDiv * ((S.uv[q][lb][Y][X + 1].x - S.uv[q][lb][Y][X - 1].x) +
                      (S.uv[q][lb][Y + 1][X].y - S.uv[q][lb][Y - 1][X].y));
        t += -facDiv * chi * ((S.ud[q][lb][Y][X + 1].x - S.ud[q][lb][Y][X - 1].x) +
                              (S.ud[q][lb][Y + 1][X].y - S.ud[q][lb][Y - 1][X].y));
        for (int f = 0; f < 4; ++f)
          if (edge[f] && S.kind[lb][f] == kFiner) t = t + S.corr[0][lb][f][along[f]];
      } else {
        t = P.tmp[cell];
      }
      if (pres) {
        const double p0 = S.p[q][lb][Y][X];
        t -= ((S.p[q][lb][Y][X - 1] + S.p[q][lb][Y][X + 1]) + (S.p[q][lb][Y - 1][X] + S.p[q][lb][Y + 1][X])) -
             4.0 * p0;
        for (int f = 0; f < 4; ++f)
          if (edge[f] && S.kind[lb][f] == kFiner) t = t + S.corr[1][lb][f][along[f]];
        P.pold[cell] = p0;
      }
      P.tmp[cell] = t;
    }
    code = code_next;
    // the next iteration's first barrier orders these reads of buffer q
    // before that iteration's copies into it
  }
  cp_async_wait_n<0>();  // nothing may land after return
}

__global__ void __launch_bounds__(kProjThreads, 4) k_pressure_correction(const __grid_constant__ Geo G, double dt,
                                                                           const double* __restrict__ pres,
                                                                           double* __restrict__ vel) {
  __shared__ ProjSmem S;
  const int lb = threadIdx.x >> 6, c = threadIdx.x & 63, ix = c & 7, iy = c >> 3;
  const bool gthr = c < 4 * kBS;
  const Fld Q{pres, 1};
  const int64_t ngroups = (G.F.nb + kLabBlocks - 1) / kLabBlocks;
  auto fetch = [&](int64_t grp, Prefetch& q) {
    const int64_t b = grp * kLabBlocks + lb;
    if (b >= G.F.nb) return;
    const int64_t cell = b * kBLEN + c;
    q.p = __ldg(pres + cell);
    q.u = reinterpret_cast<const double2*>(vel)[cell];  // updated in place: no read-only path
    if (gthr) q.code = __ldg(G.nbr + 4 * b + (c >> 3));
  };
  Prefetch cur{}, nxt{};
  int64_t grp = blockIdx.x;
  if (grp < ngroups) fetch(grp, cur);
  for (; grp < ngroups; grp += gridDim.x) {
    const int64_t b = grp * kLabBlocks + lb;
    const bool valid = b < G.F.nb;
    const int64_t cell = b * kBLEN + c;
    if (valid) labv(S, kLabP, lb, ix, iy) = cur.p;
    if (grp + gridDim.x < ngroups) fetch(grp + gridDim.x, nxt);
    if (valid && gthr) {
      const Ghost gh(G, b, c, G.side_from_code(b, c >> 3, cur.code));
      const int k = c & 7, f = gh.f;
      if (k == 0) S.kind[lb][f] = gh.s.kind;
      const int gx = gh.ix + (f == 0 ? -1 : f == 1 ? 1 : 0), gy = gh.iy + (f == 2 ? -1 : f == 3 ? 1 : 0);
      const double g = gh.value(Q, 0, false);
      labv(S, kLabP, lb, gx, gy) = g;
      if (gh.s.kind == kFiner) {
        const double pFac = -0.5 * dt * cell_h(G.F, G.F.level[b]);
        const double own = grad_face(f, pFac, g, Q.v(gh.cell, 0));
        int64_t fb;
        int k0;
        gh.fine_cells(fb, k0);
        const double pFacF = -0.5 * dt * cell_h(G.F, G.F.level[fb]);
        double fs[2];
        for (int q = 0; q < 2; ++q)
          fs[q] = grad_face(f ^ 1, pFacF, gh.fine_ghost(Q, 0, fb, k0, q), Q.v(gh.fine_cell(fb, k0, q, 0), 0));
        S.corr[0][lb][f][k] = own + (fs[0] + fs[1]);
      }
    }
    __syncthreads();
    if (valid) {
      const double h = cell_h(G.F, G.F.level[b]);
      const double pFac = -0.5 * dt * h;
      double tv[2];
      tv[0] = pFac * (labv(S, kLabP, lb, ix + 1, iy) - labv(S, kLabP, lb, ix - 1, iy));
      tv[1] = pFac * (labv(S, kLabP, lb, ix, iy + 1) - labv(S, kLabP, lb, ix, iy - 1));
      const bool edge[4] = {ix == 0, ix == kBS - 1, iy == 0, iy == kBS - 1};
      const int along[4] = {iy, iy, ix, ix};
      for (int f = 0; f < 4; ++f)
        if (edge[f] && S.kind[lb][f] == kFiner) tv[f < 2 ? 0 : 1] = tv[f < 2 ? 0 : 1] + S.corr[0][lb][f][along[f]];
      const double ih2 = 1.0 / h / h;
      double2 v = cur.u;
      v.x += tv[0] * ih2;
      v.y += tv[1] * ih2;
      reinterpret_cast<double2*>(vel)[cell] = v;
    }
    __syncthreads();
    cur = nxt;
  }
}

// Persistent grid: the co-resident CTAs of a kernel (queried once per device).
int persistent_grid(const void* fn, int which, int64_t ngroups) {
  static std::atomic<int> cap[64][2];
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 0;
  int g = cap[dev][which].load(std::memory_order_acquire);
  if (g <= 0) {
    int sms = 0, per_sm = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kProjThreads, 0) != cudaSuccess)
      return 0;
    g = std::max(1, sms * per_sm);
    cap[dev][which].store(g, std::memory_order_release);
  }
  return (int)std::min<int64_t>(g, ngroups);
}

}  // namespace

cudaError_t launch_pressure_rhs(const ForestView& F, const int32_t* nbr, double dt, const ProjFields& f,
                                cudaStream_t s) {
  if (F.nb <= 0) return cudaSuccess;
  const int grid = persistent_grid((const void*)k_pressure_rhs, 0, (F.nb + kLabBlocks - 1) / kLabBlocks);
  if (grid <= 0) return cudaErrorInvalidConfiguration;
  k_pressure_rhs<<<grid, kProjThreads, 0, s>>>(Geo{F, nbr}, dt, f);
  return cudaGetLastError();
}

cudaError_t launch_pressure_correction(const ForestView& F, const int32_t* nbr, double dt, const double* pres,
                                       double* vel, cudaStream_t s) {
  if (F.nb <= 0) return cudaSuccess;
  const int grid = persistent_grid((const void*)k_pressure_correction, 1, (F.nb + kLabBlocks - 1) / kLabBlocks);
  if (grid <= 0) return cudaErrorInvalidConfiguration;
  k_pressure_correction<<<grid, kProjThreads, 0, s>>>(Geo{F, nbr}, dt, pres, vel);
  return cudaGetLastError();
}

}  // namespace cup2d
