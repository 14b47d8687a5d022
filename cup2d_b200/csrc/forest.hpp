// Host-side 2D block-AMR forest: the block list that CUP2D gets from Cubism.
//
// A forest is a set of leaf blocks (level, bx, by) over bpdx x bpdy root
// blocks of 8x8 cells.  Cubism (an un-vendored submodule of CUP2D) owns this
// structure in the reference; the Poisson path only needs, per block, its
// level, its (i,j) index at that level, and the neighbour queries
// Exists / CheckCoarser / CheckFiner used by ExpAMRSolver::getMat
// (source/Poisson/ExpAMRSolver.cpp:141-177, 217-256).
//
// This file builds synthetic forests: refinement to the finest level near
// disks, face-and-corner 2:1 balance, and a Morton (Z) order of the leaves.
// Block order only permutes the linear system, so any bijective order works.
#pragma once
#include <cstdint>
#include <vector>

namespace cup2d {

struct Disk {
  double cx, cy, r;
};

struct ForestSpec {
  int bpdx = 1, bpdy = 1;  // root blocks per direction
  int level_max = 1;       // number of levels (finest = level_max - 1)
  double extent = 1.0;     // length of the longer domain side
  bool periodic_x = false, periodic_y = false;
};

struct Forest {
  ForestSpec spec;
  std::vector<int32_t> level, bx, by;
  int64_t size() const { return (int64_t)level.size(); }
};

// Grid spacing of a cell at `level` (Cubism: extent / (max(bpd)*8*2^level)).
double cell_h(const ForestSpec& s, int level);

// Refine every block whose rectangle meets the band {p : | |p-c| - r | <= band}
// of any disk, down to level_max-1; then enforce 2:1 balance across faces and
// corners and sort the leaves in Morton order.
Forest build_disk_forest(const ForestSpec& s, const std::vector<Disk>& disks,
                         double band);

// Uniform forest: every block at `level`.
Forest build_uniform_forest(const ForestSpec& s, int level);

// Validates a leaf set: leaves tile the domain exactly once and face/corner
// neighbours differ by at most one level.  Returns 0 if valid, otherwise a
// non-zero code (1 overlap/hole, 2 balance violation, 3 out of range).
int validate_forest(const Forest& f);

// Seeded synthetic right-hand side: b = 0.5*h*(u(x+h)-u(x-h) + v(y+h)-v(y-h))
// (the divergence stencil of PressureSingle.cpp:339-346 with dt=1) of a
// random Fourier velocity field with wave-vectors 0<|k|<=kmax and amplitude
// |k|^-2, N(0,1) coefficients from std::mt19937_64(seed).  The result is
// projected to zero entry-sum (Neumann compatibility).  Layout: block-major,
// b[block*64 + iy*8 + ix].
void fourier_rhs(const Forest& f, uint64_t seed, int kmax, double* b);

// Same, with coefficients a_k(t) = rho*a_k(t-1) + sqrt(1-rho^2)*xi: the
// AR(1) sequence of a time-stepping run.  `coef` holds 4 doubles per mode and
// is advanced in place when step > 0.
int fourier_num_modes(int kmax);
void fourier_init_coefs(uint64_t seed, int kmax, double* coef);
void fourier_advance_coefs(uint64_t seed, int kmax, double rho, int64_t step,
                           double* coef);
void fourier_rhs_from_coefs(const Forest& f, int kmax, const double* coef,
                            double* b);

}  // namespace cup2d
