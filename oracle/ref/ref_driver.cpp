// ORACLE — test infrastructure only.  C entry points of the reference checker:
// CUP2D's own ExpAMRSolver (source/Poisson/ExpAMRSolver.cpp, compiled
// unchanged from the reference tree by oracle/ref/build.py) run on a forest
// given as a block list, through the same call the pressure step makes,
// ExpAMRSolver::solve(sim.tmp, sim.pres) (PressureSingle.cpp:851).
//
// Two builds share this file:
//   * CPU (liboracle_ref_cpu.so): the solver stage is solver_capture.cpp, so
//     a "solve" runs the reference's P^-1 construction (ctor, :25-99),
//     getMat (:180-313), getVec (:315-352) and LocalSpMatDnVec::make, and
//     records P^-1 and the COO system for ref_copy_pinv / ref_copy_system.
//   * GPU (liboracle_ref_gpu.so): the reference's BiCGSTAB.cu
//     (cuBLAS/cuSPARSE) solves the system, and the solve's mean removal
//     (:383-415) writes the result into the pressure grid.  The solver's own
//     progress lines (|A x0|, initial norm, restarts, iterations, final error;
//     BiCGSTAB.cu:449-452,490-493,549,600-606) go to std::cout, which this
//     driver redirects into the caller's log buffer for parsing.
//
// The SimulationData members this path reads are set from the arguments:
// step (tolerances apply from step 10 on, ExpAMRSolver.cpp:366-368),
// PoissonTol, PoissonTolRel, maxPoissonRestarts, bMeanConstraint.
#include <cstdint>
#include <cstring>
#include <iostream>
#include <memory>
#include <sstream>
#include <string>

#include "ExpAMRSolver.h"
#include "ref_capture.hpp"

BCflag cubismBCX = wall;
BCflag cubismBCY = wall;

// SimulationData's out-of-line members live in the reference's
// SimulationData.cpp, which needs the rest of CUP2D; the checker defines the
// ones this path touches.
SimulationData::SimulationData() {}
SimulationData::~SimulationData() { delete profiler; }
void SimulationData::startProfiler(std::string) {}
void SimulationData::stopProfiler() {}

RefCapture& ref_capture() {
  static RefCapture c;
  return c;
}

extern "C" {

typedef struct ref_forest {
  int32_t bpdx, bpdy, level_max, periodic_x, periodic_y;
  double extent;
  int64_t nblocks;
  const int32_t* level;
  const int32_t* bx;
  const int32_t* by;
} ref_forest;

// Runs ExpAMRSolver::solve on the forest with right-hand side b (the h^2-scaled
// divergence in sim.tmp) and initial guess x (sim.pres); on return x holds the
// reference's mean-removed solution (GPU build) or is unchanged apart from the
// mean removal (CPU build).  Vectors are block-major, 64 cells per block in
// iy*8+ix order.  Returns 0, or -1 with the exception text in the log.
// With mean_constraint != 0 the solve runs with sim.bMeanConstraint set.
int ref_solve_mc(const ref_forest* f, const double* b, double* x, double tol_abs, double tol_rel, int max_restarts,
                 int step, int mean_constraint, char* log, int64_t log_cap) {
  std::ostringstream out;
  std::streambuf* saved = std::cout.rdbuf(out.rdbuf());
  int rc = 0;
  try {
    ref_capture() = RefCapture{};
    cubismBCX = f->periodic_x ? periodic : wall;
    cubismBCY = f->periodic_y ? periodic : wall;
    auto tmp = std::make_unique<ScalarGrid>();
    auto pres = std::make_unique<ScalarGrid>();
    tmp->standin_setup(f->bpdx, f->bpdy, f->level_max, f->extent, f->nblocks, f->level, f->bx, f->by);
    pres->standin_setup(f->bpdx, f->bpdy, f->level_max, f->extent, f->nblocks, f->level, f->bx, f->by);
    for (int64_t k = 0; k < f->nblocks; k++) {
      ScalarBlock& B = tmp->standin_block(k);
      ScalarBlock& P = pres->standin_block(k);
      for (int iy = 0; iy < 8; iy++)
        for (int ix = 0; ix < 8; ix++) {
          B(ix, iy).s = b[k * 64 + iy * 8 + ix];
          P(ix, iy).s = x[k * 64 + iy * 8 + ix];
        }
    }
    {
      SimulationData sim;
      sim.comm = MPI_COMM_WORLD;
      sim.rank = 0;
      sim.bpdx = f->bpdx;
      sim.bpdy = f->bpdy;
      sim.levelMax = f->level_max;
      sim.extent = f->extent;
      sim.step = step;
      sim.PoissonTol = tol_abs;
      sim.PoissonTolRel = tol_rel;
      sim.maxPoissonRestarts = max_restarts;
      sim.bMeanConstraint = mean_constraint;
      sim.verbose = false;
      sim.tmp = tmp.get();
      sim.pres = pres.get();
      {
        ExpAMRSolver solver(sim);
        solver.solve(sim.tmp, sim.pres);
      }
      sim.tmp = nullptr;
      sim.pres = nullptr;
    }
    for (int64_t k = 0; k < f->nblocks; k++) {
      ScalarBlock& P = pres->standin_block(k);
      for (int iy = 0; iy < 8; iy++)
        for (int ix = 0; ix < 8; ix++) x[k * 64 + iy * 8 + ix] = P(ix, iy).s;
    }
  } catch (const std::exception& e) {
    out << "\nERROR: " << e.what() << "\n";
    rc = -1;
  }
  std::cout.rdbuf(saved);
  const std::string s = out.str();
  if (log && log_cap > 0) {
    const size_t n = std::min<size_t>(s.size(), (size_t)log_cap - 1);
    std::memcpy(log, s.data(), n);
    log[n] = '\0';
  }
  return rc;
}

int ref_solve(const ref_forest* f, const double* b, double* x, double tol_abs, double tol_rel, int max_restarts,
              int step, char* log, int64_t log_cap) {
  return ref_solve_mc(f, b, x, tol_abs, tol_rel, max_restarts, step, 0, log, log_cap);
}

// The row getMat recorded for bMeanConstraint in the last ref_solve (CPU
// build; -1 when the constraint was off).
int ref_mean_row(void) { return ref_capture().have_system ? ref_capture().mean_row : -2; }

// P^-1 recorded by the last ref_solve (CPU build): 64x64, row-major.
int ref_copy_pinv(double* P) {
  const RefCapture& c = ref_capture();
  if (c.pinv.size() != 64 * 64) return -1;
  std::memcpy(P, c.pinv.data(), sizeof(double) * 64 * 64);
  return 0;
}

// Size of the system recorded by the last ref_solve (CPU build).
int ref_system_size(int64_t* m, int64_t* nnz) {
  const RefCapture& c = ref_capture();
  if (!c.have_system) return -1;
  *m = c.m;
  *nnz = (int64_t)c.val.size();
  return 0;
}

// The recorded COO (rows in ascending order, as LocalSpMatDnVec holds it),
// b, x0 and h^2 per block.
int ref_copy_system(int32_t* row, int32_t* col, double* val, double* b, double* x0, double* h2) {
  const RefCapture& c = ref_capture();
  if (!c.have_system) return -1;
  const size_t nnz = c.val.size();
  for (size_t i = 0; i < nnz; i++) {
    row[i] = c.row[i];
    col[i] = c.col[i];
  }
  std::memcpy(val, c.val.data(), sizeof(double) * nnz);
  std::memcpy(b, c.b.data(), sizeof(double) * c.b.size());
  std::memcpy(x0, c.x0.data(), sizeof(double) * c.x0.size());
  std::memcpy(h2, c.h2.data(), sizeof(double) * c.h2.size());
  return 0;
}

}  // extern "C"
