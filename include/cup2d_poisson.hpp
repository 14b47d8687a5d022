// cup2d_poisson.hpp — C++ drop-in over the C ABI (cup2d_poisson.h).
//
// Mirrors CUP2D's solver boundary (paths in the CUP2D tree):
//   class PoissonSolver { virtual void solve(const ScalarGrid*, ScalarGrid*) = 0; }
//                                                   source/Poisson/Base.h:8-13
//   std::shared_ptr<PoissonSolver> makePoissonSolver(SimulationData&)
//                                                   source/Poisson/Base.cpp:8-30
//   ExpAMRSolver::solve: step<10 tolerances, re-assembly on
//   UpdateFluxCorrection, mean removal              source/Poisson/ExpAMRSolver.cpp:354-416
//
// ScalarGrid here is the block list plus one value per cell (block-major,
// data[block*64 + iy*8 + ix]); a CUP2D build fills it from sim.tmp / sim.pres
// (ScalarBlock is 8x8 row-major, the same layout).  Errors throw
// std::runtime_error carrying the status string; nothing exits.
#pragma once

#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "cup2d_poisson.h"

namespace cup2d_b200 {

struct ScalarGrid {
  cup2d_forest forest;   // the block list (arrays owned by the caller)
  double* data;          // 64 values per block, host memory
};

// The fields of SimulationData the Poisson path reads
// (source/Simulation.cpp:239-245, ExpAMRSolver.cpp:366-372).
struct SimulationData {
  std::string poissonSolver = "cuda_iterative";
  double PoissonTol = 1e-6;
  double PoissonTolRel = 0.0;
  int maxPoissonRestarts = 30;
  int maxPoissonIterations = 1000;  // BiCGSTAB.cu:468 fixes 1000
  int bMeanConstraint = 0;
  int step = 0;
  bool mixedPrecision = false;
  bool UpdateFluxCorrection = true;  // set when the mesh changed
};

inline void check(int status, const char* where) {
  if (status != CUP2D_OK && status != CUP2D_NOT_CONVERGED && status != CUP2D_BREAKDOWN_LIMIT)
    throw std::runtime_error(std::string(where) + ": " + cup2d_status_string(status));
}

class PoissonSolver {
 public:
  virtual ~PoissonSolver() = default;
  virtual void solve(const ScalarGrid* input, ScalarGrid* output) = 0;
};

// "cuda_iterative": BiCGSTAB + 64x64 block-Jacobi on the GPU.
class ExpAMRSolver : public PoissonSolver {
 public:
  ExpAMRSolver(SimulationData& s, const cup2d_forest& forest) : sim_(s) {
    if (s.bMeanConstraint != 0) throw std::invalid_argument("bMeanConstraint != 0 is not supported");
    cup2d_solve_opts o = opts();
    check(cup2d_poisson_create(&forest, &o, &h_), "cup2d_poisson_create");
    sim_.UpdateFluxCorrection = false;
  }
  ~ExpAMRSolver() override { cup2d_poisson_destroy(h_); }
  ExpAMRSolver(const ExpAMRSolver&) = delete;
  ExpAMRSolver& operator=(const ExpAMRSolver&) = delete;

  // input: RHS (sim.tmp); output: initial guess in, solution out (sim.pres)
  void solve(const ScalarGrid* input, ScalarGrid* output) override {
    if (sim_.UpdateFluxCorrection) {
      sim_.UpdateFluxCorrection = false;
      check(cup2d_poisson_update_mesh(h_, &input->forest), "cup2d_poisson_update_mesh");
    }
    cup2d_solve_opts o = opts();
    check(cup2d_poisson_set_opts(h_, &o), "cup2d_poisson_set_opts");
    check(cup2d_poisson_solve(h_, input->data, output->data, &last_), "cup2d_poisson_solve");
  }
  const cup2d_solve_stats& last_stats() const { return last_; }

 private:
  cup2d_solve_opts opts() const {
    cup2d_solve_opts o;
    cup2d_default_opts(&o);
    const bool early = sim_.step < 10;
    o.tol_abs = early ? 0.0 : sim_.PoissonTol;
    o.tol_rel = early ? 0.0 : sim_.PoissonTolRel;
    o.max_restarts = early ? 100 : sim_.maxPoissonRestarts;
    o.max_iter = sim_.maxPoissonIterations;
    o.precision = sim_.mixedPrecision ? CUP2D_PREC_MIXED : CUP2D_PREC_FP64;
    return o;
  }
  SimulationData& sim_;
  cup2d_poisson* h_ = nullptr;
  cup2d_solve_stats last_{};
};

inline std::shared_ptr<PoissonSolver> makePoissonSolver(SimulationData& s, const cup2d_forest& forest) {
  if (s.poissonSolver == "cuda_iterative") return std::make_shared<ExpAMRSolver>(s, forest);
  if (s.poissonSolver == "iterative")
    throw std::invalid_argument("Poisson solver \"iterative\" (the CPU AMRSolver) is not part of cup2d_b200");
  throw std::invalid_argument("Poisson solver: \"" + s.poissonSolver + "\" unrecognized!");
}

}  // namespace cup2d_b200
