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

#include <algorithm>
#include <memory>
#include <stdexcept>
#include <utility>
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
    o.mean_constraint = sim_.bMeanConstraint;
    return o;
  }
  SimulationData& sim_;
  cup2d_poisson* h_ = nullptr;
  cup2d_solve_stats last_{};
};

// Many independent problems in one persistent launch (cup2d_batch_*): each
// problem gets exactly the solve above.  Host-buffer solves, device-pointer
// solves, the launch-shape autotuner and CUDA-graph replay.
class BatchSolver {
 public:
  BatchSolver(const std::vector<cup2d_forest>& forests, const cup2d_solve_opts& opts) {
    check(cup2d_batch_create((int32_t)forests.size(), forests.data(), &opts, &b_), "cup2d_batch_create");
  }
  ~BatchSolver() { cup2d_batch_destroy(b_); }
  BatchSolver(const BatchSolver&) = delete;
  BatchSolver& operator=(const BatchSolver&) = delete;

  int32_t size() const { return cup2d_batch_size(b_); }
  // host buffers: b[i] the RHS, x[i] initial guess in, solution out
  std::vector<cup2d_solve_stats> solve(const std::vector<const double*>& b, const std::vector<double*>& x) {
    std::vector<cup2d_solve_stats> st((size_t)size());
    check(cup2d_batch_solve(b_, b.data(), x.data(), st.data()), "cup2d_batch_solve");
    return st;
  }
  // device pointers, on `stream` (a cudaStream_t)
  std::vector<cup2d_solve_stats> solve_device(const std::vector<const double*>& d_b,
                                              const std::vector<double*>& d_x, void* stream = nullptr) {
    std::vector<cup2d_solve_stats> st((size_t)size());
    check(cup2d_batch_solve_device(b_, d_b.data(), d_x.data(), st.data(), stream), "cup2d_batch_solve_device");
    return st;
  }
  // the fastest (team, CTAs per SM) among the candidates, kept for later solves
  std::pair<int32_t, int32_t> tune(const std::vector<const double*>& d_b, const std::vector<double*>& d_x,
                                   const std::vector<int32_t>& teams, const std::vector<int32_t>& ctas_per_sm,
                                   int32_t iters = 0) {
    std::vector<double> rates(teams.size() * std::max<size_t>(1, ctas_per_sm.size()));
    int32_t team = 0, cps = 0;
    check(cup2d_batch_tune(b_, d_b.data(), d_x.data(), teams.data(), (int32_t)teams.size(), ctas_per_sm.data(),
                           (int32_t)ctas_per_sm.size(), iters, rates.data(), &team, &cps),
          "cup2d_batch_tune");
    return {team, cps};
  }
  void capture(const std::vector<const double*>& d_b, const std::vector<double*>& d_x, bool zero_x = false) {
    check(cup2d_batch_capture(b_, d_b.data(), d_x.data(), zero_x ? CUP2D_GRAPH_ZERO_X : 0), "cup2d_batch_capture");
  }
  void replay(void* stream = nullptr) { check(cup2d_batch_replay(b_, stream), "cup2d_batch_replay"); }
  std::vector<cup2d_solve_stats> replay_stats() {
    std::vector<cup2d_solve_stats> st((size_t)size());
    check(cup2d_batch_replay_stats(b_, st.data()), "cup2d_batch_replay_stats");
    return st;
  }

 private:
  cup2d_batch* b_ = nullptr;
};

inline std::shared_ptr<PoissonSolver> makePoissonSolver(SimulationData& s, const cup2d_forest& forest) {
  if (s.poissonSolver == "cuda_iterative") return std::make_shared<ExpAMRSolver>(s, forest);
  if (s.poissonSolver == "iterative")
    throw std::invalid_argument("Poisson solver \"iterative\" (the CPU AMRSolver) is not part of cup2d_b200");
  throw std::invalid_argument("Poisson solver: \"" + s.poissonSolver + "\" unrecognized!");
}

}  // namespace cup2d_b200
