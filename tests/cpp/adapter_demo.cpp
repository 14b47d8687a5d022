// Uses the C++ drop-in the way CUP2D's PressureSingle does
// (source/Operators/PressureSingle.cpp:851): solve(tmp, pres).
// Exit codes: 0 solved to tolerance, 2 no CUDA device, 1 anything else.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "cup2d_poisson.hpp"

int main() {
  const double disk[3] = {0.6, 0.5, 0.1};
  cup2d_mesh* mesh = nullptr;
  if (cup2d_mesh_disks(4, 2, 4, 2.0, 0, 0, 1, disk, 0.15, &mesh) != CUP2D_OK) return 1;
  cup2d_forest f;
  cup2d_mesh_forest(mesh, &f);
  const size_t n = (size_t)f.nblocks * 64;
  std::vector<double> tmp(n), pres(n, 0.0);
  cup2d_rhs_fourier(&f, 7, 8, tmp.data());
  cup2d_b200::SimulationData sim;
  sim.step = 20;
  sim.PoissonTol = 0.0;
  sim.PoissonTolRel = 1e-8;
  sim.maxPoissonRestarts = 100;
  sim.maxPoissonIterations = 5000;
  int rc = 0;
  try {
    auto solver = cup2d_b200::makePoissonSolver(sim, f);
    cup2d_b200::ScalarGrid in{f, tmp.data()}, out{f, pres.data()};
    solver->solve(&in, &out);
    const auto& st = static_cast<cup2d_b200::ExpAMRSolver&>(*solver).last_stats();
    std::printf("status %d iterations %d rel_res_inf %.3e\n", st.status, st.iterations, st.rel_res_inf);
    rc = (st.status == CUP2D_OK && st.rel_res_inf <= 1e-8) ? 0 : 1;
  } catch (const std::exception& e) {
    std::printf("error: %s\n", e.what());
    rc = std::strstr(e.what(), "no CUDA device") ? 2 : 1;
  }
  cup2d_mesh_destroy(mesh);
  return rc;
}
