// C++ caller of the batch wrapper: three uneven forests in one launch from
// host buffers.  Exit code 2 when no CUDA device is present.
#include <cstdio>
#include <stdexcept>
#include <vector>

#include "cup2d_poisson.hpp"

int main() {
  const double disk_a[3] = {0.6, 0.5, 0.1};
  const double disk_b[3] = {1.2, 0.4, 0.1};
  cup2d_mesh* m[2] = {nullptr, nullptr};
  if (cup2d_mesh_disks(4, 2, 4, 2.0, 0, 0, 1, disk_a, 0.15, &m[0]) ||
      cup2d_mesh_disks(4, 2, 3, 2.0, 0, 0, 1, disk_b, 0.1, &m[1]))
    return 1;
  std::vector<cup2d_forest> forests(2);
  std::vector<std::vector<double>> b(2), x(2);
  for (int i = 0; i < 2; ++i) {
    cup2d_mesh_forest(m[i], &forests[i]);
    b[i].resize(64 * forests[i].nblocks);
    x[i].assign(64 * forests[i].nblocks, 0.0);
    cup2d_rhs_fourier(&forests[i], 7 + i, 8, b[i].data());
  }
  cup2d_solve_opts opts;
  cup2d_default_opts(&opts);
  opts.tol_rel = 1e-8;
  opts.max_iter = 5000;
  int rc = 0;
  try {
    cup2d_b200::BatchSolver batch(forests, opts);
    const auto st = batch.solve({b[0].data(), b[1].data()}, {x[0].data(), x[1].data()});
    for (size_t i = 0; i < st.size(); ++i) std::printf("problem %zu: status %d\n", i, st[i].status);
  } catch (const std::runtime_error& e) {
    std::printf("%s\n", e.what());
    rc = 2;
  }
  cup2d_mesh_destroy(m[0]);
  cup2d_mesh_destroy(m[1]);
  return rc;
}
