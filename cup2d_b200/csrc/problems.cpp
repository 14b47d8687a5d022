// C ABI for synthetic forests and right-hand sides (include/cup2d_poisson.h).
#include <cstring>
#include <new>
#include <vector>

#include "../../include/cup2d_poisson.h"
#include "forest.hpp"

using cup2d::Forest;
using cup2d::ForestSpec;

struct cup2d_mesh {
  Forest f;
};

namespace {

bool to_forest(const cup2d_forest* in, Forest& out) {
  if (!in || in->nblocks < 0 || (in->nblocks > 0 && (!in->level || !in->bx || !in->by))) return false;
  out.spec.bpdx = in->bpdx;
  out.spec.bpdy = in->bpdy;
  out.spec.level_max = in->level_max;
  out.spec.extent = in->extent;
  out.spec.periodic_x = in->periodic_x != 0;
  out.spec.periodic_y = in->periodic_y != 0;
  out.level.assign(in->level, in->level + in->nblocks);
  out.bx.assign(in->bx, in->bx + in->nblocks);
  out.by.assign(in->by, in->by + in->nblocks);
  return true;
}

bool spec_ok(int32_t bpdx, int32_t bpdy, int32_t level_max, double extent) {
  return bpdx >= 1 && bpdy >= 1 && level_max >= 1 && level_max <= 20 && extent > 0.0 &&
         (int64_t)bpdx * bpdy <= (1 << 20);
}

}  // namespace

extern "C" {

int cup2d_mesh_disks(int32_t bpdx, int32_t bpdy, int32_t level_max, double extent, int32_t periodic_x,
                     int32_t periodic_y, int32_t ndisks, const double* disks, double band, cup2d_mesh** out) {
  if (!out || !spec_ok(bpdx, bpdy, level_max, extent) || ndisks < 0 || (ndisks > 0 && !disks) || !(band >= 0.0))
    return CUP2D_INVALID_ARGUMENT;
  ForestSpec s;
  s.bpdx = bpdx;
  s.bpdy = bpdy;
  s.level_max = level_max;
  s.extent = extent;
  s.periodic_x = periodic_x != 0;
  s.periodic_y = periodic_y != 0;
  std::vector<cup2d::Disk> d(ndisks);
  for (int i = 0; i < ndisks; ++i) d[i] = {disks[3 * i], disks[3 * i + 1], disks[3 * i + 2]};
  auto* m = new (std::nothrow) cup2d_mesh();
  if (!m) return CUP2D_OOM;
  m->f = cup2d::build_disk_forest(s, d, band);
  *out = m;
  return CUP2D_OK;
}

int cup2d_mesh_uniform(int32_t bpdx, int32_t bpdy, int32_t level_max, int32_t level, double extent,
                       int32_t periodic_x, int32_t periodic_y, cup2d_mesh** out) {
  if (!out || !spec_ok(bpdx, bpdy, level_max, extent) || level < 0 || level >= level_max)
    return CUP2D_INVALID_ARGUMENT;
  ForestSpec s;
  s.bpdx = bpdx;
  s.bpdy = bpdy;
  s.level_max = level_max;
  s.extent = extent;
  s.periodic_x = periodic_x != 0;
  s.periodic_y = periodic_y != 0;
  auto* m = new (std::nothrow) cup2d_mesh();
  if (!m) return CUP2D_OOM;
  m->f = cup2d::build_uniform_forest(s, level);
  *out = m;
  return CUP2D_OK;
}

int cup2d_mesh_forest(const cup2d_mesh* m, cup2d_forest* out) {
  if (!m || !out) return CUP2D_INVALID_ARGUMENT;
  const Forest& f = m->f;
  out->bpdx = f.spec.bpdx;
  out->bpdy = f.spec.bpdy;
  out->level_max = f.spec.level_max;
  out->periodic_x = f.spec.periodic_x;
  out->periodic_y = f.spec.periodic_y;
  out->extent = f.spec.extent;
  out->nblocks = f.size();
  out->level = f.level.data();
  out->bx = f.bx.data();
  out->by = f.by.data();
  return CUP2D_OK;
}

int cup2d_mesh_destroy(cup2d_mesh* m) {
  delete m;
  return CUP2D_OK;
}

int cup2d_forest_validate(const cup2d_forest* in) {
  Forest f;
  if (!to_forest(in, f)) return CUP2D_INVALID_ARGUMENT;
  return cup2d::validate_forest(f) == 0 ? CUP2D_OK : CUP2D_BAD_MESH;
}

int cup2d_forest_cell_h(const cup2d_forest* in, double* h_out) {
  if (!in || !h_out || !(in->extent > 0.0)) return CUP2D_INVALID_ARGUMENT;
  ForestSpec s;
  s.bpdx = in->bpdx;
  s.bpdy = in->bpdy;
  s.extent = in->extent;
  for (int64_t b = 0; b < in->nblocks; ++b) h_out[b] = cup2d::cell_h(s, in->level[b]);
  return CUP2D_OK;
}

int cup2d_rhs_fourier(const cup2d_forest* in, uint64_t seed, int32_t kmax, double* b) {
  Forest f;
  if (!b || kmax < 1 || kmax > 31 || !to_forest(in, f)) return CUP2D_INVALID_ARGUMENT;
  cup2d::fourier_rhs(f, seed, kmax, b);
  return CUP2D_OK;
}

int32_t cup2d_fourier_num_modes(int32_t kmax) {
  return (kmax < 1 || kmax > 31) ? 0 : cup2d::fourier_num_modes(kmax);
}

int cup2d_fourier_coefs(uint64_t seed, int32_t kmax, double* coef) {
  if (!coef || kmax < 1 || kmax > 31) return CUP2D_INVALID_ARGUMENT;
  cup2d::fourier_init_coefs(seed, kmax, coef);
  return CUP2D_OK;
}

int cup2d_fourier_advance(uint64_t seed, int32_t kmax, double rho, int64_t step, double* coef) {
  if (!coef || kmax < 1 || kmax > 31 || !(rho >= -1.0 && rho <= 1.0)) return CUP2D_INVALID_ARGUMENT;
  cup2d::fourier_advance_coefs(seed, kmax, rho, step, coef);
  return CUP2D_OK;
}

int cup2d_rhs_from_coefs(const cup2d_forest* in, int32_t kmax, const double* coef, double* b) {
  Forest f;
  if (!b || !coef || kmax < 1 || kmax > 31 || !to_forest(in, f)) return CUP2D_INVALID_ARGUMENT;
  cup2d::fourier_rhs_from_coefs(f, kmax, coef, b);
  return CUP2D_OK;
}

}  // extern "C"
