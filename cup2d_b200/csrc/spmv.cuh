// Block-structured SpMV on one 8x8 block per warp (two cells per lane).
//
// Lane l owns cells c0 = l (rows iy = 0..3) and c1 = l + 32 (rows 4..7) of
// the block.  In-block neighbours come from warp shuffles; the cells across
// a same-level face are read from the neighbour block (L2, bypassing L1:
// they are written by other CTAs between grid barriers).  Rows of cells on a
// coarse/fine face are evaluated from their stored CSR row.
#pragma once
#include "common.cuh"

namespace cup2d {

template <class T>
__device__ __forceinline__ T ldcg(const T* p) {
  return __ldcg(p);
}

template <class T>
__device__ __forceinline__ const T* row_vals(const MeshView& M);
template <>
__device__ __forceinline__ const double* row_vals<double>(const MeshView& M) { return M.xval; }
template <>
__device__ __forceinline__ const float* row_vals<float>(const MeshView& M) { return M.xval32; }

template <class T>
__device__ __forceinline__ T explicit_row(const MeshView& M, int r, const T* __restrict__ z) {
  const int k0 = __ldg(M.xptr + r), k1 = __ldg(M.xptr + r + 1);
  const T* __restrict__ vals = row_vals<T>(M);
  T s = T(0);
  for (int k = k0; k < k1; ++k) s += __ldg(vals + k) * ldcg(z + __ldg(M.xcol + k));
  return s;
}

// y = (A z) for the two cells of this lane; z0/z1 are this lane's values.
template <class T>
__device__ __forceinline__ void spmv_block(const MeshView& M, int64_t blk, const T* __restrict__ z,
                                           int lane, T z0, T z1, T& y0, T& y1) {
  const int ix = lane & 7, iy0 = lane >> 3;
  const int4 nb4 = __ldg(reinterpret_cast<const int4*>(M.nbr) + blk);
  const T l0 = __shfl_up_sync(kFull, z0, 1), r0 = __shfl_down_sync(kFull, z0, 1);
  const T l1 = __shfl_up_sync(kFull, z1, 1), r1 = __shfl_down_sync(kFull, z1, 1);
  const T d0 = __shfl_up_sync(kFull, z0, 8);
  const T u0a = __shfl_down_sync(kFull, z0, 8), u0b = __shfl_sync(kFull, z1, (lane + 8) & 31);
  const T u1 = __shfl_down_sync(kFull, z1, 8);
  const T d1a = __shfl_up_sync(kFull, z1, 8), d1b = __shfl_sync(kFull, z0, (lane + 24) & 31);
  T a0 = T(0), a1 = T(0);
  int n0 = 0, n1 = 0;
  // x direction
  if (ix > 0) {
    a0 += l0; a1 += l1; ++n0; ++n1;
  } else if (nb4.x >= 0) {
    const T* q = z + (int64_t)nb4.x * kBLEN + iy0 * kBS + 7;
    a0 += ldcg(q); a1 += ldcg(q + 32); ++n0; ++n1;
  }
  if (ix < 7) {
    a0 += r0; a1 += r1; ++n0; ++n1;
  } else if (nb4.y >= 0) {
    const T* q = z + (int64_t)nb4.y * kBLEN + iy0 * kBS;
    a0 += ldcg(q); a1 += ldcg(q + 32); ++n0; ++n1;
  }
  // y direction: c0 rows 0..3, c1 rows 4..7
  if (iy0 > 0) {
    a0 += d0; ++n0;
  } else if (nb4.z >= 0) {
    a0 += ldcg(z + (int64_t)nb4.z * kBLEN + 56 + ix); ++n0;
  }
  a0 += (lane < 24) ? u0a : u0b; ++n0;
  a1 += (lane >= 8) ? d1a : d1b; ++n1;
  if (iy0 < 3) {
    a1 += u1; ++n1;
  } else if (nb4.w >= 0) {
    a1 += ldcg(z + (int64_t)nb4.w * kBLEN + ix); ++n1;
  }
  y0 = a0 - T(n0) * z0;
  y1 = a1 - T(n1) * z1;
  if (nb4.x == kExplicit || nb4.y == kExplicit || nb4.z == kExplicit || nb4.w == kExplicit) {
    const unsigned long long m = __ldg(M.xmask + blk);
    const int base = __ldg(M.xbase + blk);
    if ((m >> lane) & 1ull) y0 = explicit_row<T>(M, base + __popcll(m & ((1ull << lane) - 1ull)), z);
    if ((m >> (lane + 32)) & 1ull)
      y1 = explicit_row<T>(M, base + __popcll(m & ((1ull << (lane + 32)) - 1ull)), z);
  }
}

}  // namespace cup2d
