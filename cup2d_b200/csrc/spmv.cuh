// Block-structured SpMV: y = A z over a range of 8x8 blocks.
//
// Phase 1 (stencil): one warp per block, two cells per lane; lane l owns
// cells c0 = l (rows iy = 0..3) and c1 = l + 32 (rows 4..7).  In-block
// neighbours come from warp shuffles; cells across a same-level face are
// read from the neighbour block, and a wall face contributes no flux.
// Loads of two blocks (and the epilogue's operands) are issued before either
// is computed so that each warp keeps two blocks' worth of requests in
// flight.  Rows of cells on a coarse/fine face are skipped here.
//
// Phase 2 (explicit rows): every thread of the CTA takes explicit rows of
// the range (they are numbered contiguously by block), one row each.
//
// Values written by other CTAs between grid barriers are read with
// ld.global.cg (L2), never from a possibly stale L1 line.
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
#pragma unroll 4
  for (int k = k0; k < k1; ++k) s += __ldg(vals + k) * ldcg(z + __ldg(M.xcol + k));
  return s;
}

template <class T>
struct BlockGather {
  int4 nb;
  T z0, z1;                  // this lane's cells
  T xm0, xm1, xp0, xp1;      // across the x faces (lanes with ix = 0 / 7)
  T ym, yp;                  // across the y faces (rows 0 / 7)
};

template <class T>
__device__ __forceinline__ void gather_block_nb(const int4& nb, int64_t blk, const T* __restrict__ z, int lane,
                                                BlockGather<T>& g) {
  const int ix = lane & 7, iy0 = lane >> 3;
  g.nb = nb;
  const int64_t o = blk * kBLEN;
  g.z0 = ldcg(z + o + lane);
  g.z1 = ldcg(z + o + lane + 32);
  g.xm0 = g.xm1 = g.xp0 = g.xp1 = g.ym = g.yp = T(0);
  if (ix == 0 && g.nb.x >= 0) {
    const T* q = z + (int64_t)g.nb.x * kBLEN + iy0 * kBS + 7;
    g.xm0 = ldcg(q);
    g.xm1 = ldcg(q + 32);
  }
  if (ix == 7 && g.nb.y >= 0) {
    const T* q = z + (int64_t)g.nb.y * kBLEN + iy0 * kBS;
    g.xp0 = ldcg(q);
    g.xp1 = ldcg(q + 32);
  }
  if (iy0 == 0 && g.nb.z >= 0) g.ym = ldcg(z + (int64_t)g.nb.z * kBLEN + 56 + ix);
  if (iy0 == 3 && g.nb.w >= 0) g.yp = ldcg(z + (int64_t)g.nb.w * kBLEN + ix);
}

__device__ __forceinline__ int4 block_nbr(const MeshView& M, int64_t blk) {
  return __ldg(reinterpret_cast<const int4*>(M.nbr) + blk);
}

template <class T>
__device__ __forceinline__ void gather_block(const MeshView& M, int64_t blk, const T* __restrict__ z, int lane,
                                             BlockGather<T>& g) {
  gather_block_nb<T>(block_nbr(M, blk), blk, z, lane, g);
}

// Stencil rows of the gathered block (explicit rows get meaningless values).
template <class T>
__device__ __forceinline__ void stencil_block(const BlockGather<T>& g, int lane, T& y0, T& y1) {
  const int ix = lane & 7, iy0 = lane >> 3;
  const T l0 = __shfl_up_sync(kFull, g.z0, 1), r0 = __shfl_down_sync(kFull, g.z0, 1);
  const T l1 = __shfl_up_sync(kFull, g.z1, 1), r1 = __shfl_down_sync(kFull, g.z1, 1);
  const T d0 = __shfl_up_sync(kFull, g.z0, 8);
  const T u0a = __shfl_down_sync(kFull, g.z0, 8), u0b = __shfl_sync(kFull, g.z1, (lane + 8) & 31);
  const T u1 = __shfl_down_sync(kFull, g.z1, 8);
  const T d1a = __shfl_up_sync(kFull, g.z1, 8), d1b = __shfl_sync(kFull, g.z0, (lane + 24) & 31);
  T a0 = T(0), a1 = T(0);
  int n0 = 0, n1 = 0;
  if (ix > 0) { a0 += l0; a1 += l1; n0++; n1++; }
  else if (g.nb.x >= 0) { a0 += g.xm0; a1 += g.xm1; n0++; n1++; }
  if (ix < 7) { a0 += r0; a1 += r1; n0++; n1++; }
  else if (g.nb.y >= 0) { a0 += g.xp0; a1 += g.xp1; n0++; n1++; }
  if (iy0 > 0) { a0 += d0; n0++; }
  else if (g.nb.z >= 0) { a0 += g.ym; n0++; }
  a0 += (lane < 24) ? u0a : u0b; n0++;
  a1 += (lane >= 8) ? d1a : d1b; n1++;
  if (iy0 < 3) { a1 += u1; n1++; }
  else if (g.nb.w >= 0) { a1 += g.yp; n1++; }
  y0 = a0 - T(n0) * g.z0;
  y1 = a1 - T(n1) * g.z1;
}

template <class T>
__device__ __forceinline__ unsigned long long explicit_mask(const MeshView& M, int64_t blk, const int4& nb) {
  if (nb.x == kExplicit || nb.y == kExplicit || nb.z == kExplicit || nb.w == kExplicit) return __ldg(M.xmask + blk);
  return 0ull;
}

// y = A z for the two cells of this lane (single-block form, complete rows).
template <class T>
__device__ __forceinline__ void spmv_block(const MeshView& M, int64_t blk, const T* __restrict__ z, int lane,
                                           T& y0, T& y1) {
  BlockGather<T> g;
  gather_block<T>(M, blk, z, lane, g);
  stencil_block<T>(g, lane, y0, y1);
  const unsigned long long m = explicit_mask<T>(M, blk, g.nb);
  if (m) {
    const int base = __ldg(M.xbase + blk);
    if ((m >> lane) & 1ull) y0 = explicit_row<T>(M, base + __popcll(m & ((1ull << lane) - 1ull)), z);
    if ((m >> (lane + 32)) & 1ull) y1 = explicit_row<T>(M, base + __popcll(m & ((1ull << (lane + 32)) - 1ull)), z);
  }
}

// y = A z over blocks [b0, b1) by the whole CTA.  The epilogue is a functor
// with `Pre load(i)`, the operands it needs at cell i (loaded together with
// the gather, before y is known), and `operator()(i, y, pre)`, called once
// per cell by the thread that computed it, in no particular order.  The
// neighbour tables of a warp's next block pair are fetched while it
// computes the current pair, so each pair costs one round trip to memory.
template <class T, class Epi>
__device__ __forceinline__ void spmv_range(const MeshView& M, const T* __restrict__ z, int64_t b0, int64_t b1,
                                           Epi& epi) {
  using Pre = typename Epi::Pre;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  int64_t blk = b0 + w;
  int4 na = make_int4(0, 0, 0, 0), nbb = make_int4(0, 0, 0, 0);
  if (blk < b1) na = block_nbr(M, blk);
  if (blk + nw < b1) nbb = block_nbr(M, blk + nw);
  for (; blk < b1; blk += 2 * nw) {
    const bool two = blk + nw < b1;  // warp-uniform
    BlockGather<T> ga, gb;
    gather_block_nb<T>(na, blk, z, lane, ga);
    const int64_t oa = blk * kBLEN, ob = (blk + nw) * kBLEN;
    const Pre pa0 = epi.load(oa + lane), pa1 = epi.load(oa + lane + 32);
    Pre pb0{}, pb1{};
    if (two) {
      gather_block_nb<T>(nbb, blk + nw, z, lane, gb);
      pb0 = epi.load(ob + lane);
      pb1 = epi.load(ob + lane + 32);
    }
    const int64_t nxt = blk + 2 * nw;
    if (nxt < b1) na = block_nbr(M, nxt);
    if (nxt + nw < b1) nbb = block_nbr(M, nxt + nw);
    T y0, y1;
    stencil_block<T>(ga, lane, y0, y1);
    unsigned long long m = explicit_mask<T>(M, blk, ga.nb);
    if (!((m >> lane) & 1ull)) epi(oa + lane, y0, pa0);
    if (!((m >> (lane + 32)) & 1ull)) epi(oa + lane + 32, y1, pa1);
    if (two) {
      stencil_block<T>(gb, lane, y0, y1);
      m = explicit_mask<T>(M, blk + nw, gb.nb);
      if (!((m >> lane) & 1ull)) epi(ob + lane, y0, pb0);
      if (!((m >> (lane + 32)) & 1ull)) epi(ob + lane + 32, y1, pb1);
    }
  }
  if (b1 > b0) {
    const int r0 = __ldg(M.xbase + b0), r1 = __ldg(M.xbase + b1);
    for (int r = r0 + threadIdx.x; r < r1; r += blockDim.x) {
      const int64_t i = (int64_t)__ldg(M.rowcell + r);
      const Pre pre = epi.load(i);
      epi(i, explicit_row<T>(M, r, z), pre);
    }
  }
}

}  // namespace cup2d
