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

// ------------------------------------------------ 16-byte lane layout ----
//
// The range passes move 16 bytes per lane and access: V = 4 consecutive
// cells of a row for FP32 (a warp covers two blocks, 16 lanes each), V = 2
// for FP64 (a warp covers one block).  A "chunk" is the CB blocks one warp
// access covers.  Lane l of a chunk owns cells cell0 .. cell0 + V - 1 of
// block bl, row iy; in-row neighbours of other lanes and the rows above and
// below come from shuffles, cells across a block face from the neighbour.

template <class T>
struct Lane {
  static constexpr int V = 16 / (int)sizeof(T);  // cells per lane
  static constexpr int LB = kBLEN / V;           // lanes per block
  static constexpr int LR = kBS / V;             // lanes per row
  static constexpr int CB = 32 / LB;             // blocks per chunk
  int sub, bl, iy, ix0, cell0;
  __device__ __forceinline__ explicit Lane(int lane) {
    sub = lane % LB;
    bl = lane / LB;
    iy = sub / LR;
    ix0 = V * (sub % LR);
    cell0 = iy * kBS + ix0;
  }
};

// N consecutive values at p (N * sizeof(T) a multiple of 8 bytes, p aligned
// to it): ld.global.cg / plain stores of 8- or 16-byte vectors.
template <int N, class T>
__device__ __forceinline__ void ldv(const T* p, T (&v)[N]) {
  static_assert(N * sizeof(T) % 8 == 0, "vector size");
  if constexpr (sizeof(T) == 4 && N == 2) {
    const float2 a = __ldcg(reinterpret_cast<const float2*>(p));
    v[0] = a.x; v[1] = a.y;
  } else if constexpr (sizeof(T) == 4) {
#pragma unroll
    for (int k = 0; k < N; k += 4) {
      const float4 a = __ldcg(reinterpret_cast<const float4*>(p + k));
      v[k] = a.x; v[k + 1] = a.y; v[k + 2] = a.z; v[k + 3] = a.w;
    }
  } else {
#pragma unroll
    for (int k = 0; k < N; k += 2) {
      const double2 a = __ldcg(reinterpret_cast<const double2*>(p + k));
      v[k] = a.x; v[k + 1] = a.y;
    }
  }
}

template <int N, class T>
__device__ __forceinline__ void stv(T* p, const T (&v)[N]) {
  static_assert(N * sizeof(T) % 8 == 0, "vector size");
  if constexpr (sizeof(T) == 4 && N == 2) {
    *reinterpret_cast<float2*>(p) = make_float2(v[0], v[1]);
  } else if constexpr (sizeof(T) == 4) {
#pragma unroll
    for (int k = 0; k < N; k += 4)
      *reinterpret_cast<float4*>(p + k) = make_float4(v[k], v[k + 1], v[k + 2], v[k + 3]);
  } else {
#pragma unroll
    for (int k = 0; k < N; k += 2) *reinterpret_cast<double2*>(p + k) = make_double2(v[k], v[k + 1]);
  }
}

template <class T>
struct ChunkGather {
  static constexpr int V = Lane<T>::V;
  int4 nb;
  T z[V];         // this lane's cells
  T xm, xp;       // across the x faces (first / last lane of a row)
  T ym[V], yp[V]; // across the y faces (rows 0 / 7)
};

template <class T>
__device__ __forceinline__ void gather_chunk(const int4& nb, int64_t blk, bool valid, const T* __restrict__ z,
                                             const Lane<T>& L, ChunkGather<T>& g) {
  constexpr int V = Lane<T>::V;
  g.nb = nb;
  g.xm = g.xp = T(0);
#pragma unroll
  for (int j = 0; j < V; ++j) g.z[j] = g.ym[j] = g.yp[j] = T(0);
  if (!valid) return;
  ldv<V>(z + blk * kBLEN + L.cell0, g.z);
  if (L.ix0 == 0 && nb.x >= 0) g.xm = ldcg(z + (int64_t)nb.x * kBLEN + L.iy * kBS + (kBS - 1));
  if (L.ix0 + V == kBS && nb.y >= 0) g.xp = ldcg(z + (int64_t)nb.y * kBLEN + L.iy * kBS);
  if (L.iy == 0 && nb.z >= 0) ldv<V>(z + (int64_t)nb.z * kBLEN + (kBS - 1) * kBS + L.ix0, g.ym);
  if (L.iy == kBS - 1 && nb.w >= 0) ldv<V>(z + (int64_t)nb.w * kBLEN + L.ix0, g.yp);
}

// Stencil rows of the lane's cells, summed left, right, below, above as the
// assembled rows are (explicit rows get meaningless values).  All lanes of
// the warp take part (shuffles).
template <class T>
__device__ __forceinline__ void stencil_chunk(const ChunkGather<T>& g, const Lane<T>& L, T (&y)[Lane<T>::V]) {
  constexpr int V = Lane<T>::V, LR = Lane<T>::LR;
  const T from_l = __shfl_up_sync(kFull, g.z[V - 1], 1);
  const T from_r = __shfl_down_sync(kFull, g.z[0], 1);
  T dn[V], up[V];
#pragma unroll
  for (int j = 0; j < V; ++j) {
    dn[j] = __shfl_up_sync(kFull, g.z[j], LR);
    up[j] = __shfl_down_sync(kFull, g.z[j], LR);
  }
  const bool left_in = (L.sub % LR) > 0, right_in = (L.sub % LR) < LR - 1;
#pragma unroll
  for (int j = 0; j < V; ++j) {
    T a = T(0);
    int n = 0;
    if (j > 0) { a += g.z[j - 1]; n++; }
    else if (left_in) { a += from_l; n++; }
    else if (g.nb.x >= 0) { a += g.xm; n++; }
    if (j < V - 1) { a += g.z[j + 1]; n++; }
    else if (right_in) { a += from_r; n++; }
    else if (g.nb.y >= 0) { a += g.xp; n++; }
    if (L.iy > 0) { a += dn[j]; n++; }
    else if (g.nb.z >= 0) { a += g.ym[j]; n++; }
    if (L.iy < kBS - 1) { a += up[j]; n++; }
    else if (g.nb.w >= 0) { a += g.yp[j]; n++; }
    y[j] = a - T(n) * g.z[j];
  }
}

// y = A z over blocks [b0, b1) by the whole CTA, in the 16-byte layout.  The
// epilogue functor provides
//   Pre load(i0) / Pre load1(i)  operands of the lane's V cells from i0 (or
//                                of one cell i, as element 0), loaded with
//                                the gather, before y is known;
//   vec(i0, y[V], pre)           the V cells (all stencil rows);
//   one(i, y, pre, j)            cell i, element j of pre (lanes owning an
//                                explicit row, and the explicit rows);
// each cell is handed over exactly once, by one thread, in no particular
// order.  A warp has two chunks in flight, and fetches the neighbour tables
// of its next two chunks while it computes the current ones.
template <class T, class Epi>
__device__ __forceinline__ void spmv_range(const MeshView& M, const T* __restrict__ z, int64_t b0, int64_t b1,
                                           Epi& epi) {
  using Pre = typename Epi::Pre;
  constexpr int V = Lane<T>::V, CB = Lane<T>::CB;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const Lane<T> L(lane);
  const int64_t nch = (b1 - b0 + CB - 1) / CB;
  auto block_of = [&](int64_t c) { return b0 + c * CB + L.bl; };
  auto nbr_of = [&](int64_t c) {
    const int64_t blk = block_of(c);
    return (c < nch && blk < b1) ? block_nbr(M, blk) : make_int4(kWall, kWall, kWall, kWall);
  };
  int64_t c = w;
  int4 na = nbr_of(c), nbb = nbr_of(c + nw);
  for (; c < nch; c += 2 * nw) {
    const int64_t ca = c, cb = c + nw;
    const int64_t ba = block_of(ca), bb = block_of(cb);
    const bool va = ba < b1, vb = cb < nch && bb < b1;
    ChunkGather<T> ga, gb;
    gather_chunk<T>(na, ba, va, z, L, ga);
    gather_chunk<T>(nbb, bb, vb, z, L, gb);
    const int64_t ia = ba * kBLEN + L.cell0, ib = bb * kBLEN + L.cell0;
    Pre pa{}, pb{};
    if (va) pa = epi.load(ia);
    if (vb) pb = epi.load(ib);
    na = nbr_of(c + 2 * nw);
    nbb = nbr_of(c + 3 * nw);
    T y[V];
    stencil_chunk<T>(ga, L, y);
    if (va) {
      const unsigned mk = (unsigned)(explicit_mask<T>(M, ba, ga.nb) >> L.cell0) & ((1u << V) - 1u);
      if (mk == 0u) {
        epi.vec(ia, y, pa);
      } else {
#pragma unroll
        for (int j = 0; j < V; ++j)
          if (!((mk >> j) & 1u)) epi.one(ia + j, y[j], pa, j);
      }
    }
    stencil_chunk<T>(gb, L, y);
    if (vb) {
      const unsigned mk = (unsigned)(explicit_mask<T>(M, bb, gb.nb) >> L.cell0) & ((1u << V) - 1u);
      if (mk == 0u) {
        epi.vec(ib, y, pb);
      } else {
#pragma unroll
        for (int j = 0; j < V; ++j)
          if (!((mk >> j) & 1u)) epi.one(ib + j, y[j], pb, j);
      }
    }
  }
  if (b1 > b0) {
    const int r0 = __ldg(M.xbase + b0), r1 = __ldg(M.xbase + b1);
    for (int r = r0 + threadIdx.x; r < r1; r += blockDim.x) {
      const int64_t i = (int64_t)__ldg(M.rowcell + r);
      const Pre pre = epi.load1(i);
      epi.one(i, explicit_row<T>(M, r, z), pre, 0);
    }
  }
}

}  // namespace cup2d
