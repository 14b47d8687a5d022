// Block-structured SpMV: y = A z over a range of 8x8 blocks.
//
// Stencil rows: the range passes (spmv_range) move 16 bytes per lane (see
// Lane below); in-row and vertical neighbours come from the warp's block row
// in shared memory, cells across a same-level face from the neighbour
// block, and a wall face contributes no flux.  Rows of cells on a
// coarse/fine face are skipped there.
//
// Explicit rows (coarse/fine faces): stored as CSR, numbered contiguously by
// block; every thread of the CTA takes rows of the CTA's row range.
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

__device__ __forceinline__ int4 block_nbr(const MeshView& M, int blk) {
  return __ldg(reinterpret_cast<const int4*>(M.nbr) + blk);
}

template <class T>
__device__ __forceinline__ unsigned long long explicit_mask(const MeshView& M, int blk, const int4& nb) {
  if (nb.x == kExplicit || nb.y == kExplicit || nb.z == kExplicit || nb.w == kExplicit) return __ldg(M.xmask + blk);
  return 0ull;
}

// Entries of an explicit row whose loads are issued as one batch: 8 in FP32,
// 4 in FP64 (whose batch kernels run at 80 registers a thread).
template <class T>
constexpr int kRowBatch = sizeof(T) == 4 ? 8 : 4;

// sum_k vals[k] z[xcol[k]] of an explicit row, k ascending over [k0, k1).
// The columns and values of the first kRowBatch entries are requested
// together, then their gathers together (two dependent round trips for a
// row of up to kRowBatch entries; coarse/fine rows hold 7-8); the rest of a
// longer row follows in a plain loop.  The sum is accumulated in k order, as the
// assembled row is.
template <class T>
__device__ __forceinline__ T explicit_row(const MeshView& M, const T* __restrict__ z, int k0, int k1) {
  constexpr int W = kRowBatch<T>;
  const T* __restrict__ vals = row_vals<T>(M);
  int col[W];
  T v[W], g[W];
#pragma unroll
  for (int j = 0; j < W; ++j) {
    const bool in = k0 + j < k1;
    col[j] = in ? __ldg(M.xcol + k0 + j) : 0;
    v[j] = in ? __ldg(vals + k0 + j) : T(0);
  }
#pragma unroll
  for (int j = 0; j < W; ++j) g[j] = k0 + j < k1 ? ldcg(z + col[j]) : T(0);
  T acc = T(0);
#pragma unroll
  for (int j = 0; j < W; ++j)
    if (k0 + j < k1) acc += v[j] * g[j];
  for (int k = k0 + W; k < k1; ++k) acc += __ldg(vals + k) * ldcg(z + __ldg(M.xcol + k));
  return acc;
}

// ------------------------------------------------ 16-byte lane layout ----
//
// The range passes move 16 bytes per lane and access: V = 4 consecutive
// cells of a row for FP32 (a warp covers two blocks, 16 lanes each), V = 2
// for FP64 (a warp covers one block).  A "chunk" is the CB blocks one warp
// access covers.  Lane l of a chunk owns cells cell0 .. cell0 + V - 1 of
// block bl, row iy; in-row neighbours of other lanes and the rows above and
// below come from the warp's block row in shared memory, cells across a
// block face from the neighbour block.

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

// N consecutive values from shared memory as one 16-byte vector.
template <int N, class T>
__device__ __forceinline__ void lds16(const T* p, T (&v)[N]) {
  static_assert(N * sizeof(T) == 16, "one 16-byte vector");
  if constexpr (sizeof(T) == 4) {
    const float4 a = *reinterpret_cast<const float4*>(p);
    v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
  } else {
    const double2 a = *reinterpret_cast<const double2*>(p);
    v[0] = a.x; v[1] = a.y;
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

// Loads of the lane's cells and of the halos across block faces.
template <class T>
__device__ __forceinline__ void gather_chunk(const int4& nb, int blk, bool valid, const T* __restrict__ z,
                                             const Lane<T>& L, ChunkGather<T>& g) {
  constexpr int V = Lane<T>::V;
  g.nb = nb;
  g.xm = g.xp = T(0);
#pragma unroll
  for (int j = 0; j < V; ++j) g.z[j] = g.ym[j] = g.yp[j] = T(0);
  if (!valid) return;
  ldv<V>(z + blk * kBLEN + L.cell0, g.z);
  if (L.ix0 == 0 && nb.x >= 0) g.xm = ldcg(z + nb.x * kBLEN + L.iy * kBS + (kBS - 1));
  if (L.ix0 + V == kBS && nb.y >= 0) g.xp = ldcg(z + nb.y * kBLEN + L.iy * kBS);
  if (L.iy == 0 && nb.z >= 0) ldv<V>(z + nb.z * kBLEN + (kBS - 1) * kBS + L.ix0, g.ym);
  if (L.iy == kBS - 1 && nb.w >= 0) ldv<V>(z + nb.w * kBLEN + L.ix0, g.yp);
}

// Stencil rows of the lane's cells, summed left, right, below, above as the
// assembled rows are (explicit rows get meaningless values).  The warp
// writes its chunk to its block row in shared memory (`row`: kBLEN values,
// 16-byte aligned) and reads the in-block neighbours back from there (a
// lane's row above and below as whole vectors); cells across a block face
// come from the halo loads.  All lanes of the warp take part.  Shuffling the
// neighbours instead took more instructions (two per FP64 value) and kept
// more registers live: measured 8 % slower on the mixed batch.
template <class T>
__device__ __forceinline__ void stencil_chunk_smem(const ChunkGather<T>& g, const Lane<T>& L, T* row,
                                                   T (&y)[Lane<T>::V]) {
  constexpr int V = Lane<T>::V;
  stv<V>(row + L.cell0, g.z);
  __syncwarp();
  const bool has_l = L.ix0 > 0 || g.nb.x >= 0, has_r = L.ix0 + V < kBS || g.nb.y >= 0;
  const bool has_d = L.iy > 0 || g.nb.z >= 0, has_u = L.iy < kBS - 1 || g.nb.w >= 0;
  const T vl = L.ix0 > 0 ? row[L.cell0 - 1] : g.xm;
  const T vr = L.ix0 + V < kBS ? row[L.cell0 + V] : g.xp;
  T dn[V], up[V];
  if (L.iy > 0) {
    const T* p = row + L.cell0 - kBS;
#pragma unroll
    for (int j = 0; j < V; ++j) dn[j] = p[j];
  } else {
#pragma unroll
    for (int j = 0; j < V; ++j) dn[j] = g.ym[j];
  }
  if (L.iy < kBS - 1) {
    const T* p = row + L.cell0 + kBS;
#pragma unroll
    for (int j = 0; j < V; ++j) up[j] = p[j];
  } else {
#pragma unroll
    for (int j = 0; j < V; ++j) up[j] = g.yp[j];
  }
  __syncwarp();
#pragma unroll
  for (int j = 0; j < V; ++j) {
    T a = T(0);
    int n = 0;
    if (j > 0) { a += g.z[j - 1]; n++; } else if (has_l) { a += vl; n++; }
    if (j < V - 1) { a += g.z[j + 1]; n++; } else if (has_r) { a += vr; n++; }
    if (has_d) { a += dn[j]; n++; }
    if (has_u) { a += up[j]; n++; }
    y[j] = a - T(n) * g.z[j];
  }
}

template <class T, class Epi>
__device__ __forceinline__ void chunk_epilogue(const MeshView& M, const ChunkGather<T>& g, const Lane<T>& L,
                                               int blk, bool valid, const typename Epi::Pre& pre, Epi& epi,
                                               T* row) {
  constexpr int V = Lane<T>::V;
  T y[V];
  stencil_chunk_smem<T>(g, L, row, y);
  if (!valid) return;
  const int i0 = blk * kBLEN + L.cell0;
  const unsigned mk = (unsigned)(explicit_mask<T>(M, blk, g.nb) >> L.cell0) & ((1u << V) - 1u);
  if (mk == 0u) {
    epi.vec(i0, y, pre);
  } else {
#pragma unroll
    for (int j = 0; j < V; ++j)
      if (!((mk >> j) & 1u)) epi.one(i0 + j, y[j], pre, j);
  }
}

// y = A z: the stencil rows of blocks [b0, b1) and the explicit rows
// [r0, r1), by the whole CTA, in the 16-byte layout; `row` is the lane's
// block row of the warp's shared-memory scratch.  The epilogue functor
// provides
//   Pre load(i0) / Pre load1(i)  operands of the lane's V cells from i0 (or
//                                of one cell i, as element 0), loaded with
//                                the gather, before y is known;
//   vec(i0, y[V], pre)           the V cells (all stencil rows);
//   one(i, y, pre, j)            cell i, element j of pre (lanes owning an
//                                explicit row, and the explicit rows);
// each cell of the ranges is handed over exactly once, by one thread, in no
// particular order.  A warp takes one chunk (CB consecutive blocks) per step
// and fetches the neighbour table of its next chunk while it computes the
// current one; the halos across block faces are loaded from the neighbours
// (one chunk in flight per warp keeps the solver kernels' register state
// small: two chunks with halos shuffled between Morton siblings spilled more
// and measured 10 % slower on the mixed batch).  The explicit rows' offsets
// are fetched before the stencil loop.
template <class T, class Epi>
__device__ __forceinline__ void spmv_range(const MeshView& M, const T* __restrict__ z, int b0, int b1,
                                           int r0, int r1, Epi& epi, T* row) {
  using Pre = typename Epi::Pre;
  constexpr int CB = Lane<T>::CB;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const Lane<T> L(lane);
  // explicit rows: this thread's first row, its offsets and cell, early
  int r = r0 + threadIdx.x;
  int k0 = 0, k1 = 0;
  int cell = 0;
  if (r < r1) {
    k0 = __ldg(M.xptr + r);
    k1 = __ldg(M.xptr + r + 1);
    cell = __ldg(M.rowcell + r);
  }
  const int nch = (b1 - b0 + CB - 1) / CB;
  auto nbr_of = [&](int blk) {
    return blk < b1 ? block_nbr(M, blk) : make_int4(kWall, kWall, kWall, kWall);
  };
  int ch = w;
  int4 na = nbr_of(b0 + ch * CB + L.bl);
  for (; ch < nch; ch += nw) {
    const int ba = b0 + ch * CB + L.bl;
    const bool va = ba < b1;
    ChunkGather<T> ga;
    gather_chunk<T>(na, ba, va, z, L, ga);
    Pre pa{};
    if (va) pa = epi.load(ba * kBLEN + L.cell0);
    na = nbr_of(b0 + (ch + nw) * CB + L.bl);
    chunk_epilogue<T>(M, ga, L, ba, va, pa, epi, row);
  }
  for (; r < r1; r += blockDim.x) {
    // the next row's offsets are requested before this row's gathers
    const int rn = r + blockDim.x;
    int k0n = 0, k1n = 0, celln = 0;
    if (rn < r1) {
      k0n = __ldg(M.xptr + rn);
      k1n = __ldg(M.xptr + rn + 1);
      celln = __ldg(M.rowcell + rn);
    }
    const Pre pre = epi.load1(cell);
    epi.one(cell, explicit_row<T>(M, z, k0, k1), pre, 0);
    k0 = k0n;
    k1 = k1n;
    cell = celln;
  }
}

// ------------------------------------------- staged SpMV (passes B, D) ----
//
// The SpMV passes of the solve move 12-24 bytes per cell and were bound by
// how many loads a warp keeps in flight: with the operands gathered into
// registers a warp has one chunk outstanding.  Here every lane issues its
// chunk's copies with cp.async (16-byte cells of the operand z and of the
// epilogue's vector, the halo values across the block faces) into a
// per-warp ring of kSpmvStages chunk slots in shared memory, kSpmvStages - 1 chunks
// ahead of the one it computes; copies in flight hold no registers.  The
// rows are then summed from shared memory in the same order as
// stencil_chunk_smem (so both give the same bits).  The neighbour table of
// the next chunk to issue is read into registers one step ahead (its halo
// addresses depend on it).  The explicit rows are done between the first
// copies and the first chunk, so that their dependent loads (offsets,
// columns, gathered z) overlap the copies in flight.

constexpr int kSpmvStages = 2;

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// cp.async of B bytes (4, 8 or 16; both addresses B-aligned); n < B copies n
// bytes and zero-fills the rest (n = 0: nothing is read).
template <int B>
__device__ __forceinline__ void cp_async_n(void* dst, const void* src, int n) {
  if constexpr (B == 16)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_u32(dst)), "l"(src), "r"(n) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;" ::"r"(smem_u32(dst)), "l"(src), "n"(B), "r"(n)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit_group() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait_n() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// One warp's ring of chunk slots.
template <class T>
struct SpmvStage {
  static constexpr int CB = Lane<T>::CB;
  alignas(16) T z[kSpmvStages][CB * kBLEN];
  alignas(16) T op[kSpmvStages][CB * kBLEN];
  alignas(16) T halo[kSpmvStages][CB][4][kBS];  // 0 Xm (col 7 of the left block), 1 Xp (col 0), 2 Ym (row 7), 3 Yp (row 0)
  alignas(16) int4 nb[kSpmvStages][CB];
};

// y = A z over blocks [b0, b1) and explicit rows [r0, r1) with the epilogue
// operand `op` (the vector Epi's dot products read) staged beside z.  Epi
// provides struct Pre { T v[V]; }, load1(i) for the explicit rows, vec() and
// one() as for spmv_range.  `st` is this warp's stage ring.
template <class T, class Epi>
__device__ __forceinline__ void spmv_range_staged(const MeshView& M, const T* __restrict__ z,
                                                  const T* __restrict__ op, int b0, int b1, int r0, int r1,
                                                  Epi& epi, SpmvStage<T>& st) {
  using Pre = typename Epi::Pre;
  constexpr int V = Lane<T>::V, CB = Lane<T>::CB, S = kSpmvStages;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const Lane<T> L(lane);
  // explicit rows: this thread's first row, its offsets and cell, early
  int r = r0 + threadIdx.x;
  int k0 = 0, k1 = 0;
  int cell = 0;
  if (r < r1) {
    k0 = __ldg(M.xptr + r);
    k1 = __ldg(M.xptr + r + 1);
    cell = __ldg(M.rowcell + r);
  }
  const int nch = (b1 - b0 + CB - 1) / CB;
  auto blk_of = [&](int k) { return b0 + (w + k * nw) * CB + L.bl; };
  auto nbr_of = [&](int k) {
    const int blk = blk_of(k);
    return blk < b1 ? block_nbr(M, blk) : make_int4(kWall, kWall, kWall, kWall);
  };
  // the copies of the warp's k-th chunk into slot k % S
  auto issue = [&](int k, const int4& nb) {
    const int s = k % S, blk = blk_of(k);
    const bool valid = blk < b1;
    const int own = valid ? blk : b0;  // an address inside the range for zero-fills
    cp_async_n<16>(&st.z[s][L.bl * kBLEN + L.cell0], z + own * kBLEN + L.cell0, valid ? 16 : 0);
    cp_async_n<16>(&st.op[s][L.bl * kBLEN + L.cell0], op + own * kBLEN + L.cell0, valid ? 16 : 0);
    if (L.sub == 0) st.nb[s][L.bl] = nb;
    if (L.ix0 == 0 && nb.x >= 0)
      cp_async_n<sizeof(T)>(&st.halo[s][L.bl][0][L.iy], z + nb.x * kBLEN + L.iy * kBS + (kBS - 1), sizeof(T));
    if (L.ix0 + V == kBS && nb.y >= 0)
      cp_async_n<sizeof(T)>(&st.halo[s][L.bl][1][L.iy], z + nb.y * kBLEN + L.iy * kBS, sizeof(T));
    if (L.iy == 0 && nb.z >= 0)
      cp_async_n<16>(&st.halo[s][L.bl][2][L.ix0], z + nb.z * kBLEN + (kBS - 1) * kBS + L.ix0, 16);
    if (L.iy == kBS - 1 && nb.w >= 0)
      cp_async_n<16>(&st.halo[s][L.bl][3][L.ix0], z + nb.w * kBLEN + L.ix0, 16);
    cp_async_commit_group();
  };
  const int K = w < nch ? (nch - w + nw - 1) / nw : 0;  // chunks of this warp
  // chunks 0 .. S-2 ahead (past the end: zero-fills only, an empty group)
  if (K > 0) {
#pragma unroll
    for (int k = 0; k < S - 1; ++k) issue(k, nbr_of(k));
  }
  int4 nn = nbr_of(S - 1);
  // the explicit rows while the first chunks' copies are in flight: their
  // dependent loads (offsets, columns, gathered z) overlap the copies
  for (; r < r1; r += blockDim.x) {
    // the next row's offsets are requested before this row's gathers
    const int rn = r + blockDim.x;
    int k0n = 0, k1n = 0, celln = 0;
    if (rn < r1) {
      k0n = __ldg(M.xptr + rn);
      k1n = __ldg(M.xptr + rn + 1);
      celln = __ldg(M.rowcell + rn);
    }
    const Pre pre = epi.load1(cell);
    epi.one(cell, explicit_row<T>(M, z, k0, k1), pre, 0);
    k0 = k0n;
    k1 = k1n;
    cell = celln;
  }
  for (int k = 0; k < K; ++k) {
    cp_async_wait_n<S - 2>();  // this lane's copies of chunk k have landed
    __syncwarp();              // ... and every lane's; slot (k+S-1)%S was last read in step k-1
    issue(k + S - 1, nn);
    nn = nbr_of(k + S);
    const int s = k % S, blk = blk_of(k);
    if (blk >= b1) continue;
    const T* zs = &st.z[s][L.bl * kBLEN];
    const T(*h)[kBS] = st.halo[s][L.bl];
    const int4 nb = st.nb[s][L.bl];
    T zc[V], dn[V], up[V];
    Pre pre;
    lds16<V>(zs + L.cell0, zc);
    lds16<V>(&st.op[s][L.bl * kBLEN + L.cell0], pre.v);
    const bool has_l = L.ix0 > 0 || nb.x >= 0, has_r = L.ix0 + V < kBS || nb.y >= 0;
    const bool has_d = L.iy > 0 || nb.z >= 0, has_u = L.iy < kBS - 1 || nb.w >= 0;
    const T vl = L.ix0 > 0 ? zs[L.cell0 - 1] : h[0][L.iy];
    const T vr = L.ix0 + V < kBS ? zs[L.cell0 + V] : h[1][L.iy];
    lds16<V>(L.iy > 0 ? zs + L.cell0 - kBS : &h[2][L.ix0], dn);
    lds16<V>(L.iy < kBS - 1 ? zs + L.cell0 + kBS : &h[3][L.ix0], up);
    T y[V];
#pragma unroll
    for (int j = 0; j < V; ++j) {
      T a = T(0);
      int n = 0;
      if (j > 0) { a += zc[j - 1]; n++; } else if (has_l) { a += vl; n++; }
      if (j < V - 1) { a += zc[j + 1]; n++; } else if (has_r) { a += vr; n++; }
      if (has_d) { a += dn[j]; n++; }
      if (has_u) { a += up[j]; n++; }
      y[j] = a - T(n) * zc[j];
    }
    const int i0 = blk * kBLEN + L.cell0;
    const unsigned mk = (unsigned)(explicit_mask<T>(M, blk, nb) >> L.cell0) & ((1u << V) - 1u);
    if (mk == 0u) {
      epi.vec(i0, y, pre);
    } else {
#pragma unroll
      for (int j = 0; j < V; ++j)
        if (!((mk >> j) & 1u)) epi.one(i0 + j, y[j], pre, j);
    }
  }
  cp_async_wait_n<0>();  // the empty tail groups; nothing may land after return
}

}  // namespace cup2d
