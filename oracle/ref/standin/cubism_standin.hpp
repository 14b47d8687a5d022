// ORACLE — test infrastructure only.  A minimal stand-in for the parts of the
// Cubism AMR grid library that CUP2D's ExpAMRSolver.cpp and the headers it
// pulls in (source/Definitions.h, source/SimulationData.h) name.  Cubism is an
// un-vendored submodule of CUP2D, so the reference's assembly cannot be
// compiled against the real library; this header supplies the same names with
// the semantics getMat relies on (source/Poisson/ExpAMRSolver.cpp:180-313):
//
//   * BlockInfo: level, index[3], Z, Znei[3][3][3], Zparent, Zchild[2][2][2],
//     blockID, h, ptrBlock.  Z is this stand-in's own key of a block position
//     at a level (row-major, j * NX(level) + i); every Z-valued field uses the
//     same key, so lookups are consistent.  Znei wraps around the domain in
//     both directions (getMat queries all four neighbours and uses those
//     across a non-periodic wall only when the flux is periodic).
//   * Grid::Tree(level, Z): Exists() for a leaf, CheckCoarser() when an
//     ancestor is a leaf, CheckFiner() when a leaf lies below the position,
//     none of the three for a hole; rank() is 0 (one rank) for a leaf.
//   * Grid::getBlockInfoAll(level, Z): the BlockInfo of any position, created
//     on first use; leaves carry their position in the block list as
//     blockID, so the assembled rows use the caller's block order.
//   * GridBlock / ScalarElement: an 8x8 block of cells, element .s.
//
// Templates that Definitions.h only names in aliases (BlockLab,
// BlockLabNeumann, BlockLabMPI, MeshAdaptation) are empty shells.
#pragma once

#include <algorithm>
#include <array>
#include <cstdint>
#include <iostream>  // the real Cubism headers bring in <iostream>, which the
                     // reference's sources use without including it
#include <limits>
#include <map>
#include <memory>
#include <set>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include <mpi.h>

namespace cubism {

struct BlockInfo {
  long long blockID = -1;
  long long Z = 0;
  long long Znei[3][3][3] = {};
  long long Zparent = 0;
  long long Zchild[2][2][2] = {};
  double h = 0.0;
  double origin[3] = {0.0, 0.0, 0.0};
  int index[3] = {0, 0, 0};
  int level = 0;
  void* ptrBlock = nullptr;
};

class TreePosition {
 public:
  // >= 0: a leaf owned by that rank; -1: a coarser leaf covers it;
  // -2: refined; -3: nothing (a hole)
  int position = -3;
  bool Exists() const { return position >= 0; }
  int rank() const { return position; }
  bool CheckCoarser() const { return position == -1; }
  bool CheckFiner() const { return position == -2; }
};

template <typename T>
struct ScalarElement {
  T s = 0;
};

template <int dim, typename T>
struct VectorElement {
  T u[dim] = {};
};

template <int blocksize, int dim, typename TElement>
struct GridBlock {
  static constexpr int sizeX = blocksize;
  static constexpr int sizeY = blocksize;
  static constexpr int sizeZ = dim > 2 ? blocksize : 1;
  using ElementType = TElement;
  TElement data[sizeZ][sizeY][sizeX];
  TElement& operator()(int ix, int iy = 0, int iz = 0) { return data[iz][iy][ix]; }
  const TElement& operator()(int ix, int iy = 0, int iz = 0) const { return data[iz][iy][ix]; }
};

// The forest behind a grid: leaves in the caller's order, plus lazily created
// BlockInfo/TreePosition records for every queried position.
class StandinForest {
 public:
  void setup(int bpdx, int bpdy, int level_max, double extent, long long nblocks, const int32_t* level,
             const int32_t* bx, const int32_t* by) {
    bpdx_ = bpdx;
    bpdy_ = bpdy;
    level_max_ = level_max;
    extent_ = extent;
    leaves_.clear();
    all_.clear();
    tree_.clear();
    leaf_of_.clear();
    leaves_.reserve((size_t)nblocks);
    refined_.clear();
    for (long long b = 0; b < nblocks; b++) {
      const long long Z = key(level[b], bx[b], by[b]);
      leaf_of_[{level[b], Z}] = b;
      // every ancestor position of a leaf is refined
      long long i = bx[b], j = by[b];
      for (int l = level[b] - 1; l >= 0; l--) {
        i >>= 1;
        j >>= 1;
        refined_.insert({l, key(l, i, j)});
      }
    }
    for (long long b = 0; b < nblocks; b++) leaves_.push_back(make(level[b], key(level[b], bx[b], by[b])));
  }

  std::vector<BlockInfo>& leaves() { return leaves_; }
  std::array<int, 3> max_blocks() const { return {bpdx_, bpdy_, 1}; }

  BlockInfo& info(int level, long long Z) {
    auto it = all_.find({level, Z});
    if (it == all_.end()) it = all_.emplace(std::make_pair(level, Z), make(level, Z)).first;
    return it->second;
  }

  TreePosition& tree(int level, long long Z) {
    auto it = tree_.find({level, Z});
    if (it != tree_.end()) return it->second;
    TreePosition t;
    if (leaf_of_.count({level, Z})) {
      t.position = 0;
    } else {
      // refined when a leaf lies below it; "coarser" when an ancestor is a
      // leaf; neither (a hole in the forest) otherwise
      t.position = refined_.count({level, Z}) ? -2 : -3;
      long long i = Z % nx(level), j = Z / nx(level);
      for (int l = level - 1; l >= 0 && t.position == -3; l--) {
        i >>= 1;
        j >>= 1;
        if (leaf_of_.count({l, key(l, i, j)})) t.position = -1;
      }
    }
    return tree_.emplace(std::make_pair(level, Z), t).first->second;
  }

 private:
  long long nx(int level) const { return (long long)bpdx_ << level; }
  long long ny(int level) const { return (long long)bpdy_ << level; }
  long long key(int level, long long i, long long j) const { return j * nx(level) + i; }

  BlockInfo make(int level, long long Z) const {
    BlockInfo b;
    b.level = level;
    b.Z = Z;
    const long long NX = nx(level), NY = ny(level);
    const long long i = Z % NX, j = Z / NX;
    b.index[0] = (int)i;
    b.index[1] = (int)j;
    b.index[2] = 0;
    // cell spacing: the domain's longer side spans max(bpdx, bpdy) root blocks
    b.h = extent_ / ((double)std::max(bpdx_, bpdy_) * 8.0 * (double)(1ll << level));
    b.origin[0] = (double)i * 8 * b.h;
    b.origin[1] = (double)j * 8 * b.h;
    for (int dx = -1; dx <= 1; dx++)
      for (int dy = -1; dy <= 1; dy++) {
        const long long ii = ((i + dx) % NX + NX) % NX, jj = ((j + dy) % NY + NY) % NY;
        for (int dz = 0; dz < 3; dz++) b.Znei[dx + 1][dy + 1][dz] = key(level, ii, jj);
      }
    b.Zparent = level > 0 ? key(level - 1, i / 2, j / 2) : 0;
    for (int cx = 0; cx < 2; cx++)
      for (int cy = 0; cy < 2; cy++)
        for (int cz = 0; cz < 2; cz++) b.Zchild[cx][cy][cz] = key(level + 1, 2 * i + cx, 2 * j + cy);
    auto it = leaf_of_.find({level, Z});
    if (it != leaf_of_.end()) b.blockID = it->second;
    return b;
  }

  int bpdx_ = 1, bpdy_ = 1, level_max_ = 1;
  double extent_ = 1.0;
  std::vector<BlockInfo> leaves_;
  std::map<std::pair<int, long long>, BlockInfo> all_;
  std::map<std::pair<int, long long>, TreePosition> tree_;
  std::map<std::pair<int, long long>, long long> leaf_of_;
  std::set<std::pair<int, long long>> refined_;
};

template <typename Block, template <typename X> class allocator = std::allocator>
class Grid {
 public:
  using BlockType = Block;
  bool UpdateFluxCorrection = true;

  void standin_setup(int bpdx, int bpdy, int level_max, double extent, long long nblocks, const int32_t* level,
                     const int32_t* bx, const int32_t* by) {
    forest_.setup(bpdx, bpdy, level_max, extent, nblocks, level, bx, by);
    blocks_.assign((size_t)nblocks, Block{});
    auto& L = forest_.leaves();
    for (size_t b = 0; b < L.size(); b++) {
      L[b].ptrBlock = &blocks_[b];
      forest_.info(L[b].level, L[b].Z).ptrBlock = &blocks_[b];
    }
  }
  Block& standin_block(long long b) { return blocks_[(size_t)b]; }

  std::vector<BlockInfo>& getBlocksInfo() { return forest_.leaves(); }
  std::array<int, 3> getMaxBlocks() const { return forest_.max_blocks(); }
  void UpdateBlockInfoAll_States(bool = false) {}
  BlockInfo& getBlockInfoAll(int level, long long Z) { return forest_.info(level, Z); }
  TreePosition& Tree(int level, long long Z) { return forest_.tree(level, Z); }
  TreePosition& Tree(const BlockInfo& info) { return forest_.tree(info.level, info.Z); }

 private:
  StandinForest forest_;
  std::vector<Block> blocks_;
};

template <typename TGrid>
class GridMPI : public TGrid {};

template <typename TGrid, template <typename X> class allocator = std::allocator>
class BlockLab {
 public:
  virtual ~BlockLab() = default;
  virtual bool is_xperiodic() { return false; }
  virtual bool is_yperiodic() { return false; }
  virtual bool is_zperiodic() { return false; }
  virtual void _apply_bc(const BlockInfo&, const double = 0, const bool = false) {}
};

template <typename TGrid, int dim, template <typename X> class allocator = std::allocator>
class BlockLabNeumann : public BlockLab<TGrid, allocator> {};

template <typename MyBlockLab>
class BlockLabMPI : public MyBlockLab {};

template <typename TLab>
class MeshAdaptation {};

class Profiler {};
class ArgumentParser {};
struct StencilInfo {};

}  // namespace cubism
