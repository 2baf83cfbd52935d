// Layouts: how a global array of the FFT index space is stored in a buffer.
//
// A layout is a topology of virtual ranks plus, per rank, a local block with
// an axis permutation ("map": local dim i holds logical axis map[i]) in C or
// Fortran memory order.  Blocks are concatenated in rank order.  With the
// topology all ones it is a plain (optionally permuted) global array.
//
// For the device, a layout becomes lookup tables:
//   separable form (every rank has the same local extents, i.e. every split
//   axis divides evenly, or padded blocks): offset(c) = sum_k off_k[c_k];
//   general form (ragged bins):
//     r = sum_k rk_k[c_k];  offset(c) = rbase[r] + sum_k loc_k[c_k] * rstride[r][k].
#pragma once

#include <cstdint>
#include <vector>

#include "plan_core.hpp"

namespace dfft {

constexpr int kMaxRank = 4;

struct Layout {
  Ext gext;                // global extents (logical axis order)
  Ext topo;                // ranks per axis
  bool rank_right = true;  // rank_to_coord order
  Ext map;                 // local dim i <-> logical axis map[i]
  bool view_right = true;  // memory order of the local blocks
  bool complex = true;     // element type: complex or real
  // Padded blocks (an exchange buffer of one rank): when not empty, every
  // block is stored with these extents (logical axis order) instead of its
  // own local extents, and block r starts at r * prod(pad); the entries past
  // a block's local extents are padding that no kernel reads or writes.
  Ext pad;

  std::size_t nprocs() const { return total_size(topo); }
  bool operator==(const Layout& o) const {
    return gext == o.gext && topo == o.topo && rank_right == o.rank_right && map == o.map &&
           view_right == o.view_right && complex == o.complex && pad == o.pad;
  }
  bool operator!=(const Layout& o) const { return !(*this == o); }
};

// Geometry of one rank's block.
struct RankBlock {
  Ext coords, starts, local;  // logical axis order
  Ext mapped;                 // local extents in memory-dim order (local[map[i]])
  Ext stride;                 // element stride of each logical axis
  std::size_t size = 0;
  std::size_t base = 0;  // element offset of the block in the buffer
};

std::vector<RankBlock> layout_blocks(const Layout& L);
// Elements of the buffer that holds the layout (padding included).
std::size_t layout_elements(const Layout& L);
bool layout_separable(const Layout& L);
// Logical axis with unit stride (the fastest-varying axis of every block).
std::size_t layout_fast_axis(const Layout& L);

// Every split axis divides evenly (the blocks along it have equal extents).
bool layout_even(const Layout& L);

// Host image of the device tables of a layout, packed in one int64 array.
struct LayoutTables {
  int mode = 0;  // 0 separable, 1 general
  int nd = 0;
  std::vector<std::int64_t> data;
  // offsets (in int64 units) into `data`
  std::int64_t off[kMaxRank] = {0, 0, 0, 0};  // mode 0: off_k, length gext[k]
  std::int64_t rk[kMaxRank] = {0, 0, 0, 0};   // mode 1
  std::int64_t loc[kMaxRank] = {0, 0, 0, 0};  // mode 1
  std::int64_t rbase = 0, rstride = 0;        // mode 1
};
LayoutTables build_layout_tables(const Layout& L);

}  // namespace dfft
