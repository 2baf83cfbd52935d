// The reference's data-movement layer on virtual ranks: pack, all-to-all and
// unpack as functions of their own, and the TransBlock that chains them.
//
//   pack / unpack  KokkosFFT_Distributed_PackUnpack.hpp:439-499 (one rank's
//                  view and buffer, exactly the reference's arguments)
//   all2all        KokkosFFT_Distributed_MPI_All2All.hpp:23-58 (MPI_Alltoall
//                  over the world or a Cartesian row / column communicator,
//                  KokkosFFT_Distributed_PencilPlan.hpp:32-71), here over the
//                  concatenated buffers of all virtual ranks
//   TransBlock     KokkosFFT_Distributed_TransBlock.hpp:38-107 (pack, all2all,
//                  unpack; backward swaps the maps and axes)
//
// All of them run the same device kernels as the plans' literal programs
// (csrc/transpose.cu), so the reference's own unit-test vectors for these
// functions pin the kernels the plans use.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "dev_types.h"
#include "layout.hpp"

namespace dfft {

// Exchange group of virtual rank r: its rank within the group and the group's
// members by sub-rank.  comm_axis < 0: all ranks (the slab plans' world
// communicator).  comm_axis 0 / 1: the row / column communicator that
// MPI_Cart_sub keeps from MPI_Cart_create over the entries of cart_topology
// larger than one (row-major coordinates, no reordering).
struct ExchangeGroup {
  std::size_t sub = 0;
  std::vector<std::size_t> members;
};
ExchangeGroup exchange_group(std::size_t nprocs, const Ext& cart_topology, int comm_axis, std::size_t rank);

// Appends the per-rank geometry table of dev::XposeArgs (block starts and
// extents in layout L, sub-rank, members) for an exchange over groups of pc
// ranks.
void append_exchange_geo(std::vector<std::int64_t>& out, const Layout& L, const Ext& cart_topology, int comm_axis,
                         std::size_t pc);

// Device view of layout tables uploaded at `base`.
dev::DevLayout device_layout_at(const LayoutTables& T, const std::int64_t* base);

// pack(exec, src, dst, map, axis) of one rank: src is a view of rank D with
// extents src_extents (in its own dimension order, i.e. the local extents
// permuted by map), dst a buffer of rank D + 1 with buffer_extents.
void pack_local(const Ext& src_extents, const Ext& map, std::size_t axis, const Ext& buffer_extents, bool layout_right,
                int elem_bytes, const void* src, void* dst, cudaStream_t stream);
// unpack(exec, src, dst, map, axis) of one rank: src is the buffer, dst a
// view with extents dst_extents (permuted by map).
void unpack_local(const Ext& buffer_extents, const Ext& map, std::size_t axis, const Ext& dst_extents,
                  bool layout_right, int elem_bytes, const void* src, void* dst, cudaStream_t stream);
// all2all(send, recv, comm) of every virtual rank at once: send / recv hold
// nprocs buffers of buffer_extents, rank after rank.
void all2all_virtual(std::size_t nprocs, const Ext& buffer_extents, bool layout_right, const Ext& cart_topology,
                     int comm_axis, int elem_bytes, const void* send, void* recv, cudaStream_t stream);

// TransBlock over every virtual rank of a topology pair.
struct TransBlockDesc {
  Ext gext;                     // global extents
  Ext in_topo, out_topo;        // topologies of the forward input / output
  bool in_right = true, out_right = true;
  Ext src_map, dst_map;         // maps of the forward input / output views
  std::size_t src_axis = 0;     // forward: split on send
  std::size_t dst_axis = 0;     // forward: merged on receive
  bool view_right = true;
  int elem_bytes = 8;
  int comm_axis = -1;           // see exchange_group
  Ext cart_topology;            // see exchange_group (empty: in_topo)
};

class TransBlockExec {
 public:
  explicit TransBlockExec(const TransBlockDesc& d);
  ~TransBlockExec();
  TransBlockExec(const TransBlockExec&) = delete;
  TransBlockExec& operator=(const TransBlockExec&) = delete;

  // in / out: every rank's block concatenated (forward: in-topology blocks
  // with src_map -> out-topology blocks with dst_map; backward the reverse);
  // send / recv: nprocs buffers of buffer_extents each.
  void execute(const void* in, void* out, void* send, void* recv, bool forward, cudaStream_t stream) const;

  const Ext& buffer_extents() const { return bext_; }
  std::size_t nprocs() const { return P_; }
  const Layout& layout(bool of_input) const { return of_input ? lin_ : lout_; }

 private:
  TransBlockDesc d_;
  std::size_t P_ = 0;
  Ext bext_;
  Layout lin_, lout_;
  std::int64_t* d_tables_ = nullptr;
  dev::XposeArgs pack_[2]{}, a2a_[2]{}, unpack_[2]{};  // [0] forward, [1] backward
};

}  // namespace dfft
