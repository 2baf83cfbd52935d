// Host-side planning for the distributed 3D FFT execute path.
//
// This is a runtime-rank restatement of the reference library's planning
// layer (topology chains, block analyses, extents, mappings).  Every function
// cites the reference header it follows (paths relative to the reference's
// `distributed/src/`).  There is no MPI here: the ranks of a topology are
// virtual, and the per-rank results that the reference gathers with
// MPI_Allgather / MPI_Allreduce are evaluated for every rank on the host.
#pragma once

#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

namespace dfft {

using Ext = std::vector<std::size_t>;  // extents, topologies, maps (size = view rank)

// Error raised by planning and validation; the C-ABI turns it into a status.
struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

// Status codes shared with include/dfft.h.
enum : int {
  kOk = 0,
  kErrInvalidArgument = 1,
  kErrInvalidTopology = 2,
  kErrInvalidExtents = 3,
  kErrUnsupported = 4,
  kErrCuda = 5,
  kErrAlloc = 6,
  kErrInternal = 7,
  kErrTimeout = 8,
};

[[noreturn]] void fail(int code, const std::string& msg);

// KokkosFFT_Distributed_Types.hpp:19-49
enum class TopologyType { Empty, Shared, Slab, Pencil, Brick, Invalid };
enum class BlockType { Transpose, FFT };

// KokkosFFT_Distributed_Types.hpp:61-154 (BlockInfo<DIM>)
struct BlockInfo {
  Ext in_topology, out_topology;
  Ext in_extents, out_extents;
  Ext buffer_extents;  // size rank+1
  Ext in_map, out_map;
  std::size_t in_axis = 0, out_axis = 0;
  std::size_t fft_dim = 0;
  std::size_t comm_axis = 0;
  BlockType block_type = BlockType::FFT;
  std::size_t block_idx = 0;
  bool operator==(const BlockInfo& o) const;
};

// ---- container helpers (KokkosFFT_Distributed_ContainerAnalyses.hpp) ----
std::size_t total_size(const Ext& v);
std::size_t count_non_ones(const Ext& v);                                        // :19-30
std::vector<std::size_t> extract_different_indices(const Ext& a, const Ext& b);  // :38-55
std::vector<std::size_t> extract_different_value_set(const Ext& a, const Ext& b);  // :64-81
std::vector<std::size_t> extract_non_one_indices(const Ext& a, const Ext& b);    // :90-106
Ext extract_non_one_values(const Ext& a);                                        // :114-126
bool has_identical_non_ones(const Ext& non_ones);                                // :135-147
Ext swap_elements(const Ext& arr, std::size_t i, std::size_t j);                 // :158-164
Ext merge_topology(const Ext& in, const Ext& out);                               // :182-229
std::size_t diff_topology(const Ext& in, const Ext& out);                        // :240-258

// ---- topology analyses (KokkosFFT_Distributed_Topologies.hpp) ----
TopologyType to_topology_type(const Ext& topo);                        // :26-41
TopologyType get_common_topology_type(const std::vector<Ext>& topos);  // :66-89
void slab_in_out_axes(const Ext& in, const Ext& out, std::size_t& in_axis,
                      std::size_t& out_axis);  // :109-133
void pencil_in_out_axes(const Ext& in, const Ext& out, std::size_t& in_axis,
                        std::size_t& out_axis);  // :153-175
Ext propose_mid_array(const Ext& in, const Ext& out);  // :191-242
std::vector<std::vector<std::size_t>> decompose_axes(const std::vector<Ext>& topos,
                                                     const Ext& axes);  // :259-331
std::size_t compute_trans_axis(const Ext& in, const Ext& out,
                               std::size_t first_non_one);  // :352-399
std::vector<Ext> get_all_slab_topologies(const Ext& in, const Ext& out,
                                         const Ext& axes);  // :421-618
struct PencilChain {
  std::vector<Ext> topologies;
  std::vector<std::size_t> trans_axes;
  std::vector<std::size_t> layouts;  // 1 = LayoutRight rank order, 0 = LayoutLeft
};
PencilChain get_all_pencil_topologies(const Ext& in, bool in_right, const Ext& out, bool out_right,
                                      const Ext& axes);  // :645-811

// ---- layout math ----
// KokkosFFT_Distributed_PackUnpack.hpp:40-46
void bin_mapping(std::int64_t n, std::int64_t nbins, std::int64_t ibin, std::int64_t& start,
                 std::int64_t& length);
// KokkosFFT_Distributed_MPI_Extents.hpp:492-523
Ext rank_to_coord(const Ext& topology, std::size_t rank, bool layout_right);
// KokkosFFT_Distributed_MPI_Extents.hpp:202-233
Ext compute_local_extents(const Ext& extents, const Ext& topology, const Ext& map, std::size_t rank,
                          bool layout_right);
// Starts of a rank's block: KokkosFFT_Distributed_MPI_Extents.hpp:56-98,159-169
Ext compute_local_starts(const Ext& extents, const Ext& topology, std::size_t rank, bool layout_right);
// KokkosFFT_Distributed_Extents.hpp:35-61
Ext compute_buffer_extents(const Ext& extents, const Ext& in_topo, const Ext& out_topo,
                           bool view_layout_right);
// KokkosFFT_Distributed_Extents.hpp:116-137
Ext compute_fft_extents(const Ext& in_extents, const Ext& out_extents, const Ext& axes);
// KokkosFFT_Distributed_Mapping.hpp:39-100
Ext permute_map_by_axes(const Ext& src_map, const Ext& axes, bool view_layout_right);
// kokkos-fft Impl::get_map_axes, restated as permute_map_by_axes on the identity
Ext get_map_axes(std::size_t rank, const Ext& axes, bool view_layout_right);
Ext compute_mapped_extents(const Ext& extents, const Ext& map);
Ext identity_map(std::size_t rank);
std::size_t get_index(const Ext& v, std::size_t value);  // position of value, v.size() if absent

// ---- block analyses (KokkosFFT_Distributed_BlockAnalyses.hpp) ----
struct BlockAnalyses {
  std::vector<BlockInfo> blocks;
  std::size_t max_buffer_size = 0;  // this rank's max (elements of the real type)
};

// SlabBlockAnalysesInternal (:391-445) for one virtual rank.
BlockAnalyses slab_block_analyses(const Ext& in_extents, const Ext& gin, const Ext& gout, const Ext& in_topo,
                                  const Ext& out_topo, const Ext& axes, bool real_input, bool view_layout_right,
                                  std::size_t rank);
// PencilBlockAnalysesInternal (:447-506) for one virtual rank.
BlockAnalyses pencil_block_analyses(const Ext& in_extents, const Ext& gin, const Ext& gout, const Ext& in_topo,
                                    bool in_right, const Ext& out_topo, bool out_right, const Ext& axes,
                                    bool real_input, bool view_layout_right, std::size_t rank);

// propose_transpose_block (KokkosFFT_Distributed_BlockAnalyses.hpp:93-136):
// one transpose block and its max buffer size (elements of the real type).
BlockInfo propose_transpose(const Ext& map, const Ext& in_topo, const Ext& out_topo, const Ext& in_extents,
                            const Ext& global_extents, const Ext& axes, std::size_t rank, bool is_layout_right,
                            bool is_last, std::size_t in_axis, std::size_t out_axis, std::size_t comm_axis,
                            std::size_t block_idx, std::size_t size_factor, bool view_layout_right,
                            std::size_t* max_buffer_size);

// Validation of the global extents for a transform (are_valid_extents,
// KokkosFFT_Distributed_MPI_Extents.hpp:322-417).  `real_input` selects R2C.
void check_valid_extents(const Ext& gin, const Ext& gout, const Ext& axes, bool real_input,
                         bool view_layout_right);

std::string ext_str(const Ext& e);

}  // namespace dfft
