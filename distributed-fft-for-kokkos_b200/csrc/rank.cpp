// Per-rank programs: the block sequence of ONE world rank, for one process
// per GPU with a real all-to-all between the processes.
//
// The reference runs every rank's InternalPlan on its own local views and
// moves data with TransBlock (pack, MPI_Alltoall / ncclAllToAll over the
// world or a Cartesian row / column communicator, unpack;
// KokkosFFT_Distributed_TransBlock.hpp:76-107,
// KokkosFFT_Distributed_NCCL_All2All.hpp:21-89,
// KokkosFFT_Distributed_PencilPlan.hpp:32-71).  Here a direction of one
// rank's program is a chain of segments separated by exchanges:
//
//   * the local array of every topology of the chain is kept in logical axis
//     order (the reference's local transposes only change which axes are
//     innermost; the pack buffer is indexed by logical axes whatever the
//     source order, so the exchanged bytes are the reference's own);
//   * the FFT stage that ends a segment writes its lines straight into the
//     send buffer in the reference's [group size, buffer extents] order (the
//     pack folded into the stage's stores), and the first stage of the next
//     segment reads the recv buffer in place (the unpack folded into its
//     loads): both are padded layouts over the rank's local extents, split
//     into group-size bins along the exchanged axis;
//   * where the register kernels cannot address such a side (a buffer split
//     along the stage's own FFT axis), the stage runs on a plain local array
//     and a copy stage does the pack or unpack;
//   * the caller moves the send buffer to the recv buffer with its own
//     communicator (equal chunks of elements x element bytes / group size).
#include <cstring>
#include <string>

#include "plan.hpp"

namespace dfft {

// Rank d_.rank's local array in chain topology k, logical axis order.
Layout Plan::rank_layout(std::size_t k, bool complex) const {
  const std::size_t D = d_.gin.size();
  Layout L;
  L.gext = compute_local_extents(complex ? d_.gout : d_.gin, chain_.at(k), identity_map(D),
                                 static_cast<std::size_t>(d_.rank), chain_layouts_.at(k) != 0);
  L.topo.assign(D, 1);
  L.map = identity_map(D);
  L.view_right = d_.view_right;
  L.complex = complex;
  return L;
}

// The exchange buffer of transpose block b seen from the local array of
// chain topology k: group-size bins along split_axis (bin p holds what goes
// to / comes from group member p), every bin padded to the block's buffer
// extents (the reference's pack / unpack buffer).
Layout Plan::rank_buffer_layout(std::size_t k, bool complex, std::size_t split_axis, const BlockInfo& b) const {
  Layout L = rank_layout(k, complex);
  const std::size_t D = L.gext.size();
  const std::size_t pc = d_.view_right ? b.buffer_extents.front() : b.buffer_extents.back();
  L.topo[split_axis] = pc;
  L.pad.assign(D, 0);
  for (std::size_t i = 0; i < D; ++i) L.pad[i] = b.buffer_extents[d_.view_right ? i + 1 : i];
  for (const RankBlock& rb : layout_blocks(L))
    for (std::size_t i = 0; i < D; ++i)
      if (rb.local[i] > L.pad[i]) fail(kErrInternal, "a pack bin is larger than the buffer extents");
  return L;
}

ExchangeGroup Plan::exchange_group_of(bool forward, std::size_t k, std::size_t rank) const {
  const auto& xs = xch_[forward ? 0 : 1];
  if (k >= xs.size()) fail(kErrInvalidArgument, "exchange index out of range");
  if (rank >= nprocs()) fail(kErrInvalidArgument, "rank must be less than topology size.");
  return exchange_group(nprocs(), d_.in_topo, xs[k].comm_axis, rank);
}

Ext Plan::rank_local_extents(int which) const {
  const Layout& L = which == 0 ? lin_ : lout_;
  return compute_local_extents(L.gext, L.topo, identity_map(L.gext.size()), static_cast<std::size_t>(d_.rank),
                               L.rank_right);
}

// Host side of a direction: one Exchange per transpose block, in execution
// order (forward: block order; backward: reversed).
void Plan::rank_exchanges(bool forward) {
  auto& xs = xch_[forward ? 0 : 1];
  xs.clear();
  const std::size_t r = static_cast<std::size_t>(d_.rank), D = d_.gin.size();
  const auto& blocks = per_rank_.at(r).blocks;
  const std::size_t nbl = blocks.size();
  // the rank's blocks at both ends of the chain must be its input / output blocks
  const bool c0 = chain_layouts_.at(0) != 0, c1 = chain_layouts_.back() != 0;
  if (compute_local_starts(d_.gin, chain_.front(), r, c0) != compute_local_starts(d_.gin, d_.in_topo, r, d_.in_right) ||
      compute_local_starts(d_.gout, chain_.back(), r, c1) !=
          compute_local_starts(d_.gout, d_.out_topo, r, d_.out_right))
    fail(kErrUnsupported, "per-rank plans need the topology chain to start and end at the plan's topologies");
  std::vector<std::size_t> order(nbl);
  for (std::size_t i = 0; i < nbl; ++i) order[i] = forward ? i : nbl - 1 - i;
  std::vector<std::size_t> topo_index(nbl);
  for (std::size_t i = 0, t = 0; i < nbl; ++i) {
    topo_index[i] = t;
    if (blocks[i].block_type == BlockType::Transpose) ++t;
  }
  // element type at each point: real until the first FFT block of the
  // forward walk (R2C), complex after it
  std::size_t first_fft = nbl;
  for (std::size_t i = 0; i < nbl; ++i)
    if (blocks[i].block_type == BlockType::FFT) {
      first_fft = i;
      break;
    }
  for (std::size_t i : order) {
    const BlockInfo& b = blocks[i];
    if (b.block_type != BlockType::Transpose) continue;
    const bool complex = !d_.r2c || i > first_fft;
    Exchange x;
    x.block = i;
    x.comm_axis = type_ == TopologyType::Pencil ? static_cast<int>(b.comm_axis) : -1;
    x.elements = total_size(b.buffer_extents);
    x.elem_bytes = (complex ? 2 : 1) * (d_.dbl ? 8 : 4);
    const std::size_t k = topo_index[i];
    // send side: forward packs the chain-k array along in_axis, backward the
    // chain-(k+1) array along out_axis
    const Layout S = forward ? rank_buffer_layout(k, complex, b.in_axis, b)
                             : rank_buffer_layout(k + 1, complex, b.out_axis, b);
    std::size_t valid = 0;
    for (const RankBlock& rb : layout_blocks(S)) valid += total_size(rb.local);
    x.padded = valid < x.elements;
    x.group = exchange_group(nprocs(), d_.in_topo, x.comm_axis, r);
    const std::size_t pc = d_.view_right ? b.buffer_extents.front() : b.buffer_extents.back();
    if (x.group.members.size() != pc) fail(kErrInternal, "exchange group size differs from the buffer's rank extent");
    (void)D;
    xs.push_back(x);
  }
}

void Plan::build_rank(bool forward) {
  const int dir = forward ? 0 : 1;
  auto& prog = prog_[dir];
  prog.clear();
  auto& ends = seg_end_[dir];
  ends.clear();
  const std::size_t r = static_cast<std::size_t>(d_.rank), D = d_.gin.size();
  const auto& blocks = per_rank_.at(r).blocks;
  const std::size_t nbl = blocks.size();
  std::vector<std::size_t> topo_index(nbl);
  for (std::size_t i = 0, t = 0; i < nbl; ++i) {
    topo_index[i] = t;
    if (blocks[i].block_type == BlockType::Transpose) ++t;
  }
  const std::size_t last_k = chain_.size() - 1;
  auto other_scratch = [](int b) { return b == kBufScratch0 ? kBufScratch1 : kBufScratch0; };
  auto scratch_for = [&](int cur_b) { return (cur_b == kBufScratch0 || cur_b == kBufScratch1) ? other_scratch(cur_b) : kBufScratch0; };
  int cur_l, cur_b;
  auto copy_to = [&](const Layout& L, int dst_b) {
    const int nl = add_layout(L);
    Op op = make_stage(cur_l, nl, layout_fast_axis(layouts_[cur_l]), dev::kCopy, false, 1.0);
    op.src = cur_b;
    op.dst = dst_b;
    prog.push_back(op);
    cur_l = nl;
    cur_b = dst_b;
  };
  auto plain = [](Layout L) {
    L.topo.assign(L.topo.size(), 1);
    L.pad.clear();
    return L;
  };
  // One FFT stage from the current array into (L, dst_b).  A side split
  // along the FFT axis that keeps the stage off the register kernels gets
  // its own copy (pack / unpack) through a plain local array.
  auto fft_stage = [&](const Layout& L, int dst_b, std::size_t a, int kind, bool inv, double scale) {
    const int nl = add_layout(L);
    Op op = make_stage(cur_l, nl, a, kind, inv, scale);
    const bool src_split = layouts_[cur_l].topo[a] > 1, dst_split = L.topo[a] > 1;
    if (!op.fast && !op.blue && op.four_n1 == 0 && (src_split || dst_split) &&
        dev::fast_stage_supported(op.sa.n)) {
      if (src_split) copy_to(plain(layouts_[cur_l]), scratch_for(cur_b));
      const Layout mid = dst_split ? plain(L) : L;
      const int ml = add_layout(mid);
      Op f = make_stage(cur_l, ml, a, kind, inv, scale);
      f.src = cur_b;
      f.dst = dst_split ? scratch_for(cur_b) : dst_b;
      push_stage(prog, f);
      cur_l = ml;
      cur_b = f.dst;
      if (dst_split) copy_to(L, dst_b);
      return;
    }
    op.src = cur_b;
    op.dst = dst_b;
    push_stage(prog, op);
    cur_l = nl;
    cur_b = dst_b;
  };
  const auto& xs = xch_[dir];
  std::size_t xi = 0;
  auto end_segment = [&](std::size_t block) {
    if (xi >= xs.size() || xs[xi].block != block) fail(kErrInternal, "per-rank exchanges out of order");
    ends.push_back(prog.size());
    ++xi;
  };

  if (forward) {
    bool complex = !d_.r2c;
    cur_l = add_layout(rank_layout(0, complex));
    cur_b = kBufIn;
    for (std::size_t i = 0; i < nbl; ++i) {
      const BlockInfo& b = blocks[i];
      const std::size_t k = topo_index[i];
      if (b.block_type == BlockType::FFT) {
        for (std::size_t j = 0; j < b.fft_dim; ++j) {
          const std::size_t a = d_.view_right ? b.in_map[D - 1 - j] : b.in_map[j];
          const int kind = complex ? dev::kC2C : dev::kR2C;
          complex = true;
          Layout L = rank_layout(k, true);
          int dst_b = scratch_for(cur_b);
          double scale = 1.0;
          if (j + 1 == b.fft_dim && i + 1 < nbl && blocks[i + 1].block_type == BlockType::Transpose) {
            L = rank_buffer_layout(k, true, blocks[i + 1].in_axis, blocks[i + 1]);
            dst_b = kBufSend;
          } else if (j + 1 == b.fft_dim && i + 1 == nbl) {
            dst_b = kBufOut;
            scale = scale_fwd_;
          }
          fft_stage(L, dst_b, a, kind, false, scale);
        }
      } else {
        const Layout S = rank_buffer_layout(k, complex, b.in_axis, b);
        if (cur_b != kBufSend || layouts_[cur_l] != S) copy_to(S, kBufSend);
        end_segment(i);
        cur_l = add_layout(rank_buffer_layout(k + 1, complex, b.out_axis, b));
        cur_b = kBufRecv;
      }
    }
    if (cur_b != kBufOut) finalize_program(prog, cur_l, cur_b, rank_layout(last_k, true), scale_fwd_, true);
  } else {
    bool complex = true;
    cur_l = add_layout(rank_layout(last_k, true));
    cur_b = kBufIn;
    for (std::size_t ii = nbl; ii-- > 0;) {
      const BlockInfo& b = blocks[ii];
      const std::size_t k = topo_index[ii];
      if (b.block_type == BlockType::FFT) {
        for (std::size_t jj = b.fft_dim; jj-- > 0;) {
          const std::size_t a = d_.view_right ? b.in_map[D - 1 - jj] : b.in_map[jj];
          const bool c2r = d_.r2c && b.block_idx == 0 && jj == 0;
          if (c2r) complex = false;
          Layout L = rank_layout(k, complex);
          int dst_b = scratch_for(cur_b);
          double scale = 1.0;
          if (jj == 0 && ii > 0 && blocks[ii - 1].block_type == BlockType::Transpose) {
            L = rank_buffer_layout(k, complex, blocks[ii - 1].out_axis, blocks[ii - 1]);
            dst_b = kBufSend;
          } else if (jj == 0 && ii == 0) {
            dst_b = kBufOut;
            scale = scale_bwd_;
          }
          fft_stage(L, dst_b, a, c2r ? dev::kC2R : dev::kC2C, true, scale);
        }
      } else {
        const Layout S = rank_buffer_layout(k + 1, complex, b.out_axis, b);
        if (cur_b != kBufSend || layouts_[cur_l] != S) copy_to(S, kBufSend);
        end_segment(ii);
        cur_l = add_layout(rank_buffer_layout(k, complex, b.in_axis, b));
        cur_b = kBufRecv;
      }
    }
    if (cur_b != kBufOut) finalize_program(prog, cur_l, cur_b, rank_layout(0, complex), scale_bwd_, complex);
  }
  if (xi != xs.size()) fail(kErrInternal, "per-rank program skipped an exchange");
  ends.push_back(prog.size());
}

void Plan::execute_segment(bool forward, std::size_t segment, const void* in, void* out, void* send, void* recv,
                           cudaStream_t stream) const {
  if (!is_rank_plan()) fail(kErrInvalidArgument, "segments belong to per-rank plans (dfft_plan_create_rank)");
  if (!on_device_) fail(kErrInvalidArgument, "plan was created by dfft_plan_analyze_rank and cannot execute");
  const int dir = forward ? 0 : 1;
  const auto& ends = seg_end_[dir];
  if (segment >= ends.size()) fail(kErrInvalidArgument, "segment index out of range");
  const std::size_t begin = segment == 0 ? 0 : ends[segment - 1], end = ends[segment];
  const bool first = segment == 0, last = segment + 1 == ends.size();
  const std::size_t real = d_.dbl ? 8 : 4;
  auto need = [&](const void* p, std::size_t align, const char* which) {
    if (!p) fail(kErrInvalidArgument, std::string("null ") + which + " buffer");
    if (reinterpret_cast<std::uintptr_t>(p) % align != 0)
      fail(kErrInvalidArgument, std::string(which) + " buffer is not aligned to its element type (" +
                                    std::to_string(align) + " bytes)");
  };
  // forward: real input for R2C; backward: real output for R2C
  if (first) need(in, (forward ? lin_.complex : true) ? 2 * real : real, "input");
  if (last) need(out, (forward ? true : lin_.complex) ? 2 * real : real, "output");
  const auto& xs = xch_[dir];
  if (!last) need(send, xs[segment].elem_bytes, "send");
  if (!first) need(recv, xs[segment - 1].elem_bytes, "recv");
  if (first && last && in == out) fail(kErrInvalidArgument, "in-place execution is not supported: in and out must differ");
  if (!first && !last && send == recv) fail(kErrInvalidArgument, "send and recv buffers must differ");
  run_program(prog_[dir], in, out, stream, begin, end, send, recv);
}

}  // namespace dfft
