// extern "C" entry points declared in include/dfft.h.  Every call catches
// the planner's exceptions and turns them into a dfft_status plus a
// thread-local message (the reference throws std::runtime_error via
// KOKKOSFFT_THROW_IF; nothing may unwind across a C ABI).
#include <algorithm>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/dfft.h"
#include "batch.hpp"
#include "exchange.hpp"
#include "ns.hpp"
#include "plan.hpp"

struct dfft_plan_s {
  dfft::Plan* impl;
};

struct dfft_ns_s {
  dfft::NsState* impl;
};

struct dfft_graph_s {
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};

struct dfft_batch_s {
  dfft::Batch* impl;
};

namespace {

thread_local std::string g_last_error;

dfft_status set_error(int code, const std::string& msg) {
  g_last_error = msg;
  return static_cast<dfft_status>(code);
}

template <typename F>
dfft_status guarded(F&& f) {
  try {
    f();
    g_last_error.clear();
    return DFFT_SUCCESS;
  } catch (const dfft::Error& e) {
    return set_error(e.code, e.what());
  } catch (const std::bad_alloc&) {
    return set_error(DFFT_ERROR_ALLOC, "host allocation failed");
  } catch (const std::exception& e) {
    return set_error(DFFT_ERROR_INTERNAL, e.what());
  } catch (...) {
    return set_error(DFFT_ERROR_INTERNAL, "unknown error");
  }
}

dfft::PlanDesc to_desc(const dfft_plan_desc* d) {
  if (!d) dfft::fail(dfft::kErrInvalidArgument, "null descriptor");
  if (d->rank < 2 || d->rank > DFFT_MAX_RANK) dfft::fail(dfft::kErrInvalidArgument, "view rank must be in [2, 4]");
  if (d->fft_rank < 1 || d->fft_rank > 3 || d->fft_rank > d->rank)
    dfft::fail(dfft::kErrInvalidArgument, "the Rank of FFT axes must be between 1 and 3");
  dfft::PlanDesc p;
  const std::size_t D = static_cast<std::size_t>(d->rank);
  for (int i = 0; i < d->fft_rank; ++i) {
    int a = d->axes[i];
    if (a < 0) a += d->rank;  // convert_negative_axes
    if (a < 0 || a >= d->rank) dfft::fail(dfft::kErrInvalidArgument, "input axes are not valid for the view");
    p.axes.push_back(static_cast<std::size_t>(a));
  }
  for (std::size_t k = 0; k < D; ++k) {
    p.gin.push_back(d->in_extents[k]);
    p.gout.push_back(d->out_extents[k]);
    p.in_topo.push_back(d->in_topology[k]);
    p.out_topo.push_back(d->out_topology[k]);
  }
  p.in_right = d->in_topology_layout_right != 0;
  p.out_right = d->out_topology_layout_right != 0;
  p.view_right = d->view_layout_right != 0;
  if (d->kind != DFFT_KIND_C2C && d->kind != DFFT_KIND_R2C) dfft::fail(dfft::kErrInvalidArgument, "unknown kind");
  if (d->precision != DFFT_PREC_F64 && d->precision != DFFT_PREC_F32 && d->precision != DFFT_PREC_F32_COMPENSATED)
    dfft::fail(dfft::kErrInvalidArgument, "unknown precision");
  if (d->exec_mode != DFFT_EXEC_FUSED && d->exec_mode != DFFT_EXEC_LITERAL && d->exec_mode != DFFT_EXEC_LITERAL_CAPTURE)
    dfft::fail(dfft::kErrInvalidArgument, "unknown execution mode");
  p.r2c = d->kind == DFFT_KIND_R2C;
  p.dbl = d->precision == DFFT_PREC_F64;
  p.comp = d->precision == DFFT_PREC_F32_COMPENSATED;
  p.norm = d->normalization;
  p.exec_mode = d->exec_mode;
  p.stream = static_cast<cudaStream_t>(d->stream);
  return p;
}

const dfft::Plan& impl_of(const dfft_plan* p) {
  if (!p || !p->impl) dfft::fail(dfft::kErrInvalidArgument, "null plan");
  return *p->impl;
}

const dfft::Plan& rank_impl_of(const dfft_plan* p) {
  const auto& impl = impl_of(p);
  if (!impl.is_rank_plan())
    dfft::fail(dfft::kErrInvalidArgument, "not a per-rank plan (dfft_plan_create_rank / dfft_plan_analyze_rank)");
  return impl;
}

bool forward_of(int32_t direction) {
  if (direction != DFFT_FORWARD && direction != DFFT_BACKWARD)
    dfft::fail(dfft::kErrInvalidArgument, "Invalid FFT direction specified.");
  return direction == DFFT_FORWARD;
}

void copy_ext(const dfft::Ext& e, uint64_t* dst, std::size_t n) {
  for (std::size_t i = 0; i < n; ++i) dst[i] = i < e.size() ? e[i] : 0;
}

dfft_status create(dfft_plan** out, const dfft_plan_desc* desc, bool on_device, int64_t rank = -1) {
  return guarded([&] {
    if (!out) dfft::fail(dfft::kErrInvalidArgument, "null output pointer");
    *out = nullptr;
    auto p = to_desc(desc);
    if (rank < -1) dfft::fail(dfft::kErrInvalidArgument, "rank must be non-negative");
    p.rank = rank;
    auto* impl = new dfft::Plan(p, on_device);
    *out = new dfft_plan_s{impl};
  });
}

}  // namespace

// Capture `body` (work enqueued on one stream) into an instantiated graph.
template <typename F>
static dfft_graph_s* capture_graph(F&& body) {
  auto ck = [](cudaError_t e, const char* what) {
    if (e != cudaSuccess) dfft::fail(dfft::kErrCuda, std::string(what) + ": " + cudaGetErrorString(e));
  };
  cudaStream_t cap = nullptr;
  ck(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking), "stream create");
  cudaGraph_t g = nullptr;
  try {
    ck(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal), "begin capture");
    try {
      body(cap);
    } catch (...) {
      cudaGraph_t dead = nullptr;
      cudaStreamEndCapture(cap, &dead);
      if (dead) cudaGraphDestroy(dead);
      throw;
    }
    ck(cudaStreamEndCapture(cap, &g), "end capture");
  } catch (...) {
    cudaStreamDestroy(cap);
    throw;
  }
  cudaStreamDestroy(cap);
  auto* out = new dfft_graph_s;
  out->graph = g;
  if (cudaGraphInstantiate(&out->exec, g, 0) != cudaSuccess) {
    cudaGetLastError();
    cudaGraphDestroy(g);
    delete out;
    dfft::fail(dfft::kErrCuda, "cudaGraphInstantiate failed");
  }
  return out;
}

extern "C" {

void dfft_plan_desc_init(dfft_plan_desc* d) {
  if (!d) return;
  std::memset(d, 0, sizeof(*d));
  d->rank = 3;
  d->fft_rank = 3;
  d->axes[0] = 0;
  d->axes[1] = 1;
  d->axes[2] = 2;
  for (int k = 0; k < DFFT_MAX_RANK; ++k) {
    d->in_topology[k] = 1;
    d->out_topology[k] = 1;
  }
  d->in_topology_layout_right = 1;
  d->out_topology_layout_right = 1;
  d->view_layout_right = 1;
  d->kind = DFFT_KIND_C2C;
  d->precision = DFFT_PREC_F64;
  d->normalization = DFFT_NORM_BACKWARD;
  d->exec_mode = DFFT_EXEC_FUSED;
  d->stream = nullptr;
}

dfft_status dfft_plan_create(dfft_plan** plan, const dfft_plan_desc* desc) { return create(plan, desc, true); }

dfft_status dfft_plan_analyze(dfft_plan** plan, const dfft_plan_desc* desc) { return create(plan, desc, false); }

dfft_status dfft_plan_destroy(dfft_plan* plan) {
  return guarded([&] {
    if (!plan) return;
    delete plan->impl;
    delete plan;
  });
}

dfft_status dfft_execute_on_stream(const dfft_plan* plan, const void* in, void* out, int32_t direction,
                                   void* stream) {
  return guarded([&] {
    const auto& p = impl_of(plan);
    if (direction != DFFT_FORWARD && direction != DFFT_BACKWARD)
      dfft::fail(dfft::kErrInvalidArgument, "Invalid FFT direction specified.");
    p.execute(in, out, direction == DFFT_FORWARD, static_cast<cudaStream_t>(stream));
  });
}

dfft_status dfft_execute_adjoint(const dfft_plan* plan, const void* in, void* out, int32_t direction, void* stream) {
  return guarded([&] {
    const auto& p = impl_of(plan);
    if (direction != DFFT_FORWARD && direction != DFFT_BACKWARD)
      dfft::fail(dfft::kErrInvalidArgument, "Invalid FFT direction specified.");
    p.execute_adjoint(in, out, direction == DFFT_FORWARD, static_cast<cudaStream_t>(stream));
  });
}

dfft_status dfft_execute(const dfft_plan* plan, const void* in, void* out, int32_t direction) {
  if (!plan || !plan->impl) return set_error(DFFT_ERROR_INVALID_ARGUMENT, "null plan");
  return dfft_execute_on_stream(plan, in, out, direction, plan->impl->desc().stream);
}

const char* dfft_plan_name(const dfft_plan* plan) {
  if (!plan || !plan->impl) return "";
  return plan->impl->name().c_str();
}

dfft_status dfft_get_nprocs(const dfft_plan* plan, int64_t* nprocs) {
  return guarded([&] {
    if (!nprocs) dfft::fail(dfft::kErrInvalidArgument, "null output");
    *nprocs = static_cast<int64_t>(impl_of(plan).nprocs());
  });
}

dfft_status dfft_get_local_extents(const dfft_plan* plan, int64_t rank, int32_t which, uint64_t* extents,
                                   uint64_t* starts) {
  return guarded([&] {
    const auto& p = impl_of(plan);
    if (rank < 0 || static_cast<std::size_t>(rank) >= p.nprocs())
      dfft::fail(dfft::kErrInvalidArgument, "rank must be less than topology size.");
    const dfft::Layout& L = which == 0 ? p.in_layout() : p.out_layout();
    const std::size_t D = L.gext.size();
    dfft::Ext ext = dfft::compute_local_extents(L.gext, L.topo, dfft::identity_map(D), rank, L.rank_right);
    dfft::Ext st = dfft::compute_local_starts(L.gext, L.topo, rank, L.rank_right);
    if (extents) copy_ext(ext, extents, DFFT_MAX_RANK);
    if (starts) copy_ext(st, starts, DFFT_MAX_RANK);
  });
}

dfft_status dfft_get_local_offset(const dfft_plan* plan, int64_t rank, int32_t which, uint64_t* offset) {
  return guarded([&] {
    const auto& p = impl_of(plan);
    if (rank < 0 || static_cast<std::size_t>(rank) >= p.nprocs())
      dfft::fail(dfft::kErrInvalidArgument, "rank must be less than topology size.");
    if (!offset) dfft::fail(dfft::kErrInvalidArgument, "null output");
    auto blocks = dfft::layout_blocks(which == 0 ? p.in_layout() : p.out_layout());
    *offset = blocks[rank].base;
  });
}

dfft_status dfft_get_buffer_elements(const dfft_plan* plan, int32_t which, uint64_t* count) {
  return guarded([&] {
    const auto& p = impl_of(plan);
    if (!count) dfft::fail(dfft::kErrInvalidArgument, "null output");
    *count = dfft::layout_elements(which == 0 ? p.in_layout() : p.out_layout());
  });
}

dfft_status dfft_get_num_blocks(const dfft_plan* plan, int64_t* nblocks) {
  return guarded([&] {
    if (!nblocks) dfft::fail(dfft::kErrInvalidArgument, "null output");
    *nblocks = static_cast<int64_t>(impl_of(plan).analyses().at(0).blocks.size());
  });
}

static void fill_block_info(const dfft::BlockInfo& b, dfft_block_info* info) {
  std::memset(info, 0, sizeof(*info));
  info->block_type = b.block_type == dfft::BlockType::FFT ? 1 : 0;
  info->block_idx = static_cast<int32_t>(b.block_idx);
  info->fft_dim = static_cast<int32_t>(b.fft_dim);
  info->in_axis = static_cast<int32_t>(b.in_axis);
  info->out_axis = static_cast<int32_t>(b.out_axis);
  info->comm_axis = static_cast<int32_t>(b.comm_axis);
  copy_ext(b.in_topology, info->in_topology, DFFT_MAX_RANK);
  copy_ext(b.out_topology, info->out_topology, DFFT_MAX_RANK);
  copy_ext(b.in_extents, info->in_extents, DFFT_MAX_RANK);
  copy_ext(b.out_extents, info->out_extents, DFFT_MAX_RANK);
  copy_ext(b.buffer_extents, info->buffer_extents, DFFT_MAX_RANK + 1);
  copy_ext(b.in_map, info->in_map, DFFT_MAX_RANK);
  copy_ext(b.out_map, info->out_map, DFFT_MAX_RANK);
}

dfft_status dfft_get_block_info(const dfft_plan* plan, int64_t rank, int64_t block, dfft_block_info* info) {
  return guarded([&] {
    const auto& p = impl_of(plan);
    if (!info) dfft::fail(dfft::kErrInvalidArgument, "null output");
    if (rank < 0 || static_cast<std::size_t>(rank) >= p.nprocs())
      dfft::fail(dfft::kErrInvalidArgument, "rank must be less than topology size.");
    const auto& blocks = p.analyses().at(rank).blocks;
    if (block < 0 || static_cast<std::size_t>(block) >= blocks.size())
      dfft::fail(dfft::kErrInvalidArgument, "block index out of range");
    fill_block_info(blocks[block], info);
  });
}

dfft_status dfft_get_device_error(const dfft_plan* plan, int32_t reset, int32_t* code) {
  return guarded([&] {
    if (!code) dfft::fail(dfft::kErrInvalidArgument, "null output");
    *code = impl_of(plan).device_error(reset != 0);
  });
}

dfft_status dfft_get_max_buffer_size(const dfft_plan* plan, uint64_t* size) {
  return guarded([&] {
    if (!size) dfft::fail(dfft::kErrInvalidArgument, "null output");
    *size = impl_of(plan).max_buffer_size();
  });
}

dfft_status dfft_plan_create_rank(dfft_plan** plan, const dfft_plan_desc* desc, int64_t rank) {
  return create(plan, desc, true, rank);
}

dfft_status dfft_plan_analyze_rank(dfft_plan** plan, const dfft_plan_desc* desc, int64_t rank) {
  return create(plan, desc, false, rank);
}

dfft_status dfft_get_num_exchanges(const dfft_plan* plan, int32_t direction, int64_t* n) {
  return guarded([&] {
    const auto& p = rank_impl_of(plan);
    if (!n) dfft::fail(dfft::kErrInvalidArgument, "null output");
    *n = static_cast<int64_t>(p.exchanges(forward_of(direction)).size());
  });
}

dfft_status dfft_get_exchange_info(const dfft_plan* plan, int32_t direction, int64_t k, dfft_exchange_info* info) {
  return guarded([&] {
    const auto& p = rank_impl_of(plan);
    if (!info) dfft::fail(dfft::kErrInvalidArgument, "null output");
    const auto& xs = p.exchanges(forward_of(direction));
    if (k < 0 || static_cast<std::size_t>(k) >= xs.size())
      dfft::fail(dfft::kErrInvalidArgument, "exchange index out of range");
    const dfft::Exchange& x = xs[k];
    info->block = static_cast<int64_t>(x.block);
    info->comm_axis = x.comm_axis;
    info->padded = x.padded ? 1 : 0;
    info->elements = x.elements;
    info->element_bytes = x.elem_bytes;
    info->group_size = static_cast<int64_t>(x.group.members.size());
  });
}

dfft_status dfft_get_exchange_group(const dfft_plan* plan, int32_t direction, int64_t k, int64_t rank,
                                    int64_t* sub_rank, int64_t* members) {
  return guarded([&] {
    const auto& p = rank_impl_of(plan);
    if (k < 0 || rank < 0) dfft::fail(dfft::kErrInvalidArgument, "negative index");
    const dfft::ExchangeGroup g =
        p.exchange_group_of(forward_of(direction), static_cast<std::size_t>(k), static_cast<std::size_t>(rank));
    if (sub_rank) *sub_rank = static_cast<int64_t>(g.sub);
    if (members)
      for (std::size_t j = 0; j < g.members.size(); ++j) members[j] = static_cast<int64_t>(g.members[j]);
  });
}

dfft_status dfft_execute_segment(const dfft_plan* plan, int32_t direction, int64_t segment, const void* in,
                                 void* out, void* send, void* recv, void* stream) {
  return guarded([&] {
    const auto& p = rank_impl_of(plan);
    if (segment < 0) dfft::fail(dfft::kErrInvalidArgument, "segment index out of range");
    p.execute_segment(forward_of(direction), static_cast<std::size_t>(segment), in, out, send, recv,
                      static_cast<cudaStream_t>(stream));
  });
}

dfft_status dfft_execute_exchanged(const dfft_plan* plan, const void* in, void* out, int32_t direction, void* send,
                                   void* recv, dfft_exchange_fn exchange, void* user, void* stream) {
  return guarded([&] {
    const auto& p = rank_impl_of(plan);
    const bool fwd = forward_of(direction);
    const auto& xs = p.exchanges(fwd);
    if (!xs.empty() && !exchange) dfft::fail(dfft::kErrInvalidArgument, "null exchange callback");
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    for (std::size_t s = 0; s <= xs.size(); ++s) {
      p.execute_segment(fwd, s, in, out, send, recv, st);
      if (s == xs.size()) break;
      const uint64_t per_peer = xs[s].elements / xs[s].group.members.size() * xs[s].elem_bytes;
      const int32_t rc = exchange(user, static_cast<int64_t>(s), send, recv, per_peer, stream);
      if (rc != 0) dfft::fail(dfft::kErrCuda, "exchange callback returned " + std::to_string(rc));
    }
  });
}

dfft_status dfft_get_topology_chain(const dfft_plan* plan, int64_t* n, uint64_t* topologies, int64_t* trans_axes,
                                    int64_t* layouts) {
  return guarded([&] {
    const auto& p = impl_of(plan);
    if (!n) dfft::fail(dfft::kErrInvalidArgument, "null output");
    const auto& ch = p.chain();
    const int64_t cap = *n;
    *n = static_cast<int64_t>(ch.size());
    if (cap < static_cast<int64_t>(ch.size())) return;
    const std::size_t D = p.desc().gin.size();
    for (std::size_t i = 0; i < ch.size(); ++i) {
      if (topologies)
        for (std::size_t k = 0; k < D; ++k) topologies[i * D + k] = ch[i][k];
      if (layouts) layouts[i] = static_cast<int64_t>(p.chain_layouts().at(i));
      if (trans_axes && i + 1 < ch.size())
        trans_axes[i] = i < p.chain_trans_axes().size() ? static_cast<int64_t>(p.chain_trans_axes()[i]) : 0;
    }
  });
}

dfft_status dfft_debug_export_buffers(const dfft_plan* plan, int32_t direction, int64_t block, int32_t which,
                                      void* host_dst, uint64_t capacity_bytes) {
  return guarded([&] {
    if (!host_dst) dfft::fail(dfft::kErrInvalidArgument, "null host buffer");
    if (block < 0) dfft::fail(dfft::kErrInvalidArgument, "block index out of range");
    impl_of(plan).export_buffers(direction == DFFT_FORWARD, static_cast<std::size_t>(block), which, host_dst,
                                 capacity_bytes);
  });
}

dfft_status dfft_get_launch_count(const dfft_plan* plan, int32_t direction, int64_t* launches) {
  return guarded([&] {
    if (!launches) dfft::fail(dfft::kErrInvalidArgument, "null output");
    *launches = static_cast<int64_t>(impl_of(plan).launches(direction == DFFT_FORWARD));
  });
}

dfft_status dfft_get_workspace_bytes(const dfft_plan* plan, uint64_t* bytes) {
  return guarded([&] {
    if (!bytes) dfft::fail(dfft::kErrInvalidArgument, "null output");
    *bytes = impl_of(plan).workspace_bytes();
  });
}

dfft_status dfft_get_all_topologies(int32_t pencil, int32_t rank, const uint64_t* in_topology,
                                    int32_t in_layout_right, const uint64_t* out_topology, int32_t out_layout_right,
                                    int32_t fft_rank, const int32_t* axes, int64_t* n, uint64_t* topologies,
                                    int64_t* trans_axes, int64_t* layouts) {
  return guarded([&] {
    if (!in_topology || !out_topology || !axes || !n) dfft::fail(dfft::kErrInvalidArgument, "null argument");
    if (rank < 1 || rank > 8 || fft_rank < 1 || fft_rank > 3) dfft::fail(dfft::kErrInvalidArgument, "bad rank");
    dfft::Ext in(in_topology, in_topology + rank), out(out_topology, out_topology + rank), ax;
    for (int i = 0; i < fft_rank; ++i) {
      int a = axes[i] < 0 ? axes[i] + rank : axes[i];
      ax.push_back(static_cast<std::size_t>(a));
    }
    std::vector<dfft::Ext> chain;
    std::vector<std::size_t> tr, lay;
    if (pencil) {
      auto ch = dfft::get_all_pencil_topologies(in, in_layout_right != 0, out, out_layout_right != 0, ax);
      chain = ch.topologies;
      tr = ch.trans_axes;
      lay = ch.layouts;
    } else {
      chain = dfft::get_all_slab_topologies(in, out, ax);
    }
    const int64_t cap = *n;
    *n = static_cast<int64_t>(chain.size());
    if (cap < *n) return;
    for (std::size_t i = 0; i < chain.size(); ++i) {
      if (topologies)
        for (int k = 0; k < rank; ++k) topologies[i * rank + k] = chain[i][k];
      if (layouts) layouts[i] = i < lay.size() ? static_cast<int64_t>(lay[i]) : 0;
      if (trans_axes && i < tr.size()) trans_axes[i] = static_cast<int64_t>(tr[i]);
    }
  });
}

}  // extern "C"

dfft_status dfft_noalloc_impl(const void* in, void* out, int64_t n0, int64_t n1, int64_t n2, int32_t precision,
                              int32_t direction, int32_t normalization, void* stream, const char** err);

extern "C" {

dfft_status dfft_execute_local_c2c_noalloc(const void* in, void* out, int64_t n0, int64_t n1, int64_t n2,
                                           int32_t precision, int32_t direction, int32_t normalization,
                                           void* stream) {
  const char* err = "";
  const dfft_status st = dfft_noalloc_impl(in, out, n0, n1, n2, precision, direction, normalization, stream, &err);
  if (st != DFFT_SUCCESS) return set_error(st, err);
  g_last_error.clear();
  return DFFT_SUCCESS;
}

dfft_status dfft_graph_create(dfft_graph** graph, const dfft_plan* const* plans, const void* const* ins,
                              void* const* outs, const int32_t* directions, const int32_t* branch_ids,
                              int64_t count) {
  return guarded([&] {
    if (!graph || !plans || !ins || !outs || !directions || count <= 0)
      dfft::fail(dfft::kErrInvalidArgument, "null argument or empty batch");
    *graph = nullptr;
    for (int64_t i = 0; i < count; ++i) {
      impl_of(plans[i]);
      if (directions[i] != DFFT_FORWARD && directions[i] != DFFT_BACKWARD)
        dfft::fail(dfft::kErrInvalidArgument, "Invalid FFT direction specified.");
    }
    auto ck = [](cudaError_t e, const char* what) {
      if (e != cudaSuccess) dfft::fail(dfft::kErrCuda, std::string(what) + ": " + cudaGetErrorString(e));
    };
    // branch of every item: its id in branch_ids, or its own
    std::vector<int> bidx(static_cast<std::size_t>(count));
    std::vector<int32_t> ids;
    for (int64_t i = 0; i < count; ++i) {
      const int32_t id = branch_ids ? branch_ids[i] : static_cast<int32_t>(i);
      auto it = std::find(ids.begin(), ids.end(), id);
      if (it == ids.end()) {
        bidx[i] = static_cast<int>(ids.size());
        ids.push_back(id);
      } else {
        bidx[i] = static_cast<int>(it - ids.begin());
      }
    }
    // a plan's transforms share its two scratch arrays: all of them must run
    // in order on one branch
    for (int64_t i = 0; i < count; ++i)
      for (int64_t j = 0; j < i; ++j)
        if (plans[i] == plans[j] && bidx[i] != bidx[j])
          dfft::fail(dfft::kErrInvalidArgument,
                     "a plan appears on two branches (items " + std::to_string(j) + " and " + std::to_string(i) +
                         "): its transforms share the plan's scratch and must be on one branch");
    const std::size_t nb = ids.size();
    cudaStream_t cap = nullptr;
    ck(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking), "stream create");
    std::vector<cudaStream_t> branches(nb, nullptr);
    std::vector<cudaEvent_t> done(nb, nullptr);
    cudaEvent_t fork = nullptr;
    cudaGraph_t g = nullptr;
    auto cleanup = [&]() {
      for (auto s2 : branches)
        if (s2) cudaStreamDestroy(s2);
      for (auto e : done)
        if (e) cudaEventDestroy(e);
      if (fork) cudaEventDestroy(fork);
      if (cap) cudaStreamDestroy(cap);
    };
    try {
      ck(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming), "event create");
      for (std::size_t b = 0; b < nb; ++b) {
        ck(cudaStreamCreateWithFlags(&branches[b], cudaStreamNonBlocking), "stream create");
        ck(cudaEventCreateWithFlags(&done[b], cudaEventDisableTiming), "event create");
      }
      ck(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal), "begin capture");
      try {
        ck(cudaEventRecord(fork, cap), "fork record");
        for (std::size_t b = 0; b < nb; ++b) ck(cudaStreamWaitEvent(branches[b], fork, 0), "fork wait");
        for (int64_t i = 0; i < count; ++i)
          plans[i]->impl->execute(ins[i], outs[i], directions[i] == DFFT_FORWARD, branches[bidx[i]]);
        for (std::size_t b = 0; b < nb; ++b) {
          ck(cudaEventRecord(done[b], branches[b]), "join record");
          ck(cudaStreamWaitEvent(cap, done[b], 0), "join wait");
        }
      } catch (...) {
        cudaGraph_t dead = nullptr;
        cudaStreamEndCapture(cap, &dead);
        if (dead) cudaGraphDestroy(dead);
        throw;
      }
      ck(cudaStreamEndCapture(cap, &g), "end capture");
      auto* out = new dfft_graph_s;
      out->graph = g;
      if (cudaGraphInstantiate(&out->exec, g, 0) != cudaSuccess) {
        cudaGetLastError();
        cudaGraphDestroy(g);
        delete out;
        dfft::fail(dfft::kErrCuda, "cudaGraphInstantiate failed");
      }
      *graph = out;
    } catch (...) {
      cleanup();
      throw;
    }
    cleanup();
  });
}

static const dfft::Batch& batch_of(const dfft_batch* b) {
  if (!b || !b->impl) dfft::fail(dfft::kErrInvalidArgument, "null batch");
  return *b->impl;
}

dfft_status dfft_batch_create(dfft_batch** batch, const dfft_plan* const* plans, int64_t count) {
  return guarded([&] {
    if (!batch || !plans || count <= 0) dfft::fail(dfft::kErrInvalidArgument, "null argument or empty batch");
    *batch = nullptr;
    std::vector<const dfft::Plan*> ps;
    for (int64_t i = 0; i < count; ++i) ps.push_back(&impl_of(plans[i]));
    auto* impl = new dfft::Batch(std::move(ps));
    *batch = new dfft_batch_s{impl};
  });
}

dfft_status dfft_batch_execute(const dfft_batch* batch, const void* const* ins, void* const* outs, int32_t direction,
                               void* stream) {
  return guarded([&] {
    if (direction != DFFT_FORWARD && direction != DFFT_BACKWARD)
      dfft::fail(dfft::kErrInvalidArgument, "Invalid FFT direction specified.");
    batch_of(batch).execute(ins, outs, direction == DFFT_FORWARD, static_cast<cudaStream_t>(stream));
  });
}

dfft_status dfft_batch_get_launch_count(const dfft_batch* batch, int32_t direction, int64_t* launches) {
  return guarded([&] {
    if (!launches) dfft::fail(dfft::kErrInvalidArgument, "null output");
    *launches = static_cast<int64_t>(batch_of(batch).launches(direction == DFFT_FORWARD));
  });
}

dfft_status dfft_batch_destroy(dfft_batch* batch) {
  return guarded([&] {
    if (!batch) return;
    delete batch->impl;
    delete batch;
  });
}

dfft_status dfft_ns_graph_create(dfft_graph** graph, dfft_ns* const* states, void* const* uks, int64_t count,
                                 int32_t batched) {
  return guarded([&] {
    if (!graph || !states || !uks || count <= 0) dfft::fail(dfft::kErrInvalidArgument, "null argument or empty batch");
    *graph = nullptr;
    std::vector<dfft::NsState*> ss;
    std::vector<const dfft::Plan*> ps;
    for (int64_t i = 0; i < count; ++i) {
      if (!states[i] || !states[i]->impl || !uks[i]) dfft::fail(dfft::kErrInvalidArgument, "null state or buffer");
      ss.push_back(states[i]->impl);
      ps.push_back(dfft::ns_plan(states[i]->impl));
    }
    for (int64_t i = 0; i < count; ++i)
      for (int64_t j = 0; j < i; ++j)
        if (ss[i] == ss[j]) dfft::fail(dfft::kErrInvalidArgument, "a Navier-Stokes state appears twice");
    if (batched) {
      const dfft::Batch batch(ps);
      *graph = capture_graph([&](cudaStream_t st) {
        dfft::ns_batch_step(ss.data(), uks, static_cast<int>(count), batch, st);
      });
      return;
    }
    // per-field steps on up to four concurrent branches; fields that share a
    // plan (and so its scratch) stay on one branch
    auto ck = [](cudaError_t e, const char* what) {
      if (e != cudaSuccess) dfft::fail(dfft::kErrCuda, std::string(what) + ": " + cudaGetErrorString(e));
    };
    std::vector<const dfft::Plan*> distinct;
    std::vector<int> branch(static_cast<std::size_t>(count));
    for (int64_t i = 0; i < count; ++i) {
      auto it = std::find(distinct.begin(), distinct.end(), ps[i]);
      if (it == distinct.end()) {
        branch[i] = static_cast<int>(distinct.size());
        distinct.push_back(ps[i]);
      } else {
        branch[i] = static_cast<int>(it - distinct.begin());
      }
    }
    const int nb = static_cast<int>(std::min<std::size_t>(4, distinct.size()));
    for (auto& b : branch) b %= nb;
    std::vector<cudaStream_t> streams(nb, nullptr);
    std::vector<cudaEvent_t> done(nb, nullptr);
    cudaEvent_t fork = nullptr;
    auto cleanup = [&]() {
      for (auto x : streams)
        if (x) cudaStreamDestroy(x);
      for (auto e : done)
        if (e) cudaEventDestroy(e);
      if (fork) cudaEventDestroy(fork);
    };
    try {
      ck(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming), "event create");
      for (int b = 0; b < nb; ++b) {
        ck(cudaStreamCreateWithFlags(&streams[b], cudaStreamNonBlocking), "stream create");
        ck(cudaEventCreateWithFlags(&done[b], cudaEventDisableTiming), "event create");
      }
      *graph = capture_graph([&](cudaStream_t st) {
        ck(cudaEventRecord(fork, st), "fork record");
        for (int b = 0; b < nb; ++b) ck(cudaStreamWaitEvent(streams[b], fork, 0), "fork wait");
        for (int64_t i = 0; i < count; ++i) dfft::ns_step(ss[i], uks[i], streams[branch[i]]);
        for (int b = 0; b < nb; ++b) {
          ck(cudaEventRecord(done[b], streams[b]), "join record");
          ck(cudaStreamWaitEvent(st, done[b], 0), "join wait");
        }
      });
    } catch (...) {
      cleanup();
      throw;
    }
    cleanup();
  });
}

dfft_status dfft_graph_launch(const dfft_graph* graph, void* stream) {
  return guarded([&] {
    if (!graph || !graph->exec) dfft::fail(dfft::kErrInvalidArgument, "null graph");
    const cudaError_t e = cudaGraphLaunch(graph->exec, static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) dfft::fail(dfft::kErrCuda, std::string("cudaGraphLaunch: ") + cudaGetErrorString(e));
  });
}

dfft_status dfft_graph_destroy(dfft_graph* graph) {
  return guarded([&] {
    if (!graph) return;
    if (graph->exec) cudaGraphExecDestroy(graph->exec);
    if (graph->graph) cudaGraphDestroy(graph->graph);
    delete graph;
  });
}

dfft_status dfft_ns_create(dfft_ns** ns, const dfft_plan* plan, double nu, double dt, double lx) {
  return guarded([&] {
    if (!ns) dfft::fail(dfft::kErrInvalidArgument, "null output pointer");
    *ns = nullptr;
    const auto& p = impl_of(plan);
    if (!p.on_device()) dfft::fail(dfft::kErrInvalidArgument, "plan was created by dfft_plan_analyze");
    auto* impl = dfft::ns_create(&p, nu, dt, lx);
    *ns = new dfft_ns_s{impl};
  });
}

static dfft::NsState* ns_of(dfft_ns* ns) {
  if (!ns || !ns->impl) dfft::fail(dfft::kErrInvalidArgument, "null Navier-Stokes state");
  return ns->impl;
}

dfft_status dfft_ns_init_taylor_green(dfft_ns* ns, void* uk, double v0, void* stream) {
  return guarded([&] {
    if (!uk) dfft::fail(dfft::kErrInvalidArgument, "null buffer");
    dfft::ns_taylor_green(ns_of(ns), uk, v0, static_cast<cudaStream_t>(stream));
  });
}

dfft_status dfft_ns_rhs(dfft_ns* ns, void* uk, void* dukdt, void* stream) {
  return guarded([&] {
    if (!uk || !dukdt) dfft::fail(dfft::kErrInvalidArgument, "null buffer");
    dfft::ns_rhs(ns_of(ns), uk, dukdt, static_cast<cudaStream_t>(stream));
  });
}

dfft_status dfft_ns_step(dfft_ns* ns, void* uk, void* stream) {
  return guarded([&] {
    if (!uk) dfft::fail(dfft::kErrInvalidArgument, "null buffer");
    dfft::ns_step(ns_of(ns), uk, static_cast<cudaStream_t>(stream));
  });
}

dfft_status dfft_ns_energy(dfft_ns* ns, const void* uk, double* energy, void* stream) {
  return guarded([&] {
    if (!uk || !energy) dfft::fail(dfft::kErrInvalidArgument, "null argument");
    *energy = dfft::ns_energy(ns_of(ns), uk, static_cast<cudaStream_t>(stream));
  });
}

dfft_status dfft_ns_velocity(dfft_ns* ns, const void* uk, void* u, void* stream) {
  return guarded([&] {
    if (!uk || !u) dfft::fail(dfft::kErrInvalidArgument, "null buffer");
    dfft::ns_velocity(ns_of(ns), uk, u, static_cast<cudaStream_t>(stream));
  });
}

dfft_status dfft_ns_vorticity(dfft_ns* ns, const void* uk, void* vor, void* stream) {
  return guarded([&] {
    if (!uk || !vor) dfft::fail(dfft::kErrInvalidArgument, "null buffer");
    dfft::ns_vorticity(ns_of(ns), uk, vor, static_cast<cudaStream_t>(stream));
  });
}

static_assert(DFFT_NS_MAX_BINS == dfft::kNsMaxBins, "spectrum bin limit");

dfft_status dfft_ns_diagnostics(dfft_ns* ns, const void* uk, int32_t num_bins, double* e_spec, double* k_vals,
                                dfft_ns_diag* out, void* stream) {
  return guarded([&] {
    if (!uk || !out) dfft::fail(dfft::kErrInvalidArgument, "null argument");
    const dfft::NsDiag d = dfft::ns_diagnostics(ns_of(ns), uk, num_bins, e_spec, k_vals,
                                                static_cast<cudaStream_t>(stream));
    out->energy = d.energy;
    out->enstrophy = d.enstrophy;
    out->divergence_l2 = d.divergence_l2;
  });
}

dfft_status dfft_ns_write_diagnostics(dfft_ns* ns, const void* uk, const char* out_dir, int32_t iter,
                                      int32_t num_bins, dfft_ns_diag* out, void* stream) {
  return guarded([&] {
    if (!uk || !out_dir) dfft::fail(dfft::kErrInvalidArgument, "null argument");
    const dfft::NsDiag d = dfft::ns_write_diagnostics(ns_of(ns), uk, out_dir, iter, num_bins,
                                                      static_cast<cudaStream_t>(stream));
    if (out) {
      out->energy = d.energy;
      out->enstrophy = d.enstrophy;
      out->divergence_l2 = d.divergence_l2;
    }
  });
}

dfft_status dfft_ns_rhs_adjoint(dfft_ns* ns, const void* uk, const void* lambda, void* grad, void* stream) {
  return guarded([&] {
    if (!uk || !lambda || !grad) dfft::fail(dfft::kErrInvalidArgument, "null buffer");
    if (grad == uk || grad == lambda) dfft::fail(dfft::kErrInvalidArgument, "grad must not alias uk or lambda");
    dfft::ns_rhs_adjoint(ns_of(ns), uk, lambda, grad, static_cast<cudaStream_t>(stream));
  });
}

dfft_status dfft_ns_step_adjoint(dfft_ns* ns, const void* uk, void* lambda, void* stream) {
  return guarded([&] {
    if (!uk || !lambda) dfft::fail(dfft::kErrInvalidArgument, "null buffer");
    if (uk == lambda) dfft::fail(dfft::kErrInvalidArgument, "lambda must not alias uk");
    dfft::ns_step_adjoint(ns_of(ns), uk, lambda, static_cast<cudaStream_t>(stream));
  });
}

dfft_status dfft_ns_destroy(dfft_ns* ns) {
  return guarded([&] {
    if (!ns) return;
    dfft::ns_destroy(ns->impl);
    delete ns;
  });
}

// ---- data-movement layer ----
static dfft::Ext ext_of(const uint64_t* v, int32_t n, const char* what) {
  if (!v) dfft::fail(dfft::kErrInvalidArgument, std::string("null ") + what);
  if (n < 1 || n > DFFT_MAX_RANK + 1) dfft::fail(dfft::kErrInvalidArgument, std::string("bad rank of ") + what);
  return dfft::Ext(v, v + n);
}

static dfft::Ext map_of(const int32_t* v, int32_t n, const char* what) {
  if (!v) dfft::fail(dfft::kErrInvalidArgument, std::string("null ") + what);
  dfft::Ext m;
  for (int32_t i = 0; i < n; ++i) {
    if (v[i] < 0 || v[i] >= n) dfft::fail(dfft::kErrInvalidArgument, std::string(what) + " entry out of range");
    m.push_back(static_cast<std::size_t>(v[i]));
  }
  return m;
}

static void check_view_rank(int32_t rank) {
  if (rank < 2 || rank > DFFT_MAX_RANK) dfft::fail(dfft::kErrInvalidArgument, "view rank must be in [2, 4]");
}

dfft_status dfft_pack(int32_t rank, const uint64_t* src_extents, const int32_t* src_map, int32_t axis,
                      const uint64_t* buffer_extents, int32_t layout_right, int32_t element_bytes, const void* src,
                      void* dst, void* stream) {
  return guarded([&] {
    check_view_rank(rank);
    if (axis < 0 || axis >= rank) dfft::fail(dfft::kErrInvalidArgument, "axis out of range");
    dfft::pack_local(ext_of(src_extents, rank, "src_extents"), map_of(src_map, rank, "src_map"),
                     static_cast<std::size_t>(axis), ext_of(buffer_extents, rank + 1, "buffer_extents"),
                     layout_right != 0, element_bytes, src, dst, static_cast<cudaStream_t>(stream));
  });
}

dfft_status dfft_unpack(int32_t rank, const uint64_t* buffer_extents, const int32_t* dst_map, int32_t axis,
                        const uint64_t* dst_extents, int32_t layout_right, int32_t element_bytes, const void* src,
                        void* dst, void* stream) {
  return guarded([&] {
    check_view_rank(rank);
    if (axis < 0 || axis >= rank) dfft::fail(dfft::kErrInvalidArgument, "axis out of range");
    dfft::unpack_local(ext_of(buffer_extents, rank + 1, "buffer_extents"), map_of(dst_map, rank, "dst_map"),
                       static_cast<std::size_t>(axis), ext_of(dst_extents, rank, "dst_extents"), layout_right != 0,
                       element_bytes, src, dst, static_cast<cudaStream_t>(stream));
  });
}

dfft_status dfft_all2all(int64_t nprocs, int32_t buffer_rank, const uint64_t* buffer_extents, int32_t layout_right,
                         int32_t comm_axis, int32_t cart_rank, const uint64_t* cart_topology, int32_t element_bytes,
                         const void* send, void* recv, void* stream) {
  return guarded([&] {
    if (nprocs <= 0) dfft::fail(dfft::kErrInvalidArgument, "nprocs must be positive");
    dfft::Ext cart;
    if (comm_axis >= 0) cart = ext_of(cart_topology, cart_rank, "cart_topology");
    dfft::all2all_virtual(static_cast<std::size_t>(nprocs), ext_of(buffer_extents, buffer_rank, "buffer_extents"),
                          layout_right != 0, cart, comm_axis, element_bytes, send, recv,
                          static_cast<cudaStream_t>(stream));
  });
}

struct dfft_trans_block_s {
  dfft::TransBlockExec* impl;
};

dfft_status dfft_trans_block_create(dfft_trans_block** tb, const dfft_trans_block_desc* d) {
  return guarded([&] {
    if (!tb || !d) dfft::fail(dfft::kErrInvalidArgument, "null argument");
    *tb = nullptr;
    check_view_rank(d->rank);
    const int32_t D = d->rank;
    dfft::TransBlockDesc t;
    t.gext = ext_of(d->global_extents, D, "global_extents");
    t.in_topo = ext_of(d->in_topology, D, "in_topology");
    t.out_topo = ext_of(d->out_topology, D, "out_topology");
    t.in_right = d->in_topology_layout_right != 0;
    t.out_right = d->out_topology_layout_right != 0;
    t.src_map = map_of(d->src_map, D, "src_map");
    t.dst_map = map_of(d->dst_map, D, "dst_map");
    if (d->src_axis < 0 || d->src_axis >= D || d->dst_axis < 0 || d->dst_axis >= D)
      dfft::fail(dfft::kErrInvalidArgument, "axis out of range");
    t.src_axis = static_cast<std::size_t>(d->src_axis);
    t.dst_axis = static_cast<std::size_t>(d->dst_axis);
    t.view_right = d->view_layout_right != 0;
    t.elem_bytes = d->element_bytes;
    t.comm_axis = d->comm_axis;
    bool any = false;
    for (int32_t k = 0; k < D; ++k) any = any || d->cart_topology[k] != 0;
    if (any) t.cart_topology = ext_of(d->cart_topology, D, "cart_topology");
    auto* impl = new dfft::TransBlockExec(t);
    *tb = new dfft_trans_block_s{impl};
  });
}

static const dfft::TransBlockExec& tb_of(const dfft_trans_block* tb) {
  if (!tb || !tb->impl) dfft::fail(dfft::kErrInvalidArgument, "null trans block");
  return *tb->impl;
}

dfft_status dfft_trans_block_buffer_extents(const dfft_trans_block* tb, uint64_t* extents) {
  return guarded([&] {
    if (!extents) dfft::fail(dfft::kErrInvalidArgument, "null output");
    const auto& b = tb_of(tb).buffer_extents();
    for (std::size_t k = 0; k < b.size(); ++k) extents[k] = b[k];
  });
}

dfft_status dfft_trans_block_execute(const dfft_trans_block* tb, const void* in, void* out, void* send, void* recv,
                                     int32_t direction, void* stream) {
  return guarded([&] {
    if (direction != DFFT_FORWARD && direction != DFFT_BACKWARD)
      dfft::fail(dfft::kErrInvalidArgument, "Invalid FFT direction specified.");
    tb_of(tb).execute(in, out, send, recv, direction == DFFT_FORWARD, static_cast<cudaStream_t>(stream));
  });
}

dfft_status dfft_trans_block_destroy(dfft_trans_block* tb) {
  return guarded([&] {
    if (!tb) return;
    delete tb->impl;
    delete tb;
  });
}

// ---- layout math ----
dfft_status dfft_rank_to_coord(int32_t rank, const uint64_t* topology, int32_t layout_right, int64_t rank_id,
                               uint64_t* coord) {
  return guarded([&] {
    if (!coord) dfft::fail(dfft::kErrInvalidArgument, "null output");
    const dfft::Ext topo = ext_of(topology, rank, "topology");
    if (rank_id < 0 || static_cast<std::size_t>(rank_id) >= dfft::total_size(topo))
      dfft::fail(dfft::kErrInvalidArgument, "rank must be less than topology size.");
    const dfft::Ext c = dfft::rank_to_coord(topo, static_cast<std::size_t>(rank_id), layout_right != 0);
    for (std::size_t k = 0; k < c.size(); ++k) coord[k] = c[k];
  });
}

dfft_status dfft_compute_local_extents_and_starts(int32_t rank, const uint64_t* global_extents,
                                                  const uint64_t* topology, int32_t layout_right, int64_t rank_id,
                                                  uint64_t* extents, uint64_t* starts) {
  return guarded([&] {
    if (!extents || !starts) dfft::fail(dfft::kErrInvalidArgument, "null output");
    const dfft::Ext g = ext_of(global_extents, rank, "global_extents"), topo = ext_of(topology, rank, "topology");
    if (rank_id < 0 || static_cast<std::size_t>(rank_id) >= dfft::total_size(topo))
      dfft::fail(dfft::kErrInvalidArgument, "rank must be less than topology size.");
    const std::size_t r = static_cast<std::size_t>(rank_id);
    const dfft::Ext e = dfft::compute_local_extents(g, topo, dfft::identity_map(g.size()), r, layout_right != 0);
    const dfft::Ext st = dfft::compute_local_starts(g, topo, r, layout_right != 0);
    for (std::size_t k = 0; k < g.size(); ++k) {
      extents[k] = e[k];
      starts[k] = st[k];
    }
  });
}

dfft_status dfft_compute_buffer_extents(int32_t rank, const uint64_t* global_extents, const uint64_t* in_topology,
                                        const uint64_t* out_topology, int32_t layout_right,
                                        uint64_t* buffer_extents) {
  return guarded([&] {
    if (!buffer_extents) dfft::fail(dfft::kErrInvalidArgument, "null output");
    const dfft::Ext b = dfft::compute_buffer_extents(ext_of(global_extents, rank, "global_extents"),
                                                     ext_of(in_topology, rank, "in_topology"),
                                                     ext_of(out_topology, rank, "out_topology"), layout_right != 0);
    for (std::size_t k = 0; k < b.size(); ++k) buffer_extents[k] = b[k];
  });
}

dfft_status dfft_permute_map_by_axes(int32_t rank, const int32_t* src_map, int32_t naxes, const int32_t* axes,
                                     int32_t layout_right, int32_t* out_map) {
  return guarded([&] {
    if (!out_map) dfft::fail(dfft::kErrInvalidArgument, "null output");
    const dfft::Ext m = map_of(src_map, rank, "src_map");
    dfft::Ext ax;
    for (int32_t i = 0; i < naxes; ++i) {
      if (!axes || axes[i] < 0 || axes[i] >= rank) dfft::fail(dfft::kErrInvalidArgument, "axes out of range");
      ax.push_back(static_cast<std::size_t>(axes[i]));
    }
    const dfft::Ext r = dfft::permute_map_by_axes(m, ax, layout_right != 0);
    for (std::size_t k = 0; k < r.size(); ++k) out_map[k] = static_cast<int32_t>(r[k]);
  });
}

dfft_status dfft_propose_transpose_block(int32_t rank, const int32_t* map, const uint64_t* in_topology,
                                         const uint64_t* out_topology, const uint64_t* in_extents,
                                         const uint64_t* global_extents, int32_t naxes, const int32_t* axes,
                                         int64_t rank_id, int32_t is_layout_right, int32_t is_last, int32_t in_axis,
                                         int32_t out_axis, int32_t comm_axis, int64_t block_idx,
                                         int64_t size_factor, int32_t view_layout_right, dfft_block_info* info,
                                         uint64_t* max_buffer_size) {
  return guarded([&] {
    if (!info) dfft::fail(dfft::kErrInvalidArgument, "null output");
    check_view_rank(rank);
    dfft::Ext ax;
    for (int32_t i = 0; i < naxes; ++i) {
      if (!axes || axes[i] < 0 || axes[i] >= rank) dfft::fail(dfft::kErrInvalidArgument, "axes out of range");
      ax.push_back(static_cast<std::size_t>(axes[i]));
    }
    if (in_axis < 0 || out_axis < 0 || comm_axis < 0 || block_idx < 0 || size_factor < 0 || rank_id < 0)
      dfft::fail(dfft::kErrInvalidArgument, "negative index");
    std::size_t mb = 0;
    const dfft::BlockInfo b = dfft::propose_transpose(
        map_of(map, rank, "map"), ext_of(in_topology, rank, "in_topology"), ext_of(out_topology, rank, "out_topology"),
        ext_of(in_extents, rank, "in_extents"), ext_of(global_extents, rank, "global_extents"), ax,
        static_cast<std::size_t>(rank_id), is_layout_right != 0, is_last != 0, static_cast<std::size_t>(in_axis),
        static_cast<std::size_t>(out_axis), static_cast<std::size_t>(comm_axis), static_cast<std::size_t>(block_idx),
        static_cast<std::size_t>(size_factor), view_layout_right != 0, &mb);
    fill_block_info(b, info);
    if (max_buffer_size) *max_buffer_size = mb;
  });
}

const char* dfft_last_error_string(void) { return g_last_error.c_str(); }

const char* dfft_version(void) { return "dfft-b200 0.1.0"; }

}  // extern "C"
