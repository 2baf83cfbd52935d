// Pack, all-to-all, unpack and TransBlock on virtual ranks (see exchange.hpp).
#include "exchange.hpp"

#include <algorithm>
#include <cstring>
#include <numeric>
#include <string>

namespace dfft {

namespace {

void cuda_ok(cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    cudaGetLastError();
    fail(kErrCuda, std::string(what) + ": " + cudaGetErrorString(e));
  }
}

void check_elem(int eb) {
  if (eb != 4 && eb != 8 && eb != 16) fail(kErrInvalidArgument, "element size must be 4, 8 or 16 bytes");
}

void check_ptr(const void* p, int eb, const char* which) {
  if (!p) fail(kErrInvalidArgument, std::string("null ") + which + " buffer");
  if (reinterpret_cast<std::uintptr_t>(p) % static_cast<std::uintptr_t>(eb) != 0)
    fail(kErrInvalidArgument, std::string(which) + " buffer is not aligned to its element size");
}

void check_map(const Ext& map, std::size_t D, const char* which) {
  if (map.size() != D) fail(kErrInvalidArgument, std::string(which) + " must have the view rank");
  Ext s = map;
  std::sort(s.begin(), s.end());
  for (std::size_t i = 0; i < D; ++i)
    if (s[i] != i) fail(kErrInvalidArgument, std::string(which) + " must be a permutation of the view's axes");
}

// Logical extents of a view whose dimension i holds logical axis map[i].
Ext unmap_extents(const Ext& mapped, const Ext& map) {
  Ext l(mapped.size());
  for (std::size_t i = 0; i < map.size(); ++i) l[map[i]] = mapped[i];
  return l;
}

bool overlap(const void* a, std::size_t na, const void* b, std::size_t nb) {
  const auto pa = reinterpret_cast<std::uintptr_t>(a), pb = reinterpret_cast<std::uintptr_t>(b);
  return pa < pb + nb && pb < pa + na;
}

// One rank's local view as a layout (topology of ones).
Layout local_layout(const Ext& lext, const Ext& map, bool right, int eb) {
  Layout L;
  L.gext = lext;
  L.topo.assign(lext.size(), 1);
  L.rank_right = true;
  L.map = map;
  L.view_right = right;
  L.complex = eb != 4;
  return L;
}

dev::XposeArgs base_args(const Ext& bext, bool right, std::size_t nprocs, std::size_t pc) {
  dev::XposeArgs X;
  std::memset(&X, 0, sizeof(X));
  X.nd = static_cast<int>(bext.size() - 1);
  X.nprocs = static_cast<int>(nprocs);
  X.pc = static_cast<int>(pc);
  X.rs = static_cast<int>(9 + pc);
  for (std::size_t k = 0; k < bext.size(); ++k) X.bext[k] = static_cast<std::int64_t>(bext[k]);
  X.buf_right = right ? 1 : 0;
  X.bufsize = static_cast<std::int64_t>(total_size(bext));
  return X;
}

// Pack (op 0) or unpack (op 2) of one rank's view through the transpose kernels.
void local_xpose(int op, const Ext& view_ext, const Ext& map, std::size_t axis, const Ext& bext, bool right, int eb,
                 const void* src, void* dst, cudaStream_t st) {
  const std::size_t D = view_ext.size();
  if (D < 2 || D > static_cast<std::size_t>(kMaxRank)) fail(kErrInvalidArgument, "view rank must be in [2, 4]");
  if (bext.size() != D + 1) fail(kErrInvalidArgument, "the buffer rank must be the view rank + 1");
  check_map(map, D, "map");
  if (axis >= D) fail(kErrInvalidArgument, "axis out of range");
  check_elem(eb);
  check_ptr(src, eb, "source");
  check_ptr(dst, eb, "destination");
  const Ext lext = unmap_extents(view_ext, map);
  const std::size_t pc = right ? bext.front() : bext.back();
  if (pc == 0) fail(kErrInvalidArgument, "the buffer has no process dimension");
  const std::size_t nview = total_size(view_ext), nbuf = total_size(bext);
  if (op == 0 ? overlap(src, nview * eb, dst, nbuf * eb) : overlap(src, nbuf * eb, dst, nview * eb))
    fail(kErrInvalidArgument, "source and destination must not alias");
  if (nbuf == 0 || nview == 0) return;
  const Layout L = local_layout(lext, map, right, eb);
  const LayoutTables T = build_layout_tables(L);
  std::vector<std::int64_t> tab = T.data;
  const std::size_t geo_at = tab.size();
  for (int k = 0; k < 4; ++k) tab.push_back(0);  // starts
  for (int k = 0; k < 4; ++k) tab.push_back(k < static_cast<int>(D) ? static_cast<std::int64_t>(lext[k]) : 0);
  tab.push_back(0);                                  // sub-rank (unused by pack / unpack)
  for (std::size_t j = 0; j < pc; ++j) tab.push_back(0);  // members (unused)
  std::int64_t* d = nullptr;
  cuda_ok(cudaMallocAsync(reinterpret_cast<void**>(&d), tab.size() * sizeof(std::int64_t), st), "table allocation");
  cudaError_t e = cudaMemcpyAsync(d, tab.data(), tab.size() * sizeof(std::int64_t), cudaMemcpyHostToDevice, st);
  dev::XposeArgs X = base_args(bext, right, 1, pc);
  X.axis = static_cast<int>(axis);
  X.merged = static_cast<std::int64_t>(lext[axis]);
  X.geo = d + geo_at;
  X.lay = device_layout_at(T, d);
  X.src = src;
  X.dst = dst;
  if (e == cudaSuccess) e = dev::launch_xpose(op, X, eb, st);
  const cudaError_t ef = cudaFreeAsync(d, st);
  cuda_ok(e, op == 0 ? "pack" : "unpack");
  cuda_ok(ef, "table release");
}

}  // namespace

ExchangeGroup exchange_group(std::size_t nprocs, const Ext& cart_topology, int comm_axis, std::size_t rank) {
  ExchangeGroup g;
  if (comm_axis < 0) {
    g.sub = rank;
    g.members.resize(nprocs);
    std::iota(g.members.begin(), g.members.end(), std::size_t(0));
    return g;
  }
  std::vector<std::size_t> dims;
  for (auto t : cart_topology)
    if (t > 1) dims.push_back(t);
  if (dims.size() != 2)
    fail(kErrInvalidTopology, "a row / column communicator needs a Cartesian topology with two split axes");
  if (dims[0] * dims[1] != nprocs) fail(kErrInvalidTopology, "the Cartesian topology does not cover every rank");
  const std::size_t t1 = dims[1], c0 = rank / t1, c1 = rank % t1;
  if (comm_axis == 0) {
    g.sub = c0;
    for (std::size_t j = 0; j < dims[0]; ++j) g.members.push_back(j * t1 + c1);
  } else if (comm_axis == 1) {
    g.sub = c1;
    for (std::size_t j = 0; j < dims[1]; ++j) g.members.push_back(c0 * t1 + j);
  } else {
    fail(kErrInvalidArgument, "comm_axis must be -1 (all ranks), 0 (row) or 1 (column)");
  }
  return g;
}

void append_exchange_geo(std::vector<std::int64_t>& out, const Layout& L, const Ext& cart_topology, int comm_axis,
                         std::size_t pc) {
  const std::size_t P = L.nprocs();
  const auto blocks = layout_blocks(L);
  const std::size_t D = L.gext.size();
  for (std::size_t r = 0; r < P; ++r) {
    for (std::size_t k = 0; k < 4; ++k) out.push_back(k < D ? static_cast<std::int64_t>(blocks[r].starts[k]) : 0);
    for (std::size_t k = 0; k < 4; ++k) out.push_back(k < D ? static_cast<std::int64_t>(blocks[r].local[k]) : 0);
    const ExchangeGroup g = exchange_group(P, cart_topology, comm_axis, r);
    if (g.members.size() != pc) fail(kErrInternal, "communicator size does not match the buffer's process extent");
    out.push_back(static_cast<std::int64_t>(g.sub));
    for (auto m : g.members) out.push_back(static_cast<std::int64_t>(m));
  }
}

dev::DevLayout device_layout_at(const LayoutTables& T, const std::int64_t* base) {
  dev::DevLayout L;
  std::memset(&L, 0, sizeof(L));
  L.t = base;
  L.mode = T.mode;
  for (int k = 0; k < 4; ++k) {
    L.off[k] = T.off[k];
    L.rk[k] = T.rk[k];
    L.loc[k] = T.loc[k];
  }
  L.rbase = T.rbase;
  L.rstride = T.rstride;
  return L;
}

void pack_local(const Ext& src_extents, const Ext& map, std::size_t axis, const Ext& buffer_extents, bool layout_right,
                int elem_bytes, const void* src, void* dst, cudaStream_t stream) {
  local_xpose(0, src_extents, map, axis, buffer_extents, layout_right, elem_bytes, src, dst, stream);
}

void unpack_local(const Ext& buffer_extents, const Ext& map, std::size_t axis, const Ext& dst_extents,
                  bool layout_right, int elem_bytes, const void* src, void* dst, cudaStream_t stream) {
  local_xpose(2, dst_extents, map, axis, buffer_extents, layout_right, elem_bytes, src, dst, stream);
}

void all2all_virtual(std::size_t nprocs, const Ext& buffer_extents, bool layout_right, const Ext& cart_topology,
                     int comm_axis, int elem_bytes, const void* send, void* recv, cudaStream_t stream) {
  if (nprocs == 0) fail(kErrInvalidArgument, "nprocs must be positive");
  if (buffer_extents.size() < 2) fail(kErrInvalidArgument, "all2all: View rank must be larger than or equal to 2");
  check_elem(elem_bytes);
  check_ptr(send, elem_bytes, "send");
  check_ptr(recv, elem_bytes, "recv");
  const std::size_t pc = layout_right ? buffer_extents.front() : buffer_extents.back();
  const std::size_t gsize = exchange_group(nprocs, cart_topology, comm_axis, 0).members.size();
  // KokkosFFT_Distributed_MPI_All2All.hpp:43-51
  if (pc != gsize)
    fail(kErrInvalidArgument, "Extent of dimension to be transposed of send (" + std::to_string(pc) + ") or recv (" +
                                  std::to_string(pc) + ") buffer does not match MPI size: " + std::to_string(gsize));
  const std::size_t per = total_size(buffer_extents);
  if (overlap(send, nprocs * per * elem_bytes, recv, nprocs * per * elem_bytes))
    fail(kErrInvalidArgument, "send and recv buffers must not alias");
  if (per == 0) return;
  std::vector<std::int64_t> tab;
  for (std::size_t r = 0; r < nprocs; ++r) {
    for (int k = 0; k < 8; ++k) tab.push_back(0);
    const ExchangeGroup g = exchange_group(nprocs, cart_topology, comm_axis, r);
    tab.push_back(static_cast<std::int64_t>(g.sub));
    for (auto m : g.members) tab.push_back(static_cast<std::int64_t>(m));
  }
  std::int64_t* d = nullptr;
  cuda_ok(cudaMallocAsync(reinterpret_cast<void**>(&d), tab.size() * sizeof(std::int64_t), stream), "table allocation");
  cudaError_t e = cudaMemcpyAsync(d, tab.data(), tab.size() * sizeof(std::int64_t), cudaMemcpyHostToDevice, stream);
  dev::XposeArgs X = base_args(buffer_extents, layout_right, nprocs, pc);
  X.geo = d;
  X.src = send;
  X.dst = recv;
  if (e == cudaSuccess) e = dev::launch_xpose(1, X, elem_bytes, stream);
  const cudaError_t ef = cudaFreeAsync(d, stream);
  cuda_ok(e, "all2all");
  cuda_ok(ef, "table release");
}

TransBlockExec::TransBlockExec(const TransBlockDesc& d) : d_(d) {
  const std::size_t D = d.gext.size();
  if (D < 2 || D > static_cast<std::size_t>(kMaxRank)) fail(kErrInvalidArgument, "view rank must be in [2, 4]");
  if (d.in_topo.size() != D || d.out_topo.size() != D)
    fail(kErrInvalidArgument, "topologies must have the view rank");
  for (std::size_t k = 0; k < D; ++k)
    if (d.gext[k] == 0 || d.in_topo[k] == 0 || d.out_topo[k] == 0)
      fail(kErrInvalidArgument, "extents and topologies must be positive");
  check_map(d.src_map, D, "src_map");
  check_map(d.dst_map, D, "dst_map");
  if (d.src_axis >= D || d.dst_axis >= D) fail(kErrInvalidArgument, "axis out of range");
  check_elem(d.elem_bytes);
  P_ = total_size(d.in_topo);
  if (P_ != total_size(d.out_topo))
    fail(kErrInvalidTopology, "in_topology and out_topology must have the same size.");
  const Ext cart = d.cart_topology.empty() ? d.in_topo : d.cart_topology;
  bext_ = compute_buffer_extents(d.gext, d.in_topo, d.out_topo, d.view_right);
  const std::size_t pc = d.view_right ? bext_.front() : bext_.back();
  auto make = [&](const Ext& topo, bool rr, const Ext& map) {
    Layout L;
    L.gext = d.gext;
    L.topo = topo;
    L.rank_right = rr;
    L.map = map;
    L.view_right = d.view_right;
    L.complex = d.elem_bytes != 4;
    return L;
  };
  lin_ = make(d.in_topo, d.in_right, d.src_map);
  lout_ = make(d.out_topo, d.out_right, d.dst_map);
  // TransBlock::good (KokkosFFT_Distributed_TransBlock.hpp:120-186): every
  // rank's view must fit its buffer
  const std::size_t per = total_size(bext_);
  for (const Layout* L : {&lin_, &lout_})
    for (const auto& b : layout_blocks(*L))
      if (b.size > per)
        fail(kErrInvalidArgument, "Input view size must be smaller than the send buffer size");
  const LayoutTables Ti = build_layout_tables(lin_), To = build_layout_tables(lout_);
  std::vector<std::int64_t> tab = Ti.data;
  const std::size_t at_o = tab.size();
  tab.insert(tab.end(), To.data.begin(), To.data.end());
  const std::size_t geo_i = tab.size();
  append_exchange_geo(tab, lin_, cart, d.comm_axis, pc);
  const std::size_t geo_o = tab.size();
  append_exchange_geo(tab, lout_, cart, d.comm_axis, pc);
  cuda_ok(cudaMalloc(reinterpret_cast<void**>(&d_tables_), tab.size() * sizeof(std::int64_t)), "table allocation");
  const cudaError_t e =
      cudaMemcpy(d_tables_, tab.data(), tab.size() * sizeof(std::int64_t), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    cudaFree(d_tables_);
    d_tables_ = nullptr;
    cuda_ok(e, "table upload");
  }
  const dev::DevLayout Di = device_layout_at(Ti, d_tables_), Do = device_layout_at(To, d_tables_ + at_o);
  const dev::XposeArgs X = base_args(bext_, d.view_right, P_, pc);
  // forward: pack the input layout along src_axis, merge dst_axis into the
  // output layout; backward: the reverse (TransBlock.hpp:97-101)
  for (int dir = 0; dir < 2; ++dir) {
    const bool fwd = dir == 0;
    const std::size_t pa = fwd ? d.src_axis : d.dst_axis, ua = fwd ? d.dst_axis : d.src_axis;
    pack_[dir] = X;
    pack_[dir].axis = static_cast<int>(pa);
    pack_[dir].merged = static_cast<std::int64_t>(d.gext[pa]);
    pack_[dir].lay = fwd ? Di : Do;
    pack_[dir].geo = d_tables_ + (fwd ? geo_i : geo_o);
    a2a_[dir] = X;
    a2a_[dir].geo = pack_[dir].geo;
    unpack_[dir] = X;
    unpack_[dir].axis = static_cast<int>(ua);
    unpack_[dir].merged = static_cast<std::int64_t>(d.gext[ua]);
    unpack_[dir].lay = fwd ? Do : Di;
    unpack_[dir].geo = d_tables_ + (fwd ? geo_o : geo_i);
  }
}

TransBlockExec::~TransBlockExec() {
  if (d_tables_) cudaFree(d_tables_);
}

void TransBlockExec::execute(const void* in, void* out, void* send, void* recv, bool forward,
                             cudaStream_t stream) const {
  const int eb = d_.elem_bytes;
  check_ptr(in, eb, "input");
  check_ptr(out, eb, "output");
  check_ptr(send, eb, "send");
  check_ptr(recv, eb, "recv");
  const std::size_t nin = layout_elements(forward ? lin_ : lout_) * eb;
  const std::size_t nout = layout_elements(forward ? lout_ : lin_) * eb;
  const std::size_t nbuf = P_ * total_size(bext_) * eb;
  // TransBlock.hpp:166-185
  if (overlap(in, nin, send, nbuf)) fail(kErrInvalidArgument, "Input view must not be aliasing with send buffer");
  if (overlap(out, nout, recv, nbuf)) fail(kErrInvalidArgument, "Output view must not be aliasing with receive buffer");
  if (overlap(send, nbuf, recv, nbuf)) fail(kErrInvalidArgument, "send and recv buffers must not alias");
  if (total_size(bext_) == 0) return;
  const int dir = forward ? 0 : 1;
  dev::XposeArgs X = pack_[dir];
  X.src = in;
  X.dst = send;
  cuda_ok(dev::launch_xpose(0, X, eb, stream), "pack");
  X = a2a_[dir];
  X.src = send;
  X.dst = recv;
  cuda_ok(dev::launch_xpose(1, X, eb, stream), "all2all");
  X = unpack_[dir];
  X.src = recv;
  X.dst = out;
  cuda_ok(dev::launch_xpose(2, X, eb, stream), "unpack");
}

}  // namespace dfft
