// Plan construction and execution.
//
// Validation follows internal_plan_factory (KokkosFFT_Distributed_Plan.hpp:46-113)
// and the Slab/Pencil plan constructors; the block lists come from the
// restated block analyses; normalisation follows the SlabPlan / PencilPlan
// wrappers (KokkosFFT_Distributed_SlabPlan.hpp:1344-1358,
// KokkosFFT_Distributed_PencilPlan.hpp:1680-1690).
//
// Two device programs exist per direction:
//   fused   - one FFT stage kernel per FFT axis.  The first stage gathers from
//             the caller's input blocks, the last scatters into the caller's
//             output blocks, the stages in between use a plain global array.
//             Every exchange of the reference (pack, all-to-all, unpack, local
//             transposes) is a re-addressing inside those gathers / scatters,
//             and the normalisation is a factor in the last scatter.
//   literal - the reference's block sequence kernel by kernel on per-rank
//             blocks: local transpose, per-axis FFTs, pack, all-to-all,
//             unpack, normalisation pass.  Its send / recv buffers are kept
//             for bit-exact comparison with the reference's buffers.
#include "plan.hpp"

#include <cuda.h>

#include "exchange.hpp"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <fstream>
#include <limits>
#include <mutex>
#include <sstream>
#include <cstring>

namespace dfft {

namespace {

void cuda_check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) fail(kErrCuda, std::string(what) + ": " + cudaGetErrorString(e));
}

// Radix plan of a transform length: passes of 8 (with 4,4 or 4 or 2 to finish
// a power of two), then 3, 5, 7, 11, 13.
std::vector<int> radix_plan(std::size_t n) {
  std::vector<int> r;
  if (n == 0) fail(kErrInvalidExtents, "FFT length 0");
  std::size_t m = n;
  int k2 = 0;
  while (m % 2 == 0) {
    m /= 2;
    ++k2;
  }
  int q = k2 / 3, rem = k2 % 3;
  if (rem == 1) {
    if (q >= 1) {
      --q;
      r.push_back(4);
      r.push_back(4);
    } else {
      r.push_back(2);
    }
  } else if (rem == 2) {
    r.push_back(4);
  }
  for (int i = 0; i < q; ++i) r.push_back(8);
  for (int p : {3, 5, 7, 11, 13}) {
    while (m % static_cast<std::size_t>(p) == 0) {
      m /= static_cast<std::size_t>(p);
      r.push_back(p);
    }
  }
  if (m != 1)
    fail(kErrUnsupported, "FFT length " + std::to_string(n) + " has a prime factor larger than 13");
  if (r.size() > static_cast<std::size_t>(dev::kMaxPasses)) fail(kErrUnsupported, "too many FFT passes");
  return r;
}

// Whether radix_plan covers n (prime factors up to 13, few enough passes).
bool radix_supported(std::size_t n) {
  if (n == 0) return false;
  std::size_t m = n;
  int k2 = 0;
  while (m % 2 == 0) {
    m /= 2;
    ++k2;
  }
  int passes = k2 / 3 + (k2 % 3 != 0 ? 1 : 0);  // the radix-8 / 4 / 2 passes of radix_plan
  for (std::size_t p : {3, 5, 7, 11, 13})
    while (m % p == 0) {
      m /= p;
      ++passes;
    }
  return m == 1 && passes <= dev::kMaxPasses;
}

// In-place radix-2 FFT (exp(-2 pi i jk / m)) of m = 2^k long double values.
void host_fft(std::vector<long double>& re, std::vector<long double>& im) {
  const std::size_t m = re.size();
  for (std::size_t i = 1, j = 0; i < m; ++i) {
    std::size_t bit = m >> 1;
    for (; j & bit; bit >>= 1) j ^= bit;
    j ^= bit;
    if (i < j) {
      std::swap(re[i], re[j]);
      std::swap(im[i], im[j]);
    }
  }
  const long double pi = 3.141592653589793238462643383279502884L;
  for (std::size_t len = 2; len <= m; len <<= 1) {
    for (std::size_t k = 0; k < len / 2; ++k) {
      const long double ang = -2.0L * pi * static_cast<long double>(k) / static_cast<long double>(len);
      const long double wr = cosl(ang), wi = sinl(ang);
      for (std::size_t i = k; i < m; i += len) {
        const std::size_t j = i + len / 2;
        const long double xr = re[j] * wr - im[j] * wi, xi = re[j] * wi + im[j] * wr;
        re[j] = re[i] - xr;
        im[j] = im[i] - xi;
        re[i] += xr;
        im[i] += xi;
      }
    }
  }
}

}  // namespace

// ---------------------------------------------------------------------------
// Construction
// ---------------------------------------------------------------------------
Plan::Plan(const PlanDesc& d, bool on_device) : d_(d), on_device_(on_device) {
  analyze();
  if (is_rank_plan()) {
    if (static_cast<std::size_t>(d_.rank) >= nprocs())
      fail(kErrInvalidArgument, "rank must be less than topology size.");
    if (d_.exec_mode != 0) fail(kErrInvalidArgument, "per-rank plans run the fused execution mode only");
    rank_exchanges(true);
    rank_exchanges(false);
  }
  if (!on_device_) return;
  try {
    if (is_rank_plan()) {
      build_rank(true);
      build_rank(false);
      allocate_device();
      autotune();
      return;
    }
    build_fused(true);
    build_fused(false);
    build_adjoint(true);
    build_adjoint(false);
    if (d_.exec_mode == 1 || d_.exec_mode == 2) {
      prog_[0].clear();
      prog_[1].clear();
      build_literal(true);
      build_literal(false);
    }
    allocate_device();
    autotune();
  } catch (...) {
    for (auto p : bufs_)
      if (p) cudaFree(p);
    for (auto& kv : twiddles_) cudaFree(kv.second);
    if (d_tables_) cudaFree(d_tables_);
    if (d_err_) cudaFree(d_err_);
    for (auto& kv : blue_tables_)
      for (void* p : kv.second) cudaFree(p);
    throw;
  }
}

Plan::~Plan() {
  for (auto p : bufs_)
    if (p) cudaFree(p);
  for (auto& kv : twiddles_) cudaFree(kv.second);
  if (d_tables_) cudaFree(d_tables_);
  if (d_err_) cudaFree(d_err_);
  for (auto& kv : blue_tables_)
    for (void* p : kv.second) cudaFree(p);
}

void Plan::analyze() {
  const std::size_t D = d_.gin.size();
  if (D < 2 || D > static_cast<std::size_t>(kMaxRank)) fail(kErrInvalidArgument, "view rank must be in [2, 4]");
  if (d_.gout.size() != D || d_.in_topo.size() != D || d_.out_topo.size() != D)
    fail(kErrInvalidArgument, "extents and topologies must have the view rank");
  for (std::size_t k = 0; k < D; ++k) {
    if (d_.gin[k] == 0 || d_.gout[k] == 0) fail(kErrInvalidExtents, "extents must be positive");
    if (d_.gin[k] >= (1u << 30) || d_.gout[k] >= (1u << 30)) fail(kErrUnsupported, "extent too large");
  }
  // internal_plan_factory (Plan.hpp:59-72)
  if (total_size(d_.in_topo) != total_size(d_.out_topo))
    fail(kErrInvalidTopology, "in_topology and out_topology must have the same size.");
  check_valid_extents(d_.gin, d_.gout, d_.axes, d_.r2c, d_.view_right);

  type_ = get_common_topology_type({d_.in_topo, d_.out_topo});
  switch (type_) {
    case TopologyType::Shared: name_ = "SharedPlan"; break;
    case TopologyType::Slab: name_ = "SlabPlan"; break;
    case TopologyType::Pencil:
      if (D < 3) fail(kErrInvalidTopology, "Pencil plan supports 3D or higher dimensional Views");
      name_ = "PencilPlan";
      break;
    case TopologyType::Empty: fail(kErrInvalidTopology, "Empty topology is not supported for FFT plan.");
    case TopologyType::Brick: fail(kErrInvalidTopology, "Brick topology is not supported for FFT plan.");
    default: fail(kErrInvalidTopology, "Unsupported topology for FFT plan.");
  }

  const std::size_t P = nprocs();
  if (type_ == TopologyType::Slab) {
    chain_ = get_all_slab_topologies(d_.in_topo, d_.out_topo, d_.axes);
    chain_layouts_.assign(chain_.size(), 1);
    trans_axes_.assign(chain_.size() - 1, 0);
  } else if (type_ == TopologyType::Pencil) {
    auto ch = get_all_pencil_topologies(d_.in_topo, d_.in_right, d_.out_topo, d_.out_right, d_.axes);
    chain_ = ch.topologies;
    trans_axes_ = ch.trans_axes;
    chain_layouts_ = ch.layouts;
  } else {
    chain_ = {d_.in_topo};
    chain_layouts_ = {d_.in_right ? 1u : 0u};
  }

  per_rank_.resize(P);
  for (std::size_t r = 0; r < P; ++r) {
    Ext in_ext = compute_local_extents(d_.gin, d_.in_topo, identity_map(D), r, d_.in_right);
    if (type_ == TopologyType::Slab) {
      per_rank_[r] = slab_block_analyses(in_ext, d_.gin, d_.gout, d_.in_topo, d_.out_topo, d_.axes, d_.r2c,
                                         d_.view_right, r);
      if (per_rank_[r].blocks.empty() || per_rank_[r].blocks.size() > 5)
        fail(kErrInternal, "Number blocks must be in [1, 5]");
    } else if (type_ == TopologyType::Pencil) {
      per_rank_[r] = pencil_block_analyses(in_ext, d_.gin, d_.gout, d_.in_topo, d_.in_right, d_.out_topo,
                                           d_.out_right, d_.axes, d_.r2c, d_.view_right, r);
      if (per_rank_[r].blocks.empty() || per_rank_[r].blocks.size() > 8)
        fail(kErrInternal, "Number blocks must be in [1, 8]");
    } else {
      // SharedPlan (KokkosFFT_Distributed_SharedPlan.hpp:15-84): one local FFT.
      BlockInfo b;
      Ext map = get_map_axes(D, d_.axes, d_.view_right);
      b.block_type = BlockType::FFT;
      b.fft_dim = d_.axes.size();
      b.in_map = b.out_map = map;
      b.in_extents = compute_mapped_extents(d_.gin, map);
      b.out_extents = compute_mapped_extents(d_.gout, map);
      b.in_topology.assign(D, 0);
      b.out_topology.assign(D, 0);
      b.buffer_extents.assign(D + 1, 0);
      per_rank_[r].blocks = {b};
      per_rank_[r].max_buffer_size = total_size(d_.gout) * 2;
    }
    max_buffer_size_ = std::max(max_buffer_size_, per_rank_[r].max_buffer_size);
  }

  // Normalisation (KokkosFFT::Impl::normalize semantics).
  Ext fft_ext = compute_fft_extents(d_.gin, d_.gout, d_.axes);
  const double N = static_cast<double>(total_size(fft_ext));
  switch (d_.norm) {
    case 0: scale_fwd_ = 1.0; scale_bwd_ = 1.0 / N; break;
    case 1: scale_fwd_ = 1.0 / N; scale_bwd_ = 1.0; break;
    case 2: scale_fwd_ = scale_bwd_ = 1.0 / std::sqrt(N); break;
    case 3: scale_fwd_ = scale_bwd_ = 1.0; break;
    default: fail(kErrInvalidArgument, "unknown normalization");
  }

  lin_.gext = d_.gin;
  lin_.topo = d_.in_topo;
  lin_.rank_right = d_.in_right;
  lin_.map = identity_map(D);
  lin_.view_right = d_.view_right;
  lin_.complex = !d_.r2c;
  lout_.gext = d_.gout;
  lout_.topo = d_.out_topo;
  lout_.rank_right = d_.out_right;
  lout_.map = identity_map(D);
  lout_.view_right = d_.view_right;
  lout_.complex = true;
}

int Plan::add_layout(const Layout& L) {
  for (std::size_t i = 0; i < layouts_.size(); ++i)
    if (layouts_[i] == L) return static_cast<int>(i);
  layouts_.push_back(L);
  tables_.push_back(build_layout_tables(L));
  layout_base_.push_back(static_cast<std::int64_t>(host_tables_.size()));
  auto& t = tables_.back().data;
  host_tables_.insert(host_tables_.end(), t.begin(), t.end());
  return static_cast<int>(layouts_.size() - 1);
}

Layout Plan::block_layout(const Ext& topo, bool rank_right, const Ext& map, bool complex) const {
  Layout L;
  L.gext = complex ? d_.gout : d_.gin;
  L.topo = topo;
  L.rank_right = rank_right;
  L.map = map;
  L.view_right = d_.view_right;
  L.complex = complex;
  return L;
}

// FFT axes in the order the reference transforms them in the forward
// direction: FFT blocks in sequence, each block's axes from the innermost
// (unit-stride) one outwards.  The first axis is the R2C axis.
std::vector<std::size_t> Plan::fft_axis_order() const {
  std::vector<std::size_t> order;
  const std::size_t D = d_.gin.size();
  for (auto& b : per_rank_.at(0).blocks) {
    if (b.block_type != BlockType::FFT) continue;
    for (std::size_t i = 0; i < b.fft_dim; ++i) order.push_back(d_.view_right ? b.in_map[D - 1 - i] : b.in_map[i]);
  }
  Ext sorted_order(order.begin(), order.end()), sorted_axes = d_.axes;
  std::sort(sorted_order.begin(), sorted_order.end());
  std::sort(sorted_axes.begin(), sorted_axes.end());
  if (sorted_order != sorted_axes) fail(kErrInternal, "FFT blocks do not cover the FFT axes");
  return order;
}

const void* Plan::twiddle(std::size_t n) {
  auto key = std::make_pair(n, d_.dbl);
  auto it = twiddles_.find(key);
  if (it != twiddles_.end()) return it->second;
  const long double pi = 3.141592653589793238462643383279502884L;
  std::vector<double> hd(2 * n);
  std::vector<float> hf(2 * n);
  for (std::size_t k = 0; k < n; ++k) {
    const long double ang = 2.0L * pi * static_cast<long double>(k) / static_cast<long double>(n);
    const long double c = cosl(ang), s = -sinl(ang);
    hd[2 * k] = static_cast<double>(c);
    hd[2 * k + 1] = static_cast<double>(s);
    hf[2 * k] = static_cast<float>(c);
    hf[2 * k + 1] = static_cast<float>(s);
  }
  void* p = nullptr;
  const std::size_t bytes = n * (d_.dbl ? 16 : 8);
  if (cudaMalloc(&p, bytes) != cudaSuccess) fail(kErrAlloc, "cudaMalloc of twiddle table failed");
  twiddles_[key] = p;
  workspace_bytes_ += bytes;
  cuda_check(cudaMemcpy(p, d_.dbl ? static_cast<const void*>(hd.data()) : static_cast<const void*>(hf.data()), bytes,
                        cudaMemcpyHostToDevice),
             "twiddle upload");
  return p;
}

// Chirp and filter tables of an n-point chirp-z stage with m-point FFTs, in
// the plan's precision: chirp c_j = exp(-i pi (j^2 mod 2n) / n), j < n; the
// forward filter is FFT_m(b) / m with b_j = conj(c_j) for j < n, b_{m-j} = b_j
// for 0 < j < n and 0 elsewhere, the inverse filter the same for the
// conjugate chirp.  Computed in long double on the host.
void Plan::bluestein_tables(std::size_t n, std::size_t m, const void** chirp, const void** ffwd, const void** finv) {
  auto key = std::make_pair(n, m);
  auto it = blue_tables_.find(key);
  if (it == blue_tables_.end()) {
    const long double pi = 3.141592653589793238462643383279502884L;
    std::vector<long double> cr(n), ci(n);
    for (std::size_t j = 0; j < n; ++j) {
      const unsigned long long q = (static_cast<unsigned long long>(j) * j) % (2ull * n);
      const long double ang = -pi * static_cast<long double>(q) / static_cast<long double>(n);
      cr[j] = cosl(ang);
      ci[j] = sinl(ang);
    }
    std::vector<std::vector<long double>> tabs;  // chirp (re, im interleaved), filters
    std::vector<long double> ch(2 * n);
    for (std::size_t j = 0; j < n; ++j) {
      ch[2 * j] = cr[j];
      ch[2 * j + 1] = ci[j];
    }
    tabs.push_back(ch);
    for (int dir = 0; dir < 2; ++dir) {
      // forward chirp c: b = conj(c); inverse chirp conj(c): b = c
      std::vector<long double> br(m, 0.0L), bi(m, 0.0L);
      for (std::size_t j = 0; j < n; ++j) {
        const long double im = dir == 0 ? -ci[j] : ci[j];
        br[j] = cr[j];
        bi[j] = im;
        if (j > 0) {
          br[m - j] = cr[j];
          bi[m - j] = im;
        }
      }
      host_fft(br, bi);
      std::vector<long double> f(2 * m);
      for (std::size_t k = 0; k < m; ++k) {
        f[2 * k] = br[k] / static_cast<long double>(m);
        f[2 * k + 1] = bi[k] / static_cast<long double>(m);
      }
      tabs.push_back(f);
    }
    std::vector<void*> ptrs;
    for (auto& t : tabs) {
      const std::size_t bytes = t.size() * (d_.dbl ? 8 : 4);
      void* p = nullptr;
      if (cudaMalloc(&p, bytes) != cudaSuccess) {
        cudaGetLastError();
        for (void* q : ptrs) cudaFree(q);
        fail(kErrAlloc, "cudaMalloc of chirp-z tables failed");
      }
      ptrs.push_back(p);
      workspace_bytes_ += bytes;
      cudaError_t e;
      if (d_.dbl) {
        std::vector<double> h(t.begin(), t.end());
        e = cudaMemcpy(p, h.data(), bytes, cudaMemcpyHostToDevice);
      } else {
        std::vector<float> h(t.begin(), t.end());
        e = cudaMemcpy(p, h.data(), bytes, cudaMemcpyHostToDevice);
      }
      if (e != cudaSuccess) {
        for (void* q : ptrs) cudaFree(q);
        fail(kErrCuda, std::string("chirp-z table upload: ") + cudaGetErrorString(e));
      }
    }
    it = blue_tables_.emplace(key, ptrs).first;
  }
  *chirp = it->second[0];
  *ffwd = it->second[1];
  *finv = it->second[2];
}

void Plan::push_stage(std::vector<Op>& prog, const Op& op) {
  if (op.four_n1 > 0) {
    // four-step: z = the lines as (lines, n2, n1) arrays (j = j1 + n1 j2);
    // FFT over j2, twiddle w_n^(j1 k2), FFT over j1, scatter k = k2 + n2 k1
    const std::size_t nl = static_cast<std::size_t>(op.blue_lines);
    const std::size_t n1 = static_cast<std::size_t>(op.four_n1), n2 = static_cast<std::size_t>(op.four_n2);
    Layout Z;
    Z.gext = {nl, n2, n1};
    Z.topo = {1, 1, 1};
    Z.map = identity_map(3);
    Z.view_right = true;
    Z.complex = true;
    const int lz = add_layout(Z);
    const std::size_t zb = nl * n1 * n2 * (d_.dbl ? 16 : 8);
    const int z1 = debug_buffer(-3, 0, 0, zb), z2 = debug_buffer(-3, 0, 1, zb);
    Op pre = op;
    pre.type = Op::BluePre;
    pre.dst = z1;
    prog.push_back(pre);
    Op f1 = make_stage(lz, lz, 1, dev::kC2C, op.inverse, 1.0);
    f1.src = z1;
    f1.dst = z2;
    push_stage(prog, f1);
    Op tw = op;
    tw.type = Op::FourTwiddle;
    tw.src = tw.dst = z2;
    prog.push_back(tw);
    Op f2 = make_stage(lz, lz, 2, dev::kC2C, op.inverse, 1.0);
    f2.src = z2;
    f2.dst = z1;
    push_stage(prog, f2);
    Op post = op;
    post.type = Op::BluePost;
    post.src = z1;
    prog.push_back(post);
    return;
  }
  if (!op.blue) {
    prog.push_back(op);
    return;
  }
  const std::size_t nl = static_cast<std::size_t>(op.blue_lines), m = static_cast<std::size_t>(op.blue_m);
  Layout Z;
  Z.gext = {nl, m};
  Z.topo = {1, 1};
  Z.map = identity_map(2);
  Z.view_right = true;
  Z.complex = true;
  const int lz = add_layout(Z);
  const std::size_t zb = nl * m * (d_.dbl ? 16 : 8);
  const int z1 = debug_buffer(-2, 0, 0, zb), z2 = debug_buffer(-2, 0, 1, zb);
  Op pre = op;
  pre.type = Op::BluePre;
  pre.dst = z1;
  prog.push_back(pre);
  Op f1 = make_stage(lz, lz, 1, dev::kC2C, false, 1.0);  // may itself be a four-step stage
  f1.src = z1;
  f1.dst = z2;
  push_stage(prog, f1);
  Op mul = op;
  mul.type = Op::BlueMul;
  mul.src = mul.dst = z2;
  prog.push_back(mul);
  Op f2 = make_stage(lz, lz, 1, dev::kC2C, true, 1.0);
  f2.src = z2;
  f2.dst = z1;
  push_stage(prog, f2);
  Op post = op;
  post.type = Op::BluePost;
  post.src = z1;
  prog.push_back(post);
}

Op Plan::make_stage(int src_l, int dst_l, std::size_t a, int kind, bool inverse, double scale) {
  const Layout& S = layouts_[src_l];
  const Layout& Dl = layouts_[dst_l];
  const std::size_t D = S.gext.size();
  Op op;
  op.type = Op::Stage;
  op.kind = kind;
  op.inverse = inverse;
  op.src_layout = src_l;
  op.dst_layout = dst_l;
  dev::StageArgs& A = op.sa;
  std::memset(&A, 0, sizeof(A));
  const std::size_t n = (kind == dev::kC2R) ? Dl.gext[a] : S.gext[a];
  A.nd = static_cast<int>(D);
  A.a = static_cast<int>(a);
  A.n = static_cast<int>(n);
  A.na_in = static_cast<int>(S.gext[a]);
  A.na_out = static_cast<int>(Dl.gext[a]);
  if (kind == dev::kCopy && !S.complex) {
    op.kind = kind = dev::kCopyReal;
  }
  const bool is_copy = kind == dev::kCopy || kind == dev::kCopyReal;
  if (is_copy && (A.na_in != A.na_out || S.complex != Dl.complex))
    fail(kErrInternal, "copy stage between different extents or element types");
  const std::size_t fs = layout_fast_axis(S), fd = layout_fast_axis(Dl);
  std::size_t b;
  if (fd != a) b = fd;
  else if (fs != a) b = fs;
  else {
    // lines contiguous on both sides: tile along the longest other axis so
    // that short axes (e.g. the 3 components of a batched 4D view) do not
    // leave most lines of a tile empty
    b = (a == 0) ? 1 : 0;
    for (std::size_t k = 0; k < D; ++k)
      if (k != a && Dl.gext[k] > Dl.gext[b]) b = k;
  }
  A.b = static_cast<int>(b);
  int others[2] = {-1, -1}, no = 0;
  for (std::size_t k = 0; k < D; ++k)
    if (k != a && k != b) others[no++] = static_cast<int>(k);
  A.o0 = others[0];
  A.o1 = others[1];
  A.Eb = static_cast<int>(Dl.gext[b]);
  A.Eo0 = A.o0 >= 0 ? static_cast<int>(Dl.gext[A.o0]) : 1;
  A.Eo1 = A.o1 >= 0 ? static_cast<int>(Dl.gext[A.o1]) : 1;
  A.load_afast = fs == a ? 1 : 0;
  A.store_afast = fd == a ? 1 : 0;
  A.scale = scale;

  if (!is_copy && !radix_supported(n)) {
    // chirp-z stage: a circular convolution of length m >= 2n - 1
    std::size_t m = 1;
    while (m < 2 * n - 1) m <<= 1;
    op.blue = true;
    op.blue_m = static_cast<int>(m);
    op.blue_lines = static_cast<long long>(A.Eb) * A.Eo0 * A.Eo1;
    const void *chirp = nullptr, *ffwd = nullptr, *finv = nullptr;
    bluestein_tables(n, m, &chirp, &ffwd, &finv);
    op.blue_chirp = chirp;
    op.blue_filter = inverse ? finv : ffwd;
    op.tiles = 1;
    return op;
  }
  if (!is_copy) {
    auto radices = radix_plan(n);
    A.npass = static_cast<int>(radices.size());
    unsigned long long code = 0;
    for (std::size_t p = 0; p < radices.size(); ++p) code |= static_cast<unsigned long long>(radices[p]) << (4 * p);
    A.radix_code = code;
  }

  const std::size_t ce = d_.dbl ? 16 : 8;
  const bool pairs = kind == dev::kR2C || kind == dev::kC2R;
  const std::size_t base = kind == dev::kC2R ? 2 * (n / 2 + 1) : n;
  const std::size_t pitch = base | 1;
  auto smem_for = [&](std::size_t B) {
    const std::size_t nl = pairs ? (B + 1) / 2 : B;
    return ((n + 1) & ~static_cast<std::size_t>(1)) * ce + 2 * nl * pitch * ce;
  };
  std::size_t B = std::min<std::size_t>(d_.dbl ? 8 : 16, Dl.gext[b]);
  if (pairs && B > 1 && (B & 1)) ++B;
  // shrink the tile to <= 100 KB of shared memory (pairs keep 2 lines)
  const std::size_t Bmin = pairs ? 2 : 1;
  while (B > Bmin && smem_for(B) > 100 * 1024) B = std::max(Bmin, B - (pairs ? 2 : 1));
  if (smem_for(B) > 227 * 1024) {
    if (is_copy) fail(kErrUnsupported, "line of " + std::to_string(n) + " elements too large for one copy stage");
    // four-step stage: n = n1 n2 with n1 the largest divisor <= sqrt(n)
    std::size_t n1 = 1;
    for (std::size_t d = 2; d * d <= n; ++d)
      if (n % d == 0) n1 = d;
    if (n1 == 1) fail(kErrUnsupported, "FFT length " + std::to_string(n) + " too large for one stage");
    op.four_n1 = static_cast<int>(n1);
    op.four_n2 = static_cast<int>(n / n1);
    op.four_tw = twiddle(n);
    op.blue_m = static_cast<int>(n);
    op.blue_lines = static_cast<long long>(A.Eb) * A.Eo0 * A.Eo1;
    op.tiles = 1;
    return op;
  }
  A.B = static_cast<int>(B);
  A.nl = static_cast<int>(pairs ? (B + 1) / 2 : B);
  A.pitch = static_cast<int>(pitch);
  A.tiles_b = static_cast<int>((Dl.gext[b] + B - 1) / B);
  const unsigned long long tiles = static_cast<unsigned long long>(A.tiles_b) * A.Eo0 * A.Eo1;
  if (tiles >= (1ull << 31)) fail(kErrUnsupported, "too many tiles");
  op.tiles = static_cast<unsigned>(tiles);
  op.smem = smem_for(B);
  op.nthreads = 256;
  if (!is_copy) A.tw = twiddle(n);

  // Register-resident kernels.  Each side of the stage either has separable
  // tables (per-axis offset tables; lines read along a must then be one
  // contiguous run) or general tables whose rank blocks do not split axis a
  // (every line is affine, base + p * stride; lines read along a have unit
  // stride because a is the layout's fast axis).
  auto side_ok = [&](int l, const Layout& L, std::size_t len, bool afast, int* affine, int* atab,
                     std::int64_t* abase, std::int64_t* astride) {
    const LayoutTables& T = tables_[l];
    *atab = 0;
    if (T.mode == 0) {
      // separable: the offsets along a must be affine (unit stride when the
      // lines are read along a)
      *affine = 0;
      const std::int64_t* off = T.data.data() + T.off[a];
      const std::int64_t st = len > 1 ? off[1] - off[0] : 1;
      bool aff = !afast || st == 1;
      for (std::size_t c = 1; aff && c < len; ++c)
        if (off[c] != off[0] + static_cast<std::int64_t>(c) * st) aff = false;
      // the kernels take 32-bit offsets along a line
      if (aff && static_cast<std::int64_t>(len - 1) * (st < 0 ? -st : st) >= (std::int64_t(1) << 31)) aff = false;
      if (aff) {
        *abase = off[0];
        *astride = st;
        return true;
      }
      // an exchange buffer split into bins along a (per-rank programs): the
      // general-layout kernel variant reads positions from the axis table
      if (!L.pad.empty() && L.topo[a] > 1 && (!afast || layout_fast_axis(L) == a)) {
        *atab = 1;
        *abase = 0;
        *astride = 1;
        return true;
      }
      return false;
    }
    *affine = 1;
    return L.topo[a] == 1 && (!afast || layout_fast_axis(L) == a);
  };
  // the register kernels take the coordinates along o0 / o1 from a grid of
  // (tiles, Eo0, Eo1) CTAs
  const bool grid_ok = A.Eo0 <= dev::fast_stage_max_grid_yz() && A.Eo1 <= dev::fast_stage_max_grid_yz();
  const std::size_t Bf = (grid_ok && dev::fast_stage_supported(static_cast<int>(n)))
                             ? static_cast<std::size_t>(dev::fast_stage_lines(d_.dbl, static_cast<int>(n)))
                             : 0;
  int saff = 0, daff = 0, satab = 0, datab = 0;
  std::int64_t sab = 0, sas = 0, dab = 0, das = 0;
  // C2C: lines of n points on both sides, the same row orientation
  if (kind == dev::kC2C && Bf && A.load_afast == A.store_afast && S.gext[a] == n && Dl.gext[a] == n &&
      side_ok(src_l, S, n, A.load_afast != 0, &saff, &satab, &sab, &sas) &&
      side_ok(dst_l, Dl, n, A.load_afast != 0, &daff, &datab, &dab, &das)) {
    op.fast = true;
    A.B = static_cast<int>(Bf);
    A.tiles_b = static_cast<int>((Dl.gext[b] + Bf - 1) / Bf);
  }
  // R2C (first) / C2R (last): lines of n reals and n/2+1 complex values, both
  // read along a; two real lines per register line
  const std::size_t nr = n, nc = n / 2 + 1;
  const std::size_t ns = kind == dev::kR2C ? nr : nc, ndst = kind == dev::kR2C ? nc : nr;
  if ((kind == dev::kR2C || kind == dev::kC2R) && Bf && A.load_afast && A.store_afast && S.gext[a] == ns &&
      Dl.gext[a] == ndst && side_ok(src_l, S, ns, true, &saff, &satab, &sab, &sas) &&
      side_ok(dst_l, Dl, ndst, true, &daff, &datab, &dab, &das)) {
    op.fast = true;
    A.B = static_cast<int>(Bf);
    A.tiles_b = static_cast<int>((Dl.gext[b] + 2 * Bf - 1) / (2 * Bf));
  }
  if (op.fast) {
    A.src_line_affine = saff;
    A.dst_line_affine = daff;
    A.src_atab = satab;
    A.dst_atab = datab;
    A.src_abase = sab;
    A.src_astride = sas;
    A.dst_abase = dab;
    A.dst_astride = das;
    // Two complex64 lines per thread: C2C of 2^k points on separable sides;
    // b-fast tiles move both lines of a pair with one 16-byte access, so
    // every pair must start on an even element on both sides.
    auto pair_aligned = [&](int l, std::int64_t abase, std::int64_t astride, bool atab) {
      const LayoutTables& T = tables_[l];
      if (T.mode != 0) return false;
      if (atab) {
        const std::int64_t* oa = T.data.data() + T.off[a];
        for (std::size_t c = 0; c < layouts_[l].gext[a]; ++c)
          if (oa[c] & 1) return false;
      } else if ((abase & 1) || (astride & 1)) {
        return false;
      }
      const std::int64_t* ob = T.data.data() + T.off[b];
      for (std::size_t c = 0; c + 1 < static_cast<std::size_t>(A.Eb); c += 2)
        if ((ob[c] & 1) || ob[c + 1] != ob[c] + 1) return false;
      if ((A.Eb & 1) && (ob[A.Eb - 1] & 1)) return false;
      for (int o : {A.o0, A.o1}) {
        if (o < 0) continue;
        const std::int64_t* oo = T.data.data() + T.off[o];
        for (std::size_t c = 0; c < layouts_[l].gext[o]; ++c)
          if (oo[c] & 1) return false;
      }
      return true;
    };
    // (axis-table sides: the two-line kernel takes the positions along a from
    // the table; b-fast pairs need every offset even)
    const bool atab = satab || datab;
    if (kind == dev::kC2C && !d_.dbl && dev::pair_stage_supported(static_cast<int>(n)) && !saff && !daff &&
        (A.load_afast || (pair_aligned(src_l, sab, sas, satab) && pair_aligned(dst_l, dab, das, datab)))) {
      int opts[3];
      dev::pair_stage_line_options(static_cast<int>(n), A.load_afast != 0, opts);
      op.single_B = A.B;
      A.pairs = 1;
      A.B = opts[0];
      A.tiles_b = static_cast<int>((Dl.gext[b] + opts[0] - 1) / opts[0]);
      // b-fast source tiles moved by TMA when a tensor map can describe the
      // source layout (the default; the tuner may pick another variant)
      const int tl = dev::pair_tma_lines(static_cast<int>(n));
      if (!A.load_afast && tl > 0 && !atab && tma_source(src_l, A, &op.tma) &&
          (!op.tma.b_split || op.tma.lb % tl == 0)) {
        op.pair_B = A.B;
        A.pairs = 3;
        A.B = tl;
        A.tiles_b = static_cast<int>((Dl.gext[b] + tl - 1) / tl);
      }
      // compensated last pass: the default tiles of the two kernels above
      // (not on axis-table sides: plain FP32 there)
      if (d_.comp && !atab) A.comp = 1;
    }
    const unsigned long long ft = static_cast<unsigned long long>(A.tiles_b) * A.Eo0 * A.Eo1;
    if (ft >= (1ull << 31)) fail(kErrUnsupported, "too many tiles");
    op.tiles = static_cast<unsigned>(ft);
  }
  return op;
}

// Tensor-map description of the source layout of a b-fast stage for the
// TMA-fed kernel: dimension 0 is the tile axis b inside a rank block (unit
// stride), then the FFT axis a, the other axes inside a block and, for every
// split axis, its rank coordinate (stride: rank stride x block size), sorted
// by stride; at most 5 dimensions of extent > 1.  The box is A.B lines along b
// (set at launch) by min(n, 256) along a, so a tile lands in shared memory as
// n rows of A.B elements.  Needs a separable layout (equal blocks) and even
// element strides (16-byte multiples); when b is split the launch also needs
// rank blocks a whole number of tiles wide along b (a box never crosses into
// the next block).
bool Plan::tma_source(int l, const dev::StageArgs& A, TmaSource* out) const {
  const Layout& L = layouts_[l];
  const std::size_t D = L.gext.size();
  if (!layout_even(L) || A.n > 1024) return false;
  const auto blocks = layout_blocks(L);
  const RankBlock& b0 = blocks.at(0);
  const std::size_t a = static_cast<std::size_t>(A.a), b = static_cast<std::size_t>(A.b);
  if (L.topo[a] != 1 || b0.stride[b] != 1 || b0.local[a] != static_cast<std::size_t>(A.n)) return false;
  Ext rs(D, 1);
  std::size_t acc = 1;
  if (L.rank_right) {
    for (long k = static_cast<long>(D) - 1; k >= 0; --k) {
      rs[k] = acc;
      acc *= L.topo[k];
    }
  } else {
    for (std::size_t k = 0; k < D; ++k) {
      rs[k] = acc;
      acc *= L.topo[k];
    }
  }
  struct Dim {
    int which, rank_part;
    std::uint64_t extent, stride, lk;
  };
  auto role = [&](std::size_t k) { return k == b ? 0 : k == a ? 1 : static_cast<int>(k) == A.o0 ? 2 : 3; };
  std::vector<Dim> dims;
  dims.push_back({0, 0, b0.local[b], 1, b0.local[b]});
  for (std::size_t k = 0; k < D; ++k) {
    if (k == b) continue;
    if (b0.local[k] > 1) dims.push_back({role(k), 0, b0.local[k], b0.stride[k], b0.local[k]});
  }
  for (std::size_t k = 0; k < D; ++k)
    if (L.topo[k] > 1) dims.push_back({role(k), 1, L.topo[k], rs[k] * b0.size, b0.local[k]});
  if (dims.size() > 5) return false;
  std::sort(dims.begin() + 1, dims.end(), [](const Dim& x, const Dim& y) { return x.stride < y.stride; });
  TmaSource t;
  std::uint64_t span = 16;
  for (std::size_t d = 0; d < dims.size(); ++d) {
    const std::uint64_t sb = dims[d].stride * 8;  // complex64
    if (d > 0 && (sb % 16 != 0 || sb >= (std::uint64_t(1) << 40))) return false;
    if (dims[d].extent >= (std::uint64_t(1) << 31)) return false;
    t.dim[d] = dims[d].extent;
    t.stride[d] = sb;
    t.coords.which[d] = dims[d].which;
    t.coords.rank_part[d] = dims[d].rank_part;
    t.coords.lk[d] = static_cast<int>(dims[d].lk);
    span = std::max(span, sb * dims[d].extent);
  }
  for (std::size_t d = dims.size(); d < 5; ++d) {
    t.dim[d] = 1;
    t.stride[d] = (span + 15) / 16 * 16;
    t.coords.which[d] = 4;
    t.coords.rank_part[d] = 0;
    t.coords.lk[d] = 1;
  }
  const int boxa = std::min(A.n, 256);
  for (std::size_t d = 0; d < 5; ++d) t.box[d] = 1;
  t.lb = b0.local[b];
  t.b_split = L.topo[b] > 1;
  for (std::size_t d = 1; d < dims.size(); ++d)
    if (dims[d].which == 1) t.box[d] = static_cast<std::uint32_t>(boxa);
  t.coords.boxa = boxa;
  t.coords.nchunks = A.n / boxa;
  t.ok = true;
  *out = t;
  return true;
}

// Launch of a register-resident stage (C2C, R2C or C2R).
static cudaError_t launch_fast_op(const dev::StageArgs& A, bool dbl, int kind, bool inverse, cudaStream_t st) {
  if (kind == dev::kR2C || kind == dev::kC2R) return dev::launch_fft_fast_real(A, dbl, kind == dev::kC2R, st);
  if (A.pairs) return dev::launch_fft_pair(A, inverse, A.load_afast != 0, st);
  return dev::launch_fft_fast(A, dbl, inverse, A.load_afast != 0, st);
}

// One stage launch with the run-time fallbacks of the two-line variants: the
// TMA kernel needs a source the tensor map can address (16-byte aligned
// pointer); the two-line b-fast kernels need 16-byte aligned buffers.
cudaError_t Plan::launch_stage(const Op& op, dev::StageArgs A, cudaStream_t stream) const {
  if (!op.fast) return dev::launch_fft_stage(A, d_.dbl, op.kind, op.inverse, op.nthreads, op.smem, op.tiles, stream);
  const bool misaligned = ((reinterpret_cast<std::uintptr_t>(A.in) | reinterpret_cast<std::uintptr_t>(A.out)) & 15) != 0;
  if (A.pairs == 3) {
    alignas(64) CUtensorMap map;
    TmaSource t = op.tma;
    t.box[0] = static_cast<std::uint32_t>(A.B);
    if (!misaligned && (!t.b_split || t.lb % static_cast<std::uint64_t>(A.B) == 0) && tma_encode(&map, A.in, t))
      return dev::launch_fft_pair_tma(A, &map, t.coords, op.inverse, stream);
    A.pairs = 1;
    A.B = op.pair_B;
    A.tiles_b = (A.Eb + A.B - 1) / A.B;
  }
  if (A.pairs && !A.load_afast && misaligned) {
    // a caller buffer off a 16-byte boundary: the one-line kernel (plain
    // FP32 arithmetic)
    A.pairs = 0;
    A.comp = 0;
    A.B = op.single_B;
    A.tiles_b = (A.Eb + A.B - 1) / A.B;
  }
  return launch_fast_op(A, d_.dbl, op.kind, op.inverse, stream);
}

int Plan::device_error(bool reset) const {
  if (!d_err_) return 0;
  int v = 0;
  cuda_check(cudaDeviceSynchronize(), "device error word");
  cuda_check(cudaMemcpy(&v, d_err_, sizeof(int), cudaMemcpyDeviceToHost), "device error word");
  if (reset) cuda_check(cudaMemset(d_err_, 0, sizeof(int)), "device error word");
  return v;
}

// ---------------------------------------------------------------------------
// Fused program
// ---------------------------------------------------------------------------
void Plan::build_fused(bool forward) {
  auto& prog = prog_[forward ? 0 : 1];
  prog.clear();
  auto order = fft_axis_order();
  const std::size_t S = order.size();
  Layout I;
  I.gext = d_.gout;
  I.topo.assign(d_.gout.size(), 1);
  I.map = identity_map(d_.gout.size());
  I.view_right = d_.view_right;
  I.complex = true;
  const int li = add_layout(I), lin = add_layout(lin_), lout = add_layout(lout_);
  if (!forward) std::reverse(order.begin(), order.end());
  for (std::size_t s = 0; s < S; ++s) {
    const bool first = s == 0, last = s == S - 1;
    int src_l, dst_l, kind;
    if (forward) {
      src_l = first ? lin : li;
      dst_l = last ? lout : li;
      kind = (first && d_.r2c) ? dev::kR2C : dev::kC2C;
    } else {
      src_l = first ? lout : li;
      dst_l = last ? lin : li;
      kind = (last && d_.r2c) ? dev::kC2R : dev::kC2C;
    }
    Op op = make_stage(src_l, dst_l, order[s], kind, !forward, last ? (forward ? scale_fwd_ : scale_bwd_) : 1.0);
    op.src = first ? kBufIn : (((s - 1) % 2 == 0) ? kBufScratch0 : kBufScratch1);
    op.dst = last ? kBufOut : ((s % 2 == 0) ? kBufScratch0 : kBufScratch1);
    push_stage(prog, op);
  }
}

// ---------------------------------------------------------------------------
// Adjoint programs.  For C2C the adjoint of s * DFT is s * (unnormalised
// inverse DFT), i.e. the opposite fused program with the other scale.  For
// R2C (real x, half spectrum along the R2C axis): adjoint(R2C) = C2R * diag(1/w)
// and adjoint(C2R) = diag(w) * R2C with w = 2 on the interior modes (doubled by
// the Hermitian extension) and 1 on DC / Nyquist; the weights commute with the
// C2C transforms along the other axes and are applied to a complex
// intermediate through the layout tables.
// ---------------------------------------------------------------------------
void Plan::build_adjoint(bool of_forward) {
  auto& prog = adj_[of_forward ? 0 : 1];
  prog.clear();
  auto order = fft_axis_order();
  const std::size_t S = order.size();
  const std::size_t ar = order.front();  // R2C axis
  Layout I;
  I.gext = d_.gout;
  I.topo.assign(d_.gout.size(), 1);
  I.map = identity_map(d_.gout.size());
  I.view_right = d_.view_right;
  I.complex = true;
  const int li = add_layout(I), lin = add_layout(lin_), lout = add_layout(lout_);
  const double scale = of_forward ? scale_fwd_ : scale_bwd_;
  auto weight_op = [&](int layout, int buf, double factor) {
    Op w;
    w.type = Op::Weight;
    w.src = w.dst = buf;
    w.src_layout = layout;
    w.w_axis = static_cast<int>(ar);
    w.w_n = static_cast<int>(d_.gin[ar]);
    w.scale = factor;
    return w;
  };
  if (of_forward) {
    // output layout -> input layout: inverse transforms, C2R last
    std::reverse(order.begin(), order.end());
    int cur_l = lout, cur_b = kBufIn;
    if (d_.r2c && S == 1) {
      Op c = make_stage(lout, li, layout_fast_axis(lout_), dev::kCopy, false, 1.0);
      c.src = kBufIn;
      c.dst = kBufScratch0;
      prog.push_back(c);
      prog.push_back(weight_op(li, kBufScratch0, 0.5));
      cur_l = li;
      cur_b = kBufScratch0;
    }
    for (std::size_t s = 0; s < S; ++s) {
      const bool last = s == S - 1;
      const int kind = (last && d_.r2c) ? dev::kC2R : dev::kC2C;
      const int dst_l = last ? lin : li;
      Op op = make_stage(cur_l, dst_l, order[s], kind, true, last ? scale : 1.0);
      op.src = cur_b;
      op.dst = last ? kBufOut : (cur_b == kBufScratch0 ? kBufScratch1 : kBufScratch0);
      push_stage(prog, op);
      cur_l = dst_l;
      cur_b = op.dst;
      if (s == 0 && d_.r2c && S >= 2) prog.push_back(weight_op(li, cur_b, 0.5));
    }
  } else {
    // input layout -> output layout: forward transforms, R2C first
    int cur_l = lin, cur_b = kBufIn;
    for (std::size_t s = 0; s < S; ++s) {
      const bool first = s == 0, last = s == S - 1;
      const int kind = (first && d_.r2c) ? dev::kR2C : dev::kC2C;
      const int dst_l = last ? lout : li;
      Op op = make_stage(cur_l, dst_l, order[s], kind, false, last ? scale : 1.0);
      op.src = cur_b;
      op.dst = last ? kBufOut : (cur_b == kBufScratch0 ? kBufScratch1 : kBufScratch0);
      push_stage(prog, op);
      cur_l = dst_l;
      cur_b = op.dst;
      if (first && d_.r2c) prog.push_back(weight_op(cur_l, cur_b, 2.0));
    }
  }
}

// ---------------------------------------------------------------------------
// Literal program (reference block sequence)
// ---------------------------------------------------------------------------
std::int64_t Plan::add_geo(const Layout& L, const BlockInfo& b, std::size_t pc) {
  // Exchange groups: the whole communicator for slabs; for pencils the row /
  // column communicators of MPI_Cart_create over the non-one entries of the
  // input topology (reorder = 0, row-major) split by MPI_Cart_sub
  // (KokkosFFT_Distributed_PencilPlan.hpp:32-71), picked by comm_axis.
  const std::int64_t base = static_cast<std::int64_t>(host_tables_.size());
  append_exchange_geo(host_tables_, L, d_.in_topo, type_ == TopologyType::Pencil ? static_cast<int>(b.comm_axis) : -1,
                      pc);
  return base;
}

int Plan::debug_buffer(int dir, std::size_t block, int which, std::size_t bytes) {
  const auto key = std::make_pair(dir, static_cast<int>(block * 4 + which));
  auto it = debug_bufs_.find(key);
  if (it != debug_bufs_.end()) {
    buf_bytes_[it->second] = std::max(buf_bytes_[it->second], bytes);
    return it->second;
  }
  const int id = static_cast<int>(kBufFirstDebug + debug_bufs_.size());
  debug_bufs_[key] = id;
  buf_bytes_.resize(std::max<std::size_t>(buf_bytes_.size(), id + 1), 0);
  buf_bytes_[id] = bytes;
  return id;
}

void Plan::build_literal(bool forward) {
  auto& prog = prog_[forward ? 0 : 1];
  prog.clear();
  const auto& blocks = per_rank_.at(0).blocks;
  const std::size_t D = d_.gin.size();
  const std::size_t nbl = blocks.size();
  std::vector<std::size_t> topo_index(nbl);  // chain index of each block
  {
    std::size_t t = 0;
    for (std::size_t i = 0; i < nbl; ++i) {
      topo_index[i] = t;
      if (blocks[i].block_type == BlockType::Transpose) ++t;
    }
  }
  auto flag = [&](std::size_t k) { return chain_layouts_.at(k) != 0; };
  auto other_scratch = [](int b) { return b == kBufScratch0 ? kBufScratch1 : kBufScratch0; };
  auto copy_to = [&](int& cur_l, int& cur_b, const Layout& L) {
    const int nl = add_layout(L);
    if (nl == cur_l) return;
    // a local transpose: lines along the source's unit-stride axis
    Op op = make_stage(cur_l, nl, layout_fast_axis(layouts_[cur_l]), dev::kCopy, false, 1.0);
    op.src = cur_b;
    op.dst = other_scratch(cur_b);
    prog.push_back(op);
    cur_l = nl;
    cur_b = op.dst;
  };
  auto fft_stage = [&](int& cur_l, int& cur_b, const Layout& dstL, std::size_t a, int kind, bool inv) {
    const int nl = add_layout(dstL);
    Op op = make_stage(cur_l, nl, a, kind, inv, 1.0);
    op.src = cur_b;
    // in place on scratch; out of place when reading the caller's buffer or changing type
    op.dst = (cur_b == kBufIn || kind == dev::kR2C || kind == dev::kC2R) ? other_scratch(cur_b) : cur_b;
    push_stage(prog, op);
    cur_l = nl;
    cur_b = op.dst;
  };
  auto xpose = [&](int& cur_l, int& cur_b, const BlockInfo& b, const Layout& Ls, const Layout& Ld,
                   std::size_t pack_axis, std::size_t unpack_axis, int dir) {
    const int ls = add_layout(Ls), ld = add_layout(Ld);
    if (ls != cur_l) copy_to(cur_l, cur_b, Ls);
    const std::size_t pc = d_.view_right ? b.buffer_extents.front() : b.buffer_extents.back();
    const std::size_t bufsize = total_size(b.buffer_extents);
    const int eb = Ls.complex ? (d_.dbl ? 16 : 8) : (d_.dbl ? 8 : 4);
    std::size_t block_index = 0;
    for (std::size_t i = 0; i < nbl; ++i)
      if (&blocks[i] == &b) block_index = i;
    const bool capture = d_.exec_mode == 2;
    const std::size_t xbytes = nprocs() * bufsize * eb;
    int ids[2];
    if (capture) {
      ids[0] = debug_buffer(dir, block_index, 0, xbytes);
      ids[1] = debug_buffer(dir, block_index, 1, xbytes);
      Op c;
      c.type = Op::Copy;
      c.src = cur_b;
      c.dst = debug_buffer(dir, block_index, 2, layout_elements(Ls) * eb);
      c.bytes = layout_elements(Ls) * eb;
      prog.push_back(c);
    } else {
      // send / recv buffers shared by every exchange of the plan
      ids[0] = debug_buffer(-1, 0, 0, xbytes);
      ids[1] = debug_buffer(-1, 0, 1, xbytes);
    }
    dev::XposeArgs X;
    std::memset(&X, 0, sizeof(X));
    X.rs = static_cast<int>(9 + pc);
    X.nd = static_cast<int>(D);
    X.nprocs = static_cast<int>(nprocs());
    X.pc = static_cast<int>(pc);
    for (std::size_t k = 0; k < b.buffer_extents.size(); ++k) X.bext[k] = static_cast<std::int64_t>(b.buffer_extents[k]);
    X.buf_right = d_.view_right ? 1 : 0;
    X.bufsize = static_cast<std::int64_t>(bufsize);
    Op pack;
    pack.type = Op::Pack;
    pack.xa = X;
    pack.xa.axis = static_cast<int>(pack_axis);
    pack.xa.merged = static_cast<std::int64_t>(Ls.gext[pack_axis]);
    pack.src_layout = ls;
    pack.xa.geo = reinterpret_cast<const std::int64_t*>(add_geo(Ls, b, pc));  // offset, resolved later
    pack.elem_bytes = eb;
    pack.src = cur_b;
    pack.dst = ids[0];
    pack.block = static_cast<int>(block_index);
    Op a2a = pack;
    a2a.type = Op::All2All;
    a2a.src = ids[0];
    a2a.dst = ids[1];
    Op unpack;
    unpack.type = Op::Unpack;
    unpack.xa = X;
    unpack.xa.axis = static_cast<int>(unpack_axis);
    unpack.xa.merged = static_cast<std::int64_t>(Ld.gext[unpack_axis]);
    unpack.dst_layout = ld;
    unpack.xa.geo = reinterpret_cast<const std::int64_t*>(add_geo(Ld, b, pc));
    unpack.elem_bytes = eb;
    unpack.src = ids[1];
    unpack.dst = other_scratch(cur_b);
    unpack.block = static_cast<int>(block_index);
    prog.push_back(pack);
    prog.push_back(a2a);
    prog.push_back(unpack);
    cur_l = ld;
    cur_b = unpack.dst;
    if (capture) {
      Op c;
      c.type = Op::Copy;
      c.src = cur_b;
      c.dst = debug_buffer(dir, block_index, 3, layout_elements(Ld) * eb);
      c.bytes = layout_elements(Ld) * eb;
      prog.push_back(c);
    }
  };

  const int dir = forward ? 0 : 1;
  if (forward) {
    int cur_l = add_layout(lin_), cur_b = kBufIn;
    bool complex = lin_.complex;
    for (std::size_t i = 0; i < nbl; ++i) {
      const BlockInfo& b = blocks[i];
      const std::size_t k = topo_index[i];
      if (b.block_type == BlockType::FFT) {
        Layout Lb = block_layout(chain_[k], flag(k), b.in_map, complex);
        copy_to(cur_l, cur_b, Lb);
        for (std::size_t j = 0; j < b.fft_dim; ++j) {
          const std::size_t a = d_.view_right ? b.in_map[D - 1 - j] : b.in_map[j];
          if (!complex) {
            complex = true;
            fft_stage(cur_l, cur_b, block_layout(chain_[k], flag(k), b.in_map, true), a, dev::kR2C, false);
          } else {
            fft_stage(cur_l, cur_b, layouts_[cur_l], a, dev::kC2C, false);
          }
        }
      } else {
        Layout Ls = block_layout(chain_[k], flag(k), b.in_map, complex);
        Layout Ld = block_layout(chain_[k + 1], flag(k + 1), b.out_map, complex);
        xpose(cur_l, cur_b, b, Ls, Ld, b.in_axis, b.out_axis, dir);
      }
    }
    finalize_program(prog, cur_l, cur_b, lout_, scale_fwd_, true);
  } else {
    int cur_l = add_layout(lout_), cur_b = kBufIn;
    bool complex = true;
    for (std::size_t ii = nbl; ii-- > 0;) {
      const BlockInfo& b = blocks[ii];
      const std::size_t k = topo_index[ii];
      if (b.block_type == BlockType::FFT) {
        Layout Lb = block_layout(chain_[k], flag(k), b.in_map, true);
        copy_to(cur_l, cur_b, Lb);
        for (std::size_t jj = b.fft_dim; jj-- > 0;) {
          const std::size_t a = d_.view_right ? b.in_map[D - 1 - jj] : b.in_map[jj];
          const bool c2r = d_.r2c && b.block_idx == 0 && jj == 0;
          if (c2r) {
            complex = false;
            fft_stage(cur_l, cur_b, block_layout(chain_[k], flag(k), b.in_map, false), a, dev::kC2R, true);
          } else {
            fft_stage(cur_l, cur_b, layouts_[cur_l], a, dev::kC2C, true);
          }
        }
      } else {
        Layout Ls = block_layout(chain_[k + 1], flag(k + 1), b.out_map, complex);
        Layout Ld = block_layout(chain_[k], flag(k), b.in_map, complex);
        xpose(cur_l, cur_b, b, Ls, Ld, b.out_axis, b.in_axis, dir);
      }
    }
    finalize_program(prog, cur_l, cur_b, lin_, scale_bwd_, lin_.complex);
  }
}

// Route the result of the program into the caller's output buffer (the last
// op writes there directly when it already produces the output layout,
// otherwise a local-transpose copy is appended), then normalise.
void Plan::finalize_program(std::vector<Op>& prog, int cur_l, int cur_b, const Layout& final_layout, double scale,
                            bool final_complex) {
  const int lf = add_layout(final_layout);
  if (cur_l == lf && !prog.empty() && prog.back().dst == cur_b && cur_b != kBufIn) {
    prog.back().dst = kBufOut;
  } else {
    Op op = make_stage(cur_l, lf, layout_fast_axis(layouts_[cur_l]), dev::kCopy, false, 1.0);
    op.src = cur_b;
    op.dst = kBufOut;
    prog.push_back(op);
  }
  if (scale != 1.0) {
    Op s;
    s.type = Op::Scale;
    s.src = s.dst = kBufOut;
    s.n_real = static_cast<std::int64_t>(layout_elements(final_layout) * (final_complex ? 2 : 1));
    s.scale = scale;
    prog.push_back(s);
  }
}

// ---------------------------------------------------------------------------
// Device resources
// ---------------------------------------------------------------------------
void Plan::allocate_device() {
  // Scratch: the largest global array the programs hold (per-rank programs:
  // the largest layout they use, so that the tuner's trial launches of the
  // stages that read or write the exchange buffers fit).
  std::size_t max_elems = std::max(layout_elements(lin_), layout_elements(lout_));
  if (is_rank_plan()) {
    max_elems = 0;
    for (const Layout& L : layouts_) max_elems = std::max(max_elems, layout_elements(L));
  }
  const std::size_t scratch_bytes = max_elems * (d_.dbl ? 16 : 8);
  buf_bytes_.resize(std::max<std::size_t>(buf_bytes_.size(), kBufFirstDebug), 0);
  buf_bytes_[kBufScratch0] = scratch_bytes;
  buf_bytes_[kBufScratch1] = scratch_bytes;
  bufs_.assign(buf_bytes_.size(), nullptr);
  // only allocate the scratch buffers the programs use
  std::vector<bool> used(buf_bytes_.size(), false);
  for (auto* progs : {&prog_[0], &prog_[1], &adj_[0], &adj_[1]})
    for (auto& op : *progs) {
      if (op.src >= kBufScratch0) used[op.src] = true;
      if (op.dst >= kBufScratch0) used[op.dst] = true;
    }
  for (std::size_t i = kBufScratch0; i < buf_bytes_.size(); ++i) {
    if (!used[i] || buf_bytes_[i] == 0) continue;
    if (cudaMalloc(&bufs_[i], buf_bytes_[i]) != cudaSuccess) {
      cudaGetLastError();
      fail(kErrAlloc, "cudaMalloc of " + std::to_string(buf_bytes_[i]) + " bytes of plan scratch failed");
    }
    workspace_bytes_ += buf_bytes_[i];
  }
  const std::size_t tb = std::max<std::size_t>(host_tables_.size(), 1) * sizeof(std::int64_t);
  if (cudaMalloc(&d_tables_, tb) != cudaSuccess) {
    cudaGetLastError();
    fail(kErrAlloc, "cudaMalloc of layout tables failed");
  }
  workspace_bytes_ += tb;
  if (cudaMalloc(reinterpret_cast<void**>(&d_err_), sizeof(int)) != cudaSuccess) {
    cudaGetLastError();
    fail(kErrAlloc, "cudaMalloc of the device error word failed");
  }
  cuda_check(cudaMemset(d_err_, 0, sizeof(int)), "device error word");
  if (!host_tables_.empty())
    cuda_check(cudaMemcpy(d_tables_, host_tables_.data(), host_tables_.size() * sizeof(std::int64_t),
                          cudaMemcpyHostToDevice),
               "table upload");
  auto dev_layout = [&](int l) {
    dev::DevLayout L;
    std::memset(&L, 0, sizeof(L));
    const LayoutTables& T = tables_.at(l);
    L.t = d_tables_ + layout_base_.at(l);
    L.mode = T.mode;
    for (int k = 0; k < 4; ++k) {
      L.off[k] = T.off[k];
      L.rk[k] = T.rk[k];
      L.loc[k] = T.loc[k];
    }
    L.rbase = T.rbase;
    L.rstride = T.rstride;
    return L;
  };
  for (auto* progs : {&prog_[0], &prog_[1], &adj_[0], &adj_[1]}) {
    for (auto& op : *progs) {
      if (op.type == Op::Weight) op.sa.dst = dev_layout(op.src_layout);
      if (op.type == Op::Stage || op.type == Op::BluePre || op.type == Op::BluePost) {
        op.sa.src = dev_layout(op.src_layout);
        op.sa.dst = dev_layout(op.dst_layout);
        op.sa.err = d_err_;
      } else if (op.type == Op::Pack || op.type == Op::All2All || op.type == Op::Unpack) {
        op.xa.geo = d_tables_ + reinterpret_cast<std::intptr_t>(op.xa.geo);
        if (op.type == Op::Pack) op.xa.lay = dev_layout(op.src_layout);
        if (op.type == Op::Unpack) op.xa.lay = dev_layout(op.dst_layout);
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Autotuner: kernel variant (one or two lines per thread, streaming, TMA-fed)
// and lines per CTA of every register-resident stage, timed on the plan's
// scratch buffers at plan creation and cached per stage signature (line
// length, precision, direction, row orientation, tile grid, the topologies of
// both sides and the line strides) for the process; DFFT_TUNE_CACHE=<file>
// also persists the choices across processes and DFFT_AUTOTUNE=0 keeps the
// defaults.
// ---------------------------------------------------------------------------
namespace {
std::mutex g_tune_mutex;
std::map<std::string, int> g_tune_cache;
bool g_tune_loaded = false;

void load_tune_cache_locked() {
  if (g_tune_loaded) return;
  g_tune_loaded = true;
  const char* path = std::getenv("DFFT_TUNE_CACHE");
  if (!path) return;
  std::ifstream f(path);
  std::string key;
  int val;
  while (f >> key >> val) g_tune_cache[key] = val;
}

void store_tune_locked(const std::string& key, int val) {
  g_tune_cache[key] = val;
  const char* path = std::getenv("DFFT_TUNE_CACHE");
  if (!path) return;
  std::ofstream f(path, std::ios::app);
  f << key << " " << val << "\n";
}
}  // namespace

void Plan::autotune() {
  const char* env = std::getenv("DFFT_AUTOTUNE");
  if (env && std::string(env) == "0") return;
  if (bufs_.size() <= kBufScratch1 || !bufs_[kBufScratch0] || !bufs_[kBufScratch1]) return;
  cudaStream_t st = d_.stream;
  bool cleared = false;
  std::lock_guard<std::mutex> lock(g_tune_mutex);
  load_tune_cache_locked();
  for (auto* progs : {&prog_[0], &prog_[1], &adj_[0], &adj_[1]}) {
    for (auto& op : *progs) {
      if (op.type != Op::Stage || !op.fast) continue;
      dev::StageArgs& A = op.sa;

      // Trial buffers: the op's own plan-owned buffers, else the scratch
      // pair; each must hold the whole layout the stage reads / writes
      // (chirp-z stages run their FFTs on arrays larger than the scratch).
      auto elem_bytes = [&](int l) { return layouts_[l].complex ? (d_.dbl ? 16u : 8u) : (d_.dbl ? 8u : 4u); };
      const std::size_t need_in = layout_elements(layouts_[op.src_layout]) * elem_bytes(op.src_layout);
      const std::size_t need_out = layout_elements(layouts_[op.dst_layout]) * elem_bytes(op.dst_layout);
      const int tin = op.src >= kBufScratch0 ? op.src : kBufScratch0;
      int tout = op.dst >= kBufScratch0 ? op.dst : kBufScratch1;
      if (tout == tin && op.src != op.dst) tout = tin == kBufScratch0 ? kBufScratch1 : kBufScratch0;
      if (!bufs_.at(tin) || !bufs_.at(tout) || buf_bytes_.at(tin) < need_in || buf_bytes_.at(tout) < need_out)
        continue;  // no trial buffers large enough: keep the default tile
      void* t_in = bufs_[tin];
      void* t_out = bufs_[tout];
      std::ostringstream k;
      const bool real = op.kind == dev::kR2C || op.kind == dev::kC2R;  // two real lines per register line
      const bool pair_ok = op.single_B != 0;                            // eligible for two lines per thread
      const bool tma_ok = op.tma.ok;                                    // eligible for the TMA-fed kernel
      k << "fast:n" << A.n << (d_.dbl ? "f64" : "f32") << (op.inverse ? "i" : "f") << (A.load_afast ? "a" : "b")
        << (op.kind == dev::kR2C ? "r2c" : op.kind == dev::kC2R ? "c2r" : "") << (pair_ok ? "P" : "")
        << (tma_ok ? "T" : "") << (A.comp ? "C" : "")
        << (A.src_line_affine || A.dst_line_affine || A.src_atab || A.dst_atab ? "G" : "") << ":" << A.Eb << "x"
        << A.Eo0 << "x" << A.Eo1;
      // the topologies and line strides of both sides: stages of one shape
      // that read or write differently blocked layouts are tuned apart
      for (int side : {op.src_layout, op.dst_layout}) {
        const Layout& Ls = layouts_[side];
        k << ":" << (Ls.rank_right ? "R" : "L");
        for (std::size_t t : Ls.topo) k << t << ".";
      }
      k << ":" << A.src_astride << "." << A.dst_astride;
      const std::string key = k.str();
      // a configuration: lines per tile of the one-line kernel; kPairCode +
      // lines per tile of the two-line kernel; kStreamCode + tiles per CTA of
      // its streaming variant; kTmaCode + lines per tile of the TMA-fed kernel
      constexpr int kPairCode = 100000, kStreamCode = 200000, kTmaCode = 300000;
      auto apply = [&](int code) {
        if (code >= kTmaCode) {
          A.pairs = 3;
          A.B = code - kTmaCode;
        } else if (code >= kStreamCode) {
          A.pairs = 2;
          A.tpc = code - kStreamCode;
          A.B = dev::pair_stage_stream_lines(A.n, A.load_afast != 0);
        } else {
          A.pairs = code >= kPairCode ? 1 : 0;
          A.B = code % kPairCode;
        }
        A.tiles_b = real ? (A.Eb + 2 * A.B - 1) / (2 * A.B) : (A.Eb + A.B - 1) / A.B;
        op.tiles = static_cast<unsigned>(static_cast<unsigned long long>(A.tiles_b) * A.Eo0 * A.Eo1);
      };
      auto it = g_tune_cache.find(key);
      if (it != g_tune_cache.end() && (it->second < kPairCode || pair_ok) && (it->second < kTmaCode || tma_ok)) {
        apply(it->second);
        continue;
      }
      if (!cleared) {
        // every plan-owned buffer starts cleared (trial launches read them)
        for (std::size_t i = kBufScratch0; i < bufs_.size(); ++i)
          if (bufs_[i]) cuda_check(cudaMemsetAsync(bufs_[i], 0, buf_bytes_[i], st), "tuner clear");
        cleared = true;
      }
      std::vector<int> cand;
      int opts[4];
      if (A.comp) {
        // compensated stages: the default tiles of the TMA and two-line kernels
        if (tma_ok) cand.push_back(kTmaCode + dev::pair_tma_lines(A.n));
        dev::pair_stage_line_options(A.n, A.load_afast != 0, opts);
        cand.push_back(kPairCode + opts[0]);
      } else if (tma_ok) {
        const int nt = dev::pair_tma_line_options(A.n, opts);
        for (int i = 0; i < nt; ++i)
          if (!op.tma.b_split || op.tma.lb % static_cast<std::uint64_t>(opts[i]) == 0) cand.push_back(kTmaCode + opts[i]);
      }
      const bool atab = A.src_atab || A.dst_atab;
      if (pair_ok && !A.comp && atab) {
        // axis-table sides: the two-line kernel's default tile only
        dev::pair_stage_line_options(A.n, A.load_afast != 0, opts);
        cand.push_back(kPairCode + opts[0]);
      } else if (pair_ok && !A.comp) {
        const int np = dev::pair_stage_line_options(A.n, A.load_afast != 0, opts);
        for (int i = 0; i < np; ++i) cand.push_back(kPairCode + opts[i]);
        const int sb = dev::pair_stage_stream_lines(A.n, A.load_afast != 0);
        const int tiles = sb > 0 ? (A.Eb + sb - 1) / sb : 0;
        for (int tpc : {4, 8, 16})
          if (tiles >= 2 * tpc) cand.push_back(kStreamCode + tpc);
      }
      const int nopt = A.comp ? 0 : dev::fast_stage_line_options(d_.dbl, A.n, opts);
      for (int i = 0; i < nopt; ++i) cand.push_back(opts[i]);
      int best = A.pairs == 3 ? kTmaCode + A.B : A.pairs == 2 ? kStreamCode + A.tpc : (A.pairs ? kPairCode : 0) + A.B;
      float best_ms = std::numeric_limits<float>::max();
      cudaEvent_t e0, e1;
      cuda_check(cudaEventCreate(&e0), "tuner event");
      cuda_check(cudaEventCreate(&e1), "tuner event");
      for (int code : cand) {
        apply(code);
        dev::StageArgs T = A;
        T.in = t_in;
        T.out = t_out;
        if (launch_stage(op, T, st) != cudaSuccess) {
          cudaGetLastError();
          continue;
        }
        cudaEventRecord(e0, st);
        for (int r = 0; r < 3; ++r) launch_stage(op, T, st);
        cudaEventRecord(e1, st);
        cuda_check(cudaEventSynchronize(e1), "tuner sync");
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best_ms) {
          best_ms = ms;
          best = code;
        }
      }
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      apply(best);
      store_tune_locked(key, best);
    }
  }
}

// ---------------------------------------------------------------------------
// Execution
// ---------------------------------------------------------------------------
void Plan::run_program(const std::vector<Op>& prog, const void* in, void* out, cudaStream_t stream,
                       std::size_t begin, std::size_t end, void* send, void* recv) const {
  if (!on_device_) fail(kErrInvalidArgument, "plan was created by dfft_plan_analyze and cannot execute");
  auto buf = [&](int id) -> void* {
    if (id == kBufIn) return const_cast<void*>(in);
    if (id == kBufOut) return out;
    if (id == kBufSend) return send;
    if (id == kBufRecv) return recv;
    return bufs_.at(id);
  };
  end = std::min(end, prog.size());
  for (std::size_t oi = begin; oi < end; ++oi) {
    const Op& op0 = prog[oi];
    cudaError_t e = cudaSuccess;
    switch (op0.type) {
      case Op::Stage: {
        if (op0.tiles == 0) break;
        dev::StageArgs A = op0.sa;
        A.in = buf(op0.src);
        A.out = buf(op0.dst);
        e = launch_stage(op0, A, stream);
        break;
      }
      case Op::Pack:
      case Op::All2All:
      case Op::Unpack: {
        dev::XposeArgs X = op0.xa;
        X.src = buf(op0.src);
        X.dst = buf(op0.dst);
        if (X.bufsize * X.nprocs == 0) break;
        e = dev::launch_xpose(op0.type == Op::Pack ? 0 : (op0.type == Op::All2All ? 1 : 2), X, op0.elem_bytes, stream);
        break;
      }
      case Op::BluePre:
      case Op::BlueMul:
      case Op::BluePost:
      case Op::FourTwiddle: {
        dev::BlueArgs B;
        std::memset(&B, 0, sizeof(B));
        B.S = op0.sa;
        B.kind = op0.kind;
        B.inverse = op0.inverse ? 1 : 0;
        B.m = op0.blue_m;
        B.nlines = op0.blue_lines;
        B.chirp = op0.blue_chirp;
        B.filter = op0.blue_filter;
        B.four_n1 = op0.four_n1;
        B.four_n2 = op0.four_n2;
        B.tw = op0.four_tw;
        int which = 0;
        if (op0.type == Op::BluePre) {
          B.S.in = buf(op0.src);
          B.zout = buf(op0.dst);
        } else if (op0.type == Op::BlueMul || op0.type == Op::FourTwiddle) {
          which = op0.type == Op::BlueMul ? 1 : 3;
          B.zout = buf(op0.dst);
        } else {
          which = 2;
          B.zin = buf(op0.src);
          B.S.out = buf(op0.dst);
        }
        e = dev::launch_bluestein(which, B, d_.dbl, stream);
        break;
      }
      case Op::Scale: e = dev::launch_scale(buf(op0.dst), op0.n_real, d_.dbl, op0.scale, stream); break;
      case Op::Copy: e = cudaMemcpyAsync(buf(op0.dst), buf(op0.src), op0.bytes, cudaMemcpyDeviceToDevice, stream); break;
      case Op::Weight: {
        const Layout& L = layouts_[op0.src_layout];
        std::int64_t ext[4] = {1, 1, 1, 1};
        for (std::size_t k = 0; k < L.gext.size(); ++k) ext[k] = static_cast<std::int64_t>(L.gext[k]);
        e = dev::launch_weight(op0.sa.dst, buf(op0.dst), d_.dbl, static_cast<int>(L.gext.size()), ext, op0.w_axis,
                               op0.w_n, op0.scale, stream);
        break;
      }
    }
    if (e != cudaSuccess) fail(kErrCuda, std::string("kernel launch failed: ") + cudaGetErrorString(e));
  }
}

// The kernels move whole real / complex elements: a buffer off its element
// alignment would fault on the device, so it is refused before any launch.
void Plan::check_alignment(const void* p, bool complex, const char* which) const {
  const std::uintptr_t real = d_.dbl ? 8 : 4;
  const std::uintptr_t align = complex ? 2 * real : real;
  if (reinterpret_cast<std::uintptr_t>(p) % align != 0)
    fail(kErrInvalidArgument, std::string(which) + " buffer is not aligned to its element type (" +
                                  std::to_string(align) + " bytes)");
}

void Plan::check_buffers(const void* in, const void* out, bool forward) const {
  if (!on_device_) fail(kErrInvalidArgument, "plan was created by dfft_plan_analyze and cannot execute");
  if (!in || !out) fail(kErrInvalidArgument, "null buffer");
  if (in == out) fail(kErrInvalidArgument, "in-place execution is not supported: in and out must differ");
  // forward: input layout -> complex output layout; backward: the reverse
  check_alignment(in, forward ? lin_.complex : true, "input");
  check_alignment(out, forward ? true : lin_.complex, "output");
}

void Plan::execute(const void* in, void* out, bool forward, cudaStream_t stream) const {
  if (is_rank_plan())
    fail(kErrInvalidArgument, "a per-rank plan executes segment by segment around the caller's exchanges");
  check_buffers(in, out, forward);
  run_program(prog_[forward ? 0 : 1], in, out, stream);
}

bool Plan::can_premultiply() const {
  if (is_rank_plan() || !on_device_ || prog_[1].empty()) return false;
  const Op& op = prog_[1].front();
  return op.type == Op::Stage && op.fast && op.kind == dev::kC2C && op.src == kBufIn &&
         dev::fast_stage_supported(op.sa.n);
}

void Plan::execute_backward_premul(const void* in, void* out, const dev::StageArgs& pre, cudaStream_t stream) const {
  if (!can_premultiply()) fail(kErrInternal, "the first backward stage cannot pre-multiply its loads");
  check_buffers(in, out, false);
  const auto& prog = prog_[1];
  Op op = prog.front();
  dev::StageArgs A = op.sa;
  // the one-line kernel, general-layout variant: the tuned tile of a
  // one-line stage, else the default one
  if (A.pairs) A.B = dev::fast_stage_lines(d_.dbl, A.n);
  A.pairs = 0;
  A.comp = 0;
  A.tiles_b = (A.Eb + A.B - 1) / A.B;
  op.tiles = static_cast<unsigned>(static_cast<unsigned long long>(A.tiles_b) * A.Eo0 * A.Eo1);
  A.pre_mode = pre.pre_mode;
  A.pre_n[0] = pre.pre_n[0];
  A.pre_n[1] = pre.pre_n[1];
  for (int k = 0; k < 3; ++k) A.pre_cut[k] = pre.pre_cut[k];
  A.pre_kscale = pre.pre_kscale;
  A.in = const_cast<void*>(in);
  A.out = op.dst == kBufOut ? out : bufs_.at(op.dst);
  const cudaError_t e = launch_stage(op, A, stream);
  if (e != cudaSuccess) fail(kErrCuda, std::string("kernel launch failed: ") + cudaGetErrorString(e));
  run_program(prog, in, out, stream, 1);
}

void Plan::execute_adjoint(const void* in, void* out, bool of_forward, cudaStream_t stream) const {
  if (is_rank_plan()) fail(kErrInvalidArgument, "per-rank plans have no adjoint programs");
  if (!in || !out) fail(kErrInvalidArgument, "null buffer");
  if (in == out) fail(kErrInvalidArgument, "in-place execution is not supported: in and out must differ");
  // adjoint of forward: complex output layout -> input layout; of backward: the reverse
  check_alignment(in, of_forward ? true : lin_.complex, "input");
  check_alignment(out, of_forward ? lin_.complex : true, "output");
  run_program(adj_[of_forward ? 0 : 1], in, out, stream);
}

dev::DevLayout Plan::device_layout(bool output) const {
  if (!on_device_) fail(kErrInvalidArgument, "plan has no device tables");
  Layout L = output ? lout_ : lin_;
  for (std::size_t i = 0; i < layouts_.size(); ++i) {
    if (layouts_[i] == L) {
      dev::DevLayout D;
      std::memset(&D, 0, sizeof(D));
      const LayoutTables& T = tables_[i];
      D.t = d_tables_ + layout_base_[i];
      D.mode = T.mode;
      for (int k = 0; k < 4; ++k) {
        D.off[k] = T.off[k];
        D.rk[k] = T.rk[k];
        D.loc[k] = T.loc[k];
      }
      D.rbase = T.rbase;
      D.rstride = T.rstride;
      return D;
    }
  }
  fail(kErrInternal, "layout not registered");
}

void Plan::export_buffers(bool forward, std::size_t block, int which, void* host, std::size_t capacity) const {
  if (!on_device_) fail(kErrInvalidArgument, "plan has no device buffers");
  if (which < 0 || which > 3) fail(kErrInvalidArgument, "which must be 0 (send), 1 (recv), 2 (pack input) or 3 (unpack output)");
  auto it = debug_bufs_.find({forward ? 0 : 1, static_cast<int>(block * 4 + which)});
  if (it == debug_bufs_.end())
    fail(kErrInvalidArgument, "no recorded buffers for this block (capturing literal execution of a transpose block only)");
  const std::size_t bytes = buf_bytes_.at(it->second);
  if (capacity < bytes) fail(kErrInvalidArgument, "host buffer too small: need " + std::to_string(bytes) + " bytes");
  cuda_check(cudaDeviceSynchronize(), "synchronize before export");
  cuda_check(cudaMemcpy(host, bufs_.at(it->second), bytes, cudaMemcpyDeviceToHost), "export copy");
}

}  // namespace dfft
