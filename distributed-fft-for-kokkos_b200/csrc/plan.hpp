// Execution plan: validation (internal_plan_factory), per-rank block
// analyses, and the device programs that execute the forward and backward
// transforms.
#pragma once

#include <cuda_runtime.h>

#include <map>
#include <memory>
#include <string>
#include <vector>

#include "dev_types.h"
#include "exchange.hpp"
#include "layout.hpp"
#include "plan_core.hpp"

namespace dfft {

struct PlanDesc {
  Ext axes;  // non-negative
  Ext gin, gout, in_topo, out_topo;
  bool in_right = true, out_right = true, view_right = true;
  bool r2c = false;
  bool dbl = true;
  bool comp = false;  // FP32 with the compensated last radix pass of two-line stages
  int norm = 0;       // 0 backward, 1 forward, 2 ortho, 3 none
  int exec_mode = 0;  // 0 fused, 1 literal, 2 literal with capture of every exchange
  cudaStream_t stream = nullptr;
  // >= 0: the program of this one world rank (one process per GPU): its local
  // blocks only, with the exchanges left to the caller's communicator
  long long rank = -1;
};

// Buffer ids used by the device programs (send / recv: the caller's exchange
// buffers of a per-rank program).
enum : int { kBufRecv = -3, kBufSend = -2, kBufIn = 0, kBufOut = 1, kBufScratch0 = 2, kBufScratch1 = 3,
             kBufFirstDebug = 4 };

// One all-to-all of a per-rank program: the send buffer (the reference's
// [group size, buffer extents] pack buffer of transpose block `block`) goes
// out in equal chunks, one per group member, and the recv buffer of the same
// size comes back.
struct Exchange {
  std::size_t block = 0;
  int comm_axis = -1;  // -1 whole communicator; 0 / 1 row / column communicator
  std::size_t elements = 0;
  std::size_t elem_bytes = 0;
  bool padded = false;  // the send buffer has entries past the bins that must stay zero
  ExchangeGroup group;  // this rank's group (world ranks by sub-rank)
};

// Tiled tensor-map description of a TMA-fed stage's source layout (5
// dimensions, unused ones of extent 1): byte strides of dimensions 1..4, the
// box, and how the kernel forms a tile's coordinates.
struct TmaSource {
  bool ok = false;
  std::uint64_t lb = 0;  // extent of the tile axis b inside a rank block
  bool b_split = false;  // b split across ranks: tiles must not cross a block
  std::uint64_t dim[5] = {1, 1, 1, 1, 1};
  std::uint64_t stride[5] = {0, 0, 0, 0, 0};
  std::uint32_t box[5] = {1, 1, 1, 1, 1};
  dev::TmaCoords coords{};
};

// Encode `t` for source address `base` into the 128-byte CUtensorMap at `map`
// (64-byte aligned); false if the driver has no tensor-map support or refuses
// the description (tma.cpp).
bool tma_encode(void* map, const void* base, const TmaSource& t);

struct Op {
  enum Type { Stage, Pack, All2All, Unpack, Scale, Copy, Weight, BluePre, BlueMul, BluePost, FourTwiddle } type;
  int src = -1, dst = -1;  // buffer ids
  // Stage
  dev::StageArgs sa{};
  int kind = 0;
  bool inverse = false;
  bool fast = false;  // register-resident kernel (fft_fast.cu, or fft_pair.cu when sa.pairs)
  int single_B = 0;   // lines per tile of the one-line kernel, for b-fast pair stages whose
                      // caller buffers turn out not to be 16-byte aligned
  int pair_B = 0;     // lines per tile of the two-line kernel, for TMA stages whose source
                      // cannot be described by a tensor map at run time
  TmaSource tma;      // source description of a TMA-eligible b-fast pair stage
  // chirp-z stage (line length with a prime factor above 13): make_stage marks
  // it, push_stage expands it into pre / FFT / mul / inverse FFT / post ops
  bool blue = false;
  int blue_m = 0;
  long long blue_lines = 0;
  const void* blue_chirp = nullptr;
  const void* blue_filter = nullptr;
  // four-step stage (a line too long for one stage, n = four_n1 * four_n2):
  // pre / strided FFT / twiddle / contiguous FFT / post, sharing the chirp-z
  // gather and scatter kernels
  int four_n1 = 0, four_n2 = 0;
  const void* four_tw = nullptr;
  int nthreads = 256;
  std::size_t smem = 0;
  unsigned tiles = 0;
  int src_layout = -1, dst_layout = -1;
  // Pack / All2All / Unpack
  dev::XposeArgs xa{};
  int elem_bytes = 0;
  int block = -1;  // transpose block index in the block list
  // Weight (Hermitian weights of an R2C spectrum)
  int w_axis = 0, w_n = 0;
  // Scale / Copy
  std::int64_t n_real = 0;
  std::size_t bytes = 0;
  double scale = 1.0;
};

class Plan {
 public:
  Plan(const PlanDesc& d, bool on_device);
  ~Plan();
  Plan(const Plan&) = delete;
  Plan& operator=(const Plan&) = delete;

  void execute(const void* in, void* out, bool forward, cudaStream_t stream) const;
  // Adjoint (conjugate transpose) of the forward (of_forward) or backward
  // transform, normalisation included: of_forward maps the output layout to the
  // input layout, the other the input layout to the output layout.
  void execute_adjoint(const void* in, void* out, bool of_forward, cudaStream_t stream) const;

  const std::string& name() const { return name_; }
  std::size_t nprocs() const { return total_size(d_.in_topo); }
  const PlanDesc& desc() const { return d_; }
  const std::vector<BlockAnalyses>& analyses() const { return per_rank_; }
  std::size_t max_buffer_size() const { return max_buffer_size_; }
  const std::vector<Ext>& chain() const { return chain_; }
  const std::vector<std::size_t>& chain_trans_axes() const { return trans_axes_; }
  const std::vector<std::size_t>& chain_layouts() const { return chain_layouts_; }
  const Layout& in_layout() const { return lin_; }
  const Layout& out_layout() const { return lout_; }
  std::size_t launches(bool forward) const { return prog_[forward ? 0 : 1].size(); }
  std::size_t workspace_bytes() const { return workspace_bytes_; }
  bool on_device() const { return on_device_; }
  // Device error word (0 or the code a kernel's bounded wait left); reset clears it.
  int device_error(bool reset) const;
  // Batched execution (batch.cpp): the fused program of a direction, the
  // plan's device buffers by id, one op's launch, and the checks of execute.
  const std::vector<Op>& program(bool forward) const { return prog_[forward ? 0 : 1]; }
  void* device_buffer(int id) const { return bufs_.at(id); }
  cudaError_t launch_op(const Op& op, const dev::StageArgs& A, cudaStream_t stream) const {
    return launch_stage(op, A, stream);
  }
  void check_buffers(const void* in, const void* out, bool forward) const;
  // Device tables of the caller-facing input / output layouts.
  dev::DevLayout device_layout(bool output) const;
  // Copy a buffer recorded by a capturing literal execution of transpose
  // block `block` to host: which = 0 send, 1 recv, 2 pack input, 3 unpack output.
  void export_buffers(bool forward, std::size_t block, int which, void* host, std::size_t capacity) const;

  // Backward transform whose first stage multiplies every loaded value by a
  // spectral factor (dev::StageArgs::pre_mode and the geometry in pre; the
  // stage runs the general-layout one-line kernel).  can_premultiply(): the
  // first backward stage is a register C2C stage, else the caller applies the
  // factor itself.
  bool can_premultiply() const;
  void execute_backward_premul(const void* in, void* out, const dev::StageArgs& pre, cudaStream_t stream) const;

  // Per-rank programs (desc().rank >= 0, rank.cpp).  A direction runs as
  // segments: segment 0 reads `in`, every segment but the last ends by
  // writing exchange k's send buffer, the caller's all-to-all fills its recv
  // buffer, which segment k + 1 reads; the last segment writes `out`.
  bool is_rank_plan() const { return d_.rank >= 0; }
  const std::vector<Exchange>& exchanges(bool forward) const { return xch_[forward ? 0 : 1]; }
  // Exchange group of any world rank for exchange k of a direction.
  ExchangeGroup exchange_group_of(bool forward, std::size_t k, std::size_t rank) const;
  void execute_segment(bool forward, std::size_t segment, const void* in, void* out, void* send, void* recv,
                       cudaStream_t stream) const;
  // Local extents (logical order) of this rank's input (which 0) / output (1) block.
  Ext rank_local_extents(int which) const;

 private:
  PlanDesc d_;
  bool on_device_;
  std::string name_;
  TopologyType type_;
  std::vector<Ext> chain_;
  std::vector<std::size_t> trans_axes_, chain_layouts_;
  std::vector<BlockAnalyses> per_rank_;
  std::size_t max_buffer_size_ = 0;
  double scale_fwd_ = 1.0, scale_bwd_ = 1.0;
  Layout lin_, lout_;

  // device programs and resources
  std::vector<Layout> layouts_;
  std::vector<LayoutTables> tables_;
  std::vector<std::int64_t> host_tables_;
  std::vector<std::int64_t> layout_base_;  // offset of each layout's tables
  std::int64_t* d_tables_ = nullptr;
  std::vector<Op> prog_[2];
  std::vector<Op> adj_[2];  // adjoint of forward, adjoint of backward
  std::vector<void*> bufs_;                 // device buffers by id (in/out are null)
  std::vector<std::size_t> buf_bytes_;
  std::map<std::pair<std::size_t, bool>, void*> twiddles_;
  std::map<std::pair<int, int>, int> debug_bufs_;  // (dir, block*4 + which) -> buffer id
  int debug_buffer(int dir, std::size_t block, int which, std::size_t bytes);
  std::size_t workspace_bytes_ = 0;
  int* d_err_ = nullptr;  // device error word (dev::StageArgs::err)

  void analyze();
  int add_layout(const Layout& L);
  std::vector<std::size_t> fft_axis_order() const;
  Layout block_layout(const Ext& topo, bool rank_right, const Ext& map, bool complex) const;
  Op make_stage(int src_layout, int dst_layout, std::size_t a, int kind, bool inverse, double scale);
  // Append a stage op, or the five ops of a chirp-z stage.
  void push_stage(std::vector<Op>& prog, const Op& op);
  std::map<std::pair<std::size_t, std::size_t>, std::vector<void*>> blue_tables_;  // (n, m) -> chirp, filter fwd / inv
  void bluestein_tables(std::size_t n, std::size_t m, const void** chirp, const void** ffwd, const void** finv);
  std::int64_t add_geo(const Layout& L, const BlockInfo& b, std::size_t pc);
  void build_fused(bool forward);
  void build_literal(bool forward);
  void build_adjoint(bool of_forward);
  void run_program(const std::vector<Op>& prog, const void* in, void* out, cudaStream_t stream,
                   std::size_t begin = 0, std::size_t end = ~std::size_t(0), void* send = nullptr,
                   void* recv = nullptr) const;
  void check_alignment(const void* p, bool complex, const char* which) const;
  void finalize_program(std::vector<Op>& prog, int cur_layout, int cur_buf, const Layout& final_layout,
                        double scale, bool final_complex);
  void allocate_device();
  void autotune();
  // per-rank programs
  std::vector<Exchange> xch_[2];
  std::vector<std::size_t> seg_end_[2];  // op index one past each segment's last op
  Layout rank_layout(std::size_t chain_index, bool complex) const;
  Layout rank_buffer_layout(std::size_t chain_index, bool complex, std::size_t split_axis, const BlockInfo& b) const;
  void rank_exchanges(bool forward);
  void build_rank(bool forward);
  bool tma_source(int layout, const dev::StageArgs& A, TmaSource* out) const;
  cudaError_t launch_stage(const Op& op, dev::StageArgs A, cudaStream_t stream) const;
  const void* twiddle(std::size_t n);
};

}  // namespace dfft
