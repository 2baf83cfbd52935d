// Batched execution (see batch.hpp).
#include "batch.hpp"

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <map>
#include <set>
#include <string>
#include <tuple>

namespace dfft {

namespace {

// A stage the batched kernels run: a register-resident C2C, R2C or C2R stage
// whose line length has a batched tile body.
bool batchable(const Op& op) {
  if (op.type != Op::Stage || !op.fast) return false;
  if (op.kind != dev::kC2C && op.kind != dev::kR2C && op.kind != dev::kC2R) return false;
  return dev::batch_stage_supported(op.sa.n);
}

// kind, inverse, a-fast rows, line length, two-line tiles: one batched launch
// per group
using GroupKey = std::tuple<int, bool, bool, int, bool>;

// complex64 C2C stages the one-tile launches would run two lines per thread
// (separable sides, pair-aligned: op.single_B is set) take the batched
// two-line tiles
bool pair_batchable(const Op& op, bool dbl) {
  return !dbl && op.kind == dev::kC2C && op.single_B != 0 && dev::batch_pair_lines(op.sa.n, op.sa.load_afast != 0) > 0;
}

void ck(cudaError_t e) {
  if (e != cudaSuccess) fail(kErrCuda, std::string("batch stream fork / join: ") + cudaGetErrorString(e));
}

}  // namespace

Batch::Batch(std::vector<const Plan*> plans) : plans_(std::move(plans)) {
  if (plans_.empty()) fail(kErrInvalidArgument, "a batch needs at least one plan");
  std::set<const Plan*> seen;
  for (const Plan* p : plans_) {
    if (!p) fail(kErrInvalidArgument, "null plan in batch");
    if (!p->on_device()) fail(kErrInvalidArgument, "plan was created by dfft_plan_analyze and cannot execute");
    if (!seen.insert(p).second)
      fail(kErrInvalidArgument, "a plan appears twice in the batch (its scratch arrays would be shared)");
    if (p->desc().exec_mode != 0) fail(kErrInvalidArgument, "batched execution needs fused plans");
    if (p->is_rank_plan()) fail(kErrInvalidArgument, "batched execution needs plans over all ranks, not per-rank plans");
    for (bool fwd : {true, false})
      for (const Op& op : p->program(fwd))
        if (op.type != Op::Stage)
          fail(kErrInvalidArgument, "batched execution needs fused plans whose stages are all FFT stage kernels");
  }
  dbl_ = plans_[0]->desc().dbl;
  for (const Plan* p : plans_)
    if (p->desc().dbl != dbl_) fail(kErrInvalidArgument, "all plans of a batch must have the same precision");
  bool ok = cudaEventCreateWithFlags(&fork_, cudaEventDisableTiming) == cudaSuccess;
  for (int i = 0; ok && i < kAux; ++i)
    ok = cudaStreamCreateWithFlags(&aux_[i], cudaStreamNonBlocking) == cudaSuccess &&
         cudaEventCreateWithFlags(&join_[i], cudaEventDisableTiming) == cudaSuccess;
  if (!ok) {
    cudaGetLastError();
    release();
    fail(kErrCuda, "batch stream / event creation failed");
  }
}

Batch::~Batch() { release(); }

void Batch::release() {
  for (int i = 0; i < kAux; ++i) {
    if (aux_[i]) cudaStreamDestroy(aux_[i]);
    if (join_[i]) cudaEventDestroy(join_[i]);
    aux_[i] = nullptr;
    join_[i] = nullptr;
  }
  if (fork_) cudaEventDestroy(fork_);
  fork_ = nullptr;
}

std::size_t Batch::launches(bool forward) const {
  std::size_t nst = 0, n = 0;
  for (const Plan* p : plans_) nst = std::max(nst, p->program(forward).size());
  for (std::size_t s = 0; s < nst; ++s) {
    std::map<GroupKey, std::size_t> groups;
    for (const Plan* p : plans_) {
      const auto& prog = p->program(forward);
      if (s >= prog.size() || prog[s].tiles == 0) continue;
      const Op& op = prog[s];
      if (batchable(op))
        ++groups[GroupKey(op.kind, op.inverse, op.sa.load_afast != 0, op.sa.n, pair_batchable(op, dbl_))];
      else
        ++n;
    }
    for (auto& g : groups) n += (g.second + dev::kMaxBatchFields - 1) / dev::kMaxBatchFields;
  }
  return n;
}

void Batch::execute(const void* const* ins, void* const* outs, bool forward, cudaStream_t st) const {
  if (!ins || !outs) fail(kErrInvalidArgument, "null buffer arrays");
  for (std::size_t f = 0; f < plans_.size(); ++f) plans_[f]->check_buffers(ins[f], outs[f], forward);
  std::size_t nst = 0;
  for (const Plan* p : plans_) nst = std::max(nst, p->program(forward).size());
  for (std::size_t s = 0; s < nst; ++s) {
    std::map<GroupKey, std::vector<dev::StageArgs>> groups;
    for (std::size_t f = 0; f < plans_.size(); ++f) {
      const Plan* p = plans_[f];
      const auto& prog = p->program(forward);
      if (s >= prog.size()) continue;
      const Op& op = prog[s];
      if (op.tiles == 0) continue;
      dev::StageArgs A = op.sa;
      A.in = op.src == kBufIn ? const_cast<void*>(ins[f]) : op.src == kBufOut ? outs[f] : p->device_buffer(op.src);
      A.out = op.dst == kBufIn ? const_cast<void*>(ins[f]) : op.dst == kBufOut ? outs[f] : p->device_buffer(op.dst);
      if (!batchable(op)) {
        const cudaError_t e = p->launch_op(op, A, st);
        if (e != cudaSuccess) fail(kErrCuda, std::string("kernel launch failed: ") + cudaGetErrorString(e));
        continue;
      }
      // the batched tile bodies: two lines per thread where the one-tile
      // launch could run them, else one line per thread group; lines per
      // tile fixed by the line length
      // (b-fast pairs move 16 bytes at a time: both buffers on 16-byte boundaries)
      const bool aligned = ((reinterpret_cast<std::uintptr_t>(A.in) | reinterpret_cast<std::uintptr_t>(A.out)) & 15) == 0;
      const bool pair = pair_batchable(op, dbl_) && (A.load_afast || aligned);
      A.pairs = 0;
      A.comp = 0;
      A.B = pair ? dev::batch_pair_lines(A.n, A.load_afast != 0) : dev::batch_stage_lines(A.n);
      const int per = (op.kind == dev::kC2C) ? A.B : 2 * A.B;
      A.tiles_b = (A.Eb + per - 1) / per;
      groups[GroupKey(op.kind, op.inverse, A.load_afast != 0, A.n, pair)].push_back(A);
    }
    // one launch per group (and per kMaxBatchFields fields of it); within a
    // launch the largest fields come first, so the last work items the
    // persistent CTAs pick up are small tiles and the launch ends evenly
    int nl = 0;
    for (auto& g : groups) nl += static_cast<int>((g.second.size() + dev::kMaxBatchFields - 1) / dev::kMaxBatchFields);
    fork(st, nl);
    auto tiles_of = [](const dev::StageArgs& A) { return static_cast<long long>(A.tiles_b) * A.Eo0 * A.Eo1; };
    int li = 0;
    for (auto& g : groups) {
      auto list = g.second;
      std::stable_sort(list.begin(), list.end(),
                       [&](const dev::StageArgs& x, const dev::StageArgs& y) { return tiles_of(x) > tiles_of(y); });
      for (std::size_t c = 0; c < list.size(); c += dev::kMaxBatchFields, ++li) {
        dev::BatchParams P;
        std::memset(&P, 0, sizeof(P));
        P.nfields = static_cast<int>(std::min<std::size_t>(dev::kMaxBatchFields, list.size() - c));
        P.prefix[0] = 0;
        for (int i = 0; i < P.nfields; ++i) {
          P.f[i] = list[c + i];
          const long long tiles = tiles_of(P.f[i]);
          if (tiles >= (1ll << 31)) fail(kErrUnsupported, "too many tiles in one field of a batch");
          P.prefix[i + 1] = P.prefix[i] + tiles;
        }
        const cudaStream_t ls = lane(st, li);
        const cudaError_t e = std::get<4>(g.first)
                                  ? dev::launch_fft_batch_pair(P, std::get<1>(g.first), std::get<2>(g.first), ls)
                                  : dev::launch_fft_batch(P, dbl_, std::get<0>(g.first), std::get<1>(g.first),
                                                          std::get<2>(g.first), ls);
        if (e != cudaSuccess) fail(kErrCuda, std::string("batched stage launch failed: ") + cudaGetErrorString(e));
      }
    }
    join(st, nl);
  }
}

void Batch::fork(cudaStream_t st, int lanes) const {
  if (lanes <= 1) return;
  ck(cudaEventRecord(fork_, st));
  for (int i = 0; i < std::min(lanes - 1, kAux); ++i) ck(cudaStreamWaitEvent(aux_[i], fork_, 0));
}

void Batch::join(cudaStream_t st, int lanes) const {
  if (lanes <= 1) return;
  for (int i = 0; i < std::min(lanes - 1, kAux); ++i) {
    ck(cudaEventRecord(join_[i], aux_[i]));
    ck(cudaStreamWaitEvent(st, join_[i], 0));
  }
}

}  // namespace dfft
