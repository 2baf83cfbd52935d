// Batched execution (see batch.hpp).
#include "batch.hpp"

#include <algorithm>
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

// kind, inverse, a-fast rows, value class (3 * 2^k lengths or powers of two):
// one batched launch per group
using GroupKey = std::tuple<int, bool, bool, bool>;

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
        ++groups[GroupKey(op.kind, op.inverse, op.sa.load_afast != 0, op.sa.n % 3 == 0)];
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
      // the batched tile bodies: one line per thread group, lines per tile
      // fixed by the line length
      A.pairs = 0;
      A.comp = 0;
      A.B = dev::batch_stage_lines(A.n);
      const int per = (op.kind == dev::kC2C) ? A.B : 2 * A.B;
      A.tiles_b = (A.Eb + per - 1) / per;
      groups[GroupKey(op.kind, op.inverse, A.load_afast != 0, A.n % 3 == 0)].push_back(A);
    }
    for (auto& g : groups) {
      const auto& list = g.second;
      for (std::size_t c = 0; c < list.size(); c += dev::kMaxBatchFields) {
        dev::BatchParams P;
        std::memset(&P, 0, sizeof(P));
        P.nfields = static_cast<int>(std::min<std::size_t>(dev::kMaxBatchFields, list.size() - c));
        P.prefix[0] = 0;
        for (int i = 0; i < P.nfields; ++i) {
          P.f[i] = list[c + i];
          const long long tiles = static_cast<long long>(P.f[i].tiles_b) * P.f[i].Eo0 * P.f[i].Eo1;
          if (tiles >= (1ll << 31)) fail(kErrUnsupported, "too many tiles in one field of a batch");
          P.prefix[i + 1] = P.prefix[i] + tiles;
        }
        const cudaError_t e = dev::launch_fft_batch(P, dbl_, std::get<0>(g.first), std::get<1>(g.first),
                                                    std::get<2>(g.first), st);
        if (e != cudaSuccess) fail(kErrCuda, std::string("batched stage launch failed: ") + cudaGetErrorString(e));
      }
    }
  }
}

}  // namespace dfft
