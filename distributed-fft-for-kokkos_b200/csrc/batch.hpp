// Batched execution of many plans (fields of uneven sizes): every stage index
// of the fused programs runs as one persistent launch per group of stages
// that share kind, direction and row orientation (fft_batch.cu), instead of
// one launch per field.
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "plan.hpp"

namespace dfft {

class Batch {
 public:
  // Distinct, executable plans of one precision with fused programs.
  explicit Batch(std::vector<const Plan*> plans);
  ~Batch();
  Batch(const Batch&) = delete;
  Batch& operator=(const Batch&) = delete;
  // Field f: ins[f] -> outs[f] in `forward` direction (plan buffers as for
  // Plan::execute), all on one stream.
  void execute(const void* const* ins, void* const* outs, bool forward, cudaStream_t st) const;
  // Kernel launches of one execute in a direction.
  std::size_t launches(bool forward) const;
  std::size_t size() const { return plans_.size(); }
  const std::vector<const Plan*>& plans() const { return plans_; }

  // The launches of one stage index that belong to different groups touch
  // different fields: they run concurrently, forked from the caller's stream
  // onto kAux auxiliary streams and joined back (graph-capturable).  Callers
  // with per-field work of their own (the Navier-Stokes phases) use the same
  // lanes: lane 0 is the caller's stream, lane i > 0 aux stream i - 1.
  static constexpr int kAux = 3;
  void fork(cudaStream_t st, int lanes) const;
  void join(cudaStream_t st, int lanes) const;
  cudaStream_t lane(cudaStream_t st, int i) const { return i == 0 ? st : aux_[(i - 1) % kAux]; }

 private:
  std::vector<const Plan*> plans_;
  bool dbl_ = false;
  cudaStream_t aux_[kAux] = {};
  cudaEvent_t fork_ = nullptr;
  cudaEvent_t join_[kAux] = {};
  void release();
};

}  // namespace dfft
