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
  // Field f: ins[f] -> outs[f] in `forward` direction (plan buffers as for
  // Plan::execute), all on one stream.
  void execute(const void* const* ins, void* const* outs, bool forward, cudaStream_t st) const;
  // Kernel launches of one execute in a direction.
  std::size_t launches(bool forward) const;
  std::size_t size() const { return plans_.size(); }
  const std::vector<const Plan*>& plans() const { return plans_; }

 private:
  std::vector<const Plan*> plans_;
  bool dbl_ = false;
};

}  // namespace dfft
