// Batched register stages, separable-layout instantiation (see fft_batch.cu).
#include "fft_batch.cuh"

namespace dfft {
namespace dev {
namespace batch {
template <>
cudaError_t launch_batch_variant<false>(BatchParams& P, bool dbl, int kind, bool inverse, bool afast,
                                        cudaStream_t st) {
  return dbl ? launch_batch_t<double, false>(P, kind, inverse, afast, st)
             : launch_batch_t<float, false>(P, kind, inverse, afast, st);
}
}  // namespace batch
}  // namespace dev
}  // namespace dfft
