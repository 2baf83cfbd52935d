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

#define DFFT_BATCH_PAIR_LENGTHS(X) X(16) X(32) X(64) X(128) X(256) X(512) X(1024) X(2048)

int batch_pair_lines(int n, bool afast) {
  switch (n) {
#define DFFT_LINES(N_) \
  case N_: return 2 * (afast ? batch::BatchPairs<N_, true>::value : batch::BatchPairs<N_, false>::value);
    DFFT_BATCH_PAIR_LENGTHS(DFFT_LINES)
#undef DFFT_LINES
    default: return 0;
  }
}

cudaError_t launch_fft_batch_pair(BatchParams& P, bool inverse, bool afast, cudaStream_t st) {
  if (P.nfields < 1 || P.nfields > kMaxBatchFields) return cudaErrorInvalidValue;
  const int n = P.f[0].n;
  for (int i = 0; i < P.nfields; ++i)
    if (P.f[i].n != n || P.f[i].B != batch_pair_lines(n, afast)) return cudaErrorInvalidValue;
  switch (n) {
#define DFFT_CASE(N_)                                                                          \
  case N_:                                                                                     \
    if (inverse)                                                                               \
      return afast ? batch::launch_batch_pair_n<true, true, N_>(P, st)                         \
                   : batch::launch_batch_pair_n<true, false, N_>(P, st);                       \
    return afast ? batch::launch_batch_pair_n<false, true, N_>(P, st)                          \
                 : batch::launch_batch_pair_n<false, false, N_>(P, st);
    DFFT_BATCH_PAIR_LENGTHS(DFFT_CASE)
#undef DFFT_CASE
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace dev
}  // namespace dfft
