// Batched register FFT stages (sm_100a): one persistent launch runs one stage
// of many fields of uneven sizes that share the stage's line length.
//
// A CTA of kBatchThreads threads walks work items blockIdx.x, +gridDim.x, ...
// of a table that concatenates the tiles of every field; for each item it
// finds the field (the item index only grows, so the field index only
// advances), decodes the tile (tb, co0, co1) of that field's stage and runs
// the tile body of the line length with B = kBatchThreads / (N / V) lines,
// the same bodies as the one-tile-per-CTA kernels (fft_tile.cuh), at the
// register budget of those kernels.  The twiddles are staged once per CTA; a
// barrier separates consecutive tiles.  The host launches the lengths of one
// stage index concurrently (batch.cpp).
#include "fft_batch.cuh"

namespace dfft {
namespace dev {

namespace batch {
template <>
cudaError_t launch_batch_variant<true>(BatchParams& P, bool dbl, int kind, bool inverse, bool afast,
                                       cudaStream_t st) {
  return dbl ? launch_batch_t<double, true>(P, kind, inverse, afast, st)
             : launch_batch_t<float, true>(P, kind, inverse, afast, st);
}
}  // namespace batch

using namespace batch;

bool batch_stage_supported(int n) {
  switch (n) {
#define DFFT_OK(N_) case N_:
    DFFT_BATCH_LENGTHS(DFFT_OK)
#undef DFFT_OK
    return true;
    default: return false;
  }
}

int batch_stage_lines(int n) {
  switch (n) {
#define DFFT_LINES(N_) \
  case N_: return BatchLines<N_>::value;
    DFFT_BATCH_LENGTHS(DFFT_LINES)
#undef DFFT_LINES
    default: return 0;
  }
}

cudaError_t launch_fft_batch(BatchParams& P, bool dbl, int kind, bool inverse, bool afast, cudaStream_t st) {
  static_assert(sizeof(BatchParams) <= 32000, "batch parameters must fit the kernel parameter space");
  if (P.nfields < 1 || P.nfields > kMaxBatchFields) return cudaErrorInvalidValue;
  // separable sides on every field: the variant without the general-layout
  // addressing (fewer registers)
  bool general = false;
  for (int i = 0; i < P.nfields; ++i) general = general || P.f[i].src_line_affine || P.f[i].dst_line_affine || P.f[i].src_atab || P.f[i].dst_atab;
  return general ? launch_batch_variant<true>(P, dbl, kind, inverse, afast, st)
                 : launch_batch_variant<false>(P, dbl, kind, inverse, afast, st);
}

}  // namespace dev
}  // namespace dfft
