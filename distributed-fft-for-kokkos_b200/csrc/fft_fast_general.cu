// General-layout instantiations of the register FFT stage kernels
// (fft_fast.cuh): lines addressed as base + p * stride from the general layout
// tables, exchange-buffer sides addressed through the axis table, and the
// spectral pre-multiplier of the Navier-Stokes backward transforms.  A
// translation unit of its own so that it compiles beside fft_fast.cu.
#include "fft_fast.cuh"

namespace dfft {
namespace dev {

namespace {

template <typename T, int N, bool INV, bool AF>
cudaError_t general_fast_n(const StageArgs& A, cudaStream_t st) {
  constexpr int B0 = fast_lines<T>(N);
  constexpr int B1 = B0 / 2 > 0 ? B0 / 2 : 1;
  constexpr int B2 = B0 / 4 > 0 ? B0 / 4 : 1;
  if (A.B == B0) return launch_fast_b<T, N, INV, AF, B0, true>(A, st);
  if (A.B == B1) return launch_fast_b<T, N, INV, AF, B1, true>(A, st);
  if (A.B == B2) return launch_fast_b<T, N, INV, AF, B2, true>(A, st);
  return cudaErrorInvalidValue;
}

template <typename T, int N>
cudaError_t general_fast_t(const StageArgs& A, bool inverse, bool afast, cudaStream_t st) {
  if (inverse) return afast ? general_fast_n<T, N, true, true>(A, st) : general_fast_n<T, N, true, false>(A, st);
  return afast ? general_fast_n<T, N, false, true>(A, st) : general_fast_n<T, N, false, false>(A, st);
}

template <typename T, int N, bool C2R>
cudaError_t general_real_n(const StageArgs& A, cudaStream_t st) {
  constexpr int B0 = fast_lines<T>(N);
  constexpr int B1 = B0 / 2 > 0 ? B0 / 2 : 1;
  constexpr int B2 = B0 / 4 > 0 ? B0 / 4 : 1;
  if (A.B == B0) return launch_real_b<T, N, C2R, B0, true>(A, st);
  if (A.B == B1) return launch_real_b<T, N, C2R, B1, true>(A, st);
  if (A.B == B2) return launch_real_b<T, N, C2R, B2, true>(A, st);
  return cudaErrorInvalidValue;
}

}  // namespace

#define DFFT_GENERAL_LENGTHS(X) \
  X(16) X(32) X(64) X(128) X(256) X(512) X(1024) X(2048) X(4096) X(24) X(48) X(96) X(192) X(384) X(768)

cudaError_t launch_fast_general(const StageArgs& A, bool dbl, bool inverse, bool afast, cudaStream_t st) {
  switch (A.n) {
#define DFFT_CASE(N_) \
  case N_:            \
    return dbl ? general_fast_t<double, N_>(A, inverse, afast, st) : general_fast_t<float, N_>(A, inverse, afast, st);
    DFFT_GENERAL_LENGTHS(DFFT_CASE)
#undef DFFT_CASE
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_real_general(const StageArgs& A, bool dbl, bool c2r, cudaStream_t st) {
  switch (A.n) {
#define DFFT_CASE(N_)                                                                                          \
  case N_:                                                                                                     \
    if (dbl) return c2r ? general_real_n<double, N_, true>(A, st) : general_real_n<double, N_, false>(A, st); \
    return c2r ? general_real_n<float, N_, true>(A, st) : general_real_n<float, N_, false>(A, st);
    DFFT_GENERAL_LENGTHS(DFFT_CASE)
#undef DFFT_CASE
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace dev
}  // namespace dfft
