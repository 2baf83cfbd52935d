// Register-resident FFT stage for lines of 2^k or 3 * 2^k points (sm_100a).
//
// Used when both the source and the destination have unit stride along the
// FFT axis a ("a-fast": every line is one contiguous run) or along the tile
// axis b ("b-fast": at every position along a, neighbouring lines of the tile
// are neighbours in memory, except where a rank block ends).  Per-line base
// offsets come from the separable layout tables, so the stage still performs
// the reference's pack / all-to-all / unpack / local transpose by addressing.
//
// Each line of length N is transformed by N/V threads holding V values each
// (V = 8 for powers of two, V = 24 for 3 * 2^k; every radix of the plan
// divides V, so each pass is V/R butterflies per thread).
// The first radix pass reads its inputs straight from global memory and the
// last pass writes its outputs straight to global memory (consecutive threads
// touch consecutive addresses for either row orientation); the passes in
// between exchange values through padded shared memory (one pad element per
// 256 bytes, which keeps the stride-R Stockham writes conflict-light).
#include "fft_fast.cuh"

namespace dfft {
namespace dev {

template <typename T, int N, bool INV, bool AF>
static cudaError_t launch_fast_n(const StageArgs& A, cudaStream_t st) {
  constexpr int B0 = fast_lines<T>(N);
  constexpr int B1 = B0 / 2 > 0 ? B0 / 2 : 1;
  constexpr int B2 = B0 / 4 > 0 ? B0 / 4 : 1;
  if (A.B == B0) return launch_fast_b<T, N, INV, AF, B0>(A, st);
  if (A.B == B1) return launch_fast_b<T, N, INV, AF, B1>(A, st);
  if (A.B == B2) return launch_fast_b<T, N, INV, AF, B2>(A, st);
  return cudaErrorInvalidValue;
}

template <typename T, int N>
static cudaError_t launch_fast_t(const StageArgs& A, bool inverse, bool afast, cudaStream_t st) {
  if (inverse) {
    return afast ? launch_fast_n<T, N, true, true>(A, st) : launch_fast_n<T, N, true, false>(A, st);
  }
  return afast ? launch_fast_n<T, N, false, true>(A, st) : launch_fast_n<T, N, false, false>(A, st);
}

template <typename T, int N, bool C2R>
static cudaError_t launch_real_n(const StageArgs& A, cudaStream_t st) {
  constexpr int B0 = fast_lines<T>(N);
  constexpr int B1 = B0 / 2 > 0 ? B0 / 2 : 1;
  constexpr int B2 = B0 / 4 > 0 ? B0 / 4 : 1;
  if (A.B == B0) return launch_real_b<T, N, C2R, B0>(A, st);
  if (A.B == B1) return launch_real_b<T, N, C2R, B1>(A, st);
  if (A.B == B2) return launch_real_b<T, N, C2R, B2>(A, st);
  return cudaErrorInvalidValue;
}

int fast_stage_lines(bool dbl, int n) { return dbl ? fast_lines<double>(n) : fast_lines<float>(n); }

int fast_stage_line_options(bool dbl, int n, int* opts) {
  const int b0 = fast_stage_lines(dbl, n);
  int k = 0;
  opts[k++] = b0;
  if (b0 / 2 >= 1 && b0 / 2 != b0) opts[k++] = b0 / 2;
  if (b0 / 4 >= 1 && b0 / 4 != b0 / 2) opts[k++] = b0 / 4;
  return k;
}

bool fast_stage_supported(int n) {
  return n == 16 || n == 32 || n == 64 || n == 128 || n == 256 || n == 512 || n == 1024 || n == 2048 || n == 4096 ||
         n == 24 || n == 48 || n == 96 || n == 192 || n == 384 || n == 768;
}

cudaError_t launch_fft_fast(const StageArgs& A, bool dbl, bool inverse, bool afast, cudaStream_t st) {
  if (A.Eo0 > fast_stage_max_grid_yz() || A.Eo1 > fast_stage_max_grid_yz()) return cudaErrorInvalidValue;
  if (general_stage(A)) return launch_fast_general(A, dbl, inverse, afast, st);
#define DFFT_CASE(N_)                                                                 \
  case N_:                                                                            \
    return dbl ? launch_fast_t<double, N_>(A, inverse, afast, st)                     \
               : launch_fast_t<float, N_>(A, inverse, afast, st);
  switch (A.n) {
    DFFT_CASE(16)
    DFFT_CASE(32)
    DFFT_CASE(64)
    DFFT_CASE(128)
    DFFT_CASE(256)
    DFFT_CASE(512)
    DFFT_CASE(1024)
    DFFT_CASE(2048)
    DFFT_CASE(4096)
    DFFT_CASE(24)
    DFFT_CASE(48)
    DFFT_CASE(96)
    DFFT_CASE(192)
    DFFT_CASE(384)
    DFFT_CASE(768)
    default: return cudaErrorInvalidValue;
  }
#undef DFFT_CASE
}

cudaError_t launch_fft_fast_real(const StageArgs& A, bool dbl, bool c2r, cudaStream_t st) {
  if (A.Eo0 > fast_stage_max_grid_yz() || A.Eo1 > fast_stage_max_grid_yz()) return cudaErrorInvalidValue;
  if (general_stage(A)) return launch_real_general(A, dbl, c2r, st);
#define DFFT_CASE(N_)                                                                          \
  case N_:                                                                                     \
    if (dbl) return c2r ? launch_real_n<double, N_, true>(A, st) : launch_real_n<double, N_, false>(A, st); \
    return c2r ? launch_real_n<float, N_, true>(A, st) : launch_real_n<float, N_, false>(A, st);
  switch (A.n) {
    DFFT_CASE(16)
    DFFT_CASE(32)
    DFFT_CASE(64)
    DFFT_CASE(128)
    DFFT_CASE(256)
    DFFT_CASE(512)
    DFFT_CASE(1024)
    DFFT_CASE(2048)
    DFFT_CASE(4096)
    DFFT_CASE(24)
    DFFT_CASE(48)
    DFFT_CASE(96)
    DFFT_CASE(192)
    DFFT_CASE(384)
    DFFT_CASE(768)
    default: return cudaErrorInvalidValue;
  }
#undef DFFT_CASE
}

}  // namespace dev
}  // namespace dfft
