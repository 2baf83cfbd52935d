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
#include "fft_tile.cuh"

namespace dfft {
namespace dev {

using namespace radix;


// B lines per CTA, N/V threads per line.
// AFF: the general-layout variant (affine lines on the sides that set
// src_line_affine / dst_line_affine); the separable variant carries none of
// its code, which keeps its register count.
// Resident CTAs per SM the register budget is sized for.  Left alone, the
// compiler spends registers on scheduling freedom: the separable 8-value
// kernels take a few more than the budget of their natural occupancy (b-fast
// 1024-thread tiles lose half their resident threads at 33+ registers) and
// the 24-value kernels anything up to 150.  So 8-value kernels are held to
// 2048 (b-fast) or 1536 (a-fast) complex64 threads, or 1024 complex128
// threads, per SM, and 24-value kernels to 768 complex64 or 384 complex128
// threads (about 85 / 170 registers).  The general-layout 8-value variant
// keeps the compiler's choice.
template <typename T, int N, int THREADS, bool AFAST, bool AFF>
struct MinBlocks {
  static constexpr bool v8 = Vals<N>::value == 8;
  static constexpr bool bound = !(v8 && AFF);
  static constexpr int target = v8 ? (sizeof(T) == 4 ? (AFAST ? 1536 : 2048) : 1024) : (sizeof(T) == 4 ? 768 : 384);
  static constexpr int v = target / THREADS;
  static constexpr int value = (bound && v > 0) ? v : 1;
};

template <typename T, bool INV, int N, int B, bool AFAST, bool AFF>
__global__ void __launch_bounds__(N / Vals<N>::value * B,
                                  (MinBlocks<T, N, N / Vals<N>::value * B, AFAST, AFF>::value))
    fft_fast_kernel(const StageArgs A) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  // grid (tiles_b, Eo0, Eo1): tile along b, coordinates along o0 and o1
  fast_tile<T, INV, N, B, AFAST, AFF>(A, blockIdx.x, blockIdx.y, blockIdx.z, smem_raw);
}

template <typename T, bool C2R, int N, int B, bool AFF>
__global__ void __launch_bounds__(N / Vals<N>::value * B) fft_real_kernel(const StageArgs A) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  // grid (tiles_b, Eo0, Eo1): tile along b, coordinates along o0 and o1
  real_tile<T, C2R, N, B, AFF>(A, blockIdx.x, blockIdx.y, blockIdx.z, smem_raw);
}

// Default lines per CTA: at least 128-byte rows for b-fast tiles (16
// complex64 or 8 complex128), at least 256 threads, at most 1024 threads
// (N/V per line).  The launcher also has variants with 1/2 and 1/4 of it.
template <typename T>
constexpr int fast_lines(int n) {
  const int tt = n % 3 == 0 ? n / 24 : n / 8;
  const int rows = sizeof(T) == 4 ? 16 : 8;
  const int want = rows > 256 / tt ? rows : 256 / tt;
  const int cap = 1024 / tt;
  return want < cap ? want : cap;
}

template <typename T, int N, bool INV, bool AF, int B, bool AFF = false>
static cudaError_t launch_fast_b(const StageArgs& A, cudaStream_t st) {
  constexpr int LP = SmemShape<T, N, B, AF>::LP;
  const size_t smem = sizeof(cplx<T>) * (N + static_cast<size_t>(B) * LP);
  auto k = fft_fast_kernel<T, INV, N, B, AF, AFF>;
  const cudaError_t e = raise_smem_limit(reinterpret_cast<const void*>(k), smem);
  if (e != cudaSuccess) return e;
  k<<<fast_grid(A), N / Vals<N>::value * B, smem, st>>>(with_table_offsets(A));
  return cudaGetLastError();
}

template <typename T, int N, bool INV, bool AF>
static cudaError_t launch_fast_n(const StageArgs& A, cudaStream_t st) {
  constexpr int B0 = fast_lines<T>(N);
  constexpr int B1 = B0 / 2 > 0 ? B0 / 2 : 1;
  constexpr int B2 = B0 / 4 > 0 ? B0 / 4 : 1;
  if (A.src_line_affine || A.dst_line_affine || A.src_atab || A.dst_atab || A.pre_mode)  // general layouts: default tile only
    return A.B == B0 ? launch_fast_b<T, N, INV, AF, B0, true>(A, st) : cudaErrorInvalidValue;
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

template <typename T, int N, bool C2R, int B, bool AFF = false>
static cudaError_t launch_real_b(const StageArgs& A, cudaStream_t st) {
  constexpr int LP = SmemShape<T, N, B, true>::LP;
  const size_t smem = sizeof(cplx<T>) * (N + static_cast<size_t>(B) * LP);
  auto k = fft_real_kernel<T, C2R, N, B, AFF>;
  const cudaError_t e = raise_smem_limit(reinterpret_cast<const void*>(k), smem);
  if (e != cudaSuccess) return e;
  k<<<fast_grid(A), N / Vals<N>::value * B, smem, st>>>(with_table_offsets(A));
  return cudaGetLastError();
}

template <typename T, int N, bool C2R>
static cudaError_t launch_real_n(const StageArgs& A, cudaStream_t st) {
  constexpr int B0 = fast_lines<T>(N);
  constexpr int B1 = B0 / 2 > 0 ? B0 / 2 : 1;
  constexpr int B2 = B0 / 4 > 0 ? B0 / 4 : 1;
  if (A.src_line_affine || A.dst_line_affine || A.src_atab || A.dst_atab || A.pre_mode)
    return A.B == B0 ? launch_real_b<T, N, C2R, B0, true>(A, st) : cudaErrorInvalidValue;
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
