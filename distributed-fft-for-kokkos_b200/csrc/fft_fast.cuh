// Register-resident FFT stage kernels (fft_fast.cu describes them) and their
// per-tile launchers, shared by the separable-layout instantiations
// (fft_fast.cu) and the general-layout ones (fft_fast_general.cu), which
// compile as two translation units.
#pragma once

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
inline cudaError_t launch_fast_b(const StageArgs& A, cudaStream_t st) {
  constexpr int LP = SmemShape<T, N, B, AF>::LP;
  const size_t smem = sizeof(cplx<T>) * (N + static_cast<size_t>(B) * LP);
  auto k = fft_fast_kernel<T, INV, N, B, AF, AFF>;
  const cudaError_t e = raise_smem_limit(reinterpret_cast<const void*>(k), smem);
  if (e != cudaSuccess) return e;
  k<<<fast_grid(A), N / Vals<N>::value * B, smem, st>>>(with_table_offsets(A));
  return cudaGetLastError();
}

template <typename T, int N, bool C2R, int B, bool AFF = false>
inline cudaError_t launch_real_b(const StageArgs& A, cudaStream_t st) {
  constexpr int LP = SmemShape<T, N, B, true>::LP;
  const size_t smem = sizeof(cplx<T>) * (N + static_cast<size_t>(B) * LP);
  auto k = fft_real_kernel<T, C2R, N, B, AFF>;
  const cudaError_t e = raise_smem_limit(reinterpret_cast<const void*>(k), smem);
  if (e != cudaSuccess) return e;
  k<<<fast_grid(A), N / Vals<N>::value * B, smem, st>>>(with_table_offsets(A));
  return cudaGetLastError();
}

// Launch of a general-layout stage (affine lines, axis-table sides or a
// spectral pre-multiplier; fft_fast_general.cu): lines per tile A.B among
// fast_lines, 1/2 and 1/4 of it.
cudaError_t launch_fast_general(const StageArgs& A, bool dbl, bool inverse, bool afast, cudaStream_t st);
cudaError_t launch_real_general(const StageArgs& A, bool dbl, bool c2r, cudaStream_t st);

inline bool general_stage(const StageArgs& A) {
  return A.src_line_affine || A.dst_line_affine || A.src_atab || A.dst_atab || A.pre_mode;
}

}  // namespace dev
}  // namespace dfft
