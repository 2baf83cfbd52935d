// Kernels of the batched register stages (see fft_batch.cu): the tile bodies
// of fft_tile.cuh behind a persistent work-table loop.  Instantiated for
// general-layout sides (AFF, fft_batch.cu) and separable sides only
// (fft_batch_sep.cu, fewer registers) in two translation units.
#pragma once

#include <cstring>

#include "fft_pair.cuh"
#include "fft_tile.cuh"

namespace dfft {
namespace dev {
namespace batch {

using namespace radix;


constexpr int kBatchThreads = 256;

// A launch covers the fields of one line length N, so each kernel carries one
// tile body at a register budget of its own: resident threads per SM for
// 8-value bodies 1536 complex64 / 768 complex128, for 24-value bodies 512 /
// 256 (one step below the one-tile kernels of fft_fast.cu, which leaves the
// work-table loop its registers without spilling); the general-layout
// 8-value variant keeps the compiler's choice.
template <typename T, int N, bool AFAST, bool AFF>
struct BatchMinBlocks {
  static constexpr bool v8 = Vals<N>::value == 8;
  static constexpr int target = v8 ? (sizeof(T) == 4 ? 1536 : 768) : (sizeof(T) == 4 ? 512 : 256);
  static constexpr int v = target / kBatchThreads;
  static constexpr int value = (!(v8 && AFF) && v > 0) ? v : 1;
};

template <int N>
struct BatchLines {
  static constexpr int value = kBatchThreads / (N / Vals<N>::value);
};

#define DFFT_BATCH_LENGTHS(X) \
  X(16) X(32) X(64) X(128) X(256) X(512) X(1024) X(2048) X(24) X(48) X(96) X(192) X(384) X(768)

// tile (tb, co0, co1) of a field's stage from its local work index (32-bit:
// the host keeps every field's tile count below 2^31)
__device__ __forceinline__ void decode(const StageArgs& A, unsigned local, int* tb, int* co0, int* co1) {
  const unsigned tbs = static_cast<unsigned>(A.tiles_b);
  *tb = static_cast<int>(local % tbs);
  const unsigned rest = local / tbs;
  *co0 = static_cast<int>(rest % static_cast<unsigned>(A.Eo0));
  *co1 = static_cast<int>(rest / static_cast<unsigned>(A.Eo0));
}

template <typename T, bool INV, bool AFAST, bool AFF, int N>
__global__ void __launch_bounds__(kBatchThreads, (BatchMinBlocks<T, N, AFAST, AFF>::value))
    fft_batch_c2c_kernel(const __grid_constant__ BatchParams P) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const long long total = P.prefix[P.nfields];
  int f = 0;
  bool first = true;  // the twiddles of N are staged by the CTA's first tile
  for (long long w = blockIdx.x; w < total; w += gridDim.x) {
    while (w >= P.prefix[f + 1]) ++f;
    const StageArgs& A = P.f[f];
    int tb, co0, co1;
    decode(A, static_cast<unsigned>(w - P.prefix[f]), &tb, &co0, &co1);
    fast_tile<T, INV, N, BatchLines<N>::value, AFAST, AFF>(A, tb, co0, co1, smem_raw, first);
    first = false;
    __syncthreads();  // the next tile restages its lines
  }
}

template <typename T, bool C2R, bool AFF, int N>
__global__ void __launch_bounds__(kBatchThreads, (BatchMinBlocks<T, N, true, AFF>::value))
    fft_batch_real_kernel(const __grid_constant__ BatchParams P) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const long long total = P.prefix[P.nfields];
  int f = 0;
  bool first = true;
  for (long long w = blockIdx.x; w < total; w += gridDim.x) {
    while (w >= P.prefix[f + 1]) ++f;
    const StageArgs& A = P.f[f];
    int tb, co0, co1;
    decode(A, static_cast<unsigned>(w - P.prefix[f]), &tb, &co0, &co1);
    real_tile<T, C2R, N, BatchLines<N>::value, AFF>(A, tb, co0, co1, smem_raw, first);
    first = false;
    __syncthreads();
  }
}

// Two-line (complex64, separable, 2^k points) batched C2C stage: the tile
// body of fft_pair_kernel with its default pairs per tile, N/8 threads per
// pair, at that kernel's register budget (1024 resident threads per SM).
template <int N, bool AFAST>
struct BatchPairs {
  static constexpr int value = pair_option(N, AFAST, 0);
  static constexpr int threads = N / 8 * value;
  static constexpr int min_blocks = 1024 / threads > 0 ? 1024 / threads : 1;
};

template <bool INV, bool AFAST, int N>
__global__ void __launch_bounds__(BatchPairs<N, AFAST>::threads, (BatchPairs<N, AFAST>::min_blocks))
    fft_batch_pair_kernel(const __grid_constant__ BatchParams P) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const long long total = P.prefix[P.nfields];
  int f = 0;
  bool first = true;
  for (long long w = blockIdx.x; w < total; w += gridDim.x) {
    while (w >= P.prefix[f + 1]) ++f;
    const StageArgs& A = P.f[f];
    int tb, co0, co1;
    decode(A, static_cast<unsigned>(w - P.prefix[f]), &tb, &co0, &co1);
    pair_tile<INV, N, BatchPairs<N, AFAST>::value, AFAST>(A, tb, co0, co1, smem_raw, first);
    first = false;
    __syncthreads();
  }
}

template <typename T>
size_t tile_smem(int n, bool afast) {
  switch (n) {
#define DFFT_SMEM(N_)                                                                                        \
  case N_:                                                                                                   \
    return sizeof(cplx<T>) * (N_ + static_cast<size_t>(BatchLines<N_>::value) *                              \
                                       (afast ? SmemShape<T, N_, BatchLines<N_>::value, true>::LP         \
                                              : SmemShape<T, N_, BatchLines<N_>::value, false>::LP));
    DFFT_BATCH_LENGTHS(DFFT_SMEM)
#undef DFFT_SMEM
    default: return 0;
  }
}

template <int THREADS = kBatchThreads, typename K>
cudaError_t launch_persistent(K kernel, BatchParams& P, size_t smem, cudaStream_t st) {
  cudaError_t e = raise_smem_limit(reinterpret_cast<const void*>(kernel), smem);
  if (e != cudaSuccess) return e;
  int dev = 0, sms = 0, per_sm = 0;
  if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
  if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
  if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, THREADS, smem)) != cudaSuccess)
    return e;
  long long grid = static_cast<long long>(sms) * (per_sm > 0 ? per_sm : 1);
  const long long total = P.prefix[P.nfields];
  if (grid > total) grid = total;
  if (grid < 1) return cudaSuccess;
  kernel<<<static_cast<unsigned>(grid), THREADS, smem, st>>>(P);
  return cudaGetLastError();
}

template <bool INV, bool AFAST, int N>
cudaError_t launch_batch_pair_n(BatchParams& P, cudaStream_t st) {
  constexpr size_t smem = pair_tile_smem<N, BatchPairs<N, AFAST>::value, AFAST>();
  for (int i = 0; i < P.nfields; ++i) P.f[i] = with_table_offsets(P.f[i]);
  return launch_persistent<BatchPairs<N, AFAST>::threads>(fft_batch_pair_kernel<INV, AFAST, N>, P, smem, st);
}

template <typename T, bool AFF, int N>
cudaError_t launch_batch_n(BatchParams& P, size_t smem, int kind, bool inverse, bool afast, cudaStream_t st) {
  if (kind == kC2C) {
    if (inverse)
      return afast ? launch_persistent(fft_batch_c2c_kernel<T, true, true, AFF, N>, P, smem, st)
                   : launch_persistent(fft_batch_c2c_kernel<T, true, false, AFF, N>, P, smem, st);
    return afast ? launch_persistent(fft_batch_c2c_kernel<T, false, true, AFF, N>, P, smem, st)
                 : launch_persistent(fft_batch_c2c_kernel<T, false, false, AFF, N>, P, smem, st);
  }
  if (kind == kR2C) return launch_persistent(fft_batch_real_kernel<T, false, AFF, N>, P, smem, st);
  if (kind == kC2R) return launch_persistent(fft_batch_real_kernel<T, true, AFF, N>, P, smem, st);
  return cudaErrorInvalidValue;
}

// every field of P has the same line length (the host groups them)
template <typename T, bool AFF>
cudaError_t launch_batch_t(BatchParams& P, int kind, bool inverse, bool afast, cudaStream_t st) {
  const int n = P.f[0].n;
  const size_t smem = tile_smem<T>(n, kind == kC2C ? afast : true);
  if (smem == 0) return cudaErrorInvalidValue;
  for (int i = 0; i < P.nfields; ++i) {
    if (P.f[i].n != n) return cudaErrorInvalidValue;
    P.f[i] = with_table_offsets(P.f[i]);
  }
  switch (n) {
#define DFFT_LAUNCH(N_) \
  case N_: return launch_batch_n<T, AFF, N_>(P, smem, kind, inverse, afast, st);
    DFFT_BATCH_LENGTHS(DFFT_LAUNCH)
#undef DFFT_LAUNCH
    default: return cudaErrorInvalidValue;
  }
}

// the launcher of one addressing variant (AFF: general-layout sides),
// defined in fft_batch.cu (AFF = true) and fft_batch_sep.cu (AFF = false)
template <bool AFF>
cudaError_t launch_batch_variant(BatchParams& P, bool dbl, int kind, bool inverse, bool afast, cudaStream_t st);
template <>
cudaError_t launch_batch_variant<true>(BatchParams& P, bool dbl, int kind, bool inverse, bool afast, cudaStream_t st);
template <>
cudaError_t launch_batch_variant<false>(BatchParams& P, bool dbl, int kind, bool inverse, bool afast, cudaStream_t st);

}  // namespace batch
}  // namespace dev
}  // namespace dfft
