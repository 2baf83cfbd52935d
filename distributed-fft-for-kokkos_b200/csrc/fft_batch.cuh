// Kernels of the batched register stages (see fft_batch.cu): the tile bodies
// of fft_tile.cuh behind a persistent work-table loop.  Instantiated for
// general-layout sides (AFF, fft_batch.cu) and separable sides only
// (fft_batch_sep.cu, fewer registers) in two translation units.
#pragma once

#include <cstring>

#include "fft_tile.cuh"

namespace dfft {
namespace dev {
namespace batch {

using namespace radix;


constexpr int kBatchThreads = 256;

// A launch covers the lengths of one value class VC (8 values a thread:
// powers of two; 24: 3 * 2^k), so each kernel's register budget is its own
// class's: resident CTAs per SM for complex64 4 (64 registers) for 8-value
// tiles and 3 (85 registers, the budget of the one-tile 24-value kernels)
// for 24-value tiles; for complex128 2 and 1.
template <typename T, int VC>
struct BatchMinBlocks {
  static constexpr int value = sizeof(T) == 4 ? (VC == 8 ? 4 : 3) : (VC == 8 ? 2 : 1);
};

template <int N>
struct BatchLines {
  static constexpr int value = kBatchThreads / (N / Vals<N>::value);
};

#define DFFT_BATCH_LENGTHS8(X) X(16) X(32) X(64) X(128) X(256) X(512) X(1024) X(2048)
#define DFFT_BATCH_LENGTHS24(X) X(24) X(48) X(96) X(192) X(384) X(768)
#define DFFT_BATCH_LENGTHS(X) DFFT_BATCH_LENGTHS8(X) DFFT_BATCH_LENGTHS24(X)

// tile (tb, co0, co1) of a field's stage from its local work index (32-bit:
// the host keeps every field's tile count below 2^31)
__device__ __forceinline__ void decode(const StageArgs& A, unsigned local, int* tb, int* co0, int* co1) {
  const unsigned tbs = static_cast<unsigned>(A.tiles_b);
  *tb = static_cast<int>(local % tbs);
  const unsigned rest = local / tbs;
  *co0 = static_cast<int>(rest % static_cast<unsigned>(A.Eo0));
  *co1 = static_cast<int>(rest / static_cast<unsigned>(A.Eo0));
}

template <typename T, bool INV, bool AFAST, bool AFF, int VC>
__global__ void __launch_bounds__(kBatchThreads, (BatchMinBlocks<T, VC>::value)) fft_batch_c2c_kernel(const __grid_constant__ BatchParams P) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const long long total = P.prefix[P.nfields];
  int f = 0, cur_n = 0;
  for (long long w = blockIdx.x; w < total; w += gridDim.x) {
    while (w >= P.prefix[f + 1]) ++f;
    const StageArgs& A = P.f[f];
    int tb, co0, co1;
    decode(A, static_cast<unsigned>(w - P.prefix[f]), &tb, &co0, &co1);
    const bool stage_tw = A.n != cur_n;
    cur_n = A.n;
#define DFFT_TILE(N_) \
  case N_: fast_tile<T, INV, N_, BatchLines<N_>::value, AFAST, AFF>(A, tb, co0, co1, smem_raw, stage_tw); break;
    if constexpr (VC == 8) {
      switch (A.n) { DFFT_BATCH_LENGTHS8(DFFT_TILE) default: break; }
    } else {
      switch (A.n) { DFFT_BATCH_LENGTHS24(DFFT_TILE) default: break; }
    }
#undef DFFT_TILE
    __syncthreads();  // the next tile restages twiddles and lines
  }
}

template <typename T, bool C2R, bool AFF, int VC>
__global__ void __launch_bounds__(kBatchThreads, (BatchMinBlocks<T, VC>::value)) fft_batch_real_kernel(const __grid_constant__ BatchParams P) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const long long total = P.prefix[P.nfields];
  int f = 0, cur_n = 0;
  for (long long w = blockIdx.x; w < total; w += gridDim.x) {
    while (w >= P.prefix[f + 1]) ++f;
    const StageArgs& A = P.f[f];
    int tb, co0, co1;
    decode(A, static_cast<unsigned>(w - P.prefix[f]), &tb, &co0, &co1);
    const bool stage_tw = A.n != cur_n;
    cur_n = A.n;
#define DFFT_TILE(N_) \
  case N_: real_tile<T, C2R, N_, BatchLines<N_>::value, AFF>(A, tb, co0, co1, smem_raw, stage_tw); break;
    if constexpr (VC == 8) {
      switch (A.n) { DFFT_BATCH_LENGTHS8(DFFT_TILE) default: break; }
    } else {
      switch (A.n) { DFFT_BATCH_LENGTHS24(DFFT_TILE) default: break; }
    }
#undef DFFT_TILE
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

template <typename K>
cudaError_t launch_persistent(K kernel, BatchParams& P, size_t smem, cudaStream_t st) {
  cudaError_t e = raise_smem_limit(reinterpret_cast<const void*>(kernel), smem);
  if (e != cudaSuccess) return e;
  int dev = 0, sms = 0, per_sm = 0;
  if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
  if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
  if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kBatchThreads, smem)) != cudaSuccess)
    return e;
  long long grid = static_cast<long long>(sms) * (per_sm > 0 ? per_sm : 1);
  const long long total = P.prefix[P.nfields];
  if (grid > total) grid = total;
  if (grid < 1) return cudaSuccess;
  kernel<<<static_cast<unsigned>(grid), kBatchThreads, smem, st>>>(P);
  return cudaGetLastError();
}

template <typename T, bool AFF, int VC>
cudaError_t launch_batch_vc(BatchParams& P, size_t smem, int kind, bool inverse, bool afast, cudaStream_t st) {
  if (kind == kC2C) {
    if (inverse)
      return afast ? launch_persistent(fft_batch_c2c_kernel<T, true, true, AFF, VC>, P, smem, st)
                   : launch_persistent(fft_batch_c2c_kernel<T, true, false, AFF, VC>, P, smem, st);
    return afast ? launch_persistent(fft_batch_c2c_kernel<T, false, true, AFF, VC>, P, smem, st)
                 : launch_persistent(fft_batch_c2c_kernel<T, false, false, AFF, VC>, P, smem, st);
  }
  if (kind == kR2C) return launch_persistent(fft_batch_real_kernel<T, false, AFF, VC>, P, smem, st);
  if (kind == kC2R) return launch_persistent(fft_batch_real_kernel<T, true, AFF, VC>, P, smem, st);
  return cudaErrorInvalidValue;
}

// every field of P has line lengths of one value class (the host groups them)
template <typename T, bool AFF>
cudaError_t launch_batch_t(BatchParams& P, int kind, bool inverse, bool afast, cudaStream_t st) {
  size_t smem = 0;
  const bool v24 = P.f[0].n % 3 == 0;
  for (int i = 0; i < P.nfields; ++i) {
    const size_t b = tile_smem<T>(P.f[i].n, kind == kC2C ? afast : true);
    if (b == 0 || (P.f[i].n % 3 == 0) != v24) return cudaErrorInvalidValue;
    if (b > smem) smem = b;
    P.f[i] = with_table_offsets(P.f[i]);
  }
  return v24 ? launch_batch_vc<T, AFF, 24>(P, smem, kind, inverse, afast, st)
             : launch_batch_vc<T, AFF, 8>(P, smem, kind, inverse, afast, st);
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
