// Batched register FFT stages (sm_100a): one persistent launch runs one stage
// of many fields of uneven sizes.
//
// A CTA of kBatchThreads threads walks work items blockIdx.x, +gridDim.x, ...
// of a table that concatenates the tiles of every field; for each item it
// finds the field (the item index only grows, so the field index only
// advances), decodes the tile (tb, co0, co1) of that field's stage and runs
// the tile body of the stage's line length with B = kBatchThreads / (N / V)
// lines, the same bodies as the one-tile-per-CTA kernels (fft_tile.cuh).
// The switch on the line length is uniform across the CTA.  Shared memory is
// sized for the largest tile of the launch and the twiddles are staged per
// tile; a barrier separates consecutive tiles.
#include <cstring>

#include "fft_tile.cuh"

namespace dfft {
namespace dev {

using namespace radix;

namespace {

constexpr int kBatchThreads = 256;

// resident CTAs per SM the register budget is sized for: three for complex64
// (85 registers, the budget of the one-tile 24-value kernels), one for
// complex128
template <typename T>
struct BatchMinBlocks {
  static constexpr int value = sizeof(T) == 4 ? 3 : 1;
};

template <int N>
struct BatchLines {
  static constexpr int value = kBatchThreads / (N / Vals<N>::value);
};

#define DFFT_BATCH_LENGTHS(X) \
  X(16) X(32) X(64) X(128) X(256) X(512) X(1024) X(2048) X(24) X(48) X(96) X(192) X(384) X(768)

__device__ __forceinline__ void decode(const StageArgs& A, long long local, int tiles_b, int* tb, int* co0, int* co1) {
  *tb = static_cast<int>(local % tiles_b);
  const long long rest = local / tiles_b;
  *co0 = static_cast<int>(rest % A.Eo0);
  *co1 = static_cast<int>(rest / A.Eo0);
}

template <typename T, bool INV, bool AFAST>
__global__ void __launch_bounds__(kBatchThreads, BatchMinBlocks<T>::value) fft_batch_c2c_kernel(const __grid_constant__ BatchParams P) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const long long total = P.prefix[P.nfields];
  int f = 0;
  for (long long w = blockIdx.x; w < total; w += gridDim.x) {
    while (w >= P.prefix[f + 1]) ++f;
    const StageArgs& A = P.f[f];
    int tb, co0, co1;
    decode(A, w - P.prefix[f], A.tiles_b, &tb, &co0, &co1);
    switch (A.n) {
#define DFFT_TILE(N_) \
  case N_: fast_tile<T, INV, N_, BatchLines<N_>::value, AFAST, true>(A, tb, co0, co1, smem_raw); break;
      DFFT_BATCH_LENGTHS(DFFT_TILE)
#undef DFFT_TILE
      default: break;
    }
    __syncthreads();  // the next tile restages twiddles and lines
  }
}

template <typename T, bool C2R>
__global__ void __launch_bounds__(kBatchThreads, BatchMinBlocks<T>::value) fft_batch_real_kernel(const __grid_constant__ BatchParams P) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const long long total = P.prefix[P.nfields];
  int f = 0;
  for (long long w = blockIdx.x; w < total; w += gridDim.x) {
    while (w >= P.prefix[f + 1]) ++f;
    const StageArgs& A = P.f[f];
    int tb, co0, co1;
    decode(A, w - P.prefix[f], A.tiles_b, &tb, &co0, &co1);
    switch (A.n) {
#define DFFT_TILE(N_) \
  case N_: real_tile<T, C2R, N_, BatchLines<N_>::value, true>(A, tb, co0, co1, smem_raw); break;
      DFFT_BATCH_LENGTHS(DFFT_TILE)
#undef DFFT_TILE
      default: break;
    }
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

template <typename T>
cudaError_t launch_batch_t(BatchParams& P, int kind, bool inverse, bool afast, cudaStream_t st) {
  size_t smem = 0;
  for (int i = 0; i < P.nfields; ++i) {
    const size_t b = tile_smem<T>(P.f[i].n, kind == kC2C ? afast : true);
    if (b == 0) return cudaErrorInvalidValue;
    if (b > smem) smem = b;
    P.f[i] = with_table_offsets(P.f[i]);
  }
  if (kind == kC2C) {
    if (inverse)
      return afast ? launch_persistent(fft_batch_c2c_kernel<T, true, true>, P, smem, st)
                   : launch_persistent(fft_batch_c2c_kernel<T, true, false>, P, smem, st);
    return afast ? launch_persistent(fft_batch_c2c_kernel<T, false, true>, P, smem, st)
                 : launch_persistent(fft_batch_c2c_kernel<T, false, false>, P, smem, st);
  }
  if (kind == kR2C) return launch_persistent(fft_batch_real_kernel<T, false>, P, smem, st);
  if (kind == kC2R) return launch_persistent(fft_batch_real_kernel<T, true>, P, smem, st);
  return cudaErrorInvalidValue;
}

}  // namespace

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
  return dbl ? launch_batch_t<double>(P, kind, inverse, afast, st) : launch_batch_t<float>(P, kind, inverse, afast, st);
}

}  // namespace dev
}  // namespace dfft
