// Pack / all-to-all / unpack kernels over all virtual ranks at once, and the
// normalisation pass.  They reproduce the reference's TransBlock data flow
// (KokkosFFT_Distributed_TransBlock.hpp:76-107) buffer for buffer:
//   pack    KokkosFFT_Distributed_PackUnpack.hpp:85-251   (gather, zero fill)
//   all2all KokkosFFT_Distributed_MPI_All2All.hpp:23-58   (recv_r[j] = send_{g_j}[s(r)])
//   unpack  KokkosFFT_Distributed_PackUnpack.hpp:258-420  (scatter, skip padding)
// Instead of walking each rank's local view they address the global array
// through the layout tables, so the same kernels also materialise the
// reference's buffers from any other layout of the same data.
#include "fft_stage.cuh"

namespace dfft {
namespace dev {

// KokkosFFT_Distributed_PackUnpack.hpp:40-46
__device__ __forceinline__ void bin_map(int64_t n, int64_t nb, int64_t ib, int64_t& s, int64_t& l) {
  const int64_t base = n / nb, rem = n % nb;
  l = base + (ib < rem ? 1 : 0);
  s = ib * base + (ib < rem ? ib : rem);
}

// Decode a buffer linear index into (p, i[0..nd)) in logical axis order.
__device__ __forceinline__ void decode_buffer(const XposeArgs& X, int64_t e, int64_t& p, int64_t* i) {
  if (X.buf_right) {
#pragma unroll
    for (int k = 3; k >= 0; --k) {
      if (k < X.nd) {
        const int64_t ext = X.bext[k + 1];
        i[k] = e % ext;
        e /= ext;
      }
    }
  } else {
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      if (k < X.nd) {
        const int64_t ext = X.bext[k];
        i[k] = e % ext;
        e /= ext;
      }
    }
  }
  p = e;
}

// Global coordinate of buffer element (p, i) of rank r; false for padding.
// Along `axis` the index is merged with the bin of p (merge_indices,
// PackUnpack.hpp:62-73); along the other axes it must fall inside rank r's
// block.
__device__ __forceinline__ bool buffer_coord(const XposeArgs& X, int64_t r, int64_t p, const int64_t* i, int* c) {
  const int64_t* g = X.geo + r * X.rs;
  int64_t s, l;
  bin_map(X.merged, X.pc, p, s, l);
  bool ok = true;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    c[k] = 0;
    if (k < X.nd) {
      if (k == X.axis) {
        ok = ok && (i[k] < l);
        c[k] = static_cast<int>(s + i[k]);
      } else {
        ok = ok && (i[k] < g[4 + k]);
        c[k] = static_cast<int>(g[k] + i[k]);
      }
    }
  }
  return ok;
}

template <typename E>
__global__ void pack_kernel(const XposeArgs X) {
  const int64_t total = X.bufsize * X.nprocs;
  for (int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; t < total;
       t += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t r = t / X.bufsize, e = t - r * X.bufsize;
    int64_t p, i[4] = {0, 0, 0, 0};
    decode_buffer(X, e, p, i);
    int c[4];
    E v;
    memset(&v, 0, sizeof(E));
    if (buffer_coord(X, r, p, i, c)) v = reinterpret_cast<const E*>(X.src)[layout_offset(X.lay, c, X.nd)];
    reinterpret_cast<E*>(X.dst)[t] = v;
  }
}

template <typename E>
__global__ void unpack_kernel(const XposeArgs X) {
  const int64_t total = X.bufsize * X.nprocs;
  for (int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; t < total;
       t += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t r = t / X.bufsize, e = t - r * X.bufsize;
    int64_t p, i[4] = {0, 0, 0, 0};
    decode_buffer(X, e, p, i);
    int c[4];
    if (buffer_coord(X, r, p, i, c))
      reinterpret_cast<E*>(X.dst)[layout_offset(X.lay, c, X.nd)] = reinterpret_cast<const E*>(X.src)[t];
  }
}

// recv_r[j*cnt + q] = send_{g(r,j)}[s(r)*cnt + q]   (MPI_Alltoall over the group)
template <typename E>
__global__ void all2all_kernel(const XposeArgs X) {
  const int64_t total = X.bufsize * X.nprocs;
  const int64_t cnt = X.bufsize / X.pc;
  for (int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; t < total;
       t += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t r = t / X.bufsize, e = t - r * X.bufsize;
    const int64_t j = e / cnt, q = e - j * cnt;
    const int64_t src_rank = X.geo[r * X.rs + 9 + j];
    const int64_t s = X.geo[r * X.rs + 8];
    reinterpret_cast<E*>(X.dst)[t] = reinterpret_cast<const E*>(X.src)[src_rank * X.bufsize + s * cnt + q];
  }
}

template <typename T>
__global__ void scale_kernel(T* p, int64_t n, T s) {
  for (int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; t < n;
       t += static_cast<int64_t>(gridDim.x) * blockDim.x)
    p[t] *= s;
}

static unsigned grid_for(int64_t n, int threads) {
  int64_t g = (n + threads - 1) / threads;
  const int64_t cap = 148 * 32;
  if (g > cap) g = cap;
  if (g < 1) g = 1;
  return static_cast<unsigned>(g);
}

cudaError_t launch_xpose(int op, const XposeArgs& X, int elem_bytes, cudaStream_t st) {
  const int threads = 256;
  const unsigned grid = grid_for(X.bufsize * X.nprocs, threads);
  switch (op) {
    case 0:
      if (elem_bytes == 4) pack_kernel<float><<<grid, threads, 0, st>>>(X);
      else if (elem_bytes == 8) pack_kernel<float2><<<grid, threads, 0, st>>>(X);
      else pack_kernel<double2><<<grid, threads, 0, st>>>(X);
      break;
    case 1:
      if (elem_bytes == 4) all2all_kernel<float><<<grid, threads, 0, st>>>(X);
      else if (elem_bytes == 8) all2all_kernel<float2><<<grid, threads, 0, st>>>(X);
      else all2all_kernel<double2><<<grid, threads, 0, st>>>(X);
      break;
    case 2:
      if (elem_bytes == 4) unpack_kernel<float><<<grid, threads, 0, st>>>(X);
      else if (elem_bytes == 8) unpack_kernel<float2><<<grid, threads, 0, st>>>(X);
      else unpack_kernel<double2><<<grid, threads, 0, st>>>(X);
      break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t launch_scale(void* p, int64_t n_real, bool dbl, double s, cudaStream_t st) {
  const int threads = 256;
  const unsigned grid = grid_for(n_real, threads);
  if (dbl) scale_kernel<double><<<grid, threads, 0, st>>>(static_cast<double*>(p), n_real, s);
  else scale_kernel<float><<<grid, threads, 0, st>>>(static_cast<float*>(p), n_real, static_cast<float>(s));
  return cudaGetLastError();
}

}  // namespace dev
}  // namespace dfft
