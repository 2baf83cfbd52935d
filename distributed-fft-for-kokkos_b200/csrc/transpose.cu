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

// Hermitian weight of an R2C spectrum: every element whose index k along the
// R2C axis is an interior mode (k != 0 and 2k != n_real) is multiplied by f.
// Walks the global index space and addresses any layout through its tables.
template <typename C>
__global__ void hermitian_weight_kernel(const DevLayout L, C* data, int nd, int64_t e0, int64_t e1, int64_t e2,
                                        int64_t e3, int axis, int n_real, double f) {
  const int64_t total = e0 * e1 * e2 * e3;
  for (int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; t < total;
       t += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    int64_t r = t;
    int c[4];
    c[3] = static_cast<int>(r % e3);
    r /= e3;
    c[2] = static_cast<int>(r % e2);
    r /= e2;
    c[1] = static_cast<int>(r % e1);
    c[0] = static_cast<int>(r / e1);
    int k = c[0];
#pragma unroll
    for (int q = 1; q < 4; ++q)
      if (axis == q) k = c[q];
    if (k == 0 || 2 * k == n_real) continue;
    // logical coordinates of the nd-dimensional array sit in the last nd slots
    int cc[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) cc[q] = (q < nd) ? c[q + 4 - nd] : 0;
    C& v = data[layout_offset(L, cc, nd)];
    v.x *= f;
    v.y *= f;
  }
}

static unsigned grid_for(int64_t n, int threads);

cudaError_t launch_weight(const DevLayout& L, void* data, bool dbl, int nd, const int64_t* ext, int axis, int n_real,
                          double factor, cudaStream_t st) {
  int64_t e[4] = {1, 1, 1, 1};
  for (int q = 0; q < nd; ++q) e[4 - nd + q] = ext[q];
  const int a4 = axis + 4 - nd;
  const int64_t total = e[0] * e[1] * e[2] * e[3];
  const unsigned grid = grid_for(total, 256);
  if (dbl)
    hermitian_weight_kernel<double2><<<grid, 256, 0, st>>>(L, static_cast<double2*>(data), nd, e[0], e[1], e[2], e[3],
                                                            a4, n_real, factor);
  else
    hermitian_weight_kernel<float2><<<grid, 256, 0, st>>>(L, static_cast<float2*>(data), nd, e[0], e[1], e[2], e[3],
                                                           a4, n_real, factor);
  return cudaGetLastError();
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
