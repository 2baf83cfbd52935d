// Chirp-z (Bluestein) stage kernels: the gather / chirp, filter and chirp /
// scatter steps around two m-point FFTs (see BlueArgs in dev_types.h); the
// same gather / scatter (without chirp) and a twiddle step serve the
// four-step stages of lines too long for one stage.  The FFTs themselves are
// ordinary register or generic stages on a plain (lines, m) array.
// These kernels address the rank-blocked layouts element by element through
// the layout tables: the path serves line lengths the radix passes cannot
// (a prime factor above 13), not the hot shapes.
#include "fft_stage.cuh"

namespace dfft {
namespace dev {
namespace {

template <typename T>
__device__ __forceinline__ cplx<T> chirp_at(const BlueArgs& B, int j) {
  if (B.four_n1 > 0) return mk<T>(T(1), T(0));  // four-step: plain copy
  cplx<T> c = reinterpret_cast<const cplx<T>*>(B.chirp)[j];
  if (B.inverse) c.y = -c.y;
  return c;
}

__device__ __forceinline__ void line_coords(const StageArgs& S, long long line, int* c) {
  c[0] = c[1] = c[2] = c[3] = 0;
  const int ib = static_cast<int>(line % S.Eb);
  const long long rest = line / S.Eb;
  c[S.b] = ib;
  if (S.o0 >= 0) c[S.o0] = static_cast<int>(rest % S.Eo0);
  if (S.o1 >= 0) c[S.o1] = static_cast<int>(rest / S.Eo0);
}

template <typename T>
__global__ void blue_pre_kernel(const BlueArgs B) {
  using C = cplx<T>;
  const StageArgs& S = B.S;
  const int n = S.n, m = B.m;
  const long long total = B.nlines * m;
  C* z = reinterpret_cast<C*>(B.zout);
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<long long>(gridDim.x) * blockDim.x) {
    const long long line = i / m;
    const int j = static_cast<int>(i % m);
    C v = mk<T>(T(0), T(0));
    if (j < n) {
      int c[4];
      line_coords(S, line, c);
      if (B.kind == kR2C) {
        c[S.a] = j;
        v = mk<T>(reinterpret_cast<const T*>(S.in)[layout_offset(S.src, c, S.nd)], T(0));
      } else if (B.kind == kC2R) {
        // full line from the half spectrum: x_j = X_j (j <= n/2), conj X_{n-j}
        const bool mirror = 2 * j > n;
        c[S.a] = mirror ? n - j : j;
        v = reinterpret_cast<const C*>(S.in)[layout_offset(S.src, c, S.nd)];
        if (mirror) v.y = -v.y;
        if (j == 0 || 2 * j == n) v.y = T(0);
      } else {
        c[S.a] = j;
        v = reinterpret_cast<const C*>(S.in)[layout_offset(S.src, c, S.nd)];
      }
      v = cmul(v, chirp_at<T>(B, j));
    }
    z[i] = v;
  }
}

template <typename T>
__global__ void blue_mul_kernel(const BlueArgs B) {
  using C = cplx<T>;
  const long long total = B.nlines * B.m;
  C* z = reinterpret_cast<C*>(B.zout);
  const C* f = reinterpret_cast<const C*>(B.filter);
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<long long>(gridDim.x) * blockDim.x)
    z[i] = cmul(z[i], f[i % B.m]);
}

// four-step twiddle: z[line][k2][j1] *= w_n^(j1 k2)
template <typename T>
__global__ void four_twiddle_kernel(const BlueArgs B) {
  using C = cplx<T>;
  const int n = B.S.n, n1 = B.four_n1;
  const long long total = B.nlines * n;
  C* z = reinterpret_cast<C*>(B.zout);
  const C* tw = reinterpret_cast<const C*>(B.tw);
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int p = static_cast<int>(i % n);
    const long long j1 = p % n1, k2 = p / n1;
    C w = tw[(j1 * k2) % n];
    if (B.inverse) w.y = -w.y;
    z[i] = cmul(z[i], w);
  }
}

template <typename T>
__global__ void blue_post_kernel(const BlueArgs B) {
  using C = cplx<T>;
  const StageArgs& S = B.S;
  const int n = S.n, m = B.m;
  const int nout = B.kind == kR2C ? n / 2 + 1 : n;
  const long long total = B.nlines * nout;
  const C* z = reinterpret_cast<const C*>(B.zin);
  const T sc = T(S.scale);
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<long long>(gridDim.x) * blockDim.x) {
    const long long line = i / nout;
    const int k = static_cast<int>(i % nout);
    const long long src = B.four_n1 > 0 ? (k % B.four_n2) * static_cast<long long>(B.four_n1) + k / B.four_n2 : k;
    const C v = cscale(cmul(z[line * m + src], chirp_at<T>(B, k)), sc);
    int c[4];
    line_coords(S, line, c);
    c[S.a] = k;
    const int64_t o = layout_offset(S.dst, c, S.nd);
    if (B.kind == kC2R)
      reinterpret_cast<T*>(S.out)[o] = v.x;
    else
      reinterpret_cast<C*>(S.out)[o] = v;
  }
}

unsigned grid_for(long long n) {
  long long g = (n + 255) / 256;
  if (g > 148 * 32) g = 148 * 32;
  return static_cast<unsigned>(g < 1 ? 1 : g);
}

template <typename T>
cudaError_t launch_t(int op, const BlueArgs& B, cudaStream_t st) {
  const int n = B.S.n;
  const long long work = op == 2 ? B.nlines * (B.kind == kR2C ? n / 2 + 1 : n) : B.nlines * B.m;
  if (work <= 0) return cudaSuccess;
  if (op == 0)
    blue_pre_kernel<T><<<grid_for(work), 256, 0, st>>>(B);
  else if (op == 1)
    blue_mul_kernel<T><<<grid_for(work), 256, 0, st>>>(B);
  else if (op == 2)
    blue_post_kernel<T><<<grid_for(work), 256, 0, st>>>(B);
  else
    four_twiddle_kernel<T><<<grid_for(work), 256, 0, st>>>(B);
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_bluestein(int op, const BlueArgs& B, bool dbl, cudaStream_t st) {
  if (op < 0 || op > 3) return cudaErrorInvalidValue;
  return dbl ? launch_t<double>(op, B, st) : launch_t<float>(op, B, st);
}

}  // namespace dev
}  // namespace dfft
