// Per-axis FFT stage kernel (sm_100a).
//
// One CTA owns a tile of B lines of the global FFT index space: the lines run
// along the FFT axis `a` and are adjacent along the tile axis `b` (chosen on
// the host as the unit-stride axis of the destination, or of the source).
//   1. gather:  tile <- source layout, table-driven.  This is where the
//               reference's unpack and the all-to-all of the preceding
//               transpose block land.  R2C packs two real lines into one
//               complex line; C2R rebuilds the full Hermitian spectrum.
//   2. Stockham autosort mixed-radix passes (radices 2,3,4,5,7,8,11,13) that
//      ping-pong between two shared-memory buffers.
//   3. scatter: tile -> destination layout with the normalisation folded in
//               (this is where the reference's pack lands).
// Twiddles come from a host table (long double, rounded to the stage
// precision) staged in shared memory.
#include <map>
#include <mutex>

#include "fft_stage.cuh"

namespace dfft {
namespace dev {

// ---------------------------------------------------------------------------
// Radix-R DFTs on registers.  Forward: X_q = sum_r v_r exp(-2 pi i r q / R).
// ---------------------------------------------------------------------------
template <bool INV, typename C>
__device__ __forceinline__ void dft4(C& v0, C& v1, C& v2, C& v3) {
  C s02 = cadd(v0, v2), d02 = csub(v0, v2);
  C s13 = cadd(v1, v3), d13 = rot<INV>(csub(v1, v3));
  v0 = cadd(s02, s13);
  v2 = csub(s02, s13);
  v1 = cadd(d02, d13);
  v3 = csub(d02, d13);
}

template <typename T, bool INV>
__device__ __forceinline__ void dft8(cplx<T>* v) {
  using C = cplx<T>;
  const T h = T(0.70710678118654752440084436210484903928);  // sqrt(1/2)
  C e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
  C o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
  dft4<INV>(e0, e1, e2, e3);
  dft4<INV>(o0, o1, o2, o3);
  // w^1 o1, w^2 o2, w^3 o3 with w = exp(-/+ i pi / 4)
  C t1, t3;
  if (INV) {
    t1 = mk<T>(h * (o1.x - o1.y), h * (o1.x + o1.y));
    t3 = mk<T>(-h * (o3.x + o3.y), h * (o3.x - o3.y));
  } else {
    t1 = mk<T>(h * (o1.x + o1.y), h * (o1.y - o1.x));
    t3 = mk<T>(h * (o3.y - o3.x), -h * (o3.x + o3.y));
  }
  C t2 = rot<INV>(o2);
  v[0] = cadd(e0, o0);
  v[4] = csub(e0, o0);
  v[1] = cadd(e1, t1);
  v[5] = csub(e1, t1);
  v[2] = cadd(e2, t2);
  v[6] = csub(e2, t2);
  v[3] = cadd(e3, t3);
  v[7] = csub(e3, t3);
}

template <typename T, bool INV>
__device__ __forceinline__ void dft3(cplx<T>* v) {
  using C = cplx<T>;
  const T c3 = T(0.86602540378443864676372317075293618347);  // sqrt(3)/2
  C t = cadd(v[1], v[2]);
  C d = rot<INV>(cscale(csub(v[1], v[2]), c3));
  C m = csub(v[0], cscale(t, T(0.5)));
  v[0] = cadd(v[0], t);
  v[1] = cadd(m, d);
  v[2] = csub(m, d);
}

template <typename T, bool INV>
__device__ __forceinline__ void dft5(cplx<T>* v) {
  using C = cplx<T>;
  // cos(2pi/5) = (sqrt5-1)/4, cos(4pi/5) = -(sqrt5+1)/4,
  // sin(2pi/5) = sqrt((5+sqrt5)/8), sin(4pi/5) = sqrt((5-sqrt5)/8)
  const T c1 = T(0.30901699437494742410229341718281905886);
  const T c2 = T(-0.80901699437494742410229341718281905886);
  const T s1 = T(0.95105651629515357211643933337938214340);
  const T s2 = T(0.58778525229247312916870595463907276860);
  C t1 = cadd(v[1], v[4]), t2 = cadd(v[2], v[3]);
  C d1 = csub(v[1], v[4]), d2 = csub(v[2], v[3]);
  C a1 = cadd(v[0], cadd(cscale(t1, c1), cscale(t2, c2)));
  C a2 = cadd(v[0], cadd(cscale(t1, c2), cscale(t2, c1)));
  C b1 = rot<INV>(cadd(cscale(d1, s1), cscale(d2, s2)));
  C b2 = rot<INV>(csub(cscale(d1, s2), cscale(d2, s1)));
  v[0] = cadd(v[0], cadd(t1, t2));
  v[1] = cadd(a1, b1);
  v[4] = csub(a1, b1);
  v[2] = cadd(a2, b2);
  v[3] = csub(a2, b2);
}

// Odd radix R: pairwise form; cos and sin of 2 pi m / R are read from the
// stage twiddle table (tw[m * n / R] = exp(-2 pi i m / R)).
template <typename T, bool INV, int R>
__device__ __forceinline__ void dft_odd(cplx<T>* v, const cplx<T>* tw, int n) {
  using C = cplx<T>;
  constexpr int H = (R - 1) / 2;
  C t[H], d[H];
#pragma unroll
  for (int m = 1; m <= H; ++m) {
    t[m - 1] = cadd(v[m], v[R - m]);
    d[m - 1] = csub(v[m], v[R - m]);
  }
  const int step = n / R;
  C out[R];
  C s0 = v[0];
#pragma unroll
  for (int m = 0; m < H; ++m) s0 = cadd(s0, t[m]);
  out[0] = s0;
#pragma unroll
  for (int q = 1; q <= H; ++q) {
    C re = v[0];
    C im = mk<T>(T(0), T(0));
#pragma unroll
    for (int m = 1; m <= H; ++m) {
      const int e = (m * q) % R;
      const C w = tw[e * step];  // (cos, -sin) of 2 pi e / R
      re = cadd(re, cscale(t[m - 1], w.x));
      im = cadd(im, cscale(d[m - 1], -w.y));
    }
    const C r = rot<INV>(im);
    out[q] = cadd(re, r);
    out[R - q] = csub(re, r);
  }
#pragma unroll
  for (int q = 0; q < R; ++q) v[q] = out[q];
}

template <typename T, bool INV, int R>
__device__ __forceinline__ void dft(cplx<T>* v, const cplx<T>* tw, int n) {
  if constexpr (R == 2) {
    const cplx<T> t = v[0];
    v[0] = cadd(t, v[1]);
    v[1] = csub(t, v[1]);
  } else if constexpr (R == 3) {
    dft3<T, INV>(v);
  } else if constexpr (R == 4) {
    dft4<INV>(v[0], v[1], v[2], v[3]);
  } else if constexpr (R == 5) {
    dft5<T, INV>(v);
  } else if constexpr (R == 8) {
    dft8<T, INV>(v);
  } else {
    dft_odd<T, INV, R>(v, tw, n);
  }
}

// One Stockham pass of radix R over `nl` lines of length n (line pitch
// `pitch`), reading `src` and writing `dst`.  Ns is the product of the radices
// of the previous passes.
template <typename T, bool INV, int R>
__device__ __forceinline__ void stockham_pass(const cplx<T>* __restrict__ src, cplx<T>* __restrict__ dst, int pitch,
                                              int nl, int n, int Ns, const cplx<T>* tw) {
  using C = cplx<T>;
  const int m = n / R;
  const int total = nl * m;
  const int tstride = n / (Ns * R);
  for (int bf = threadIdx.x; bf < total; bf += blockDim.x) {
    const int line = bf / m, j = bf - line * m;
    const int k = j % Ns;
    const C* s = src + line * pitch + j;
    C v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = s[r * m];
    if (Ns > 1) {
#pragma unroll
      for (int r = 1; r < R; ++r) {
        C w = tw[k * r * tstride];
        if (INV) w.y = -w.y;
        v[r] = cmul(v[r], w);
      }
    }
    dft<T, INV, R>(v, tw, n);
    C* d = dst + line * pitch + (j - k) * R + k;
#pragma unroll
    for (int r = 0; r < R; ++r) d[r * Ns] = v[r];
  }
}

template <typename T, bool INV>
__device__ __forceinline__ void run_pass(int R, const cplx<T>* src, cplx<T>* dst, int pitch, int nl, int n, int Ns,
                                         const cplx<T>* tw) {
  switch (R) {
    case 2: stockham_pass<T, INV, 2>(src, dst, pitch, nl, n, Ns, tw); break;
    case 3: stockham_pass<T, INV, 3>(src, dst, pitch, nl, n, Ns, tw); break;
    case 4: stockham_pass<T, INV, 4>(src, dst, pitch, nl, n, Ns, tw); break;
    case 5: stockham_pass<T, INV, 5>(src, dst, pitch, nl, n, Ns, tw); break;
    case 7: stockham_pass<T, INV, 7>(src, dst, pitch, nl, n, Ns, tw); break;
    case 8: stockham_pass<T, INV, 8>(src, dst, pitch, nl, n, Ns, tw); break;
    case 11: stockham_pass<T, INV, 11>(src, dst, pitch, nl, n, Ns, tw); break;
    case 13: stockham_pass<T, INV, 13>(src, dst, pitch, nl, n, Ns, tw); break;
    default: break;  // rejected on the host
  }
}

// Coordinates of (pos along a, line along b) in the current tile.
__device__ __forceinline__ void tile_coord(int* c, const int* cbase, int a, int pos, int b, int lb) {
#pragma unroll
  for (int k = 0; k < 4; ++k) c[k] = (k == a) ? pos : ((k == b) ? lb : cbase[k]);
}

template <typename T, int KIND, bool INV>
__global__ void __launch_bounds__(256) fft_stage_kernel(const StageArgs A) {
  using C = cplx<T>;
  const DevLayout lsrc = A.src, ldst = A.dst;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* tw = reinterpret_cast<C*>(smem_raw);
  C* buf0 = tw + ((A.n + 1) & ~1);
  C* buf1 = buf0 + A.nl * A.pitch;

  // Which tile: (tb, o0, o1)
  int t = blockIdx.x;
  const int tb = t % A.tiles_b;
  t /= A.tiles_b;
  int co0 = 0, co1 = 0;
  if (A.o0 >= 0) {
    co0 = t % A.Eo0;
    t /= A.Eo0;
  }
  if (A.o1 >= 0) co1 = t;
  const int b0 = tb * A.B;
  const int nb = min(A.B, A.Eb - b0);
  const int nt = blockDim.x;
  int cbase[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) cbase[k] = (k == A.o0) ? co0 : ((k == A.o1) ? co1 : 0);

  if (KIND != kCopy && KIND != kCopyReal) {
    const C* gtw = reinterpret_cast<const C*>(A.tw);
    for (int i = threadIdx.x; i < A.n; i += nt) tw[i] = gtw[i];
  }

  // ---------------- gather ----------------
  {
    const int na = A.na_in;
    const int Bl = (KIND == kR2C || KIND == kC2R) ? 2 * A.nl : A.B;  // lines incl. pair padding
    const int total = Bl * na;
    for (int e = threadIdx.x; e < total; e += nt) {
      int line, pos;
      if (A.load_afast) {
        line = e / na;
        pos = e - line * na;
      } else {
        pos = e / Bl;
        line = e - pos * Bl;
      }
      const bool valid = line < nb;
      int c[4];
      tile_coord(c, cbase, A.a, pos, A.b, b0 + line);
      if (KIND == kR2C) {
        T v = T(0);
        if (valid) v = reinterpret_cast<const T*>(A.in)[layout_offset(lsrc, c, A.nd)];
        T* slot = reinterpret_cast<T*>(buf0 + (line >> 1) * A.pitch + pos);
        slot[line & 1] = v;
      } else if (KIND == kC2R) {
        C v = mk<T>(T(0), T(0));
        if (valid) v = reinterpret_cast<const C*>(A.in)[layout_offset(lsrc, c, A.nd)];
        buf0[(line >> 1) * A.pitch + (line & 1) * na + pos] = v;
      } else if (KIND == kCopyReal) {
        if (valid) buf0[line * A.pitch + pos] = mk<T>(reinterpret_cast<const T*>(A.in)[layout_offset(lsrc, c, A.nd)], T(0));
      } else {
        if (valid) buf0[line * A.pitch + pos] = reinterpret_cast<const C*>(A.in)[layout_offset(lsrc, c, A.nd)];
      }
    }
  }
  __syncthreads();

  C* cur = buf0;
  C* nxt = buf1;
  if (KIND == kC2R) {
    // Z = X0 + i X1 over the full length n from the two half spectra stored
    // side by side in each line of buf0; the imaginary parts of the DC and
    // (even n) Nyquist bins are dropped, as a C2R transform does.
    const int h = A.n / 2 + 1;
    const int total = A.nl * h;
    for (int it = threadIdx.x; it < total; it += nt) {
      const int m = it / h, k = it - m * h;
      const C x0 = buf0[m * A.pitch + k];
      const C x1 = buf0[m * A.pitch + h + k];
      C* line = buf1 + m * A.pitch;
      if (k == 0 || 2 * k == A.n) {
        line[k] = mk<T>(x0.x, x1.x);
      } else {
        line[k] = mk<T>(x0.x - x1.y, x0.y + x1.x);
        line[A.n - k] = mk<T>(x0.x + x1.y, x1.x - x0.y);
      }
    }
    __syncthreads();
    cur = buf1;
    nxt = buf0;
  }

  if (KIND != kCopy && KIND != kCopyReal) {
    int Ns = 1;
    unsigned long long code = A.radix_code;
    for (int p = 0; p < A.npass; ++p) {
      const int R = static_cast<int>(code & 0xFull);
      code >>= 4;
      run_pass<T, INV>(R, cur, nxt, A.pitch, A.nl, A.n, Ns, tw);
      __syncthreads();
      C* tmp = cur;
      cur = nxt;
      nxt = tmp;
      Ns *= R;
    }
  }

  // ---------------- scatter ----------------
  {
    const int na = A.na_out;
    const int total = A.B * na;
    const T s = T(A.scale);
    for (int e = threadIdx.x; e < total; e += nt) {
      int line, pos;
      if (A.store_afast) {
        line = e / na;
        pos = e - line * na;
      } else {
        pos = e / A.B;
        line = e - pos * A.B;
      }
      if (line >= nb) continue;
      int c[4];
      tile_coord(c, cbase, A.a, pos, A.b, b0 + line);
      const int64_t o = layout_offset(ldst, c, A.nd);
      if (KIND == kR2C) {
        const C* zl = cur + (line >> 1) * A.pitch;
        const C z = zl[pos];
        const C zc = cconj(zl[pos == 0 ? 0 : A.n - pos]);
        C x;
        if ((line & 1) == 0) {
          x = cscale(cadd(z, zc), T(0.5) * s);
        } else {
          const C d = csub(z, zc);
          x = mk<T>(d.y * (T(0.5) * s), -d.x * (T(0.5) * s));
        }
        reinterpret_cast<C*>(A.out)[o] = x;
      } else if (KIND == kC2R) {
        const C z = cur[(line >> 1) * A.pitch + pos];
        reinterpret_cast<T*>(A.out)[o] = ((line & 1) ? z.y : z.x) * s;
      } else if (KIND == kCopyReal) {
        reinterpret_cast<T*>(A.out)[o] = cur[line * A.pitch + pos].x * s;
      } else {
        reinterpret_cast<C*>(A.out)[o] = cscale(cur[line * A.pitch + pos], s);
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Host-callable launcher
// ---------------------------------------------------------------------------
template <typename T>
static cudaError_t launch_stage_t(const StageArgs& A, int kind, bool inverse, int nthreads, size_t smem,
                                  unsigned tiles, cudaStream_t st) {
  void (*k)(StageArgs) = nullptr;
  switch (kind) {
    case kC2C: k = inverse ? fft_stage_kernel<T, kC2C, true> : fft_stage_kernel<T, kC2C, false>; break;
    case kR2C: k = fft_stage_kernel<T, kR2C, false>; break;
    case kC2R: k = fft_stage_kernel<T, kC2R, true>; break;
    case kCopy: k = fft_stage_kernel<T, kCopy, false>; break;
    case kCopyReal: k = fft_stage_kernel<T, kCopyReal, false>; break;
    default: return cudaErrorInvalidValue;
  }
  const cudaError_t e = raise_smem_limit(reinterpret_cast<const void*>(k), smem);
  if (e != cudaSuccess) return e;
  k<<<tiles, nthreads, smem, st>>>(A);
  return cudaGetLastError();
}

cudaError_t raise_smem_limit(const void* kernel, size_t smem) {
  if (smem <= 48 * 1024) return cudaSuccess;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  static std::mutex mu;
  static std::map<std::pair<const void*, int>, size_t> raised;
  std::lock_guard<std::mutex> lock(mu);
  size_t& done = raised[std::make_pair(kernel, dev)];
  if (smem <= done) return cudaSuccess;
  e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
  if (e == cudaSuccess) done = smem;
  return e;
}

cudaError_t launch_fft_stage(const StageArgs& A, bool dbl, int kind, bool inverse, int nthreads, size_t smem,
                             unsigned tiles, cudaStream_t st) {
  return dbl ? launch_stage_t<double>(A, kind, inverse, nthreads, smem, tiles, st)
             : launch_stage_t<float>(A, kind, inverse, nthreads, smem, tiles, st);
}

}  // namespace dev
}  // namespace dfft
