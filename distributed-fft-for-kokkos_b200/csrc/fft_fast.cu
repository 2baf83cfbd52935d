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
#include "fft_radix.cuh"

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
  using C = cplx<T>;
  constexpr int V = Vals<N>::value;
  constexpr int TT = N / V;                  // threads per line
  constexpr int NPASS = Radix<N, 0>::npass;
  using SH = SmemShape<T, N, B, AFAST>;
  constexpr int LP = SH::LP;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* tw = reinterpret_cast<C*>(smem_raw);
  C* tile = tw + N;
  const DevLayout ls = A.src, ld = A.dst;

  // grid (tiles_b, Eo0, Eo1): tile along b, coordinates along o0 and o1
  const int tb = blockIdx.x, co0 = blockIdx.y, co1 = blockIdx.z;
  const int b0 = tb * B;
  const int nb = min(B, A.Eb - b0);

  // thread -> (line, t): lines contiguous in the warp for b-fast rows
  int line, t;
  if (AFAST) {
    t = threadIdx.x % TT;
    line = threadIdx.x / TT;
  } else {
    line = threadIdx.x % B;
    t = threadIdx.x / B;
  }
  const bool active = line < nb;

  {
    const C* gtw = reinterpret_cast<const C*>(A.tw);
    for (int i = threadIdx.x; i < N; i += blockDim.x) tw[i] = gtw[i];
  }

  // offsets shared by the whole tile (separable tables)
  int64_t so = 0, dof = 0;
  const bool saff = AFF && A.src_line_affine, daff = AFF && A.dst_line_affine;
  if constexpr (!AFF) {
    if (A.o0 >= 0) {
      so += __ldg(ls.t + A.s_to0 + co0);
      dof += __ldg(ld.t + A.d_to0 + co0);
    }
    if (A.o1 >= 0) {
      so += __ldg(ls.t + A.s_to1 + co1);
      dof += __ldg(ld.t + A.d_to1 + co1);
    }
  } else {
    if (!saff) {
      if (A.o0 >= 0) so += __ldg(ls.t + A.s_to0 + co0);
      if (A.o1 >= 0) so += __ldg(ls.t + A.s_to1 + co1);
    }
    if (!daff) {
      if (A.o0 >= 0) dof += __ldg(ld.t + A.d_to0 + co0);
      if (A.o1 >= 0) dof += __ldg(ld.t + A.d_to1 + co1);
    }
  }

  C v[V];
  constexpr int R0 = Radix<N, 0>::value, Q0 = V / R0;
  const C* in = reinterpret_cast<const C*>(A.in);
  if (active) {
    if constexpr (AFF) {
      // general-layout variant: each side is one affine line, base + p * stride
      int64_t base, stride;
      if (saff) {
        line_affine(ls, A, b0 + line, co0, co1, &base, &stride);
      } else {
        base = so + __ldg(ls.t + A.s_tb + b0 + line) + A.src_abase;
        stride = A.src_astride;
      }
      const C* row = in + base;
#pragma unroll
      for (int q = 0; q < Q0; ++q)
#pragma unroll
        for (int r = 0; r < R0; ++r) v[q * R0 + r] = row[in_pos<N, 0, TT>(t, q, r) * stride];
    } else if (AFAST) {
      const C* row = in + so + __ldg(ls.t + A.s_tb + b0 + line) + A.src_abase;
#pragma unroll
      for (int q = 0; q < Q0; ++q)
#pragma unroll
        for (int r = 0; r < R0; ++r) v[q * R0 + r] = row[in_pos<N, 0, TT>(t, q, r)];
    } else if constexpr (V == 8) {
      // (N - 1) * stride < 2^31 (host check): 32-bit offsets along the line
      const int st = static_cast<int>(A.src_astride);
      const C* row = in + so + __ldg(ls.t + A.s_tb + b0 + line) + A.src_abase + static_cast<int64_t>(t) * st;
#pragma unroll
      for (int q = 0; q < Q0; ++q)
#pragma unroll
        for (int r = 0; r < R0; ++r) v[q * R0 + r] = row[(TT * q + r * (N / R0)) * st];  // in_pos - t
    } else {
      // 24 values a thread: offsets read from the axis table one at a time
      // keep fewer addresses live than 24 precomputed products
      const C* col = in + so + __ldg(ls.t + A.s_tb + b0 + line);
#pragma unroll
      for (int q = 0; q < Q0; ++q)
#pragma unroll
        for (int r = 0; r < R0; ++r) v[q * R0 + r] = col[__ldg(ls.t + A.s_ta + in_pos<N, 0, TT>(t, q, r))];
    }
  } else {
#pragma unroll
    for (int e = 0; e < V; ++e) v[e] = mk<T>(T(0), T(0));
  }
  __syncthreads();  // twiddles staged

  run_fft<T, INV, N, 0, TT, SH::S>(v, t, tw, tile + line * LP);

  constexpr int RL = Radix<N, NPASS - 1>::value, QL = V / RL;
  if (A.scale != 1.0) {  // only the normalised direction's last stage scales
    const T s = T(A.scale);
#pragma unroll
    for (int e = 0; e < V; ++e) v[e] = cscale(v[e], s);
  }
  C* out = reinterpret_cast<C*>(A.out);
  if (active) {
    if constexpr (AFF) {
      int64_t base, stride;
      if (daff) {
        line_affine(ld, A, b0 + line, co0, co1, &base, &stride);
      } else {
        base = dof + __ldg(ld.t + A.d_tb + b0 + line) + A.dst_abase;
        stride = A.dst_astride;
      }
      C* row = out + base;
#pragma unroll
      for (int q = 0; q < QL; ++q)
#pragma unroll
        for (int r = 0; r < RL; ++r) row[(t + last_rel<N, TT>(q, r)) * stride] = v[q * RL + r];
    } else if (AFAST) {
      C* row = out + dof + __ldg(ld.t + A.d_tb + b0 + line) + A.dst_abase;
#pragma unroll
      for (int q = 0; q < QL; ++q)
#pragma unroll
        for (int r = 0; r < RL; ++r) row[t + last_rel<N, TT>(q, r)] = v[q * RL + r];
    } else if constexpr (V == 8) {
      const int st = static_cast<int>(A.dst_astride);
      C* row = out + dof + __ldg(ld.t + A.d_tb + b0 + line) + A.dst_abase + static_cast<int64_t>(t) * st;
#pragma unroll
      for (int q = 0; q < QL; ++q)
#pragma unroll
        for (int r = 0; r < RL; ++r) row[last_rel<N, TT>(q, r) * st] = v[q * RL + r];
    } else {
      C* col = out + dof + __ldg(ld.t + A.d_tb + b0 + line);
#pragma unroll
      for (int q = 0; q < QL; ++q)
#pragma unroll
        for (int r = 0; r < RL; ++r) col[__ldg(ld.t + A.d_ta + t + last_rel<N, TT>(q, r))] = v[q * RL + r];
    }
  }
}

// Real-to-complex first stage / complex-to-real last stage on lines that are
// contiguous on both sides.  Each CTA line carries two real lines of the tile
// (rows 2l and 2l+1 along the tile axis) as one complex line z = x0 + i x1.
//   R2C: the N-point FFT of z goes to shared memory, and the two half spectra
//        X0[k] = (Z[k] + conj Z[N-k]) / 2, X1[k] = (Z[k] - conj Z[N-k]) / 2i,
//        k = 0..N/2, are written with the scale folded in.
//   C2R: Z[k] = X0[k] + i X1[k] and Z[N-k] = conj X0[k] + i conj X1[k] are
//        assembled in shared memory (imaginary parts of DC and Nyquist
//        dropped), inverse FFT, x0 = Re z and x1 = Im z are written.
template <typename T, bool C2R, int N, int B, bool AFF>
__global__ void __launch_bounds__(N / Vals<N>::value * B) fft_real_kernel(const StageArgs A) {
  using C = cplx<T>;
  constexpr int V = Vals<N>::value;
  constexpr int TT = N / V;
  constexpr int NPASS = Radix<N, 0>::npass;
  constexpr int H = N / 2;
  using SH = SmemShape<T, N, B, true>;
  constexpr int LP = SH::LP;
  constexpr int S = SH::S;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* tw = reinterpret_cast<C*>(smem_raw);
  C* tile = tw + N;
  const DevLayout ls = A.src, ld = A.dst;

  // grid (tiles_b, Eo0, Eo1): tile along b, coordinates along o0 and o1
  const int tb = blockIdx.x, co0 = blockIdx.y, co1 = blockIdx.z;
  const int b0 = tb * 2 * B;               // first real line of the tile
  const int nbr = min(2 * B, A.Eb - b0);   // real lines in the tile
  const int t = threadIdx.x % TT;
  const int line = threadIdx.x / TT;
  const int r0 = 2 * line, r1 = 2 * line + 1;
  const bool act0 = r0 < nbr, act1 = r1 < nbr;
  C* ln = tile + line * LP;

  {
    const C* gtw = reinterpret_cast<const C*>(A.tw);
    for (int i = threadIdx.x; i < N; i += blockDim.x) tw[i] = gtw[i];
  }
  // row bases (offset of position 0 of each real / complex line); lines are
  // contiguous along a on both sides
  int64_t srow0 = 0, srow1 = 0, drow0 = 0, drow1 = 0, unused;
  if (AFF && A.src_line_affine) {
    if (act0) line_affine(ls, A, b0 + r0, co0, co1, &srow0, &unused);
    if (act1) line_affine(ls, A, b0 + r1, co0, co1, &srow1, &unused);
  } else {
    int64_t so = A.src_abase;
    if (A.o0 >= 0) so += __ldg(ls.t + A.s_to0 + co0);
    if (A.o1 >= 0) so += __ldg(ls.t + A.s_to1 + co1);
    srow0 = so + (act0 ? __ldg(ls.t + A.s_tb + b0 + r0) : 0);
    srow1 = so + (act1 ? __ldg(ls.t + A.s_tb + b0 + r1) : 0);
  }
  if (AFF && A.dst_line_affine) {
    if (act0) line_affine(ld, A, b0 + r0, co0, co1, &drow0, &unused);
    if (act1) line_affine(ld, A, b0 + r1, co0, co1, &drow1, &unused);
  } else {
    int64_t dof = A.dst_abase;
    if (A.o0 >= 0) dof += __ldg(ld.t + A.d_to0 + co0);
    if (A.o1 >= 0) dof += __ldg(ld.t + A.d_to1 + co1);
    drow0 = dof + (act0 ? __ldg(ld.t + A.d_tb + b0 + r0) : 0);
    drow1 = dof + (act1 ? __ldg(ld.t + A.d_tb + b0 + r1) : 0);
  }
  const T s = T(A.scale);

  C v[V];
  constexpr int R0 = Radix<N, 0>::value, Q0 = V / R0;
  if constexpr (!C2R) {
    const T* in = reinterpret_cast<const T*>(A.in);
    const T* row0 = in + srow0;
    const T* row1 = in + srow1;
#pragma unroll
    for (int q = 0; q < Q0; ++q)
#pragma unroll
      for (int r = 0; r < R0; ++r) {
        const int p = in_pos<N, 0, TT>(t, q, r);
        v[q * R0 + r] = mk<T>(act0 ? row0[p] : T(0), act1 ? row1[p] : T(0));
      }
    __syncthreads();  // twiddles staged
  } else {
    const C* in = reinterpret_cast<const C*>(A.in);
    const C* row0 = in + srow0;
    const C* row1 = in + srow1;
    for (int k = t; k <= H; k += TT) {
      const C x0 = act0 ? row0[k] : mk<T>(T(0), T(0));
      const C x1 = act1 ? row1[k] : mk<T>(T(0), T(0));
      if (k == 0 || k == H) {
        ln[padpos<S>(k)] = mk<T>(x0.x, x1.x);
      } else {
        ln[padpos<S>(k)] = mk<T>(x0.x - x1.y, x0.y + x1.x);
        ln[padpos<S>(N - k)] = mk<T>(x0.x + x1.y, x1.x - x0.y);
      }
    }
    __syncthreads();  // spectrum and twiddles staged
#pragma unroll
    for (int q = 0; q < Q0; ++q)
#pragma unroll
      for (int r = 0; r < R0; ++r) v[q * R0 + r] = ln[padpos<S>(in_pos<N, 0, TT>(t, q, r))];
    __syncthreads();  // every line read before the first exchange overwrites it
  }

  run_fft<T, C2R, N, 0, TT, S>(v, t, tw, ln);

  constexpr int RL = Radix<N, NPASS - 1>::value, QL = V / RL;
  if constexpr (!C2R) {
    // the last exchange ended with a barrier: the line buffer is free
#pragma unroll
    for (int q = 0; q < QL; ++q)
#pragma unroll
      for (int r = 0; r < RL; ++r) ln[padpos<S>(t + last_rel<N, TT>(q, r))] = v[q * RL + r];
    __syncthreads();
    C* out = reinterpret_cast<C*>(A.out);
    C* row0 = out + drow0;
    C* row1 = out + drow1;
    const T hs = T(0.5) * s;
    for (int k = t; k <= H; k += TT) {
      const C z = ln[padpos<S>(k)];
      const C zc = cconj(ln[padpos<S>(k == 0 ? 0 : N - k)]);
      if (act0) row0[k] = cscale(cadd(z, zc), hs);
      if (act1) {
        const C d = csub(z, zc);
        row1[k] = mk<T>(d.y * hs, -d.x * hs);
      }
    }
  } else {
    T* out = reinterpret_cast<T*>(A.out);
    T* row0 = out + drow0;
    T* row1 = out + drow1;
#pragma unroll
    for (int q = 0; q < QL; ++q)
#pragma unroll
      for (int r = 0; r < RL; ++r) {
        const int p = t + last_rel<N, TT>(q, r);
        if (act0) row0[p] = v[q * RL + r].x * s;
        if (act1) row1[p] = v[q * RL + r].y * s;
      }
  }
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
  if (A.src_line_affine || A.dst_line_affine)  // general layouts: default tile only
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
  if (A.src_line_affine || A.dst_line_affine)
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
