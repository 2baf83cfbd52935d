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
#include "fft_stage.cuh"

namespace dfft {
namespace dev {

namespace {

template <bool INV, typename C>
__device__ __forceinline__ void r4(C& v0, C& v1, C& v2, C& v3) {
  C s02 = cadd(v0, v2), d02 = csub(v0, v2);
  C s13 = cadd(v1, v3), d13 = rot<INV>(csub(v1, v3));
  v0 = cadd(s02, s13);
  v2 = csub(s02, s13);
  v1 = cadd(d02, d13);
  v3 = csub(d02, d13);
}

template <typename T, bool INV>
__device__ __forceinline__ void r8(cplx<T>* v) {
  using C = cplx<T>;
  const T h = T(0.70710678118654752440084436210484903928);
  C e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
  C o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
  r4<INV>(e0, e1, e2, e3);
  r4<INV>(o0, o1, o2, o3);
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
__device__ __forceinline__ void r3(cplx<T>* v) {
  using C = cplx<T>;
  const T c3 = T(0.86602540378443864676372317075293618347);  // sqrt(3)/2
  const C t = cadd(v[1], v[2]);
  const C d = rot<INV>(cscale(csub(v[1], v[2]), c3));
  const C m = csub(v[0], cscale(t, T(0.5)));
  v[0] = cadd(v[0], t);
  v[1] = cadd(m, d);
  v[2] = csub(m, d);
}

template <typename T, bool INV, int R>
__device__ __forceinline__ void dftR(cplx<T>* v) {
  if constexpr (R == 3) {
    r3<T, INV>(v);
  } else if constexpr (R == 2) {
    const cplx<T> t = v[0];
    v[0] = cadd(t, v[1]);
    v[1] = csub(t, v[1]);
  } else if constexpr (R == 4) {
    r4<INV>(v[0], v[1], v[2], v[3]);
  } else {
    r8<T, INV>(v);
  }
}

// radix of pass P of an N-point plan: the first pass is radix 8 whenever N
// allows it; the radix-3 pass of 3 * 2^k plans is the last one.
template <int N, int P>
struct Radix;
#define DFFT_PLAN(N_, ...)                                       \
  template <int P>                                               \
  struct Radix<N_, P> {                                          \
    static constexpr int list[] = {__VA_ARGS__};                 \
    static constexpr int npass = sizeof(list) / sizeof(int);     \
    static constexpr int value = P < npass ? list[P < npass ? P : 0] : 1; \
  };
DFFT_PLAN(16, 2, 8)
DFFT_PLAN(32, 4, 8)
DFFT_PLAN(64, 8, 8)
DFFT_PLAN(128, 8, 2, 8)
DFFT_PLAN(256, 8, 4, 8)
DFFT_PLAN(512, 8, 8, 8)
DFFT_PLAN(1024, 8, 4, 4, 8)
DFFT_PLAN(2048, 8, 4, 8, 8)
DFFT_PLAN(4096, 8, 8, 8, 8)
DFFT_PLAN(24, 8, 3)
DFFT_PLAN(48, 8, 2, 3)
DFFT_PLAN(96, 8, 4, 3)
DFFT_PLAN(192, 8, 8, 3)
DFFT_PLAN(384, 8, 4, 4, 3)
DFFT_PLAN(768, 8, 8, 4, 3)
#undef DFFT_PLAN

// values per thread
template <int N>
struct Vals {
  static constexpr int value = (N % 3 == 0) ? 24 : 8;
};

template <int N, int P>
struct NsOf {
  static constexpr int value = NsOf<N, P - 1>::value * Radix<N, P - 1>::value;
};
template <int N>
struct NsOf<N, 0> {
  static constexpr int value = 1;
};

// Shared-memory layout of a line: position p is stored at p + (p >> S) and
// lines are LP elements apart.  S and the pitch offset were chosen by an
// offline model of the bank wavefronts of every exchange of every plan and
// thread mapping (one pad per 8 elements, or per 16 for complex64 lines of
// 128+ points read along the line), which keeps the exchanges within ~1.1x of
// conflict-free.
template <typename T, int N, int B, bool AFAST>
struct SmemShape {
  static constexpr bool f32 = sizeof(T) == 4;
  static constexpr int S = (f32 && ((AFAST && N >= 128) || (!AFAST && B == 1))) ? 4 : 3;
  static constexpr int extra_afast = (N <= (f32 ? 64 : 32)) ? 1 : 0;
  static constexpr int full = f32 ? 16 : 8;
  static constexpr int extra_bfast = (B >= full) ? 0 : (B * 2 == full) ? 3 : (B * 4 == full) ? 5 : (B * 8 == full) ? 9 : 0;
  static constexpr int LP = (N - 1) + ((N - 1) >> S) + 1 + (AFAST ? extra_afast : extra_bfast);
};

template <int S>
__device__ __forceinline__ int padpos(int p) {
  return p + (p >> S);
}

// element position of value (q, r) of thread t at the input of pass P
template <int N, int P, int TT>
__device__ __forceinline__ int in_pos(int t, int q, int r) {
  constexpr int R = Radix<N, P>::value;
  return (t + TT * q) + r * (N / R);
}

// element position of value (q, r) of thread t at the output of pass P
template <int N, int P, int TT>
__device__ __forceinline__ int out_pos(int t, int q, int r) {
  constexpr int R = Radix<N, P>::value;
  constexpr int Ns = NsOf<N, P>::value;
  const int j = t + TT * q;
  const int k = j % Ns;
  return (j - k) * R + k + r * Ns;
}

// Output position of value (q, r) of thread t after the last pass, minus t.
// The earlier passes multiply to Ns = N / R_last and j = t + TT q < Ns, so the
// Stockham index (j - j % Ns) R + j % Ns + r Ns reduces to j + r Ns: the
// position is t plus a compile-time constant (no modulo by a 3 * 2^k Ns).
template <int N, int TT>
__device__ __forceinline__ constexpr int last_rel(int q, int r) {
  constexpr int RL = Radix<N, Radix<N, 0>::npass - 1>::value;
  static_assert(NsOf<N, Radix<N, 0>::npass - 1>::value * RL == N, "radix plan must multiply to N");
  return TT * q + r * (N / RL);
}

template <typename T, bool INV, int N, int P, int TT>
__device__ __forceinline__ void compute_pass(cplx<T>* v, int t, const cplx<T>* tw) {
  using C = cplx<T>;
  constexpr int R = Radix<N, P>::value;
  constexpr int Ns = NsOf<N, P>::value;
  constexpr int Q = Vals<N>::value / R;
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    if (Ns > 1) {
      const int k = (t + TT * q) % Ns;
      const int m = k * (N / (Ns * R));  // w = tw[m] = exp(-2 pi i k / (Ns R))
      if constexpr (R == 8) {
        // three table reads (w, w^2, w^4); the other powers are products of
        // at most two of them
        C w1 = tw[m], w2 = tw[2 * m], w4 = tw[4 * m];
        if (INV) {
          w1.y = -w1.y;
          w2.y = -w2.y;
          w4.y = -w4.y;
        }
        const C w3 = cmul(w1, w2);
        v[q * R + 1] = cmul(v[q * R + 1], w1);
        v[q * R + 2] = cmul(v[q * R + 2], w2);
        v[q * R + 3] = cmul(v[q * R + 3], w3);
        v[q * R + 4] = cmul(v[q * R + 4], w4);
        v[q * R + 5] = cmul(v[q * R + 5], cmul(w1, w4));
        v[q * R + 6] = cmul(v[q * R + 6], cmul(w2, w4));
        v[q * R + 7] = cmul(v[q * R + 7], cmul(w3, w4));
      } else {
#pragma unroll
        for (int r = 1; r < R; ++r) {
          C w = tw[r * m];
          if (INV) w.y = -w.y;
          v[q * R + r] = cmul(v[q * R + r], w);
        }
      }
    }
    dftR<T, INV, R>(v + q * R);
  }
}

template <typename T, bool INV, int N, int P, int TT, int S>
__device__ __forceinline__ void exchange(cplx<T>* v, int t, cplx<T>* line) {
  constexpr int V = Vals<N>::value;
  constexpr int R = Radix<N, P>::value, Q = V / R;
  constexpr int R2 = Radix<N, P + 1>::value, Q2 = V / R2;
#pragma unroll
  for (int q = 0; q < Q; ++q)
#pragma unroll
    for (int r = 0; r < R; ++r) line[padpos<S>(out_pos<N, P, TT>(t, q, r))] = v[q * R + r];
  __syncthreads();
#pragma unroll
  for (int q = 0; q < Q2; ++q)
#pragma unroll
    for (int r = 0; r < R2; ++r) v[q * R2 + r] = line[padpos<S>(in_pos<N, P + 1, TT>(t, q, r))];
  __syncthreads();
}

template <typename T, bool INV, int N, int P, int TT, int S>
__device__ __forceinline__ void run_fft(cplx<T>* v, int t, const cplx<T>* tw, cplx<T>* line) {
  compute_pass<T, INV, N, P, TT>(v, t, tw);
  if constexpr (P + 1 < Radix<N, 0>::npass) {
    exchange<T, INV, N, P, TT, S>(v, t, line);
    run_fft<T, INV, N, P + 1, TT, S>(v, t, tw, line);
  }
}

// Base offset and stride along a of line (b = lb, o0 = c0, o1 = c1) of a
// layout whose rank blocks do not split axis a.
__device__ __forceinline__ void line_affine(const DevLayout& L, const StageArgs& A, int lb, int c0, int c1,
                                            int64_t* base, int64_t* stride) {
  int c[4] = {0, 0, 0, 0};
  c[A.b] = lb;
  if (A.o0 >= 0) c[A.o0] = c0;
  if (A.o1 >= 0) c[A.o1] = c1;
  *base = layout_offset(L, c, A.nd);
  c[A.a] = 1;
  *stride = layout_offset(L, c, A.nd) - *base;
}

}  // namespace

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

// Grid of a stage and the table offsets the kernels read (host side).
static dim3 fast_grid(const StageArgs& A) {
  return dim3(static_cast<unsigned>(A.tiles_b), static_cast<unsigned>(A.Eo0), static_cast<unsigned>(A.Eo1));
}

static StageArgs with_table_offsets(const StageArgs& A) {
  StageArgs R = A;
  R.s_ta = A.src.off[A.a];
  R.d_ta = A.dst.off[A.a];
  R.s_tb = A.src.off[A.b];
  R.d_tb = A.dst.off[A.b];
  R.s_to0 = A.o0 >= 0 ? A.src.off[A.o0] : 0;
  R.d_to0 = A.o0 >= 0 ? A.dst.off[A.o0] : 0;
  R.s_to1 = A.o1 >= 0 ? A.src.off[A.o1] : 0;
  R.d_to1 = A.o1 >= 0 ? A.dst.off[A.o1] : 0;
  return R;
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
