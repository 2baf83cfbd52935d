// Register-resident radix passes shared by the register FFT kernels
// (fft_fast.cu: one line per thread group; fft_pair.cu: two complex64 lines
// per thread).  A line of N points is transformed by N/V threads holding V
// values each (V = 8 for powers of two, V = 24 for 3 * 2^k); pass P is a
// Stockham pass of radix Radix<N, P>, and values move between passes through
// padded shared memory.
#pragma once

#include "fft_stage.cuh"

namespace dfft {
namespace dev {
namespace radix {

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
// conflict-free.  Lines of 3 * 2^k points read along the line (a-fast: 8
// threads of a line, 4 lines per warp) up to 192 points in complex64 and every
// such length in complex128 take S = 3 and one more pad: with the general
// rule their exchanges and the R2C / C2R half-spectrum passes ran at 2x the
// conflict-free wavefronts (measured: 8M bank conflicts per 192-point R2C
// launch of 340 MB), with this shape within 1.09x.
template <typename T, int N, int B, bool AFAST>
struct SmemShape {
  static constexpr bool f32 = sizeof(T) == 4;
  static constexpr bool v24 = AFAST && N % 3 == 0 && !(f32 && N >= 384);
  static constexpr int S = v24 ? 3 : (f32 && ((AFAST && N >= 128) || (!AFAST && B == 1))) ? 4 : 3;
  static constexpr int extra_afast = (v24 || N <= (f32 ? 64 : 32)) ? 1 : 0;
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

// ---- Compensated final radix-8 pass (complex64) ----
// Each value of the pass is carried as an unevaluated sum hi + lo of two
// floats: the twiddle products are split exactly with fused multiply-adds
// (p = a b rounded, e = fma(a, b, -p) = a b - p exactly), every addition of
// the butterfly is an error-free two-sum (Knuth: s = a + b rounded,
// e = (a - (s - (s - a))) + (b - (s - a)) = a + b - s exactly) whose error
// term is carried in lo, the 1/sqrt(2) rotations use a two-float constant,
// and each output is rounded once, hi + lo.  The intrinsics (__fadd_rn,
// __fmul_rn) keep the compiler from contracting the additions and products
// into fused multiply-adds, which would break the error-free identities.
// All seven twiddles are read from the table (no products of twiddles).
struct DFloat {
  float hi, lo;
};
struct DCplx {
  DFloat x, y;
};

__device__ __forceinline__ DFloat two_sum(float a, float b) {
  const float s = __fadd_rn(a, b);
  const float bb = __fadd_rn(s, -a);
  const float e = __fadd_rn(__fadd_rn(a, -__fadd_rn(s, -bb)), __fadd_rn(b, -bb));
  return DFloat{s, e};
}
__device__ __forceinline__ DFloat df_add(DFloat a, DFloat b) {
  DFloat r = two_sum(a.hi, b.hi);
  r.lo = __fadd_rn(r.lo, __fadd_rn(a.lo, b.lo));
  return r;
}
__device__ __forceinline__ DFloat df_neg(DFloat a) { return DFloat{-a.hi, -a.lo}; }
__device__ __forceinline__ DFloat df_sub(DFloat a, DFloat b) { return df_add(a, df_neg(b)); }
__device__ __forceinline__ DCplx dc_add(DCplx a, DCplx b) { return DCplx{df_add(a.x, b.x), df_add(a.y, b.y)}; }
__device__ __forceinline__ DCplx dc_sub(DCplx a, DCplx b) { return DCplx{df_sub(a.x, b.x), df_sub(a.y, b.y)}; }
// s i z, s = -1 forward, +1 inverse (exact)
template <bool INV>
__device__ __forceinline__ DCplx dc_rot(DCplx z) {
  return INV ? DCplx{df_neg(z.y), z.x} : DCplx{z.y, df_neg(z.x)};
}
// a * (1/sqrt 2) with the constant as the two floats kH + kHl
__device__ __forceinline__ DFloat df_mul_h(DFloat a) {
  constexpr double hd = 0.70710678118654752440084436210484903928;
  constexpr float kH = static_cast<float>(hd);
  constexpr float kHl = static_cast<float>(hd - static_cast<double>(kH));
  const float p = __fmul_rn(a.hi, kH);
  const float pe = __fmaf_rn(a.hi, kH, -p);
  return DFloat{p, __fadd_rn(pe, __fadd_rn(__fmul_rn(a.lo, kH), __fmul_rn(a.hi, kHl)))};
}
// exact product of two complex64 values as hi + lo pairs
__device__ __forceinline__ DCplx dc_mul_exact(float2 v, float2 w) {
  float p = __fmul_rn(v.x, w.x), pe = __fmaf_rn(v.x, w.x, -p);
  float q = __fmul_rn(v.y, w.y), qe = __fmaf_rn(v.y, w.y, -q);
  DCplx r;
  r.x = two_sum(p, -q);
  r.x.lo = __fadd_rn(r.x.lo, __fadd_rn(pe, -qe));
  p = __fmul_rn(v.x, w.y);
  pe = __fmaf_rn(v.x, w.y, -p);
  q = __fmul_rn(v.y, w.x);
  qe = __fmaf_rn(v.y, w.x, -q);
  r.y = two_sum(p, q);
  r.y.lo = __fadd_rn(r.y.lo, __fadd_rn(pe, qe));
  return r;
}

template <bool INV>
__device__ __forceinline__ void dc_r4(DCplx& v0, DCplx& v1, DCplx& v2, DCplx& v3) {
  const DCplx s02 = dc_add(v0, v2), d02 = dc_sub(v0, v2);
  const DCplx s13 = dc_add(v1, v3), d13 = dc_rot<INV>(dc_sub(v1, v3));
  v0 = dc_add(s02, s13);
  v2 = dc_sub(s02, s13);
  v1 = dc_add(d02, d13);
  v3 = dc_sub(d02, d13);
}

// Final radix-8 pass P (twiddled, Ns = N / 8 > 1) of one line in compensated
// arithmetic; same data movement as compute_pass.
template <bool INV, int N, int P, int TT>
__device__ __forceinline__ void compute_pass_comp(float2* v, int t, const float2* tw) {
  constexpr int R = Radix<N, P>::value;
  constexpr int Ns = NsOf<N, P>::value;
  static_assert(R == 8 && Vals<N>::value == 8, "compensated pass: radix 8, 8 values per thread");
  DCplx d[8];
  d[0] = DCplx{DFloat{v[0].x, 0.f}, DFloat{v[0].y, 0.f}};
  if (Ns > 1) {
    const int k = t % Ns;
    const int m = k * (N / (Ns * R));
#pragma unroll
    for (int r = 1; r < 8; ++r) {
      float2 w = tw[r * m];
      if (INV) w.y = -w.y;
      d[r] = dc_mul_exact(v[r], w);
    }
  } else {
#pragma unroll
    for (int r = 1; r < 8; ++r) d[r] = DCplx{DFloat{v[r].x, 0.f}, DFloat{v[r].y, 0.f}};
  }
  DCplx e0 = d[0], e1 = d[2], e2 = d[4], e3 = d[6];
  DCplx o0 = d[1], o1 = d[3], o2 = d[5], o3 = d[7];
  dc_r4<INV>(e0, e1, e2, e3);
  dc_r4<INV>(o0, o1, o2, o3);
  DCplx t1, t3;
  if (INV) {
    t1 = DCplx{df_mul_h(df_sub(o1.x, o1.y)), df_mul_h(df_add(o1.x, o1.y))};
    t3 = DCplx{df_neg(df_mul_h(df_add(o3.x, o3.y))), df_mul_h(df_sub(o3.x, o3.y))};
  } else {
    t1 = DCplx{df_mul_h(df_add(o1.x, o1.y)), df_mul_h(df_sub(o1.y, o1.x))};
    t3 = DCplx{df_mul_h(df_sub(o3.y, o3.x)), df_neg(df_mul_h(df_add(o3.x, o3.y)))};
  }
  const DCplx t2 = dc_rot<INV>(o2);
  const DCplx out[8] = {dc_add(e0, o0), dc_add(e1, t1), dc_add(e2, t2), dc_add(e3, t3),
                        dc_sub(e0, o0), dc_sub(e1, t1), dc_sub(e2, t2), dc_sub(e3, t3)};
#pragma unroll
  for (int r = 0; r < 8; ++r)
    v[r] = make_float2(__fadd_rn(out[r].x.hi, out[r].x.lo), __fadd_rn(out[r].y.hi, out[r].y.lo));
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
// general-layout side whose rank blocks do not split axis a: the line lies in
// one rank block, found from the other coordinates (axis a contributes rank
// 0 and local index 0 at position 0), and its stride is that block's stride
// of axis a.
__device__ __forceinline__ void line_affine(const DevLayout& L, const StageArgs& A, int lb, int c0, int c1,
                                            int64_t* base, int64_t* stride) {
  int c[4] = {0, 0, 0, 0};
  c[A.b] = lb;
  if (A.o0 >= 0) c[A.o0] = c0;
  if (A.o1 >= 0) c[A.o1] = c1;
  int64_t r = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k)
    if (k < A.nd && k != A.a) r += __ldg(L.t + L.rk[k] + c[k]);
  int64_t o = __ldg(L.t + L.rbase + r);
#pragma unroll
  for (int k = 0; k < 4; ++k)
    if (k < A.nd && k != A.a) o += __ldg(L.t + L.loc[k] + c[k]) * __ldg(L.t + L.rstride + r * 4 + k);
  *base = o;
  *stride = __ldg(L.t + L.rstride + r * 4 + A.a);
}


}  // namespace radix

// Grid of a stage and the table offsets the kernels read (host side).
inline dim3 fast_grid(const StageArgs& A) {
  return dim3(static_cast<unsigned>(A.tiles_b), static_cast<unsigned>(A.Eo0), static_cast<unsigned>(A.Eo1));
}

inline StageArgs with_table_offsets(const StageArgs& A) {
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

}  // namespace dev
}  // namespace dfft
