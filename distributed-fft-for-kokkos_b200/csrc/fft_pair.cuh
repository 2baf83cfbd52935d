// Device code of the two-complex64-lines-per-thread register stages, shared
// by fft_pair.cu (per-thread global loads) and fft_tma.cu (TMA-fed tiles).
// See fft_pair.cu for the thread mapping.
#pragma once

#include "fft_radix.cuh"

namespace dfft {
namespace dev {
namespace radix {


// One exchange of pass P for both lines of a pair: position p of the pair
// lives at padpos(p) of the pair's shared-memory line as (x0, y0, x1, y1).
template <int N, int P, int TT, int S>
__device__ __forceinline__ void exchange_pair(float2* v0, float2* v1, int t, float4* line) {
  constexpr int V = 8;
  constexpr int R = Radix<N, P>::value, Q = V / R;
  constexpr int R2 = Radix<N, P + 1>::value, Q2 = V / R2;
#pragma unroll
  for (int q = 0; q < Q; ++q)
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const float2 a = v0[q * R + r], b = v1[q * R + r];
      line[padpos<S>(out_pos<N, P, TT>(t, q, r))] = make_float4(a.x, a.y, b.x, b.y);
    }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < Q2; ++q)
#pragma unroll
    for (int r = 0; r < R2; ++r) {
      const float4 w = line[padpos<S>(in_pos<N, P + 1, TT>(t, q, r))];
      v0[q * R2 + r] = make_float2(w.x, w.y);
      v1[q * R2 + r] = make_float2(w.z, w.w);
    }
  __syncthreads();
}

// One radix pass of both lines: the compensated variant for the last pass
// when COMP is set.
template <bool INV, int N, int P, int TT, bool COMP>
__device__ __forceinline__ void pass_pair(float2* v0, float2* v1, int t, const float2* tw) {
  if constexpr (COMP && P + 1 == Radix<N, 0>::npass) {
    compute_pass_comp<INV, N, P, TT>(v0, t, tw);
    compute_pass_comp<INV, N, P, TT>(v1, t, tw);
  } else {
    // both lines read the same twiddles (same t): the second pass reuses them
    compute_pass<float, INV, N, P, TT>(v0, t, tw);
    compute_pass<float, INV, N, P, TT>(v1, t, tw);
  }
}

template <bool INV, int N, int P, int TT, int S, bool COMP = false>
__device__ __forceinline__ void run_fft_pair(float2* v0, float2* v1, int t, const float2* tw, float4* line) {
  pass_pair<INV, N, P, TT, COMP>(v0, v1, t, tw);
  if constexpr (P + 1 < Radix<N, 0>::npass) {
    exchange_pair<N, P, TT, S>(v0, v1, t, line);
    run_fft_pair<INV, N, P + 1, TT, S, COMP>(v0, v1, t, tw, line);
  }
}

// Loads the pair (l0, l1) of one tile (first line b0) into v0 / v1.
// b-fast: positions p of the pair at (line l0 offset) + p * stride; stride and
// offsets are even (host check) and (N - 1) * stride < 2^31.
// ATAB: a side whose offsets along a come from the axis table (an exchange
// buffer cut into bins along a; StageArgs::src_atab / dst_atab).
template <int N, bool AFAST, bool ATAB = false>
__device__ __forceinline__ void load_pair(const StageArgs& A, const float2* in, int64_t so, int b0, int l0, int l1,
                                          bool act0, bool act1, int t, float2* v0, float2* v1) {
  using C = float2;
  constexpr int V = 8, TT = N / V;
  constexpr int R0 = Radix<N, 0>::value, Q0 = V / R0;
  const DevLayout& ls = A.src;
  const C zero = make_float2(0.f, 0.f);
  if (AFAST) {
    const C* row0 = in + so + (act0 ? __ldg(ls.t + A.s_tb + b0 + l0) : 0);
    const C* row1 = in + so + (act1 ? __ldg(ls.t + A.s_tb + b0 + l1) : 0);
#pragma unroll
    for (int q = 0; q < Q0; ++q)
#pragma unroll
      for (int r = 0; r < R0; ++r) {
        const int pos = in_pos<N, 0, TT>(t, q, r);
        const int64_t p = (ATAB && A.src_atab) ? __ldg(ls.t + A.s_ta + pos) : pos;
        v0[q * R0 + r] = act0 ? row0[p] : zero;
        v1[q * R0 + r] = act1 ? row1[p] : zero;
      }
  } else if (ATAB && A.src_atab) {
    // b-fast pair rows at the axis-table offsets of their positions (even,
    // host check: 16-byte aligned pairs)
    const C* line = in + so + (act0 ? __ldg(ls.t + A.s_tb + b0 + l0) : 0);
#pragma unroll
    for (int q = 0; q < Q0; ++q)
#pragma unroll
      for (int r = 0; r < R0; ++r) {
        const int64_t o = __ldg(ls.t + A.s_ta + in_pos<N, 0, TT>(t, q, r));
        if (act1) {
          const float4 w = *reinterpret_cast<const float4*>(line + o);
          v0[q * R0 + r] = make_float2(w.x, w.y);
          v1[q * R0 + r] = make_float2(w.z, w.w);
        } else {
          v0[q * R0 + r] = act0 ? line[o] : zero;
          v1[q * R0 + r] = zero;
        }
      }
  } else {
    const int st = static_cast<int>(A.src_astride);
    const int64_t base = so + (act0 ? __ldg(ls.t + A.s_tb + b0 + l0) : 0) + static_cast<int64_t>(t) * st;
    if (act1) {
      const float4* row = reinterpret_cast<const float4*>(in + base);
      const int st2 = st / 2;
#pragma unroll
      for (int q = 0; q < Q0; ++q)
#pragma unroll
        for (int r = 0; r < R0; ++r) {
          const float4 w = row[(TT * q + r * (N / R0)) * st2];
          v0[q * R0 + r] = make_float2(w.x, w.y);
          v1[q * R0 + r] = make_float2(w.z, w.w);
        }
    } else {
      const C* row = in + base;
#pragma unroll
      for (int q = 0; q < Q0; ++q)
#pragma unroll
        for (int r = 0; r < R0; ++r) {
          v0[q * R0 + r] = act0 ? row[(TT * q + r * (N / R0)) * st] : zero;
          v1[q * R0 + r] = zero;
        }
    }
  }
}

// Scales (when the stage scales) and stores the pair after the last pass.
template <int N, bool AFAST, bool ATAB = false>
__device__ __forceinline__ void store_pair(const StageArgs& A, float2* out, int64_t dof, int b0, int l0, int l1,
                                           bool act0, bool act1, int t, float2* v0, float2* v1) {
  using C = float2;
  constexpr int V = 8, TT = N / V;
  constexpr int NPASS = Radix<N, 0>::npass;
  constexpr int RL = Radix<N, NPASS - 1>::value, QL = V / RL;
  const DevLayout& ld = A.dst;
  if (A.scale != 1.0) {
    const float s = static_cast<float>(A.scale);
#pragma unroll
    for (int e = 0; e < V; ++e) {
      v0[e] = cscale(v0[e], s);
      v1[e] = cscale(v1[e], s);
    }
  }
  if (AFAST) {
    C* row0 = out + dof + (act0 ? __ldg(ld.t + A.d_tb + b0 + l0) : 0);
    C* row1 = out + dof + (act1 ? __ldg(ld.t + A.d_tb + b0 + l1) : 0);
#pragma unroll
    for (int q = 0; q < QL; ++q)
#pragma unroll
      for (int r = 0; r < RL; ++r) {
        const int pos = t + last_rel<N, TT>(q, r);
        const int64_t p = (ATAB && A.dst_atab) ? __ldg(ld.t + A.d_ta + pos) : pos;
        if (act0) row0[p] = v0[q * RL + r];
        if (act1) row1[p] = v1[q * RL + r];
      }
  } else if (ATAB && A.dst_atab) {
    if (!act0) return;
    C* line = out + dof + __ldg(ld.t + A.d_tb + b0 + l0);
#pragma unroll
    for (int q = 0; q < QL; ++q)
#pragma unroll
      for (int r = 0; r < RL; ++r) {
        const int64_t o = __ldg(ld.t + A.d_ta + t + last_rel<N, TT>(q, r));
        const C a = v0[q * RL + r], b = v1[q * RL + r];
        if (act1)
          *reinterpret_cast<float4*>(line + o) = make_float4(a.x, a.y, b.x, b.y);
        else
          line[o] = a;
      }
  } else if (act0) {
    const int st = static_cast<int>(A.dst_astride);
    const int64_t base = dof + __ldg(ld.t + A.d_tb + b0 + l0) + static_cast<int64_t>(t) * st;
    if (act1) {
      float4* row = reinterpret_cast<float4*>(out + base);
      const int st2 = st / 2;
#pragma unroll
      for (int q = 0; q < QL; ++q)
#pragma unroll
        for (int r = 0; r < RL; ++r) {
          const C a = v0[q * RL + r], b = v1[q * RL + r];
          row[last_rel<N, TT>(q, r) * st2] = make_float4(a.x, a.y, b.x, b.y);
        }
    } else {
      C* row = out + base;
#pragma unroll
      for (int q = 0; q < QL; ++q)
#pragma unroll
        for (int r = 0; r < RL; ++r) row[last_rel<N, TT>(q, r) * st] = v0[q * RL + r];
    }
  }
}

// One tile (tile tb along b, coordinates co0 / co1) of a two-line C2C stage:
// PB line pairs, N/8 threads per pair, `smem_raw` holding N complex64
// twiddles and PB * LP 16-byte line elements (pair_tile_smem).  Called by
// fft_pair_kernel (one tile per CTA) and by the batched stage kernels, whose
// CTAs walk tiles of many fields (stage_tw = false: the twiddles of this N
// are already staged).  Separable sides only.
template <bool INV, int N, int PB, bool AFAST, bool COMP = false, bool ATAB = false>
__device__ __forceinline__ void pair_tile(const StageArgs& A, int tb, int co0, int co1, unsigned char* smem_raw,
                                          bool stage_tw = true) {
  using C = float2;
  constexpr int V = 8;
  static_assert(Vals<N>::value == V, "two-line kernel: lines of 2^k points");
  constexpr int TT = N / V;
  using SH = SmemShape<double, N, PB, AFAST>;  // 16-byte elements: the complex128 line layout
  constexpr int LP = SH::LP;
  C* tw = reinterpret_cast<C*>(smem_raw);
  float4* tile = reinterpret_cast<float4*>(smem_raw + sizeof(C) * N);
  const DevLayout ls = A.src, ld = A.dst;

  const int b0 = tb * 2 * PB;
  const int nb = min(2 * PB, A.Eb - b0);
  int lp, t;
  if (AFAST) {
    t = threadIdx.x % TT;
    lp = threadIdx.x / TT;
  } else {
    lp = threadIdx.x % PB;
    t = threadIdx.x / PB;
  }
  const int l0 = AFAST ? lp : 2 * lp, l1 = AFAST ? lp + PB : 2 * lp + 1;
  const bool act0 = l0 < nb, act1 = l1 < nb;

  if (stage_tw) {
    const C* gtw = reinterpret_cast<const C*>(A.tw);
    for (int i = threadIdx.x; i < N; i += blockDim.x) tw[i] = gtw[i];
  }
  int64_t so = A.src_abase, dof = A.dst_abase;
  if (A.o0 >= 0) {
    so += __ldg(ls.t + A.s_to0 + co0);
    dof += __ldg(ld.t + A.d_to0 + co0);
  }
  if (A.o1 >= 0) {
    so += __ldg(ls.t + A.s_to1 + co1);
    dof += __ldg(ld.t + A.d_to1 + co1);
  }

  C v0[V], v1[V];
  const C* in = reinterpret_cast<const C*>(A.in);
  load_pair<N, AFAST, ATAB>(A, in, so, b0, l0, l1, act0, act1, t, v0, v1);
  __syncthreads();  // twiddles staged

  run_fft_pair<INV, N, 0, TT, SH::S, COMP>(v0, v1, t, tw, tile + lp * LP);

  store_pair<N, AFAST, ATAB>(A, reinterpret_cast<C*>(A.out), dof, b0, l0, l1, act0, act1, t, v0, v1);
}

template <int N, int PB, bool AFAST>
constexpr size_t pair_tile_smem() {
  return sizeof(float2) * N + sizeof(float4) * static_cast<size_t>(PB) * SmemShape<double, N, PB, AFAST>::LP;
}

// Line pairs per CTA, option i (0 default, 1 half, 2 double or quarter):
//   b-fast: 8 pairs (16-line, 128-byte rows) or enough for 256 threads;
//   a-fast: enough pairs for 128 threads;  at most 1024 threads.
constexpr int pair_option(int n, bool afast, int i) {
  const int tt = n / 8;
  const int cap = 1024 / tt > 0 ? 1024 / tt : 1;
  int p0 = afast ? (128 / tt > 1 ? 128 / tt : 1) : (256 / tt > 8 ? 256 / tt : 8);
  if (p0 > cap) p0 = cap;
  if (i == 0) return p0;
  if (i == 1) return p0 / 2 > 0 ? p0 / 2 : 0;
  if (p0 * 2 <= cap) return p0 * 2;
  return p0 / 4 > 0 ? p0 / 4 : 0;
}

// Line pairs per CTA of the streaming variant: the default, at most 512
// threads (about 110 registers a thread leave room for one 512-thread CTA).
constexpr int pair_stream_pairs(int n, bool afast) {
  const int p0 = pair_option(n, afast, 0);
  const int cap = 512 / (n / 8) > 0 ? 512 / (n / 8) : 1;
  return p0 < cap ? p0 : cap;
}

// b-fast tiles
constexpr int pair_stream_pairs(int n) { return pair_stream_pairs(n, false); }

}  // namespace radix
}  // namespace dev
}  // namespace dfft
