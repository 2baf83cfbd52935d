// Tile bodies of the register-resident stages (one line per thread group):
// fast_tile (C2C, lines of 2^k or 3 * 2^k points) and real_tile (R2C first /
// C2R last stage, two real lines per register line).  fft_fast.cu launches
// one tile per CTA; fft_batch.cu's persistent CTAs walk tiles of many fields.
#pragma once

#include "fft_radix.cuh"

namespace dfft {
namespace dev {
namespace radix {

// One tile (tile tb along b, coordinates co0 / co1 along o0 / o1) of a C2C
// stage, run by N/V*B threads with `smem_raw` of (N + B*LP) complex elements.
// Called by fft_fast_kernel (one tile per CTA) and by the batched stage
// kernels (fft_batch.cu), whose CTAs walk tiles of several fields.
template <typename T, bool INV, int N, int B, bool AFAST, bool AFF>
// stage_tw = false: the twiddles of this N are already in smem_raw (the
// previous tile of the CTA had the same line length)
__device__ __forceinline__ void fast_tile(const StageArgs& A, int tb, int co0, int co1, unsigned char* smem_raw,
                                          bool stage_tw = true) {
  using C = cplx<T>;
  constexpr int V = Vals<N>::value;
  constexpr int TT = N / V;                  // threads per line
  constexpr int NPASS = Radix<N, 0>::npass;
  using SH = SmemShape<T, N, B, AFAST>;
  constexpr int LP = SH::LP;
  C* tw = reinterpret_cast<C*>(smem_raw);
  C* tile = tw + N;
  const DevLayout ls = A.src, ld = A.dst;

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
    if (stage_tw)
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
      if (A.src_atab) {
#pragma unroll
        for (int q = 0; q < Q0; ++q)
#pragma unroll
          for (int r = 0; r < R0; ++r) v[q * R0 + r] = row[__ldg(ls.t + A.s_ta + in_pos<N, 0, TT>(t, q, r))];
      } else {
#pragma unroll
        for (int q = 0; q < Q0; ++q)
#pragma unroll
          for (int r = 0; r < R0; ++r) v[q * R0 + r] = row[in_pos<N, 0, TT>(t, q, r) * stride];
      }
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
  if constexpr (AFF) {
    if (A.pre_mode && active) {
      // global spatial coordinates of the line (axes 1..3 of the 4D view):
      // the one along a varies with the position, the others are fixed
      int fixed[3], along = -1;
#pragma unroll
      for (int k = 1; k <= 3; ++k) {
        fixed[k - 1] = k == A.b ? b0 + line : k == A.o0 ? co0 : k == A.o1 ? co1 : 0;
        if (k == A.a) along = k - 1;
      }
#pragma unroll
      for (int q = 0; q < Q0; ++q)
#pragma unroll
        for (int r = 0; r < R0; ++r) {
          const int p = in_pos<N, 0, TT>(t, q, r);
          int m[3];
#pragma unroll
          for (int k = 0; k < 3; ++k) m[k] = along == k ? p : fixed[k];
#pragma unroll
          for (int k = 0; k < 2; ++k) m[k] = 2 * m[k] < A.pre_n[k] ? m[k] : m[k] - A.pre_n[k];
          const bool keep = abs(m[0]) <= A.pre_cut[0] && abs(m[1]) <= A.pre_cut[1] && m[2] <= A.pre_cut[2];
          C x = v[q * R0 + r];
          if (!keep) x = mk<T>(T(0), T(0));
          if (A.pre_mode >= 2) {
            const int c = A.pre_mode - 2;
            const T kc = T((c == 0 ? m[0] : c == 1 ? m[1] : m[2]) * A.pre_kscale);
            x = mk<T>(-kc * x.y, kc * x.x);  // i k_c x
          }
          v[q * R0 + r] = x;
        }
    }
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
      if (A.dst_atab) {
#pragma unroll
        for (int q = 0; q < QL; ++q)
#pragma unroll
          for (int r = 0; r < RL; ++r) row[__ldg(ld.t + A.d_ta + t + last_rel<N, TT>(q, r))] = v[q * RL + r];
      } else {
#pragma unroll
        for (int q = 0; q < QL; ++q)
#pragma unroll
          for (int r = 0; r < RL; ++r) row[(t + last_rel<N, TT>(q, r)) * stride] = v[q * RL + r];
      }
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
__device__ __forceinline__ void real_tile(const StageArgs& A, int tb, int co0, int co1, unsigned char* smem_raw,
                                          bool stage_tw = true) {
  using C = cplx<T>;
  constexpr int V = Vals<N>::value;
  constexpr int TT = N / V;
  constexpr int NPASS = Radix<N, 0>::npass;
  constexpr int H = N / 2;
  using SH = SmemShape<T, N, B, true>;
  constexpr int LP = SH::LP;
  constexpr int S = SH::S;
  C* tw = reinterpret_cast<C*>(smem_raw);
  C* tile = tw + N;
  const DevLayout ls = A.src, ld = A.dst;

  const int b0 = tb * 2 * B;               // first real line of the tile
  const int nbr = min(2 * B, A.Eb - b0);   // real lines in the tile
  const int t = threadIdx.x % TT;
  const int line = threadIdx.x / TT;
  const int r0 = 2 * line, r1 = 2 * line + 1;
  const bool act0 = r0 < nbr, act1 = r1 < nbr;
  C* ln = tile + line * LP;

  {
    const C* gtw = reinterpret_cast<const C*>(A.tw);
    if (stage_tw)
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
  // position p of a line -> offset from its row base: p, or (general-layout
  // variant, a side split into bins along a) the axis table
  const bool satab = AFF && A.src_atab, datab = AFF && A.dst_atab;
  auto spos = [&](int p) -> int64_t { return satab ? __ldg(ls.t + A.s_ta + p) : p; };
  auto dpos = [&](int p) -> int64_t { return datab ? __ldg(ld.t + A.d_ta + p) : p; };

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
        const int64_t p = spos(in_pos<N, 0, TT>(t, q, r));
        v[q * R0 + r] = mk<T>(act0 ? row0[p] : T(0), act1 ? row1[p] : T(0));
      }
    __syncthreads();  // twiddles staged
  } else {
    const C* in = reinterpret_cast<const C*>(A.in);
    const C* row0 = in + srow0;
    const C* row1 = in + srow1;
    for (int k = t; k <= H; k += TT) {
      const int64_t pk = spos(k);
      const C x0 = act0 ? row0[pk] : mk<T>(T(0), T(0));
      const C x1 = act1 ? row1[pk] : mk<T>(T(0), T(0));
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
      const int64_t pk = dpos(k);
      if (act0) row0[pk] = cscale(cadd(z, zc), hs);
      if (act1) {
        const C d = csub(z, zc);
        row1[pk] = mk<T>(d.y * hs, -d.x * hs);
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
        const int64_t p = dpos(t + last_rel<N, TT>(q, r));
        if (act0) row0[p] = v[q * RL + r].x * s;
        if (act1) row1[p] = v[q * RL + r].y * s;
      }
  }
}

}  // namespace radix
}  // namespace dev
}  // namespace dfft
