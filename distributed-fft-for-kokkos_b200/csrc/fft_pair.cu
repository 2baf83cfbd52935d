// Register-resident FFT stage with two complex64 lines per thread (sm_100a).
//
// The same radix passes as fft_fast.cu (8 values a line per thread, lines of
// 2^k points, 16..4096), but every thread carries two lines of the tile:
//   b-fast tiles (unit stride along the tile axis b): lines 2l and 2l+1, which
//     are neighbours in memory, so one 16-byte access moves the same position
//     of both (the host checks that every pair starts on a 16-byte boundary);
//   a-fast tiles (unit stride along the FFT axis a): lines l and l + B/2, each
//     read as a contiguous row by consecutive threads.
// The exchanges between passes move both lines' values of a position as one
// 16-byte shared-memory element (the complex128 layout of the single-line
// kernel, which keeps them conflict-free), and the twiddle reads, index and
// address arithmetic of a thread serve 16 values instead of 8.  Separable
// layouts only (per-axis offset tables, affine along a).
#include "fft_pair.cuh"

namespace dfft {
namespace dev {

using namespace radix;

namespace {

// 1024 resident threads per SM: 64 registers for 16 complex64 values a thread
// (the compensated variant, with twice the live values in its last pass,
// keeps the compiler's choice)
template <int THREADS, bool COMP>
struct PairMinBlocks {
  static constexpr int v = 1024 / THREADS;
  static constexpr int value = (v > 0 && !COMP) ? v : 1;
};

// PB line pairs per CTA (2 PB lines), N/8 threads per pair.  COMP: the last
// radix pass in compensated arithmetic (compute_pass_comp).
template <bool INV, int N, int PB, bool AFAST, bool COMP = false, bool ATAB = false>
__global__ void __launch_bounds__(N / 8 * PB, (PairMinBlocks<N / 8 * PB, COMP>::value))
    fft_pair_kernel(const StageArgs A) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  // grid (tiles_b, Eo0, Eo1)
  pair_tile<INV, N, PB, AFAST, COMP, ATAB>(A, blockIdx.x, blockIdx.y, blockIdx.z, smem_raw);
}

// Streaming variant: a CTA walks A.tpc consecutive tiles along b (grid
// (ceil(tiles_b / tpc), Eo0, Eo1)) and issues the loads of tile i + 1 into
// registers before it transforms tile i, so each thread keeps one tile's
// loads in flight while it computes.  The table offsets along o0 / o1 and the
// twiddles are set up once per CTA.  About 100 registers: one CTA per SM.
template <bool INV, int N, int PB, bool AFAST>
__global__ void __launch_bounds__(N / 8 * PB, 1) fft_pair_stream_kernel(const StageArgs A) {
  using C = float2;
  constexpr int V = 8;
  static_assert(Vals<N>::value == V, "two-line kernel: lines of 2^k points");
  constexpr int TT = N / V;
  using SH = SmemShape<double, N, PB, AFAST>;
  constexpr int LP = SH::LP;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* tw = reinterpret_cast<C*>(smem_raw);
  float4* tile = reinterpret_cast<float4*>(smem_raw + sizeof(C) * N);
  const DevLayout ls = A.src, ld = A.dst;

  const int first = blockIdx.x * A.tpc, co0 = blockIdx.y, co1 = blockIdx.z;
  const int last = min(first + A.tpc, A.tiles_b);
  int lp, t;
  if (AFAST) {
    t = threadIdx.x % TT;
    lp = threadIdx.x / TT;
  } else {
    lp = threadIdx.x % PB;
    t = threadIdx.x / PB;
  }
  const int l0 = AFAST ? lp : 2 * lp, l1 = AFAST ? lp + PB : 2 * lp + 1;
  {
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
  const C* in = reinterpret_cast<const C*>(A.in);
  C* out = reinterpret_cast<C*>(A.out);

  C v0[V], v1[V], w0[V], w1[V];
  int b0 = first * 2 * PB;
  int nb = min(2 * PB, A.Eb - b0);
  load_pair<N, AFAST>(A, in, so, b0, l0, l1, l0 < nb, l1 < nb, t, v0, v1);
  __syncthreads();  // twiddles staged
  for (int k = first; k < last; ++k) {
    const int bn = b0 + 2 * PB;
    const int nbn = min(2 * PB, A.Eb - bn);
    if (k + 1 < last) load_pair<N, AFAST>(A, in, so, bn, l0, l1, l0 < nbn, l1 < nbn, t, w0, w1);
    run_fft_pair<INV, N, 0, TT, SH::S>(v0, v1, t, tw, tile + lp * LP);  // ends on a barrier
    store_pair<N, AFAST>(A, out, dof, b0, l0, l1, l0 < nb, l1 < nb, t, v0, v1);
#pragma unroll
    for (int e = 0; e < V; ++e) {
      v0[e] = w0[e];
      v1[e] = w1[e];
    }
    b0 = bn;
    nb = nbn;
  }
}

template <int N, bool INV, bool AF, int PB, bool COMP = false, bool ATAB = false>
static cudaError_t launch_pair_b(const StageArgs& A, cudaStream_t st) {
  if constexpr (PB <= 0) {
    return cudaErrorInvalidValue;
  } else {
    constexpr int LP = SmemShape<double, N, PB, AF>::LP;
    const size_t smem = sizeof(float2) * N + sizeof(float4) * static_cast<size_t>(PB) * LP;
    auto k = fft_pair_kernel<INV, N, PB, AF, COMP, ATAB>;
    const cudaError_t e = raise_smem_limit(reinterpret_cast<const void*>(k), smem);
    if (e != cudaSuccess) return e;
    k<<<fast_grid(A), N / 8 * PB, smem, st>>>(with_table_offsets(A));
    return cudaGetLastError();
  }
}

template <int N, bool INV, bool AF>
static cudaError_t launch_pair_stream(const StageArgs& A, cudaStream_t st) {
  constexpr int PB = pair_stream_pairs(N, AF);
  if (A.B != 2 * PB || A.tpc < 1) return cudaErrorInvalidValue;
  constexpr int LP = SmemShape<double, N, PB, AF>::LP;
  const size_t smem = sizeof(float2) * N + sizeof(float4) * static_cast<size_t>(PB) * LP;
  auto k = fft_pair_stream_kernel<INV, N, PB, AF>;
  const cudaError_t e = raise_smem_limit(reinterpret_cast<const void*>(k), smem);
  if (e != cudaSuccess) return e;
  const dim3 grid(static_cast<unsigned>((A.tiles_b + A.tpc - 1) / A.tpc), static_cast<unsigned>(A.Eo0),
                  static_cast<unsigned>(A.Eo1));
  k<<<grid, N / 8 * PB, smem, st>>>(with_table_offsets(A));
  return cudaGetLastError();
}

template <int N, bool INV, bool AF>
static cudaError_t launch_pair_n(const StageArgs& A, cudaStream_t st) {
  constexpr int P0 = pair_option(N, AF, 0), P1 = pair_option(N, AF, 1), P2 = pair_option(N, AF, 2);
  if (A.src_atab || A.dst_atab) {
    // sides read or written through the axis table: the default tile, plain FP32
    if (!A.comp && A.B == 2 * P0) return launch_pair_b<N, INV, AF, P0, false, true>(A, st);
    return cudaErrorInvalidValue;
  }
  if (A.comp) return A.B == 2 * P0 ? launch_pair_b<N, INV, AF, P0, true>(A, st) : cudaErrorInvalidValue;
  if (A.B == 2 * P0) return launch_pair_b<N, INV, AF, P0>(A, st);
  if (P1 > 0 && A.B == 2 * P1) return launch_pair_b<N, INV, AF, P1>(A, st);
  if (P2 > 0 && A.B == 2 * P2) return launch_pair_b<N, INV, AF, P2>(A, st);
  return cudaErrorInvalidValue;
}

template <int N>
static cudaError_t launch_pair_t(const StageArgs& A, bool inverse, bool afast, cudaStream_t st) {
  if (A.pairs == 2) {
    if (A.comp || A.src_atab || A.dst_atab) return cudaErrorInvalidValue;
    if (inverse) return afast ? launch_pair_stream<N, true, true>(A, st) : launch_pair_stream<N, true, false>(A, st);
    return afast ? launch_pair_stream<N, false, true>(A, st) : launch_pair_stream<N, false, false>(A, st);
  }
  if (inverse) return afast ? launch_pair_n<N, true, true>(A, st) : launch_pair_n<N, true, false>(A, st);
  return afast ? launch_pair_n<N, false, true>(A, st) : launch_pair_n<N, false, false>(A, st);
}

}  // namespace

bool pair_stage_supported(int n) { return n >= 16 && n <= 4096 && (n & (n - 1)) == 0; }

int pair_stage_stream_lines(int n, bool afast) {
  switch (n) {
#define DFFT_OPT(N_) \
  case N_: return 2 * pair_stream_pairs(N_, afast);
    DFFT_OPT(16) DFFT_OPT(32) DFFT_OPT(64) DFFT_OPT(128) DFFT_OPT(256) DFFT_OPT(512) DFFT_OPT(1024) DFFT_OPT(2048)
    DFFT_OPT(4096)
#undef DFFT_OPT
    default: return 0;
  }
}

int pair_stage_line_options(int n, bool afast, int* opts) {
  int k = 0;
  for (int i = 0; i < 3; ++i) {
    int p = 0;
    switch (n) {
#define DFFT_OPT(N_) \
  case N_: p = pair_option(N_, afast, i); break;
      DFFT_OPT(16) DFFT_OPT(32) DFFT_OPT(64) DFFT_OPT(128) DFFT_OPT(256) DFFT_OPT(512) DFFT_OPT(1024) DFFT_OPT(2048)
      DFFT_OPT(4096)
#undef DFFT_OPT
      default: break;
    }
    if (p > 0) opts[k++] = 2 * p;
  }
  return k;
}

cudaError_t launch_fft_pair(const StageArgs& A, bool inverse, bool afast, cudaStream_t st) {
  if (A.Eo0 > fast_stage_max_grid_yz() || A.Eo1 > fast_stage_max_grid_yz()) return cudaErrorInvalidValue;
  switch (A.n) {
    case 16: return launch_pair_t<16>(A, inverse, afast, st);
    case 32: return launch_pair_t<32>(A, inverse, afast, st);
    case 64: return launch_pair_t<64>(A, inverse, afast, st);
    case 128: return launch_pair_t<128>(A, inverse, afast, st);
    case 256: return launch_pair_t<256>(A, inverse, afast, st);
    case 512: return launch_pair_t<512>(A, inverse, afast, st);
    case 1024: return launch_pair_t<1024>(A, inverse, afast, st);
    case 2048: return launch_pair_t<2048>(A, inverse, afast, st);
    case 4096: return launch_pair_t<4096>(A, inverse, afast, st);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace dev
}  // namespace dfft
