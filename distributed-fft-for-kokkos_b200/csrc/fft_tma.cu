// TMA-fed register FFT stage for b-fast tiles of complex64 lines (sm_100a).
//
// A b-fast stage transforms lines along the FFT axis a whose neighbours along
// the tile axis b are neighbours in memory: a tile of L = 2 PB lines is a 2D
// box of L consecutive elements along b by N positions along a, i.e. N rows
// of L * 8 bytes with a large stride between rows.  Here the source tiles are
// moved by the tensor memory accelerator: one thread issues
// cp.async.bulk.tensor loads of the whole box into shared memory against an
// mbarrier, two tiles ahead of the one being transformed, so the CTA keeps
// two tiles (2 x L x N x 8 bytes) of loads in flight without holding them in
// registers.  The CTA is persistent: it walks tiles blockIdx.x, +gridDim.x,
// ... of the stage, with the twiddles staged once.
//
// Per tile, every thread reads its line pair's pass-0 values from the landing
// buffer (one 16-byte element per position: a quarter warp reads one or more
// whole consecutive rows, no bank conflicts), the tile is released to the
// next TMA load, the radix passes run as in fft_pair.cu (two lines per
// thread, 16-byte exchanges through the padded line buffer) and the last pass
// stores straight to global memory.
//
// The tensor map describes the source layout: the local block axes of a
// rank-blocked separable layout plus one dimension per split axis for the
// rank coordinate (at most 5); the host builds it per launch for the actual
// source pointer.  Waits on the mbarriers are bounded (about one second of
// %globaltimer): a wait that runs out sets *A.err, waits (bounded again) for
// the CTA's other load in flight and returns.
#include <cuda.h>

#include <cstring>

#include "fft_pair.cuh"

namespace dfft {
namespace dev {

using namespace radix;

namespace {

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Bounded wait for phase `parity` of `bar`: false after ~1 s.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = global_ns();
  for (uint32_t i = 1;; ++i) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((i & 63) == 0 && global_ns() - t0 > 1000000000ull) return false;
  }
}

// Orders this thread's earlier generic-proxy shared-memory accesses (made
// visible to it by the preceding barrier) before its following async-proxy
// (TMA) accesses.
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Tiled TMA load of a 5D box (no multicast) into this CTA's shared memory.
__device__ __forceinline__ void tma_load_5d(void* dst, const CUtensorMap* map, uint64_t* bar, const int* c) {
  asm volatile(
      "cp.async.bulk.tensor.5d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4, %5, %6}], [%7];" ::"r"(smem_addr(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c[0]), "r"(c[1]), "r"(c[2]), "r"(c[3]), "r"(c[4]),
      "r"(smem_addr(bar))
      : "memory");
}

// Issue the loads of tile (tb, co0, co1) into `dst`: N / boxa boxes of
// L x boxa along (b, a).  Thread 0 only.
template <int N, int L>
__device__ __forceinline__ void issue_tile(const CUtensorMap* map, const TmaCoords& T, int tb, int co0, int co1,
                                           float2* dst, uint64_t* bar) {
  mbar_expect_tx(bar, static_cast<uint32_t>(N * L * sizeof(float2)));
  int c[5];
#pragma unroll
  for (int d = 0; d < 5; ++d) {
    const int w = T.which[d];
    const int v = w == 0 ? tb * L : w == 2 ? co0 : w == 3 ? co1 : 0;
    c[d] = (w == 4 || w == 1) ? 0 : (T.rank_part[d] ? v / T.lk[d] : v % T.lk[d]);
  }
  for (int j = 0; j < T.nchunks; ++j) {
#pragma unroll
    for (int d = 0; d < 5; ++d)
      if (T.which[d] == 1) c[d] = j * T.boxa;
    tma_load_5d(dst + static_cast<int64_t>(j) * T.boxa * L, map, bar, c);
  }
}

// Tile coordinates of a persistent CTA: tile index i = tb + tiles_b (co0 +
// Eo0 co1), advanced by a fixed step with carries instead of divisions.
struct TileWalk {
  int tb, co0, co1;
  __device__ void init(unsigned i, const StageArgs& A) {
    tb = static_cast<int>(i % static_cast<unsigned>(A.tiles_b));
    const unsigned rest = i / static_cast<unsigned>(A.tiles_b);
    co0 = static_cast<int>(rest % static_cast<unsigned>(A.Eo0));
    co1 = static_cast<int>(rest / static_cast<unsigned>(A.Eo0));
  }
  __device__ void advance(int step_b, int step_r, const StageArgs& A) {
    tb += step_b;
    int carry = 0;
    if (tb >= A.tiles_b) {
      tb -= A.tiles_b;
      carry = 1;
    }
    co0 += step_r + carry;
    while (co0 >= A.Eo0) {
      co0 -= A.Eo0;
      ++co1;
    }
  }
};

// Exchange of pass P through the tile's own landing buffer, in its dense
// layout: position p of line pair lp at element row(p) * PB + lp (16 bytes),
// row(p) = p ^ ((p >> 3) & (8 / PB - 1)).  A quarter warp (8 lanes) covers 8 /
// PB consecutive values of t; the Stockham positions they touch in one access
// are either consecutive or 8 apart (radix-8 first pass), and the XOR spreads
// rows 8 apart over different 16-byte bank groups, so the accesses of a
// quarter warp stay (nearly) conflict-free for every PB.  With PB >= 8 a
// quarter warp shares t and the map is the identity.
template <int PB>
__device__ __forceinline__ int dense_row(int p) {
  constexpr int mask = PB >= 8 ? 0 : 8 / PB - 1;
  return mask ? (p ^ ((p >> 3) & mask)) : p;
}

template <int N, int P, int TT, int PB>
__device__ __forceinline__ void exchange_dense(float2* v0, float2* v1, int t, float4* buf) {
  constexpr int V = 8;
  constexpr int R = Radix<N, P>::value, Q = V / R;
  constexpr int R2 = Radix<N, P + 1>::value, Q2 = V / R2;
#pragma unroll
  for (int q = 0; q < Q; ++q)
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const float2 a = v0[q * R + r], b = v1[q * R + r];
      buf[dense_row<PB>(out_pos<N, P, TT>(t, q, r)) * PB] = make_float4(a.x, a.y, b.x, b.y);
    }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < Q2; ++q)
#pragma unroll
    for (int r = 0; r < R2; ++r) {
      const float4 w = buf[dense_row<PB>(in_pos<N, P + 1, TT>(t, q, r)) * PB];
      v0[q * R2 + r] = make_float2(w.x, w.y);
      v1[q * R2 + r] = make_float2(w.z, w.w);
    }
  __syncthreads();
}

template <bool INV, int N, int P, int TT, int PB, bool COMP>
__device__ __forceinline__ void run_fft_dense(float2* v0, float2* v1, int t, const float2* tw, float4* buf) {
  pass_pair<INV, N, P, TT, COMP>(v0, v1, t, tw);
  if constexpr (P + 1 < Radix<N, 0>::npass) {
    exchange_dense<N, P, TT, PB>(v0, v1, t, buf);
    run_fft_dense<INV, N, P + 1, TT, PB, COMP>(v0, v1, t, tw, buf);
  }
}

// Scales (when the stage scales) and stores a b-fast line pair after the last
// pass; dof is the offset of line 2 lp at position 0 (table lookups done by
// the caller).
template <int N>
__device__ __forceinline__ void store_pair_at(const StageArgs& A, float2* out, int64_t dof, int t, bool act0,
                                              bool act1, float2* v0, float2* v1) {
  using C = float2;
  constexpr int V = 8, TT = N / V;
  constexpr int NPASS = Radix<N, 0>::npass;
  constexpr int RL = Radix<N, NPASS - 1>::value, QL = V / RL;
  if (A.scale != 1.0) {
    const float sc = static_cast<float>(A.scale);
#pragma unroll
    for (int e = 0; e < V; ++e) {
      v0[e] = cscale(v0[e], sc);
      v1[e] = cscale(v1[e], sc);
    }
  }
  if (!act0) return;
  const int st = static_cast<int>(A.dst_astride);
  const int64_t base = dof + static_cast<int64_t>(t) * st;
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

constexpr int kTmaStages = 3;

// PB line pairs (L = 2 PB lines) per tile, N/8 threads per pair.  Three
// tile buffers: tile k lands in buffer k % 3, is transformed there (the
// exchanges reuse it) and, once its last exchange has been read, the buffer
// takes the load of tile k + 3; tiles k + 1 and k + 2 are in flight meanwhile.
template <int N, int PB>
constexpr size_t tma_smem_bytes() {
  return sizeof(float2) * (static_cast<size_t>(kTmaStages) * N * 2 * PB + N) + kTmaStages * sizeof(uint64_t);
}

// CTAs per SM the shared memory admits (register budget sized for them)
template <int N, int PB>
struct TmaMinBlocks {
  static constexpr int by_smem = static_cast<int>((227 * 1024) / tma_smem_bytes<N, PB>());
  static constexpr int by_threads = 2048 / (N / 8 * PB);
  static constexpr int v = by_smem < by_threads ? by_smem : by_threads;
  static constexpr int value = v > 0 ? v : 1;
};

template <bool INV, int N, int PB, bool COMP>
__global__ void __launch_bounds__(N / 8 * PB, (TmaMinBlocks<N, PB>::value))
    fft_pair_tma_kernel(const __grid_constant__ CUtensorMap map, const StageArgs A, const TmaCoords T) {
  using C = float2;
  constexpr int V = 8, TT = N / V, L = 2 * PB;
  constexpr int R0 = Radix<N, 0>::value, Q0 = V / R0;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  // [tile buffers 0..2 | twiddles | 3 mbarriers]
  C* land = reinterpret_cast<C*>(smem_raw);
  C* tw = land + kTmaStages * N * L;
  uint64_t* bars = reinterpret_cast<uint64_t*>(tw + N);

  const unsigned ntiles = static_cast<unsigned>(A.tiles_b) * A.Eo0 * A.Eo1;
  const int lp = threadIdx.x % PB, t = threadIdx.x / PB;
  const unsigned first = blockIdx.x, step = gridDim.x;
  const int step_b = static_cast<int>(step % static_cast<unsigned>(A.tiles_b));
  const int step_r = static_cast<int>(step / static_cast<unsigned>(A.tiles_b));
  if (threadIdx.x == 0) {
#pragma unroll
    for (int i = 0; i < kTmaStages; ++i) mbar_init(bars + i, 1);
    mbar_fence_init();
  }
  {
    const C* gtw = reinterpret_cast<const C*>(A.tw);
    for (int i = threadIdx.x; i < N; i += blockDim.x) tw[i] = gtw[i];
  }
  __syncthreads();
  TileWalk cur, nxt;  // the tile being transformed; the next tile to load (thread 0)
  cur.init(first, A);
  nxt = cur;
  unsigned issued = first;
  if (threadIdx.x == 0) {
    for (int i = 0; i < kTmaStages && issued < ntiles; ++i, issued += step) {
      issue_tile<N, L>(&map, T, nxt.tb, nxt.co0, nxt.co1, land + i * N * L, bars + i);
      nxt.advance(step_b, step_r, A);
    }
  }
  const DevLayout ld = A.dst;
  C* out = reinterpret_cast<C*>(A.out);
  int s = 0;
  uint32_t phase = 0;
  for (unsigned tile = first; tile < ntiles; tile += step) {
    C* buf = land + s * N * L;
    // destination offsets of this tile's line pair, loaded while the tile
    // is transformed
    const int b0 = cur.tb * L, nb = min(L, A.Eb - b0);
    const bool act0 = 2 * lp < nb, act1 = 2 * lp + 1 < nb;
    int64_t dof = A.dst_abase + (act0 ? __ldg(ld.t + A.d_tb + b0 + 2 * lp) : 0);
    if (A.o0 >= 0) dof += __ldg(ld.t + A.d_to0 + cur.co0);
    if (A.o1 >= 0) dof += __ldg(ld.t + A.d_to1 + cur.co1);

    const bool ok = mbar_wait_bounded(bars + s, phase);
    C v0[V], v1[V];
    if (ok) {
      const float4* row = reinterpret_cast<const float4*>(buf) + lp;
#pragma unroll
      for (int q = 0; q < Q0; ++q)
#pragma unroll
        for (int r = 0; r < R0; ++r) {
          const float4 w = row[(t + TT * q + r * (N / R0)) * PB];
          v0[q * R0 + r] = make_float2(w.x, w.y);
          v1[q * R0 + r] = make_float2(w.z, w.w);
        }
    }
    // all pass-0 reads are done before the first exchange writes the buffer
    if (__syncthreads_or(!ok)) {
      // a load that never completed: record it, let the other loads in
      // flight land before the shared memory is released, return
      if (threadIdx.x == 0) {
        atomicExch(A.err, 1);
        uint32_t ph = phase;
        int ss = s;
        for (unsigned u = tile + step; u < issued; u += step) {
          if (++ss == kTmaStages) {
            ss = 0;
            ph ^= 1u;
          }
          mbar_wait_bounded(bars + ss, ph);
        }
      }
      return;
    }
    run_fft_dense<INV, N, 0, TT, PB, COMP>(v0, v1, t, tw, reinterpret_cast<float4*>(buf) + lp);  // ends on a barrier
    if (threadIdx.x == 0 && issued < ntiles) {
      fence_proxy_async();
      issue_tile<N, L>(&map, T, nxt.tb, nxt.co0, nxt.co1, buf, bars + s);
      nxt.advance(step_b, step_r, A);
      issued += step;
    }
    store_pair_at<N>(A, out, dof, t, act0, act1, v0, v1);
    cur.advance(step_b, step_r, A);
    if (++s == kTmaStages) {
      s = 0;
      phase ^= 1u;
    }
  }
}

template <int N, bool INV, int PB, bool COMP = false>
cudaError_t launch_tma_pb(const StageArgs& A, const void* map, const TmaCoords& T, cudaStream_t st) {
  if constexpr (PB < 1) {
    return cudaErrorInvalidValue;
  } else {
    constexpr size_t smem = tma_smem_bytes<N, PB>();
    static_assert(smem <= 227 * 1024, "TMA stage tiles do not fit in shared memory");
    auto k = fft_pair_tma_kernel<INV, N, PB, COMP>;
    cudaError_t e = raise_smem_limit(reinterpret_cast<const void*>(k), smem);
    if (e != cudaSuccess) return e;
    int per_sm = 0, sms = 0, dev = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, N / 8 * PB, smem)) != cudaSuccess) return e;
    const long long ntiles = static_cast<long long>(A.tiles_b) * A.Eo0 * A.Eo1;
    long long grid = static_cast<long long>(sms) * (per_sm > 0 ? per_sm : 1);
    if (grid > ntiles) grid = ntiles;
    if (grid < 1) return cudaSuccess;
    CUtensorMap m;
    static_assert(sizeof(CUtensorMap) == 128, "tensor map size");
    memcpy(&m, map, sizeof(m));
    k<<<static_cast<unsigned>(grid), N / 8 * PB, smem, st>>>(m, with_table_offsets(A), T);
    return cudaGetLastError();
  }
}

// line-pair options of the TMA stage: the b-fast streaming default (rows of
// 16 complex64 = 128 bytes for n >= 256) and its half (two CTAs per SM); a
// quarter (32-byte rows) measured 1.6x slower at n = 512 and is not offered
constexpr int tma_pairs(int n, int i) {
  const int p = pair_stream_pairs(n) >> i;
  return p >= 1 ? p : 0;
}

template <int N, bool INV>
cudaError_t launch_tma_n(const StageArgs& A, const void* map, const TmaCoords& T, cudaStream_t st) {
  if (A.comp) return A.B == 2 * tma_pairs(N, 0) ? launch_tma_pb<N, INV, tma_pairs(N, 0), true>(A, map, T, st)
                                                 : cudaErrorInvalidValue;
  if (A.B == 2 * tma_pairs(N, 0)) return launch_tma_pb<N, INV, tma_pairs(N, 0)>(A, map, T, st);
  if (A.B == 2 * tma_pairs(N, 1)) return launch_tma_pb<N, INV, tma_pairs(N, 1)>(A, map, T, st);
  return cudaErrorInvalidValue;
}

}  // namespace

bool pair_tma_supported(int n) { return n >= 16 && n <= 1024 && (n & (n - 1)) == 0; }

int pair_tma_lines(int n) { return pair_tma_supported(n) ? 2 * pair_stream_pairs(n) : 0; }

int pair_tma_line_options(int n, int* opts) {
  if (!pair_tma_supported(n)) return 0;
  int k = 0;
  for (int i = 0; i < 2; ++i) {
    const int p = pair_stream_pairs(n) >> i;
    if (p >= 1) opts[k++] = 2 * p;
  }
  return k;
}

cudaError_t launch_fft_pair_tma(const StageArgs& A, const void* map, const TmaCoords& T, bool inverse,
                                cudaStream_t st) {
  if (!A.err) return cudaErrorInvalidValue;
  switch (A.n) {
#define DFFT_TMA(N_) \
  case N_: return inverse ? launch_tma_n<N_, true>(A, map, T, st) : launch_tma_n<N_, false>(A, map, T, st);
    DFFT_TMA(16) DFFT_TMA(32) DFFT_TMA(64) DFFT_TMA(128) DFFT_TMA(256) DFFT_TMA(512) DFFT_TMA(1024)
#undef DFFT_TMA
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace dev
}  // namespace dfft
