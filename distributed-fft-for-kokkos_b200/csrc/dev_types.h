// Host-visible argument structs and launchers of the device kernels.
#pragma once

#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>

namespace dfft {
namespace dev {

// Layout lookup tables (see layout.hpp).  Offsets index into `t`.
struct DevLayout {
  const int64_t* t;
  int mode;  // 0 separable, 1 general
  int64_t off[4], rk[4], loc[4], rbase, rstride;
};

enum StageKind { kC2C = 0, kR2C = 1, kC2R = 2, kCopy = 3, kCopyReal = 4 };

constexpr int kMaxPasses = 16;

struct StageArgs {
  DevLayout src, dst;
  const void* in;
  void* out;
  const void* tw;     // n twiddles exp(-2*pi*i*k/n) in the stage precision
  int nd;             // view rank
  int a, b, o0, o1;   // FFT axis, tile axis, remaining axes (-1 if absent)
  int n;              // transform length (real length for R2C / C2R)
  int na_in, na_out;  // extents along a in the source / destination
  int Eb, Eo0, Eo1;   // extents along b, o0, o1
  int B;              // lines per tile (real lines for R2C / C2R)
  int nl;             // shared-memory lines (B, or ceil(B/2) for R2C / C2R)
  int pitch;          // shared-memory line pitch (complex elements)
  int tiles_b;        // ceil(Eb / B)
  int load_afast, store_afast;  // thread order of the gather / scatter
  double scale;                 // applied on store
  int npass;
  unsigned long long radix_code;  // radix of pass p in bits [4p, 4p+4)
  // register kernels: 1 = address each line as base + p * stride, both taken
  // from the general layout tables (axis a lies inside one rank block)
  int src_line_affine, dst_line_affine;
  // register kernels, separable sides: the offset table of axis a is affine,
  // off_a[p] = abase + p * astride (checked on the host), so positions along
  // the line are addressed without a table read
  int64_t src_abase, dst_abase, src_astride, dst_astride;
  // register kernels, general-layout variant: 1 = a separable side whose
  // offsets along a are not affine (an exchange buffer split into bins along
  // a): positions along the line are read from the axis table (abase = 0)
  int src_atab, dst_atab;
  // register kernels, separable sides: start of the offset tables of axes a,
  // b, o0, o1 in src.t / dst.t (filled by the launcher from src.off /
  // dst.off, so the kernels select no table at run time)
  int64_t s_ta, s_tb, s_to0, s_to1, d_ta, d_tb, d_to0, d_to1;
  // register kernels: 1 = two complex64 lines per thread (fft_pair.cu), 2 =
  // the same streaming tpc consecutive tiles along b per CTA
  int pairs;
  int tpc;
  // device error word of the plan: kernels with bounded waits set it when a
  // wait runs out (1: a TMA tile load never completed)
  int* err;
  // two-line kernels: 1 = last radix pass in compensated arithmetic (the
  // default tile of fft_pair_kernel and of the TMA kernel only)
  int comp;
  // spectral pre-multiplier of the loaded values, general-layout variant of
  // the one-line C2C kernel only (the first backward stage of a
  // Navier-Stokes right-hand side on a 4D (3, nx, ny, nz / 2 + 1) spectrum):
  // 0 none; 1 the 2/3-rule mask (keep |m_x| <= cut[0], |m_y| <= cut[1],
  // m_z <= cut[2], signed modes m of axes 1 and 2, the half axis 3 has modes
  // 0 .. n / 2); 2 + c: i k_c times the mask, k_c = m_c * kscale (c = 0, 1, 2)
  int pre_mode;
  int pre_n[2];    // extents of axes 1 and 2 (signed modes)
  int pre_cut[3];  // cutoffs of axes 1, 2, 3
  double pre_kscale;
};

// How the TMA-fed stage forms the 5 coordinates of a tile's box from the
// tile's global coordinates: dimension d takes axis which[d] (0 b, 1 a, 2 o0,
// 3 o1, 4 none: coordinate 0), either its position inside the rank block
// (rank_part 0: g % lk) or its rank coordinate (rank_part 1: g / lk).  The a
// axis is loaded in nchunks boxes of boxa positions.
struct TmaCoords {
  int which[5];
  int rank_part[5];
  int lk[5];
  int boxa, nchunks;
};

// Per-rank geometry of one transpose, packed as int64:
//   [r*rs + 0..3]   starts of rank r's block (logical axes)
//   [r*rs + 4..7]   extents of rank r's block (logical axes)
//   [r*rs + 8]      sub-rank of r in its exchange group
//   [r*rs + 9..]    world ranks of the group members, by sub-rank (pc entries)
struct XposeArgs {
  const int64_t* geo;
  int rs;           // int64 per rank in geo
  int nd;           // view rank
  int nprocs;       // world size P
  int pc;           // exchange group size (buffer extent of the rank dim)
  int axis;         // pack: split axis; unpack: merged axis
  int64_t merged;   // global extent along `axis`
  int64_t bext[5];  // buffer extents (reference order)
  int buf_right;    // buffer memory order: rank dim first (LayoutRight) or last
  int64_t bufsize;  // elements per rank buffer
  DevLayout lay;    // global array layout (pack source / unpack destination)
  const void* src;
  void* dst;
};

// Raise `kernel`'s dynamic shared-memory limit to `smem` bytes on the current
// device when a launch needs more than the default 48 KB there.  The attribute
// belongs to the device, so it is recorded per (kernel, device), under a lock
// (plans may be built and executed from several host threads).
cudaError_t raise_smem_limit(const void* kernel, size_t smem);

cudaError_t launch_fft_stage(const StageArgs& A, bool dbl, int kind, bool inverse, int nthreads, size_t smem,
                             unsigned tiles, cudaStream_t st);
// Register-resident power-of-two stage (fft_fast.cu): line lengths 16..4096,
// C2C, rows contiguous on both sides.
bool fast_stage_supported(int n);
int fast_stage_lines(bool dbl, int n);
// Lines-per-CTA variants the launcher accepts (A.B must be one of them).
int fast_stage_line_options(bool dbl, int n, int* opts);
// R2C first stage (c2r = false) or C2R last stage (c2r = true) of the
// register-resident kernel; lines contiguous on both sides; A.B complex lines
// (2 A.B real lines) per tile
// The register kernels run a grid of (tiles_b, Eo0, Eo1) CTAs; Eo0 and Eo1
// must be at most fast_stage_max_grid_yz().
cudaError_t launch_fft_fast_real(const StageArgs& A, bool dbl, bool c2r, cudaStream_t st);
cudaError_t launch_fft_fast(const StageArgs& A, bool dbl, bool inverse, bool afast, cudaStream_t st);
constexpr int fast_stage_max_grid_yz() { return 65535; }
// Two complex64 lines per thread (fft_pair.cu): C2C stages of 2^k points
// (16..4096) on separable layouts; for b-fast tiles every line pair must start
// on a 16-byte boundary (even offsets and stride along a).  A.B is the lines
// per tile (twice the pairs), one of pair_stage_line_options().
bool pair_stage_supported(int n);
int pair_stage_line_options(int n, bool afast, int* opts);
// Lines per tile of the streaming two-line variant (A.pairs = 2).
int pair_stage_stream_lines(int n, bool afast);
cudaError_t launch_fft_pair(const StageArgs& A, bool inverse, bool afast, cudaStream_t st);
// TMA-fed two-line stage (fft_tma.cu): b-fast C2C tiles of 2^k complex64
// points (16..1024) whose source is described by a tiled tensor map `map`
// (a CUtensorMap, 128 bytes) with boxes of A.B x min(n, 256);
// A.B must be one of pair_tma_line_options(n) and A.err a device int.
bool pair_tma_supported(int n);
int pair_tma_lines(int n);
// Lines-per-tile options of the TMA stage (A.B must be one of them).
int pair_tma_line_options(int n, int* opts);
cudaError_t launch_fft_pair_tma(const StageArgs& A, const void* map, const TmaCoords& T, bool inverse,
                                cudaStream_t st);
// Batched register stage (fft_batch.cu): one persistent launch runs the same
// stage (kind, direction, row orientation) of up to kMaxBatchFields fields
// of one line length; field f owns work items prefix[f] .. prefix[f+1] - 1,
// its tiles (tb + tiles_b (co0 + Eo0 co1)).  Every field's StageArgs
// must have B = batch_stage_lines(n) (complex lines per tile) and the tiles_b
// that goes with it; the args are taken by value (kernel parameter space).
constexpr int kMaxBatchFields = 48;
// Two-line variant (fft_batch_sep.cu): complex64 C2C stages of 2^k points
// (16..2048) on separable sides whose line pairs start on 16-byte
// boundaries; every field's StageArgs with B = batch_pair_lines(n, afast).
int batch_pair_lines(int n, bool afast);
struct BatchParams {
  int nfields;
  long long prefix[kMaxBatchFields + 1];
  StageArgs f[kMaxBatchFields];
};
bool batch_stage_supported(int n);
int batch_stage_lines(int n);
// kind: kC2C, kR2C or kC2R (R2C / C2R: lines along a on both sides)
cudaError_t launch_fft_batch(BatchParams& P, bool dbl, int kind, bool inverse, bool afast, cudaStream_t st);
cudaError_t launch_fft_batch_pair(BatchParams& P, bool inverse, bool afast, cudaStream_t st);
// Chirp-z (Bluestein) stage for line lengths the radix passes do not cover
// (a prime factor above 13): X_k = c_k sum_j (x_j c_j) conj(c_{k-j}),
// c_j = exp(-i pi j^2 / n) (conjugated for the inverse), as a circular
// convolution of length m >= 2n - 1 through two m-point FFTs (bluestein.cu).
//   pre:  z[line][j] = x_j c_j (j < n), 0 (n <= j < m), x read through the
//         stage's source layout (R2C: real x; C2R: the full line rebuilt from
//         the half spectrum, imaginary parts of DC / Nyquist dropped)
//   mul:  z[line][k] *= filter[k] (the m-point FFT of the conjugate chirp,
//         divided by m, so that the unnormalised inverse FFT gives the
//         convolution)
//   post: X_k = c_k z[line][k] * scale written through the stage's
//         destination layout (R2C: k <= n/2; C2R: real parts)
// Lines are the stage's (b, o0, o1) coordinates, line = ib + Eb (io0 + Eo0 io1).
struct BlueArgs {
  StageArgs S;         // stage geometry (layouts, axes, extents, n, kind via `kind`)
  int kind;            // kC2C, kR2C or kC2R
  int inverse;
  int m;
  long long nlines;
  const void* chirp;   // n complex values exp(-i pi (j^2 mod 2n) / n) of the stage precision
  const void* filter;  // m complex values
  const void* zin;     // post: z (nlines x m complex)
  void* zout;          // pre: z
  // four-step mode (four_n1 > 0; lines too long for one stage, n = n1 n2):
  // pre copies the line without chirp (m = n), z viewed as (line, j2, j1)
  // with j = j1 + n1 j2; twiddle multiplies z[line][k2][j1] by
  // w_n^(j1 k2) (tw: the n-point table exp(-2 pi i k / n), conjugated for
  // the inverse); post reads X_k at (k mod n2) n1 + k / n2
  int four_n1, four_n2;
  const void* tw;
};
// op: 0 pre, 1 mul (on zout), 2 post, 3 four-step twiddle (on zout)
cudaError_t launch_bluestein(int op, const BlueArgs& B, bool dbl, cudaStream_t st);
// op: 0 pack, 1 all-to-all, 2 unpack
cudaError_t launch_xpose(int op, const XposeArgs& X, int elem_bytes, cudaStream_t st);
cudaError_t launch_scale(void* p, int64_t n_real, bool dbl, double s, cudaStream_t st);
// Multiply the interior modes (k != 0, 2k != n_real along `axis`) of a complex
// array stored in layout L by `factor`.
cudaError_t launch_weight(const DevLayout& L, void* data, bool dbl, int nd, const int64_t* ext, int axis, int n_real,
                          double factor, cudaStream_t st);

}  // namespace dev
}  // namespace dfft
