// dfft_execute_local_c2c_noalloc: a 3D complex-to-complex FFT of one local
// C-order array that allocates no device memory.
//
// Some callers cannot call cudaMalloc: programs whose device memory is owned
// up front by another allocator (a framework's caching pool that reserved the
// GPU), and latency-critical loops that must not hit cudaMalloc / cudaFree,
// which can synchronise the device.  This entry point runs the same three
// register-resident FFT stages as a plan's fused program (z, then y, then x),
// but keeps the intermediate array between the stages in a file-scope
// __device__ array of fixed size instead of plan scratch, and its layout
// tables and twiddles in file-scope arrays as well.
//
// Limits and behaviour:
//  * every extent a power of two in [16, 4096]; n0*n1*n2 complex elements of
//    the chosen precision at most DFFT_NOALLOC_MAX_BYTES (64 MiB); anything
//    else is rejected with DFFT_ERROR_UNSUPPORTED before any launch;
//  * in and out must be aligned to one complex element (8 bytes for
//    complex64, 16 for complex128); misaligned pointers are rejected with
//    DFFT_ERROR_INVALID_ARGUMENT before any launch;
//  * every GPU that loads the library holds the 64 MiB scratch (plus ~200 KB of
//    tables and twiddles) until the process exits;
//  * the first call on a device sets that device up (looks up the device
//    addresses of the arrays and uploads the twiddle tables with synchronous
//    copies); make that first call before any stream capture;
//  * all calls share the arrays: calls that overlap on the GPU (different
//    streams without ordering, several host threads) race and corrupt each
//    other's results.  Each call overwrites the layout tables and the whole
//    intermediate before reading them, so nothing needs to start at zero.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>

#include "../../include/dfft.h"
#include "fft_stage.cuh"

namespace dfft {
namespace dev {

namespace {

constexpr int kMaxLine = 4096;
constexpr int kTwiddleEntries = 2 * kMaxLine - 16;  // all powers of two 16..4096 back to back
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[DFFT_NOALLOC_MAX_BYTES];
static __device__ __align__(256) int64_t g_noalloc_tables[3 * kMaxLine];
static __device__ __align__(256) double2 g_noalloc_tw64[kTwiddleEntries];
static __device__ __align__(256) float2 g_noalloc_tw32[kTwiddleEntries];

struct DeviceState {
  bool ready = false;
  void* scratch = nullptr;
  int64_t* tables = nullptr;
  double2* tw64 = nullptr;
  float2* tw32 = nullptr;
};

std::mutex g_setup_mutex;
DeviceState g_state[kMaxDevices];
// host staging of the twiddle tables (static storage: no allocation)
double g_host_tw64[2 * kTwiddleEntries];
float g_host_tw32[2 * kTwiddleEntries];

int tw_offset(int n) { return n - 16; }  // 16 + 32 + ... + n/2 = n - 16

__global__ void fill_c_order_tables(int64_t* t, int n0, int n1, int n2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n0) t[i] = static_cast<int64_t>(i) * n1 * n2;
  if (i < n1) t[kMaxLine + i] = static_cast<int64_t>(i) * n2;
  if (i < n2) t[2 * kMaxLine + i] = i;
}

dfft_status setup_device(int dev, DeviceState** out, const char** err) {
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (dev < 0 || dev >= kMaxDevices) {
    *err = "device ordinal out of range";
    return DFFT_ERROR_UNSUPPORTED;
  }
  DeviceState& s = g_state[dev];
  if (!s.ready) {
    // In host code the __device__ arrays are only host-side stand-ins: take
    // their device addresses on this device (the caller made it current).
    if (cudaGetSymbolAddress(&s.scratch, g_noalloc_scratch) != cudaSuccess ||
        cudaGetSymbolAddress(reinterpret_cast<void**>(&s.tables), g_noalloc_tables) != cudaSuccess ||
        cudaGetSymbolAddress(reinterpret_cast<void**>(&s.tw64), g_noalloc_tw64) != cudaSuccess ||
        cudaGetSymbolAddress(reinterpret_cast<void**>(&s.tw32), g_noalloc_tw32) != cudaSuccess) {
      cudaGetLastError();
      *err = "cudaGetSymbolAddress of the no-allocation arrays failed";
      return DFFT_ERROR_CUDA;
    }
    const long double pi = 3.141592653589793238462643383279502884L;
    for (int n = 16; n <= kMaxLine; n *= 2) {
      for (int k = 0; k < n; ++k) {
        const long double ang = 2.0L * pi * static_cast<long double>(k) / static_cast<long double>(n);
        const int e = tw_offset(n) + k;
        g_host_tw64[2 * e] = static_cast<double>(cosl(ang));
        g_host_tw64[2 * e + 1] = static_cast<double>(-sinl(ang));
        g_host_tw32[2 * e] = static_cast<float>(cosl(ang));
        g_host_tw32[2 * e + 1] = static_cast<float>(-sinl(ang));
      }
    }
    if (cudaMemcpy(s.tw64, g_host_tw64, sizeof(g_host_tw64), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(s.tw32, g_host_tw32, sizeof(g_host_tw32), cudaMemcpyHostToDevice) != cudaSuccess) {
      cudaGetLastError();
      *err = "upload of the no-allocation twiddle tables failed";
      return DFFT_ERROR_CUDA;
    }
    s.ready = true;
  }
  *out = &s;
  return DFFT_SUCCESS;
}

bool pow2_in_range(int64_t n) { return n >= 16 && n <= kMaxLine && (n & (n - 1)) == 0; }

}  // namespace
}  // namespace dev
}  // namespace dfft

// Worker of dfft_execute_local_c2c_noalloc (capi.cpp keeps the error text).
dfft_status dfft_noalloc_impl(const void* in, void* out, int64_t n0, int64_t n1, int64_t n2, int32_t precision,
                              int32_t direction, int32_t normalization, void* stream, const char** err) {
  using namespace dfft::dev;
  *err = "";
  if (!in || !out) {
    *err = "null buffer";
    return DFFT_ERROR_INVALID_ARGUMENT;
  }
  if (in == out) {
    *err = "in-place execution is not supported: in and out must differ";
    return DFFT_ERROR_INVALID_ARGUMENT;
  }
  if (precision != DFFT_PREC_F64 && precision != DFFT_PREC_F32) {
    *err = "unknown precision";
    return DFFT_ERROR_INVALID_ARGUMENT;
  }
  if (direction != DFFT_FORWARD && direction != DFFT_BACKWARD) {
    *err = "Invalid FFT direction specified.";
    return DFFT_ERROR_INVALID_ARGUMENT;
  }
  if (normalization < DFFT_NORM_BACKWARD || normalization > DFFT_NORM_NONE) {
    *err = "unknown normalization";
    return DFFT_ERROR_INVALID_ARGUMENT;
  }
  if (!pow2_in_range(n0) || !pow2_in_range(n1) || !pow2_in_range(n2)) {
    *err = "no-allocation FFT: every extent must be a power of two in [16, 4096]";
    return DFFT_ERROR_UNSUPPORTED;
  }
  const bool dbl = precision == DFFT_PREC_F64;
  // the stage kernels move whole complex elements (float2 / double2): a
  // pointer off that alignment would fault on the device, so refuse it here
  const uintptr_t align = dbl ? 16 : 8;
  if (reinterpret_cast<uintptr_t>(in) % align != 0 || reinterpret_cast<uintptr_t>(out) % align != 0) {
    *err = dbl ? "no-allocation FFT: in and out must be 16-byte aligned for complex128"
               : "no-allocation FFT: in and out must be 8-byte aligned for complex64";
    return DFFT_ERROR_INVALID_ARGUMENT;
  }
  const unsigned long long bytes = static_cast<unsigned long long>(n0) * n1 * n2 * (dbl ? 16ull : 8ull);
  if (bytes > DFFT_NOALLOC_MAX_BYTES) {
    *err = "no-allocation FFT: the array exceeds the 64 MiB scratch (DFFT_NOALLOC_MAX_BYTES)";
    return DFFT_ERROR_UNSUPPORTED;
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    *err = "cudaGetDevice failed";
    return DFFT_ERROR_CUDA;
  }
  DeviceState* s = nullptr;
  const dfft_status st = setup_device(dev, &s, err);
  if (st != DFFT_SUCCESS) return st;
  cudaStream_t cs = static_cast<cudaStream_t>(stream);

  const int nmax = static_cast<int>(std::max(n0, std::max(n1, n2)));
  fill_c_order_tables<<<(nmax + 255) / 256, 256, 0, cs>>>(s->tables, static_cast<int>(n0), static_cast<int>(n1),
                                                           static_cast<int>(n2));
  if (cudaGetLastError() != cudaSuccess) {
    *err = "table fill launch failed";
    return DFFT_ERROR_CUDA;
  }

  const double N = static_cast<double>(n0) * n1 * n2;
  const bool fwd = direction == DFFT_FORWARD;
  double scale = 1.0;
  if (normalization == DFFT_NORM_BACKWARD) scale = fwd ? 1.0 : 1.0 / N;
  else if (normalization == DFFT_NORM_FORWARD) scale = fwd ? 1.0 / N : 1.0;
  else if (normalization == DFFT_NORM_ORTHO) scale = 1.0 / std::sqrt(N);

  DevLayout L;
  std::memset(&L, 0, sizeof(L));
  L.t = s->tables;
  L.mode = 0;
  L.off[0] = 0;
  L.off[1] = kMaxLine;
  L.off[2] = 2 * kMaxLine;
  const int64_t ext[3] = {n0, n1, n2};
  // stages (FFT axis, tile axis, other axis), z first as in the fused program
  const int stages[3][3] = {{2, 1, 0}, {1, 2, 0}, {0, 2, 1}};
  for (int si = 0; si < 3; ++si) {
    const int a = stages[si][0], b = stages[si][1], o = stages[si][2];
    StageArgs A;
    std::memset(&A, 0, sizeof(A));
    A.src = L;
    A.dst = L;
    A.in = si == 0 ? in : s->scratch;
    A.out = si == 2 ? out : s->scratch;  // the middle stage runs in place
    A.nd = 3;
    A.a = a;
    A.b = b;
    A.o0 = o;
    A.o1 = -1;
    A.n = static_cast<int>(ext[a]);
    A.na_in = A.na_out = A.n;
    A.Eb = static_cast<int>(ext[b]);
    A.Eo0 = static_cast<int>(ext[o]);
    A.Eo1 = 1;
    A.B = fast_stage_lines(dbl, A.n);
    A.tiles_b = (A.Eb + A.B - 1) / A.B;
    A.load_afast = A.store_afast = (a == 2) ? 1 : 0;
    // C order: position p along axis a sits at p * (product of the faster extents)
    A.src_abase = A.dst_abase = 0;
    A.src_astride = A.dst_astride = (a == 0) ? n1 * n2 : (a == 1) ? n2 : 1;
    A.scale = si == 2 ? scale : 1.0;
    A.tw = dbl ? static_cast<const void*>(s->tw64 + tw_offset(A.n))
               : static_cast<const void*>(s->tw32 + tw_offset(A.n));
    if (launch_fft_fast(A, dbl, !fwd, a == 2, cs) != cudaSuccess) {
      cudaGetLastError();
      *err = "FFT stage launch failed";
      return DFFT_ERROR_CUDA;
    }
  }
  return DFFT_SUCCESS;
}
