// Device helpers shared by the .cu translation units.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

#include "dev_types.h"

namespace dfft {
namespace dev {

template <typename T> struct CplxOf;
template <> struct CplxOf<float> { using type = float2; };
template <> struct CplxOf<double> { using type = double2; };
template <typename T> using cplx = typename CplxOf<T>::type;

template <typename T> __device__ __forceinline__ cplx<T> mk(T x, T y) { cplx<T> r; r.x = x; r.y = y; return r; }
template <typename C> __device__ __forceinline__ C cadd(C a, C b) { C r; r.x = a.x + b.x; r.y = a.y + b.y; return r; }
template <typename C> __device__ __forceinline__ C csub(C a, C b) { C r; r.x = a.x - b.x; r.y = a.y - b.y; return r; }
template <typename C> __device__ __forceinline__ C cmul(C a, C b) {
  C r;
  r.x = a.x * b.x - a.y * b.y;
  r.y = a.x * b.y + a.y * b.x;
  return r;
}
template <typename C, typename T> __device__ __forceinline__ C cscale(C a, T s) { C r; r.x = a.x * s; r.y = a.y * s; return r; }
template <typename C> __device__ __forceinline__ C cconj(C a) { a.y = -a.y; return a; }
// s*i*z with s = -1 for the forward transform and +1 for the inverse.
template <bool INV, typename C> __device__ __forceinline__ C rot(C z) {
  C r;
  if (INV) { r.x = -z.y; r.y = z.x; } else { r.x = z.y; r.y = -z.x; }
  return r;
}

// Element offset of global coordinate c (nd axes) in a layout.
__device__ __forceinline__ int64_t layout_offset(const DevLayout& L, const int* c, int nd) {
  if (L.mode == 0) {
    int64_t o = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k)
      if (k < nd) o += __ldg(L.t + L.off[k] + c[k]);
    return o;
  }
  int64_t r = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k)
    if (k < nd) r += __ldg(L.t + L.rk[k] + c[k]);
  int64_t o = __ldg(L.t + L.rbase + r);
#pragma unroll
  for (int k = 0; k < 4; ++k)
    if (k < nd) o += __ldg(L.t + L.loc[k] + c[k]) * __ldg(L.t + L.rstride + r * 4 + k);
  return o;
}

}  // namespace dev
}  // namespace dfft
