// Pseudo-spectral incompressible Navier-Stokes step of the reference's batched
// example (examples/navier-stokes-MPI-batched/main.cpp), on the buffers of a
// distributed R2C plan over 4D views (3, nx, ny, nz) with FFT axes {1,2,3}.
//
//   rhs (main.cpp:536-586): dealias u_hat in place (2/3 rule, :165-192,
//   :220-233); derivatives i k u_hat (:596-616); four backward transforms;
//   advection u . grad u (:629-645); one forward transform; dealias; combine
//   -adv - nu k^2 u_hat (:655-669); projection u - k (k . u) / k^2 (:241-260);
//   RK4 low-storage stages (examples/utils/math_utils.hpp:90-141).
//
// Every kernel walks global coordinates and addresses the rank-blocked
// buffers through the plan's layout tables, so the spectral operators see the
// global wavenumber of each element whatever the topology.  The RK4 stage
// update is fused into the combine / projection kernel.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>
#include <new>
#include <string>

#include "../../include/dfft.h"
#include "fft_stage.cuh"
#include "batch.hpp"
#include "layout.hpp"
#include "ns.hpp"

#include <algorithm>
#include "plan.hpp"

namespace dfft {
namespace dev {
namespace {

struct NsGeom {
  int nx, ny, nz, nzh;  // physical extents and nz/2+1
  int cx, cy, cz;       // 2/3-rule cutoffs on the integer mode index
  double kscale;        // wavenumber = mode index * 2 / lx
};

__device__ __forceinline__ int signed_mode(int i, int n) { return (2 * i < n) ? i : i - n; }

// (ix, iy, iz) of point t of an (nx, ny, nz) box in C order; 32-bit unsigned
// divisions whenever the index fits (every grid up to 1625^3)
__device__ __forceinline__ void decode_point(int64_t t, int nz, int ny, int* ix, int* iy, int* iz) {
  if (t < (int64_t(1) << 32)) {
    const unsigned u = static_cast<unsigned>(t), q = u / static_cast<unsigned>(nz);
    *iz = static_cast<int>(u - q * static_cast<unsigned>(nz));
    *iy = static_cast<int>(q % static_cast<unsigned>(ny));
    *ix = static_cast<int>(q / static_cast<unsigned>(ny));
  } else {
    const int64_t q = t / nz;
    *iz = static_cast<int>(t - q * nz);
    *iy = static_cast<int>(q % ny);
    *ix = static_cast<int>(q / ny);
  }
}

// offsets of the 3 components at (ix, iy, iz): the component axis is not
// split across ranks, so they are o(0) + d * step, step the component stride
// of the rank block that holds the point (one table walk for all three)
__device__ __forceinline__ void off3(const DevLayout& L, int ix, int iy, int iz, int64_t* o) {
  int64_t base, step;
  if (L.mode == 0) {
    const int64_t c0 = __ldg(L.t + L.off[0]);
    base = c0 + __ldg(L.t + L.off[1] + ix) + __ldg(L.t + L.off[2] + iy) + __ldg(L.t + L.off[3] + iz);
    step = __ldg(L.t + L.off[0] + 1) - c0;
  } else {
    const int64_t r = __ldg(L.t + L.rk[1] + ix) + __ldg(L.t + L.rk[2] + iy) + __ldg(L.t + L.rk[3] + iz);
    const int64_t* rs = L.t + L.rstride + r * 4;
    base = __ldg(L.t + L.rbase + r) + __ldg(L.t + L.loc[1] + ix) * __ldg(rs + 1) +
           __ldg(L.t + L.loc[2] + iy) * __ldg(rs + 2) + __ldg(L.t + L.loc[3] + iz) * __ldg(rs + 3);
    step = __ldg(rs + 0);
  }
  o[0] = base;
  o[1] = base + step;
  o[2] = base + 2 * step;
}

template <typename T>
__global__ void ns_prep_kernel(const DevLayout L, cplx<T>* uk, cplx<T>* dx, cplx<T>* dy, cplx<T>* dz, NsGeom g) {
  const int64_t total = static_cast<int64_t>(g.nx) * g.ny * g.nzh;
  for (int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; t < total;
       t += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    int ix, iy, iz;
    decode_point(t, g.nzh, g.ny, &ix, &iy, &iz);
    const int mx = signed_mode(ix, g.nx), my = signed_mode(iy, g.ny), mz = iz;
    const bool keep = abs(mx) <= g.cx && abs(my) <= g.cy && mz <= g.cz;
    const T kx = T(mx * g.kscale), ky = T(my * g.kscale), kz = T(mz * g.kscale);
    int64_t oc[3];
    off3(L, ix, iy, iz, oc);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const int64_t o = oc[d];
      cplx<T> v = uk[o];
      if (!keep) v = mk<T>(T(0), T(0));
      uk[o] = v;
      // i k v = (-k v.y, k v.x)
      dx[o] = mk<T>(-kx * v.y, kx * v.x);
      dy[o] = mk<T>(-ky * v.y, ky * v.x);
      dz[o] = mk<T>(-kz * v.y, kz * v.x);
    }
  }
}

template <typename T>
__global__ void ns_advection_kernel(const DevLayout L, T* u, const T* ux, const T* uy, const T* uz, NsGeom g) {
  const int64_t total = static_cast<int64_t>(g.nx) * g.ny * g.nz;
  for (int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; t < total;
       t += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    int ix, iy, iz;
    decode_point(t, g.nz, g.ny, &ix, &iy, &iz);
    int64_t o[3];
    off3(L, ix, iy, iz, o);
    const T a = u[o[0]], b = u[o[1]], c = u[o[2]];
#pragma unroll
    for (int d = 0; d < 3; ++d) u[o[d]] = a * ux[o[d]] + b * uy[o[d]] + c * uz[o[d]];
  }
}

// rhs = P( -mask * adv_hat - nu k^2 u_hat ), then RK4 stage `step` on uk
template <typename T>
__global__ void ns_rhs_rk_kernel(const DevLayout L, cplx<T>* adv, cplx<T>* uk, cplx<T>* y0, cplx<T>* k1, cplx<T>* k2,
                                 cplx<T>* k3, NsGeom g, double nu, double h, int step) {
  const int64_t total = static_cast<int64_t>(g.nx) * g.ny * g.nzh;
  for (int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; t < total;
       t += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    int ix, iy, iz;
    decode_point(t, g.nzh, g.ny, &ix, &iy, &iz);
    const int mx = signed_mode(ix, g.nx), my = signed_mode(iy, g.ny), mz = iz;
    const bool keep = abs(mx) <= g.cx && abs(my) <= g.cy && mz <= g.cz;
    const double kx = mx * g.kscale, ky = my * g.kscale, kz = mz * g.kscale;
    const double ksq = kx * kx + ky * ky + kz * kz;
    const double inv_ksq = (ix == 0 && iy == 0 && iz == 0) ? 0.0 : 1.0 / ksq;
    const T visc = T(-nu * ksq);
    int64_t o[3];
    cplx<T> r[3], um[3];
    off3(L, ix, iy, iz, o);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      cplx<T> a = adv[o[d]];
      if (!keep) a = mk<T>(T(0), T(0));
      // the dealiased state (the 2/3 rule applied to uk, main.cpp:220-233)
      um[d] = keep ? uk[o[d]] : mk<T>(T(0), T(0));
      const cplx<T> u = um[d];
      r[d] = mk<T>(-a.x + visc * u.x, -a.y + visc * u.y);
    }
    const T ikk = T(inv_ksq);
    const cplx<T> div = mk<T>((T(kx) * r[0].x + T(ky) * r[1].x + T(kz) * r[2].x) * ikk,
                              (T(kx) * r[0].y + T(ky) * r[1].y + T(kz) * r[2].y) * ikk);
    const T kk[3] = {T(kx), T(ky), T(kz)};
    const T hh = T(h);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const cplx<T> f = mk<T>(r[d].x - kk[d] * div.x, r[d].y - kk[d] * div.y);
      const cplx<T> hf = mk<T>(f.x * hh, f.y * hh);
      const int64_t q = o[d];
      if (step == 0) {
        const cplx<T> y = um[d];
        y0[q] = y;
        k1[q] = hf;
        uk[q] = mk<T>(y.x + hf.x / T(2), y.y + hf.y / T(2));
      } else if (step == 1) {
        k2[q] = hf;
        uk[q] = mk<T>(y0[q].x + hf.x / T(2), y0[q].y + hf.y / T(2));
      } else if (step == 2) {
        k3[q] = hf;
        uk[q] = mk<T>(y0[q].x + hf.x, y0[q].y + hf.y);
      } else if (step == 3) {
        const cplx<T> a = k1[q], b = k2[q], c = k3[q];
        uk[q] = mk<T>(y0[q].x + (a.x + T(2) * b.x + T(2) * c.x + hf.x) / T(6),
                      y0[q].y + (a.y + T(2) * b.y + T(2) * c.y + hf.y) / T(6));
      } else {
        adv[q] = f;  // step < 0: store the right-hand side itself
        uk[q] = um[d];  // and leave uk dealiased, as the reference's right-hand side does
      }
    }
  }
}

// initial condition in spectral space (main.cpp:358-363): dealias, then
// project onto the divergence-free space
template <typename T>
__global__ void ns_project_kernel(const DevLayout L, cplx<T>* uk, NsGeom g) {
  const int64_t total = static_cast<int64_t>(g.nx) * g.ny * g.nzh;
  for (int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; t < total;
       t += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    int ix, iy, iz;
    decode_point(t, g.nzh, g.ny, &ix, &iy, &iz);
    const int mx = signed_mode(ix, g.nx), my = signed_mode(iy, g.ny), mz = iz;
    const bool keep = abs(mx) <= g.cx && abs(my) <= g.cy && mz <= g.cz;
    const double kx = mx * g.kscale, ky = my * g.kscale, kz = mz * g.kscale;
    const double inv_ksq = (ix == 0 && iy == 0 && iz == 0) ? 0.0 : 1.0 / (kx * kx + ky * ky + kz * kz);
    int64_t o[3];
    cplx<T> r[3];
    off3(L, ix, iy, iz, o);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      r[d] = keep ? uk[o[d]] : mk<T>(T(0), T(0));
    }
    const T ikk = T(inv_ksq);
    const cplx<T> div = mk<T>((T(kx) * r[0].x + T(ky) * r[1].x + T(kz) * r[2].x) * ikk,
                              (T(kx) * r[0].y + T(ky) * r[1].y + T(kz) * r[2].y) * ikk);
    const T kk[3] = {T(kx), T(ky), T(kz)};
#pragma unroll
    for (int d = 0; d < 3; ++d) uk[o[d]] = mk<T>(r[d].x - kk[d] * div.x, r[d].y - kk[d] * div.y);
  }
}

template <typename T>
__global__ void ns_taylor_green_kernel(const DevLayout L, T* u, NsGeom g, double lx, double v0) {
  const int64_t total = static_cast<int64_t>(g.nx) * g.ny * g.nz;
  const double pi = 3.14159265358979323846;
  for (int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; t < total;
       t += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    int ix, iy, iz;
    decode_point(t, g.nz, g.ny, &ix, &iy, &iz);
    const double x = lx * pi * ix / g.nx, y = lx * pi * iy / g.ny, z = lx * pi * iz / g.nz;
    int64_t o[3];
    off3(L, ix, iy, iz, o);
    u[o[0]] = T(v0 * sin(x) * cos(y) * cos(z));
    u[o[1]] = T(-v0 * cos(x) * sin(y) * cos(z));
    u[o[2]] = T(0);
  }
}

// total kinetic energy (main.cpp:746-766): coef * sum 0.5 * factor * |u_hat|^2,
// factor 1 on the kz = 0 plane and 2 elsewhere (Hermitian half spectrum),
// coef = (lx pi)^3 / N^2; accumulated in FP64.  The reference takes the kz = 0
// plane by the local index of its output block; this takes the global one,
// which is the same whenever z is not split in the output topology.
template <typename T>
__global__ void ns_energy_kernel(const DevLayout L, const cplx<T>* uk, NsGeom g, double coef, double* out) {
  const int64_t total = static_cast<int64_t>(g.nx) * g.ny * g.nzh;
  double acc = 0.0;
  for (int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; t < total;
       t += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    int ix, iy, iz;
    decode_point(t, g.nzh, g.ny, &ix, &iy, &iz);
    const double factor = (iz == 0) ? 1.0 : 2.0;
    double e = 0.0;
    int64_t o[3];
    off3(L, ix, iy, iz, o);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const cplx<T> v = uk[o[d]];
      e += double(v.x) * double(v.x) + double(v.y) * double(v.y);
    }
    acc += 0.5 * factor * e * coef;
  }
  for (int s = 16; s > 0; s >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, s);
  if ((threadIdx.x & 31) == 0) atomicAdd(out, acc);
}

// vorticity spectrum i k x u_hat with the full (not dealiased) wavenumbers
// (compute_vorticity, main.cpp:677-698)
template <typename T>
__global__ void ns_vorticity_kernel(const DevLayout L, const cplx<T>* uk, cplx<T>* w, NsGeom g) {
  const int64_t total = static_cast<int64_t>(g.nx) * g.ny * g.nzh;
  for (int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; t < total;
       t += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    int ix, iy, iz;
    decode_point(t, g.nzh, g.ny, &ix, &iy, &iz);
    const T kx = T(signed_mode(ix, g.nx) * g.kscale), ky = T(signed_mode(iy, g.ny) * g.kscale),
            kz = T(iz * g.kscale);
    int64_t o[3];
    off3(L, ix, iy, iz, o);
    const cplx<T> u = uk[o[0]], v = uk[o[1]], q = uk[o[2]];
    // c = k x u_hat, then i c = (-c.y, c.x)
    const cplx<T> c0 = mk<T>(ky * q.x - kz * v.x, ky * q.y - kz * v.y);
    const cplx<T> c1 = mk<T>(kz * u.x - kx * q.x, kz * u.y - kx * q.y);
    const cplx<T> c2 = mk<T>(kx * v.x - ky * u.x, kx * v.y - ky * u.y);
    w[o[0]] = mk<T>(-c0.y, c0.x);
    w[o[1]] = mk<T>(-c1.y, c1.x);
    w[o[2]] = mk<T>(-c2.y, c2.x);
  }
}

// FP64 diagnostics of a spectrum (diag_energy, main.cpp:741-794, plus the
// enstrophy and the divergence): out[0] += coef * sum 0.5 f |u_hat|^2,
// out[1] += coef * sum 0.5 f |k x u_hat|^2, out[2] += coef * sum f |k . u_hat|^2,
// out[3 + i] += sum 0.5 f |u_hat|^2 over the modes with bins[i] <= |k| <
// bins[i + 1] (no coef, as the reference's E_spec), f = 1 on the kz = 0 plane
// and 2 elsewhere.  |k| is formed without fused multiply-adds so that it
// rounds as k_x^2 + k_y^2 + k_z^2 evaluated term by term.
template <typename T>
__global__ void ns_diag_kernel(const DevLayout L, const cplx<T>* uk, NsGeom g, double coef, const double* bins,
                               int nb, double* out) {
  extern __shared__ double sh[];  // bins (nb + 1), then the nb spectrum sums of this CTA
  double* sb = sh;
  double* ss = sh + nb + 1;
  for (int i = threadIdx.x; i <= nb; i += blockDim.x) sb[i] = bins[i];
  for (int i = threadIdx.x; i < nb; i += blockDim.x) ss[i] = 0.0;
  __syncthreads();
  const double delta = nb > 0 ? sb[nb] / nb : 0.0;
  const int64_t total = static_cast<int64_t>(g.nx) * g.ny * g.nzh;
  double ae = 0.0, aw = 0.0, ad = 0.0;
  for (int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; t < total;
       t += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    int ix, iy, iz;
    decode_point(t, g.nzh, g.ny, &ix, &iy, &iz);
    const double kx = signed_mode(ix, g.nx) * g.kscale, ky = signed_mode(iy, g.ny) * g.kscale, kz = iz * g.kscale;
    const double f = (iz == 0) ? 1.0 : 2.0;
    int64_t o[3];
    off3(L, ix, iy, iz, o);
    double ur[3], ui[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const cplx<T> v = uk[o[d]];
      ur[d] = double(v.x);
      ui[d] = double(v.y);
    }
    const double e = 0.5 * f * (ur[0] * ur[0] + ui[0] * ui[0] + ur[1] * ur[1] + ui[1] * ui[1] + ur[2] * ur[2] +
                                ui[2] * ui[2]);
    ae += e * coef;
    const double c0r = ky * ur[2] - kz * ur[1], c0i = ky * ui[2] - kz * ui[1];
    const double c1r = kz * ur[0] - kx * ur[2], c1i = kz * ui[0] - kx * ui[2];
    const double c2r = kx * ur[1] - ky * ur[0], c2i = kx * ui[1] - ky * ui[0];
    aw += 0.5 * f * coef * (c0r * c0r + c0i * c0i + c1r * c1r + c1i * c1i + c2r * c2r + c2i * c2i);
    const double dr = kx * ur[0] + ky * ur[1] + kz * ur[2], di = kx * ui[0] + ky * ui[1] + kz * ui[2];
    ad += f * coef * (dr * dr + di * di);
    if (nb > 0) {
      const double ksq = __dadd_rn(__dadd_rn(__dmul_rn(kx, kx), __dmul_rn(ky, ky)), __dmul_rn(kz, kz));
      const double km = sqrt(ksq);
      int i = delta > 0.0 ? static_cast<int>(km / delta) : 0;
      i = max(0, min(i, nb - 1));
      while (i > 0 && km < sb[i]) --i;
      while (i < nb - 1 && km >= sb[i + 1]) ++i;
      if (km >= sb[i] && km < sb[i + 1]) atomicAdd(ss + i, e);
    }
  }
  for (int s = 16; s > 0; s >>= 1) {
    ae += __shfl_down_sync(0xffffffffu, ae, s);
    aw += __shfl_down_sync(0xffffffffu, aw, s);
    ad += __shfl_down_sync(0xffffffffu, ad, s);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(out, ae);
    atomicAdd(out + 1, aw);
    atomicAdd(out + 2, ad);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < nb; i += blockDim.x)
    if (ss[i] != 0.0) atomicAdd(out + 3 + i, ss[i]);
}

// ---- adjoint (vector-Jacobian product) of the right-hand side ----
// f(y) = P(-D F(adv(B D y)) - nu k^2 D y), adv_j = sum_a u_a d_a u_j, u = B D y,
// d_a u = B(i k_a D y); D the 2/3 mask, P the projection, F / B the forward /
// backward transforms.  With the real inner product on the half spectrum
// (Re sum conj(a) b, as the plan's adjoint transforms use) the VJP of a
// cotangent c is
//   mu = P c,   lambda_adv = F^H(-D mu),
//   lambda_u_a = sum_j lambda_adv_j d_a u_j,   lambda_(d_a u)_j = u_a lambda_adv_j,
//   f^T c = D(-nu k^2 mu + B^H lambda_u + sum_a (-i k_a) B^H lambda_(d_a u)).

// dst = D src
template <typename T>
__global__ void ns_dealias_kernel(const DevLayout L, const cplx<T>* src, cplx<T>* dst, NsGeom g) {
  const int64_t total = static_cast<int64_t>(g.nx) * g.ny * g.nzh;
  for (int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; t < total;
       t += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    int ix, iy, iz;
    decode_point(t, g.nzh, g.ny, &ix, &iy, &iz);
    const bool keep = abs(signed_mode(ix, g.nx)) <= g.cx && abs(signed_mode(iy, g.ny)) <= g.cy && iz <= g.cz;
    int64_t o[3];
    off3(L, ix, iy, iz, o);
#pragma unroll
    for (int d = 0; d < 3; ++d) dst[o[d]] = keep ? src[o[d]] : mk<T>(T(0), T(0));
  }
}

// mu = P c (projection, 1/k^2 = 0 at the origin); advbar = -D mu
template <typename T>
__global__ void ns_adj_pre_kernel(const DevLayout L, const cplx<T>* c, cplx<T>* mu, cplx<T>* advbar, NsGeom g) {
  const int64_t total = static_cast<int64_t>(g.nx) * g.ny * g.nzh;
  for (int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; t < total;
       t += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    int ix, iy, iz;
    decode_point(t, g.nzh, g.ny, &ix, &iy, &iz);
    const int mx = signed_mode(ix, g.nx), my = signed_mode(iy, g.ny), mz = iz;
    const bool keep = abs(mx) <= g.cx && abs(my) <= g.cy && mz <= g.cz;
    const double kx = mx * g.kscale, ky = my * g.kscale, kz = mz * g.kscale;
    const double inv_ksq = (ix == 0 && iy == 0 && iz == 0) ? 0.0 : 1.0 / (kx * kx + ky * ky + kz * kz);
    int64_t o[3];
    off3(L, ix, iy, iz, o);
    cplx<T> r[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) r[d] = c[o[d]];
    const T ikk = T(inv_ksq);
    const cplx<T> div = mk<T>((T(kx) * r[0].x + T(ky) * r[1].x + T(kz) * r[2].x) * ikk,
                              (T(kx) * r[0].y + T(ky) * r[1].y + T(kz) * r[2].y) * ikk);
    const T kk[3] = {T(kx), T(ky), T(kz)};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const cplx<T> m = mk<T>(r[d].x - kk[d] * div.x, r[d].y - kk[d] * div.y);
      mu[o[d]] = m;
      advbar[o[d]] = keep ? mk<T>(-m.x, -m.y) : mk<T>(T(0), T(0));
    }
  }
}

// physical space, in place: lam <- lambda_u (sum_j lam_j d_a u_j), du[a] <-
// lambda_(d_a u) (u_a lam_j)
template <typename T>
__global__ void ns_adj_point_kernel(const DevLayout L, const T* u, T* d0, T* d1, T* d2, T* lam, NsGeom g) {
  const int64_t total = static_cast<int64_t>(g.nx) * g.ny * g.nz;
  for (int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; t < total;
       t += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    int ix, iy, iz;
    decode_point(t, g.nz, g.ny, &ix, &iy, &iz);
    int64_t o[3];
    off3(L, ix, iy, iz, o);
    T* dd[3] = {d0, d1, d2};
    T uu[3], la[3], gr[3][3];
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      uu[j] = u[o[j]];
      la[j] = lam[o[j]];
    }
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int j = 0; j < 3; ++j) gr[a][j] = dd[a][o[j]];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      lam[o[a]] = la[0] * gr[a][0] + la[1] * gr[a][1] + la[2] * gr[a][2];
#pragma unroll
      for (int j = 0; j < 3; ++j) dd[a][o[j]] = uu[a] * la[j];
    }
  }
}

// out = D(-nu k^2 mu + w + sum_a (-i k_a) h_a)
template <typename T>
__global__ void ns_adj_combine_kernel(const DevLayout L, const cplx<T>* mu, const cplx<T>* w, const cplx<T>* h0,
                                      const cplx<T>* h1, const cplx<T>* h2, cplx<T>* out, NsGeom g, double nu) {
  const int64_t total = static_cast<int64_t>(g.nx) * g.ny * g.nzh;
  for (int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; t < total;
       t += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    int ix, iy, iz;
    decode_point(t, g.nzh, g.ny, &ix, &iy, &iz);
    const int mx = signed_mode(ix, g.nx), my = signed_mode(iy, g.ny), mz = iz;
    const bool keep = abs(mx) <= g.cx && abs(my) <= g.cy && mz <= g.cz;
    const double kx = mx * g.kscale, ky = my * g.kscale, kz = mz * g.kscale;
    const T visc = T(-nu * (kx * kx + ky * ky + kz * kz));
    const T kk[3] = {T(kx), T(ky), T(kz)};
    int64_t o[3];
    off3(L, ix, iy, iz, o);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const int64_t q = o[d];
      if (!keep) {
        out[q] = mk<T>(T(0), T(0));
        continue;
      }
      const cplx<T> m = mu[q], ww = w[q], a0 = h0[q], a1 = h1[q], a2 = h2[q];
      // -i k z = (k z.y, -k z.x)
      const T sy = kk[0] * a0.y + kk[1] * a1.y + kk[2] * a2.y;
      const T sx = kk[0] * a0.x + kk[1] * a1.x + kk[2] * a2.x;
      out[q] = mk<T>(visc * m.x + ww.x + sy, visc * m.y + ww.y - sx);
    }
  }
}

// y = a + s x over whole buffers (n complex elements)
template <typename T>
__global__ void ns_axpy_kernel(const cplx<T>* a, const cplx<T>* x, cplx<T>* y, double s, int64_t n) {
  const T ss = T(s);
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const cplx<T> av = a[i], xv = x[i];
    y[i] = mk<T>(av.x + ss * xv.x, av.y + ss * xv.y);
  }
}

unsigned grid_of(int64_t n) {
  int64_t g = (n + 255) / 256;
  if (g > 148 * 16) g = 148 * 16;
  return static_cast<unsigned>(g < 1 ? 1 : g);
}

}  // namespace
}  // namespace dev

// Host object: work buffers of one field.
struct NsState {
  const Plan* plan;
  double nu, dt, lx;
  bool dbl;
  dev::NsGeom g;
  dev::DevLayout lin, lout;
  std::size_t nin, nout;  // elements of the physical / spectral buffers
  void* dk[3] = {nullptr, nullptr, nullptr};  // i k u_hat
  void* adv = nullptr;                        // advection spectrum / rhs
  void* u = nullptr;                          // physical velocity / advection
  void* du[3] = {nullptr, nullptr, nullptr};  // physical derivatives
  void* rk[4] = {nullptr, nullptr, nullptr, nullptr};  // y0, k1, k2, k3
  double* energy = nullptr;
  double* diag = nullptr;  // 3 + kNsMaxBins sums of ns_diagnostics
  double* bins = nullptr;  // kNsMaxBins + 1 bin edges
  // adjoint workspace (allocated by the first adjoint call): spectral mu, w,
  // lambda_y0, lambda_k, vjp output; physical lambda_adv
  void* adj[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
  void* ladv = nullptr;
  ~NsState() {
    for (auto p : adj) cudaFree(p);
    cudaFree(ladv);
    for (auto p : dk) cudaFree(p);
    for (auto p : du) cudaFree(p);
    for (auto p : rk) cudaFree(p);
    cudaFree(adv);
    cudaFree(u);
    cudaFree(energy);
    cudaFree(diag);
    cudaFree(bins);
  }
};

namespace {
void ck(cudaError_t e, const char* what) {
  if (e != cudaSuccess) fail(kErrCuda, std::string(what) + ": " + cudaGetErrorString(e));
}
}  // namespace

NsState* ns_create(const Plan* plan, double nu, double dt, double lx) {
  const auto& d = plan->desc();
  if (d.gin.size() != 4 || !d.r2c || d.axes != Ext{1, 2, 3} || d.gin[0] != 3 || !d.view_right ||
      d.in_topo[0] != 1 || d.out_topo[0] != 1)
    fail(kErrInvalidArgument,
         "Navier-Stokes needs an R2C plan over LayoutRight 4D views (3, nx, ny, nz) with FFT axes {1, 2, 3} and "
         "the component axis not split (topology (1, px, py, 1) / (1, 1, px, py) as in the reference)");
  auto* s = new NsState;
  s->plan = plan;
  s->nu = nu;
  s->dt = dt;
  s->lx = lx;
  s->dbl = d.dbl;
  s->g.nx = static_cast<int>(d.gin[1]);
  s->g.ny = static_cast<int>(d.gin[2]);
  s->g.nz = static_cast<int>(d.gin[3]);
  s->g.nzh = s->g.nz / 2 + 1;
  // cutoff = int(k_max * 2 / 3), k_max = n / 2  (main.cpp:167-172)
  s->g.cx = (s->g.nx / 2) * 2 / 3;
  s->g.cy = (s->g.ny / 2) * 2 / 3;
  s->g.cz = (s->g.nz / 2) * 2 / 3;
  s->g.kscale = 2.0 / lx;  // fftfreq(n, lx / (2 n))
  s->lin = plan->device_layout(false);
  s->lout = plan->device_layout(true);
  s->nin = total_size(d.gin);
  s->nout = total_size(d.gout);
  const std::size_t rb = s->dbl ? 8 : 4, cb = 2 * rb;
  try {
    for (auto& p : s->dk) ck(cudaMalloc(&p, s->nout * cb), "ns alloc");
    for (auto& p : s->rk) ck(cudaMalloc(&p, s->nout * cb), "ns alloc");
    for (auto& p : s->du) ck(cudaMalloc(&p, s->nin * rb), "ns alloc");
    ck(cudaMalloc(&s->adv, s->nout * cb), "ns alloc");
    ck(cudaMalloc(&s->u, s->nin * rb), "ns alloc");
    ck(cudaMalloc(reinterpret_cast<void**>(&s->energy), sizeof(double)), "ns alloc");
    ck(cudaMalloc(reinterpret_cast<void**>(&s->diag), (3 + kNsMaxBins) * sizeof(double)), "ns alloc");
    ck(cudaMalloc(reinterpret_cast<void**>(&s->bins), (kNsMaxBins + 1) * sizeof(double)), "ns alloc");
  } catch (...) {
    delete s;
    throw;
  }
  return s;
}

// step in 0..3: RK4 stage; step = -1: only the right-hand side, into `out`
// The three pointwise phases of one right-hand side, around the transforms:
// prep (dealias uk in place, i k uk), advection (u . grad u in physical
// space), combine (dealias, -adv - nu k^2 uk, projection, RK4 stage `step`;
// step = -1 stores the right-hand side into `adv`).
static void ns_prep_phase(NsState* s, void* uk, cudaStream_t st) {
  using namespace dev;
  const int64_t nsp = static_cast<int64_t>(s->g.nx) * s->g.ny * s->g.nzh;
  if (s->dbl)
    ns_prep_kernel<double><<<grid_of(nsp), 256, 0, st>>>(s->lout, static_cast<double2*>(uk),
                                                          static_cast<double2*>(s->dk[0]),
                                                          static_cast<double2*>(s->dk[1]),
                                                          static_cast<double2*>(s->dk[2]), s->g);
  else
    ns_prep_kernel<float><<<grid_of(nsp), 256, 0, st>>>(s->lout, static_cast<float2*>(uk),
                                                         static_cast<float2*>(s->dk[0]),
                                                         static_cast<float2*>(s->dk[1]),
                                                         static_cast<float2*>(s->dk[2]), s->g);
  ck(cudaGetLastError(), "ns prep");
}

static void ns_advection_phase(NsState* s, cudaStream_t st) {
  using namespace dev;
  const int64_t nph = static_cast<int64_t>(s->g.nx) * s->g.ny * s->g.nz;
  if (s->dbl)
    ns_advection_kernel<double><<<grid_of(nph), 256, 0, st>>>(s->lin, static_cast<double*>(s->u),
                                                               static_cast<double*>(s->du[0]),
                                                               static_cast<double*>(s->du[1]),
                                                               static_cast<double*>(s->du[2]), s->g);
  else
    ns_advection_kernel<float><<<grid_of(nph), 256, 0, st>>>(s->lin, static_cast<float*>(s->u),
                                                              static_cast<float*>(s->du[0]),
                                                              static_cast<float*>(s->du[1]),
                                                              static_cast<float*>(s->du[2]), s->g);
  ck(cudaGetLastError(), "ns advection");
}

static void ns_combine_phase(NsState* s, void* uk, void* adv, int step, cudaStream_t st) {
  using namespace dev;
  const int64_t nsp = static_cast<int64_t>(s->g.nx) * s->g.ny * s->g.nzh;
  if (s->dbl)
    ns_rhs_rk_kernel<double><<<grid_of(nsp), 256, 0, st>>>(
        s->lout, static_cast<double2*>(adv), static_cast<double2*>(uk), static_cast<double2*>(s->rk[0]),
        static_cast<double2*>(s->rk[1]), static_cast<double2*>(s->rk[2]), static_cast<double2*>(s->rk[3]), s->g, s->nu,
        s->dt, step);
  else
    ns_rhs_rk_kernel<float><<<grid_of(nsp), 256, 0, st>>>(
        s->lout, static_cast<float2*>(adv), static_cast<float2*>(uk), static_cast<float2*>(s->rk[0]),
        static_cast<float2*>(s->rk[1]), static_cast<float2*>(s->rk[2]), static_cast<float2*>(s->rk[3]), s->g, s->nu,
        s->dt, step);
  ck(cudaGetLastError(), "ns rhs");
}

// Backward transforms of the dealiased velocity and its three derivative
// spectra.  When the plan's first backward stage is a register C2C stage, the
// prep phase is folded into that stage's loads: each transform reads uk and
// multiplies by the 2/3-rule mask (and i k_c), so neither the masked spectrum
// nor the derivative spectra are written to memory (the combine phase applies
// the mask to uk itself).
static void ns_backward_phase(NsState* s, void* uk, cudaStream_t st) {
  if (!s->plan->can_premultiply()) {
    ns_prep_phase(s, uk, st);
    s->plan->execute(uk, s->u, false, st);
    for (int k = 0; k < 3; ++k) s->plan->execute(s->dk[k], s->du[k], false, st);
    return;
  }
  dev::StageArgs pre;
  std::memset(&pre, 0, sizeof(pre));
  pre.pre_n[0] = s->g.nx;
  pre.pre_n[1] = s->g.ny;
  pre.pre_cut[0] = s->g.cx;
  pre.pre_cut[1] = s->g.cy;
  pre.pre_cut[2] = s->g.cz;
  pre.pre_kscale = s->g.kscale;
  pre.pre_mode = 1;
  s->plan->execute_backward_premul(uk, s->u, pre, st);
  for (int k = 0; k < 3; ++k) {
    pre.pre_mode = 2 + k;
    s->plan->execute_backward_premul(uk, s->du[k], pre, st);
  }
}

// step in 0..3: RK4 stage; step = -1: only the right-hand side, into `out`
static void ns_rhs_stage(NsState* s, void* uk, int step, void* out, cudaStream_t st) {
  ns_backward_phase(s, uk, st);
  ns_advection_phase(s, st);
  void* adv = step < 0 ? out : s->adv;
  s->plan->execute(s->u, adv, true, st);
  ns_combine_phase(s, uk, adv, step, st);
}

// One RK4 step of several fields: the pointwise phases per field, each
// transform of all fields through one batched execution (one launch per
// stage).
void ns_batch_step(NsState* const* s, void* const* uks, int n, const Batch& batch, cudaStream_t st) {
  std::vector<const void*> ins(n);
  std::vector<void*> outs(n);
  // the pointwise phases of different fields run concurrently on the batch's
  // lanes, fields dealt to the least loaded lane, largest first
  const int lanes = std::min(n, Batch::kAux + 1);
  std::vector<int> lane_of(n, 0), order(n);
  {
    std::vector<double> load(lanes, 0.0);
    for (int f = 0; f < n; ++f) order[f] = f;
    auto size_of = [&](int f) { return static_cast<double>(s[f]->g.nx) * s[f]->g.ny * s[f]->g.nz; };
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return size_of(a) > size_of(b); });
    for (int f : order) {
      const int l = static_cast<int>(std::min_element(load.begin(), load.end()) - load.begin());
      lane_of[f] = l;
      load[l] += size_of(f);
    }
  }
  auto per_field = [&](auto&& phase) {
    batch.fork(st, lanes);
    for (int f : order) phase(f, batch.lane(st, lane_of[f]));
    batch.join(st, lanes);
  };
  for (int step = 0; step < 4; ++step) {
    per_field([&](int f, cudaStream_t ls) { ns_prep_phase(s[f], uks[f], ls); });
    for (int f = 0; f < n; ++f) {
      ins[f] = uks[f];
      outs[f] = s[f]->u;
    }
    batch.execute(ins.data(), outs.data(), false, st);
    for (int k = 0; k < 3; ++k) {
      for (int f = 0; f < n; ++f) {
        ins[f] = s[f]->dk[k];
        outs[f] = s[f]->du[k];
      }
      batch.execute(ins.data(), outs.data(), false, st);
    }
    per_field([&](int f, cudaStream_t ls) { ns_advection_phase(s[f], ls); });
    for (int f = 0; f < n; ++f) {
      ins[f] = s[f]->u;
      outs[f] = s[f]->adv;
    }
    batch.execute(ins.data(), outs.data(), true, st);
    per_field([&](int f, cudaStream_t ls) { ns_combine_phase(s[f], uks[f], s[f]->adv, step, ls); });
  }
}

const Plan* ns_plan(const NsState* s) { return s->plan; }

void ns_rhs(NsState* s, void* uk, void* dukdt, cudaStream_t st) { ns_rhs_stage(s, uk, -1, dukdt, st); }

void ns_step(NsState* s, void* uk, cudaStream_t st) {
  for (int step = 0; step < 4; ++step) ns_rhs_stage(s, uk, step, nullptr, st);
}

void ns_taylor_green(NsState* s, void* uk, double v0, cudaStream_t st) {
  using namespace dev;
  const int64_t nph = static_cast<int64_t>(s->g.nx) * s->g.ny * s->g.nz;
  if (s->dbl)
    ns_taylor_green_kernel<double><<<grid_of(nph), 256, 0, st>>>(s->lin, static_cast<double*>(s->u), s->g, s->lx, v0);
  else
    ns_taylor_green_kernel<float><<<grid_of(nph), 256, 0, st>>>(s->lin, static_cast<float*>(s->u), s->g, s->lx, v0);
  ck(cudaGetLastError(), "ns init");
  s->plan->execute(s->u, uk, true, st);
  const int64_t nsp = static_cast<int64_t>(s->g.nx) * s->g.ny * s->g.nzh;
  if (s->dbl)
    ns_project_kernel<double><<<grid_of(nsp), 256, 0, st>>>(s->lout, static_cast<double2*>(uk), s->g);
  else
    ns_project_kernel<float><<<grid_of(nsp), 256, 0, st>>>(s->lout, static_cast<float2*>(uk), s->g);
  ck(cudaGetLastError(), "ns init projection");
}

double ns_energy(NsState* s, const void* uk, cudaStream_t st) {
  using namespace dev;
  const int64_t nsp = static_cast<int64_t>(s->g.nx) * s->g.ny * s->g.nzh;
  const double N = static_cast<double>(s->g.nx) * s->g.ny * s->g.nz;
  const double vol = s->lx * 3.14159265358979323846;
  ck(cudaMemsetAsync(s->energy, 0, sizeof(double), st), "ns energy");
  if (s->dbl)
    ns_energy_kernel<double><<<grid_of(nsp), 256, 0, st>>>(s->lout, static_cast<const double2*>(uk), s->g,
                                                            vol * vol * vol / (N * N), s->energy);
  else
    ns_energy_kernel<float><<<grid_of(nsp), 256, 0, st>>>(s->lout, static_cast<const float2*>(uk), s->g,
                                                           vol * vol * vol / (N * N), s->energy);
  ck(cudaGetLastError(), "ns energy");
  double e = 0.0;
  ck(cudaMemcpyAsync(&e, s->energy, sizeof(double), cudaMemcpyDeviceToHost, st), "ns energy");
  ck(cudaStreamSynchronize(st), "ns energy");
  return e;
}

void ns_velocity(NsState* s, const void* uk, void* u, cudaStream_t st) { s->plan->execute(uk, u, false, st); }

void ns_vorticity(NsState* s, const void* uk, void* vor, cudaStream_t st) {
  using namespace dev;
  const int64_t nsp = static_cast<int64_t>(s->g.nx) * s->g.ny * s->g.nzh;
  if (s->dbl)
    ns_vorticity_kernel<double><<<grid_of(nsp), 256, 0, st>>>(s->lout, static_cast<const double2*>(uk),
                                                               static_cast<double2*>(s->adv), s->g);
  else
    ns_vorticity_kernel<float><<<grid_of(nsp), 256, 0, st>>>(s->lout, static_cast<const float2*>(uk),
                                                              static_cast<float2*>(s->adv), s->g);
  ck(cudaGetLastError(), "ns vorticity");
  s->plan->execute(s->adv, vor, false, st);
}

// Radial bins of the energy spectrum (main.cpp:471-500): k_max is the largest
// |k| of the grid, the edges linspace(0, k_max, nb + 1) with the last edge
// k_max itself, the k values the bin midpoints.
static std::vector<double> spectrum_bins(const NsState* s, int nb) {
  const double kx = (s->g.nx / 2) * s->g.kscale, ky = (s->g.ny / 2) * s->g.kscale, kz = (s->g.nz / 2) * s->g.kscale;
  volatile double sq = kx * kx;  // evaluated term by term, as on the device
  sq = sq + ky * ky;
  sq = sq + kz * kz;
  const double k_max = std::sqrt(static_cast<double>(sq));
  std::vector<double> b(static_cast<std::size_t>(nb) + 1);
  const double delta = (k_max - 0.0) / static_cast<double>(nb);
  for (int i = 0; i < nb; ++i) b[i] = 0.0 + delta * static_cast<double>(i);
  b[nb] = k_max;
  return b;
}

NsDiag ns_diagnostics(NsState* s, const void* uk, int nb, double* spec, double* kvals, cudaStream_t st) {
  using namespace dev;
  if (nb < 0 || nb > kNsMaxBins)
    fail(kErrInvalidArgument, "num_bins must be in [0, " + std::to_string(kNsMaxBins) + "]");
  if (nb > 0 && (!spec || !kvals)) fail(kErrInvalidArgument, "null spectrum output");
  const int64_t nsp = static_cast<int64_t>(s->g.nx) * s->g.ny * s->g.nzh;
  const double N = static_cast<double>(s->g.nx) * s->g.ny * s->g.nz;
  const double vol = s->lx * 3.14159265358979323846;
  std::vector<double> bins = nb > 0 ? spectrum_bins(s, nb) : std::vector<double>(1, 0.0);
  ck(cudaMemcpyAsync(s->bins, bins.data(), bins.size() * sizeof(double), cudaMemcpyHostToDevice, st), "ns diag");
  ck(cudaMemsetAsync(s->diag, 0, (3 + static_cast<std::size_t>(nb)) * sizeof(double), st), "ns diag");
  const std::size_t smem = (2 * static_cast<std::size_t>(nb) + 1) * sizeof(double);
  const double coef = vol * vol * vol / (N * N);
  if (s->dbl)
    ns_diag_kernel<double><<<grid_of(nsp), 256, smem, st>>>(s->lout, static_cast<const double2*>(uk), s->g, coef,
                                                             s->bins, nb, s->diag);
  else
    ns_diag_kernel<float><<<grid_of(nsp), 256, smem, st>>>(s->lout, static_cast<const float2*>(uk), s->g, coef,
                                                            s->bins, nb, s->diag);
  ck(cudaGetLastError(), "ns diag");
  std::vector<double> h(3 + static_cast<std::size_t>(nb));
  ck(cudaMemcpyAsync(h.data(), s->diag, h.size() * sizeof(double), cudaMemcpyDeviceToHost, st), "ns diag");
  ck(cudaStreamSynchronize(st), "ns diag");
  for (int i = 0; i < nb; ++i) {
    spec[i] = h[3 + i];
    kvals[i] = 0.5 * (bins[i] + bins[i + 1]);
  }
  NsDiag d;
  d.energy = h[0];
  d.enstrophy = h[1];
  d.divergence_l2 = std::sqrt(h[2]);
  return d;
}

// "<dir>/<label>_rx<3 digits>_ry<3 digits>_<10 digits>.dat" (main.cpp:803-818,
// IO::zfill)
static std::string dump_name(const std::string& dir, const char* label, std::size_t rx, std::size_t ry, int iter) {
  char tail[64];
  std::snprintf(tail, sizeof(tail), "_rx%03zu_ry%03zu_%010d.dat", rx, ry, iter);
  return dir + "/" + label + tail;
}

static void write_raw(const std::string& path, const void* data, std::size_t bytes) {
  std::FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) fail(kErrInvalidArgument, "Failed to open file: " + path);
  const std::size_t w = bytes ? std::fwrite(data, 1, bytes, f) : 0;
  const int c = std::fclose(f);
  if (w != bytes || c != 0) fail(kErrInternal, "short write to " + path);
}

NsDiag ns_write_diagnostics(NsState* s, const void* uk, const std::string& dir, int iter, int nb, cudaStream_t st) {
  const auto& d = s->plan->desc();
  if (d.in_topo[0] != 1 || d.in_topo[3] != 1)
    fail(kErrUnsupported, "field dumps name files by (rx, ry) of the reference's in_topology (1, px, py, 1)");
  if (iter < 0) fail(kErrInvalidArgument, "iteration must be non-negative");
  const std::size_t rb = s->dbl ? 8 : 4;
  std::vector<unsigned char> host(s->nin * rb);
  const auto blocks = layout_blocks(s->plan->in_layout());
  auto dump = [&](const char* const labels[3]) {
    ck(cudaMemcpyAsync(host.data(), s->u, host.size(), cudaMemcpyDeviceToHost, st), "ns dump");
    ck(cudaStreamSynchronize(st), "ns dump");
    for (const RankBlock& b : blocks) {
      // LayoutRight block (3, nx_loc, ny_loc, nz): component c is one contiguous run
      const std::size_t comp = b.size / 3;
      for (int c = 0; c < 3; ++c)
        write_raw(dump_name(dir, labels[c], b.coords[1], b.coords[2], iter),
                  host.data() + (b.base + c * comp) * rb, comp * rb);
    }
  };
  // diag_fields (main.cpp:711-739): velocity, then vorticity, in physical space
  ns_velocity(s, uk, s->u, st);
  static const char* const vel[3] = {"u", "v", "w"};
  dump(vel);
  ns_vorticity(s, uk, s->u, st);
  static const char* const vor[3] = {"vor_x", "vor_y", "vor_z"};
  dump(vor);
  // diag_energy (main.cpp:741-794): spectrum and bin centres, written once
  // (by rank 0 in the reference, whose coordinates are (0, 0))
  std::vector<double> spec(static_cast<std::size_t>(nb)), kv(static_cast<std::size_t>(nb));
  NsDiag r = ns_diagnostics(s, uk, nb, spec.data(), kv.data(), st);
  write_raw(dump_name(dir, "E_spec", 0, 0, iter), spec.data(), spec.size() * sizeof(double));
  write_raw(dump_name(dir, "k_vals", 0, 0, iter), kv.data(), kv.size() * sizeof(double));
  return r;
}

// ---- adjoints ----
static void ns_adj_alloc(NsState* s) {
  if (s->ladv) return;
  const std::size_t cb = (s->dbl ? 16 : 8) * s->nout, rb = (s->dbl ? 8 : 4) * s->nin;
  for (auto& p : s->adj) ck(cudaMalloc(&p, cb), "ns adjoint alloc");
  ck(cudaMalloc(&s->ladv, rb), "ns adjoint alloc");
}

template <typename T>
static void launch_dealias(NsState* s, const void* src, void* dst, cudaStream_t st) {
  using namespace dev;
  const int64_t nsp = static_cast<int64_t>(s->g.nx) * s->g.ny * s->g.nzh;
  ns_dealias_kernel<T><<<grid_of(nsp), 256, 0, st>>>(s->lout, static_cast<const cplx<T>*>(src),
                                                      static_cast<cplx<T>*>(dst), s->g);
  ck(cudaGetLastError(), "ns dealias");
}

template <typename T>
static void launch_axpy(const void* a, const void* x, void* y, double sc, std::size_t n, cudaStream_t st) {
  using namespace dev;
  ns_axpy_kernel<T><<<grid_of(static_cast<int64_t>(n)), 256, 0, st>>>(
      static_cast<const cplx<T>*>(a), static_cast<const cplx<T>*>(x), static_cast<cplx<T>*>(y), sc,
      static_cast<int64_t>(n));
  ck(cudaGetLastError(), "ns axpy");
}

// out = (d f / d y)^T c at y; y is one of the adjoint's own buffers (it is
// dealiased in place, a no-op for the dealiased states the callers pass).
template <typename T>
static void ns_vjp(NsState* s, void* y, const void* c, void* out, cudaStream_t st) {
  using namespace dev;
  using C = cplx<T>;
  const int64_t nsp = static_cast<int64_t>(s->g.nx) * s->g.ny * s->g.nzh;
  const int64_t nph = static_cast<int64_t>(s->g.nx) * s->g.ny * s->g.nz;
  // recompute u and d_a u from y (the forward pencils are not stored)
  ns_prep_kernel<T><<<grid_of(nsp), 256, 0, st>>>(s->lout, static_cast<C*>(y), static_cast<C*>(s->dk[0]),
                                                   static_cast<C*>(s->dk[1]), static_cast<C*>(s->dk[2]), s->g);
  ck(cudaGetLastError(), "ns vjp prep");
  s->plan->execute(y, s->u, false, st);
  for (int k = 0; k < 3; ++k) s->plan->execute(s->dk[k], s->du[k], false, st);
  void* mu = s->adj[0];
  void* w = s->adj[1];
  ns_adj_pre_kernel<T><<<grid_of(nsp), 256, 0, st>>>(s->lout, static_cast<const C*>(c), static_cast<C*>(mu),
                                                      static_cast<C*>(s->adv), s->g);
  ck(cudaGetLastError(), "ns vjp projection");
  s->plan->execute_adjoint(s->adv, s->ladv, true, st);  // F^H
  ns_adj_point_kernel<T><<<grid_of(nph), 256, 0, st>>>(s->lin, static_cast<const T*>(s->u),
                                                        static_cast<T*>(s->du[0]), static_cast<T*>(s->du[1]),
                                                        static_cast<T*>(s->du[2]), static_cast<T*>(s->ladv), s->g);
  ck(cudaGetLastError(), "ns vjp advection");
  s->plan->execute_adjoint(s->ladv, w, false, st);  // B^H
  for (int k = 0; k < 3; ++k) s->plan->execute_adjoint(s->du[k], s->dk[k], false, st);
  ns_adj_combine_kernel<T><<<grid_of(nsp), 256, 0, st>>>(
      s->lout, static_cast<const C*>(mu), static_cast<const C*>(w), static_cast<const C*>(s->dk[0]),
      static_cast<const C*>(s->dk[1]), static_cast<const C*>(s->dk[2]), static_cast<C*>(out), s->g, s->nu);
  ck(cudaGetLastError(), "ns vjp combine");
}

template <typename T>
static void ns_rhs_adjoint_t(NsState* s, const void* uk, const void* lam, void* grad, cudaStream_t st) {
  ns_adj_alloc(s);
  void* y = s->rk[0];
  launch_dealias<T>(s, uk, y, st);
  ns_vjp<T>(s, y, lam, grad, st);
}

// One RK4 step S(y) = D y + (k1 + 2 k2 + 2 k3 + k4) / 6, k_i = dt f(a_i),
// a1 = D y, a2 = a1 + k1 / 2, a3 = a1 + k2 / 2, a4 = a1 + k3: the stage
// states are recomputed from y (three right-hand sides), then the four VJPs
// run backwards.
template <typename T>
static void ns_step_adjoint_t(NsState* s, const void* uk, void* lam, cudaStream_t st) {
  ns_adj_alloc(s);
  const double h = s->dt;
  const std::size_t n = s->nout;
  void* a[4] = {s->rk[0], s->rk[1], s->rk[2], s->rk[3]};
  void* ly0 = s->adj[2];
  void* lk = s->adj[3];
  void* gbuf = s->adj[4];
  launch_dealias<T>(s, uk, a[0], st);
  for (int i = 1; i < 4; ++i) {
    // f(a_{i-1}) into gbuf (the right-hand side dealiases its input in place:
    // the stage states are already dealiased)
    ns_rhs_stage(s, a[i - 1], -1, gbuf, st);
    launch_axpy<T>(a[0], gbuf, a[i], i == 3 ? h : 0.5 * h, n, st);
  }
  // backward pass: ly0 accumulates the cotangent of a1, lk is the cotangent
  // of the current k_i
  ck(cudaMemcpyAsync(ly0, lam, n * sizeof(dev::cplx<T>), cudaMemcpyDeviceToDevice, st), "ns step adjoint");
  const double ck_direct[4] = {1.0 / 6.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0};  // d S / d k_i
  const double up[3] = {0.5, 0.5, 1.0};  // a2 = a1 + k1 / 2, a3 = a1 + k2 / 2, a4 = a1 + k3
  // k4 first: lk = lam / 6
  launch_axpy<T>(lam, lam, lk, ck_direct[3] - 1.0, n, st);
  for (int i = 3; i >= 0; --i) {
    // g = dt f'(a_i)^T lk
    ns_vjp<T>(s, a[i], lk, gbuf, st);
    launch_axpy<T>(ly0, gbuf, ly0, h, n, st);
    if (i > 0) {
      // cotangent of k_i (1-based; a[i] = a1 + up[i - 1] k_i): its direct
      // weight in S plus up[i - 1] times this stage's g
      launch_axpy<T>(lam, lam, lk, ck_direct[i - 1] - 1.0, n, st);
      launch_axpy<T>(lk, gbuf, lk, h * up[i - 1], n, st);
    }
  }
  launch_dealias<T>(s, ly0, lam, st);
}

void ns_rhs_adjoint(NsState* s, const void* uk, const void* lam, void* grad, cudaStream_t st) {
  if (s->dbl)
    ns_rhs_adjoint_t<double>(s, uk, lam, grad, st);
  else
    ns_rhs_adjoint_t<float>(s, uk, lam, grad, st);
}

void ns_step_adjoint(NsState* s, const void* uk, void* lam, cudaStream_t st) {
  if (s->dbl)
    ns_step_adjoint_t<double>(s, uk, lam, st);
  else
    ns_step_adjoint_t<float>(s, uk, lam, st);
}

void ns_destroy(NsState* s) { delete s; }

}  // namespace dfft
