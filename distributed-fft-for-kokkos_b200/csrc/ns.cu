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
#include <cmath>
#include <cstring>
#include <new>
#include <string>

#include "../../include/dfft.h"
#include "fft_stage.cuh"
#include "ns.hpp"
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

// offset of component d at global (ix, iy, iz) in a 4D layout
__device__ __forceinline__ int64_t off4(const DevLayout& L, int d, int ix, int iy, int iz) {
  int c[4] = {d, ix, iy, iz};
  return layout_offset(L, c, 4);
}

// offsets of the 3 components at (ix, iy, iz): the component axis is not
// split across ranks, so they are o(0) + d * (o(1) - o(0))
__device__ __forceinline__ void off3(const DevLayout& L, int ix, int iy, int iz, int64_t* o) {
  o[0] = off4(L, 0, ix, iy, iz);
  const int64_t step = off4(L, 1, ix, iy, iz) - o[0];
  o[1] = o[0] + step;
  o[2] = o[1] + step;
}

template <typename T>
__global__ void ns_prep_kernel(const DevLayout L, cplx<T>* uk, cplx<T>* dx, cplx<T>* dy, cplx<T>* dz, NsGeom g) {
  const int64_t total = static_cast<int64_t>(g.nx) * g.ny * g.nzh;
  for (int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; t < total;
       t += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int iz = static_cast<int>(t % g.nzh);
    const int iy = static_cast<int>((t / g.nzh) % g.ny);
    const int ix = static_cast<int>(t / (static_cast<int64_t>(g.nzh) * g.ny));
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
    const int iz = static_cast<int>(t % g.nz);
    const int iy = static_cast<int>((t / g.nz) % g.ny);
    const int ix = static_cast<int>(t / (static_cast<int64_t>(g.nz) * g.ny));
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
    const int iz = static_cast<int>(t % g.nzh);
    const int iy = static_cast<int>((t / g.nzh) % g.ny);
    const int ix = static_cast<int>(t / (static_cast<int64_t>(g.nzh) * g.ny));
    const int mx = signed_mode(ix, g.nx), my = signed_mode(iy, g.ny), mz = iz;
    const bool keep = abs(mx) <= g.cx && abs(my) <= g.cy && mz <= g.cz;
    const double kx = mx * g.kscale, ky = my * g.kscale, kz = mz * g.kscale;
    const double ksq = kx * kx + ky * ky + kz * kz;
    const double inv_ksq = (ix == 0 && iy == 0 && iz == 0) ? 0.0 : 1.0 / ksq;
    const T visc = T(-nu * ksq);
    int64_t o[3];
    cplx<T> r[3];
    off3(L, ix, iy, iz, o);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      cplx<T> a = adv[o[d]];
      if (!keep) a = mk<T>(T(0), T(0));
      const cplx<T> u = uk[o[d]];
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
        const cplx<T> y = uk[q];
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
    const int iz = static_cast<int>(t % g.nzh);
    const int iy = static_cast<int>((t / g.nzh) % g.ny);
    const int ix = static_cast<int>(t / (static_cast<int64_t>(g.nzh) * g.ny));
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
    const int iz = static_cast<int>(t % g.nz);
    const int iy = static_cast<int>((t / g.nz) % g.ny);
    const int ix = static_cast<int>(t / (static_cast<int64_t>(g.nz) * g.ny));
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
    const int iz = static_cast<int>(t % g.nzh);
    const int iy = static_cast<int>((t / g.nzh) % g.ny);
    const int ix = static_cast<int>(t / (static_cast<int64_t>(g.nzh) * g.ny));
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
  ~NsState() {
    for (auto p : dk) cudaFree(p);
    for (auto p : du) cudaFree(p);
    for (auto p : rk) cudaFree(p);
    cudaFree(adv);
    cudaFree(u);
    cudaFree(energy);
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
  } catch (...) {
    delete s;
    throw;
  }
  return s;
}

// step in 0..3: RK4 stage; step = -1: only the right-hand side, into `out`
static void ns_rhs_stage(NsState* s, void* uk, int step, void* out, cudaStream_t st) {
  using namespace dev;
  const int64_t nsp = static_cast<int64_t>(s->g.nx) * s->g.ny * s->g.nzh;
  const int64_t nph = static_cast<int64_t>(s->g.nx) * s->g.ny * s->g.nz;
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
  s->plan->execute(uk, s->u, false, st);
  for (int k = 0; k < 3; ++k) s->plan->execute(s->dk[k], s->du[k], false, st);
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
  void* adv = step < 0 ? out : s->adv;
  s->plan->execute(s->u, adv, true, st);
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

void ns_destroy(NsState* s) { delete s; }

}  // namespace dfft
