// Navier-Stokes step of the reference's batched example on a plan's buffers
// (implemented in ns.cu).
#pragma once

#include <cuda_runtime.h>

#include <string>

#include "plan.hpp"

namespace dfft {
struct NsState;
constexpr int kNsMaxBins = 2048;
struct NsDiag {
  double energy, enstrophy, divergence_l2;
};
NsState* ns_create(const Plan* plan, double nu, double dt, double lx);
void ns_rhs(NsState* s, void* uk, void* dukdt, cudaStream_t st);
void ns_step(NsState* s, void* uk, cudaStream_t st);
void ns_taylor_green(NsState* s, void* uk, double v0, cudaStream_t st);
double ns_energy(NsState* s, const void* uk, cudaStream_t st);
// physical velocity / vorticity (plan input layout) of a spectrum; uk is not modified
void ns_velocity(NsState* s, const void* uk, void* u, cudaStream_t st);
void ns_vorticity(NsState* s, const void* uk, void* vor, cudaStream_t st);
// FP64 energy, enstrophy, divergence and nb-bin energy spectrum; synchronises st
NsDiag ns_diagnostics(NsState* s, const void* uk, int nb, double* spec, double* kvals, cudaStream_t st);
// the reference's diag_fields + diag_energy files for every virtual rank
NsDiag ns_write_diagnostics(NsState* s, const void* uk, const std::string& dir, int iter, int nb, cudaStream_t st);
// VJPs with the real inner product of the half spectrum: grad = (d f / d uk)^T
// lam for f(uk) = rhs(D uk); lam <- (d S / d uk)^T lam for one RK4 step S
// (the stage states are recomputed from uk, not stored); uk is not modified
void ns_rhs_adjoint(NsState* s, const void* uk, const void* lam, void* grad, cudaStream_t st);
void ns_step_adjoint(NsState* s, const void* uk, void* lam, cudaStream_t st);
void ns_destroy(NsState* s);
class Batch;
// one RK4 step of n fields (distinct states), the transforms of all fields
// batched through `batch`, whose plans are the states' plans in order
void ns_batch_step(NsState* const* s, void* const* uks, int n, const Batch& batch, cudaStream_t st);
const Plan* ns_plan(const NsState* s);
}  // namespace dfft
