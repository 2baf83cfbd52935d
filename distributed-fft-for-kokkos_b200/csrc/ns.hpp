// Navier-Stokes step of the reference's batched example on a plan's buffers
// (implemented in ns.cu).
#pragma once

#include <cuda_runtime.h>

#include "plan.hpp"

namespace dfft {
struct NsState;
NsState* ns_create(const Plan* plan, double nu, double dt, double lx);
void ns_rhs(NsState* s, void* uk, void* dukdt, cudaStream_t st);
void ns_step(NsState* s, void* uk, cudaStream_t st);
void ns_taylor_green(NsState* s, void* uk, double v0, cudaStream_t st);
double ns_energy(NsState* s, const void* uk, cudaStream_t st);
void ns_destroy(NsState* s);
}  // namespace dfft
