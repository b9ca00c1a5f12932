// Smoothed-aggregation algebraic multigrid (the 'amg' preconditioner): host-side
// interface used by the solver handle (graph engine, precond KCFD_PREC_AMG). The C ABI
// (kcfd_amg_*) is declared in kcfd.h.
#pragma once
#include <cuda_runtime.h>

#include "kcfd.h"

namespace kcfd {
namespace amg {

// Numeric set-up from the level-0 values (the caller's CSR values, same pattern as at
// creation): every level's smoother, prolongator and Galerkin operator, and the
// coarsest level's dense inverse. Kernels only; no host synchronisation.
int setup(kcfd_amg* h, const double* vals64, cudaStream_t st);

// out = M^-1 in (one V(1,1) cycle). `active` (device int, may be null): every kernel
// returns at once when it reads 0 (the graph engine's loop flag). pdl: launch with
// programmatic dependent launch (the kernels wait for their predecessor first).
int vcycle(const kcfd_amg* h, const double* in, double* out, const int* active, cudaStream_t st, bool pdl);

int levels(const kcfd_amg* h);

}  // namespace amg
}  // namespace kcfd
