// Generic FVM operators on the device, accumulating into a device linear system
// (CSR values + tracked diagonal + rhs), in the reference's operator-by-operator style:
//   core/fvm_operators.py:59-100   diffusion_operator          -> kcfd_op_diffusion
//   core/fvm_operators.py:103-129  convection_operator_upwind  -> kcfd_op_convection_upwind
//   core/fvm_operators.py:132-148  temporal_operator           -> kcfd_op_temporal
//   core/fvm_operators.py:151-175  source_term / linearized_source -> kcfd_op_source
//   core/fvm_operators.py:178-225  apply_boundary_conditions   -> kcfd_op_boundary
//   core/fvm_operators.py:228-240  under_relax                 -> kcfd_op_under_relax
//   core/interpolation.py:227-303  muscl_deferred_correction   -> kcfd_muscl_correction
// Each operator ADDS its contributions, like the reference's COO triplets summed by
// to_sparse(). The tracked diagonal `diag` is the reference's FVMSystem.diag: every
// add_diagonal contribution goes to both the CSR diagonal slot and diag, and
// under_relax reads diag (which a caller may floor on its own, as the two-fluid model
// does). Face operators run one launch per face colour (conflict-free scatter).
#include <cuda_runtime.h>

#include <algorithm>

#include "kcfd_common.h"

namespace kcfd {
namespace {

constexpr int kT = 256;
inline int nblk(int64_t n) { return (int)std::max<int64_t>(1, std::min<int64_t>((n + kT - 1) / kT, 1 << 20)); }

__device__ __forceinline__ double lim_psi(int lim, double r) {
    switch (lim) {
        case 0: return fmax(0.0, fmin(1.0, r));
        case 1: return fmax(0.0, fmax(fmin(2.0 * r, 1.0), fmin(r, 2.0)));
        case 2: return r > 0 ? (r * r + r) / (r * r + 1.0) : 0.0;
        default: return r > 0 ? 2.0 * r / (1.0 + r) : 0.0;
    }
}

__global__ void k_diff(kcfd_dmesh_t m, int f0, int f1, const double* __restrict__ gamma, double* __restrict__ v,
                       double* __restrict__ diag) {
    for (int f = f0 + blockIdx.x * blockDim.x + threadIdx.x; f < f1; f += gridDim.x * blockDim.x) {
        const double d = m.dlen[f];
        if (d < 1e-30) continue;
        const int o = m.owner[f], nb = m.neigh[f];
        const double gO = gamma[o], gN = gamma[nb];
        const double gf = (gO + gN > 1e-30) ? 2.0 * gO * gN / (gO + gN) : 0.0;
        const double c = gf * m.area[f] / d;
        v[m.diag_slot[o]] += c;
        v[m.diag_slot[nb]] += c;
        v[m.slot_on[f]] += -c;
        v[m.slot_no[f]] += -c;
        diag[o] += c;
        diag[nb] += c;
    }
}

__global__ void k_conv_int(kcfd_dmesh_t m, int f0, int f1, const double* __restrict__ mf, double* __restrict__ v,
                           double* __restrict__ diag) {
    for (int f = f0 + blockIdx.x * blockDim.x + threadIdx.x; f < f1; f += gridDim.x * blockDim.x) {
        const int o = m.owner[f], nb = m.neigh[f];
        const double F = mf[f];
        v[m.diag_slot[o]] += fmax(F, 0.0);
        v[m.slot_on[f]] += fmin(F, 0.0);
        v[m.diag_slot[nb]] += fmax(-F, 0.0);
        v[m.slot_no[f]] += fmin(-F, 0.0);
        diag[o] += fmax(F, 0.0);
        diag[nb] += fmax(-F, 0.0);
    }
}

__global__ void k_conv_bnd(kcfd_dmesh_t m, int f0, int f1, const double* __restrict__ mf, double* __restrict__ v,
                           double* __restrict__ diag) {
    for (int f = f0 + blockIdx.x * blockDim.x + threadIdx.x; f < f1; f += gridDim.x * blockDim.x) {
        const double F = mf[f];
        if (F >= 0) {
            const int o = m.owner[f];
            v[m.diag_slot[o]] += F;
            diag[o] += F;
        }
    }
}

// bt: 0 zero_gradient, 1 dirichlet, 2 neumann (per boundary face); bv: phi_b; bg:
// neumann gradient value.
__global__ void k_bc(kcfd_dmesh_t m, int f0, int f1, const int8_t* __restrict__ bt, const double* __restrict__ bv,
                     const double* __restrict__ bg, const double* __restrict__ gamma, const double* __restrict__ mf,
                     double* __restrict__ v, double* __restrict__ diag, double* __restrict__ rhs) {
    for (int f = f0 + blockIdx.x * blockDim.x + threadIdx.x; f < f1; f += gridDim.x * blockDim.x) {
        const double d = m.dlen[f];
        if (d < 1e-30) continue;
        const int o = m.owner[f], bi = f - m.n_internal;
        const int t = bt[bi];
        if (t == 1) {
            const double phib = bv[bi];
            const double c = gamma[o] * m.area[f] / d;
            v[m.diag_slot[o]] += c;
            diag[o] += c;
            double add = c * phib;
            const double F = mf[f];
            if (F < 0) add = add + (-F) * phib;
            rhs[o] += add;
        } else if (t == 2) {
            rhs[o] += bg[bi] * m.area[f];
        } else if (t == 0) {
            const double F = mf[f];
            if (F < 0) {
                v[m.diag_slot[o]] += -F;
                diag[o] += -F;
            }
        }
    }
}

__global__ void k_cells(int n, const int* __restrict__ diag_slot, const double* __restrict__ vol, int kind, double a0,
                        double a1, const double* __restrict__ p0, const double* __restrict__ p1,
                        double* __restrict__ v, double* __restrict__ diag, double* __restrict__ rhs) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double V = vol[i];
        if (kind == 0) {  // temporal: rho V / dt on the diagonal, coeff * phi_old on the rhs
            const double c = a0 * V / a1;
            v[diag_slot[i]] += c;
            diag[i] += c;
            rhs[i] += c * p0[i];
        } else if (kind == 1) {  // source: S V
            rhs[i] += p0[i] * V;
        } else if (kind == 2) {  // linearised source: -Sp V diagonal, Su V rhs
            const double c = -p0[i] * V;
            v[diag_slot[i]] += c;
            diag[i] += c;
            rhs[i] += p1[i] * V;
        } else {  // under-relaxation (alpha = a0) with the tracked diagonal
            const double ap = diag[i];
            const double add = ap * (1.0 - a0) / a0;
            v[diag_slot[i]] += add;
            diag[i] += add;
            rhs[i] += add * p0[i];
        }
    }
}

__global__ void k_muscl(kcfd_dmesh_t m, int f0, int f1, int lim, const double* __restrict__ phi,
                        const double* __restrict__ mf, const double* __restrict__ grad, double* __restrict__ corr) {
    const int D = m.ndim;
    for (int f = f0 + blockIdx.x * blockDim.x + threadIdx.x; f < f1; f += gridDim.x * blockDim.x) {
        const int o = m.owner[f], nb = m.neigh[f];
        const double F = mf[f];
        const bool pos = F >= 0;
        const int up = pos ? o : nb, dn = pos ? nb : o;
        const double phiU = phi[up], phiD = phi[dn];
        double dot = 0.0;
        for (int k = 0; k < D; ++k) dot = dot + grad[up * D + k] * (m.fcenter[f * D + k] - m.ccenter[up * D + k]);
        const double lin = phiU + dot;
        const double dcd = phiD - phiU;
        if (fabs(dcd) < 1e-15) continue;
        const double r = 2.0 * (lin - phiU) / dcd - 1.0;
        const double psi = lim_psi(lim, r);
        const double fc = fabs(F) * ((phiU + 0.5 * psi * dcd) - phiU);
        corr[up] -= fc;
        corr[dn] += fc;
    }
}

template <class Fn>
void colours(const kcfd_dmesh_t* m, bool internal, Fn fn) {
    const int c0 = internal ? 0 : m->n_colors_int;
    const int c1 = internal ? m->n_colors_int : m->n_colors_int + m->n_colors_bnd;
    for (int c = c0; c < c1; ++c) {
        const int f0 = m->color_ptr[c], f1 = m->color_ptr[c + 1];
        if (f1 > f0) fn(f0, f1, nblk(f1 - f0));
    }
}

int check(const kcfd_dmesh_t* m) {
    KCFD_REQUIRE(m && m->owner && m->color_ptr && m->diag_slot, "kcfd_op: NULL mesh descriptor");
    return KCFD_OK;
}

}  // namespace
}  // namespace kcfd

using namespace kcfd;

extern "C" {

int kcfd_op_diffusion(const kcfd_dmesh_t* m, const double* gamma, double* vals, double* diag, void* stream) {
    if (int e = check(m)) return e;
    KCFD_REQUIRE(gamma && vals && diag, "kcfd_op_diffusion: NULL argument");
    cudaStream_t st = (cudaStream_t)stream;
    colours(m, true, [&](int f0, int f1, int nb) { k_diff<<<nb, kT, 0, st>>>(*m, f0, f1, gamma, vals, diag); });
    KCFD_CUDA(cudaGetLastError());
    return KCFD_OK;
}

int kcfd_op_convection_upwind(const kcfd_dmesh_t* m, const double* mf, double* vals, double* diag, void* stream) {
    if (int e = check(m)) return e;
    KCFD_REQUIRE(mf && vals && diag, "kcfd_op_convection_upwind: NULL argument");
    cudaStream_t st = (cudaStream_t)stream;
    colours(m, true, [&](int f0, int f1, int nb) { k_conv_int<<<nb, kT, 0, st>>>(*m, f0, f1, mf, vals, diag); });
    colours(m, false, [&](int f0, int f1, int nb) { k_conv_bnd<<<nb, kT, 0, st>>>(*m, f0, f1, mf, vals, diag); });
    KCFD_CUDA(cudaGetLastError());
    return KCFD_OK;
}

int kcfd_op_boundary(const kcfd_dmesh_t* m, const int8_t* btype, const double* bval, const double* bgrad,
                     const double* gamma, const double* mf, double* vals, double* diag, double* rhs, void* stream) {
    if (int e = check(m)) return e;
    KCFD_REQUIRE(btype && bval && bgrad && gamma && mf && vals && diag && rhs, "kcfd_op_boundary: NULL argument");
    cudaStream_t st = (cudaStream_t)stream;
    colours(m, false, [&](int f0, int f1, int nb) {
        k_bc<<<nb, kT, 0, st>>>(*m, f0, f1, btype, bval, bgrad, gamma, mf, vals, diag, rhs);
    });
    KCFD_CUDA(cudaGetLastError());
    return KCFD_OK;
}

int kcfd_op_cells(const kcfd_dmesh_t* m, int32_t kind, double a0, double a1, const double* p0, const double* p1,
                  double* vals, double* diag, double* rhs, void* stream) {
    if (int e = check(m)) return e;
    KCFD_REQUIRE(kind >= 0 && kind <= 3, "kcfd_op_cells: kind must be 0..3");
    KCFD_REQUIRE(vals && diag && rhs && (kind == 3 || p0) && (kind != 2 || p1), "kcfd_op_cells: NULL argument");
    KCFD_REQUIRE(kind != 3 || a0 > 0, "kcfd_op_cells: under-relaxation needs alpha > 0");
    k_cells<<<nblk(m->n_cells), kT, 0, (cudaStream_t)stream>>>(m->n_cells, m->diag_slot, m->volume, kind, a0, a1, p0,
                                                               p1, vals, diag, rhs);
    KCFD_CUDA(cudaGetLastError());
    return KCFD_OK;
}

int kcfd_muscl_correction(const kcfd_dmesh_t* m, int32_t limiter, const double* phi, const double* mf,
                          const double* grad, double* corr, void* stream) {
    if (int e = check(m)) return e;
    KCFD_REQUIRE(limiter >= 0 && limiter <= 3, "kcfd_muscl_correction: unknown limiter %d", limiter);
    KCFD_REQUIRE(phi && mf && grad && corr, "kcfd_muscl_correction: NULL argument");
    cudaStream_t st = (cudaStream_t)stream;
    KCFD_CUDA(cudaMemsetAsync(corr, 0, sizeof(double) * m->n_cells, st));
    colours(m, true, [&](int f0, int f1, int nb) { k_muscl<<<nb, kT, 0, st>>>(*m, f0, f1, limiter, phi, mf, grad, corr); });
    KCFD_CUDA(cudaGetLastError());
    return KCFD_OK;
}

}  // extern "C"
