// FVM assembly of the SIMPLE inner loop on sm_100a.
//
// Replaces the Python face loops of the K-CFD reference:
//   models/single_phase.py:124-144  _face_mass_flux        -> kcfd_mass_flux
//   models/single_phase.py:147-258  _momentum_eq (assembly) -> kcfd_momentum_assemble
//   models/single_phase.py:274-348  _pressure_correction    -> kcfd_pressure_assemble
//   core/gradient.py:12-48          green_gauss_gradient    -> kcfd_gg_gradient
//   core/interpolation.py:227-303   muscl_deferred_correction (fused into momentum)
//   models/single_phase.py:355-377  velocity / pressure correction -> kcfd_simple_correct
//
// Layout and scatter: faces live on the device colour by colour (no two faces of a
// colour share a cell). One launch per colour processes its faces with one thread
// each: off-diagonal coefficients go straight into their CSR slots (face -> slot
// map, each slot written by exactly one face), and the owner/neighbour sums (aP,
// rhs, gradients) are plain read-modify-writes that cannot collide inside a colour
// -- no atomics, and a fixed colour order makes the sums deterministic. A final cell
// kernel applies the cell terms (time, relaxation, diagonal, pin).
#include <cuda_runtime.h>

#include <algorithm>

#include "kcfd_common.h"
#include "team.cuh"

namespace kcfd {

constexpr int kThreads = 256;

inline int blocks_for(int64_t n) { return (int)std::max<int64_t>(1, std::min<int64_t>((n + kThreads - 1) / kThreads, 1 << 20)); }

struct DM {
    int D, n, F, Fi;
    const int* __restrict__ owner;
    const int* __restrict__ neigh;
    const double* __restrict__ area;
    const double* __restrict__ normal;
    const double* __restrict__ fcenter;
    const double* __restrict__ cc;
    const double* __restrict__ vol;
    const double* __restrict__ gc;
    const double* __restrict__ dlen;
    const double* __restrict__ dorth;
    const int* __restrict__ slot_on;
    const int* __restrict__ slot_no;
    const int* __restrict__ diag_slot;
    const int* __restrict__ indptr;
    const int* __restrict__ cf_ptr;
    const int* __restrict__ cf_face;
};

static DM to_dm(const kcfd_dmesh_t* m) {
    DM d;
    d.D = m->ndim; d.n = m->n_cells; d.F = m->n_faces; d.Fi = m->n_internal;
    d.owner = m->owner; d.neigh = m->neigh; d.area = m->area; d.normal = m->normal; d.fcenter = m->fcenter;
    d.cc = m->ccenter; d.vol = m->volume; d.gc = m->gc; d.dlen = m->dlen; d.dorth = m->dorth;
    d.slot_on = m->slot_on; d.slot_no = m->slot_no; d.diag_slot = m->diag_slot; d.indptr = m->indptr;
    d.cf_ptr = m->cf_ptr; d.cf_face = m->cf_face;
    return d;
}

__device__ __forceinline__ double limiter_psi(int lim, double r) {
    switch (lim) {
        case 0: return fmax(0.0, fmin(1.0, r));                                // minmod
        case 1: return fmax(0.0, fmax(fmin(2.0 * r, 1.0), fmin(r, 2.0)));     // superbee
        case 2: return r > 0 ? (r * r + r) / (r * r + 1.0) : 0.0;             // van Albada
        default: return r > 0 ? 2.0 * r / (1.0 + r) : 0.0;                    // van Leer
    }
}

// ------------------------------------------------------------------ mass flux --
template <int D>
__global__ void k_mass_flux(DM m, const int8_t* __restrict__ ut, const double* __restrict__ ub,
                            const double* __restrict__ U, double rho, double* __restrict__ mf) {
    for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < m.F; f += gridDim.x * blockDim.x) {
        const int o = m.owner[f];
        double uf[D];
        if (f < m.Fi) {
            const int nb = m.neigh[f];
            const double g = m.gc[f];
#pragma unroll
            for (int k = 0; k < D; ++k) uf[k] = g * U[o * D + k] + (1.0 - g) * U[nb * D + k];
        } else {
            const int bi = f - m.Fi;
            const bool dir = ut[bi] == 1;
#pragma unroll
            for (int k = 0; k < D; ++k) uf[k] = dir ? ub[bi * D + k] : U[o * D + k];
        }
        double dot = 0.0;
#pragma unroll
        for (int k = 0; k < D; ++k) dot = dot + uf[k] * m.normal[f * D + k];
        mf[f] = rho * dot * m.area[f];
    }
}

// ------------------------------------------------------------------ momentum ----
// Internal faces of one colour. MUSCL and non-orthogonal corrections read the
// Green-Gauss gradients gU [n][D][D] (component-major).
template <int D, bool MUSCL, bool NONORTH>
__global__ void k_mom_int(DM m, int f0, int f1, double mu_f, int lim, const double* __restrict__ U,
                          const double* __restrict__ p, const double* __restrict__ mf, const double* __restrict__ gU,
                          double* __restrict__ aP, double* __restrict__ b, double* __restrict__ v64,
                          float* __restrict__ v32) {
    for (int f = f0 + blockIdx.x * blockDim.x + threadIdx.x; f < f1; f += gridDim.x * blockDim.x) {
        const int o = m.owner[f], nb = m.neigh[f];
        const double F = mf[f], A = m.area[f];
        double co = 0.0, cn = 0.0;  // off-diagonal values (o,nb) and (nb,o)
        if (!(m.dlen[f] < 1e-30)) {
            const double Df = mu_f * A / m.dorth[f];
            aP[o] += Df + fmax(F, 0.0);
            aP[nb] += Df + fmax(-F, 0.0);
            co = -(Df + fmax(-F, 0.0));
            cn = -(Df + fmax(F, 0.0));
        }
        v64[m.slot_on[f]] = co;
        v64[m.slot_no[f]] = cn;
        if (v32) {
            v32[m.slot_on[f]] = (float)co;
            v32[m.slot_no[f]] = (float)cn;
        }
        const double pf = 0.5 * (p[o] + p[nb]);
        double add_o[D], add_n[D];
#pragma unroll
        for (int c = 0; c < D; ++c) {
            const double src = pf * m.normal[f * D + c] * A;
            add_o[c] = -src;
            add_n[c] = src;
        }
        if (MUSCL) {
            const bool pos = F >= 0;
            const int up = pos ? o : nb, dn = pos ? nb : o;
            double dx[D];
#pragma unroll
            for (int k = 0; k < D; ++k) dx[k] = m.fcenter[f * D + k] - m.cc[up * D + k];
#pragma unroll
            for (int c = 0; c < D; ++c) {
                const double phiU = U[up * D + c], phiD = U[dn * D + c];
                double dot = 0.0;
#pragma unroll
                for (int k = 0; k < D; ++k) dot = dot + gU[(up * D + c) * D + k] * dx[k];
                const double lin = phiU + dot;
                const double dcd = phiD - phiU;
                if (fabs(dcd) < 1e-15) continue;
                const double r = 2.0 * (lin - phiU) / dcd - 1.0;
                const double psi = limiter_psi(lim, r);
                const double fc = fabs(F) * ((phiU + 0.5 * psi * dcd) - phiU);
                // upwind cell loses, downwind cell gains
                if (pos) { add_o[c] -= fc; add_n[c] += fc; }
                else { add_n[c] -= fc; add_o[c] += fc; }
            }
        }
        if (NONORTH) {
            const double g = m.gc[f];
            const double s = A / m.dorth[f];
            double kv[D];
#pragma unroll
            for (int k = 0; k < D; ++k) kv[k] = m.normal[f * D + k] * A - s * (m.cc[nb * D + k] - m.cc[o * D + k]);
#pragma unroll
            for (int c = 0; c < D; ++c) {
                double kd = 0.0;
#pragma unroll
                for (int k = 0; k < D; ++k) {
                    const double gf = g * gU[(o * D + c) * D + k] + (1.0 - g) * gU[(nb * D + c) * D + k];
                    kd = kd + kv[k] * gf;
                }
                const double flux = mu_f * kd;
                add_o[c] += flux;
                add_n[c] -= flux;
            }
        }
#pragma unroll
        for (int c = 0; c < D; ++c) {
            b[o * D + c] += add_o[c];
            b[nb * D + c] += add_n[c];
        }
    }
}

// Boundary faces of one colour (each touches only its owner).
template <int D>
__global__ void k_mom_bnd(DM m, int f0, int f1, double mu, const int8_t* __restrict__ ut, const double* __restrict__ ub,
                          const int8_t* __restrict__ pt, const double* __restrict__ pv, const double* __restrict__ p,
                          const double* __restrict__ mf, double* __restrict__ aP, double* __restrict__ b) {
    for (int f = f0 + blockIdx.x * blockDim.x + threadIdx.x; f < f1; f += gridDim.x * blockDim.x) {
        const int o = m.owner[f];
        const int bi = f - m.Fi;
        const double F = mf[f], A = m.area[f], d = m.dlen[f];
        double add[D];
#pragma unroll
        for (int c = 0; c < D; ++c) add[c] = 0.0;
        double ap = 0.0;
        if (!(d < 1e-30)) {
            const double Df = mu * A / d;
            if (ut[bi] == 1) {
                ap += Df;
#pragma unroll
                for (int c = 0; c < D; ++c) add[c] += Df * ub[bi * D + c];
                if (F >= 0) ap += F;
                else {
#pragma unroll
                    for (int c = 0; c < D; ++c) add[c] += (-F) * ub[bi * D + c];
                }
            } else {
                ap += (F >= 0) ? F : -F;
            }
        }
        const double pf = (pt[bi] == 1) ? pv[bi] : p[o];
#pragma unroll
        for (int c = 0; c < D; ++c) add[c] -= pf * m.normal[f * D + c] * A;
        aP[o] += ap;
#pragma unroll
        for (int c = 0; c < D; ++c) b[o * D + c] += add[c];
    }
}

template <int D>
__global__ void k_mom_cells(DM m, double alpha, double rho, double dt, const double* __restrict__ U,
                            const double* __restrict__ Uold, double* __restrict__ aP, double* __restrict__ b,
                            double* __restrict__ v64, float* __restrict__ v32, double* __restrict__ dP) {
    const double relax = (1.0 - alpha) / alpha;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m.n; i += gridDim.x * blockDim.x) {
        double a = aP[i];
        if (dt > 0) {
            const double ct = rho * m.vol[i] / dt;
            a += ct;
#pragma unroll
            for (int c = 0; c < D; ++c) b[i * D + c] += ct * Uold[i * D + c];
        }
#pragma unroll
        for (int c = 0; c < D; ++c) b[i * D + c] += relax * a * U[i * D + c];
        const double ar = a / alpha;
        v64[m.diag_slot[i]] = ar;
        if (v32) v32[m.diag_slot[i]] = (float)ar;
        const double phys = ar * alpha;
        aP[i] = phys;
        double sum = phys;
#pragma unroll
        for (int c = 1; c < D; ++c) sum = sum + phys;
        dP[i] = m.vol[i] / fmax(sum / D, 1e-30);
    }
}

// -------------------------------------------------------- pressure correction ---
__global__ void k_pp_int(DM m, int f0, int f1, double rho, const double* __restrict__ dP, const double* __restrict__ mf,
                         double* __restrict__ aP, double* __restrict__ b, double* __restrict__ v64,
                         float* __restrict__ v32) {
    for (int f = f0 + blockIdx.x * blockDim.x + threadIdx.x; f < f1; f += gridDim.x * blockDim.x) {
        const int o = m.owner[f], nb = m.neigh[f];
        double val = 0.0;
        if (!(m.dlen[f] < 1e-30)) {
            const double df = rho * 0.5 * (dP[o] + dP[nb]) * m.area[f] / m.dorth[f];
            aP[o] += df;
            aP[nb] += df;
            val = -df;
            b[o] -= mf[f];
            b[nb] += mf[f];
        }
        v64[m.slot_on[f]] = val;
        v64[m.slot_no[f]] = val;
        if (v32) {
            v32[m.slot_on[f]] = (float)val;
            v32[m.slot_no[f]] = (float)val;
        }
    }
}

__global__ void k_pp_bnd(DM m, int f0, int f1, double rho, const int8_t* __restrict__ pt, const double* __restrict__ dP,
                         const double* __restrict__ mf, double* __restrict__ aP, double* __restrict__ b) {
    for (int f = f0 + blockIdx.x * blockDim.x + threadIdx.x; f < f1; f += gridDim.x * blockDim.x) {
        const int o = m.owner[f];
        b[o] -= mf[f];
        if (pt[f - m.Fi] == 1) {
            const double d = m.dlen[f];
            if (d > 1e-30) aP[o] += rho * dP[o] * m.area[f] / d;
        }
    }
}

__global__ void k_pp_cells(DM m, int pin, const double* __restrict__ aP, double* __restrict__ b,
                           double* __restrict__ v64, float* __restrict__ v32) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m.n; i += gridDim.x * blockDim.x) {
        if (pin && i == 0) {
            for (int k = m.indptr[0]; k < m.indptr[1]; ++k) {
                v64[k] = 0.0;
                if (v32) v32[k] = 0.0f;
            }
            v64[m.diag_slot[0]] = 0.0 + 1.0;
            if (v32) v32[m.diag_slot[0]] = 1.0f;
            b[0] = 0.0;
        } else {
            v64[m.diag_slot[i]] = aP[i];
            if (v32) v32[m.diag_slot[i]] = (float)aP[i];
        }
    }
}

// ------------------------------------------------------------- Green-Gauss ------
template <int D, int K>
__global__ void k_gg_int(DM m, int f0, int f1, const double* __restrict__ phi, double* __restrict__ g) {
    for (int f = f0 + blockIdx.x * blockDim.x + threadIdx.x; f < f1; f += gridDim.x * blockDim.x) {
        const int o = m.owner[f], nb = m.neigh[f];
        const double w = m.gc[f], A = m.area[f];
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const double pf = w * phi[o * K + k] + (1.0 - w) * phi[nb * K + k];
#pragma unroll
            for (int d = 0; d < D; ++d) {
                const double fl = pf * m.normal[f * D + d] * A;
                g[(o * K + k) * D + d] += fl;
                g[(nb * K + k) * D + d] -= fl;
            }
        }
    }
}

template <int D, int K>
__global__ void k_gg_bnd(DM m, int f0, int f1, const double* __restrict__ phi, const int8_t* __restrict__ bt,
                         const double* __restrict__ bv, double* __restrict__ g) {
    for (int f = f0 + blockIdx.x * blockDim.x + threadIdx.x; f < f1; f += gridDim.x * blockDim.x) {
        const int o = m.owner[f], bi = f - m.Fi;
        const double A = m.area[f];
        const bool use = bt[bi] == 1;
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const double pf = use ? bv[bi * K + k] : phi[o * K + k];
#pragma unroll
            for (int d = 0; d < D; ++d) g[(o * K + k) * D + d] += pf * m.normal[f * D + d] * A;
        }
    }
}

// 1/V per gradient entry, flat over [n][KD] so that loads and stores coalesce.
__global__ void k_gg_cells(int n, int KD, const double* __restrict__ vol, double* __restrict__ g) {
    const int64_t m = (int64_t)n * KD;
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < m; j += (int64_t)gridDim.x * blockDim.x) {
        const double v = vol[j / KD];
        if (v > 1e-30) g[j] = g[j] / v;
    }
}

// Green-Gauss per cell: the cell sums the fluxes of its own faces in ascending
// reference face id (the order in which core/gradient.py:12-48 accumulates them),
// adding on the owner side and subtracting on the neighbour side, and writes its
// gradient once, divided by the volume. No face colours, no read-modify-write.
template <int D, int K>
__global__ void k_gg_cell(DM m, const double* __restrict__ phi, const int8_t* __restrict__ bt,
                          const double* __restrict__ bv, double* __restrict__ g) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m.n; i += gridDim.x * blockDim.x) {
        double acc[K][D];
#pragma unroll
        for (int k = 0; k < K; ++k)
#pragma unroll
            for (int d = 0; d < D; ++d) acc[k][d] = 0.0;
        const int e1 = m.cf_ptr[i + 1];
        for (int e = m.cf_ptr[i]; e < e1; ++e) {
            const int f = m.cf_face[e];
            const int o = m.owner[f];
            const double A = m.area[f];
            double pf[K];
            bool own = true;
            if (f < m.Fi) {
                const int nb = m.neigh[f];
                own = (o == i);
                const double w = m.gc[f];
#pragma unroll
                for (int k = 0; k < K; ++k) pf[k] = w * phi[o * K + k] + (1.0 - w) * phi[nb * K + k];
            } else {
                const int bi = f - m.Fi;
                const bool use = bt[bi] == 1;
#pragma unroll
                for (int k = 0; k < K; ++k) pf[k] = use ? bv[bi * K + k] : phi[o * K + k];
            }
#pragma unroll
            for (int k = 0; k < K; ++k)
#pragma unroll
                for (int d = 0; d < D; ++d) {
                    const double fl = pf[k] * m.normal[f * D + d] * A;
                    if (own) acc[k][d] += fl;
                    else acc[k][d] -= fl;
                }
        }
        const double v = m.vol[i];
#pragma unroll
        for (int k = 0; k < K; ++k)
#pragma unroll
            for (int d = 0; d < D; ++d) g[(i * K + k) * D + d] = (v > 1e-30) ? acc[k][d] / v : acc[k][d];
    }
}

// Least-squares gradient per cell (core/gradient.py:51-99): over the cell's faces,
// dx = x_N - x_P (internal, N the other cell) or x_f - x_P (boundary, with the face's
// boundary value), dphi likewise; grad solves (A^T A) g = A^T dphi by Gaussian
// elimination with partial pivoting (as LAPACK's gesv), zero for cells with fewer
// than D faces or an exactly singular A^T A.
template <int D>
__global__ void k_lsq(DM m, const double* __restrict__ phi, const double* __restrict__ pb, double* __restrict__ g) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m.n; i += gridDim.x * blockDim.x) {
        double M[D][D + 1];
#pragma unroll
        for (int p = 0; p < D; ++p)
#pragma unroll
            for (int q = 0; q <= D; ++q) M[p][q] = 0.0;
        double xp[D];
#pragma unroll
        for (int d = 0; d < D; ++d) xp[d] = m.cc[i * D + d];
        const double pi = phi[i];
        const int e0 = m.cf_ptr[i], e1 = m.cf_ptr[i + 1];
        for (int e = e0; e < e1; ++e) {
            const int f = m.cf_face[e];
            double dx[D], dp;
            if (f < m.Fi) {
                const int o = m.owner[f];
                const int nb = (o == i) ? m.neigh[f] : o;
#pragma unroll
                for (int d = 0; d < D; ++d) dx[d] = m.cc[nb * D + d] - xp[d];
                dp = phi[nb] - pi;
            } else {
#pragma unroll
                for (int d = 0; d < D; ++d) dx[d] = m.fcenter[f * D + d] - xp[d];
                dp = pb[f - m.Fi] - pi;
            }
#pragma unroll
            for (int p = 0; p < D; ++p) {
#pragma unroll
                for (int q = 0; q < D; ++q) M[p][q] += dx[p] * dx[q];
                M[p][D] += dx[p] * dp;
            }
        }
        double out[D];
#pragma unroll
        for (int d = 0; d < D; ++d) out[d] = 0.0;
        bool ok = (e1 - e0) >= D;
        if (ok) {
#pragma unroll
            for (int c = 0; c < D; ++c) {
                int piv = c;
                double best = fabs(M[c][c]);
#pragma unroll
                for (int r = c + 1; r < D; ++r)
                    if (fabs(M[r][c]) > best) {
                        best = fabs(M[r][c]);
                        piv = r;
                    }
                if (best == 0.0) ok = false;
                if (piv != c) {
#pragma unroll
                    for (int q = 0; q <= D; ++q) {
                        const double t = M[c][q];
                        M[c][q] = M[piv][q];
                        M[piv][q] = t;
                    }
                }
                if (ok) {
#pragma unroll
                    for (int r = c + 1; r < D; ++r) {
                        const double l = M[r][c] / M[c][c];
#pragma unroll
                        for (int q = c; q <= D; ++q) M[r][q] -= l * M[c][q];
                    }
                }
            }
            if (ok) {
#pragma unroll
                for (int r = D - 1; r >= 0; --r) {
                    double v = M[r][D];
#pragma unroll
                    for (int q = r + 1; q < D; ++q) v -= M[r][q] * out[q];
                    out[r] = v / M[r][r];
                }
            }
        }
#pragma unroll
        for (int d = 0; d < D; ++d) g[i * D + d] = ok ? out[d] : 0.0;
    }
}

// ------------------------------------------------------------- reductions --------
constexpr int kRedBlocks = 1024;

template <int K>
__device__ __forceinline__ void store_partials(double (&v)[K], double* scratch) {
    __shared__ double smem[32 * kMaxK];
    block_sum<K>(v, smem);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < K; ++k) scratch[k * kRedBlocks + blockIdx.x] = v[k];
    }
}

__global__ void k_finalize(int K, int nblocks, const double* __restrict__ scratch, double* __restrict__ out) {
    // one warp per value: fixed strided order, fixed xor tree
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (w < K) {
        double t = 0.0;
        for (int j = lane; j < nblocks; j += 32) t += scratch[w * kRedBlocks + j];
        t = warp_sum(t);
        if (lane == 0) out[w] = t;
    }
}

template <int D>
__global__ void k_correct(DM m, double alpha_p, const double* __restrict__ pp, const double* __restrict__ gpp,
                          const double* __restrict__ dP, double* __restrict__ U, double* __restrict__ p,
                          double* __restrict__ scratch) {
    double v[2] = {0.0, 0.0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m.n; i += gridDim.x * blockDim.x) {
        const double d = dP[i];
#pragma unroll
        for (int c = 0; c < D; ++c) U[i * D + c] -= d * gpp[i * D + c];
        const double q = pp[i];
        const double pn = p[i] + alpha_p * q;
        p[i] = pn;
        v[0] += q * q;
        v[1] += pn * pn;
    }
    store_partials<2>(v, scratch);
}

template <int NRHS>
__global__ void k_resid(int n, const int* __restrict__ ip, const int* __restrict__ ix, const double* __restrict__ val,
                        const double* __restrict__ x, const double* __restrict__ b, double* __restrict__ scratch) {
    double v[2 * NRHS];
#pragma unroll
    for (int k = 0; k < 2 * NRHS; ++k) v[k] = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double acc[NRHS];
#pragma unroll
        for (int c = 0; c < NRHS; ++c) acc[c] = 0.0;
        for (int k = ip[i]; k < ip[i + 1]; ++k) {
            const double a = val[k];
            const int j = ix[k];
#pragma unroll
            for (int c = 0; c < NRHS; ++c) acc[c] += a * x[(size_t)j * NRHS + c];
        }
#pragma unroll
        for (int c = 0; c < NRHS; ++c) {
            const double bb = b[(size_t)i * NRHS + c];
            const double r = acc[c] - bb;
            v[2 * c] += r * r;
            v[2 * c + 1] += bb * bb;
        }
    }
    store_partials<2 * NRHS>(v, scratch);
}

__global__ void k_simple_residual(int ndim, const double* __restrict__ mom, const double* __restrict__ pn,
                                  double* __restrict__ state, double* __restrict__ hist, int* __restrict__ itp,
                                  int max_hist) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const int it = *itp;
    double res = 0.0;
    for (int c = 0; c < ndim; ++c) {
        const double r = sqrt(mom[2 * c]) / fmax(sqrt(mom[2 * c + 1]), 1e-15);
        res = (c == 0) ? r : fmax(res, r);
    }
    const double rp = sqrt(pn[0]) / fmax(sqrt(pn[1]) + 1e-10, 1e-10);
    res = fmax(res, rp);
    if (state[0] <= 0.0 && res > 1e-30) state[0] = res;
    const double r0 = state[0];
    if (it >= 0 && it < max_hist) hist[it] = (r0 > 1e-30) ? res / r0 : res;
    state[1] = res;
    *itp = it + 1;
}

template <int K>
__global__ void k_norms2(int n, const double* __restrict__ x, double* __restrict__ scratch) {
    double v[K];
#pragma unroll
    for (int c = 0; c < K; ++c) v[c] = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
#pragma unroll
        for (int c = 0; c < K; ++c) {
            const double t = x[(size_t)i * K + c];
            v[c] += t * t;
        }
    }
    store_partials<K>(v, scratch);
}

__global__ void k_record_norm(const double* __restrict__ n2, double* __restrict__ h, const int* __restrict__ it,
                              int max_hist) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        const int i = *it;
        if (i >= 0 && i < max_hist) h[i] = sqrt(n2[0]);
    }
}

}  // namespace kcfd

using namespace kcfd;

namespace {
template <typename Fn>
int for_colors(const kcfd_dmesh_t* m, bool internal, Fn fn) {
    const int c0 = internal ? 0 : m->n_colors_int;
    const int c1 = internal ? m->n_colors_int : m->n_colors_int + m->n_colors_bnd;
    for (int c = c0; c < c1; ++c) {
        const int f0 = m->color_ptr[c], f1 = m->color_ptr[c + 1];
        if (f1 > f0) fn(f0, f1, blocks_for(f1 - f0));
    }
    return KCFD_OK;
}

int check_mesh(const kcfd_dmesh_t* m) {
    KCFD_REQUIRE(m && m->owner && m->area && m->normal && m->color_ptr, "kcfd: NULL mesh descriptor");
    KCFD_REQUIRE(m->ndim == 2 || m->ndim == 3, "kcfd: mesh ndim must be 2 or 3");
    KCFD_REQUIRE(m->n_internal >= 0 && m->n_internal <= m->n_faces, "kcfd: bad face counts");
    KCFD_REQUIRE(m->color_ptr[0] == 0 && m->color_ptr[m->n_colors_int] == m->n_internal &&
                     m->color_ptr[m->n_colors_int + m->n_colors_bnd] == m->n_faces,
                 "kcfd: colour ranges do not cover the faces");
    return KCFD_OK;
}
}  // namespace

extern "C" {

int kcfd_mass_flux(const kcfd_dmesh_t* m, const kcfd_bc_t* bc, const double* U, double rho, double* mf, void* stream) {
    if (int e = check_mesh(m)) return e;
    KCFD_REQUIRE(bc && U && mf, "kcfd_mass_flux: NULL argument");
    cudaStream_t st = (cudaStream_t)stream;
    DM d = to_dm(m);
    if (d.D == 2) k_mass_flux<2><<<blocks_for(d.F), kThreads, 0, st>>>(d, bc->u_type, bc->u_val, U, rho, mf);
    else k_mass_flux<3><<<blocks_for(d.F), kThreads, 0, st>>>(d, bc->u_type, bc->u_val, U, rho, mf);
    KCFD_CUDA(cudaGetLastError());
    return KCFD_OK;
}

int kcfd_momentum_assemble(const kcfd_dmesh_t* m, const kcfd_bc_t* bc, const kcfd_mom_params_t* prm,
                           const double* U, const double* U_old, const double* p, const double* mf,
                           const double* gradU, double* aP, double* vals64, float* vals32, double* b,
                           double* dP, void* stream) {
    if (int e = check_mesh(m)) return e;
    KCFD_REQUIRE(bc && prm && U && p && mf && aP && vals64 && b && dP, "kcfd_momentum_assemble: NULL argument");
    KCFD_REQUIRE(prm->alpha_u > 0, "kcfd_momentum_assemble: alpha_u must be > 0");
    const bool muscl = prm->limiter >= 0, nonorth = prm->nonorth != 0;
    KCFD_REQUIRE(!(muscl || nonorth) || gradU, "kcfd_momentum_assemble: MUSCL / non-orthogonal need gradU");
    KCFD_REQUIRE(prm->dt <= 0 || U_old, "kcfd_momentum_assemble: transient needs U_old");
    cudaStream_t st = (cudaStream_t)stream;
    DM d = to_dm(m);
    const int D = d.D;
    KCFD_CUDA(cudaMemsetAsync(aP, 0, sizeof(double) * d.n, st));
    KCFD_CUDA(cudaMemsetAsync(b, 0, sizeof(double) * d.n * D, st));
    const double mu = prm->mu;
    const double mu_f = 2 * mu * mu / fmax(mu + mu, 1e-30);
    const int lim = prm->limiter;
    for_colors(m, true, [&](int f0, int f1, int nb) {
#define KC_MOM(DD, MU, NO) k_mom_int<DD, MU, NO><<<nb, kThreads, 0, st>>>(d, f0, f1, mu_f, lim, U, p, mf, gradU, aP, b, vals64, vals32)
        if (D == 2) {
            if (muscl && nonorth) KC_MOM(2, true, true); else if (muscl) KC_MOM(2, true, false);
            else if (nonorth) KC_MOM(2, false, true); else KC_MOM(2, false, false);
        } else {
            if (muscl && nonorth) KC_MOM(3, true, true); else if (muscl) KC_MOM(3, true, false);
            else if (nonorth) KC_MOM(3, false, true); else KC_MOM(3, false, false);
        }
#undef KC_MOM
    });
    for_colors(m, false, [&](int f0, int f1, int nb) {
        if (D == 2) k_mom_bnd<2><<<nb, kThreads, 0, st>>>(d, f0, f1, mu, bc->u_type, bc->u_val, bc->p_type, bc->p_val, p, mf, aP, b);
        else k_mom_bnd<3><<<nb, kThreads, 0, st>>>(d, f0, f1, mu, bc->u_type, bc->u_val, bc->p_type, bc->p_val, p, mf, aP, b);
    });
    if (D == 2) k_mom_cells<2><<<blocks_for(d.n), kThreads, 0, st>>>(d, prm->alpha_u, prm->rho, prm->dt, U, U_old, aP, b, vals64, vals32, dP);
    else k_mom_cells<3><<<blocks_for(d.n), kThreads, 0, st>>>(d, prm->alpha_u, prm->rho, prm->dt, U, U_old, aP, b, vals64, vals32, dP);
    KCFD_CUDA(cudaGetLastError());
    return KCFD_OK;
}

int kcfd_pressure_assemble(const kcfd_dmesh_t* m, const kcfd_bc_t* bc, double rho, const double* dP,
                           const double* mf, double* aP, double* vals64, float* vals32, double* b, void* stream) {
    if (int e = check_mesh(m)) return e;
    KCFD_REQUIRE(bc && dP && mf && aP && vals64 && b, "kcfd_pressure_assemble: NULL argument");
    cudaStream_t st = (cudaStream_t)stream;
    DM d = to_dm(m);
    KCFD_CUDA(cudaMemsetAsync(aP, 0, sizeof(double) * d.n, st));
    KCFD_CUDA(cudaMemsetAsync(b, 0, sizeof(double) * d.n, st));
    for_colors(m, true, [&](int f0, int f1, int nb) {
        k_pp_int<<<nb, kThreads, 0, st>>>(d, f0, f1, rho, dP, mf, aP, b, vals64, vals32);
    });
    for_colors(m, false, [&](int f0, int f1, int nb) {
        k_pp_bnd<<<nb, kThreads, 0, st>>>(d, f0, f1, rho, bc->p_type, dP, mf, aP, b);
    });
    k_pp_cells<<<blocks_for(d.n), kThreads, 0, st>>>(d, bc->has_p_dirichlet ? 0 : 1, aP, b, vals64, vals32);
    KCFD_CUDA(cudaGetLastError());
    return KCFD_OK;
}

int kcfd_gg_gradient(const kcfd_dmesh_t* m, int32_t ncomp, const double* phi, const int8_t* btype, const double* bval,
                     double* grad, void* stream) {
    if (int e = check_mesh(m)) return e;
    KCFD_REQUIRE(phi && btype && grad, "kcfd_gg_gradient: NULL argument");
    KCFD_REQUIRE(ncomp == 1 || ncomp == m->ndim, "kcfd_gg_gradient: ncomp must be 1 or ndim");
    cudaStream_t st = (cudaStream_t)stream;
    DM d = to_dm(m);
    if (d.cf_ptr && d.cf_face) {
        const int nb = blocks_for(d.n);
        if (d.D == 2 && ncomp == 1) k_gg_cell<2, 1><<<nb, kThreads, 0, st>>>(d, phi, btype, bval, grad);
        else if (d.D == 2) k_gg_cell<2, 2><<<nb, kThreads, 0, st>>>(d, phi, btype, bval, grad);
        else if (ncomp == 1) k_gg_cell<3, 1><<<nb, kThreads, 0, st>>>(d, phi, btype, bval, grad);
        else k_gg_cell<3, 3><<<nb, kThreads, 0, st>>>(d, phi, btype, bval, grad);
        KCFD_CUDA(cudaGetLastError());
        return KCFD_OK;
    }
    KCFD_CUDA(cudaMemsetAsync(grad, 0, sizeof(double) * d.n * ncomp * d.D, st));
#define KC_GG(DD, KK)                                                                                   \
    for_colors(m, true, [&](int f0, int f1, int nb) { k_gg_int<DD, KK><<<nb, kThreads, 0, st>>>(d, f0, f1, phi, grad); }); \
    for_colors(m, false, [&](int f0, int f1, int nb) { k_gg_bnd<DD, KK><<<nb, kThreads, 0, st>>>(d, f0, f1, phi, btype, bval, grad); });
    if (d.D == 2 && ncomp == 1) { KC_GG(2, 1) }
    else if (d.D == 2) { KC_GG(2, 2) }
    else if (ncomp == 1) { KC_GG(3, 1) }
    else { KC_GG(3, 3) }
#undef KC_GG
    k_gg_cells<<<blocks_for(d.n), kThreads, 0, st>>>(d.n, ncomp * d.D, d.vol, grad);
    KCFD_CUDA(cudaGetLastError());
    return KCFD_OK;
}

int kcfd_lsq_gradient(const kcfd_dmesh_t* m, const double* phi, const double* phi_b, double* grad, void* stream) {
    if (int e = check_mesh(m)) return e;
    KCFD_REQUIRE(phi && phi_b && grad, "kcfd_lsq_gradient: NULL argument");
    KCFD_REQUIRE(m->cf_ptr && m->cf_face, "kcfd_lsq_gradient: the mesh descriptor has no cell-face list");
    cudaStream_t st = (cudaStream_t)stream;
    DM d = to_dm(m);
    if (d.D == 2) k_lsq<2><<<blocks_for(d.n), kThreads, 0, st>>>(d, phi, phi_b, grad);
    else k_lsq<3><<<blocks_for(d.n), kThreads, 0, st>>>(d, phi, phi_b, grad);
    KCFD_CUDA(cudaGetLastError());
    return KCFD_OK;
}

int kcfd_simple_correct(const kcfd_dmesh_t* m, double alpha_p, const double* pp, const double* grad_pp,
                        const double* dP, double* U, double* p, double* norms2, double* scratch, void* stream) {
    if (int e = check_mesh(m)) return e;
    KCFD_REQUIRE(pp && grad_pp && dP && U && p && norms2 && scratch, "kcfd_simple_correct: NULL argument");
    cudaStream_t st = (cudaStream_t)stream;
    DM d = to_dm(m);
    const int nb = std::min(kRedBlocks, blocks_for(d.n));
    if (d.D == 2) k_correct<2><<<nb, kThreads, 0, st>>>(d, alpha_p, pp, grad_pp, dP, U, p, scratch);
    else k_correct<3><<<nb, kThreads, 0, st>>>(d, alpha_p, pp, grad_pp, dP, U, p, scratch);
    k_finalize<<<1, 32 * 8, 0, st>>>(2, nb, scratch, norms2);
    KCFD_CUDA(cudaGetLastError());
    return KCFD_OK;
}

int kcfd_residual_norms(const kcfd_csr_t* A, const double* x, const double* b, int32_t nrhs, double* norms2,
                        double* scratch, void* stream) {
    KCFD_REQUIRE(A && A->vals64 && x && b && norms2 && scratch, "kcfd_residual_norms: NULL argument");
    KCFD_REQUIRE(nrhs >= 1 && nrhs <= 3, "kcfd_residual_norms: nrhs must be 1..3");
    cudaStream_t st = (cudaStream_t)stream;
    const int nb = std::min(kRedBlocks, blocks_for(A->n));
    if (nrhs == 1) k_resid<1><<<nb, kThreads, 0, st>>>(A->n, A->indptr, A->indices, A->vals64, x, b, scratch);
    else if (nrhs == 2) k_resid<2><<<nb, kThreads, 0, st>>>(A->n, A->indptr, A->indices, A->vals64, x, b, scratch);
    else k_resid<3><<<nb, kThreads, 0, st>>>(A->n, A->indptr, A->indices, A->vals64, x, b, scratch);
    k_finalize<<<1, 32 * 8, 0, st>>>(2 * nrhs, nb, scratch, norms2);
    KCFD_CUDA(cudaGetLastError());
    return KCFD_OK;
}

int kcfd_simple_residual(int32_t ndim, const double* mom_norms2, const double* p_norms2, double* state, double* hist,
                         int32_t* it, int32_t max_hist, void* stream) {
    KCFD_REQUIRE(mom_norms2 && p_norms2 && state && hist && it && max_hist >= 0, "kcfd_simple_residual: bad argument");
    k_simple_residual<<<1, 32, 0, (cudaStream_t)stream>>>(ndim, mom_norms2, p_norms2, state, hist, it, max_hist);
    KCFD_CUDA(cudaGetLastError());
    return KCFD_OK;
}

int kcfd_vec_norms2(int32_t n, int32_t k, const double* x, double* out2, double* scratch, void* stream) {
    KCFD_REQUIRE(n >= 0 && k >= 1 && k <= 6 && x && out2 && scratch, "kcfd_vec_norms2: bad argument");
    cudaStream_t st = (cudaStream_t)stream;
    const int nb = std::min(kRedBlocks, blocks_for(std::max(n, 1)));
    switch (k) {
        case 1: k_norms2<1><<<nb, kThreads, 0, st>>>(n, x, scratch); break;
        case 2: k_norms2<2><<<nb, kThreads, 0, st>>>(n, x, scratch); break;
        case 3: k_norms2<3><<<nb, kThreads, 0, st>>>(n, x, scratch); break;
        case 4: k_norms2<4><<<nb, kThreads, 0, st>>>(n, x, scratch); break;
        case 5: k_norms2<5><<<nb, kThreads, 0, st>>>(n, x, scratch); break;
        default: k_norms2<6><<<nb, kThreads, 0, st>>>(n, x, scratch); break;
    }
    k_finalize<<<1, 32 * 8, 0, st>>>(k, nb, scratch, out2);
    KCFD_CUDA(cudaGetLastError());
    return KCFD_OK;
}

int kcfd_record_norm(const double* norm2, double* chist, const int32_t* it, int32_t max_hist, void* stream) {
    KCFD_REQUIRE(norm2 && chist && it && max_hist >= 0, "kcfd_record_norm: bad argument");
    k_record_norm<<<1, 32, 0, (cudaStream_t)stream>>>(norm2, chist, it, max_hist);
    KCFD_CUDA(cudaGetLastError());
    return KCFD_OK;
}

}  // extern "C"
