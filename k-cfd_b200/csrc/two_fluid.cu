// Two-fluid (Euler-Euler) system set on the device: the per-cell closures, face
// fluxes, source terms, two-phase pressure correction and field updates that
// models/two_fluid.py assembles around the generic FVM operators.
//   closures              models/closure.py:13-34,72-92 (Schiller-Naumann drag),
//                         :95-115 (Ranz-Marshall), :146-164 (Sato viscosity)
//   phase change (Lee)    models/two_fluid.py:334-360
//   interfacial h_i a_i   models/two_fluid.py:395-410
//   phase momentum        models/two_fluid.py:520-639
//   two-phase p'          models/two_fluid.py:641-725
//   volume fraction       models/two_fluid.py:727-783
//   phase energy          models/two_fluid.py:412-518
//   boundary refresh      models/two_fluid.py:224-250; mass flux core/interpolation.py:163-182
// Face kernels run one launch per face colour (no two faces of a colour share a
// cell), so every scatter is free of write conflicts and of atomics; per-element
// arithmetic follows the reference's expression order.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "kcfd_common.h"

namespace kcfd {
namespace {

constexpr int kT = 256;
inline int nblk(int64_t n) { return (int)std::max<int64_t>(1, std::min<int64_t>((n + kT - 1) / kT, 1 << 20)); }

template <class Fn>
void tf_colours(const kcfd_dmesh_t* m, bool internal, Fn fn) {
    const int c0 = internal ? 0 : m->n_colors_int;
    const int c1 = internal ? m->n_colors_int : m->n_colors_int + m->n_colors_bnd;
    for (int c = c0; c < c1; ++c) {
        const int f0 = m->color_ptr[c], f1 = m->color_ptr[c + 1];
        if (f1 > f0) fn(f0, f1, nblk(f1 - f0));
    }
}

__device__ __forceinline__ double rel_speed(const double* Ug, const double* Ul, int i, int nd) {
    double s = 0.0;
    for (int k = 0; k < nd; ++k) {
        const double d = Ug[i * nd + k] - Ul[i * nd + k];
        s = s + d * d;
    }
    return sqrt(s);
}

__global__ void k_drag(int n, int nd, kcfd_tf_params_t P, const double* __restrict__ ag, const double* __restrict__ Ug,
                       const double* __restrict__ Ul, double* __restrict__ K) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double mag = fmax(rel_speed(Ug, Ul, i, nd), 1e-15);
        double re = P.rho_l * mag * P.d_b / P.mu_l;
        re = fmax(re, 1e-10);
        const double cd = re < 1000.0 ? 24.0 / re * (1.0 + 0.15 * pow(re, 0.687)) : 0.44;
        K[i] = 0.75 * cd * ag[i] * P.rho_l * mag / P.d_b;
    }
}

__global__ void k_interfacial(int n, int nd, kcfd_tf_params_t P, const double* __restrict__ ag,
                              const double* __restrict__ Ug, const double* __restrict__ Ul,
                              const double* __restrict__ vol, double* __restrict__ hiaiV) {
    const double pr = P.mu_l * P.cp_l / P.k_l;
    const double pr333 = pow(pr, 0.333);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double mag = fmax(rel_speed(Ug, Ul, i, nd), 1e-15);
        const double re = P.rho_l * mag * P.d_b / P.mu_l;
        const double nu = 2.0 + 0.6 * sqrt(fmax(re, 1e-10)) * pr333;
        const double hi = P.h_i_coeff * nu * P.k_l / P.d_b;
        const double ai = P.a_i_coeff * 6.0 * ag[i] / fmax(P.d_b, 1e-15);
        hiaiV[i] = hi * ai * vol[i];
    }
}

__global__ void k_phase_change(int n, kcfd_tf_params_t P, const double* __restrict__ al, const double* __restrict__ ag,
                               const double* __restrict__ Tl, const double* __restrict__ Tg, double* __restrict__ dm) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double d = 0.0;
        if (Tl[i] > P.T_sat && al[i] > 1e-6) d += P.r_phase_change * al[i] * P.rho_l * (Tl[i] - P.T_sat) / P.T_sat;
        if (Tg[i] < P.T_sat && ag[i] > 1e-6) d -= P.r_phase_change * ag[i] * P.rho_g * (P.T_sat - Tg[i]) / P.T_sat;
        dm[i] = d;
    }
}

// kind 0: alpha * coef; kind 1 (liquid momentum): alpha mu_l + alpha mu_BIT (Sato).
__global__ void k_gamma(int n, int nd, int kind, kcfd_tf_params_t P, const double* __restrict__ alpha, double coef,
                        const double* __restrict__ ag, const double* __restrict__ Ug, const double* __restrict__ Ul,
                        double* __restrict__ gamma) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double g = alpha[i] * coef;
        if (kind == 1) {
            const double mu_bit = 0.6 * P.rho_l * ag[i] * P.d_b * rel_speed(Ug, Ul, i, nd);
            g = g + alpha[i] * mu_bit;
        }
        gamma[i] = g;
    }
}

// kind 0: mf alpha[owner] (momentum); kind 1: mf alpha_upwind cp (energy; owner on
// boundary faces).
__global__ void k_face_flux(kcfd_dmesh_t m, int kind, const double* __restrict__ mf, const double* __restrict__ alpha,
                            double cp, double* __restrict__ out) {
    for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < m.n_faces; f += gridDim.x * blockDim.x) {
        const int o = m.owner[f];
        const double F = mf[f];
        if (kind == 0) {
            out[f] = F * alpha[o];
        } else {
            const double a = (f < m.n_internal && F < 0) ? alpha[m.neigh[f]] : alpha[o];
            out[f] = F * a * cp;
        }
    }
}

__global__ void k_mass_flux_b(kcfd_dmesh_t m, double rho, const double* __restrict__ U, const double* __restrict__ Ub,
                              double* __restrict__ mf) {
    const int nd = m.ndim;
    for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < m.n_faces; f += gridDim.x * blockDim.x) {
        const int o = m.owner[f];
        double dot = 0.0;
        if (f < m.n_internal) {
            const int nb = m.neigh[f];
            const double g = m.gc[f];
            for (int k = 0; k < nd; ++k) dot = dot + (g * U[o * nd + k] + (1.0 - g) * U[nb * nd + k]) * m.normal[f * nd + k];
        } else {
            const int bi = f - m.n_internal;
            for (int k = 0; k < nd; ++k) dot = dot + Ub[bi * nd + k] * m.normal[f * nd + k];
        }
        mf[f] = rho * dot * m.area[f];
    }
}

__global__ void k_zero_grad(kcfd_dmesh_t m, const int8_t* __restrict__ mask, const double* __restrict__ fld, int nc,
                            double* __restrict__ bv) {
    const int fb = m.n_faces - m.n_internal;
    for (int bi = blockIdx.x * blockDim.x + threadIdx.x; bi < fb; bi += gridDim.x * blockDim.x) {
        if (!mask[bi]) continue;
        const int o = m.owner[m.n_internal + bi];
        for (int c = 0; c < nc; ++c) bv[bi * nc + c] = fld[o * nc + c];
    }
}

// Momentum cell terms: temporal (alpha rho V / dt), implicit drag (K V), gravity.
__global__ void k_mom_cells_tf(int n, int nd, int comp0, int nc, kcfd_tf_params_t P, double rho,
                               const int* __restrict__ diag_slot, const double* __restrict__ vol,
                               const double* __restrict__ alpha, const double* __restrict__ K,
                               const double* __restrict__ Uo, const double* __restrict__ old, double* __restrict__ v,
                               double* __restrict__ diag, double* __restrict__ rhs) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double V = vol[i];
        double add = 0.0;
        if (old) {
            const double c = alpha[i] * rho * V / P.dt;
            add += c;
            diag[i] += c;
            for (int c2 = 0; c2 < nc; ++c2) rhs[i * nc + c2] += c * old[i * nd + comp0 + c2];
        }
        const double kv = K[i] * V;
        v[diag_slot[i]] += add;
        v[diag_slot[i]] += kv;
        diag[i] += kv;
        for (int c2 = 0; c2 < nc; ++c2) {
            rhs[i * nc + c2] += kv * Uo[i * nd + comp0 + c2];
            rhs[i * nc + c2] += alpha[i] * rho * P.g[comp0 + c2] * V;
        }
    }
}

// Pressure force -alpha p_f n A per face (owner: -alpha_O p_f n A; neighbour: the
// negative of -alpha_N p_f n A), p_f the face mean, the owner value on boundaries.
__global__ void k_mom_pressure(kcfd_dmesh_t m, int f0, int f1, int comp0, int nc, const double* __restrict__ alpha,
                               const double* __restrict__ p, double* __restrict__ rhs) {
    const int nd = m.ndim;
    for (int f = f0 + blockIdx.x * blockDim.x + threadIdx.x; f < f1; f += gridDim.x * blockDim.x) {
        const int o = m.owner[f];
        const bool in = f < m.n_internal;
        const int nb = in ? m.neigh[f] : o;
        const double pf = in ? 0.5 * (p[o] + p[nb]) : p[o];
        for (int c = 0; c < nc; ++c) {
            const double nn = m.normal[f * nd + comp0 + c];
            rhs[o * nc + c] += -alpha[o] * pf * nn * m.area[f];
            if (in) {
                const double fnb = -alpha[nb] * pf * nn * m.area[f];
                rhs[nb * nc + c] += -fnb;
            }
        }
    }
}

// apply_boundary_conditions for nc right-hand sides sharing one matrix.
__global__ void k_bc_tf(kcfd_dmesh_t m, int f0, int f1, const int8_t* __restrict__ bt, const double* __restrict__ bv,
                        const double* __restrict__ bg, int nc, const double* __restrict__ gamma,
                        const double* __restrict__ mf, double* __restrict__ v, double* __restrict__ diag,
                        double* __restrict__ rhs) {
    for (int f = f0 + blockIdx.x * blockDim.x + threadIdx.x; f < f1; f += gridDim.x * blockDim.x) {
        const double d = m.dlen[f];
        if (d < 1e-30) continue;
        const int o = m.owner[f], bi = f - m.n_internal;
        const int t = bt[bi];
        const double F = mf[f];
        if (t == 1) {
            const double c = gamma[o] * m.area[f] / d;
            v[m.diag_slot[o]] += c;
            diag[o] += c;
            for (int k = 0; k < nc; ++k) {
                const double phib = bv[bi * nc + k];
                double add = c * phib;
                if (F < 0) add = add + (-F) * phib;
                rhs[o * nc + k] += add;
            }
        } else if (t == 2) {
            for (int k = 0; k < nc; ++k) rhs[o * nc + k] += bg[bi] * m.area[f];
        } else if (t == 0) {
            if (F < 0) {
                v[m.diag_slot[o]] += -F;
                diag[o] += -F;
            }
        }
    }
}

// Diagonal floor of the tracked diagonal (models/two_fluid.py:611-614 and the
// like), then under_relax with it for nc right-hand sides.
__global__ void k_relax_tf(int n, int nc, int floor_diag, double alpha, const int* __restrict__ diag_slot,
                           const double* __restrict__ phi, double* __restrict__ v, double* __restrict__ diag,
                           double* __restrict__ rhs) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (floor_diag && diag[i] < 1e-20) diag[i] = 1e-10;
        if (alpha >= 1.0) continue;
        const double ap = diag[i];
        const double add = ap * (1.0 - alpha) / alpha;
        v[diag_slot[i]] += add;
        diag[i] += add;
        for (int c = 0; c < nc; ++c) rhs[i * nc + c] += add * phi[i * nc + c];
    }
}

__global__ void k_update_ap(int n, const double* __restrict__ diag, double* __restrict__ ap, int first) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double cur = fmax(diag[i], 1e-20);
        ap[i] = first ? cur : fmax(ap[i], cur);
    }
}

__global__ void k_pp_int_tf(kcfd_dmesh_t m, int f0, int f1, kcfd_tf_params_t P, const double* __restrict__ al,
                            const double* __restrict__ ag, const double* __restrict__ apl,
                            const double* __restrict__ apg, const double* __restrict__ mfl,
                            const double* __restrict__ mfg, double* __restrict__ v, double* __restrict__ diag,
                            double* __restrict__ rhs) {
    for (int f = f0 + blockIdx.x * blockDim.x + threadIdx.x; f < f1; f += gridDim.x * blockDim.x) {
        const double d = m.dlen[f];
        if (d < 1e-30) continue;
        const int o = m.owner[f], nb = m.neigh[f];
        const double al_f = 0.5 * (al[o] + al[nb]);
        const double ag_f = 0.5 * (ag[o] + ag[nb]);
        const double apl_f = 0.5 * (apl[o] + apl[nb]);
        const double apg_f = 0.5 * (apg[o] + apg[nb]);
        const double vol_f = 0.5 * (m.volume[o] + m.volume[nb]);
        const double cl = P.rho_l * al_f * vol_f / fmax(apl_f, 1e-30);
        const double cg = P.rho_g * ag_f * vol_f / fmax(apg_f, 1e-30);
        const double c = (cl + cg) * m.area[f] / d;
        v[m.diag_slot[o]] += c;
        v[m.diag_slot[nb]] += c;
        v[m.slot_on[f]] += -c;
        v[m.slot_no[f]] += -c;
        diag[o] += c;
        diag[nb] += c;
        const double tot = mfl[f] * al[o] + mfg[f] * ag[o];
        rhs[o] += -tot;
        rhs[nb] += tot;
    }
}

__global__ void k_pp_bnd_tf(kcfd_dmesh_t m, int f0, int f1, const double* __restrict__ al,
                            const double* __restrict__ ag, const double* __restrict__ mfl,
                            const double* __restrict__ mfg, double* __restrict__ rhs) {
    for (int f = f0 + blockIdx.x * blockDim.x + threadIdx.x; f < f1; f += gridDim.x * blockDim.x) {
        const int o = m.owner[f];
        const double tot = mfl[f] * al[o] + mfg[f] * ag[o];
        rhs[o] += -tot;
    }
}

__global__ void k_pin(const int* __restrict__ diag_slot, double* __restrict__ v, double* __restrict__ diag) {
    v[diag_slot[0]] += 1e10;
    diag[0] += 1e10;
}

__global__ void k_grad_diff(kcfd_dmesh_t m, int f0, int f1, const double* __restrict__ pp, double* __restrict__ grad) {
    const int nd = m.ndim;
    for (int f = f0 + blockIdx.x * blockDim.x + threadIdx.x; f < f1; f += gridDim.x * blockDim.x) {
        const int o = m.owner[f], nb = m.neigh[f];
        const double dp = pp[nb] - pp[o];
        for (int k = 0; k < nd; ++k) {
            const double fl = dp * m.normal[f * nd + k] * m.area[f];
            grad[o * nd + k] += fl;
            grad[nb * nd + k] -= fl;
        }
    }
}

__global__ void k_correct_tf(int n, int nd, double alpha_p, const double* __restrict__ vol, const double* __restrict__ pp,
                             const double* __restrict__ al, const double* __restrict__ ag,
                             const double* __restrict__ apl, const double* __restrict__ apg,
                             const double* __restrict__ grad, double* __restrict__ Ul, double* __restrict__ Ug,
                             double* __restrict__ p) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double V = vol[i];
        p[i] = p[i] + alpha_p * pp[i];
        for (int k = 0; k < nd; ++k) {
            double g = grad[i * nd + k];
            if (V > 1e-30) g = g / V;
            const double cl = -al[i] * V / fmax(apl[i], 1e-20) * g;
            const double cg = -ag[i] * V / fmax(apg[i], 1e-20) * g;
            Ul[i * nd + k] += alpha_p * cl;
            Ug[i * nd + k] += alpha_p * cg;
        }
    }
}

__global__ void k_alpha_source(int n, double rho_g, const double* __restrict__ dm, const double* __restrict__ vol,
                               double* __restrict__ rhs) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        if (fabs(dm[i]) > 1e-30) rhs[i] += dm[i] / rho_g * vol[i];
}

// Phase energy cell terms: temporal (alpha rho cp V / dt), interfacial exchange
// (Su = h a V T_other, Sp = -h a V), latent heat (-dot_m h_fg V).
__global__ void k_energy_cells(int n, kcfd_tf_params_t P, double rho, double cp, const int* __restrict__ diag_slot,
                               const double* __restrict__ vol, const double* __restrict__ alpha,
                               const double* __restrict__ Told, const double* __restrict__ Tother,
                               const double* __restrict__ hiaiV, const double* __restrict__ dm, double dm_sign,
                               double* __restrict__ v, double* __restrict__ diag, double* __restrict__ rhs) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double V = vol[i];
        if (Told) {
            const double c = alpha[i] * rho * cp * V / P.dt;
            v[diag_slot[i]] += c;
            diag[i] += c;
            rhs[i] += c * Told[i];
        }
        const double h = hiaiV[i];
        rhs[i] += h * Tother[i];
        v[diag_slot[i]] += h;
        diag[i] += h;
        const double d = dm_sign * dm[i];
        rhs[i] += -d * P.h_fg * V;
    }
}

// Wall heat flux q A alpha_phase[owner] on the boundary faces of heated patches.
__global__ void k_wall_flux(kcfd_dmesh_t m, int f0, int f1, const int8_t* __restrict__ qmask,
                            const double* __restrict__ q, const double* __restrict__ aw, double* __restrict__ rhs) {
    for (int f = f0 + blockIdx.x * blockDim.x + threadIdx.x; f < f1; f += gridDim.x * blockDim.x) {
        const int bi = f - m.n_internal;
        if (!qmask[bi]) continue;
        const int o = m.owner[f];
        rhs[o] += q[bi] * m.area[f] * aw[o];
    }
}

__global__ void k_nan_flag(int64_t m, const double* __restrict__ x, int with_inf, int* __restrict__ flag) {
    int bad = 0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x) {
        const double v = x[i];
        if (isnan(v) || (with_inf && isinf(v))) bad = 1;
    }
    if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(flag, 1);
}

// mode 0: restore old when flagged; 1: restore old when flagged, else clip to
// [lo, hi]; 2: zero when flagged.
__global__ void k_guard(int64_t m, int mode, double lo, double hi, const int* __restrict__ flag,
                        const double* __restrict__ old, double* __restrict__ x) {
    const int f = *flag;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x) {
        if (f) x[i] = (mode == 2) ? 0.0 : old[i];
        else if (mode == 1) x[i] = fmin(fmax(x[i], lo), hi);
    }
}

// alpha_g clipped to [0, 1], alpha_l = 1 - alpha_g, max |alpha_g - alpha_old|
// (an order-free max: the bits of non-negative doubles order like the values).
__global__ void k_alpha_finish(int n, double* __restrict__ ag, double* __restrict__ al,
                               const double* __restrict__ aold, unsigned long long* __restrict__ maxbits) {
    unsigned long long mx = 0ull;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double a = fmin(fmax(ag[i], 0.0), 1.0);
        ag[i] = a;
        al[i] = 1.0 - a;
        const double d = fabs(a - aold[i]);
        const unsigned long long b = (unsigned long long)__double_as_longlong(d);
        mx = b > mx ? b : mx;
    }
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long t = __shfl_xor_sync(0xffffffffu, mx, o);
        mx = t > mx ? t : mx;
    }
    if ((threadIdx.x & 31) == 0) atomicMax(maxbits, mx);
}

__global__ void k_strided_copy(int n, int nc_copy, const double* __restrict__ src, int ss, int so,
                               double* __restrict__ dst, int ds, int dof) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        for (int c = 0; c < nc_copy; ++c) dst[(int64_t)i * ds + dof + c] = src[(int64_t)i * ss + so + c];
}

int chk(const kcfd_dmesh_t* m) {
    KCFD_REQUIRE(m && m->owner && m->color_ptr && m->diag_slot, "kcfd_tf: NULL mesh descriptor");
    KCFD_REQUIRE(m->ndim == 2 || m->ndim == 3, "kcfd_tf: ndim must be 2 or 3");
    return KCFD_OK;
}

}  // namespace
}  // namespace kcfd

using namespace kcfd;

extern "C" {

int kcfd_tf_drag(const kcfd_dmesh_t* m, const kcfd_tf_params_t* P, const double* alpha_g, const double* U_g,
                 const double* U_l, double* K, void* stream) {
    if (int e = chk(m)) return e;
    KCFD_REQUIRE(P && alpha_g && U_g && U_l && K, "kcfd_tf_drag: NULL argument");
    k_drag<<<nblk(m->n_cells), kT, 0, (cudaStream_t)stream>>>(m->n_cells, m->ndim, *P, alpha_g, U_g, U_l, K);
    KCFD_CUDA(cudaGetLastError());
    return KCFD_OK;
}

int kcfd_tf_interfacial(const kcfd_dmesh_t* m, const kcfd_tf_params_t* P, const double* alpha_g, const double* U_g,
                        const double* U_l, double* hiaiV, void* stream) {
    if (int e = chk(m)) return e;
    KCFD_REQUIRE(P && alpha_g && U_g && U_l && hiaiV, "kcfd_tf_interfacial: NULL argument");
    k_interfacial<<<nblk(m->n_cells), kT, 0, (cudaStream_t)stream>>>(m->n_cells, m->ndim, *P, alpha_g, U_g, U_l,
                                                                     m->volume, hiaiV);
    KCFD_CUDA(cudaGetLastError());
    return KCFD_OK;
}

int kcfd_tf_phase_change(const kcfd_dmesh_t* m, const kcfd_tf_params_t* P, const double* alpha_l,
                         const double* alpha_g, const double* T_l, const double* T_g, double* dot_m, void* stream) {
    if (int e = chk(m)) return e;
    KCFD_REQUIRE(P && alpha_l && alpha_g && T_l && T_g && dot_m, "kcfd_tf_phase_change: NULL argument");
    k_phase_change<<<nblk(m->n_cells), kT, 0, (cudaStream_t)stream>>>(m->n_cells, *P, alpha_l, alpha_g, T_l, T_g,
                                                                      dot_m);
    KCFD_CUDA(cudaGetLastError());
    return KCFD_OK;
}

int kcfd_tf_gamma(const kcfd_dmesh_t* m, const kcfd_tf_params_t* P, int32_t kind, const double* alpha, double coef,
                  const double* alpha_g, const double* U_g, const double* U_l, double* gamma, void* stream) {
    if (int e = chk(m)) return e;
    KCFD_REQUIRE(P && alpha && gamma && (kind == 0 || (kind == 1 && alpha_g && U_g && U_l)),
                 "kcfd_tf_gamma: bad arguments");
    k_gamma<<<nblk(m->n_cells), kT, 0, (cudaStream_t)stream>>>(m->n_cells, m->ndim, kind, *P, alpha, coef, alpha_g,
                                                               U_g, U_l, gamma);
    KCFD_CUDA(cudaGetLastError());
    return KCFD_OK;
}

int kcfd_tf_face_flux(const kcfd_dmesh_t* m, int32_t kind, const double* mf, const double* alpha, double cp,
                      double* out, void* stream) {
    if (int e = chk(m)) return e;
    KCFD_REQUIRE((kind == 0 || kind == 1) && mf && alpha && out, "kcfd_tf_face_flux: bad arguments");
    k_face_flux<<<nblk(m->n_faces), kT, 0, (cudaStream_t)stream>>>(*m, kind, mf, alpha, cp, out);
    KCFD_CUDA(cudaGetLastError());
    return KCFD_OK;
}

int kcfd_tf_mass_flux(const kcfd_dmesh_t* m, double rho, const double* U, const double* U_b, double* mf,
                      void* stream) {
    if (int e = chk(m)) return e;
    KCFD_REQUIRE(U && U_b && mf, "kcfd_tf_mass_flux: NULL argument");
    k_mass_flux_b<<<nblk(m->n_faces), kT, 0, (cudaStream_t)stream>>>(*m, rho, U, U_b, mf);
    KCFD_CUDA(cudaGetLastError());
    return KCFD_OK;
}

int kcfd_tf_zero_gradient(const kcfd_dmesh_t* m, const int8_t* mask, const double* field, int32_t nc, double* bval,
                          void* stream) {
    if (int e = chk(m)) return e;
    KCFD_REQUIRE(mask && field && bval && nc >= 1 && nc <= 3, "kcfd_tf_zero_gradient: bad arguments");
    k_zero_grad<<<nblk(m->n_faces - m->n_internal), kT, 0, (cudaStream_t)stream>>>(*m, mask, field, nc, bval);
    KCFD_CUDA(cudaGetLastError());
    return KCFD_OK;
}

int kcfd_tf_momentum_sources(const kcfd_dmesh_t* m, const kcfd_tf_params_t* P, int32_t comp0, int32_t nc, double rho,
                             const double* alpha, const double* p, const double* K, const double* U_other,
                             const double* U_old, double* vals, double* diag, double* rhs, void* stream) {
    if (int e = chk(m)) return e;
    KCFD_REQUIRE(P && alpha && p && K && U_other && vals && diag && rhs, "kcfd_tf_momentum_sources: NULL argument");
    KCFD_REQUIRE(comp0 >= 0 && nc >= 1 && comp0 + nc <= m->ndim, "kcfd_tf_momentum_sources: bad components");
    cudaStream_t st = (cudaStream_t)stream;
    k_mom_cells_tf<<<nblk(m->n_cells), kT, 0, st>>>(m->n_cells, m->ndim, comp0, nc, *P, rho, m->diag_slot, m->volume,
                                                    alpha, K, U_other, U_old, vals, diag, rhs);
    auto pf = [&](int f0, int f1, int nb) { k_mom_pressure<<<nb, kT, 0, st>>>(*m, f0, f1, comp0, nc, alpha, p, rhs); };
    tf_colours(m, true, pf);
    tf_colours(m, false, pf);
    KCFD_CUDA(cudaGetLastError());
    return KCFD_OK;
}

int kcfd_tf_boundary(const kcfd_dmesh_t* m, const int8_t* btype, const double* bval, const double* bgrad, int32_t nc,
                     const double* gamma, const double* mf, double* vals, double* diag, double* rhs, void* stream) {
    if (int e = chk(m)) return e;
    KCFD_REQUIRE(btype && bval && bgrad && gamma && mf && vals && diag && rhs && nc >= 1 && nc <= 3,
                 "kcfd_tf_boundary: bad arguments");
    cudaStream_t st = (cudaStream_t)stream;
    tf_colours(m, false, [&](int f0, int f1, int nb) {
        k_bc_tf<<<nb, kT, 0, st>>>(*m, f0, f1, btype, bval, bgrad, nc, gamma, mf, vals, diag, rhs);
    });
    KCFD_CUDA(cudaGetLastError());
    return KCFD_OK;
}

int kcfd_tf_relax(const kcfd_dmesh_t* m, double alpha, const double* phi, int32_t nc, int32_t floor_diag, double* vals,
                  double* diag, double* rhs, void* stream) {
    if (int e = chk(m)) return e;
    KCFD_REQUIRE(phi && vals && diag && rhs && nc >= 1 && nc <= 3 && alpha > 0, "kcfd_tf_relax: bad arguments");
    k_relax_tf<<<nblk(m->n_cells), kT, 0, (cudaStream_t)stream>>>(m->n_cells, nc, floor_diag, alpha, m->diag_slot, phi,
                                                                  vals, diag, rhs);
    KCFD_CUDA(cudaGetLastError());
    return KCFD_OK;
}

int kcfd_tf_update_ap(const kcfd_dmesh_t* m, const double* diag, double* aP, int32_t first, void* stream) {
    if (int e = chk(m)) return e;
    KCFD_REQUIRE(diag && aP, "kcfd_tf_update_ap: NULL argument");
    k_update_ap<<<nblk(m->n_cells), kT, 0, (cudaStream_t)stream>>>(m->n_cells, diag, aP, first);
    KCFD_CUDA(cudaGetLastError());
    return KCFD_OK;
}

int kcfd_tf_pressure_assemble(const kcfd_dmesh_t* m, const kcfd_tf_params_t* P, const double* alpha_l,
                              const double* alpha_g, const double* aP_l, const double* aP_g, const double* mf_l,
                              const double* mf_g, double* vals, double* diag, double* rhs, void* stream) {
    if (int e = chk(m)) return e;
    KCFD_REQUIRE(P && alpha_l && alpha_g && aP_l && aP_g && mf_l && mf_g && vals && diag && rhs,
                 "kcfd_tf_pressure_assemble: NULL argument");
    cudaStream_t st = (cudaStream_t)stream;
    tf_colours(m, true, [&](int f0, int f1, int nb) {
        k_pp_int_tf<<<nb, kT, 0, st>>>(*m, f0, f1, *P, alpha_l, alpha_g, aP_l, aP_g, mf_l, mf_g, vals, diag, rhs);
    });
    tf_colours(m, false, [&](int f0, int f1, int nb) {
        k_pp_bnd_tf<<<nb, kT, 0, st>>>(*m, f0, f1, alpha_l, alpha_g, mf_l, mf_g, rhs);
    });
    k_pin<<<1, 1, 0, st>>>(m->diag_slot, vals, diag);
    KCFD_CUDA(cudaGetLastError());
    return KCFD_OK;
}

int kcfd_tf_correct(const kcfd_dmesh_t* m, double alpha_p, const double* pp, const double* alpha_l,
                    const double* alpha_g, const double* aP_l, const double* aP_g, double* grad, double* U_l,
                    double* U_g, double* p, void* stream) {
    if (int e = chk(m)) return e;
    KCFD_REQUIRE(pp && alpha_l && alpha_g && aP_l && aP_g && grad && U_l && U_g && p, "kcfd_tf_correct: NULL argument");
    cudaStream_t st = (cudaStream_t)stream;
    KCFD_CUDA(cudaMemsetAsync(grad, 0, sizeof(double) * (size_t)m->n_cells * m->ndim, st));
    tf_colours(m, true, [&](int f0, int f1, int nb) { k_grad_diff<<<nb, kT, 0, st>>>(*m, f0, f1, pp, grad); });
    k_correct_tf<<<nblk(m->n_cells), kT, 0, st>>>(m->n_cells, m->ndim, alpha_p, m->volume, pp, alpha_l, alpha_g, aP_l,
                                                  aP_g, grad, U_l, U_g, p);
    KCFD_CUDA(cudaGetLastError());
    return KCFD_OK;
}

int kcfd_tf_alpha_source(const kcfd_dmesh_t* m, double rho_g, const double* dot_m, double* rhs, void* stream) {
    if (int e = chk(m)) return e;
    KCFD_REQUIRE(dot_m && rhs, "kcfd_tf_alpha_source: NULL argument");
    k_alpha_source<<<nblk(m->n_cells), kT, 0, (cudaStream_t)stream>>>(m->n_cells, rho_g, dot_m, m->volume, rhs);
    KCFD_CUDA(cudaGetLastError());
    return KCFD_OK;
}

int kcfd_tf_energy_sources(const kcfd_dmesh_t* m, const kcfd_tf_params_t* P, double rho, double cp,
                           const double* alpha, const double* T_old, const double* T_other, const double* hiaiV,
                           const double* dot_m, double dm_sign, const int8_t* qmask, const double* q_b,
                           const double* alpha_wall, double* vals, double* diag, double* rhs, void* stream) {
    if (int e = chk(m)) return e;
    KCFD_REQUIRE(P && alpha && T_other && hiaiV && dot_m && qmask && q_b && alpha_wall && vals && diag && rhs,
                 "kcfd_tf_energy_sources: NULL argument");
    cudaStream_t st = (cudaStream_t)stream;
    k_energy_cells<<<nblk(m->n_cells), kT, 0, st>>>(m->n_cells, *P, rho, cp, m->diag_slot, m->volume, alpha, T_old,
                                                    T_other, hiaiV, dot_m, dm_sign, vals, diag, rhs);
    tf_colours(m, false, [&](int f0, int f1, int nb) {
        k_wall_flux<<<nb, kT, 0, st>>>(*m, f0, f1, qmask, q_b, alpha_wall, rhs);
    });
    KCFD_CUDA(cudaGetLastError());
    return KCFD_OK;
}

int kcfd_tf_guard(int64_t count, double* x, const double* old, int32_t mode, double lo, double hi, int32_t* flag,
                  void* stream) {
    KCFD_REQUIRE(x && flag && (mode == 2 || old) && mode >= 0 && mode <= 2, "kcfd_tf_guard: bad arguments");
    cudaStream_t st = (cudaStream_t)stream;
    KCFD_CUDA(cudaMemsetAsync(flag, 0, sizeof(int32_t), st));
    k_nan_flag<<<nblk(count), kT, 0, st>>>(count, x, mode == 1, flag);
    k_guard<<<nblk(count), kT, 0, st>>>(count, mode, lo, hi, flag, old, x);
    KCFD_CUDA(cudaGetLastError());
    return KCFD_OK;
}

int kcfd_tf_alpha_finish(int32_t n, double* alpha_g, double* alpha_l, const double* alpha_old, double* maxdiff,
                         void* stream) {
    KCFD_REQUIRE(n > 0 && alpha_g && alpha_l && alpha_old && maxdiff, "kcfd_tf_alpha_finish: bad arguments");
    cudaStream_t st = (cudaStream_t)stream;
    KCFD_CUDA(cudaMemsetAsync(maxdiff, 0, sizeof(double), st));
    k_alpha_finish<<<nblk(n), kT, 0, st>>>(n, alpha_g, alpha_l, alpha_old, (unsigned long long*)maxdiff);
    KCFD_CUDA(cudaGetLastError());
    return KCFD_OK;
}

int kcfd_tf_copy(int32_t n, int32_t ncopy, const double* src, int32_t src_stride, int32_t src_off, double* dst,
                 int32_t dst_stride, int32_t dst_off, void* stream) {
    KCFD_REQUIRE(n >= 0 && ncopy >= 1 && src && dst && src_off + ncopy <= src_stride && dst_off + ncopy <= dst_stride,
                 "kcfd_tf_copy: bad arguments");
    if (n == 0) return KCFD_OK;
    k_strided_copy<<<nblk(n), kT, 0, (cudaStream_t)stream>>>(n, ncopy, src, src_stride, src_off, dst, dst_stride,
                                                             dst_off);
    KCFD_CUDA(cudaGetLastError());
    return KCFD_OK;
}

}  // extern "C"
