// BiCGSTAB on sm_100a: one persistent launch per solve (or per batch of systems).
//
// Replaces the solve path of the K-CFD reference:
//   core/gpu_solver.py:82-155   gpu_bicgstab / _gpu_bicgstab_cupy (KCFD_STOP_GPU)
//   core/linear_solver.py:50-62 scipy bicgstab with create_preconditioner's M
//                               (KCFD_STOP_SCIPY; Jacobi core/preconditioner.py:43-47,
//                               ILU(0) in place of the SuperLU spilu at :49-54)
//
// Design
//  * A team of CTAs owns one system for the whole solve: a single CTA (small or
//    batched systems) or the whole cooperative grid (large systems). Each CTA owns a
//    contiguous row range; SpMV runs sub-warps of `lanes` threads per row and fuses the
//    dot products the next scalar needs into its epilogue; vector phases are fused
//    (p-update + preconditioner, s + preconditioner, x/r update + dots), so an
//    iteration streams 21 vectors and two SpMVs and crosses 5 team barriers.
//  * Dot products accumulate in FP64 with fixed-order trees (team.cuh), so every CTA
//    derives the same alpha/beta/omega and the same stopping decision without a host
//    round trip.
//  * MIXED: FP32 matrix and vectors in the inner iterations, FP64 outer residual
//    r = b - A x (FP64 matrix values), FP64 solution update, FP64 dots.
//  * nrhs = 3 solves the momentum components together: one matrix, three vectors
//    interleaved [n][3], per-component scalars and stopping.
//  * ILU(0): structural, in a level order (a cell colouring, or natural-order
//    dependency levels); factorisation and both sweeps proceed level by level with a
//    team barrier between levels.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "kcfd_common.h"
#include "team.cuh"

namespace kcfd {

constexpr double kEps2 = 4.930380657631324e-32;  // float64 eps^2 (scipy rhotol/omegatol)

struct SolveArgs {
    int n;
    int lanes;
    const int* indptr;
    const int* indices;
    const double* vals64;
    const float* vals32;
    // preconditioner
    void* dinv;           // Jacobi inverse diagonal, V
    const int* ilu_col;   // [nnz] columns of each row in level order
    const int* ilu_diag;  // [n] absolute position of the diagonal in the ILU layout
    void* lu;             // [nnz] factors, V
    void* ludinv;         // [n] 1 / u_ii, V
    const int* lev_ptr;
    const int* lev_rows;
    int nlev;
    // vectors
    void* work;           // 9 V vectors of n*nrhs
    double* x;            // [n*nrhs] FP64 solution (x0 on entry)
    const double* b;      // [n*nrhs] FP64 right-hand side
    double* r64;          // [n*nrhs] MIXED outer residual
    // control
    int stop;
    int maxiter;
    int max_refine;
    double rtol, atol, inner_rtol;
    int* iters_out;
    double* relres_out;
    int* status_out;
    TeamCtl ctl;
};

template <typename V>
struct Vecs {
    V *r, *rh, *p, *v, *t, *ph, *sh, *xi, *bi;
    __device__ Vecs(void* base, size_t len) {
        V* w = (V*)base;
        r = w;
        rh = w + len;
        p = w + 2 * len;
        v = w + 3 * len;
        t = w + 4 * len;
        ph = w + 5 * len;
        sh = w + 6 * len;
        xi = w + 7 * len;
        bi = w + 8 * len;
    }
};

template <class Team>
__device__ __forceinline__ void my_range(const Team& tm, int n, int& r0, int& r1) {
    int per = (n + tm.size - 1) / tm.size;
    r0 = min(n, tm.rank * per);
    r1 = min(n, r0 + per);
}

// y = A x over rows [r0, r1) with sub-warps of L lanes per row. epi(row, acc) runs on
// the first lane of the sub-warp.
template <typename VM, typename VX, int NRHS, class Epi>
__device__ __forceinline__ void spmv_range(const int* __restrict__ ip, const int* __restrict__ ix,
                                           const VM* __restrict__ val, const VX* __restrict__ x, int r0,
                                           int r1, int L, Epi epi) {
    const int lane = threadIdx.x & 31;
    const int sub = lane / L, sl = lane % L;
    const int rows_per_warp = 32 / L;
    const int warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    for (int base = r0 + warp * rows_per_warp; base < r1; base += nwarps * rows_per_warp) {
        const int row = base + sub;
        double acc[NRHS];
#pragma unroll
        for (int c = 0; c < NRHS; ++c) acc[c] = 0.0;
        if (row < r1) {
            const int kb = __ldg(ip + row), ke = __ldg(ip + row + 1);
            for (int k = kb + sl; k < ke; k += L) {
                const int j = __ldg(ix + k);
                const double a = (double)val[k];
#pragma unroll
                for (int c = 0; c < NRHS; ++c) acc[c] += a * (double)x[(size_t)j * NRHS + c];
            }
        }
        for (int o = L >> 1; o > 0; o >>= 1) {
#pragma unroll
            for (int c = 0; c < NRHS; ++c) acc[c] += __shfl_xor_sync(0xffffffffu, acc[c], o);
        }
        if (row < r1 && sl == 0) epi(row, acc);
    }
}

// Preconditioner z = M^{-1} q on this team's rows (Jacobi) or over all levels (ILU).
template <typename V, int NRHS, int PREC, class Team>
__device__ __forceinline__ bool apply_prec(Team& tm, const SolveArgs& a, const V* __restrict__ q,
                                           V* __restrict__ z, int r0, int r1) {
    if (PREC == KCFD_PREC_NONE) {
        for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x)
#pragma unroll
            for (int c = 0; c < NRHS; ++c) z[(size_t)i * NRHS + c] = q[(size_t)i * NRHS + c];
        return true;
    } else if (PREC == KCFD_PREC_JACOBI) {
        const V* dinv = (const V*)a.dinv;
        for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
            const V d = dinv[i];
#pragma unroll
            for (int c = 0; c < NRHS; ++c) z[(size_t)i * NRHS + c] = d * q[(size_t)i * NRHS + c];
        }
        return true;
    } else {
        // the sweeps read other teams' rows: the caller's q must be complete
        if (!tm.sync()) return false;
        const V* lu = (const V*)a.lu;
        const V* ldi = (const V*)a.ludinv;
        for (int l = 0; l < a.nlev; ++l) {
            const int b0 = a.lev_ptr[l], m = a.lev_ptr[l + 1] - b0;
            const int per = (m + tm.size - 1) / tm.size;
            const int s0 = min(m, tm.rank * per), s1 = min(m, s0 + per);
            for (int k = s0 + threadIdx.x; k < s1; k += blockDim.x) {
                const int i = a.lev_rows[b0 + k];
                double acc[NRHS];
#pragma unroll
                for (int c = 0; c < NRHS; ++c) acc[c] = (double)q[(size_t)i * NRHS + c];
                const int kb = a.indptr[i], kd = a.ilu_diag[i];
                for (int kk = kb; kk < kd; ++kk) {
                    const int j = a.ilu_col[kk];
                    const double lv = (double)lu[kk];
#pragma unroll
                    for (int c = 0; c < NRHS; ++c) acc[c] -= lv * (double)z[(size_t)j * NRHS + c];
                }
#pragma unroll
                for (int c = 0; c < NRHS; ++c) z[(size_t)i * NRHS + c] = (V)acc[c];
            }
            if (!tm.sync()) return false;
        }
        for (int l = a.nlev - 1; l >= 0; --l) {
            const int b0 = a.lev_ptr[l], m = a.lev_ptr[l + 1] - b0;
            const int per = (m + tm.size - 1) / tm.size;
            const int s0 = min(m, tm.rank * per), s1 = min(m, s0 + per);
            for (int k = s0 + threadIdx.x; k < s1; k += blockDim.x) {
                const int i = a.lev_rows[b0 + k];
                double acc[NRHS];
#pragma unroll
                for (int c = 0; c < NRHS; ++c) acc[c] = (double)z[(size_t)i * NRHS + c];
                const int kd = a.ilu_diag[i], ke = a.indptr[i + 1];
                for (int kk = kd + 1; kk < ke; ++kk) {
                    const int j = a.ilu_col[kk];
                    const double uv = (double)lu[kk];
#pragma unroll
                    for (int c = 0; c < NRHS; ++c) acc[c] -= uv * (double)z[(size_t)j * NRHS + c];
                }
                const double di = (double)ldi[i];
#pragma unroll
                for (int c = 0; c < NRHS; ++c) z[(size_t)i * NRHS + c] = (V)(acc[c] * di);
            }
            if (!tm.sync()) return false;
        }
        return true;
    }
}

// Per-rhs state of one BiCGSTAB run (identical in every thread of the team).
template <int NRHS>
struct KState {
    double rho[NRHS], rho_prev[NRHS], alpha[NRHS], omega[NRHS], thr[NRHS], bnorm[NRHS], rnorm[NRHS];
    int done[NRHS], status[NRHS], iters[NRHS];
};

// BiCGSTAB over this team's rows. Solves A xv = bv from xv's initial contents.
//   stop == KCFD_STOP_SCIPY: scipy.sparse.linalg.bicgstab's loop, threshold
//       max(atol, rtol ||b||) (rtol/atol passed in), eps^2 breakdown tests.
//   stop == KCFD_STOP_GPU: core/gpu_solver.py:127-153 (relative tests, 1e-30 guards).
// Per-rhs results land in st. Returns false if a team barrier failed.
template <typename V, typename VM, int NRHS, int PREC, class Team>
__device__ bool bicgstab_body(Team& tm, const SolveArgs& a, const VM* __restrict__ vals, V* __restrict__ xv,
                              const V* __restrict__ bv, Vecs<V> w, int stop, double rtol, double atol,
                              int maxiter, KState<NRHS>& st, double* smem) {
    const int n = a.n;
    int r0, r1;
    my_range(tm, n, r0, r1);
    const int* __restrict__ ip = a.indptr;
    const int* __restrict__ ix = a.indices;
    const bool gpu = (stop == KCFD_STOP_GPU);
    // r = b - A x ; rhat = r ; ||b||^2, ||r||^2 (= rhat.r)
    {
        double red[2 * NRHS];
#pragma unroll
        for (int k = 0; k < 2 * NRHS; ++k) red[k] = 0.0;
        spmv_range<VM, V, NRHS>(ip, ix, vals, xv, r0, r1, a.lanes, [&](int i, double* acc) {
#pragma unroll
            for (int c = 0; c < NRHS; ++c) {
                const size_t q = (size_t)i * NRHS + c;
                const double bb = (double)bv[q];
                const V rr = (V)(bb - acc[c]);
                w.r[q] = rr;
                w.rh[q] = rr;
                w.p[q] = (V)0;
                w.v[q] = (V)0;
                red[c] += bb * bb;
                red[NRHS + c] += (double)rr * (double)rr;
            }
        });
        if (!tm.template allreduce<2 * NRHS>(red, 0, smem)) return false;
#pragma unroll
        for (int c = 0; c < NRHS; ++c) {
            st.bnorm[c] = sqrt(red[c]);
            st.rnorm[c] = sqrt(red[NRHS + c]);
            st.rho[c] = red[NRHS + c];  // rhat . r with rhat == r
            st.rho_prev[c] = 1.0;
            st.alpha[c] = 1.0;
            st.omega[c] = 1.0;
            st.iters[c] = 0;
            st.status[c] = KCFD_OK;
            if (gpu) {
                st.thr[c] = rtol;  // relative: ||.|| / ||b|| < tol
                st.done[c] = (st.bnorm[c] < 1e-30);
            } else {
                st.thr[c] = fmax(atol, rtol * st.bnorm[c]);
                st.done[c] = (st.bnorm[c] == 0.0);
                if (st.done[c]) {
                    // scipy returns b (== 0) as the solution
                    for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) xv[(size_t)i * NRHS + c] = (V)0;
                }
            }
        }
    }
    for (int it = 0; it < maxiter; ++it) {
        // ---- top of iteration: stopping tests, beta, p update, phat = M^-1 p ----
        int active = 0;
        double beta[NRHS];
#pragma unroll
        for (int c = 0; c < NRHS; ++c) {
            beta[c] = 0.0;
            if (st.done[c]) continue;
            if (!gpu) {
                if (st.rnorm[c] < st.thr[c]) { st.done[c] = 1; st.status[c] = KCFD_OK; continue; }
                if (fabs(st.rho[c]) < kEps2) { st.done[c] = 1; st.status[c] = KCFD_BREAKDOWN; continue; }
                if (it > 0) {
                    if (fabs(st.omega[c]) < kEps2) { st.done[c] = 1; st.status[c] = KCFD_BREAKDOWN; continue; }
                    beta[c] = (st.rho[c] / st.rho_prev[c]) * (st.alpha[c] / st.omega[c]);
                }
            } else {
                if (fabs(st.rho[c]) < 1e-30) { st.done[c] = 1; st.status[c] = KCFD_BREAKDOWN; st.iters[c] = it + 1; continue; }
                beta[c] = (fabs(st.rho_prev[c] * st.omega[c]) > 1e-30)
                              ? (st.rho[c] / st.rho_prev[c]) * (st.alpha[c] / st.omega[c]) : 0.0;
            }
            active = 1;
        }
        if (!active) return true;
        for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
#pragma unroll
            for (int c = 0; c < NRHS; ++c) {
                if (st.done[c]) continue;
                const size_t q = (size_t)i * NRHS + c;
                if (gpu) {
                    w.p[q] = (V)((double)w.r[q] + beta[c] * ((double)w.p[q] - st.omega[c] * (double)w.v[q]));
                } else if (it == 0) {
                    w.p[q] = w.r[q];
                } else {
                    w.p[q] = (V)(((double)w.p[q] - st.omega[c] * (double)w.v[q]) * beta[c] + (double)w.r[q]);
                }
            }
        }
        V* ph = w.ph;
        if (PREC == KCFD_PREC_NONE) {
            ph = w.p;
        } else if (!apply_prec<V, NRHS, PREC>(tm, a, w.p, w.ph, r0, r1)) {
            return false;
        }
        if (!tm.sync()) return false;
        // ---- v = A phat ; rv = rhat . v ----
        double red1[NRHS];
#pragma unroll
        for (int c = 0; c < NRHS; ++c) red1[c] = 0.0;
        spmv_range<VM, V, NRHS>(ip, ix, vals, ph, r0, r1, a.lanes, [&](int i, double* acc) {
#pragma unroll
            for (int c = 0; c < NRHS; ++c) {
                const size_t q = (size_t)i * NRHS + c;
                const V vv = (V)acc[c];
                w.v[q] = vv;
                red1[c] += (double)w.rh[q] * (double)vv;
            }
        });
        if (!tm.template allreduce<NRHS>(red1, 1, smem)) return false;
#pragma unroll
        for (int c = 0; c < NRHS; ++c) {
            if (st.done[c]) continue;
            if (gpu) {
                st.alpha[c] = (fabs(red1[c]) > 1e-30) ? st.rho[c] / red1[c] : 0.0;
            } else {
                if (red1[c] == 0.0) { st.done[c] = 1; st.status[c] = KCFD_BREAKDOWN; st.iters[c] = it + 1; continue; }
                st.alpha[c] = st.rho[c] / red1[c];
            }
        }
        // ---- s = r - alpha v (in place in r) ; shat = M^-1 s ; ||s||^2 ----
        double red2[NRHS];
#pragma unroll
        for (int c = 0; c < NRHS; ++c) red2[c] = 0.0;
        for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
#pragma unroll
            for (int c = 0; c < NRHS; ++c) {
                if (st.done[c]) continue;
                const size_t q = (size_t)i * NRHS + c;
                const V s = (V)((double)w.r[q] - st.alpha[c] * (double)w.v[q]);
                w.r[q] = s;
                red2[c] += (double)s * (double)s;
            }
        }
        V* sh = w.sh;
        if (PREC == KCFD_PREC_NONE) {
            sh = w.r;
        } else if (PREC == KCFD_PREC_JACOBI) {
            apply_prec<V, NRHS, PREC>(tm, a, w.r, w.sh, r0, r1);
        }
        if (!tm.template allreduce<NRHS>(red2, 2, smem)) return false;
        int any_left = 0;
#pragma unroll
        for (int c = 0; c < NRHS; ++c) {
            if (st.done[c]) continue;
            const double sn = sqrt(red2[c]);
            const bool conv = gpu ? (sn / st.bnorm[c] < st.thr[c]) : (sn < st.thr[c]);
            if (conv) {
                // x += alpha * phat, then stop
                for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
                    const size_t q = (size_t)i * NRHS + c;
                    xv[q] = (V)((double)xv[q] + st.alpha[c] * (double)ph[q]);
                }
                st.done[c] = 1;
                st.status[c] = KCFD_OK;
                st.iters[c] = it + 1;
                st.rnorm[c] = sn;
                continue;
            }
            any_left = 1;
        }
        if (!any_left) return tm.sync();
        if (PREC == KCFD_PREC_ILU0) {
            if (!apply_prec<V, NRHS, PREC>(tm, a, w.r, w.sh, r0, r1)) return false;
        }
        if (!tm.sync()) return false;
        // ---- t = A shat ; t.s, t.t ----
        double red3[2 * NRHS];
#pragma unroll
        for (int k = 0; k < 2 * NRHS; ++k) red3[k] = 0.0;
        spmv_range<VM, V, NRHS>(ip, ix, vals, sh, r0, r1, a.lanes, [&](int i, double* acc) {
#pragma unroll
            for (int c = 0; c < NRHS; ++c) {
                const size_t q = (size_t)i * NRHS + c;
                const V tt = (V)acc[c];
                w.t[q] = tt;
                red3[c] += (double)tt * (double)w.r[q];
                red3[NRHS + c] += (double)tt * (double)tt;
            }
        });
        if (!tm.template allreduce<2 * NRHS>(red3, 3, smem)) return false;
#pragma unroll
        for (int c = 0; c < NRHS; ++c) {
            if (st.done[c]) continue;
            if (gpu) st.omega[c] = (red3[NRHS + c] > 1e-30) ? red3[c] / red3[NRHS + c] : 0.0;
            else st.omega[c] = red3[c] / red3[NRHS + c];
        }
        // ---- x += alpha phat + omega shat ; r = s - omega t ; rhat.r, ||r||^2 ----
        double red4[2 * NRHS];
#pragma unroll
        for (int k = 0; k < 2 * NRHS; ++k) red4[k] = 0.0;
        for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
#pragma unroll
            for (int c = 0; c < NRHS; ++c) {
                if (st.done[c]) continue;
                const size_t q = (size_t)i * NRHS + c;
                const double al = st.alpha[c], om = st.omega[c];
                if (gpu) xv[q] = (V)((double)xv[q] + (al * (double)ph[q] + om * (double)sh[q]));
                else xv[q] = (V)(((double)xv[q] + al * (double)ph[q]) + om * (double)sh[q]);
                const V rn = (V)((double)w.r[q] - om * (double)w.t[q]);
                w.r[q] = rn;
                red4[c] += (double)w.rh[q] * (double)rn;
                red4[NRHS + c] += (double)rn * (double)rn;
            }
        }
        if (!tm.template allreduce<2 * NRHS>(red4, 4, smem)) return false;
#pragma unroll
        for (int c = 0; c < NRHS; ++c) {
            if (st.done[c]) continue;
            st.rho_prev[c] = st.rho[c];
            st.rho[c] = red4[c];
            st.rnorm[c] = sqrt(red4[NRHS + c]);
            st.iters[c] = it + 1;
            if (gpu && st.rnorm[c] / st.bnorm[c] < st.thr[c]) {
                st.done[c] = 1;
                st.status[c] = KCFD_OK;
            }
        }
    }
#pragma unroll
    for (int c = 0; c < NRHS; ++c)
        if (!st.done[c]) {
            st.status[c] = KCFD_MAXITER;
            st.iters[c] = maxiter;
        }
    return true;
}

template <int NRHS>
__device__ void write_results(const SolveArgs& a, const KState<NRHS>& st, int team_rank) {
    if (team_rank == 0 && threadIdx.x == 0) {
        for (int c = 0; c < NRHS; ++c) {
            if (a.iters_out) a.iters_out[c] = st.iters[c];
            if (a.status_out) a.status_out[c] = st.status[c];
            if (a.relres_out) a.relres_out[c] = st.bnorm[c] > 0 ? st.rnorm[c] / st.bnorm[c] : 0.0;
        }
    }
}

// FP64 solve: x in place.
template <int NRHS, int PREC, class Team>
__device__ void solve_fp64(Team& tm, const SolveArgs& a, double* smem) {
    Vecs<double> w(a.work, (size_t)a.n * NRHS);
    KState<NRHS> st;
    bool ok = bicgstab_body<double, double, NRHS, PREC>(tm, a, a.vals64, a.x, a.b, w, a.stop, a.rtol, a.atol,
                                                        a.maxiter, st, smem);
    if (!ok) return;
    write_results<NRHS>(a, st, tm.rank);
}

// MIXED solve: FP64 outer refinement around FP32 inner BiCGSTAB runs.
template <int NRHS, int PREC, class Team>
__device__ void solve_mixed(Team& tm, const SolveArgs& a, double* smem) {
    const int n = a.n;
    int r0, r1;
    my_range(tm, n, r0, r1);
    Vecs<float> w(a.work, (size_t)n * NRHS);
    KState<NRHS> out;
    double thr[NRHS], rn[NRHS], bn[NRHS];
    int done[NRHS];
    int total_it = 0;
    for (int ref = 0;; ++ref) {
        // r64 = b - A64 x ; ||b||, ||r||
        double red[2 * NRHS];
#pragma unroll
        for (int k = 0; k < 2 * NRHS; ++k) red[k] = 0.0;
        spmv_range<double, double, NRHS>(a.indptr, a.indices, a.vals64, a.x, r0, r1, a.lanes,
                                         [&](int i, double* acc) {
#pragma unroll
                                             for (int c = 0; c < NRHS; ++c) {
                                                 const size_t q = (size_t)i * NRHS + c;
                                                 const double bb = a.b[q];
                                                 const double rr = bb - acc[c];
                                                 a.r64[q] = rr;
                                                 w.bi[q] = (float)rr;
                                                 w.xi[q] = 0.0f;
                                                 red[c] += bb * bb;
                                                 red[NRHS + c] += rr * rr;
                                             }
                                         });
        if (!tm.template allreduce<2 * NRHS>(red, 5, smem)) return;
        int left = 0;
#pragma unroll
        for (int c = 0; c < NRHS; ++c) {
            bn[c] = sqrt(red[c]);
            rn[c] = sqrt(red[NRHS + c]);
            if (ref == 0) {
                thr[c] = fmax(a.atol, a.rtol * bn[c]);
                out.status[c] = KCFD_OK;
                out.iters[c] = 0;
            }
            out.bnorm[c] = bn[c];
            out.rnorm[c] = rn[c];
            done[c] = (rn[c] < thr[c]) || (bn[c] == 0.0);
            if (ref > 0 && !done[c] && out.status[c] == KCFD_BREAKDOWN) done[c] = 1;
            if (done[c] && out.status[c] != KCFD_BREAKDOWN) out.status[c] = KCFD_OK;
            left |= !done[c];
        }
        if (!left) break;
        if (ref >= a.max_refine || total_it >= a.maxiter) {
#pragma unroll
            for (int c = 0; c < NRHS; ++c)
                if (!done[c]) out.status[c] = KCFD_MAXITER;
            break;
        }
        for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
#pragma unroll
            for (int c = 0; c < NRHS; ++c)
                if (done[c]) w.bi[(size_t)i * NRHS + c] = 0.0f;
        }
        if (!tm.sync()) return;
        // inner FP32 solve A32 e = r, from e = 0, to max(inner_rtol ||r||, thr/2)
        KState<NRHS> st;
        // reuse the scipy loop; per-rhs thresholds are absolute: pass rtol=inner, atol=thr/2
        double inner_atol = thr[0] * 0.5;
        for (int c = 1; c < NRHS; ++c) inner_atol = fmin(inner_atol, thr[c] * 0.5);
        bool ok = bicgstab_body<float, float, NRHS, PREC>(tm, a, a.vals32, w.xi, w.bi, w, KCFD_STOP_SCIPY,
                                                          a.inner_rtol, inner_atol, a.maxiter - total_it, st, smem);
        if (!ok) return;
        int max_it = 0;
        int progress = 0;
#pragma unroll
        for (int c = 0; c < NRHS; ++c) {
            if (done[c]) continue;
            out.iters[c] += st.iters[c];
            max_it = max(max_it, st.iters[c]);
            if (st.iters[c] > 0) progress = 1;
            else if (st.status[c] == KCFD_BREAKDOWN) out.status[c] = KCFD_BREAKDOWN;
        }
        total_it += max(max_it, 1);
        // x += e for the rhs still running
        for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
#pragma unroll
            for (int c = 0; c < NRHS; ++c) {
                if (done[c]) continue;
                const size_t q = (size_t)i * NRHS + c;
                a.x[q] = a.x[q] + (double)w.xi[q];
            }
        }
        if (!progress) {
#pragma unroll
            for (int c = 0; c < NRHS; ++c)
                if (!done[c] && out.status[c] == KCFD_OK) out.status[c] = KCFD_BREAKDOWN;
        }
        if (!tm.sync()) return;
    }
    write_results<NRHS>(a, out, tm.rank);
}

template <int MIXED, int NRHS, int PREC>
__global__ void __launch_bounds__(512) solve_grid_kernel(SolveArgs a) {
    __shared__ double smem[32 * kMaxK];
    GridTeam tm(a.ctl);
    if (MIXED) solve_mixed<NRHS, PREC>(tm, a, smem);
    else solve_fp64<NRHS, PREC>(tm, a, smem);
}

template <int MIXED, int NRHS, int PREC>
__global__ void __launch_bounds__(1024) solve_cta_kernel(SolveArgs a) {
    __shared__ double smem[32 * kMaxK];
    CtaTeam tm;
    if (MIXED) solve_mixed<NRHS, PREC>(tm, a, smem);
    else solve_fp64<NRHS, PREC>(tm, a, smem);
}

// ---------------------------------------------------------------- set-up kernels --
template <typename V>
__global__ void jacobi_setup_kernel(int n, const int* __restrict__ ip, const int* __restrict__ ix,
                                    const double* __restrict__ vals, V* __restrict__ dinv) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double d = 0.0;
        for (int k = ip[i]; k < ip[i + 1]; ++k)
            if (ix[k] == i) d += vals[k];
        dinv[i] = (V)((fabs(d) > 1e-30) ? 1.0 / d : 0.0);
    }
}

template <typename V>
__global__ void cast_kernel(int64_t m, const double* __restrict__ s, V* __restrict__ d) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x)
        d[i] = (V)s[i];
}

constexpr int kMaxIluRow = 64;

// Structural ILU(0), IKJ order, level by level. One thread per row.
template <typename V, class Team>
__device__ void ilu0_factor_body(Team& tm, const SolveArgs& a, const int* __restrict__ src,
                                 const double* __restrict__ vals) {
    V* lu = (V*)a.lu;
    V* ldi = (V*)a.ludinv;
    for (int l = 0; l < a.nlev; ++l) {
        const int b0 = a.lev_ptr[l], m = a.lev_ptr[l + 1] - b0;
        const int per = (m + tm.size - 1) / tm.size;
        const int s0 = min(m, tm.rank * per), s1 = min(m, s0 + per);
        for (int k = s0 + threadIdx.x; k < s1; k += blockDim.x) {
            const int i = a.lev_rows[b0 + k];
            const int lo = a.indptr[i], hi = a.indptr[i + 1], dp = a.ilu_diag[i];
            double wv[kMaxIluRow];
            for (int q = lo; q < hi; ++q) wv[q - lo] = vals[src[q]];
            for (int kk = lo; kk < dp; ++kk) {
                const int kr = a.ilu_col[kk];
                const double l_ik = wv[kk - lo] * (double)ldi[kr];
                wv[kk - lo] = l_ik;
                const int ke = a.indptr[kr + 1];
                for (int jj = a.ilu_diag[kr] + 1; jj < ke; ++jj) {
                    const int j = a.ilu_col[jj];
                    for (int q = kk + 1; q < hi; ++q)
                        if (a.ilu_col[q] == j) {
                            wv[q - lo] -= l_ik * (double)lu[jj];
                            break;
                        }
                }
            }
            for (int q = lo; q < hi; ++q) lu[q] = (V)wv[q - lo];
            const double u = wv[dp - lo];
            ldi[i] = (V)((fabs(u) > 1e-300) ? 1.0 / u : 0.0);
        }
        if (!tm.sync()) return;
    }
}

template <typename V>
__global__ void __launch_bounds__(512) ilu0_factor_grid(SolveArgs a, const int* src, const double* vals) {
    GridTeam tm(a.ctl);
    ilu0_factor_body<V>(tm, a, src, vals);
}

template <typename V>
__global__ void __launch_bounds__(1024) ilu0_factor_cta(SolveArgs a, const int* src, const double* vals) {
    CtaTeam tm;
    ilu0_factor_body<V>(tm, a, src, vals);
}

}  // namespace kcfd

// =================================================================== host side ==
using namespace kcfd;

struct kcfd_solver {
    kcfd_solver_opts_t o;
    int n = 0, nnz = 0;
    int grid = 0, block = 256, team = 1, lanes = 8;
    int sm_count = 0;
    void* work = nullptr;
    double* r64 = nullptr;
    void* dinv = nullptr;
    // ILU
    int* ilu_col = nullptr;
    int* ilu_diag = nullptr;
    int* ilu_src = nullptr;
    int* lev_ptr = nullptr;
    int* lev_rows = nullptr;
    int nlev = 0;
    void* lu = nullptr;
    void* ludinv = nullptr;
    // team control
    unsigned int* bar = nullptr;
    double* partials = nullptr;
    int* err = nullptr;
};

namespace {

template <int MIXED, int NRHS, int PREC>
void* pick_kernel(bool grid) {
    return grid ? (void*)solve_grid_kernel<MIXED, NRHS, PREC> : (void*)solve_cta_kernel<MIXED, NRHS, PREC>;
}

void* solve_kernel_ptr(int mixed, int nrhs, int prec, bool grid) {
#define KC_CASE(M, R, P) \
    if (mixed == M && nrhs == R && prec == P) return pick_kernel<M, R, P>(grid);
    KC_CASE(0, 1, 0) KC_CASE(0, 1, 1) KC_CASE(0, 1, 2)
    KC_CASE(0, 2, 0) KC_CASE(0, 2, 1) KC_CASE(0, 2, 2)
    KC_CASE(0, 3, 0) KC_CASE(0, 3, 1) KC_CASE(0, 3, 2)
    KC_CASE(1, 1, 0) KC_CASE(1, 1, 1) KC_CASE(1, 1, 2)
    KC_CASE(1, 2, 0) KC_CASE(1, 2, 1) KC_CASE(1, 2, 2)
    KC_CASE(1, 3, 0) KC_CASE(1, 3, 1) KC_CASE(1, 3, 2)
#undef KC_CASE
    return nullptr;
}

int free_solver(kcfd_solver* s) {
    if (!s) return KCFD_OK;
    void* ps[] = {s->work, s->r64, s->dinv, s->ilu_col, s->ilu_diag, s->ilu_src, s->lev_ptr,
                  s->lev_rows, s->lu, s->ludinv, s->bar, s->partials, s->err};
    for (void* p : ps)
        if (p) cudaFree(p);
    delete s;
    return KCFD_OK;
}

SolveArgs make_args(const kcfd_solver* s, const kcfd_csr_t* A) {
    SolveArgs a;
    std::memset(&a, 0, sizeof(a));
    a.n = s->n;
    a.lanes = s->lanes;
    a.indptr = A->indptr;
    a.indices = A->indices;
    a.vals64 = A->vals64;
    a.vals32 = A->vals32;
    a.dinv = s->dinv;
    a.ilu_col = s->ilu_col;
    a.ilu_diag = s->ilu_diag;
    a.lu = s->lu;
    a.ludinv = s->ludinv;
    a.lev_ptr = s->lev_ptr;
    a.lev_rows = s->lev_rows;
    a.nlev = s->nlev;
    a.work = s->work;
    a.r64 = s->r64;
    a.stop = s->o.stop;
    a.maxiter = s->o.maxiter;
    a.max_refine = s->o.max_refine;
    a.rtol = s->o.rtol;
    a.atol = s->o.atol;
    a.inner_rtol = s->o.inner_rtol;
    a.ctl.bar = s->bar;
    a.ctl.partials = s->partials;
    a.ctl.err = s->err;
    a.ctl.budget = 4000000000LL;  // ~2 s at 2 GHz per barrier wait
    return a;
}

int launch(const kcfd_solver* s, void* kernel, SolveArgs& a, cudaStream_t st) {
    void* args[] = {&a};
    KCFD_CUDA(cudaMemsetAsync(s->bar, 0, 2 * sizeof(unsigned), st));
    KCFD_CUDA(cudaMemsetAsync(s->err, 0, sizeof(int), st));
    if (s->team == 2) {
        KCFD_CUDA(cudaLaunchCooperativeKernel(kernel, dim3(s->grid), dim3(s->block), args, 0, st));
    } else {
        KCFD_CUDA(cudaLaunchKernel(kernel, dim3(1), dim3(s->block), args, 0, st));
    }
    KCFD_CUDA(cudaGetLastError());
    return KCFD_OK;
}

}  // namespace

extern "C" {

int kcfd_device_info(int32_t* sm_count, int32_t* cc_major, int32_t* cc_minor) {
    int dev = 0;
    KCFD_CUDA(cudaGetDevice(&dev));
    cudaDeviceProp p;
    KCFD_CUDA(cudaGetDeviceProperties(&p, dev));
    if (sm_count) *sm_count = p.multiProcessorCount;
    if (cc_major) *cc_major = p.major;
    if (cc_minor) *cc_minor = p.minor;
    return KCFD_OK;
}

int kcfd_solver_create(const kcfd_csr_t* A, const kcfd_solver_opts_t* opts, const int32_t* level_of_row_host,
                       kcfd_solver** out) {
    KCFD_REQUIRE(A && opts && out, "kcfd_solver_create: NULL argument");
    *out = nullptr;
    KCFD_REQUIRE(A->n > 0 && A->nnz >= A->n && A->indptr && A->indices, "kcfd_solver_create: bad CSR (n=%d nnz=%d)",
                 A->n, A->nnz);
    KCFD_REQUIRE(opts->nrhs >= 1 && opts->nrhs <= 3, "kcfd_solver_create: nrhs must be 1, 2 or 3");
    KCFD_REQUIRE(opts->precond >= 0 && opts->precond <= 2, "kcfd_solver_create: bad precond");
    KCFD_REQUIRE(opts->mode == KCFD_MODE_FP64 || opts->mode == KCFD_MODE_MIXED, "kcfd_solver_create: bad mode");
    KCFD_REQUIRE(opts->stop == KCFD_STOP_SCIPY || opts->stop == KCFD_STOP_GPU, "kcfd_solver_create: bad stop rule");
    KCFD_REQUIRE(!(opts->mode == KCFD_MODE_MIXED && opts->stop == KCFD_STOP_GPU),
                 "kcfd_solver_create: MIXED mode uses the scipy stopping rule");
    KCFD_REQUIRE(opts->maxiter >= 0, "kcfd_solver_create: maxiter < 0");
    auto* s = new kcfd_solver();
    s->o = *opts;
    if (s->o.mode == KCFD_MODE_MIXED) {
        if (s->o.inner_rtol <= 0) s->o.inner_rtol = 1e-4;
        if (s->o.max_refine <= 0) s->o.max_refine = 30;
    }
    s->n = A->n;
    s->nnz = A->nnz;
    int dev = 0;
    cudaDeviceProp prop;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaGetDeviceProperties(&prop, dev) != cudaSuccess) {
        free_solver(s);
        set_error("kcfd_solver_create: no CUDA device");
        return KCFD_CUDA_ERROR;
    }
    s->sm_count = prop.multiProcessorCount;
    const int nrhs = opts->nrhs;
    const bool mixed = opts->mode == KCFD_MODE_MIXED;
    const size_t vsz = mixed ? sizeof(float) : sizeof(double);
    // row structure on the host (once per pattern)
    std::vector<int> ip(A->n + 1), ix(A->nnz);
    if (cudaMemcpy(ip.data(), A->indptr, ip.size() * 4, cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(ix.data(), A->indices, ix.size() * 4, cudaMemcpyDeviceToHost) != cudaSuccess) {
        free_solver(s);
        set_error("kcfd_solver_create: cannot read the CSR pattern (device pointers expected)");
        return KCFD_BAD_INPUT;
    }
    if (ip[0] != 0 || ip[A->n] != A->nnz) {
        free_solver(s);
        set_error("kcfd_solver_create: indptr[0] != 0 or indptr[n] != nnz");
        return KCFD_BAD_INPUT;
    }
    for (int i = 0; i < A->n; ++i) {
        if (ip[i + 1] < ip[i]) {
            free_solver(s);
            set_error("kcfd_solver_create: indptr not monotone at row %d", i);
            return KCFD_BAD_INPUT;
        }
    }
    for (int k = 0; k < A->nnz; ++k)
        if (ix[k] < 0 || ix[k] >= A->n) {
            free_solver(s);
            set_error("kcfd_solver_create: column index %d out of range at %d", ix[k], k);
            return KCFD_BAD_INPUT;
        }
    // team and launch shape
    int team = opts->team;
    if (team == 0) team = ((int64_t)A->n * nrhs <= 40000) ? 1 : 2;
    s->team = team;
    int lanes = opts->lanes;
    if (lanes <= 0) {
        double avg = (double)A->nnz / A->n;
        lanes = 1;
        while (lanes < 32 && lanes < avg) lanes <<= 1;
    }
    KCFD_REQUIRE((lanes & (lanes - 1)) == 0 && lanes >= 1 && lanes <= 32, "kcfd_solver_create: lanes must be 1..32 pow2");
    s->lanes = lanes;
    s->block = opts->block > 0 ? opts->block : (team == 1 ? 1024 : 512);
    if (team == 2 && s->block > 512) s->block = 512;
    void* kern = solve_kernel_ptr(mixed, nrhs, opts->precond, team == 2);
    if (team == 2) {
        int per_sm = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, s->block, 0) != cudaSuccess || per_sm < 1) {
            free_solver(s);
            set_error("kcfd_solver_create: solver kernel cannot be resident (block %d)", s->block);
            return KCFD_CUDA_ERROR;
        }
        // a whole number of CTAs per SM, capped so rows per CTA stay meaningful
        int g = per_sm * s->sm_count;
        int max_useful = std::max(1, (int)((A->n + s->block - 1) / s->block));
        s->grid = std::max(1, std::min(g, max_useful));
    } else {
        s->grid = 1;
    }
    // allocations
    const size_t len = (size_t)A->n * nrhs;
    bool ok = cudaMalloc(&s->work, 9 * len * vsz) == cudaSuccess;
    if (mixed) ok = ok && cudaMalloc(&s->r64, len * sizeof(double)) == cudaSuccess;
    ok = ok && cudaMalloc(&s->bar, 2 * sizeof(unsigned)) == cudaSuccess;
    ok = ok && cudaMalloc(&s->err, sizeof(int)) == cudaSuccess;
    ok = ok && cudaMalloc(&s->partials, (size_t)kSlots * kMaxK * std::max(s->grid, 1) * sizeof(double)) == cudaSuccess;
    if (ok && opts->precond == KCFD_PREC_JACOBI) ok = cudaMalloc(&s->dinv, A->n * vsz) == cudaSuccess;
    if (ok && opts->precond == KCFD_PREC_ILU0) {
        // level of each row: caller's colouring / levels, else natural-order levels
        std::vector<int> lev(A->n, 0);
        if (level_of_row_host) {
            for (int i = 0; i < A->n; ++i) lev[i] = level_of_row_host[i];
        } else {
            for (int i = 0; i < A->n; ++i)
                for (int k = ip[i]; k < ip[i + 1]; ++k)
                    if (ix[k] < i) lev[i] = std::max(lev[i], lev[ix[k]] + 1);
        }
        int nlev = 0;
        for (int i = 0; i < A->n; ++i) {
            if (lev[i] < 0) { free_solver(s); set_error("kcfd_solver_create: negative level"); return KCFD_BAD_INPUT; }
            nlev = std::max(nlev, lev[i] + 1);
        }
        std::vector<int> icol(A->nnz), isrc(A->nnz), idiag(A->n);
        std::vector<int> order;
        for (int i = 0; i < A->n; ++i) {
            const int lo = ip[i], hi = ip[i + 1];
            if (hi - lo > kMaxIluRow) {
                free_solver(s);
                set_error("kcfd_solver_create: ILU(0) row %d has %d entries (max %d)", i, hi - lo, kMaxIluRow);
                return KCFD_BAD_INPUT;
            }
            order.resize(hi - lo);
            for (int k = lo; k < hi; ++k) order[k - lo] = k;
            auto key = [&](int k) { return std::make_pair(lev[ix[k]], ix[k]); };
            std::sort(order.begin(), order.end(), [&](int x, int y) { return key(x) < key(y); });
            idiag[i] = -1;
            for (int q = 0; q < hi - lo; ++q) {
                const int k = order[q];
                icol[lo + q] = ix[k];
                isrc[lo + q] = k;
                if (ix[k] == i) idiag[i] = lo + q;
                else if (lev[ix[k]] == lev[i]) {
                    free_solver(s);
                    set_error("kcfd_solver_create: rows %d and %d are coupled but share level %d", i, ix[k], lev[i]);
                    return KCFD_BAD_INPUT;
                }
            }
            if (idiag[i] < 0) {
                free_solver(s);
                set_error("kcfd_solver_create: row %d has no diagonal entry (ILU(0) needs it)", i);
                return KCFD_BAD_INPUT;
            }
        }
        std::vector<int> lptr(nlev + 1, 0), lrows(A->n);
        for (int i = 0; i < A->n; ++i) lptr[lev[i] + 1]++;
        for (int l = 0; l < nlev; ++l) lptr[l + 1] += lptr[l];
        std::vector<int> fill(lptr.begin(), lptr.end() - 1);
        for (int i = 0; i < A->n; ++i) lrows[fill[lev[i]]++] = i;
        s->nlev = nlev;
        ok = cudaMalloc(&s->ilu_col, A->nnz * 4) == cudaSuccess && cudaMalloc(&s->ilu_src, A->nnz * 4) == cudaSuccess &&
             cudaMalloc(&s->ilu_diag, A->n * 4) == cudaSuccess && cudaMalloc(&s->lev_ptr, (nlev + 1) * 4) == cudaSuccess &&
             cudaMalloc(&s->lev_rows, A->n * 4) == cudaSuccess && cudaMalloc(&s->lu, A->nnz * vsz) == cudaSuccess &&
             cudaMalloc(&s->ludinv, A->n * vsz) == cudaSuccess;
        ok = ok && cudaMemcpy(s->ilu_col, icol.data(), A->nnz * 4, cudaMemcpyHostToDevice) == cudaSuccess &&
             cudaMemcpy(s->ilu_src, isrc.data(), A->nnz * 4, cudaMemcpyHostToDevice) == cudaSuccess &&
             cudaMemcpy(s->ilu_diag, idiag.data(), A->n * 4, cudaMemcpyHostToDevice) == cudaSuccess &&
             cudaMemcpy(s->lev_ptr, lptr.data(), (nlev + 1) * 4, cudaMemcpyHostToDevice) == cudaSuccess &&
             cudaMemcpy(s->lev_rows, lrows.data(), A->n * 4, cudaMemcpyHostToDevice) == cudaSuccess;
    }
    if (ok) ok = cudaMemset(s->bar, 0, 2 * sizeof(unsigned)) == cudaSuccess && cudaMemset(s->err, 0, sizeof(int)) == cudaSuccess;
    if (!ok) {
        free_solver(s);
        set_error("kcfd_solver_create: device allocation failed");
        return KCFD_CUDA_ERROR;
    }
    *out = s;
    return KCFD_OK;
}

void kcfd_solver_destroy(kcfd_solver* s) { free_solver(s); }

int kcfd_solver_setup(kcfd_solver* s, const kcfd_csr_t* A, void* stream) {
    KCFD_REQUIRE(s && A, "kcfd_solver_setup: NULL argument");
    KCFD_REQUIRE(A->n == s->n && A->nnz == s->nnz, "kcfd_solver_setup: matrix size differs from the bound pattern");
    KCFD_REQUIRE(A->vals64, "kcfd_solver_setup: FP64 values required");
    cudaStream_t st = (cudaStream_t)stream;
    const bool mixed = s->o.mode == KCFD_MODE_MIXED;
    const int threads = 256;
    const int blocks = std::min((s->n + threads - 1) / threads, s->sm_count * 8);
    if (s->o.precond == KCFD_PREC_JACOBI) {
        if (mixed)
            jacobi_setup_kernel<float><<<blocks, threads, 0, st>>>(s->n, A->indptr, A->indices, A->vals64, (float*)s->dinv);
        else
            jacobi_setup_kernel<double><<<blocks, threads, 0, st>>>(s->n, A->indptr, A->indices, A->vals64, (double*)s->dinv);
        KCFD_CUDA(cudaGetLastError());
    } else if (s->o.precond == KCFD_PREC_ILU0) {
        SolveArgs a = make_args(s, A);
        KCFD_CUDA(cudaMemsetAsync(s->bar, 0, 2 * sizeof(unsigned), st));
        KCFD_CUDA(cudaMemsetAsync(s->err, 0, sizeof(int), st));
        const int* src = s->ilu_src;
        const double* vals = A->vals64;
        void* args[] = {&a, (void*)&src, (void*)&vals};
        if (s->team == 2) {
            void* k = mixed ? (void*)ilu0_factor_grid<float> : (void*)ilu0_factor_grid<double>;
            KCFD_CUDA(cudaLaunchCooperativeKernel(k, dim3(s->grid), dim3(s->block), args, 0, st));
        } else {
            void* k = mixed ? (void*)ilu0_factor_cta<float> : (void*)ilu0_factor_cta<double>;
            KCFD_CUDA(cudaLaunchKernel(k, dim3(1), dim3(s->block), args, 0, st));
        }
        KCFD_CUDA(cudaGetLastError());
    }
    return KCFD_OK;
}

int kcfd_solver_solve(kcfd_solver* s, const kcfd_csr_t* A, const double* b, double* x, int32_t* iters,
                      double* relres, int32_t* status, void* stream) {
    KCFD_REQUIRE(s && A && b && x, "kcfd_solver_solve: NULL argument");
    KCFD_REQUIRE(A->n == s->n && A->nnz == s->nnz, "kcfd_solver_solve: matrix size differs from the bound pattern");
    const bool mixed = s->o.mode == KCFD_MODE_MIXED;
    KCFD_REQUIRE(A->vals64 != nullptr, "kcfd_solver_solve: FP64 values required");
    KCFD_REQUIRE(!mixed || A->vals32 != nullptr, "kcfd_solver_solve: MIXED needs FP32 values (vals32)");
    SolveArgs a = make_args(s, A);
    a.x = x;
    a.b = b;
    a.iters_out = iters;
    a.relres_out = relres;
    a.status_out = status;
    cudaStream_t st = (cudaStream_t)stream;
    void* kern = solve_kernel_ptr(mixed, s->o.nrhs, s->o.precond, s->team == 2);
    KCFD_REQUIRE(kern != nullptr, "kcfd_solver_solve: no kernel for this configuration");
    return launch(s, kern, a, st);
}

// Error flag of the last solve's team barriers (KCFD_TIMEOUT when a wait expired).
int kcfd_solver_error(kcfd_solver* s, int32_t* err, void* stream) {
    KCFD_REQUIRE(s && err, "kcfd_solver_error: NULL argument");
    KCFD_CUDA(cudaMemcpyAsync(err, s->err, sizeof(int), cudaMemcpyDeviceToHost, (cudaStream_t)stream));
    KCFD_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
    return KCFD_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------- SpMV --
namespace kcfd {
template <typename VM, typename VX, int NRHS>
__global__ void spmv_kernel(int n, const int* __restrict__ ip, const int* __restrict__ ix, const VM* __restrict__ val,
                            const VX* __restrict__ x, VX* __restrict__ y, int L) {
    const int rows_per_cta = (blockDim.x / L);
    for (int r0 = blockIdx.x * rows_per_cta; r0 < n; r0 += gridDim.x * rows_per_cta) {
        const int r1 = min(n, r0 + rows_per_cta);
        spmv_range<VM, VX, NRHS>(ip, ix, val, x, r0, r1, L, [&](int i, double* acc) {
#pragma unroll
            for (int c = 0; c < NRHS; ++c) y[(size_t)i * NRHS + c] = (VX)acc[c];
        });
    }
}

template <typename V>
int spmv_launch(const kcfd_csr_t* A, const V* vals, const V* x, V* y, int nrhs, cudaStream_t st) {
    double avg = (double)A->nnz / std::max(A->n, 1);
    int L = 1;
    while (L < 32 && L < avg) L <<= 1;
    const int threads = 256;
    int blocks = (int)std::min<int64_t>(((int64_t)A->n * L + threads - 1) / threads, 148 * 16);
    blocks = std::max(blocks, 1);
    if (nrhs == 1)
        spmv_kernel<V, V, 1><<<blocks, threads, 0, st>>>(A->n, A->indptr, A->indices, vals, x, y, L);
    else if (nrhs == 2)
        spmv_kernel<V, V, 2><<<blocks, threads, 0, st>>>(A->n, A->indptr, A->indices, vals, x, y, L);
    else if (nrhs == 3)
        spmv_kernel<V, V, 3><<<blocks, threads, 0, st>>>(A->n, A->indptr, A->indices, vals, x, y, L);
    else {
        set_error("kcfd_spmv: nrhs must be 1, 2 or 3");
        return KCFD_BAD_INPUT;
    }
    KCFD_CUDA(cudaGetLastError());
    return KCFD_OK;
}
}  // namespace kcfd

extern "C" {
int kcfd_spmv_f64(const kcfd_csr_t* A, const double* x, double* y, int32_t nrhs, void* stream) {
    KCFD_REQUIRE(A && A->vals64 && x && y, "kcfd_spmv_f64: NULL argument");
    return spmv_launch<double>(A, A->vals64, x, y, nrhs, (cudaStream_t)stream);
}
int kcfd_cast_f64_f32(int64_t m, const double* src, float* dst, void* stream) {
    KCFD_REQUIRE(m >= 0 && (m == 0 || (src && dst)), "kcfd_cast_f64_f32: bad arguments");
    if (m == 0) return KCFD_OK;
    const int threads = 256;
    const int blocks = (int)std::min<int64_t>((m + threads - 1) / threads, 148 * 32);
    cast_kernel<float><<<blocks, threads, 0, (cudaStream_t)stream>>>(m, src, dst);
    KCFD_CUDA(cudaGetLastError());
    return KCFD_OK;
}
int kcfd_spmv_f32(const kcfd_csr_t* A, const float* x, float* y, int32_t nrhs, void* stream) {
    KCFD_REQUIRE(A && A->vals32 && x && y, "kcfd_spmv_f32: NULL argument");
    return spmv_launch<float>(A, A->vals32, x, y, nrhs, (cudaStream_t)stream);
}
}
