// BiCGSTAB on sm_100a: one persistent launch per solve.
//
// Replaces the solve path of the K-CFD reference:
//   core/gpu_solver.py:82-155   gpu_bicgstab / _gpu_bicgstab_cupy (KCFD_STOP_GPU)
//   core/linear_solver.py:50-62 scipy bicgstab with create_preconditioner's M
//                               (KCFD_STOP_SCIPY; Jacobi core/preconditioner.py:43-47,
//                               structural ILU(0) in place of the SuperLU spilu at :49-54)
//
// Design
//  * A team of CTAs owns one system for the whole solve: a single CTA (small systems)
//    or the whole cooperative grid (large systems). Rows are grouped into levels
//    (one level for Jacobi / none; the ILU(0) dependency levels otherwise) and every
//    CTA owns an even slice of every level, so level-by-level work keeps all SMs busy.
//  * SpMV runs sub-warps of `lanes` threads per row and fuses the dot product the
//    next scalar needs into its epilogue; the vector phases are fused (p-update +
//    Jacobi, s + Jacobi, x/r update + dots): an iteration streams 21 vectors and two
//    SpMVs and crosses 5 team barriers (Jacobi) or 11 (two-level ILU(0)).
//  * Dot products accumulate in FP64 with fixed-order trees (team.cuh); every CTA
//    derives the same alpha/beta/omega and stopping decision with no host round trip.
//  * MIXED: FP32 matrix and vectors in the inner iterations; FP64 outer residual
//    r = b - A x with the FP64 values, FP64 solution update, FP64 dots. Inner runs are
//    capped per refinement step; a step that does not lower the FP64 residual is
//    undone and ends that right-hand side (status BREAKDOWN).
//  * nrhs 2/3 solve the momentum components together: one matrix, vectors
//    interleaved [n][nrhs], per-component scalars and stopping.
//  * ILU(0) solves the level-permuted system P A P^T: levels are contiguous row
//    ranges, the lower part of a row is exactly its columns left of the diagonal, and
//    the forward / backward sweeps read contiguous memory. b and x are permuted on
//    entry and exit inside the same launch.
//  * Large FP64 systems run on the graph engine instead (team 3, graph_engine.cuh):
//    the same iteration as lean phase kernels in one CUDA graph with a device-side
//    WHILE loop. A solve issued while its stream is being captured falls back to the
//    persistent grid kernel (the engine's graph is not nested into the capture).
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <vector>
#include <type_traits>

#include "kcfd_common.h"
#include "team.cuh"
#include "amg.h"
#include "graph_engine.cuh"

namespace kcfd {

constexpr double kEps2 = 4.930380657631324e-32;  // float64 eps^2 (scipy rhotol/omegatol)

struct SolveArgs {
    int n;
    int lanes;
    // matrix of the Krylov iterations (the level-permuted copy when perm != null)
    const int* indptr;
    const int* indices;
    const double* vals64;
    const float* vals32;
    const int* perm;     // [n] permuted row -> caller row, or null
    double* px;          // [n*nrhs] permuted FP64 solution (perm only)
    double* pb;          // [n*nrhs] permuted FP64 rhs (perm only)
    // preconditioner
    void* dinv;          // Jacobi inverse diagonal, V
    const int* diag;     // [n] position of the diagonal (ILU)
    void* lu;            // [nnz] ILU factors, V
    void* ludinv;        // [n] 1 / u_ii, V
    const int* lev_ptr;  // [nlev+1] level row ranges
    int nlev;
    // vectors
    void* work;          // 9 V vectors of n*nrhs
    double* x;           // caller FP64 solution (x0 on entry)
    const double* b;     // caller FP64 rhs
    double* r64;         // MIXED outer residual
    // control
    int stop;
    int maxiter;
    int max_refine;
    int inner_maxiter;
    int max_restarts;    // KCFD_STOP_SCIPY: restarts on rho / omega breakdown (0: scipy's stop)
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

// This CTA's slice [s0, s1) of level l. The level table is written before the
// launch and never inside it; a single level is the whole row range.
template <class Team>
__device__ __forceinline__ void level_slice(const Team& tm, const SolveArgs& a, int l, int& s0, int& s1) {
    const int b0 = (a.nlev == 1) ? 0 : a.lev_ptr[l];
    const int m = ((a.nlev == 1) ? a.n : a.lev_ptr[l + 1]) - b0;
    const int per = (m + tm.size - 1) / tm.size;
    s0 = b0 + min(m, tm.rank * per);
    s1 = b0 + min(m, tm.rank * per + per);
}

// f(s0, s1) over this CTA's slices of every level: the rows it owns.
template <class Team, class F>
__device__ __forceinline__ void for_my_rows(const Team& tm, const SolveArgs& a, F f) {
    for (int l = 0; l < a.nlev; ++l) {
        int s0, s1;
        level_slice(tm, a, l, s0, s1);
        if (s1 > s0) f(s0, s1);
    }
}

// y = A x over rows [r0, r1) with sub-warps of L lanes per row. epi(row, acc) runs on
// the first lane of the sub-warp.
// DIFF: difference form y_i = d_i x_i + sum_{j != i} a_ij (x_j - x_i), where the
// diagonal slot holds the row sum d_i = sum_j a_ij. Identical in exact arithmetic; in
// FP32 it keeps near-zero row sums (Neumann-type pressure operators) exact instead of
// leaving them to the rounding of a large diagonal.
template <typename VM, typename VX, int NRHS, bool DIFF = false, class Epi>
// Only the matrix (ip, ix, val) is read-only for the whole launch; x is rewritten
// between phases, so it is read through the coherent path.
__device__ __forceinline__ void spmv_range(const int* __restrict__ ip, const int* __restrict__ ix,
                                           const VM* __restrict__ val, const VX* x, int r0, int r1, int L,
                                           Epi epi) {
    if (L == 1) {
        // one thread per row: the first 8 columns and values are loaded before the
        // first gather of x (three memory round trips per row instead of one per
        // entry); entries are summed in row order as below
        constexpr int E = 8;
        for (int row = r0 + (int)threadIdx.x; row < r1; row += blockDim.x) {
            const int kb = __ldg(ip + row), ke = __ldg(ip + row + 1);
            int cj[E];
            double av[E];
#pragma unroll
            for (int k = 0; k < E; ++k) {
                const bool in = kb + k < ke;
                cj[k] = in ? __ldg(ix + kb + k) : row;
                av[k] = in ? (double)val[kb + k] : 0.0;
            }
            double xi[NRHS], acc[NRHS];
#pragma unroll
            for (int c = 0; c < NRHS; ++c) {
                acc[c] = 0.0;
                if (DIFF) xi[c] = (double)x[(size_t)row * NRHS + c];
            }
            auto term = [&](int j, double a) {
                if (DIFF) {
                    if (j == row) {
#pragma unroll
                        for (int c = 0; c < NRHS; ++c) acc[c] += a * xi[c];
                    } else {
#pragma unroll
                        for (int c = 0; c < NRHS; ++c) acc[c] += a * ((double)x[(size_t)j * NRHS + c] - xi[c]);
                    }
                } else {
#pragma unroll
                    for (int c = 0; c < NRHS; ++c) acc[c] += a * (double)x[(size_t)j * NRHS + c];
                }
            };
#pragma unroll
            for (int k = 0; k < E; ++k)
                if (kb + k < ke) term(cj[k], av[k]);
            for (int k = kb + E; k < ke; ++k) term(__ldg(ix + k), (double)val[k]);
            epi(row, acc);
        }
        return;
    }
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
            double xi[NRHS];
            if (DIFF) {
#pragma unroll
                for (int c = 0; c < NRHS; ++c) xi[c] = (double)x[(size_t)row * NRHS + c];
            }
#pragma unroll 4
            for (int k = kb + sl; k < ke; k += L) {
                const int j = __ldg(ix + k);
                const double av = (double)val[k];
                if (DIFF) {
                    if (j == row) {
#pragma unroll
                        for (int c = 0; c < NRHS; ++c) acc[c] += av * xi[c];
                    } else {
#pragma unroll
                        for (int c = 0; c < NRHS; ++c) acc[c] += av * ((double)x[(size_t)j * NRHS + c] - xi[c]);
                    }
                } else {
#pragma unroll
                    for (int c = 0; c < NRHS; ++c) acc[c] += av * (double)x[(size_t)j * NRHS + c];
                }
            }
        }
        for (int o = L >> 1; o > 0; o >>= 1) {
#pragma unroll
            for (int c = 0; c < NRHS; ++c) acc[c] += __shfl_xor_sync(0xffffffffu, acc[c], o);
        }
        if (row < r1 && sl == 0) epi(row, acc);
    }
}

// z = (LU)^{-1} q on the level-permuted system. Level 0 of the forward sweep and the
// last level of the backward sweep only touch rows this CTA owns, so the sweeps need
// 2 (nlev - 1) barriers; the caller syncs before anything gathers z.
template <typename V, int NRHS, class Team>
__device__ __forceinline__ bool ilu_apply(Team& tm, const SolveArgs& a, const V* q, V* z) {
    const V* lu = (const V*)a.lu;
    const V* ldi = (const V*)a.ludinv;
    for (int l = 0; l < a.nlev; ++l) {
        if (l > 0 && !tm.sync()) return false;
        int s0, s1;
        level_slice(tm, a, l, s0, s1);
        for (int i = s0 + threadIdx.x; i < s1; i += blockDim.x) {
            double acc[NRHS];
#pragma unroll
            for (int c = 0; c < NRHS; ++c) acc[c] = (double)q[(size_t)i * NRHS + c];
            const int kb = __ldg(a.indptr + i), kd = __ldg(a.diag + i);
#pragma unroll 4
            for (int k = kb; k < kd; ++k) {
                const int j = __ldg(a.indices + k);
                const double lv = (double)lu[k];
#pragma unroll
                for (int c = 0; c < NRHS; ++c) acc[c] -= lv * (double)z[(size_t)j * NRHS + c];
            }
#pragma unroll
            for (int c = 0; c < NRHS; ++c) z[(size_t)i * NRHS + c] = (V)acc[c];
        }
    }
    for (int l = a.nlev - 1; l >= 0; --l) {
        if (l < a.nlev - 1 && !tm.sync()) return false;
        int s0, s1;
        level_slice(tm, a, l, s0, s1);
        for (int i = s0 + threadIdx.x; i < s1; i += blockDim.x) {
            double acc[NRHS];
#pragma unroll
            for (int c = 0; c < NRHS; ++c) acc[c] = (double)z[(size_t)i * NRHS + c];
            const int kd = __ldg(a.diag + i), ke = __ldg(a.indptr + i + 1);
#pragma unroll 4
            for (int k = kd + 1; k < ke; ++k) {
                const int j = __ldg(a.indices + k);
                const double uv = (double)lu[k];
#pragma unroll
                for (int c = 0; c < NRHS; ++c) acc[c] -= uv * (double)z[(size_t)j * NRHS + c];
            }
            const double di = (double)ldi[i];
#pragma unroll
            for (int c = 0; c < NRHS; ++c) z[(size_t)i * NRHS + c] = (V)(acc[c] * di);
        }
    }
    return true;
}

// Per-rhs scalar state of one BiCGSTAB run. It lives in shared memory: thread 0
// writes it between block barriers, every thread reads it (identical in every CTA of
// the team, since all CTAs derive it from the same fixed-order sums).
template <int NRHS>
struct KState {
    double rho[NRHS], rho_prev[NRHS], alpha[NRHS], omega[NRHS], beta[NRHS], thr[NRHS], bnorm[NRHS], rnorm[NRHS];
    int done[NRHS], status[NRHS], iters[NRHS], nonfinite[NRHS];
    int restarts[NRHS], rs[NRHS];  // restarts used; 1 while this iteration restarts
    int active, any_left;
};

__device__ __forceinline__ bool finite(double v) { return isfinite(v); }

// BiCGSTAB on this team's rows. Solves A xv = bv from xv (x_zero: xv == 0, r = b).
//   stop == KCFD_STOP_SCIPY: scipy.sparse.linalg.bicgstab's loop, threshold
//       max(atol, rtol ||b||), eps^2 breakdown tests.
//   stop == KCFD_STOP_GPU: core/gpu_solver.py:127-153 (relative tests, 1e-30 guards).
// A non-finite scalar ends a right-hand side with KCFD_BREAKDOWN (nonfinite = 1).
// Returns false if a team barrier failed.
template <typename V, typename VM, int NRHS, int PREC, class Team>
__device__ bool bicgstab_body(Team& tm, const SolveArgs& a, const VM* __restrict__ vals, V* xv,
                              const V* bv, bool x_zero, const Vecs<V>& w, int stop, double rtol,
                              double atol, int maxiter, KState<NRHS>& st, double* smem) {
    const int* __restrict__ ip = a.indptr;
    const int* __restrict__ ix = a.indices;
    const bool gpu = (stop == KCFD_STOP_GPU);
    const V* dinv = (const V*)a.dinv;
    constexpr bool kDiff = sizeof(VM) == 4;  // FP32 operator: difference form
    constexpr int kU = (NRHS == 1) ? 4 : (NRHS == 2 ? 2 : 1);  // rows per thread in flight
    const bool t0 = threadIdx.x == 0;
    // ---- r = b - A x ; rhat = r ; ||b||^2, ||r||^2 (= rhat.r) ----
    {
        double red[2 * NRHS];
#pragma unroll
        for (int k = 0; k < 2 * NRHS; ++k) red[k] = 0.0;
        auto init_row = [&](int i, const double* acc) {
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
        };
        if (x_zero) {
            for_my_rows(tm, a, [&](int s0, int s1) {
                for (int i = s0 + threadIdx.x; i < s1; i += blockDim.x) {
                    double z[NRHS];
#pragma unroll
                    for (int c = 0; c < NRHS; ++c) z[c] = 0.0;
                    init_row(i, z);
                }
            });
        } else {
            for_my_rows(tm, a, [&](int s0, int s1) {
                spmv_range<VM, V, NRHS, kDiff>(ip, ix, vals, xv, s0, s1, a.lanes, init_row);
            });
        }
        if (!tm.template allreduce<2 * NRHS>(red, 0, smem)) return false;
        if (t0) {
            for (int c = 0; c < NRHS; ++c) {
                st.bnorm[c] = sqrt(red[c]);
                st.rnorm[c] = sqrt(red[NRHS + c]);
                st.rho[c] = red[NRHS + c];  // rhat . r with rhat == r
                st.rho_prev[c] = 1.0;
                st.alpha[c] = 1.0;
                st.omega[c] = 1.0;
                st.beta[c] = 0.0;
                st.iters[c] = 0;
                st.status[c] = KCFD_OK;
                st.restarts[c] = 0;
                st.rs[c] = 0;
                st.nonfinite[c] = !finite(red[c]) || !finite(red[NRHS + c]);
                if (gpu) {
                    st.thr[c] = rtol;  // relative: ||.|| / ||b|| < tol
                    st.done[c] = (st.bnorm[c] < 1e-30);
                } else {
                    st.thr[c] = fmax(atol, rtol * st.bnorm[c]);
                    st.done[c] = (st.bnorm[c] == 0.0);
                }
                if (st.nonfinite[c]) {
                    st.done[c] = 1;
                    st.status[c] = KCFD_BREAKDOWN;
                }
            }
        }
        __syncthreads();
        if (!gpu) {
            // scipy returns b (== 0) as the solution
#pragma unroll
            for (int c = 0; c < NRHS; ++c) {
                if (!(st.bnorm[c] == 0.0)) continue;
                for_my_rows(tm, a, [&](int s0, int s1) {
                    for (int i = s0 + threadIdx.x; i < s1; i += blockDim.x) xv[(size_t)i * NRHS + c] = (V)0;
                });
            }
        }
    }
    for (int it = 0; it < maxiter; ++it) {
        // ---- top of iteration: stopping tests, beta ----
        if (t0) {
            int active = 0;
            for (int c = 0; c < NRHS; ++c) {
                st.beta[c] = 0.0;
                if (st.done[c]) continue;
                if (!gpu) {
                    if (st.rnorm[c] < st.thr[c]) { st.done[c] = 1; st.status[c] = KCFD_OK; continue; }
                    if (fabs(st.rho[c]) < kEps2 || (it > 0 && fabs(st.omega[c]) < kEps2)) {
                        if (st.restarts[c] < a.max_restarts && st.rnorm[c] > 0.0) {
                            // restart: rhat = r, p = r (this iteration), rho = ||r||^2
                            st.restarts[c] += 1;
                            st.rs[c] = 1;
                            st.rho[c] = st.rnorm[c] * st.rnorm[c];
                            st.rho_prev[c] = st.alpha[c] = st.omega[c] = 1.0;
                            active = 1;
                            continue;
                        }
                        st.done[c] = 1;
                        st.status[c] = KCFD_BREAKDOWN;
                        continue;
                    }
                    if (it > 0) st.beta[c] = (st.rho[c] / st.rho_prev[c]) * (st.alpha[c] / st.omega[c]);
                } else {
                    if (fabs(st.rho[c]) < 1e-30) { st.done[c] = 1; st.status[c] = KCFD_BREAKDOWN; st.iters[c] = it + 1; continue; }
                    st.beta[c] = (fabs(st.rho_prev[c] * st.omega[c]) > 1e-30)
                                     ? (st.rho[c] / st.rho_prev[c]) * (st.alpha[c] / st.omega[c]) : 0.0;
                }
                if (!finite(st.beta[c])) { st.done[c] = 1; st.status[c] = KCFD_BREAKDOWN; st.nonfinite[c] = 1; continue; }
                active = 1;
            }
            st.active = active;
        }
        __syncthreads();
        if (!st.active) return true;
        // ---- p update, phat = M^-1 p ----
        for_my_rows(tm, a, [&](int s0, int s1) {
            for (int base = s0 + threadIdx.x; base < s1; base += kU * blockDim.x) {
                V rr[kU][NRHS], pp[kU][NRHS], vv[kU][NRHS], dd[kU];
#pragma unroll
                for (int u = 0; u < kU; ++u) {
                    const int i = base + u * blockDim.x;
                    if (i >= s1) continue;
                    dd[u] = (PREC == KCFD_PREC_JACOBI) ? dinv[i] : (V)1;
#pragma unroll
                    for (int c = 0; c < NRHS; ++c) {
                        if (st.done[c]) continue;
                        const size_t q = (size_t)i * NRHS + c;
                        rr[u][c] = w.r[q];
                        pp[u][c] = w.p[q];
                        vv[u][c] = w.v[q];
                    }
                }
#pragma unroll
                for (int u = 0; u < kU; ++u) {
                    const int i = base + u * blockDim.x;
                    if (i >= s1) continue;
#pragma unroll
                    for (int c = 0; c < NRHS; ++c) {
                        if (st.done[c]) continue;
                        const size_t q = (size_t)i * NRHS + c;
                        const double om = st.omega[c], be = st.beta[c];
                        V pn;
                        if (gpu) pn = (V)((double)rr[u][c] + be * ((double)pp[u][c] - om * (double)vv[u][c]));
                        else if (it == 0 || st.rs[c]) pn = rr[u][c];
                        else pn = (V)(((double)pp[u][c] - om * (double)vv[u][c]) * be + (double)rr[u][c]);
                        if (st.rs[c]) w.rh[q] = rr[u][c];
                        w.p[q] = pn;
                        if (PREC == KCFD_PREC_JACOBI) w.ph[q] = dd[u] * pn;
                    }
                }
            }
        });
        V* ph = (PREC == KCFD_PREC_NONE) ? w.p : w.ph;
        if (PREC == KCFD_PREC_ILU0 && !ilu_apply<V, NRHS>(tm, a, w.p, w.ph)) return false;
        if (!tm.sync()) return false;
        // ---- v = A phat ; rv = rhat . v ----
        double red1[NRHS];
#pragma unroll
        for (int c = 0; c < NRHS; ++c) red1[c] = 0.0;
        for_my_rows(tm, a, [&](int s0, int s1) {
            spmv_range<VM, V, NRHS, kDiff>(ip, ix, vals, ph, s0, s1, a.lanes, [&](int i, const double* acc) {
#pragma unroll
                for (int c = 0; c < NRHS; ++c) {
                    const size_t q = (size_t)i * NRHS + c;
                    const V vv = (V)acc[c];
                    w.v[q] = vv;
                    red1[c] += (double)w.rh[q] * (double)vv;
                }
            });
        });
        if (!tm.template allreduce<NRHS>(red1, 1, smem)) return false;
        if (t0) {
            for (int c = 0; c < NRHS; ++c) {
                st.rs[c] = 0;
                if (st.done[c]) continue;
                if (gpu) {
                    st.alpha[c] = (fabs(red1[c]) > 1e-30) ? st.rho[c] / red1[c] : 0.0;
                } else {
                    if (red1[c] == 0.0) { st.done[c] = 1; st.status[c] = KCFD_BREAKDOWN; st.iters[c] = it + 1; continue; }
                    st.alpha[c] = st.rho[c] / red1[c];
                }
                if (!finite(st.alpha[c])) { st.done[c] = 1; st.status[c] = KCFD_BREAKDOWN; st.nonfinite[c] = 1; st.iters[c] = it + 1; }
            }
        }
        __syncthreads();
        // ---- s = r - alpha v (in place in r) ; shat = M^-1 s (Jacobi) ; ||s||^2 ----
        double red2[NRHS];
#pragma unroll
        for (int c = 0; c < NRHS; ++c) red2[c] = 0.0;
        for_my_rows(tm, a, [&](int s0, int s1) {
            for (int base = s0 + threadIdx.x; base < s1; base += kU * blockDim.x) {
                V rr[kU][NRHS], vv[kU][NRHS], dd[kU];
#pragma unroll
                for (int u = 0; u < kU; ++u) {
                    const int i = base + u * blockDim.x;
                    if (i >= s1) continue;
                    dd[u] = (PREC == KCFD_PREC_JACOBI) ? dinv[i] : (V)1;
#pragma unroll
                    for (int c = 0; c < NRHS; ++c) {
                        if (st.done[c]) continue;
                        const size_t q = (size_t)i * NRHS + c;
                        rr[u][c] = w.r[q];
                        vv[u][c] = w.v[q];
                    }
                }
#pragma unroll
                for (int u = 0; u < kU; ++u) {
                    const int i = base + u * blockDim.x;
                    if (i >= s1) continue;
#pragma unroll
                    for (int c = 0; c < NRHS; ++c) {
                        if (st.done[c]) continue;
                        const size_t q = (size_t)i * NRHS + c;
                        const V sv = (V)((double)rr[u][c] - st.alpha[c] * (double)vv[u][c]);
                        w.r[q] = sv;
                        if (PREC == KCFD_PREC_JACOBI) w.sh[q] = dd[u] * sv;
                        red2[c] += (double)sv * (double)sv;
                    }
                }
            }
        });
        if (!tm.template allreduce<NRHS>(red2, 2, smem)) return false;
        // per-rhs convergence on ||s||: x += alpha * phat, then stop
        int conv_mask = 0;
        if (t0) {
            int any_left = 0;
            for (int c = 0; c < NRHS; ++c) {
                if (st.done[c]) continue;
                const double sn = sqrt(red2[c]);
                if (!finite(sn)) { st.done[c] = 1; st.status[c] = KCFD_BREAKDOWN; st.nonfinite[c] = 1; st.iters[c] = it + 1; continue; }
                const bool conv = gpu ? (sn / st.bnorm[c] < st.thr[c]) : (sn < st.thr[c]);
                if (conv) {
                    st.done[c] = 2;  // converged here: the x update below still applies
                    st.status[c] = KCFD_OK;
                    st.iters[c] = it + 1;
                    st.rnorm[c] = sn;
                    continue;
                }
                any_left = 1;
            }
            st.any_left = any_left;
        }
        __syncthreads();
#pragma unroll
        for (int c = 0; c < NRHS; ++c)
            if (st.done[c] == 2) conv_mask |= 1 << c;
        if (conv_mask) {
            for_my_rows(tm, a, [&](int s0, int s1) {
                for (int i = s0 + threadIdx.x; i < s1; i += blockDim.x) {
#pragma unroll
                    for (int c = 0; c < NRHS; ++c) {
                        if (!(conv_mask & (1 << c))) continue;
                        const size_t q = (size_t)i * NRHS + c;
                        xv[q] = (V)((double)xv[q] + st.alpha[c] * (double)ph[q]);
                    }
                }
            });
            __syncthreads();
            if (t0)
                for (int c = 0; c < NRHS; ++c)
                    if (st.done[c] == 2) st.done[c] = 1;
            __syncthreads();
        }
        if (!st.any_left) return true;
        V* sh = (PREC == KCFD_PREC_NONE) ? w.r : w.sh;
        if (PREC == KCFD_PREC_ILU0) {
            if (!ilu_apply<V, NRHS>(tm, a, w.r, w.sh)) return false;
            if (!tm.sync()) return false;
        }
        // ---- t = A shat ; t.s, t.t ----
        double red3[2 * NRHS];
#pragma unroll
        for (int k = 0; k < 2 * NRHS; ++k) red3[k] = 0.0;
        for_my_rows(tm, a, [&](int s0, int s1) {
            spmv_range<VM, V, NRHS, kDiff>(ip, ix, vals, sh, s0, s1, a.lanes, [&](int i, const double* acc) {
#pragma unroll
                for (int c = 0; c < NRHS; ++c) {
                    const size_t q = (size_t)i * NRHS + c;
                    const V tt = (V)acc[c];
                    w.t[q] = tt;
                    red3[c] += (double)tt * (double)w.r[q];
                    red3[NRHS + c] += (double)tt * (double)tt;
                }
            });
        });
        if (!tm.template allreduce<2 * NRHS>(red3, 3, smem)) return false;
        if (t0) {
            for (int c = 0; c < NRHS; ++c) {
                if (st.done[c]) continue;
                if (gpu) st.omega[c] = (red3[NRHS + c] > 1e-30) ? red3[c] / red3[NRHS + c] : 0.0;
                else st.omega[c] = red3[c] / red3[NRHS + c];
                if (!finite(st.omega[c])) { st.done[c] = 1; st.status[c] = KCFD_BREAKDOWN; st.nonfinite[c] = 1; st.iters[c] = it + 1; }
            }
        }
        __syncthreads();
        // ---- x += alpha phat + omega shat ; r = s - omega t ; rhat.r, ||r||^2 ----
        double red4[2 * NRHS];
#pragma unroll
        for (int k = 0; k < 2 * NRHS; ++k) red4[k] = 0.0;
        for_my_rows(tm, a, [&](int s0, int s1) {
            for (int base = s0 + threadIdx.x; base < s1; base += kU * blockDim.x) {
                V xx[kU][NRHS], hp[kU][NRHS], hs[kU][NRHS], rr[kU][NRHS], tt[kU][NRHS], rh[kU][NRHS];
#pragma unroll
                for (int u = 0; u < kU; ++u) {
                    const int i = base + u * blockDim.x;
                    if (i >= s1) continue;
#pragma unroll
                    for (int c = 0; c < NRHS; ++c) {
                        if (st.done[c]) continue;
                        const size_t q = (size_t)i * NRHS + c;
                        xx[u][c] = xv[q];
                        hp[u][c] = ph[q];
                        hs[u][c] = sh[q];
                        rr[u][c] = w.r[q];
                        tt[u][c] = w.t[q];
                        rh[u][c] = w.rh[q];
                    }
                }
#pragma unroll
                for (int u = 0; u < kU; ++u) {
                    const int i = base + u * blockDim.x;
                    if (i >= s1) continue;
#pragma unroll
                    for (int c = 0; c < NRHS; ++c) {
                        if (st.done[c]) continue;
                        const size_t q = (size_t)i * NRHS + c;
                        const double al = st.alpha[c], om = st.omega[c];
                        if (gpu) xv[q] = (V)((double)xx[u][c] + (al * (double)hp[u][c] + om * (double)hs[u][c]));
                        else xv[q] = (V)(((double)xx[u][c] + al * (double)hp[u][c]) + om * (double)hs[u][c]);
                        const V rn = (V)((double)rr[u][c] - om * (double)tt[u][c]);
                        w.r[q] = rn;
                        red4[c] += (double)rh[u][c] * (double)rn;
                        red4[NRHS + c] += (double)rn * (double)rn;
                    }
                }
            }
        });
        if (!tm.template allreduce<2 * NRHS>(red4, 4, smem)) return false;
        if (t0) {
            for (int c = 0; c < NRHS; ++c) {
                if (st.done[c]) continue;
                st.rho_prev[c] = st.rho[c];
                st.rho[c] = red4[c];
                st.rnorm[c] = sqrt(red4[NRHS + c]);
                st.iters[c] = it + 1;
                if (!finite(st.rnorm[c]) || !finite(st.rho[c])) {
                    st.done[c] = 1; st.status[c] = KCFD_BREAKDOWN; st.nonfinite[c] = 1;
                    continue;
                }
                if (gpu && st.rnorm[c] / st.bnorm[c] < st.thr[c]) {
                    st.done[c] = 1;
                    st.status[c] = KCFD_OK;
                }
            }
        }
        __syncthreads();
    }
    if (t0) {
        for (int c = 0; c < NRHS; ++c)
            if (!st.done[c]) {
                st.status[c] = KCFD_MAXITER;
                st.iters[c] = maxiter;
            }
    }
    __syncthreads();
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

// Copy the caller's x, b into the level-permuted order (own rows), or back.
template <int NRHS, class Team>
__device__ void permute_in(Team& tm, const SolveArgs& a) {
    for_my_rows(tm, a, [&](int s0, int s1) {
        for (int i = s0 + threadIdx.x; i < s1; i += blockDim.x) {
            const int o = a.perm[i];
#pragma unroll
            for (int c = 0; c < NRHS; ++c) {
                a.px[(size_t)i * NRHS + c] = a.x[(size_t)o * NRHS + c];
                a.pb[(size_t)i * NRHS + c] = a.b[(size_t)o * NRHS + c];
            }
        }
    });
}

template <int NRHS, class Team>
__device__ void permute_out(Team& tm, const SolveArgs& a) {
    for_my_rows(tm, a, [&](int s0, int s1) {
        for (int i = s0 + threadIdx.x; i < s1; i += blockDim.x) {
            const int o = a.perm[i];
#pragma unroll
            for (int c = 0; c < NRHS; ++c) a.x[(size_t)o * NRHS + c] = a.px[(size_t)i * NRHS + c];
        }
    });
}

// Verification passes of a batched FP64 solve (see solve_fp64).
constexpr int kVerifyPasses = 3;

// FP64 solve.
template <int NRHS, int PREC, class Team>
__device__ void solve_fp64(Team& tm, const SolveArgs& a, double* smem) {
    __shared__ KState<NRHS> st;
    const Vecs<double> w(a.work, (size_t)a.n * NRHS);
    double* x = a.perm ? a.px : a.x;
    const double* b = a.perm ? a.pb : a.b;
    if (a.perm) {
        permute_in<NRHS>(tm, a);
        if (!tm.sync()) return;
    }
    // With breakdown restarts (the batched solver) a system that stopped on its recursive
    // residual is checked against the true one: the next pass starts from r = b - A x
    // and ends at once (no iteration) when that meets the tolerance, else it iterates on
    // from the true residual. Iterations of all passes count against maxiter.
    const bool verify = NRHS == 1 && a.max_restarts > 0 && a.stop == KCFD_STOP_SCIPY;
    int used = 0;
    for (int pass = 0;; ++pass) {
        const bool ok = bicgstab_body<double, double, NRHS, PREC>(tm, a, a.vals64, x, b, false, w, a.stop, a.rtol,
                                                                  a.atol, a.maxiter - used, st, smem);
        if (!ok) return;
        used += st.iters[0];
        if (!verify || pass >= kVerifyPasses || st.status[0] != KCFD_OK || st.iters[0] == 0 || used >= a.maxiter) break;
        // every member's last x update is in place before any member gathers x again
        if (!tm.sync()) return;
    }
    __syncthreads();
    if (verify && threadIdx.x == 0) st.iters[0] = used;
    __syncthreads();
    if (a.perm) permute_out<NRHS>(tm, a);
    write_results<NRHS>(a, st, tm.rank);
}

// Outer (FP64) state of a MIXED solve, in shared memory like KState.
template <int NRHS>
struct MState {
    double thr[NRHS], rn[NRHS], bn[NRHS], rn_prev[NRHS];
    int done[NRHS], applied[NRHS], revert[NRHS], capped[NRHS];
    int left, stop_now, total_it, cap, grow, retry;
    double inner_atol;
};

// A refinement step that does not lower the FP64 residual is undone. If its inner run
// stopped at the iteration cap (not at the inner tolerance), it is retried from the
// same iterate with twice the cap, up to this many doublings; an inner run that met
// its tolerance and still did not help means FP32 cannot resolve the system, and the
// right-hand side stops with BREAKDOWN.
constexpr int kMaxGrow = 5;

// MIXED solve: FP64 outer refinement around capped FP32 inner BiCGSTAB runs.
template <int NRHS, int PREC, class Team>
__device__ void solve_mixed(Team& tm, const SolveArgs& a, double* smem) {
    __shared__ KState<NRHS> out;
    __shared__ KState<NRHS> st;
    __shared__ MState<NRHS> ms;
    const int n = a.n;
    const Vecs<float> w(a.work, (size_t)n * NRHS);
    double* x = a.perm ? a.px : a.x;
    const double* b = a.perm ? a.pb : a.b;
    const bool t0 = threadIdx.x == 0;
    if (a.perm) {
        permute_in<NRHS>(tm, a);
        if (!tm.sync()) return;
    }
    if (t0) {
        for (int c = 0; c < NRHS; ++c) {
            ms.applied[c] = 0;
            ms.capped[c] = 0;
            ms.done[c] = 0;
            ms.rn_prev[c] = INFINITY;
            ms.thr[c] = 0.0;
            ms.rn[c] = 0.0;
            out.status[c] = KCFD_OK;
            out.iters[c] = 0;
        }
        ms.total_it = 0;
        ms.grow = 0;
    }
    __syncthreads();
    for (int ref = 0;; ++ref) {
        // r64 = b - A64 x ; ||b||, ||r||
        double red[2 * NRHS];
#pragma unroll
        for (int k = 0; k < 2 * NRHS; ++k) red[k] = 0.0;
        for_my_rows(tm, a, [&](int s0, int s1) {
            spmv_range<double, double, NRHS>(a.indptr, a.indices, a.vals64, x, s0, s1, a.lanes,
                                             [&](int i, const double* acc) {
#pragma unroll
                                                 for (int c = 0; c < NRHS; ++c) {
                                                     const size_t q = (size_t)i * NRHS + c;
                                                     const double bb = b[q];
                                                     const double rr = bb - acc[c];
                                                     a.r64[q] = rr;
                                                     red[c] += bb * bb;
                                                     red[NRHS + c] += rr * rr;
                                                 }
                                             });
        });
        if (!tm.template allreduce<2 * NRHS>(red, 5, smem)) return;
        if (t0) {
            int left = 0;
            ms.retry = 0;
            for (int c = 0; c < NRHS; ++c) {
                ms.revert[c] = 0;
                ms.bn[c] = sqrt(red[c]);
                const double r_new = sqrt(red[NRHS + c]);
                if (ref == 0) ms.thr[c] = fmax(a.atol, a.rtol * ms.bn[c]);
                out.bnorm[c] = ms.bn[c];
                if (ms.done[c]) continue;
                if (ms.applied[c] && !(r_new < ms.rn_prev[c])) {
                    // the last refinement step did not lower the FP64 residual: undo it,
                    // then retry with a larger inner cap, or give up
                    ms.revert[c] = 1;
                    ms.rn[c] = ms.rn_prev[c];
                    if (ms.capped[c] && ms.grow < kMaxGrow && ms.total_it < a.maxiter) {
                        ms.retry = 1;
                    } else {
                        ms.done[c] = 1;
                        out.status[c] = KCFD_BREAKDOWN;
                    }
                } else if (!finite(r_new)) {
                    ms.done[c] = 1;
                    out.status[c] = KCFD_BREAKDOWN;
                    ms.rn[c] = r_new;
                } else {
                    ms.rn[c] = r_new;
                    if (r_new < ms.thr[c] || ms.bn[c] == 0.0) {
                        ms.done[c] = 1;
                        out.status[c] = KCFD_OK;
                    }
                }
                ms.applied[c] = 0;
                out.rnorm[c] = ms.rn[c];
                left |= !ms.done[c];
            }
            ms.left = left;
            ms.stop_now = 0;
            if (left && (ref >= a.max_refine || ms.total_it >= a.maxiter)) {
                for (int c = 0; c < NRHS; ++c)
                    if (!ms.done[c]) out.status[c] = KCFD_MAXITER;
                ms.stop_now = 1;
            }
            double ia = INFINITY;
            for (int c = 0; c < NRHS; ++c)
                if (!ms.done[c]) ia = fmin(ia, ms.thr[c] * 0.5);
            ms.inner_atol = ia;
            if (ms.retry) ms.grow += 1;
            ms.cap = (int)min((long long)a.inner_maxiter << ms.grow, (long long)(a.maxiter - ms.total_it));
        }
        __syncthreads();
        // own rows: undo rejected steps, load the inner rhs, zero the inner solution
        for_my_rows(tm, a, [&](int s0, int s1) {
            for (int i = s0 + threadIdx.x; i < s1; i += blockDim.x) {
#pragma unroll
                for (int c = 0; c < NRHS; ++c) {
                    const size_t q = (size_t)i * NRHS + c;
                    if (ms.revert[c]) x[q] = x[q] - (double)w.xi[q];
                    w.bi[q] = ms.done[c] ? 0.0f : (float)a.r64[q];
                    w.xi[q] = 0.0f;
                }
            }
        });
        if (!ms.left || ms.stop_now) break;
        if (ms.retry) {
            // the residual of the restored iterate is recomputed at the top
            if (!tm.sync()) return;
            continue;
        }
        // inner FP32 solve A32 e = r from e = 0 to max(inner_rtol ||r||, thr/2)
        bool ok = bicgstab_body<float, float, NRHS, PREC>(tm, a, a.vals32, w.xi, w.bi, true, w, KCFD_STOP_SCIPY,
                                                          a.inner_rtol, ms.inner_atol, ms.cap, st, smem);
        if (!ok) return;
        if (t0) {
            int max_it = 0;
            for (int c = 0; c < NRHS; ++c) {
                if (ms.done[c]) continue;
                out.iters[c] += st.iters[c];
                max_it = max(max_it, st.iters[c]);
                if (st.nonfinite[c] || st.iters[c] == 0) {
                    ms.done[c] = 1;
                    out.status[c] = KCFD_BREAKDOWN;
                } else {
                    ms.applied[c] = 1;
                    ms.rn_prev[c] = ms.rn[c];
                    ms.capped[c] = st.status[c] == KCFD_MAXITER;
                }
            }
            ms.total_it += max(max_it, 1);
        }
        __syncthreads();
        for_my_rows(tm, a, [&](int s0, int s1) {
            for (int i = s0 + threadIdx.x; i < s1; i += blockDim.x) {
#pragma unroll
                for (int c = 0; c < NRHS; ++c) {
                    if (!ms.applied[c]) continue;
                    const size_t q = (size_t)i * NRHS + c;
                    x[q] = x[q] + (double)w.xi[q];
                }
            }
        });
        if (!tm.sync()) return;
    }
    if (a.perm) permute_out<NRHS>(tm, a);
    write_results<NRHS>(a, out, tm.rank);
}

// 512 threads with up to 128 registers: the fused phases keep four rows per thread
// in flight without spilling (1024-thread CTAs would cap registers at 64).
constexpr int grid_block(int) { return 512; }

template <int MIXED, int NRHS, int PREC>
__global__ void __launch_bounds__(grid_block(NRHS), 1) solve_grid_kernel(SolveArgs a) {
    __shared__ double smem[32 * kMaxK];
    GridTeam tm(a.ctl);
    if (MIXED) solve_mixed<NRHS, PREC>(tm, a, smem);
    else solve_fp64<NRHS, PREC>(tm, a, smem);
}

// One CTA per solve. MAXB is the largest block it is launched with: 1024 threads cap
// a thread at 64 registers (the FP64 phases then spill to local memory); the
// 512-thread instance has 128.
template <int MIXED, int NRHS, int PREC, int MAXB = 1024>
__global__ void __launch_bounds__(MAXB, 1) solve_cta_kernel(SolveArgs a) {
    __shared__ double smem[32 * kMaxK];
    CtaTeam tm;
    if (MIXED) solve_mixed<NRHS, PREC>(tm, a, smem);
    else solve_fp64<NRHS, PREC>(tm, a, smem);
}

// z = M^-1 r with the handle's ILU factors (one right-hand side, FP64): r into the
// level-permuted order, the two sweeps, and back.
template <class Team>
__device__ void ilu_precond_apply(Team& tm, const SolveArgs& a) {
    for_my_rows(tm, a, [&](int s0, int s1) {
        for (int i = s0 + threadIdx.x; i < s1; i += blockDim.x) a.pb[i] = a.b[a.perm[i]];
    });
    if (!tm.sync()) return;
    if (!ilu_apply<double, 1>(tm, a, a.pb, a.px)) return;
    if (!tm.sync()) return;
    for_my_rows(tm, a, [&](int s0, int s1) {
        for (int i = s0 + threadIdx.x; i < s1; i += blockDim.x) a.x[a.perm[i]] = a.px[i];
    });
}

__global__ void __launch_bounds__(512, 1) ilu_apply_grid_kernel(SolveArgs a) {
    GridTeam tm(a.ctl);
    ilu_precond_apply(tm, a);
}

__global__ void __launch_bounds__(1024, 1) ilu_apply_cta_kernel(SolveArgs a) {
    CtaTeam tm;
    ilu_precond_apply(tm, a);
}

__global__ void jacobi_apply_kernel(int n, const double* __restrict__ dinv, const double* r, double* z) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) z[i] = dinv[i] * r[i];
}

// ------------------------------------------------------------- batched systems --
// Many independent systems of uneven size in ONE persistent launch: each CTA takes
// the next system from a queue (largest first), builds its Jacobi inverse diagonal and
// FP32 difference-form operator row by row, and solves it alone (CtaTeam: block
// barriers and block reductions only, no inter-CTA waits). A system's result does not
// depend on which CTA ran it or on what ran beside it.
struct BatchSys {
    int n, nnz;
    long long row_off;  // rows before this system in the packed vectors
    long long ptr_off;  // offset of its (n + 1) row pointers
    long long nnz_off;  // offset of its entries
};

struct BatchArgs {
    int nsys, lanes, mixed, precond, stop, maxiter, max_refine, inner_maxiter, max_restarts;
    int nq;  // systems in this launch's queue (order[0..nq))
    double rtol, atol, inner_rtol;
    const BatchSys* sys;
    const int* order;
    int* queue;
    const int* indptr;
    const int* indices;
    const double* vals64;
    float* vals32;
    void* dinv;
    int* lev;
    void* work;
    double* r64;
    double* x;
    const double* b;
    int* iters;
    double* relres;
    int* status;
};

template <typename V>
__device__ void batch_prep(const BatchArgs& B, const BatchSys& S, int sid, V* dinv, float* v32, bool mixed) {
    const int* ip = B.indptr + S.ptr_off;
    const int* ix = B.indices + S.nnz_off;
    const double* v = B.vals64 + S.nnz_off;
    for (int i = threadIdx.x; i < S.n; i += blockDim.x) {
        double d = 0.0, sum = 0.0;
        int dk = -1;
        for (int k = ip[i]; k < ip[i + 1]; ++k) {
            sum += v[k];
            if (ix[k] == i) {
                d += v[k];
                dk = k;
            } else if (mixed) {
                v32[k] = (float)v[k];
            }
        }
        if (mixed && dk >= 0) v32[dk] = (float)sum;
        if (B.precond == KCFD_PREC_JACOBI) dinv[i] = (V)((fabs(d) > 1e-30) ? 1.0 / d : 0.0);
    }
    if (threadIdx.x == 0) {
        B.lev[2 * sid] = 0;
        B.lev[2 * sid + 1] = S.n;
    }
}

// Per-system set-up in its own launch (the solve launch reads these arrays through
// the read-only path): Jacobi inverse diagonal, FP32 difference-form operator.
template <int MIXED>
__global__ void batch_prep_kernel(BatchArgs B) {
    using V = typename std::conditional<MIXED, float, double>::type;
    for (int sid = blockIdx.x; sid < B.nsys; sid += gridDim.x) {
        const BatchSys S = B.sys[sid];
        batch_prep<V>(B, S, sid, (V*)B.dinv + S.row_off, B.vals32 ? B.vals32 + S.nnz_off : nullptr, MIXED);
    }
}

// SolveArgs of system sid of a batch (everything but the team control).
template <typename V>
__device__ SolveArgs batch_args(const BatchArgs& B, int sid) {
    const BatchSys S = B.sys[sid];
    SolveArgs a;
    memset(&a, 0, sizeof(a));
    a.n = S.n;
    a.lanes = B.lanes;
    a.indptr = B.indptr + S.ptr_off;
    a.indices = B.indices + S.nnz_off;
    a.vals64 = B.vals64 + S.nnz_off;
    a.vals32 = B.vals32 ? B.vals32 + S.nnz_off : nullptr;
    a.dinv = (V*)B.dinv + S.row_off;
    a.lev_ptr = B.lev + 2 * sid;
    a.nlev = 1;
    a.work = (V*)B.work + 9 * S.row_off;
    a.x = B.x + S.row_off;
    a.b = B.b + S.row_off;
    a.r64 = B.r64 ? B.r64 + S.row_off : nullptr;
    a.stop = B.stop;
    a.maxiter = B.maxiter;
    a.max_refine = B.max_refine;
    a.inner_maxiter = B.inner_maxiter;
    a.max_restarts = B.max_restarts;
    a.rtol = B.rtol;
    a.atol = B.atol;
    a.inner_rtol = B.inner_rtol;
    a.iters_out = B.iters + sid;
    a.relres_out = B.relres + sid;
    a.status_out = B.status + sid;
    return a;
}

// Team control of the cluster tier: per cluster a barrier counter, a published queue
// entry and the reduction partials; one error flag for the launch.
struct ClusterCtl {
    unsigned int* bar;  // [clusters], zeroed before each launch
    int* slot;          // [clusters]
    double* partials;   // [clusters][kSlots * kMaxK * cluster size]
    int* err;
    long long budget;
};

// Cluster tier: the largest systems, each solved by the CTAs of one thread-block
// cluster (512 threads per CTA, one CTA per SM) as a team that splits the rows and
// meets at bounded software barriers (GridTeam over the cluster's CTAs, which the
// hardware schedules together). Rank 0 takes the next system from the queue and
// publishes it; a system's result depends only on the system and the cluster size.
template <int MIXED, int PREC>
__global__ void __launch_bounds__(512, 1) batch_cluster_kernel(BatchArgs B, ClusterCtl C) {
    __shared__ double smem[32 * kMaxK];
    using V = typename std::conditional<MIXED, float, double>::type;
    int crank, csize, cid;
    cluster_ids(crank, csize, cid);
    TeamCtl ctl;
    ctl.bar = C.bar + cid;
    ctl.partials = C.partials + (size_t)cid * kSlots * kMaxK * csize;
    ctl.err = C.err;
    ctl.budget = C.budget;
    GridTeam tm(ctl, crank, csize);
    for (;;) {
        if (crank == 0 && threadIdx.x == 0) C.slot[cid] = atomicAdd(B.queue, 1);
        if (!tm.sync()) break;
        const int q = __ldcg(C.slot + cid);
        // every member has read the entry before rank 0 can overwrite it
        if (!tm.sync()) break;
        if (q >= B.nq) break;
        const int sid = B.order[q];
        SolveArgs a = batch_args<V>(B, sid);
        a.ctl = ctl;
        if (MIXED) solve_mixed<1, PREC>(tm, a, smem);
        else solve_fp64<1, PREC>(tm, a, smem);
        if (*(volatile int*)C.err != 0) {
            // a barrier wait expired: the system has no result
            if (crank == 0 && threadIdx.x == 0) B.status[sid] = 5 /*KCFD_TIMEOUT*/;
            break;
        }
    }
}

template <int MIXED, int PREC, int BLOCK>
__global__ void __launch_bounds__(BLOCK, BLOCK == 256 ? 2 : 1) batch_kernel(BatchArgs B) {
    __shared__ double smem[32 * kMaxK];
    __shared__ int s_q;
    using V = typename std::conditional<MIXED, float, double>::type;
    CtaTeam tm;
    for (;;) {
        if (threadIdx.x == 0) s_q = atomicAdd(B.queue, 1);
        __syncthreads();
        const int q = s_q;
        __syncthreads();
        if (q >= B.nq) break;
        const int sid = B.order[q];
        SolveArgs a = batch_args<V>(B, sid);
        if (MIXED) solve_mixed<1, PREC>(tm, a, smem);
        else solve_fp64<1, PREC>(tm, a, smem);
        __syncthreads();
    }
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

// Gather the caller's values into the level-permuted CSR (FP64 and, if asked, FP32).
__global__ void permute_vals_kernel(int64_t nnz, const int* __restrict__ src, const double* __restrict__ v,
                                    double* __restrict__ p64, float* __restrict__ p32) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nnz; k += (int64_t)gridDim.x * blockDim.x) {
        const int j = src[k];
        const double x = j >= 0 ? v[j] : 0.0;  // ILU(k) fill slots hold zeros
        p64[k] = x;
        if (p32) p32[k] = (float)x;
    }
}

// FP32 operator of the MIXED inner iterations: off-diagonals rounded to FP32, the
// diagonal slot replaced by the FP64 row sum rounded once (difference form, see
// spmv_range).
__global__ void rowsum_f32_kernel(int n, const int* __restrict__ ip, const int* __restrict__ ix,
                                  const double* __restrict__ v64, float* __restrict__ v32) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double sum = 0.0;
        int dk = -1;
        for (int k = ip[i]; k < ip[i + 1]; ++k) {
            sum += v64[k];
            if (ix[k] == i) dk = k;
            else v32[k] = (float)v64[k];
        }
        if (dk >= 0) v32[dk] = (float)sum;
    }
}

constexpr int kMaxIluRow = 64;

// Structural ILU(0), IKJ order, on the level-permuted CSR: row i's lower entries
// are its columns < i (all on earlier levels), processed left to right.
template <typename V, class Team>
__device__ void ilu0_factor_body(Team& tm, const SolveArgs& a) {
    V* lu = (V*)a.lu;
    V* ldi = (V*)a.ludinv;
    const double* vals = a.vals64;
    for (int l = 0; l < a.nlev; ++l) {
        if (l > 0 && !tm.sync()) return;
        int s0, s1;
        level_slice(tm, a, l, s0, s1);
        for (int i = s0 + threadIdx.x; i < s1; i += blockDim.x) {
            const int lo = a.indptr[i], hi = a.indptr[i + 1], dp = a.diag[i];
            double wv[kMaxIluRow];
            for (int q = lo; q < hi; ++q) wv[q - lo] = vals[q];
            for (int kk = lo; kk < dp; ++kk) {
                const int kr = a.indices[kk];
                const double l_ik = wv[kk - lo] * (double)ldi[kr];
                wv[kk - lo] = l_ik;
                const int ke = a.indptr[kr + 1];
                for (int jj = a.diag[kr] + 1; jj < ke; ++jj) {
                    const int j = a.indices[jj];
                    for (int q = kk + 1; q < hi; ++q)
                        if (a.indices[q] == j) {
                            wv[q - lo] -= l_ik * (double)lu[jj];
                            break;
                        }
                }
            }
            for (int q = lo; q < hi; ++q) lu[q] = (V)wv[q - lo];
            const double u = wv[dp - lo];
            ldi[i] = (V)((fabs(u) > 1e-300) ? 1.0 / u : 0.0);
        }
    }
}

template <typename V>
__global__ void __launch_bounds__(1024, 1) ilu0_factor_grid(SolveArgs a) {
    GridTeam tm(a.ctl);
    ilu0_factor_body<V>(tm, a);
}

template <typename V>
__global__ void __launch_bounds__(1024) ilu0_factor_cta(SolveArgs a) {
    CtaTeam tm;
    ilu0_factor_body<V>(tm, a);
}

}  // namespace kcfd

// =================================================================== host side ==
using namespace kcfd;

struct kcfd_solver {
    kcfd_solver_opts_t o;
    int n = 0, nnz = 0;
    int pnnz = 0;  // entries of the permuted matrix (ILU(k): A's plus the fill)
    int grid = 0, block = 256, team = 1, lanes = 8;
    int sm_count = 0;
    void* work = nullptr;
    double* r64 = nullptr;
    void* dinv = nullptr;
    float* v32own = nullptr;  // MIXED, no permutation: FP32 difference-form operator
    int* lev_ptr = nullptr;
    int nlev = 1;
    // ILU: level-permuted CSR owned by the handle
    int* perm = nullptr;
    int* p_indptr = nullptr;
    int* p_indices = nullptr;
    int* p_src = nullptr;
    int* p_diag = nullptr;
    double* p_vals64 = nullptr;
    float* p_vals32 = nullptr;
    double* px = nullptr;
    double* pb = nullptr;
    void* lu = nullptr;
    void* ludinv = nullptr;
    // KCFD_PREC_AMG: the multigrid hierarchy (graph engine only)
    kcfd_amg* amg = nullptr;
    // team control
    unsigned int* bar = nullptr;
    double* partials = nullptr;
    int* err = nullptr;
    // graph engine (team 3)
    struct {
        ge::St* st = nullptr;
        double* part = nullptr;
        unsigned* cnt = nullptr;
        double *gx = nullptr, *gb = nullptr, *vec = nullptr;  // gx/gb: the handle's px/pb with ILU
        int* res_i = nullptr;      // [2*3] iters, status
        double* res_d = nullptr;   // [3] relres
        cudaGraph_t graph = nullptr;
        cudaGraphExec_t exec = nullptr;
        const double* vals_key = nullptr;  // caller values the graph was built for (non-permuted)
        int gmax = 0;
        int eager = 0;                     // host-driven loop instead of the graph
        bool pdl = true;                   // phase kernels with programmatic dependent launch
        bool ready = false;                // args (and graph) built
        int mix = 0;                       // MIXED: FP32 vectors and values, FP64 x, b and residuals
        ge::Args args;
        ge::ArgsT<float> args32;           // MIXED
        ge::Sell A, L, U;                  // sliced-ELL copies (L, U: ILU only)
        ge::SellT<float> A32{}, L32{}, U32{};  // MIXED: FP32 values on the same slots
        float* vec32 = nullptr;            // MIXED: the 7 Krylov vectors
        int* srcA = nullptr;               // per slot: index into the caller's values, -1 padding
        int* srcL = nullptr;               // per slot: index into the permuted CSR (lu), -1 padding
        int* srcU = nullptr;
        int64_t slotsA = 0, slotsL = 0, slotsU = 0;
    } g;
};

namespace {

template <int MIXED, int NRHS, int PREC>
void* pick_kernel(bool grid, int block) {
    if (grid) return (void*)solve_grid_kernel<MIXED, NRHS, PREC>;
    return block <= 512 ? (void*)solve_cta_kernel<MIXED, NRHS, PREC, 512> : (void*)solve_cta_kernel<MIXED, NRHS, PREC, 1024>;
}

void* solve_kernel_ptr(int mixed, int nrhs, int prec, bool grid, int block) {
#define KC_CASE(M, R, P) \
    if (mixed == M && nrhs == R && prec == P) return pick_kernel<M, R, P>(grid, block);
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
    if (s->amg) kcfd_amg_destroy(s->amg);
    if (s->g.exec) cudaGraphExecDestroy(s->g.exec);
    if (s->g.graph) cudaGraphDestroy(s->g.graph);
    {
        // with ILU the engine's x/b are the handle's permuted vectors (freed below)
        void* gx = (s->g.gx == s->px) ? nullptr : s->g.gx;
        void* gb = (s->g.gb == s->pb) ? nullptr : s->g.gb;
        void* gp[] = {s->g.st, s->g.part, s->g.cnt, gx, gb, s->g.vec, s->g.res_i, s->g.res_d,
                      (void*)s->g.A.off, (void*)s->g.A.col, (void*)s->g.A.val, (void*)s->g.L.off, (void*)s->g.L.col,
                      (void*)s->g.L.val, (void*)s->g.U.off, (void*)s->g.U.col, (void*)s->g.U.val,
                      s->g.srcA, s->g.srcL, s->g.srcU, (void*)s->g.A32.val, (void*)s->g.L32.val,
                      (void*)s->g.U32.val, (void*)s->g.vec32};
        for (void* p : gp)
            if (p) cudaFree(p);
    }
    void* ps[] = {s->work, s->r64, s->dinv, s->v32own, s->lev_ptr, s->perm, s->p_indptr, s->p_indices, s->p_src, s->p_diag,
                  s->p_vals64, s->p_vals32, s->px, s->pb, s->lu, s->ludinv, s->bar, s->partials, s->err};
    for (void* p : ps)
        if (p) cudaFree(p);
    delete s;
    return KCFD_OK;
}

// Greedy distance-d colouring of A's symmetrised graph, rows in index order: each row
// takes the smallest colour not used by any row within d edges of it. With d = k + 1
// no ILU(k) fill entry joins two rows of one colour (a level-l fill entry (i, j)
// closes a path of l + 1 edges from i to j through earlier rows).
std::vector<int> distance_colouring(int n, const std::vector<int>& ip, const std::vector<int>& ix, int d) {
    std::vector<int> deg(n + 1, 0);
    for (int i = 0; i < n; ++i)
        for (int k = ip[i]; k < ip[i + 1]; ++k)
            if (ix[k] != i) {
                deg[i + 1]++;
                deg[ix[k] + 1]++;
            }
    for (int i = 0; i < n; ++i) deg[i + 1] += deg[i];
    std::vector<int> adj(deg[n]), fill(deg.begin(), deg.end() - 1);
    for (int i = 0; i < n; ++i)
        for (int k = ip[i]; k < ip[i + 1]; ++k)
            if (ix[k] != i) {
                adj[fill[i]++] = ix[k];
                adj[fill[ix[k]]++] = i;
            }
    std::vector<int> colour(n, -1), seen(n, -1), used;
    std::vector<int> front, next;
    for (int v = 0; v < n; ++v) {
        seen[v] = v;
        front.assign(1, v);
        std::vector<int> near;
        for (int depth = 0; depth < d && !front.empty(); ++depth) {
            next.clear();
            for (int u : front)
                for (int e = deg[u]; e < deg[u + 1]; ++e) {
                    const int w = adj[e];
                    if (seen[w] == v) continue;
                    seen[w] = v;
                    next.push_back(w);
                    if (colour[w] >= 0) near.push_back(colour[w]);
                }
            front.swap(next);
        }
        int c = 0;
        std::sort(near.begin(), near.end());
        for (int x : near) {
            if (x == c) ++c;
            else if (x > c) break;
        }
        colour[v] = c;
    }
    return colour;
}

SolveArgs make_args(const kcfd_solver* s, const kcfd_csr_t* A) {
    SolveArgs a;
    std::memset(&a, 0, sizeof(a));
    a.n = s->n;
    a.lanes = s->lanes;
    if (s->perm) {
        a.indptr = s->p_indptr;
        a.indices = s->p_indices;
        a.vals64 = s->p_vals64;
        a.vals32 = s->p_vals32;
        a.perm = s->perm;
        a.px = s->px;
        a.pb = s->pb;
    } else {
        a.indptr = A->indptr;
        a.indices = A->indices;
        a.vals64 = A->vals64;
        a.vals32 = s->v32own;
    }
    a.dinv = s->dinv;
    a.diag = s->p_diag;
    a.lu = s->lu;
    a.ludinv = s->ludinv;
    a.lev_ptr = s->lev_ptr;
    a.nlev = s->nlev;
    a.work = s->work;
    a.r64 = s->r64;
    a.stop = s->o.stop;
    a.maxiter = s->o.maxiter;
    a.max_refine = s->o.max_refine;
    a.inner_maxiter = s->o.inner_maxiter;
    a.rtol = s->o.rtol;
    a.atol = s->o.atol;
    a.inner_rtol = s->o.inner_rtol;
    a.ctl.bar = s->bar;
    a.ctl.partials = s->partials;
    a.ctl.err = s->err;
    a.ctl.budget = 4000000000LL;  // ~2 s at 2 GHz per barrier wait
    return a;
}

int launch_team(const kcfd_solver* s, void* kernel, void** args, cudaStream_t st) {
    KCFD_CUDA(cudaMemsetAsync(s->bar, 0, 2 * sizeof(unsigned), st));
    KCFD_CUDA(cudaMemsetAsync(s->err, 0, sizeof(int), st));
    if (s->team >= 2) {
        KCFD_CUDA(cudaLaunchCooperativeKernel(kernel, dim3(s->grid), dim3(s->block), args, 0, st));
    } else {
        KCFD_CUDA(cudaLaunchKernel(kernel, dim3(1), dim3(s->block), args, 0, st));
    }
    KCFD_CUDA(cudaGetLastError());
    return KCFD_OK;
}

template <typename T>
bool upload(T** dst, const std::vector<T>& v) {
    if (cudaMalloc(dst, std::max<size_t>(v.size(), 1) * sizeof(T)) != cudaSuccess) return false;
    return v.empty() || cudaMemcpy(*dst, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice) == cudaSuccess;
}

// ------------------------------------------------------------ graph engine host --
int ge_fill_grid(const kcfd_solver* s, int64_t m) {
    return (int)std::max<int64_t>(1, std::min<int64_t>((m + 255) / 256, (int64_t)s->sm_count * 16));
}

// Grid of each phase kernel: its own occupancy on every SM, capped by the rows it has
// (a vector kernel takes Ilp::U rows per thread and step) and by the partial slots.
struct GeGrid {
    int init, p, fwd, bwd, sv, s, st, xr, rr;
};

template <int NRHS, int PREC, typename T>
GeGrid ge_grids(int n, int sms, int gmax) {
    auto g = [&](const void* f, int rows_per_thread) {
        int occ = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, f, ge::kBlock, 0) != cudaSuccess || occ < 1) occ = 1;
        const int64_t per = (int64_t)ge::kBlock * rows_per_thread;
        const int64_t need = ((int64_t)n + per - 1) / per;
        return (int)std::max<int64_t>(1, std::min<int64_t>({(int64_t)occ * sms, need, (int64_t)gmax}));
    };
    constexpr int U = ge::Ilp<NRHS>::U;
    GeGrid r;
    r.init = g((const void*)ge::g_init<NRHS, T>, 1);
    r.p = g((const void*)ge::g_p<NRHS, PREC, T>, U);
    r.fwd = g((const void*)ge::g_fwd<NRHS, T>, 1);
    r.bwd = g((const void*)ge::g_bwd<NRHS, T>, 1);
    r.sv = g((const void*)ge::g_spmv_v<NRHS, PREC, T>, 1);
    r.s = g((const void*)ge::g_s<NRHS, PREC, T>, U);
    r.st = g((const void*)ge::g_spmv_t<NRHS, PREC, T>, 1);
    r.xr = g((const void*)ge::g_xr<NRHS, PREC, T>, NRHS == 1 ? 2 : U);  // g_xr's rows per thread
    r.rr = ge::is_mixed<T>() ? g((const void*)ge::g_rr<NRHS, PREC, T>, 1) : 0;
    return r;
}

// Launch of one phase kernel, with programmatic dependent launch when pdl is set.
template <typename... KArgs, typename... Act>
void ge_launch(void (*k)(KArgs...), int grid, cudaStream_t cs, bool pdl, Act&&... args) {
    cudaLaunchConfig_t cfg;
    std::memset(&cfg, 0, sizeof(cfg));
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(ge::kBlock);
    cfg.stream = cs;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = pdl ? at : nullptr;
    cfg.numAttrs = pdl ? 1 : 0;
    cudaLaunchKernelEx(&cfg, k, std::forward<Act>(args)...);
}

// One loop trip: the phase kernels of one BiCGSTAB iteration.
template <int NRHS, int PREC, typename T>
void ge_body(const ge::ArgsT<T>& a, const GeGrid& G, cudaStream_t cs, bool pdl) {
    ge_launch(ge::g_p<NRHS, PREC, T>, G.p, cs, pdl, a);
    auto sweeps = [&](int which) {
        if constexpr (PREC == KCFD_PREC_AMG && !ge::is_mixed<T>()) {
            // phat = M^-1 p, shat = M^-1 s: one V-cycle each, skipped once the loop flag drops
            amg::vcycle((const kcfd_amg*)a.amg, which ? a.r : a.p, which ? a.sh : a.ph, &a.st->active, cs, pdl);
            return;
        }
        if (PREC != KCFD_PREC_ILU0) return;
        if (a.nlev == 1) {
            ge_launch(ge::g_bwd<NRHS, T>, G.bwd, cs, pdl, a, 0, which);
            return;
        }
        for (int l = 1; l < a.nlev; ++l) ge_launch(ge::g_fwd<NRHS, T>, G.fwd, cs, pdl, a, l, which);
        for (int l = a.nlev - 2; l >= 0; --l) ge_launch(ge::g_bwd<NRHS, T>, G.bwd, cs, pdl, a, l, which);
    };
    sweeps(0);
    ge_launch(ge::g_spmv_v<NRHS, PREC, T>, G.sv, cs, pdl, a);
    ge_launch(ge::g_s<NRHS, PREC, T>, G.s, cs, pdl, a);
    sweeps(1);
    ge_launch(ge::g_spmv_t<NRHS, PREC, T>, G.st, cs, pdl, a);
    ge_launch(ge::g_xr<NRHS, PREC, T>, G.xr, cs, pdl, a);
    if constexpr (ge::is_mixed<T>()) ge_launch(ge::g_rr<NRHS, PREC, T>, G.rr, cs, pdl, a);
}

// The engine's arguments of this storage type.
template <typename T>
ge::ArgsT<T>& ge_args(kcfd_solver* s);
template <>
ge::ArgsT<double>& ge_args<double>(kcfd_solver* s) { return s->g.args; }
template <>
ge::ArgsT<float>& ge_args<float>(kcfd_solver* s) { return s->g.args32; }

// Value fills at the head of every solve: the caller's FP64 values into the SELL
// copy of A, and (MIXED) its FP32 difference form.
template <typename T>
void ge_fill_values(kcfd_solver* s, const double* vals, cudaStream_t st) {
    ge::g_fill<double, double><<<ge_fill_grid(s, s->g.slotsA), 256, 0, st>>>(s->g.slotsA, s->g.srcA, vals, s->g.A.val);
    if constexpr (ge::is_mixed<T>())
        ge::g_diff32<<<ge_fill_grid(s, s->n), 256, 0, st>>>(s->n, s->g.A, s->g.A32.val);
}

// CG (one right-hand side, FP64): grids of its phase kernels, and one loop trip.
struct CgGrid {
    int init, rz, p, q, xr;
};

template <int PREC>
CgGrid cg_grids(int n, int sms, int gmax) {
    auto g = [&](const void* f, int rows_per_thread) {
        int occ = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, f, ge::kBlock, 0) != cudaSuccess || occ < 1) occ = 1;
        const int64_t per = (int64_t)ge::kBlock * rows_per_thread;
        const int64_t need = ((int64_t)n + per - 1) / per;
        return (int)std::max<int64_t>(1, std::min<int64_t>({(int64_t)occ * sms, need, (int64_t)gmax}));
    };
    CgGrid r;
    r.init = g((const void*)ge::g_cg_init, 1);
    r.rz = g((const void*)ge::g_cg_rz<PREC>, 4);
    r.p = g((const void*)ge::g_cg_p<PREC>, 4);
    r.q = g((const void*)ge::g_cg_q, 1);
    r.xr = g((const void*)ge::g_cg_xr, 2);
    return r;
}

// z = M^-1 r (ILU sweeps from r into shat, or one V-cycle), rho and beta, p, q = A p
// and alpha, then x, r and the tests. Jacobi's z is formed in g_cg_rz.
template <int PREC>
void cg_body(const ge::Args& a, const GeGrid& G, const CgGrid& C, cudaStream_t cs, bool pdl) {
    if constexpr (PREC == KCFD_PREC_AMG) {
        amg::vcycle((const kcfd_amg*)a.amg, a.r, a.sh, &a.st->active, cs, pdl);
    } else if constexpr (PREC == KCFD_PREC_ILU0) {
        for (int l = 1; l < a.nlev; ++l) ge_launch(ge::g_fwd<1, double>, G.fwd, cs, pdl, a, l, 1);
        for (int l = a.nlev - 2; l >= 0; --l) ge_launch(ge::g_bwd<1, double>, G.bwd, cs, pdl, a, l, 1);
    }
    ge_launch(ge::g_cg_rz<PREC>, C.rz, cs, pdl, a);
    ge_launch(ge::g_cg_p<PREC>, C.p, cs, pdl, a);
    ge_launch(ge::g_cg_q, C.q, cs, pdl, a);
    ge_launch(ge::g_cg_xr, C.xr, cs, pdl, a);
}

// Eager form: init, body trips in chunks with a host read of the active flag, final.
template <int NRHS, int PREC, typename T>
int ge_eager(kcfd_solver* s, cudaStream_t st) {
    const ge::ArgsT<T>& a = ge_args<T>(s);
    const GeGrid G = ge_grids<NRHS, PREC, T>(s->n, s->sm_count, s->g.gmax);
    const bool cg = s->o.method == KCFD_METHOD_CG;
    CgGrid C{};
    ge_fill_values<T>(s, s->g.vals_key, st);
    if constexpr (NRHS == 1 && !ge::is_mixed<T>()) {
        if (cg) {
            C = cg_grids<PREC>(s->n, s->sm_count, s->g.gmax);
            ge::g_cg_init<<<C.init, ge::kBlock, 0, st>>>(a);
        }
    }
    if (!cg) ge::g_init<NRHS, T><<<G.init, ge::kBlock, 0, st>>>(a);
    KCFD_CUDA(cudaGetLastError());
    constexpr int kChunk = 8;
    for (int trips = 0; trips <= a.maxiter + 2; trips += kChunk) {
        int active = 0;
        KCFD_CUDA(cudaMemcpyAsync(&active, &a.st->active, sizeof(int), cudaMemcpyDeviceToHost, st));
        KCFD_CUDA(cudaStreamSynchronize(st));
        if (!active) break;
        for (int k = 0; k < kChunk; ++k) {
            if constexpr (NRHS == 1 && !ge::is_mixed<T>()) {
                if (cg) {
                    cg_body<PREC>(a, G, C, st, s->g.pdl);
                    continue;
                }
            }
            ge_body<NRHS, PREC, T>(a, G, st, s->g.pdl);
        }
        KCFD_CUDA(cudaGetLastError());
    }
    ge::g_final<NRHS, T><<<ge_fill_grid(s, s->n), 256, 0, st>>>(a);
    KCFD_CUDA(cudaGetLastError());
    return KCFD_OK;
}

template <int NRHS, int PREC, typename T>
int ge_build(kcfd_solver* s, const kcfd_csr_t* A) {
    auto& g = s->g;
    const int n = s->n;
    constexpr bool mix = ge::is_mixed<T>();
    ge::ArgsT<T> a;
    std::memset(&a, 0, sizeof(a));
    a.n = n;
    a.nlev = s->nlev;
    a.stop = s->o.stop;
    a.maxiter = s->o.maxiter;
    a.gmax = g.gmax;
    a.rtol = s->o.rtol;
    a.atol = s->o.atol;
    a.lev = s->lev_ptr;
    if constexpr (mix) {
        a.A = g.A32;
        a.L = g.L32;
        a.U = g.U32;
    } else {
        a.A = g.A;
        a.L = g.L;
        a.U = g.U;
    }
    a.A64 = g.A;
    a.dinv = (const T*)s->dinv;
    a.ldi = (const T*)s->ludinv;
    const size_t len = (size_t)n * NRHS;
    a.x = g.gx;
    a.b = g.gb;
    T* v;
    if constexpr (mix) v = g.vec32;
    else v = g.vec;
    a.r = v; a.rh = v + len; a.p = v + 2 * len; a.v = v + 3 * len; a.t = v + 4 * len; a.ph = v + 5 * len;
    a.sh = v + 6 * len;
    a.st = g.st;
    a.part = g.part;
    a.cnt = g.cnt;
    a.out_iters = g.res_i;
    a.out_status = g.res_i + 3;
    a.out_relres = g.res_d;
    a.eager = g.eager;
    a.amg = s->amg;
    if (g.exec) cudaGraphExecDestroy(g.exec);
    if (g.graph) cudaGraphDestroy(g.graph);
    g.exec = nullptr;
    g.graph = nullptr;
    g.ready = false;
    if (g.eager) {
        // no graph: the host loop launches the same kernels (ge_eager)
        ge_args<T>(s) = a;
        g.vals_key = A->vals64;
        g.ready = true;
        return KCFD_OK;
    }
    KCFD_CUDA(cudaGraphCreate(&g.graph, 0));
    cudaGraphConditionalHandle cond;
    KCFD_CUDA(cudaGraphConditionalHandleCreate(&cond, g.graph, 1, cudaGraphCondAssignDefault));
    a.cond = cond;
    ge_args<T>(s) = a;
    const GeGrid G = ge_grids<NRHS, PREC, T>(n, s->sm_count, g.gmax);
    // node 1: the caller's values into the SELL copy (the graph holds their pointer)
    int64_t f_m = g.slotsA;
    const int* f_src = g.srcA;
    const double* f_in = A->vals64;
    double* f_out = g.A.val;
    void* fargs[] = {&f_m, &f_src, &f_in, &f_out};
    cudaKernelNodeParams kf;
    std::memset(&kf, 0, sizeof(kf));
    kf.func = (void*)ge::g_fill<double, double>;
    kf.gridDim = dim3(ge_fill_grid(s, g.slotsA));
    kf.blockDim = dim3(256);
    kf.kernelParams = fargs;
    cudaGraphNode_t n_fill, n_init, n_cond, n_fin;
    KCFD_CUDA(cudaGraphAddKernelNode(&n_fill, g.graph, nullptr, 0, &kf));
    if constexpr (mix) {
        // MIXED: the FP32 difference form of the values just filled
        int d_n = n;
        ge::Sell d_a = g.A;
        float* d_out = g.A32.val;
        void* dargs[] = {&d_n, &d_a, &d_out};
        cudaKernelNodeParams kd;
        std::memset(&kd, 0, sizeof(kd));
        kd.func = (void*)ge::g_diff32;
        kd.gridDim = dim3(ge_fill_grid(s, n));
        kd.blockDim = dim3(256);
        kd.kernelParams = dargs;
        cudaGraphNode_t n_diff;
        KCFD_CUDA(cudaGraphAddKernelNode(&n_diff, g.graph, &n_fill, 1, &kd));
        n_fill = n_diff;
    }
    const bool cg = s->o.method == KCFD_METHOD_CG;
    CgGrid C{};
    void* args[] = {&a};
    cudaKernelNodeParams kp;
    std::memset(&kp, 0, sizeof(kp));
    kp.func = (void*)ge::g_init<NRHS, T>;
    kp.gridDim = dim3(G.init);
    if constexpr (NRHS == 1 && !ge::is_mixed<T>()) {
        if (cg) {
            C = cg_grids<PREC>(n, s->sm_count, g.gmax);
            kp.func = (void*)ge::g_cg_init;
            kp.gridDim = dim3(C.init);
        }
    }
    kp.blockDim = dim3(ge::kBlock);
    kp.kernelParams = args;
    KCFD_CUDA(cudaGraphAddKernelNode(&n_init, g.graph, &n_fill, 1, &kp));
    // zero-initialised storage (the struct's default constructor is deleted)
    alignas(cudaGraphNodeParams) unsigned char cp_buf[sizeof(cudaGraphNodeParams)] = {};
    cudaGraphNodeParams& cp = *reinterpret_cast<cudaGraphNodeParams*>(cp_buf);
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = cond;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    KCFD_CUDA(cudaGraphAddNode(&n_cond, g.graph, &n_init, 1, &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    cudaStream_t cs;
    KCFD_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    cudaError_t e = cudaStreamBeginCaptureToGraph(cs, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
        bool done = false;
        if constexpr (NRHS == 1 && !ge::is_mixed<T>()) {
            if (cg) {
                cg_body<PREC>(a, G, C, cs, g.pdl);
                done = true;
            }
        }
        if (!done) ge_body<NRHS, PREC, T>(a, G, cs, g.pdl);
        cudaGraph_t outg = nullptr;
        const cudaError_t e2 = cudaStreamEndCapture(cs, &outg);
        if (e == cudaSuccess) e = e2;
    }
    const cudaError_t e3 = cudaStreamDestroy(cs);
    KCFD_CUDA(e3);
    if (e == cudaSuccess) {
        kp.func = (void*)ge::g_final<NRHS, T>;
        kp.gridDim = dim3(ge_fill_grid(s, n));
        kp.blockDim = dim3(256);
        e = cudaGraphAddKernelNode(&n_fin, g.graph, &n_cond, 1, &kp);
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(&g.exec, g.graph, 0);
    if (e != cudaSuccess && g.pdl) {
        // a driver that does not take programmatic edges inside the loop body: plain launches
        cudaGetLastError();
        if (g.exec) cudaGraphExecDestroy(g.exec);
        cudaGraphDestroy(g.graph);
        g.exec = nullptr;
        g.graph = nullptr;
        g.pdl = false;
        return ge_build<NRHS, PREC, T>(s, A);
    }
    KCFD_CUDA(e);
    g.vals_key = A->vals64;
    g.ready = true;
    return KCFD_OK;
}

// Run-time (nrhs, precond) -> template instance.
template <template <int, int, typename> class F, typename... Ts>
int ge_dispatch(const kcfd_solver* s, Ts... args) {
    const int r = s->o.nrhs, p = s->o.precond;
    const bool m = s->g.mix != 0;
#define GE_CASE(R, P) \
    if (r == R && p == P && !m) return F<R, P, double>::run(args...);
#define GE_CASE_MIX(R, P) \
    if (r == R && p == P && m) return F<R, P, float>::run(args...);
    GE_CASE(1, 0) GE_CASE(1, 1) GE_CASE(1, 2) GE_CASE(2, 0) GE_CASE(2, 1) GE_CASE(2, 2)
    GE_CASE(3, 0) GE_CASE(3, 1) GE_CASE(3, 2) GE_CASE(1, 3)
    GE_CASE_MIX(1, 0) GE_CASE_MIX(1, 1) GE_CASE_MIX(1, 2) GE_CASE_MIX(2, 0) GE_CASE_MIX(2, 1) GE_CASE_MIX(2, 2)
    GE_CASE_MIX(3, 0) GE_CASE_MIX(3, 1) GE_CASE_MIX(3, 2)
#undef GE_CASE
#undef GE_CASE_MIX
    set_error("graph engine: unsupported configuration (nrhs %d, precond %d, mixed %d)", r, p, (int)m);
    return KCFD_BAD_INPUT;
}

template <int R, int P, typename T>
struct GeBuild {
    static int run(kcfd_solver* s, const kcfd_csr_t* A) { return ge_build<R, P, T>(s, A); }
};
template <int R, int P, typename T>
struct GeEager {
    static int run(kcfd_solver* s, cudaStream_t st) { return ge_eager<R, P, T>(s, st); }
};

// Host SELL-32 of rows [0, n): row i's entries are [rb(i), re(i)) of a CSR with
// columns col; src (empty: the CSR position itself) gives each entry's value source.
struct SellHost {
    std::vector<int> off, col, src;
};

template <class RB, class RE>
bool make_sell(int n, RB rb, RE re, const std::vector<int>& col, const std::vector<int>& src, SellHost& h) {
    const int ns = (n + 31) / 32;
    h.off.assign(ns + 1, 0);
    int64_t tot = 0;
    for (int sl = 0; sl < ns; ++sl) {
        int w = 0;
        for (int i = 32 * sl; i < std::min(n, 32 * sl + 32); ++i) w = std::max(w, re(i) - rb(i));
        h.off[sl] = (int)tot;
        tot += 32LL * w;
        if (tot > INT32_MAX) return false;
    }
    h.off[ns] = (int)tot;
    h.col.assign(tot, -1);
    h.src.assign(tot, -1);
    for (int i = 0; i < n; ++i) {
        const int b = rb(i), len = re(i) - b;
        for (int k = 0; k < len; ++k) {
            const int64_t slot = h.off[i >> 5] + 32LL * k + (i & 31);
            h.col[slot] = col[b + k];
            h.src[slot] = src.empty() ? b + k : src[b + k];
        }
    }
    return true;
}

bool upload_sell(const SellHost& h, ge::Sell& d, int** src, int64_t& slots, ge::SellT<float>* d32) {
    slots = (int64_t)h.col.size();
    bool ok = upload(&d.off, h.off) && upload(&d.col, h.col) && upload(src, h.src) &&
              cudaMalloc(&d.val, std::max<int64_t>(slots, 1) * sizeof(double)) == cudaSuccess;
    if (ok && d32) {
        // MIXED: FP32 values on the same slots
        d32->off = d.off;
        d32->col = d.col;
        ok = cudaMalloc(&d32->val, std::max<int64_t>(slots, 1) * sizeof(float)) == cudaSuccess;
    }
    return ok;
}

// The engine's SELL copies: A from the rows (rowptr, cols; src maps an entry to the
// caller's value index, empty for the identity); with ILU (diag given) also the
// strict lower / upper parts, whose values come from the factor in CSR position.
int ge_build_sell(kcfd_solver* s, const std::vector<int>& rowptr, const std::vector<int>& cols,
                  const std::vector<int>& src, const std::vector<int>& diag) {
    auto& g = s->g;
    const int n = s->n;
    SellHost h;
    const bool m = g.mix != 0;
    bool ok = make_sell(n, [&](int i) { return rowptr[i]; }, [&](int i) { return rowptr[i + 1]; }, cols, src, h) &&
              upload_sell(h, g.A, &g.srcA, g.slotsA, m ? &g.A32 : nullptr);
    if (ok && !diag.empty()) {
        const std::vector<int> none;
        ok = make_sell(n, [&](int i) { return rowptr[i]; }, [&](int i) { return diag[i]; }, cols, none, h) &&
             upload_sell(h, g.L, &g.srcL, g.slotsL, m ? &g.L32 : nullptr);
        ok = ok && make_sell(n, [&](int i) { return diag[i] + 1; }, [&](int i) { return rowptr[i + 1]; }, cols, none, h) &&
             upload_sell(h, g.U, &g.srcU, g.slotsU, m ? &g.U32 : nullptr);
    }
    if (!ok) {
        set_error("graph engine: sliced-ELL copy too large or device allocation failed");
        return KCFD_CUDA_ERROR;
    }
    return KCFD_OK;
}

int ge_alloc(kcfd_solver* s) {
    auto& g = s->g;
    const size_t len = (size_t)s->n * s->o.nrhs;
    g.gmax = s->sm_count * 8;  // 256-thread blocks: at most 8 resident per SM
    bool ok = cudaMalloc(&g.st, sizeof(ge::St)) == cudaSuccess &&
              cudaMalloc(&g.part, (size_t)ge::kSlotsG * ge::kSlotK * g.gmax * sizeof(double)) == cudaSuccess &&
              cudaMalloc(&g.cnt, ge::kSlotsG * sizeof(unsigned)) == cudaSuccess &&
              (g.mix ? cudaMalloc(&g.vec32, 7 * len * sizeof(float)) : cudaMalloc(&g.vec, 7 * len * sizeof(double))) ==
                  cudaSuccess &&
              cudaMalloc(&g.res_i, 6 * sizeof(int)) == cudaSuccess && cudaMalloc(&g.res_d, 3 * sizeof(double)) == cudaSuccess;
    if (ok) {
        if (s->perm) {
            g.gx = s->px;
            g.gb = s->pb;
        } else {
            ok = cudaMalloc(&g.gx, len * sizeof(double)) == cudaSuccess &&
                 cudaMalloc(&g.gb, len * sizeof(double)) == cudaSuccess;
        }
    }
    ok = ok && cudaMemset(g.cnt, 0, ge::kSlotsG * sizeof(unsigned)) == cudaSuccess &&
         cudaMemset(g.st, 0, sizeof(ge::St)) == cudaSuccess;
    if (!ok) {
        set_error("graph engine: device allocation failed");
        return KCFD_CUDA_ERROR;
    }
    return KCFD_OK;
}

template <int NRHS>
void ge_copies(const kcfd_solver* s, bool in, const double* b, double* x, int32_t* iters, double* relres,
               int32_t* status, cudaStream_t st) {
    const int n = s->n;
    const int blocks = std::max(1, std::min((n + 255) / 256, s->sm_count * 8));
    if (in)
        ge::g_copy_in<NRHS><<<blocks, 256, 0, st>>>(n, s->perm, x, b, s->g.gx, s->g.gb);
    else
        ge::g_copy_out<NRHS><<<blocks, 256, 0, st>>>(n, s->perm, s->g.gx, x, s->g.res_i, s->g.res_d, s->g.res_i + 3,
                                                     iters, relres, status);
}

int ge_solve(kcfd_solver* s, const kcfd_csr_t* A, const double* b, double* x, int32_t* iters, double* relres,
             int32_t* status, cudaStream_t st) {
    auto& g = s->g;
    // the graph holds the caller's value pointer: rebuilt when it moves
    if (!g.ready || g.vals_key != A->vals64) {
        if (int e = ge_dispatch<GeBuild>(s, s, A)) return e;
    }
    auto copies = [&](bool in) {
        if (s->o.nrhs == 1) ge_copies<1>(s, in, b, x, iters, relres, status, st);
        else if (s->o.nrhs == 2) ge_copies<2>(s, in, b, x, iters, relres, status, st);
        else ge_copies<3>(s, in, b, x, iters, relres, status, st);
    };
    copies(true);
    KCFD_CUDA(cudaGetLastError());
    if (g.eager) {
        if (int e = ge_dispatch<GeEager>(s, s, st)) return e;
    } else {
        KCFD_CUDA(cudaGraphLaunch(g.exec, st));
    }
    copies(false);
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

// One barrier of a team of `size` members met by gridDim.x CTAs (ranks 0..gridDim.x-1).
__global__ void selftest_barrier_kernel(TeamCtl ctl, int size) {
    GridTeam tm(ctl, blockIdx.x, size);
    tm.sync();
}

int kcfd_selftest_barrier(int32_t ctas, int32_t team_size, int64_t budget_cycles, uint32_t* bar, int32_t* err,
                          void* stream) {
    KCFD_REQUIRE(bar && err, "kcfd_selftest_barrier: NULL argument");
    KCFD_REQUIRE(ctas >= 1 && ctas <= 64 && team_size >= ctas && team_size <= 65,
                 "kcfd_selftest_barrier: need 1 <= ctas <= 64 and ctas <= team_size <= 65");
    KCFD_REQUIRE(budget_cycles > 0 && budget_cycles <= 4000000000LL, "kcfd_selftest_barrier: budget out of range");
    TeamCtl ctl;
    ctl.bar = bar;
    ctl.partials = nullptr;
    ctl.err = err;
    ctl.budget = budget_cycles;
    selftest_barrier_kernel<<<ctas, 32, 0, (cudaStream_t)stream>>>(ctl, team_size);
    KCFD_CUDA(cudaGetLastError());
    return KCFD_OK;
}

struct kcfd_graph {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

int kcfd_graph_capture_begin(void* stream) {
    KCFD_REQUIRE(stream, "kcfd_graph_capture_begin: a non-default stream is required");
    KCFD_CUDA(cudaStreamBeginCapture((cudaStream_t)stream, cudaStreamCaptureModeThreadLocal));
    return KCFD_OK;
}

int kcfd_graph_capture_end(void* stream, kcfd_graph** out) {
    KCFD_REQUIRE(stream && out, "kcfd_graph_capture_end: NULL argument");
    *out = nullptr;
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture((cudaStream_t)stream, &g);
    cudaGraphExec_t x = nullptr;
    if (e == cudaSuccess) e = cudaGraphInstantiate(&x, g, 0);
    if (e != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
        set_error("kcfd_graph_capture_end: %s", cudaGetErrorString(e));
        return KCFD_CUDA_ERROR;
    }
    auto* h = new kcfd_graph();
    h->graph = g;
    h->exec = x;
    *out = h;
    return KCFD_OK;
}

int kcfd_graph_launch(kcfd_graph* g, void* stream) {
    KCFD_REQUIRE(g && g->exec, "kcfd_graph_launch: NULL graph");
    KCFD_CUDA(cudaGraphLaunch(g->exec, (cudaStream_t)stream));
    return KCFD_OK;
}

void kcfd_graph_destroy(kcfd_graph* g) {
    if (!g) return;
    if (g->exec) cudaGraphExecDestroy(g->exec);
    if (g->graph) cudaGraphDestroy(g->graph);
    delete g;
}

int kcfd_solver_create(const kcfd_csr_t* A, const kcfd_solver_opts_t* opts, const int32_t* level_of_row_host,
                       kcfd_solver** out) {
    KCFD_REQUIRE(A && opts && out, "kcfd_solver_create: NULL argument");
    *out = nullptr;
    KCFD_REQUIRE(A->n > 0 && A->nnz >= A->n && A->indptr && A->indices, "kcfd_solver_create: bad CSR (n=%d nnz=%d)",
                 A->n, A->nnz);
    KCFD_REQUIRE(opts->nrhs >= 1 && opts->nrhs <= 3, "kcfd_solver_create: nrhs must be 1, 2 or 3");
    KCFD_REQUIRE(opts->precond >= 0 && opts->precond <= 3, "kcfd_solver_create: bad precond");
    const bool amg = opts->precond == KCFD_PREC_AMG;
    KCFD_REQUIRE(!amg || opts->nrhs == 1, "kcfd_solver_create: the AMG preconditioner takes one right-hand side");
    KCFD_REQUIRE(!amg || opts->team == 0 || opts->team == 3,
                 "kcfd_solver_create: the AMG preconditioner runs on the graph engine (team 0 or 3)");
    KCFD_REQUIRE(opts->mode == KCFD_MODE_FP64 || opts->mode == KCFD_MODE_MIXED, "kcfd_solver_create: bad mode");
    KCFD_REQUIRE(opts->stop == KCFD_STOP_SCIPY || opts->stop == KCFD_STOP_GPU, "kcfd_solver_create: bad stop rule");
    KCFD_REQUIRE(!(opts->mode == KCFD_MODE_MIXED && opts->stop == KCFD_STOP_GPU),
                 "kcfd_solver_create: MIXED mode uses the scipy stopping rule");
    KCFD_REQUIRE(opts->maxiter >= 0, "kcfd_solver_create: maxiter < 0");
    KCFD_REQUIRE(opts->method == KCFD_METHOD_BICGSTAB || opts->method == KCFD_METHOD_CG, "kcfd_solver_create: bad method");
    const bool cg = opts->method == KCFD_METHOD_CG;
    KCFD_REQUIRE(!cg || (opts->nrhs == 1 && opts->mode == KCFD_MODE_FP64 && opts->stop == KCFD_STOP_SCIPY &&
                         (opts->team == 0 || opts->team == 3)),
                 "kcfd_solver_create: CG takes one right-hand side, FP64 and the scipy stop rule, and runs on the "
                 "graph engine (team 0 or 3)");
    auto* s = new kcfd_solver();
    s->o = *opts;
    // AMG: the Krylov iteration is FP64 on the graph engine; MIXED selects an FP32
    // multigrid hierarchy (below), so the handle itself runs in FP64
    const int amg_mode = opts->mode;
    if (amg) s->o.mode = KCFD_MODE_FP64;
    if (s->o.mode == KCFD_MODE_MIXED) {
        if (s->o.inner_rtol <= 0) s->o.inner_rtol = 1e-3;
        if (s->o.max_refine <= 0) s->o.max_refine = 60;
        if (s->o.inner_maxiter <= 0) s->o.inner_maxiter = 400;
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
    const bool mixed = s->o.mode == KCFD_MODE_MIXED;
    const size_t vsz = mixed ? sizeof(float) : sizeof(double);
    const int n = A->n, nnz = A->nnz;
    std::vector<int> ip(n + 1), ix(nnz);
    if (cudaMemcpy(ip.data(), A->indptr, ip.size() * 4, cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(ix.data(), A->indices, ix.size() * 4, cudaMemcpyDeviceToHost) != cudaSuccess) {
        free_solver(s);
        set_error("kcfd_solver_create: cannot read the CSR pattern (device pointers expected)");
        return KCFD_BAD_INPUT;
    }
    auto fail = [&](const char* msg, int a1 = 0, int a2 = 0, int a3 = 0) {
        free_solver(s);
        set_error(msg, a1, a2, a3);
        return KCFD_BAD_INPUT;
    };
    if (ip[0] != 0 || ip[n] != nnz) return fail("kcfd_solver_create: indptr[0] != 0 or indptr[n] != nnz");
    for (int i = 0; i < n; ++i)
        if (ip[i + 1] < ip[i]) return fail("kcfd_solver_create: indptr not monotone at row %d", i);
    for (int k = 0; k < nnz; ++k)
        if (ix[k] < 0 || ix[k] >= n) return fail("kcfd_solver_create: column index %d out of range at %d", ix[k], k);
    if (mixed) {
        // the FP32 difference form keeps each row's sum on its stored diagonal entry
        for (int i = 0; i < n; ++i) {
            bool has = false;
            for (int k = ip[i]; k < ip[i + 1] && !has; ++k) has = ix[k] == i;
            if (!has) return fail("kcfd_solver_create: MIXED mode needs a stored diagonal entry in every row (row %d)", i);
        }
    }
    // team and launch shape
    // auto: one CTA for tiny systems; the persistent grid kernel up to 40,000 unknowns
    // (and for every mixed solve); the graph engine for large FP64 systems. Measured on
    // a 4,096-row p' system: one CTA 35 us per Krylov iteration, the grid kernel 18 us,
    // the graph engine 25 us. A caller that runs many small solves concurrently (the
    // served loop) asks for one CTA explicitly, so that they overlap.
    int team = (amg || cg) ? 3 : opts->team;
    if (team == 0) {
        const int64_t unk = (int64_t)n * nrhs;
        // MIXED stays on the persistent kernel (FP32 inner iterations, FP64 refinement
        // with revert): the engine's MIXED form (team 3, asked for explicitly) keeps the
        // Krylov space across residual replacements, which diverges on near-singular
        // operators such as a pinned pressure correction at 128^3
        team = (unk <= 1024) ? 1 : ((mixed || unk <= 40000) ? 2 : 3);
    }
    if (team < 1 || team > 3) return fail("kcfd_solver_create: team must be 0..3");
    s->team = team;
    if (team == 3) {
        s->g.mix = mixed ? 1 : 0;
        const char* ev = std::getenv("KCFD_ENGINE_EAGER");
        s->g.eager = (ev && ev[0] == '1') ? 1 : 0;
        const char* pv = std::getenv("KCFD_ENGINE_PDL");
        s->g.pdl = !(pv && pv[0] == '0');
    }
    int lanes = opts->lanes;
    if (lanes <= 0) {
        // one lane streams up to ~8 entries of a row (FVM rows have 4-7): measured
        // fastest on B200 for 7-point rows; wider rows get more lanes
        const double avg = (double)nnz / n;
        lanes = 1;
        while (lanes < 32 && 8 * lanes < avg) lanes <<= 1;
    }
    if ((lanes & (lanes - 1)) != 0 || lanes < 1 || lanes > 32) return fail("kcfd_solver_create: lanes must be 1..32 pow2");
    s->lanes = lanes;
    const int max_grid_block = grid_block(nrhs);
    // one CTA: 512 threads with 128 registers (measured 30.5 us per Jacobi BiCGSTAB
    // iteration on the 64^2 cavity p' system against 32.3 us for 1024 threads at 64)
    s->block = opts->block > 0 ? opts->block : (team == 1 ? 512 : max_grid_block);
    if (team >= 2 && s->block > max_grid_block) s->block = max_grid_block;
    if (team == 1 && s->block > 1024) s->block = 1024;
    if (s->block % 32 != 0 || s->block < 32) return fail("kcfd_solver_create: block must be a multiple of 32");
    // levels
    std::vector<int> lptr;
    std::vector<int> pip, pix, psrc, pdiag;  // ILU: the level-permuted CSR (host copy)
    const int K = opts->precond == KCFD_PREC_ILU0 ? std::max(0, opts->fill_level) : 0;
    if (opts->fill_level < 0) return fail("kcfd_solver_create: fill_level < 0");
    if (opts->precond == KCFD_PREC_ILU0) {
        std::vector<int> lev(n, 0);
        if (K > 0) {
            lev = distance_colouring(n, ip, ix, K + 1);
        } else if (level_of_row_host) {
            for (int i = 0; i < n; ++i) lev[i] = level_of_row_host[i];
        } else {
            for (int i = 0; i < n; ++i)
                for (int k = ip[i]; k < ip[i + 1]; ++k)
                    if (ix[k] < i) lev[i] = std::max(lev[i], lev[ix[k]] + 1);
        }
        int nlev = 0;
        for (int i = 0; i < n; ++i) {
            if (lev[i] < 0) return fail("kcfd_solver_create: negative level at row %d", i);
            nlev = std::max(nlev, lev[i] + 1);
        }
        // permutation: rows grouped by level, row order kept inside a level
        lptr.assign(nlev + 1, 0);
        for (int i = 0; i < n; ++i) lptr[lev[i] + 1]++;
        for (int l = 0; l < nlev; ++l) lptr[l + 1] += lptr[l];
        std::vector<int> perm(n), inv(n), fill(lptr.begin(), lptr.end() - 1);
        for (int i = 0; i < n; ++i) {
            perm[fill[lev[i]]] = i;
            inv[i] = fill[lev[i]]++;
        }
        pip.assign(n + 1, 0);
        pix.clear();
        psrc.clear();
        pdiag.assign(n, -1);
        pix.reserve(nnz);
        psrc.reserve(nnz);
        std::vector<int> plev;                     // ILU(k): level of fill of each entry
        std::vector<std::pair<int, int>> row;      // (permuted column, caller slot)
        std::vector<int> cc, cl, cs;               // the row being built: column, level, slot
        for (int r = 0; r < n; ++r) {
            const int o = perm[r];
            row.clear();
            for (int k = ip[o]; k < ip[o + 1]; ++k) row.emplace_back(inv[ix[k]], k);
            std::sort(row.begin(), row.end());
            cc.clear();
            cl.clear();
            cs.clear();
            for (const auto& e : row) {
                cc.push_back(e.first);
                cl.push_back(0);
                cs.push_back(e.second);
            }
            if (K > 0) {
                // symbolic ILU(k): eliminate with every earlier row k of the factor
                // pattern (in column order, fill included); entry j of row k's upper
                // part gives fill level lev(r,k) + lev(k,j) + 1, kept when <= K
                for (size_t q = 0; q < cc.size() && cc[q] < r; ++q) {
                    const int kr = cc[q], lk = cl[q];
                    for (int e = pdiag[kr] + 1; e < pip[kr + 1]; ++e) {
                        const int nl = lk + plev[e] + 1;
                        if (nl > K) continue;
                        const int j = pix[e];
                        const auto it = std::lower_bound(cc.begin(), cc.end(), j);
                        const size_t at = it - cc.begin();
                        if (it != cc.end() && *it == j) {
                            cl[at] = std::min(cl[at], nl);
                        } else {
                            cc.insert(it, j);
                            cl.insert(cl.begin() + at, nl);
                            cs.insert(cs.begin() + at, -1);
                        }
                    }
                }
            }
            const int len = (int)cc.size();
            if (len > kMaxIluRow)
                return fail("kcfd_solver_create: ILU row %d has %d entries (max %d)", o, len, kMaxIluRow);
            pip[r + 1] = pip[r] + len;
            for (int q = 0; q < len; ++q) {
                const int c = cc[q];
                pix.push_back(c);
                psrc.push_back(cs[q]);
                plev.push_back(cl[q]);
                if (c == r) pdiag[r] = pip[r] + q;
                else if (lev[perm[c]] == lev[o]) return fail("kcfd_solver_create: coupled rows %d, %d share level %d", o, perm[c], lev[o]);
            }
            if (pdiag[r] < 0) return fail("kcfd_solver_create: row %d has no diagonal entry (ILU needs it)", o);
        }
        s->pnnz = pip[n];
        s->nlev = nlev;
        bool ok = upload(&s->perm, perm) && upload(&s->p_indptr, pip) && upload(&s->p_indices, pix) &&
                  upload(&s->p_src, psrc) && upload(&s->p_diag, pdiag);
        const size_t pn = (size_t)s->pnnz;
        ok = ok && cudaMalloc(&s->p_vals64, pn * sizeof(double)) == cudaSuccess;
        if (mixed) ok = ok && cudaMalloc(&s->p_vals32, pn * sizeof(float)) == cudaSuccess;
        ok = ok && cudaMalloc(&s->px, (size_t)n * nrhs * sizeof(double)) == cudaSuccess;
        ok = ok && cudaMalloc(&s->pb, (size_t)n * nrhs * sizeof(double)) == cudaSuccess;
        ok = ok && cudaMalloc(&s->lu, pn * vsz) == cudaSuccess;
        ok = ok && cudaMalloc(&s->ludinv, (size_t)n * vsz) == cudaSuccess;
        if (!ok) {
            free_solver(s);
            set_error("kcfd_solver_create: device allocation failed (ILU)");
            return KCFD_CUDA_ERROR;
        }
    } else {
        lptr = {0, n};
        s->nlev = 1;
    }
    if (cg && opts->precond == KCFD_PREC_ILU0 && s->nlev < 2)
        return fail("kcfd_solver_create: CG with ILU(0) needs a matrix with at least two ILU levels");
    // team 3 keeps the grid kernel's launch shape too: it factors ILU(0) with the
    // grid factor kernel and solves on the grid kernel inside stream captures
    void* kern = amg ? nullptr : solve_kernel_ptr(mixed, nrhs, opts->precond, team >= 2, s->block);
    if (amg) {
        s->grid = 1;  // no persistent kernel: AMG solves run only on the graph engine
    } else if (team >= 2) {
        int per_sm = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, s->block, 0) != cudaSuccess || per_sm < 1) {
            free_solver(s);
            set_error("kcfd_solver_create: solver kernel cannot be resident (block %d)", s->block);
            return KCFD_CUDA_ERROR;
        }
        int per_sm_f = per_sm;
        if (opts->precond == KCFD_PREC_ILU0) {
            void* fk = mixed ? (void*)ilu0_factor_grid<float> : (void*)ilu0_factor_grid<double>;
            if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_f, fk, s->block, 0) != cudaSuccess || per_sm_f < 1) {
                free_solver(s);
                set_error("kcfd_solver_create: ILU factor kernel cannot be resident");
                return KCFD_CUDA_ERROR;
            }
        }
        const int g = std::min(per_sm, per_sm_f) * s->sm_count;
        const int max_useful = std::max(1, (int)((n + s->block - 1) / s->block));
        s->grid = std::max(1, std::min(g, max_useful));
    } else {
        s->grid = 1;
    }
    const size_t len = (size_t)n * nrhs;
    bool ok = upload(&s->lev_ptr, lptr);
    ok = ok && cudaMalloc(&s->work, 9 * len * vsz) == cudaSuccess;
    if (mixed) ok = ok && cudaMalloc(&s->r64, len * sizeof(double)) == cudaSuccess;
    ok = ok && cudaMalloc(&s->bar, 2 * sizeof(unsigned)) == cudaSuccess;
    ok = ok && cudaMalloc(&s->err, sizeof(int)) == cudaSuccess;
    ok = ok && cudaMalloc(&s->partials, (size_t)kSlots * kMaxK * std::max(s->grid, 1) * sizeof(double)) == cudaSuccess;
    if (ok && opts->precond == KCFD_PREC_JACOBI) ok = cudaMalloc(&s->dinv, n * vsz) == cudaSuccess;
    if (ok && mixed && !s->perm) ok = cudaMalloc(&s->v32own, (size_t)nnz * sizeof(float)) == cudaSuccess;
    if (ok) ok = cudaMemset(s->bar, 0, 2 * sizeof(unsigned)) == cudaSuccess && cudaMemset(s->err, 0, sizeof(int)) == cudaSuccess;
    if (!ok) {
        free_solver(s);
        set_error("kcfd_solver_create: device allocation failed");
        return KCFD_CUDA_ERROR;
    }
    if (amg) {
        kcfd_amg_opts_t ao;
        std::memset(&ao, 0, sizeof(ao));
        ao.mode = amg_mode;
        ao.max_levels = opts->amg_max_levels;
        ao.coarse_max = opts->amg_coarse_max;
        if (int e = kcfd_amg_create(A, &ao, &s->amg)) {
            free_solver(s);
            return e;
        }
    }
    if (team == 3) {
        int e = ge_alloc(s);
        if (!e) e = s->perm ? ge_build_sell(s, pip, pix, psrc, pdiag) : ge_build_sell(s, ip, ix, {}, {});
        if (e) {
            free_solver(s);
            return e;
        }
    }
    *out = s;
    return KCFD_OK;
}

void kcfd_solver_destroy(kcfd_solver* s) {
    free_solver(s);
    (void)cudaGetLastError();  // a destructor reports nothing; it leaves no error behind
}

int kcfd_solver_setup(kcfd_solver* s, const kcfd_csr_t* A, void* stream) {
    KCFD_REQUIRE(s && A, "kcfd_solver_setup: NULL argument");
    {
        const cudaError_t pend = cudaGetLastError();
        if (pend != cudaSuccess) {
            set_error("kcfd_solver_setup: error left by an earlier CUDA call: %s", cudaGetErrorString(pend));
            return KCFD_CUDA_ERROR;
        }
    }
    KCFD_REQUIRE(A->n == s->n && A->nnz == s->nnz, "kcfd_solver_setup: matrix size differs from the bound pattern");
    KCFD_REQUIRE(A->vals64, "kcfd_solver_setup: FP64 values required");
    cudaStream_t st = (cudaStream_t)stream;
    const bool mixed = s->o.mode == KCFD_MODE_MIXED;
    const int threads = 256;
    const int rblocks = std::min((s->n + threads - 1) / threads, s->sm_count * 8);
    if (mixed && !s->perm) {
        rowsum_f32_kernel<<<rblocks, threads, 0, st>>>(s->n, A->indptr, A->indices, A->vals64, s->v32own);
        KCFD_CUDA(cudaGetLastError());
    }
    if (s->o.precond == KCFD_PREC_AMG) return amg::setup(s->amg, A->vals64, st);
    if (s->o.precond == KCFD_PREC_JACOBI) {
        const int blocks = std::min((s->n + threads - 1) / threads, s->sm_count * 8);
        if (mixed)
            jacobi_setup_kernel<float><<<blocks, threads, 0, st>>>(s->n, A->indptr, A->indices, A->vals64, (float*)s->dinv);
        else
            jacobi_setup_kernel<double><<<blocks, threads, 0, st>>>(s->n, A->indptr, A->indices, A->vals64, (double*)s->dinv);
        KCFD_CUDA(cudaGetLastError());
    } else if (s->o.precond == KCFD_PREC_ILU0) {
        const int blocks = (int)std::min<int64_t>(((int64_t)s->pnnz + threads - 1) / threads, s->sm_count * 16);
        permute_vals_kernel<<<blocks, threads, 0, st>>>(s->pnnz, s->p_src, A->vals64, s->p_vals64, nullptr);
        if (mixed) rowsum_f32_kernel<<<rblocks, threads, 0, st>>>(s->n, s->p_indptr, s->p_indices, s->p_vals64, s->p_vals32);
        KCFD_CUDA(cudaGetLastError());
        SolveArgs a = make_args(s, A);
        void* args[] = {&a};
        void* k = s->team >= 2 ? (mixed ? (void*)ilu0_factor_grid<float> : (void*)ilu0_factor_grid<double>)
                               : (mixed ? (void*)ilu0_factor_cta<float> : (void*)ilu0_factor_cta<double>);
        if (int e = launch_team(s, k, args, st)) return e;
        if (s->team == 3) {
            // the factor's strict lower / upper parts into the engine's SELL copies
            if (mixed) {
                const float* lu = (const float*)s->lu;
                ge::g_fill<float, float><<<ge_fill_grid(s, s->g.slotsL), 256, 0, st>>>(s->g.slotsL, s->g.srcL, lu, s->g.L32.val);
                ge::g_fill<float, float><<<ge_fill_grid(s, s->g.slotsU), 256, 0, st>>>(s->g.slotsU, s->g.srcU, lu, s->g.U32.val);
            } else {
                const double* lu = (const double*)s->lu;
                ge::g_fill<double, double><<<ge_fill_grid(s, s->g.slotsL), 256, 0, st>>>(s->g.slotsL, s->g.srcL, lu, s->g.L.val);
                ge::g_fill<double, double><<<ge_fill_grid(s, s->g.slotsU), 256, 0, st>>>(s->g.slotsU, s->g.srcU, lu, s->g.U.val);
            }
            KCFD_CUDA(cudaGetLastError());
        }
        return KCFD_OK;
    }
    return KCFD_OK;
}

int kcfd_solver_solve(kcfd_solver* s, const kcfd_csr_t* A, const double* b, double* x, int32_t* iters,
                      double* relres, int32_t* status, void* stream) {
    KCFD_REQUIRE(s && A && b && x, "kcfd_solver_solve: NULL argument");
    KCFD_REQUIRE(A->n == s->n && A->nnz == s->nnz, "kcfd_solver_solve: matrix size differs from the bound pattern");
    const bool mixed = s->o.mode == KCFD_MODE_MIXED;
    KCFD_REQUIRE(A->vals64 != nullptr, "kcfd_solver_solve: FP64 values required");
    // MIXED: the FP32 operator is the handle's own (built by kcfd_solver_setup)
    SolveArgs a = make_args(s, A);
    a.x = x;
    a.b = b;
    a.iters_out = iters;
    a.relres_out = relres;
    a.status_out = status;
    if (s->team == 3) {
        cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
        KCFD_CUDA(cudaStreamIsCapturing((cudaStream_t)stream, &cap));
        if (cap == cudaStreamCaptureStatusNone)
            return ge_solve(s, A, b, x, iters, relres, status, (cudaStream_t)stream);
        KCFD_REQUIRE(s->o.precond != KCFD_PREC_AMG,
                     "kcfd_solver_solve: an AMG solve runs as its own graph; issue it outside stream capture");
    }
    void* kern = solve_kernel_ptr(mixed, s->o.nrhs, s->o.precond, s->team >= 2, s->block);
    KCFD_REQUIRE(kern != nullptr, "kcfd_solver_solve: no kernel for this configuration");
    void* args[] = {&a};
    return launch_team(s, kern, args, (cudaStream_t)stream);
}

int kcfd_solver_apply_precond(kcfd_solver* s, const kcfd_csr_t* A, const double* r, double* z, void* stream) {
    KCFD_REQUIRE(s && A && r && z, "kcfd_solver_apply_precond: NULL argument");
    KCFD_REQUIRE(s->o.nrhs == 1, "kcfd_solver_apply_precond: one right-hand side only");
    KCFD_REQUIRE(s->o.mode == KCFD_MODE_FP64, "kcfd_solver_apply_precond: FP64 handles only");
    KCFD_REQUIRE(A->n == s->n && A->nnz == s->nnz, "kcfd_solver_apply_precond: matrix size differs from the bound pattern");
    cudaStream_t st = (cudaStream_t)stream;
    switch (s->o.precond) {
        case KCFD_PREC_NONE:
            KCFD_CUDA(cudaMemcpyAsync(z, r, (size_t)s->n * sizeof(double), cudaMemcpyDeviceToDevice, st));
            return KCFD_OK;
        case KCFD_PREC_JACOBI: {
            const int blocks = std::max(1, std::min((s->n + 255) / 256, s->sm_count * 8));
            jacobi_apply_kernel<<<blocks, 256, 0, st>>>(s->n, (const double*)s->dinv, r, z);
            KCFD_CUDA(cudaGetLastError());
            return KCFD_OK;
        }
        case KCFD_PREC_ILU0: {
            SolveArgs a = make_args(s, A);
            a.b = r;
            a.x = z;
            void* args[] = {&a};
            void* k = s->team >= 2 ? (void*)ilu_apply_grid_kernel : (void*)ilu_apply_cta_kernel;
            return launch_team(s, k, args, st);
        }
        case KCFD_PREC_AMG: return amg::vcycle(s->amg, r, z, nullptr, st, false);
        default: break;
    }
    set_error("kcfd_solver_apply_precond: unknown preconditioner");
    return KCFD_BAD_INPUT;
}

int kcfd_solver_amg(const kcfd_solver* s, kcfd_amg** out) {
    KCFD_REQUIRE(s && out, "kcfd_solver_amg: NULL argument");
    *out = s->amg;
    return KCFD_OK;
}

int kcfd_solver_info(const kcfd_solver* s, int32_t* info4) {
    KCFD_REQUIRE(s && info4, "kcfd_solver_info: NULL argument");
    info4[0] = s->team;
    info4[1] = s->lanes;
    info4[2] = s->block;
    info4[3] = s->amg ? amg::levels(s->amg) : (s->nlev > 0 ? s->nlev : 1);
    return KCFD_OK;
}

int kcfd_solver_error(kcfd_solver* s, int32_t* err, void* stream) {
    KCFD_REQUIRE(s && err, "kcfd_solver_error: NULL argument");
    KCFD_CUDA(cudaMemcpyAsync(err, s->err, sizeof(int), cudaMemcpyDeviceToHost, (cudaStream_t)stream));
    KCFD_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
    return KCFD_OK;
}

}  // extern "C"

// ---------------------------------------------------------- batched host side --
// Graded cluster tiers: a system of at least 2R, 4R, 8R rows gets 2, 4, 8 CTAs. With
// R chosen automatically (cluster_rows 0) R is the smallest of kGradedRows * 2^k for
// which the cluster teams ask for at most kClusterDemand CTAs per SM in all: a small
// batch then spreads its big systems over the GPU (its length is the slowest team's),
// a large one keeps most systems on one CTA each (its length is its total work).
// Measured on the Delaunay p' systems (FP64, Jacobi; solves/s): the first 128 of the
// 1,024, one tier of 4 CTAs from 131,072 rows 31.2, graded R = 8192 64.0, 16384 59.7,
// 24576 50.2; all 1,024: one tier 89.6, graded R = 8192 80.7, 16384 85.2, 24576 88.5.
constexpr int kGradedRows = 8192;
constexpr double kClusterDemand = 3.5;
// queue counters: [0] big tier, [1] small tier, [2 + t] cluster tier t
constexpr int kQueues = 5;

struct kcfd_batch {
    kcfd_batch_opts_t o;
    int nsys = 0;
    long long n_total = 0, nnz_total = 0;
    int grid = 0;
    BatchSys* sys = nullptr;
    int* order = nullptr;
    int* queue = nullptr;
    int* indptr = nullptr;
    int* indices = nullptr;
    float* vals32 = nullptr;
    void* dinv = nullptr;
    int* lev = nullptr;
    void* work = nullptr;
    double* r64 = nullptr;
    // tiers: order[0..nhuge) cluster teams (cluster tier t: cl_n[t] systems from
    // order[cl_first[t]], clusters of cl_size[t] CTAs, cl_ncl[t] clusters launched), then
    // nbig big systems (512-thread CTAs), then the rest
    static constexpr int kMaxClTiers = 3;
    int nhuge = 0, nbig = 0, grid_big = 0;
    int ntier = 0;
    int cl_size[kMaxClTiers] = {}, cl_n[kMaxClTiers] = {}, cl_ncl[kMaxClTiers] = {}, cl_first[kMaxClTiers] = {};
    unsigned int* cbar[kMaxClTiers] = {};  // [cl_ncl] barrier counters
    int* cslot[kMaxClTiers] = {};          // [cl_ncl] published queue entries
    double* cpart[kMaxClTiers] = {};       // [cl_ncl][kSlots][kMaxK][cl_size]
    cudaStream_t cst[kMaxClTiers] = {};
    cudaEvent_t cev[kMaxClTiers] = {};
    int* cerr = nullptr;
    cudaStream_t side = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
};

namespace {
int free_batch(kcfd_batch* b) {
    if (!b) return KCFD_OK;
    if (b->side) cudaStreamDestroy(b->side);
    if (b->ev_fork) cudaEventDestroy(b->ev_fork);
    if (b->ev_join) cudaEventDestroy(b->ev_join);
    for (int t = 0; t < kcfd_batch::kMaxClTiers; ++t) {
        if (b->cst[t]) cudaStreamDestroy(b->cst[t]);
        if (b->cev[t]) cudaEventDestroy(b->cev[t]);
        void* pt[] = {b->cbar[t], b->cslot[t], b->cpart[t]};
        for (void* p : pt)
            if (p) cudaFree(p);
    }
    void* ps[] = {b->sys, b->order, b->queue, b->indptr, b->indices, b->vals32, b->dinv, b->lev, b->work, b->r64, b->cerr};
    for (void* p : ps)
        if (p) cudaFree(p);
    delete b;
    return KCFD_OK;
}
template <int BLOCK>
void* batch_kernel_ptr_t(int mixed, int precond) {
    if (mixed)
        return precond == KCFD_PREC_JACOBI ? (void*)batch_kernel<1, KCFD_PREC_JACOBI, BLOCK>
                                           : (void*)batch_kernel<1, KCFD_PREC_NONE, BLOCK>;
    return precond == KCFD_PREC_JACOBI ? (void*)batch_kernel<0, KCFD_PREC_JACOBI, BLOCK>
                                       : (void*)batch_kernel<0, KCFD_PREC_NONE, BLOCK>;
}
void* batch_kernel_ptr(int mixed, int precond, bool big) {
    return big ? batch_kernel_ptr_t<512>(mixed, precond) : batch_kernel_ptr_t<256>(mixed, precond);
}
void* batch_cluster_ptr(int mixed, int precond) {
    if (mixed)
        return precond == KCFD_PREC_JACOBI ? (void*)batch_cluster_kernel<1, KCFD_PREC_JACOBI>
                                           : (void*)batch_cluster_kernel<1, KCFD_PREC_NONE>;
    return precond == KCFD_PREC_JACOBI ? (void*)batch_cluster_kernel<0, KCFD_PREC_JACOBI>
                                       : (void*)batch_cluster_kernel<0, KCFD_PREC_NONE>;
}
// The cluster tiers a batch asks for (largest teams first): their team sizes and row
// thresholds; graded (cluster_size 0) or one tier. Host only: whether a cluster of a
// size can be resident is checked by the caller.
int cluster_candidates(int nsys, const int32_t* n, const kcfd_batch_opts_t& o, int sms, int* cand_size, int* cand_rows) {
    int ncand = 0;
    if (o.cluster_rows < 0) return 0;
    if (o.cluster_size == 0) {
        int64_t R = o.cluster_rows;
        if (R == 0) {
            R = kGradedRows;
            for (;; R *= 2) {
                int64_t demand = 0;
                for (int s = 0; s < nsys; ++s) {
                    const int64_t q = n[s] / R;
                    demand += q >= 8 ? 8 : q >= 4 ? 4 : q >= 2 ? 2 : 0;
                }
                if (demand <= (int64_t)(kClusterDemand * sms) || R > INT32_MAX / 16) break;
            }
        }
        for (int c = 8; c >= 2; c >>= 1) {
            cand_size[ncand] = c;
            cand_rows[ncand++] = (int)std::min<int64_t>((int64_t)c * R, INT32_MAX);
        }
    } else {
        cand_size[0] = o.cluster_size;
        cand_rows[0] = o.cluster_rows == 0 ? 131072 : o.cluster_rows;
        ncand = 1;
    }
    return ncand;
}

cudaLaunchConfig_t cluster_config(int clusters, int csize, cudaStream_t st, cudaLaunchAttribute* at) {
    cudaLaunchConfig_t cfg;
    std::memset(&cfg, 0, sizeof(cfg));
    cfg.gridDim = dim3(clusters * csize);
    cfg.blockDim = dim3(512);
    cfg.stream = st;
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = csize;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cfg;
}
}  // namespace

extern "C" {

int kcfd_batch_create(int32_t nsys, const int32_t* n, const int32_t* nnz, const int32_t* indptr_host,
                      const int32_t* indices_host, const kcfd_batch_opts_t* opts, kcfd_batch** out) {
    KCFD_REQUIRE(out && opts && n && nnz && indptr_host && indices_host, "kcfd_batch_create: NULL argument");
    *out = nullptr;
    KCFD_REQUIRE(nsys > 0, "kcfd_batch_create: nsys must be > 0");
    KCFD_REQUIRE(opts->precond == KCFD_PREC_NONE || opts->precond == KCFD_PREC_JACOBI,
                 "kcfd_batch_create: precond must be none or jacobi");
    KCFD_REQUIRE(opts->mode == KCFD_MODE_FP64 || opts->mode == KCFD_MODE_MIXED, "kcfd_batch_create: bad mode");
    KCFD_REQUIRE(opts->restarts >= 0 && opts->restarts <= 1000, "kcfd_batch_create: restarts must be 0..1000");
    KCFD_REQUIRE(opts->stop == KCFD_STOP_SCIPY || (opts->stop == KCFD_STOP_GPU && opts->mode == KCFD_MODE_FP64),
                 "kcfd_batch_create: bad stop rule");
    auto* b = new kcfd_batch();
    b->o = *opts;
    if (b->o.mode == KCFD_MODE_MIXED) {
        if (b->o.inner_rtol <= 0) b->o.inner_rtol = 1e-3;
        if (b->o.max_refine <= 0) b->o.max_refine = 60;
        if (b->o.inner_maxiter <= 0) b->o.inner_maxiter = 400;
    }
    if (b->o.lanes <= 0) b->o.lanes = 1;
    b->nsys = nsys;
    std::vector<BatchSys> sys(nsys);
    long long ro = 0, po = 0, zo = 0;
    for (int s = 0; s < nsys; ++s) {
        if (n[s] <= 0 || nnz[s] < n[s]) {
            free_batch(b);
            set_error("kcfd_batch_create: system %d has n=%d nnz=%d", s, n[s], nnz[s]);
            return KCFD_BAD_INPUT;
        }
        const int32_t* ip = indptr_host + po;
        if (ip[0] != 0 || ip[n[s]] != nnz[s]) {
            free_batch(b);
            set_error("kcfd_batch_create: system %d row pointers do not span its entries", s);
            return KCFD_BAD_INPUT;
        }
        for (int i = 0; i < n[s]; ++i)
            if (ip[i + 1] < ip[i]) {
                free_batch(b);
                set_error("kcfd_batch_create: system %d row pointers not monotone", s);
                return KCFD_BAD_INPUT;
            }
        for (int k = 0; k < nnz[s]; ++k)
            if (indices_host[zo + k] < 0 || indices_host[zo + k] >= n[s]) {
                free_batch(b);
                set_error("kcfd_batch_create: system %d column index out of range", s);
                return KCFD_BAD_INPUT;
            }
        sys[s] = {n[s], nnz[s], ro, po, zo};
        ro += n[s];
        po += n[s] + 1;
        zo += nnz[s];
    }
    b->n_total = ro;
    b->nnz_total = zo;
    // largest first (longest-processing-time order for the dynamic queues). Cluster
    // teams: graded (cluster_size 0) -- a system of at least 8R, 4R or 2R rows gets a
    // cluster of 8, 4 or 2 CTAs (R = cluster_rows, 0: kGradedRows), so that a team's
    // rows per CTA, and so roughly its time per system, stay within a factor of two
    // across the big systems; or one tier of cluster_size CTAs from cluster_rows rows.
    // Then systems of at least big_rows rows go to 512-thread CTAs, the rest to
    // 256-thread CTAs.
    const bool mixed = b->o.mode == KCFD_MODE_MIXED;
    const size_t vsz = mixed ? 4 : 8;
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    std::vector<int> order(nsys);
    for (int s = 0; s < nsys; ++s) order[s] = s;
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return nnz[x] > nnz[y]; });
    const int big_rows = b->o.big_rows == 0 ? 16384 : b->o.big_rows;
    const int csize = b->o.cluster_size;
    if (csize != 0 && (csize < 2 || csize > 8)) {
        free_batch(b);
        set_error("kcfd_batch_create: cluster_size must be 0 (graded) or 2..8");
        return KCFD_BAD_INPUT;
    }
    // candidate cluster tiers (largest teams first) and their row thresholds
    int cand_size[kcfd_batch::kMaxClTiers], cand_rows[kcfd_batch::kMaxClTiers];
    const int ncand = cluster_candidates(nsys, n, b->o, sms, cand_size, cand_rows);
    // keep the tiers whose clusters can be resident (a dropped tier's systems fall to
    // the next one down)
    int ncl_max[kcfd_batch::kMaxClTiers];
    b->ntier = 0;
    for (int t = 0; t < ncand; ++t) {
        int m = 0;
        cudaLaunchAttribute at[1];
        cudaLaunchConfig_t cfg = cluster_config(1, cand_size[t], nullptr, at);
        if (cudaOccupancyMaxActiveClusters(&m, batch_cluster_ptr(mixed, b->o.precond), &cfg) != cudaSuccess) m = 0;
        cudaGetLastError();
        if (m < 1) continue;
        b->cl_size[b->ntier] = cand_size[t];
        cand_rows[b->ntier] = cand_rows[t];
        ncl_max[b->ntier++] = m;
    }
    const int nt = b->ntier;
    auto tier = [&](int x) {
        for (int t = 0; t < nt; ++t)
            if (n[x] >= cand_rows[t]) return t;
        return (big_rows > 0 && n[x] >= big_rows) ? nt : nt + 1;
    };
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return tier(x) < tier(y); });
    b->nhuge = b->nbig = 0;
    for (int s = 0; s < nsys; ++s) {
        const int t = tier(s);
        if (t < nt) b->cl_n[t]++;
        b->nhuge += t < nt ? 1 : 0;
        b->nbig += t == nt ? 1 : 0;
    }
    for (int t = 0, first = 0; t < nt; ++t) {
        b->cl_first[t] = first;
        first += b->cl_n[t];
        b->cl_ncl[t] = std::min(b->cl_n[t], ncl_max[t]);
    }
    int per_sm = 0, per_sm_big = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batch_kernel_ptr(mixed, b->o.precond, false), 256, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_big, batch_kernel_ptr(mixed, b->o.precond, true), 512, 0);
    const int nsmall = nsys - b->nbig - b->nhuge;
    b->grid = std::max(1, std::min(std::max(nsmall, 1), std::max(1, per_sm) * sms));
    b->grid_big = std::max(1, std::min(std::max(b->nbig, 1), std::max(1, per_sm_big) * sms));
    bool ok = cudaMalloc(&b->sys, nsys * sizeof(BatchSys)) == cudaSuccess &&
              cudaMemcpy(b->sys, sys.data(), nsys * sizeof(BatchSys), cudaMemcpyHostToDevice) == cudaSuccess &&
              upload(&b->order, order) && cudaMalloc(&b->queue, kQueues * sizeof(int)) == cudaSuccess &&
              cudaStreamCreateWithFlags(&b->side, cudaStreamNonBlocking) == cudaSuccess &&
              cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming) == cudaSuccess &&
              cudaEventCreateWithFlags(&b->ev_join, cudaEventDisableTiming) == cudaSuccess &&
              cudaMalloc(&b->indptr, po * 4) == cudaSuccess &&
              cudaMemcpy(b->indptr, indptr_host, po * 4, cudaMemcpyHostToDevice) == cudaSuccess &&
              cudaMalloc(&b->indices, zo * 4) == cudaSuccess &&
              cudaMemcpy(b->indices, indices_host, zo * 4, cudaMemcpyHostToDevice) == cudaSuccess &&
              cudaMalloc(&b->dinv, ro * vsz) == cudaSuccess && cudaMalloc(&b->lev, 2 * nsys * sizeof(int)) == cudaSuccess &&
              cudaMalloc(&b->work, 9 * ro * vsz) == cudaSuccess;
    if (ok && mixed) ok = cudaMalloc(&b->vals32, zo * 4) == cudaSuccess && cudaMalloc(&b->r64, ro * 8) == cudaSuccess;
    for (int t = 0; ok && t < nt; ++t) {
        if (b->cl_n[t] == 0) continue;
        const int c = b->cl_ncl[t];
        ok = cudaMalloc(&b->cbar[t], c * sizeof(unsigned int)) == cudaSuccess &&
             cudaMalloc(&b->cslot[t], c * sizeof(int)) == cudaSuccess &&
             cudaMalloc(&b->cpart[t], (size_t)c * kSlots * kMaxK * b->cl_size[t] * sizeof(double)) == cudaSuccess &&
             cudaStreamCreateWithFlags(&b->cst[t], cudaStreamNonBlocking) == cudaSuccess &&
             cudaEventCreateWithFlags(&b->cev[t], cudaEventDisableTiming) == cudaSuccess;
    }
    if (ok && b->nhuge > 0) ok = cudaMalloc(&b->cerr, sizeof(int)) == cudaSuccess;
    if (!ok) {
        free_batch(b);
        set_error("kcfd_batch_create: device allocation failed (%lld rows, %lld entries)", ro, zo);
        return KCFD_CUDA_ERROR;
    }
    *out = b;
    return KCFD_OK;
}

void kcfd_batch_destroy(kcfd_batch* b) { free_batch(b); }

int kcfd_batch_plan(int32_t nsys, const int32_t* n, const kcfd_batch_opts_t* opts, int32_t sm_count, int32_t* team) {
    KCFD_REQUIRE(n && opts && team, "kcfd_batch_plan: NULL argument");
    KCFD_REQUIRE(nsys > 0 && sm_count > 0, "kcfd_batch_plan: nsys and sm_count must be > 0");
    KCFD_REQUIRE(opts->cluster_size == 0 || (opts->cluster_size >= 2 && opts->cluster_size <= 8),
                 "kcfd_batch_plan: cluster_size must be 0 (graded) or 2..8");
    int cand_size[kcfd_batch::kMaxClTiers], cand_rows[kcfd_batch::kMaxClTiers];
    const int ncand = cluster_candidates(nsys, n, *opts, sm_count, cand_size, cand_rows);
    const int big_rows = opts->big_rows == 0 ? 16384 : opts->big_rows;
    for (int s = 0; s < nsys; ++s) {
        team[s] = (big_rows > 0 && n[s] >= big_rows) ? 1 : 0;
        for (int t = 0; t < ncand; ++t)
            if (n[s] >= cand_rows[t]) {
                team[s] = cand_size[t];
                break;
            }
    }
    return KCFD_OK;
}

int kcfd_batch_info(const kcfd_batch* b, int64_t* info) {
    KCFD_REQUIRE(b && info, "kcfd_batch_info: NULL argument");
    info[0] = b->nsys;
    info[1] = b->n_total;
    info[2] = b->nnz_total;
    info[3] = b->grid;
    return KCFD_OK;
}

int kcfd_batch_tiers(const kcfd_batch* b, int32_t* tiers) {
    KCFD_REQUIRE(b && tiers, "kcfd_batch_tiers: NULL argument");
    tiers[0] = b->nhuge;
    tiers[1] = b->nbig;
    tiers[2] = b->nsys - b->nhuge - b->nbig;
    tiers[3] = 0;
    tiers[4] = 0;
    for (int t = 0; t < b->ntier; ++t) {
        tiers[3] += b->cl_n[t] > 0 ? b->cl_ncl[t] : 0;
        if (b->cl_n[t] > 0) tiers[4] = std::max(tiers[4], b->cl_size[t]);
    }
    return KCFD_OK;
}

int kcfd_batch_solve(kcfd_batch* b, const double* vals64, const double* rhs, double* x, int32_t* iters,
                     double* relres, int32_t* status, void* stream) {
    KCFD_REQUIRE(b && vals64 && rhs && x && iters && relres && status, "kcfd_batch_solve: NULL argument");
    cudaStream_t st = (cudaStream_t)stream;
    BatchArgs B;
    std::memset(&B, 0, sizeof(B));
    B.nsys = b->nsys;
    B.lanes = b->o.lanes;
    B.mixed = b->o.mode == KCFD_MODE_MIXED;
    B.precond = b->o.precond;
    B.stop = b->o.stop;
    B.maxiter = b->o.maxiter;
    B.max_refine = b->o.max_refine;
    B.inner_maxiter = b->o.inner_maxiter;
    B.max_restarts = b->o.restarts;
    B.rtol = b->o.rtol;
    B.atol = b->o.atol;
    B.inner_rtol = b->o.inner_rtol;
    B.sys = b->sys;
    B.order = b->order;
    B.queue = b->queue;
    B.indptr = b->indptr;
    B.indices = b->indices;
    B.vals64 = vals64;
    B.vals32 = b->vals32;
    B.dinv = b->dinv;
    B.lev = b->lev;
    B.work = b->work;
    B.r64 = b->r64;
    B.x = x;
    B.b = rhs;
    B.iters = iters;
    B.relres = relres;
    B.status = status;
    KCFD_CUDA(cudaMemsetAsync(b->queue, 0, kQueues * sizeof(int), st));
    for (int t = 0; t < b->ntier; ++t)
        if (b->cl_n[t] > 0) KCFD_CUDA(cudaMemsetAsync(b->cbar[t], 0, b->cl_ncl[t] * sizeof(unsigned int), st));
    if (b->nhuge > 0) KCFD_CUDA(cudaMemsetAsync(b->cerr, 0, sizeof(int), st));
    B.nq = b->nsys;
    void* args[] = {&B};
    const int pgrid = std::max(1, std::min(b->nsys, 4 * b->grid));
    KCFD_CUDA(cudaLaunchKernel(B.mixed ? (void*)batch_prep_kernel<1> : (void*)batch_prep_kernel<0>, dim3(pgrid),
                               dim3(256), args, 0, st));
    // cluster tiers and the big tier on side streams, forked from and joined back into
    // the caller's; the cluster tiers are launched first (largest teams first) so that
    // their clusters find free SMs
    BatchArgs Bb = B, Bs = B;
    Bb.order = b->order + b->nhuge;
    Bb.nq = b->nbig;
    Bs.order = b->order + b->nhuge + b->nbig;
    Bs.queue = b->queue + 1;
    Bs.nq = b->nsys - b->nhuge - b->nbig;
    void* args_b[] = {&Bb};
    void* args_s[] = {&Bs};
    if (b->nhuge > 0 || b->nbig > 0) KCFD_CUDA(cudaEventRecord(b->ev_fork, st));
    if (b->nbig > 0) KCFD_CUDA(cudaStreamWaitEvent(b->side, b->ev_fork, 0));
    for (int t = 0; t < b->ntier; ++t) {
        if (b->cl_n[t] == 0) continue;
        KCFD_CUDA(cudaStreamWaitEvent(b->cst[t], b->ev_fork, 0));
        BatchArgs Bh = B;
        Bh.queue = b->queue + 2 + t;
        Bh.order = b->order + b->cl_first[t];
        Bh.nq = b->cl_n[t];
        ClusterCtl C;
        C.bar = b->cbar[t];
        C.slot = b->cslot[t];
        C.partials = b->cpart[t];
        C.err = b->cerr;
        C.budget = 4000000000LL;  // ~2 s at 2 GHz per barrier wait
        void* args_h[] = {&Bh, &C};
        cudaLaunchAttribute at[1];
        const cudaLaunchConfig_t cfg = cluster_config(b->cl_ncl[t], b->cl_size[t], b->cst[t], at);
        KCFD_CUDA(cudaLaunchKernelExC(&cfg, batch_cluster_ptr(B.mixed, B.precond), args_h));
    }
    if (b->nbig > 0)
        KCFD_CUDA(cudaLaunchKernel(batch_kernel_ptr(B.mixed, B.precond, true), dim3(b->grid_big), dim3(512), args_b, 0,
                                   b->side));
    if (Bs.nq > 0)
        KCFD_CUDA(cudaLaunchKernel(batch_kernel_ptr(B.mixed, B.precond, false), dim3(b->grid), dim3(256), args_s, 0, st));
    if (b->nbig > 0) {
        KCFD_CUDA(cudaEventRecord(b->ev_join, b->side));
        KCFD_CUDA(cudaStreamWaitEvent(st, b->ev_join, 0));
    }
    for (int t = 0; t < b->ntier; ++t) {
        if (b->cl_n[t] == 0) continue;
        KCFD_CUDA(cudaEventRecord(b->cev[t], b->cst[t]));
        KCFD_CUDA(cudaStreamWaitEvent(st, b->cev[t], 0));
    }
    KCFD_CUDA(cudaGetLastError());
    return KCFD_OK;
}

}  // extern "C"

// ------------------------------------------------ allocation-free entry point --
// Some callers cannot allocate device memory: code running while a CUDA graph is
// being captured (cudaMalloc is not allowed then), real-time loops that must not
// block on the allocator, and hosts that run inside a fixed, pre-reserved memory
// budget. kcfd_bicgstab_noalloc serves them: it solves one small system with the
// single-CTA BiCGSTAB kernel and takes its Krylov vectors, Jacobi diagonal and level
// table from the fixed array below instead of a solver handle's cudaMalloc'd scratch.
//
// The array is a file-scope __device__ variable: every GPU that loads libkcfd holds
// it (kNoAllocBytes) until the process exits. Host code must not pass its host-side
// symbol to a kernel; the device address is looked up once per device with
// cudaGetSymbolAddress, on the first call made on that device (so that first call
// should come before any stream capture). All calls share the array and it keeps the
// last call's contents; the kernels re-initialise every vector they read, and calls
// that overlap on the GPU (different streams) race on it.
namespace kcfd {
constexpr int kNoAllocMaxRows = 32768;                      // largest system accepted
constexpr int kNoAllocVecs = 10;                            // 9 Krylov vectors + 1/diag
constexpr size_t kNoAllocDoubles = (size_t)kNoAllocVecs * kNoAllocMaxRows + 32;  // + level table
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocDoubles];

__global__ void noalloc_prep_kernel(int n, const int* __restrict__ ip, const int* __restrict__ ix,
                                    const double* __restrict__ vals, int jacobi, double* __restrict__ dinv,
                                    int* __restrict__ lev_ptr) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (jacobi) {
            double d = 0.0;
            for (int k = ip[i]; k < ip[i + 1]; ++k)
                if (ix[k] == i) d += vals[k];
            dinv[i] = (fabs(d) > 1e-30) ? 1.0 / d : 0.0;
        }
        if (i == 0) {
            lev_ptr[0] = 0;
            lev_ptr[1] = n;
        }
    }
}

// Device address of g_noalloc_scratch per device (looked up once).
static std::mutex g_noalloc_mu;
static double* g_noalloc_ptr[64] = {};

static int noalloc_scratch(double** out, cudaStream_t st) {
    int dev = 0;
    KCFD_CUDA(cudaGetDevice(&dev));
    KCFD_REQUIRE(dev >= 0 && dev < 64, "kcfd_bicgstab_noalloc: device index %d out of range", dev);
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
        // the address look-up may not run inside a capture: refuse with a message that
        // names the cause instead of leaving the caller's capture broken
        cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
        KCFD_CUDA(cudaStreamIsCapturing(st, &cap));
        KCFD_REQUIRE(cap == cudaStreamCaptureStatusNone,
                     "kcfd_bicgstab_noalloc: the first call on device %d must come before any stream capture "
                     "(it looks up the scratch array's address)", dev);
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            set_error("kcfd_bicgstab_noalloc: cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
            return KCFD_CUDA_ERROR;
        }
        g_noalloc_ptr[dev] = (double*)p;
    }
    *out = g_noalloc_ptr[dev];
    return KCFD_OK;
}
}  // namespace kcfd

extern "C" {

int kcfd_noalloc_max_rows(void) { return kcfd::kNoAllocMaxRows; }

int kcfd_bicgstab_noalloc(const kcfd_csr_t* A, const double* b, double* x, int32_t precond, int32_t stop,
                          double rtol, double atol, int32_t maxiter, int32_t* iters, double* relres,
                          int32_t* status, void* stream) {
    KCFD_REQUIRE(A, "kcfd_bicgstab_noalloc: NULL matrix");
    KCFD_REQUIRE(A->n > 0 && A->n <= kcfd::kNoAllocMaxRows,
                 "kcfd_bicgstab_noalloc: n = %d rows; this entry point takes 1..%d rows (use a solver handle above that)",
                 A->n, kcfd::kNoAllocMaxRows);
    KCFD_REQUIRE(A->indptr && A->indices && A->vals64 && b && x, "kcfd_bicgstab_noalloc: NULL argument");
    KCFD_REQUIRE(precond == KCFD_PREC_NONE || precond == KCFD_PREC_JACOBI,
                 "kcfd_bicgstab_noalloc: precond must be KCFD_PREC_NONE or KCFD_PREC_JACOBI");
    KCFD_REQUIRE(stop == KCFD_STOP_SCIPY || stop == KCFD_STOP_GPU, "kcfd_bicgstab_noalloc: bad stop rule");
    KCFD_REQUIRE(maxiter >= 0, "kcfd_bicgstab_noalloc: maxiter < 0");
    double* scratch = nullptr;
    if (int e = kcfd::noalloc_scratch(&scratch, (cudaStream_t)stream)) return e;
    const int n = A->n;
    double* work = scratch;                                     // 9 vectors of n
    double* dinv = scratch + (size_t)9 * kcfd::kNoAllocMaxRows;  // n
    int* lev_ptr = (int*)(scratch + (size_t)kcfd::kNoAllocVecs * kcfd::kNoAllocMaxRows);
    cudaStream_t st = (cudaStream_t)stream;
    const int threads = 256;
    const int blocks = (n + threads - 1) / threads;
    kcfd::noalloc_prep_kernel<<<blocks, threads, 0, st>>>(n, A->indptr, A->indices, A->vals64,
                                                          precond == KCFD_PREC_JACOBI, dinv, lev_ptr);
    KCFD_CUDA(cudaGetLastError());
    kcfd::SolveArgs a;
    std::memset(&a, 0, sizeof(a));
    a.n = n;
    a.lanes = 1;
    a.indptr = A->indptr;
    a.indices = A->indices;
    a.vals64 = A->vals64;
    a.dinv = dinv;
    a.lev_ptr = lev_ptr;
    a.nlev = 1;
    a.work = work;
    a.x = x;
    a.b = b;
    a.stop = stop;
    a.maxiter = maxiter;
    a.rtol = rtol;
    a.atol = atol;
    a.iters_out = iters;
    a.relres_out = relres;
    a.status_out = status;
    void* args[] = {&a};
    void* kern = precond == KCFD_PREC_JACOBI ? (void*)kcfd::solve_cta_kernel<0, 1, KCFD_PREC_JACOBI>
                                             : (void*)kcfd::solve_cta_kernel<0, 1, KCFD_PREC_NONE>;
    KCFD_CUDA(cudaLaunchKernel(kern, dim3(1), dim3(1024), args, 0, st));
    KCFD_CUDA(cudaGetLastError());
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
        spmv_range<VM, VX, NRHS>(ip, ix, val, x, r0, r1, L, [&](int i, const double* acc) {
#pragma unroll
            for (int c = 0; c < NRHS; ++c) y[(size_t)i * NRHS + c] = (VX)acc[c];
        });
    }
}

// Short rows (FVM rows of 4-8 entries), one row per thread: the first kRowBatch
// columns and values of the row are all loaded before the first gather of x, so a
// thread waits for three memory round trips per row (row pointers, entries, x)
// instead of one per entry; longer rows finish in a loop. Entries are summed in row
// order, as the lane kernel does with one lane.
constexpr int kRowBatch = 8;
template <typename VM, typename VX, int NRHS>
__global__ void __launch_bounds__(256) spmv_row_kernel(int n, const int* __restrict__ ip, const int* __restrict__ ix,
                                                       const VM* __restrict__ val, const VX* __restrict__ x,
                                                       VX* __restrict__ y) {
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
        const int kb = __ldg(ip + r), ke = __ldg(ip + r + 1);
        int c[kRowBatch];
        double v[kRowBatch];
#pragma unroll
        for (int k = 0; k < kRowBatch; ++k) {
            const bool in = kb + k < ke;
            c[k] = in ? __ldg(ix + kb + k) : 0;
            v[k] = in ? (double)__ldg(val + kb + k) : 0.0;
        }
        double acc[NRHS];
#pragma unroll
        for (int q = 0; q < NRHS; ++q) acc[q] = 0.0;
#pragma unroll
        for (int k = 0; k < kRowBatch; ++k)
            if (kb + k < ke) {
#pragma unroll
                for (int q = 0; q < NRHS; ++q) acc[q] += v[k] * (double)x[(size_t)c[k] * NRHS + q];
            }
        for (int k = kb + kRowBatch; k < ke; ++k) {
            const int j = __ldg(ix + k);
            const double a = (double)__ldg(val + k);
#pragma unroll
            for (int q = 0; q < NRHS; ++q) acc[q] += a * (double)x[(size_t)j * NRHS + q];
        }
#pragma unroll
        for (int q = 0; q < NRHS; ++q) y[(size_t)r * NRHS + q] = (VX)acc[q];
    }
}

template <typename V>
int spmv_launch(const kcfd_csr_t* A, const V* vals, const V* x, V* y, int nrhs, cudaStream_t st) {
    if (nrhs < 1 || nrhs > 3) {
        set_error("kcfd_spmv: nrhs must be 1, 2 or 3");
        return KCFD_BAD_INPUT;
    }
    // one lane streams up to ~8 entries of a row, as in the solver kernels
    const double avg = (double)A->nnz / std::max(A->n, 1);
    int L = 1;
    while (L < 32 && 8 * L < avg) L <<= 1;
    const int threads = 256;
    if (L == 1) {
        // 8 resident CTAs per SM, rows taken grid-stride (measured fastest on the
        // 128^3 7-point matrix: 39.4 us against 41-43 us for one CTA per 256 rows)
        const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>(((int64_t)A->n + threads - 1) / threads, 148 * 8));
        if (nrhs == 1) spmv_row_kernel<V, V, 1><<<blocks, threads, 0, st>>>(A->n, A->indptr, A->indices, vals, x, y);
        else if (nrhs == 2) spmv_row_kernel<V, V, 2><<<blocks, threads, 0, st>>>(A->n, A->indptr, A->indices, vals, x, y);
        else spmv_row_kernel<V, V, 3><<<blocks, threads, 0, st>>>(A->n, A->indptr, A->indices, vals, x, y);
        KCFD_CUDA(cudaGetLastError());
        return KCFD_OK;
    }
    int blocks = (int)std::min<int64_t>(((int64_t)A->n * L + threads - 1) / threads, 148 * 16);
    blocks = std::max(blocks, 1);
    if (nrhs == 1)
        spmv_kernel<V, V, 1><<<blocks, threads, 0, st>>>(A->n, A->indptr, A->indices, vals, x, y, L);
    else if (nrhs == 2)
        spmv_kernel<V, V, 2><<<blocks, threads, 0, st>>>(A->n, A->indptr, A->indices, vals, x, y, L);
    else
        spmv_kernel<V, V, 3><<<blocks, threads, 0, st>>>(A->n, A->indptr, A->indices, vals, x, y, L);
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
