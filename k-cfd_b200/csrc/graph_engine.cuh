// Graph engine for large systems (solver team 3): BiCGSTAB as lean phase kernels in
// one CUDA graph whose iteration loop is a conditional WHILE node.
//
// The persistent team kernel separates phases with software grid barriers; for big
// systems the phases are long enough that kernel boundaries cost less, and lean
// kernels run at their own full occupancy (more bytes in flight per SM). Per iteration:
//   Jacobi: p-update(+M^-1) | SpMV v (+rhat.v) | s(+M^-1, ||s||) | SpMV t (+t.s, t.t) | x/r (+rhat.r, ||r||)
//   ILU(0): the same plus one forward and one backward kernel per extra level, for
//           phat and for shat (two-level colouring: 2 + 2 kernels).
// Every reduction finishes in the last block to arrive (fixed-order sum over the
// per-block partials), which also advances the scalar state in device memory and
// sets the loop condition, so nothing returns to the host until the solve is done.
// The loop is bounded twice: the state logic stops at maxiter, and block 0 of the
// last kernel stops the loop unconditionally once the trip count passes maxiter + 2.
// Eager form (KCFD_ENGINE_EAGER=1 at solver creation, for profilers that cannot see
// kernels inside graphs with conditional nodes): the same kernels with the same grids
// launched from a host loop that reads the active flag every few trips.
// Scalar formulas and stopping tests are those of bicgstab_body (scipy and GPU-path
// semantics); scalars and reductions are FP64.
//
// Storage type T of the Krylov vectors and of the matrix and preconditioner values:
//  * T = double: the plain FP64 form.
//  * T = float (MIXED): r, rhat, p, v, s, t, phat, shat, A, the ILU factors and
//    D^-1 are stored in FP32; x and b stay FP64 and every product and sum is done in
//    FP64 (loads widened). A is kept in difference form, y_i = d_i x_i +
//    sum_{j != i} a_ij (x_j - x_i) with d_i the FP64 row sum rounded once, so the
//    near-zero row sums of a pinned pressure-correction operator survive the
//    rounding. The recursive residual drifts from b - A x by the FP32 rounding of
//    the recursion; residual replacement (van der Vorst and Ye, 2000) bounds the
//    drift: once the recursive ||r|| has fallen below kReplaceEps times its value at
//    the last replacement, or below the stopping threshold, or kReplaceEvery
//    iterations after the last replacement, or at maxiter, g_rr
//    recomputes r = b - A x from the FP64 iterate with the FP64 values and continues
//    the recursion from it, keeping p and rhat (the Krylov space). Where the true
//    residual has drifted far from the recursive one (more than kDriftRestart times
//    it, or above kDriftRestart times the previous true residual) the Krylov space is
//    no longer consistent with the replaced residual, and the recursion restarts from
//    it instead (rhat = r, p = r: one step of iterative refinement). Convergence is
//    only declared on such a true residual, so the result meets the same FP64
//    stopping test as the plain form. The converged-on-s exit is not taken.
//
// Matrix layout: sliced ELL with slices of 32 rows (SELL-32). Slice s holds rows
// 32s..32s+31; entry k of row i sits at off[s] + 32 k + (i mod 32), padded to the
// slice's longest row with column -1. A warp owns one slice, so each of its matrix
// loads reads 32 consecutive values (fully coalesced) where a row-per-thread CSR
// read touches a cache line per row. Entries keep their CSR order within a row, so
// sums are the same as over the CSR. A holds whole rows (SpMV); L and U the strictly
// lower and upper parts of the level-permuted ILU(0) factors.
//
// No kernel reads through the non-coherent path anything that the same launch
// writes: x, r, p, z are read with plain loads; only the pattern, the matrix and
// preconditioner values (constant during a solve) use __ldg.
#pragma once
#include <cuda_runtime.h>

#include <type_traits>

#include "team.cuh"

namespace kcfd {
namespace ge {

constexpr int kBlock = 256;
constexpr int kSlotsG = 6;
constexpr int kSlotK = 9;  // values per reduction slot (g_rr: 3 per right-hand side)
constexpr double kEps2g = 4.930380657631324e-32;
// MIXED: replace the recursive residual once it has fallen by this factor. The drift
// of an FP32 recursion is about eps32 times the residual at the last replacement, so
// replacing every four decades keeps it near 1e-3 of the current residual; at 1e-2 a
// momentum solve (a decade per iteration) replaced every other iteration, an FP64
// residual each time (the 128^3 launch list: 30 us of 60 per Krylov iteration)
constexpr double kReplaceEps = 1e-4;
// MIXED: restart the recursion when the true residual exceeds the recursive one by this factor
constexpr double kDriftRestart = 2.0;
// MIXED: replace at least every this many iterations (an FP32 recursion on an
// ill-conditioned operator can lose its way before it has fallen by kReplaceEps)
constexpr int kReplaceEvery = 32;

struct St {
    double rho[3], rho_prev[3], alpha[3], omega[3], beta[3], thr[3], bnorm[3], rnorm[3];
    double rr_ref[3];  // MIXED: ||r|| at the last residual replacement
    int done[3], status[3], iters[3], sconv[3], zero_x[3];
    int restart[3];    // MIXED: the recursion restarts from the replaced residual (rhat = r, p = r)
    int it, active, trips, rr;  // rr: MIXED, a residual replacement is due in this trip
    int rr_last, pad;           // MIXED: iteration of the last replacement
};

template <typename V>
struct SellT {
    int* off;      // [slices + 1] first slot of each slice
    int* col;      // [slots] column, -1 for padding
    V* val;        // [slots]
};
using Sell = SellT<double>;

template <typename T>
struct ArgsT {
    int n, nlev, stop, maxiter, gmax;
    double rtol, atol;
    const int* lev;
    SellT<T> A, L, U;
    Sell A64;           // FP64 values of A for true residuals (T = double: A itself)
    const T* dinv;
    const T* ldi;
    double *x, *b;
    T *r, *rh, *p, *v, *t, *ph, *sh;
    St* st;
    double* part;       // [kSlotsG][kSlotK][gmax]
    unsigned* cnt;      // [kSlotsG]
    int* out_iters;
    double* out_relres;
    int* out_status;
    cudaGraphConditionalHandle cond;
    int eager;          // 1: launched from a host loop (no graph, no condition to set)
    const void* amg;    // KCFD_PREC_AMG: the multigrid handle (host-side, for the cycle's launches)
};
using Args = ArgsT<double>;

template <typename T>
constexpr bool is_mixed() { return std::is_same<T, float>::value; }

// Programmatic dependent launch: the phase kernels of one iteration are launched so
// that the next kernel's CTAs may be scheduled while this one drains. Each phase
// kernel first waits for the full completion (and memory visibility) of the kernel
// before it, then allows its own successor to launch. Without the launch attribute
// both instructions return at once.
__device__ __forceinline__ void pdl_enter() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// Rows per thread and per step of the vector kernels: U rows spaced by the grid
// stride, all loads issued before any store (memory-level parallelism).
template <int NRHS>
struct Ilp {
    static constexpr int U = NRHS == 1 ? 4 : (NRHS == 2 ? 2 : 1);
};

// Block partial -> partial array; the last block to arrive sums all partials in a
// fixed order and returns true with the totals in v (all threads of that block).
template <int K, typename T>
__device__ __forceinline__ bool last_block_sum(const ArgsT<T>& a, int slot, double (&v)[K]) {
    static_assert(K <= kSlotK, "reduction slot too narrow");
    __shared__ double sm[32 * kSlotK];
    __shared__ int is_last;
    block_sum<K>(v, sm);
    double* part = a.part + (size_t)slot * kSlotK * a.gmax;
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < K; ++k) part[(size_t)k * a.gmax + blockIdx.x] = v[k];
        __threadfence();
        const unsigned prev = atomicAdd(a.cnt + slot, 1u);
        is_last = (prev == gridDim.x - 1);
    }
    __syncthreads();
    if (!is_last) return false;
    __threadfence();
    // every thread of the last block sums a strided share of the partials, then the
    // block tree combines them: a fixed order for a given grid
#pragma unroll
    for (int k = 0; k < K; ++k) {
        double tsum = 0.0;
        for (int j = threadIdx.x; j < (int)gridDim.x; j += blockDim.x) tsum += __ldcg(part + (size_t)k * a.gmax + j);
        v[k] = tsum;
    }
    block_sum<K>(v, sm);
    if (threadIdx.x == 0) a.cnt[slot] = 0u;  // ready for the next use
    return true;
}

// Top of an iteration (thread 0 of a last block): stopping tests and beta.
template <int NRHS, typename T>
__device__ void top_of_iteration(const ArgsT<T>& a, St& S) {
    const bool gpu = a.stop == KCFD_STOP_GPU;
    const int it = S.it;
    int active = 0;
    for (int c = 0; c < NRHS; ++c) {
        S.beta[c] = 0.0;
        if (S.done[c]) continue;
        if (it >= a.maxiter) {
            S.done[c] = 1;
            S.status[c] = KCFD_MAXITER;
            S.iters[c] = a.maxiter;
            continue;
        }
        if (!gpu) {
            if (S.rnorm[c] < S.thr[c]) { S.done[c] = 1; S.status[c] = KCFD_OK; continue; }
            if (fabs(S.rho[c]) < kEps2g) { S.done[c] = 1; S.status[c] = KCFD_BREAKDOWN; continue; }
            if (it > 0) {
                if (fabs(S.omega[c]) < kEps2g) { S.done[c] = 1; S.status[c] = KCFD_BREAKDOWN; continue; }
                S.beta[c] = (S.rho[c] / S.rho_prev[c]) * (S.alpha[c] / S.omega[c]);
            }
        } else {
            if (fabs(S.rho[c]) < 1e-30) { S.done[c] = 1; S.status[c] = KCFD_BREAKDOWN; S.iters[c] = it + 1; continue; }
            S.beta[c] = (fabs(S.rho_prev[c] * S.omega[c]) > 1e-30) ? (S.rho[c] / S.rho_prev[c]) * (S.alpha[c] / S.omega[c]) : 0.0;
        }
        if (!isfinite(S.beta[c])) { S.done[c] = 1; S.status[c] = KCFD_BREAKDOWN; continue; }
        active = 1;
    }
    S.active = active;
}

__device__ __forceinline__ void level_range(int n, int nlev, const int* lev, int l, int& r0, int& r1) {
    r0 = (nlev == 1) ? 0 : lev[l];
    r1 = (nlev == 1) ? n : lev[l + 1];
}

// Slot of entry 0 of row i and the width of its slice.
template <typename V>
__device__ __forceinline__ void sell_row(const SellT<V>& m, int i, int& base, int& w) {
    const int sl = i >> 5;
    const int o0 = __ldg(m.off + sl), o1 = __ldg(m.off + sl + 1);
    base = o0 + (i & 31);
    w = (o1 - o0) >> 5;
}

// acc += sum_k val x[col] over the row's entries (SUB: acc -= ...), in row order;
// columns and values are loaded in batches of B before the gathers of x.
template <int NRHS, bool SUB = false, typename V, typename X>
__device__ __forceinline__ void sell_gather(const SellT<V>& m, int base, int w, const X* x, double (&acc)[NRHS]) {
    constexpr int B = NRHS == 1 ? 8 : 4;
    for (int k0 = 0; k0 < w; k0 += B) {
        int jj[B];
        double vv[B];
#pragma unroll
        for (int u = 0; u < B; ++u) {
            const bool in = k0 + u < w;
            const int slot = base + (k0 + u) * 32;
            jj[u] = in ? __ldg(m.col + slot) : -1;
            vv[u] = in ? (double)__ldg(m.val + slot) : 0.0;
        }
        double xv[B][NRHS];
#pragma unroll
        for (int u = 0; u < B; ++u)
#pragma unroll
            for (int c = 0; c < NRHS; ++c) xv[u][c] = jj[u] >= 0 ? (double)x[(size_t)jj[u] * NRHS + c] : 0.0;
#pragma unroll
        for (int u = 0; u < B; ++u)
            if (jj[u] >= 0) {
#pragma unroll
                for (int c = 0; c < NRHS; ++c) {
                    if (SUB) acc[c] -= vv[u] * xv[u][c];
                    else acc[c] += vv[u] * xv[u][c];
                }
            }
    }
}

// The SpMV gather of row i: plain (FP64 values) or, for FP32 values, the difference
// form d_i x_i + sum_{j != i} a_ij (x_j - x_i) (the diagonal slot holds d_i).
template <int NRHS, typename V, typename X>
__device__ __forceinline__ void sell_spmv_row(const SellT<V>& m, int i, int base, int w, const X* x,
                                              double (&acc)[NRHS]) {
    if constexpr (!std::is_same<V, float>::value) {
        sell_gather<NRHS>(m, base, w, x, acc);
    } else {
        constexpr int B = NRHS == 1 ? 8 : 4;
        double xi[NRHS];
#pragma unroll
        for (int c = 0; c < NRHS; ++c) xi[c] = (double)x[(size_t)i * NRHS + c];
        for (int k0 = 0; k0 < w; k0 += B) {
            int jj[B];
            double vv[B];
#pragma unroll
            for (int u = 0; u < B; ++u) {
                const bool in = k0 + u < w;
                const int slot = base + (k0 + u) * 32;
                jj[u] = in ? __ldg(m.col + slot) : -1;
                vv[u] = in ? (double)__ldg(m.val + slot) : 0.0;
            }
            double xv[B][NRHS];
#pragma unroll
            for (int u = 0; u < B; ++u)
#pragma unroll
                for (int c = 0; c < NRHS; ++c) xv[u][c] = jj[u] >= 0 ? (double)x[(size_t)jj[u] * NRHS + c] : 0.0;
#pragma unroll
            for (int u = 0; u < B; ++u) {
                if (jj[u] < 0) continue;
#pragma unroll
                for (int c = 0; c < NRHS; ++c) acc[c] += jj[u] == i ? vv[u] * xi[c] : vv[u] * (xv[u][c] - xi[c]);
            }
        }
    }
}

// The forward sweep's gather: acc -= sum_k val y[col], where y = q on the level-0
// rows (col < n0: the sweep's input, never copied) and z elsewhere; row order kept.
template <int NRHS, typename V, typename X>
__device__ __forceinline__ void sell_gather_fwd(const SellT<V>& m, int base, int w, const X* z, const X* q,
                                                int n0, double (&acc)[NRHS]) {
    constexpr int B = NRHS == 1 ? 8 : 4;
    for (int k0 = 0; k0 < w; k0 += B) {
        int jj[B];
        double vv[B];
#pragma unroll
        for (int u = 0; u < B; ++u) {
            const bool in = k0 + u < w;
            const int slot = base + (k0 + u) * 32;
            jj[u] = in ? __ldg(m.col + slot) : -1;
            vv[u] = in ? (double)__ldg(m.val + slot) : 0.0;
        }
        double xv[B][NRHS];
#pragma unroll
        for (int u = 0; u < B; ++u) {
            const X* y = jj[u] < n0 ? q : z;
#pragma unroll
            for (int c = 0; c < NRHS; ++c) xv[u][c] = jj[u] >= 0 ? (double)y[(size_t)jj[u] * NRHS + c] : 0.0;
        }
#pragma unroll
        for (int u = 0; u < B; ++u)
            if (jj[u] >= 0) {
#pragma unroll
                for (int c = 0; c < NRHS; ++c) acc[c] -= vv[u] * xv[u][c];
            }
    }
}

// SELL values from a source array: out[k] = in[src[k]], 0 for padding.
template <typename TI, typename TO>
__global__ void g_fill(int64_t m, const int* __restrict__ src, const TI* __restrict__ in, TO* __restrict__ out) {
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < m; k += (int64_t)gridDim.x * blockDim.x) {
        const int j = src[k];
        out[k] = j >= 0 ? (TO)in[j] : (TO)0;
    }
}

// MIXED: the FP32 difference-form copy of A from its FP64 SELL copy (same slots):
// off-diagonal values rounded, the diagonal slot takes the FP64 row sum (summed in
// row order) rounded once; padding 0.
__global__ void g_diff32(int n, Sell a64, float* __restrict__ v32) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        int base, w;
        sell_row(a64, i, base, w);
        double sum = 0.0;
        int dk = -1;
        for (int k = 0; k < w; ++k) {
            const int slot = base + 32 * k;
            const int j = a64.col[slot];
            const double v = a64.val[slot];
            if (j < 0) {
                v32[slot] = 0.0f;
                continue;
            }
            sum += v;
            if (j == i) dk = slot;
            else v32[slot] = (float)v;
        }
        if (dk >= 0) v32[dk] = (float)sum;
    }
}

// y = A M^-1 q on the rows of ILU level 0 is q itself: level-0 rows have no lower
// entries, so their factor rows are A's rows (u_ij = a_ij, u_ii = a_ii), and the
// backward sweep sets z_i = (q_i - sum_j a_ij z_j) / a_ii, so that
// a_ii z_i + sum_j a_ij z_j = q_i whatever the other levels hold. The SpMV kernels
// therefore take q there and multiply only the rows of the later levels (read from
// the first slice boundary at or below the level-1 start, so warps stay on slices).
// Nothing is stored for those rows: v = p and t = s there, so g_p and g_s read p and
// g_xr reads s in their place (the same values, bit for bit). (MIXED: the identity
// holds for the rounded factor rows, an operator within FP32 rounding of A's; the
// residual replacement measures every residual against the FP64 A.)
// Returns the first row the SpMV loop must treat (0 without the identity).
template <int PREC, typename T>
__device__ __forceinline__ int level0_rows(const ArgsT<T>& a) {
    return (PREC == KCFD_PREC_ILU0 && a.nlev >= 2) ? a.lev[1] : 0;
}

template <int NRHS, typename T>
__global__ void __launch_bounds__(kBlock) g_init(ArgsT<T> a) {
    St& S = *a.st;
    double red[2 * NRHS];
#pragma unroll
    for (int k = 0; k < 2 * NRHS; ++k) red[k] = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += gridDim.x * blockDim.x) {
        double acc[NRHS];
#pragma unroll
        for (int c = 0; c < NRHS; ++c) acc[c] = 0.0;
        int base, w;
        sell_row(a.A64, i, base, w);
        sell_gather<NRHS>(a.A64, base, w, a.x, acc);
#pragma unroll
        for (int c = 0; c < NRHS; ++c) {
            const size_t q = (size_t)i * NRHS + c;
            const double bb = a.b[q], rr = bb - acc[c];
            a.r[q] = (T)rr;
            a.rh[q] = (T)rr;
            a.p[q] = (T)0;
            a.v[q] = (T)0;
            red[c] += bb * bb;
            red[NRHS + c] += rr * rr;
        }
    }
    if (last_block_sum<2 * NRHS>(a, 0, red) && threadIdx.x == 0) {
        const bool gpu = a.stop == KCFD_STOP_GPU;
        for (int c = 0; c < NRHS; ++c) {
            S.bnorm[c] = sqrt(red[c]);
            S.rnorm[c] = sqrt(red[NRHS + c]);
            S.rr_ref[c] = S.rnorm[c];
            S.rho[c] = red[NRHS + c];
            S.rho_prev[c] = S.alpha[c] = S.omega[c] = 1.0;
            S.iters[c] = 0;
            S.status[c] = KCFD_OK;
            S.sconv[c] = 0;
            S.zero_x[c] = 0;
            S.restart[c] = 0;
            if (gpu) {
                S.thr[c] = a.rtol;
                S.done[c] = S.bnorm[c] < 1e-30;
            } else {
                S.thr[c] = fmax(a.atol, a.rtol * S.bnorm[c]);
                S.done[c] = S.bnorm[c] == 0.0;
                S.zero_x[c] = S.done[c];
            }
            if (!isfinite(red[c]) || !isfinite(red[NRHS + c])) {
                S.done[c] = 1;
                S.status[c] = KCFD_BREAKDOWN;
            }
        }
        S.it = 0;
        S.trips = 0;
        S.rr = 0;
        S.rr_last = 0;
        top_of_iteration<NRHS>(a, S);
        if (!a.eager) cudaGraphSetConditional(a.cond, S.active ? 1u : 0u);
    }
}

// p = r + beta (p - omega v) (scipy / GPU-path forms); phat = M^-1 p for Jacobi, or
// phat = p for a single-level ILU (with more levels the sweeps read p itself on
// level 0).
template <int NRHS, int PREC, typename T>
__global__ void __launch_bounds__(kBlock) g_p(ArgsT<T> a) {
    pdl_enter();
    const St& S = *a.st;
    if (blockIdx.x == 0 && threadIdx.x == 0) a.st->trips += 1;
    if (!S.active) return;
    constexpr int U = Ilp<NRHS>::U;
    const bool gpu = a.stop == KCFD_STOP_GPU;
    const int it = S.it;
    const int n0 = level0_rows<PREC>(a);
    double om[NRHS], be[NRHS];
    int dn[NRHS], rs[NRHS];
#pragma unroll
    for (int c = 0; c < NRHS; ++c) {
        om[c] = S.omega[c];
        be[c] = S.beta[c];
        dn[c] = S.done[c];
        rs[c] = is_mixed<T>() ? S.restart[c] : 0;
    }
    const int stride = gridDim.x * blockDim.x;
    for (int i0 = blockIdx.x * blockDim.x + threadIdx.x; i0 < a.n; i0 += U * stride) {
        double R[U][NRHS], P[U][NRHS], V[U][NRHS], D[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int i = i0 + u * stride;
            if (i < a.n) {
                if (PREC == KCFD_PREC_JACOBI) D[u] = (double)__ldg(a.dinv + i);
#pragma unroll
                for (int c = 0; c < NRHS; ++c) {
                    const size_t q = (size_t)i * NRHS + c;
                    R[u][c] = (double)a.r[q];
                    P[u][c] = (double)a.p[q];
                    // level-0 rows: v = A M^-1 p = p (never stored there)
                    V[u][c] = (i < n0) ? P[u][c] : (double)a.v[q];
                }
            }
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int i = i0 + u * stride;
            if (i >= a.n) continue;
#pragma unroll
            for (int c = 0; c < NRHS; ++c) {
                if (dn[c]) continue;
                const size_t q = (size_t)i * NRHS + c;
                double pn;
                if (gpu) pn = R[u][c] + be[c] * (P[u][c] - om[c] * V[u][c]);
                else if (it == 0 || rs[c]) pn = R[u][c];
                else pn = (P[u][c] - om[c] * V[u][c]) * be[c] + R[u][c];
                a.p[q] = (T)pn;
                if (rs[c]) a.rh[q] = a.r[q];  // restart: rhat = r
                if (PREC == KCFD_PREC_JACOBI) a.ph[q] = (T)(D[u] * pn);
                if (PREC == KCFD_PREC_ILU0 && a.nlev == 1) a.ph[q] = (T)pn;  // more levels: the sweeps read p
            }
        }
    }
}

// ILU forward sweep over level l (>= 1): z = q - L z. On the last level the backward
// scaling (no upper entries there) is applied too.
template <int NRHS, typename T>
__global__ void __launch_bounds__(kBlock) g_fwd(ArgsT<T> a, int l, int which) {
    pdl_enter();
    const St& S = *a.st;
    if (!S.active) return;
    const T* q = which ? a.r : a.p;
    T* z = which ? a.sh : a.ph;
    const int n0 = level0_rows<KCFD_PREC_ILU0>(a);  // y = q there (not copied into z)
    int dn[NRHS];
#pragma unroll
    for (int c = 0; c < NRHS; ++c) dn[c] = which ? (S.done[c] || S.sconv[c]) : S.done[c];
    int r0, r1;
    level_range(a.n, a.nlev, a.lev, l, r0, r1);
    const bool last = (l == a.nlev - 1);
    // rows from r0 rounded down to a slice boundary, so that warps and slices align
    for (int i = (r0 & ~31) + blockIdx.x * blockDim.x + threadIdx.x; i < r1; i += gridDim.x * blockDim.x) {
        if (i < r0) continue;
        const double di = last ? (double)__ldg(a.ldi + i) : 1.0;
        double acc[NRHS];
#pragma unroll
        for (int c = 0; c < NRHS; ++c) acc[c] = (double)q[(size_t)i * NRHS + c];
        int base, w;
        sell_row(a.L, i, base, w);
        sell_gather_fwd<NRHS>(a.L, base, w, (const T*)z, q, n0, acc);
#pragma unroll
        for (int c = 0; c < NRHS; ++c)
            if (!dn[c]) z[(size_t)i * NRHS + c] = (T)(acc[c] * di);
    }
}

// ILU backward sweep over level l: z = (z - U z) / u_ii. With a single level this is
// the whole preconditioner after the level-0 copy.
template <int NRHS, typename T>
__global__ void __launch_bounds__(kBlock) g_bwd(ArgsT<T> a, int l, int which) {
    pdl_enter();
    const St& S = *a.st;
    if (!S.active) return;
    T* z = which ? a.sh : a.ph;
    // level 0 of a multi-level factor starts from q (y = q there, not copied into z)
    const T* y = (l == 0 && a.nlev >= 2) ? (which ? a.r : a.p) : z;
    int dn[NRHS];
#pragma unroll
    for (int c = 0; c < NRHS; ++c) dn[c] = which ? (S.done[c] || S.sconv[c]) : S.done[c];
    int r0, r1;
    level_range(a.n, a.nlev, a.lev, l, r0, r1);
    for (int i = (r0 & ~31) + blockIdx.x * blockDim.x + threadIdx.x; i < r1; i += gridDim.x * blockDim.x) {
        if (i < r0) continue;
        const double di = (double)__ldg(a.ldi + i);
        double acc[NRHS];
#pragma unroll
        for (int c = 0; c < NRHS; ++c) acc[c] = (double)y[(size_t)i * NRHS + c];
        int base, w;
        sell_row(a.U, i, base, w);
        sell_gather<NRHS, true>(a.U, base, w, (const T*)z, acc);
#pragma unroll
        for (int c = 0; c < NRHS; ++c)
            if (!dn[c]) z[(size_t)i * NRHS + c] = (T)(acc[c] * di);
    }
}

template <int NRHS, int PREC, typename T>
__global__ void __launch_bounds__(kBlock) g_spmv_v(ArgsT<T> a) {
    pdl_enter();
    St& S = *a.st;
    if (!S.active) return;
    const T* ph = (PREC == KCFD_PREC_NONE) ? a.p : a.ph;
    double red[NRHS];
#pragma unroll
    for (int c = 0; c < NRHS; ++c) red[c] = 0.0;
    const int n0 = level0_rows<PREC>(a);
    const int stride = gridDim.x * blockDim.x;
    for (int q0 = blockIdx.x * blockDim.x + threadIdx.x; q0 < n0 * NRHS; q0 += stride) {
        // v = p on level 0: only its dot with rhat; readers take p there
        red[q0 % NRHS] += (double)a.rh[q0] * (double)a.p[q0];
    }
    for (int i = (n0 & ~31) + blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += stride) {
        if (i < n0) continue;
        int base, w;
        sell_row(a.A, i, base, w);
        double rhv[NRHS], acc[NRHS];
#pragma unroll
        for (int c = 0; c < NRHS; ++c) {
            rhv[c] = (double)a.rh[(size_t)i * NRHS + c];
            acc[c] = 0.0;
        }
        sell_spmv_row<NRHS>(a.A, i, base, w, ph, acc);
#pragma unroll
        for (int c = 0; c < NRHS; ++c) {
            a.v[(size_t)i * NRHS + c] = (T)acc[c];
            red[c] += rhv[c] * acc[c];
        }
    }
    if (last_block_sum<NRHS>(a, 1, red) && threadIdx.x == 0) {
        const bool gpu = a.stop == KCFD_STOP_GPU;
        for (int c = 0; c < NRHS; ++c) {
            S.restart[c] = 0;  // g_p has set rhat = r
            if (S.done[c]) continue;
            if (gpu) {
                S.alpha[c] = (fabs(red[c]) > 1e-30) ? S.rho[c] / red[c] : 0.0;
            } else {
                if (red[c] == 0.0) { S.done[c] = 1; S.status[c] = KCFD_BREAKDOWN; S.iters[c] = S.it + 1; continue; }
                S.alpha[c] = S.rho[c] / red[c];
            }
            if (!isfinite(S.alpha[c])) { S.done[c] = 1; S.status[c] = KCFD_BREAKDOWN; S.iters[c] = S.it + 1; }
        }
    }
}

// s = r - alpha v (in r); shat = M^-1 s for Jacobi, shat = s for a single-level ILU
// (with more levels the sweeps read s itself on level 0); ||s||.
template <int NRHS, int PREC, typename T>
__global__ void __launch_bounds__(kBlock) g_s(ArgsT<T> a) {
    pdl_enter();
    St& S = *a.st;
    if (!S.active) return;
    constexpr int U = Ilp<NRHS>::U;
    const int n0 = level0_rows<PREC>(a);
    double al[NRHS];
    int dn[NRHS];
#pragma unroll
    for (int c = 0; c < NRHS; ++c) {
        al[c] = S.alpha[c];
        dn[c] = S.done[c];
    }
    double red[NRHS];
#pragma unroll
    for (int c = 0; c < NRHS; ++c) red[c] = 0.0;
    const int stride = gridDim.x * blockDim.x;
    for (int i0 = blockIdx.x * blockDim.x + threadIdx.x; i0 < a.n; i0 += U * stride) {
        double R[U][NRHS], V[U][NRHS], D[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int i = i0 + u * stride;
            if (i < a.n) {
                if (PREC == KCFD_PREC_JACOBI) D[u] = (double)__ldg(a.dinv + i);
#pragma unroll
                for (int c = 0; c < NRHS; ++c) {
                    const size_t q = (size_t)i * NRHS + c;
                    R[u][c] = (double)a.r[q];
                    V[u][c] = (i < n0) ? (double)a.p[q] : (double)a.v[q];  // v = p on level 0
                }
            }
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int i = i0 + u * stride;
            if (i >= a.n) continue;
#pragma unroll
            for (int c = 0; c < NRHS; ++c) {
                if (dn[c]) continue;
                const size_t q = (size_t)i * NRHS + c;
                const double sv = R[u][c] - al[c] * V[u][c];
                a.r[q] = (T)sv;
                if (PREC == KCFD_PREC_JACOBI) a.sh[q] = (T)(D[u] * sv);
                if (PREC == KCFD_PREC_ILU0 && a.nlev == 1) a.sh[q] = (T)sv;  // more levels: the sweeps read s
                red[c] += sv * sv;
            }
        }
    }
    if (last_block_sum<NRHS>(a, 2, red) && threadIdx.x == 0) {
        const bool gpu = a.stop == KCFD_STOP_GPU;
        int any_left = 0;
        for (int c = 0; c < NRHS; ++c) {
            if (S.done[c]) continue;
            const double sn = sqrt(red[c]);
            if (!isfinite(sn)) { S.done[c] = 1; S.status[c] = KCFD_BREAKDOWN; S.iters[c] = S.it + 1; continue; }
            // MIXED: ||s|| is a recursive norm; convergence waits for a true residual
            const bool conv = !is_mixed<T>() && (gpu ? (sn / S.bnorm[c] < S.thr[c]) : (sn < S.thr[c]));
            if (conv) {
                S.sconv[c] = 1;  // x += alpha phat happens in g_spmv_t
                S.done[c] = 1;
                S.status[c] = KCFD_OK;
                S.iters[c] = S.it + 1;
                S.rnorm[c] = sn;
                continue;
            }
            any_left = 1;
        }
        if (!any_left) {
            S.active = 0;
            if (!a.eager) cudaGraphSetConditional(a.cond, 0u);
        }
    }
}

// Pending x += alpha phat for right-hand sides that converged on ||s||; t = A shat
// and t.s, t.t for the others.
template <int NRHS, int PREC, typename T>
__global__ void __launch_bounds__(kBlock) g_spmv_t(ArgsT<T> a) {
    pdl_enter();
    St& S = *a.st;
    int sc[NRHS], dn[NRHS];
    double al[NRHS];
    int any_sc = 0;
#pragma unroll
    for (int c = 0; c < NRHS; ++c) {
        sc[c] = S.sconv[c];
        dn[c] = S.done[c];
        al[c] = S.alpha[c];
        any_sc |= sc[c];
    }
    const bool active = S.active;
    if (!active && !any_sc) return;
    const T* ph = (PREC == KCFD_PREC_NONE) ? a.p : a.ph;
    const T* sh = (PREC == KCFD_PREC_NONE) ? a.r : a.sh;
    double red[2 * NRHS];
#pragma unroll
    for (int k = 0; k < 2 * NRHS; ++k) red[k] = 0.0;
    const int stride = gridDim.x * blockDim.x;
    if (any_sc) {
        for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += stride) {
#pragma unroll
            for (int c = 0; c < NRHS; ++c)
                if (sc[c]) a.x[(size_t)i * NRHS + c] += al[c] * (double)ph[(size_t)i * NRHS + c];
        }
    }
    const int n0 = active ? level0_rows<PREC>(a) : 0;
    if (active) {
        for (int q0 = blockIdx.x * blockDim.x + threadIdx.x; q0 < n0 * NRHS; q0 += stride) {
            const int c = q0 % NRHS;
            if (dn[c]) continue;
            const double tv = (double)a.r[q0];  // t = s on level 0 (not stored; g_xr takes s there)
            red[c] += tv * tv;
            red[NRHS + c] += tv * tv;
        }
    }
    for (int i = (n0 & ~31) + blockIdx.x * blockDim.x + threadIdx.x; active && i < a.n; i += stride) {
        if (i < n0) continue;
        int base, w;
        sell_row(a.A, i, base, w);
        double sv[NRHS], acc[NRHS];
#pragma unroll
        for (int c = 0; c < NRHS; ++c) {
            sv[c] = (double)a.r[(size_t)i * NRHS + c];
            acc[c] = 0.0;
        }
        sell_spmv_row<NRHS>(a.A, i, base, w, sh, acc);
#pragma unroll
        for (int c = 0; c < NRHS; ++c) {
            if (dn[c]) continue;
            a.t[(size_t)i * NRHS + c] = (T)acc[c];
            red[c] += acc[c] * sv[c];
            red[NRHS + c] += acc[c] * acc[c];
        }
    }
    if (last_block_sum<2 * NRHS>(a, 3, red) && threadIdx.x == 0) {
        const bool gpu = a.stop == KCFD_STOP_GPU;
        for (int c = 0; c < NRHS; ++c) {
            S.sconv[c] = 0;
            if (S.done[c]) continue;
            if (gpu) S.omega[c] = (red[NRHS + c] > 1e-30) ? red[c] / red[NRHS + c] : 0.0;
            else S.omega[c] = red[c] / red[NRHS + c];
            if (!isfinite(S.omega[c])) { S.done[c] = 1; S.status[c] = KCFD_BREAKDOWN; S.iters[c] = S.it + 1; }
        }
    }
}

// x += alpha phat + omega shat ; r = s - omega t ; rhat.r, ||r||; advance the state
// and the loop condition (MIXED: or hand both to g_rr when a replacement is due).
template <int NRHS, int PREC, typename T>
__global__ void __launch_bounds__(kBlock) g_xr(ArgsT<T> a) {
    pdl_enter();
    St& S = *a.st;
    // unconditional bound on the loop, whatever the state logic does
    if (!a.eager && blockIdx.x == 0 && threadIdx.x == 0 && S.trips > a.maxiter + 2) cudaGraphSetConditional(a.cond, 0u);
    if (!S.active) return;
    // two rows per thread for one right-hand side: 48 registers, 5 resident CTAs per SM
    // (four rows: 77 registers, 3 CTAs; measured 194.5 against 191.2 us per p' iteration)
    constexpr int U = NRHS == 1 ? 2 : Ilp<NRHS>::U;
    const bool gpu = a.stop == KCFD_STOP_GPU;
    const T* ph = (PREC == KCFD_PREC_NONE) ? a.p : a.ph;
    const T* sh = (PREC == KCFD_PREC_NONE) ? a.r : a.sh;
    double al[NRHS], om[NRHS];
    int dn[NRHS];
#pragma unroll
    for (int c = 0; c < NRHS; ++c) {
        al[c] = S.alpha[c];
        om[c] = S.omega[c];
        dn[c] = S.done[c];
    }
    double red[2 * NRHS];
#pragma unroll
    for (int k = 0; k < 2 * NRHS; ++k) red[k] = 0.0;
    const int stride = gridDim.x * blockDim.x;
    const int n0 = level0_rows<PREC>(a);
    for (int i0 = blockIdx.x * blockDim.x + threadIdx.x; i0 < a.n; i0 += U * stride) {
        double X[U][NRHS], HP[U][NRHS], HS[U][NRHS], R[U][NRHS], TT[U][NRHS], RH[U][NRHS];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int i = i0 + u * stride;
            if (i < a.n) {
#pragma unroll
                for (int c = 0; c < NRHS; ++c) {
                    const size_t q = (size_t)i * NRHS + c;
                    X[u][c] = a.x[q];
                    HP[u][c] = (double)ph[q];
                    HS[u][c] = (double)sh[q];
                    R[u][c] = (double)a.r[q];
                    TT[u][c] = (i < n0) ? R[u][c] : (double)a.t[q];  // t = s on level 0
                    RH[u][c] = (double)a.rh[q];
                }
            }
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int i = i0 + u * stride;
            if (i >= a.n) continue;
#pragma unroll
            for (int c = 0; c < NRHS; ++c) {
                if (dn[c]) continue;
                const size_t q = (size_t)i * NRHS + c;
                if (gpu) a.x[q] = X[u][c] + (al[c] * HP[u][c] + om[c] * HS[u][c]);
                else a.x[q] = (X[u][c] + al[c] * HP[u][c]) + om[c] * HS[u][c];
                const double rn = R[u][c] - om[c] * TT[u][c];
                a.r[q] = (T)rn;
                red[c] += RH[u][c] * rn;
                red[NRHS + c] += rn * rn;
            }
        }
    }
    if (last_block_sum<2 * NRHS>(a, 4, red) && threadIdx.x == 0) {
        for (int c = 0; c < NRHS; ++c) {
            if (S.done[c]) continue;
            S.rho_prev[c] = S.rho[c];
            S.rho[c] = red[c];
            S.rnorm[c] = sqrt(red[NRHS + c]);
            S.iters[c] = S.it + 1;
            if (!isfinite(S.rnorm[c]) || !isfinite(S.rho[c])) {
                S.done[c] = 1;
                S.status[c] = KCFD_BREAKDOWN;
                continue;
            }
            if (gpu && S.rnorm[c] / S.bnorm[c] < S.thr[c]) {
                S.done[c] = 1;
                S.status[c] = KCFD_OK;
            }
        }
        S.it += 1;
        if (is_mixed<T>()) {
            int due = 0;
            for (int c = 0; c < NRHS; ++c)
                if (!S.done[c] && (S.rnorm[c] < S.thr[c] || S.rnorm[c] < kReplaceEps * S.rr_ref[c] ||
                                   S.it - S.rr_last >= kReplaceEvery || S.it >= a.maxiter))
                    due = 1;
            if (due) {
                // g_rr (next in this trip) replaces r, tests and sets the condition
                S.rr = 1;
                if (!a.eager) cudaGraphSetConditional(a.cond, S.trips <= a.maxiter + 2 ? 1u : 0u);
                return;
            }
        }
        top_of_iteration<NRHS>(a, S);
        if (!a.eager) cudaGraphSetConditional(a.cond, (S.active && S.trips <= a.maxiter + 2) ? 1u : 0u);
    }
}

// MIXED residual replacement (last kernel of a trip; returns at once unless g_xr
// asked for it): r = b - A x with the FP64 values and the FP64 iterate, stored in
// FP32 for the recursion; rho = rhat.r and ||r|| from it; then the stopping tests of
// the top of the iteration on this true residual.
template <int NRHS, int PREC, typename T>
__global__ void __launch_bounds__(kBlock) g_rr(ArgsT<T> a) {
    pdl_enter();
    St& S = *a.st;
    if (!S.active || !S.rr) return;
    int dn[NRHS];
#pragma unroll
    for (int c = 0; c < NRHS; ++c) dn[c] = S.done[c];
    // rhat.r, ||r|| (FP64 residual), ||r||^2 of the stored residual (rho after a restart)
    double red[3 * NRHS];
#pragma unroll
    for (int k = 0; k < 3 * NRHS; ++k) red[k] = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += gridDim.x * blockDim.x) {
        double acc[NRHS];
#pragma unroll
        for (int c = 0; c < NRHS; ++c) acc[c] = 0.0;
        int base, w;
        sell_row(a.A64, i, base, w);
        sell_gather<NRHS>(a.A64, base, w, a.x, acc);
#pragma unroll
        for (int c = 0; c < NRHS; ++c) {
            if (dn[c]) continue;
            const size_t q = (size_t)i * NRHS + c;
            const double rr = a.b[q] - acc[c];
            const T rs = (T)rr;
            a.r[q] = rs;
            red[c] += (double)a.rh[q] * (double)rs;
            red[NRHS + c] += rr * rr;
            red[2 * NRHS + c] += (double)rs * (double)rs;
        }
    }
    if (last_block_sum<3 * NRHS>(a, 5, red) && threadIdx.x == 0) {
        int rs[NRHS];
        for (int c = 0; c < NRHS; ++c) {
            rs[c] = 0;
            if (S.done[c]) continue;
            const double rec = S.rnorm[c], tn = sqrt(red[NRHS + c]);
            // a true residual far above the recursive one, or above the previous true
            // one: the Krylov space no longer matches; restart from the true residual
            rs[c] = (tn > kDriftRestart * rec || tn > kDriftRestart * S.rr_ref[c]) ? 1 : 0;
            S.rho[c] = rs[c] ? red[2 * NRHS + c] : red[c];
            S.rnorm[c] = tn;
            S.rr_ref[c] = tn;
            if (!isfinite(S.rnorm[c]) || !isfinite(S.rho[c])) {
                S.done[c] = 1;
                S.status[c] = KCFD_BREAKDOWN;
                rs[c] = 0;
            }
        }
        S.rr = 0;
        S.rr_last = S.it;
        top_of_iteration<NRHS>(a, S);
        for (int c = 0; c < NRHS; ++c) {
            S.restart[c] = (rs[c] && !S.done[c]) ? 1 : 0;
            if (S.restart[c]) S.beta[c] = 0.0;
        }
        if (!a.eager) cudaGraphSetConditional(a.cond, (S.active && S.trips <= a.maxiter + 2) ? 1u : 0u);
    }
}

// ---------------------------------------------------------------- CG (one rhs) --
// Preconditioned conjugate gradients with scipy's loop (scipy.sparse.linalg.cg, the
// reference's solve_pressure_correction, core/linear_solver.py:73-93): r = b - A x; each
// iteration z = M^-1 r, rho = r.z, p = z (first) or z + (rho / rho_prev) p, q = A p,
// alpha = rho / p.q, x += alpha p, r -= alpha q; done once ||r|| < max(atol, rtol ||b||),
// tested before every iteration. FP64, one right-hand side. z lives in sh (r itself
// without a preconditioner), q in v.

__global__ void __launch_bounds__(kBlock) g_cg_init(Args a) {
    St& S = *a.st;
    double red[2] = {0.0, 0.0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += gridDim.x * blockDim.x) {
        double acc[1] = {0.0};
        int base, w;
        sell_row(a.A64, i, base, w);
        sell_gather<1>(a.A64, base, w, a.x, acc);
        const double bb = a.b[i], rr = bb - acc[0];
        a.r[i] = rr;
        red[0] += bb * bb;
        red[1] += rr * rr;
    }
    if (last_block_sum<2>(a, 0, red) && threadIdx.x == 0) {
        S.bnorm[0] = sqrt(red[0]);
        S.rnorm[0] = sqrt(red[1]);
        S.thr[0] = fmax(a.atol, a.rtol * S.bnorm[0]);
        S.rho[0] = S.rho_prev[0] = S.alpha[0] = S.beta[0] = 0.0;
        S.iters[0] = 0;
        S.sconv[0] = 0;
        S.status[0] = KCFD_OK;
        S.zero_x[0] = S.bnorm[0] == 0.0;  // scipy returns b
        S.done[0] = S.zero_x[0] || S.rnorm[0] < S.thr[0];
        if (!isfinite(red[0]) || !isfinite(red[1])) {
            S.done[0] = 1;
            S.status[0] = KCFD_BREAKDOWN;
        }
        if (!S.done[0] && a.maxiter <= 0) {
            S.done[0] = 1;
            S.status[0] = KCFD_MAXITER;
        }
        S.it = 0;
        S.trips = 0;
        S.active = !S.done[0];
        if (!a.eager) cudaGraphSetConditional(a.cond, S.active ? 1u : 0u);
    }
}

// rho = r.z (Jacobi: z = D^-1 r, stored); beta.
template <int PREC>
__global__ void __launch_bounds__(kBlock) g_cg_rz(Args a) {
    pdl_enter();
    St& S = *a.st;
    if (blockIdx.x == 0 && threadIdx.x == 0) S.trips += 1;
    if (!S.active) return;
    double red[1] = {0.0};
    const int stride = gridDim.x * blockDim.x;
    for (int i0 = blockIdx.x * blockDim.x + threadIdx.x; i0 < a.n; i0 += 4 * stride) {
        double R[4], Z[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int i = i0 + u * stride;
            if (i >= a.n) continue;
            R[u] = a.r[i];
            if (PREC == KCFD_PREC_JACOBI) Z[u] = __ldg(a.dinv + i) * R[u];
            else if (PREC == KCFD_PREC_NONE) Z[u] = R[u];
            else Z[u] = a.sh[i];
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int i = i0 + u * stride;
            if (i >= a.n) continue;
            if (PREC == KCFD_PREC_JACOBI) a.sh[i] = Z[u];
            red[0] += R[u] * Z[u];
        }
    }
    if (last_block_sum<1>(a, 1, red) && threadIdx.x == 0) {
        S.rho[0] = red[0];
        S.beta[0] = S.it > 0 ? S.rho[0] / S.rho_prev[0] : 0.0;
        if (S.it > 0 && !isfinite(S.beta[0])) {
            S.done[0] = 1;
            S.status[0] = KCFD_BREAKDOWN;
            S.iters[0] = S.it;
            S.active = 0;
            if (!a.eager) cudaGraphSetConditional(a.cond, 0u);
        }
    }
}

// p = z (first iteration) or z + beta p.
template <int PREC>
__global__ void __launch_bounds__(kBlock) g_cg_p(Args a) {
    pdl_enter();
    const St& S = *a.st;
    if (!S.active) return;
    const double be = S.beta[0];
    const bool first = S.it == 0;
    const double* z = PREC == KCFD_PREC_NONE ? a.r : a.sh;
    const int stride = gridDim.x * blockDim.x;
    for (int i0 = blockIdx.x * blockDim.x + threadIdx.x; i0 < a.n; i0 += 4 * stride) {
        double Z[4], P[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int i = i0 + u * stride;
            if (i >= a.n) continue;
            Z[u] = z[i];
            P[u] = first ? 0.0 : a.p[i];
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int i = i0 + u * stride;
            if (i >= a.n) continue;
            a.p[i] = first ? Z[u] : P[u] * be + Z[u];
        }
    }
}

// q = A p (in v), p.q, alpha.
__global__ void __launch_bounds__(kBlock) g_cg_q(Args a) {
    pdl_enter();
    St& S = *a.st;
    if (!S.active) return;
    double red[1] = {0.0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += gridDim.x * blockDim.x) {
        double acc[1] = {0.0};
        int base, w;
        sell_row(a.A, i, base, w);
        sell_gather<1>(a.A, base, w, a.p, acc);
        a.v[i] = acc[0];
        red[0] += a.p[i] * acc[0];
    }
    if (last_block_sum<1>(a, 2, red) && threadIdx.x == 0) {
        S.alpha[0] = S.rho[0] / red[0];
        if (!isfinite(S.alpha[0])) {
            S.done[0] = 1;
            S.status[0] = KCFD_BREAKDOWN;
            S.iters[0] = S.it;
            S.active = 0;
            if (!a.eager) cudaGraphSetConditional(a.cond, 0u);
        }
    }
}

// x += alpha p, r -= alpha q, ||r||; the stopping tests and the loop condition.
__global__ void __launch_bounds__(kBlock) g_cg_xr(Args a) {
    pdl_enter();
    St& S = *a.st;
    if (!a.eager && blockIdx.x == 0 && threadIdx.x == 0 && S.trips > a.maxiter + 2) cudaGraphSetConditional(a.cond, 0u);
    if (!S.active) return;
    const double al = S.alpha[0];
    double red[1] = {0.0};
    const int stride = gridDim.x * blockDim.x;
    for (int i0 = blockIdx.x * blockDim.x + threadIdx.x; i0 < a.n; i0 += 2 * stride) {
        double X[2], P[2], R[2], Q[2];
#pragma unroll
        for (int u = 0; u < 2; ++u) {
            const int i = i0 + u * stride;
            if (i >= a.n) continue;
            X[u] = a.x[i];
            P[u] = a.p[i];
            R[u] = a.r[i];
            Q[u] = a.v[i];
        }
#pragma unroll
        for (int u = 0; u < 2; ++u) {
            const int i = i0 + u * stride;
            if (i >= a.n) continue;
            a.x[i] = X[u] + al * P[u];
            const double rn = R[u] - al * Q[u];
            a.r[i] = rn;
            red[0] += rn * rn;
        }
    }
    if (last_block_sum<1>(a, 4, red) && threadIdx.x == 0) {
        S.rho_prev[0] = S.rho[0];
        S.rnorm[0] = sqrt(red[0]);
        S.it += 1;
        S.iters[0] = S.it;
        // scipy tests before an iteration only: after the last one it reports maxiter
        if (!isfinite(S.rnorm[0])) {
            S.done[0] = 1;
            S.status[0] = KCFD_BREAKDOWN;
        } else if (S.it >= a.maxiter) {
            S.done[0] = 1;
            S.status[0] = KCFD_MAXITER;
        } else if (S.rnorm[0] < S.thr[0]) {
            S.done[0] = 1;
            S.status[0] = KCFD_OK;
        }
        S.active = !S.done[0];
        if (!a.eager) cudaGraphSetConditional(a.cond, (S.active && S.trips <= a.maxiter + 2) ? 1u : 0u);
    }
}

// Results; x = 0 for right-hand sides with b == 0 (scipy returns b), over the grid.
template <int NRHS, typename T>
__global__ void g_final(ArgsT<T> a) {
    const St& S = *a.st;
    for (int c = 0; c < NRHS; ++c) {
        if (!S.zero_x[c]) continue;
        for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += gridDim.x * blockDim.x)
            a.x[(size_t)i * NRHS + c] = 0.0;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        for (int c = 0; c < NRHS; ++c) {
            int st = S.status[c], its = S.iters[c];
            if (!S.done[c]) {
                st = KCFD_MAXITER;
                its = a.maxiter;
            }
            a.out_status[c] = st;
            a.out_iters[c] = its;
            a.out_relres[c] = S.bnorm[c] > 0 ? S.rnorm[c] / S.bnorm[c] : 0.0;
        }
    }
}

// Copy the caller's x, b into the engine's (permuted) vectors, and back.
template <int NRHS>
__global__ void g_copy_in(int n, const int* perm, const double* x, const double* b, double* gx, double* gb) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int o = perm ? perm[i] : i;
#pragma unroll
        for (int c = 0; c < NRHS; ++c) {
            gx[(size_t)i * NRHS + c] = x[(size_t)o * NRHS + c];
            gb[(size_t)i * NRHS + c] = b[(size_t)o * NRHS + c];
        }
    }
}

template <int NRHS>
__global__ void g_copy_out(int n, const int* perm, const double* gx, double* x, const int* ri, const double* rr,
                           const int* rs, int* iters, double* relres, int* status) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int o = perm ? perm[i] : i;
#pragma unroll
        for (int c = 0; c < NRHS; ++c) x[(size_t)o * NRHS + c] = gx[(size_t)i * NRHS + c];
    }
    if (blockIdx.x == 0 && threadIdx.x < NRHS) {
        if (iters) iters[threadIdx.x] = ri[threadIdx.x];
        if (relres) relres[threadIdx.x] = rr[threadIdx.x];
        if (status) status[threadIdx.x] = rs[threadIdx.x];
    }
}

}  // namespace ge
}  // namespace kcfd
