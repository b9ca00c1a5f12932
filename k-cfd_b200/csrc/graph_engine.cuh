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
// semantics), FP64 throughout.
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

#include "team.cuh"

namespace kcfd {
namespace ge {

constexpr int kBlock = 256;
constexpr int kSlotsG = 6;
constexpr double kEps2g = 4.930380657631324e-32;

struct St {
    double rho[3], rho_prev[3], alpha[3], omega[3], beta[3], thr[3], bnorm[3], rnorm[3];
    int done[3], status[3], iters[3], sconv[3], zero_x[3];
    int it, active, trips, pad;
};

struct Sell {
    int* off;      // [slices + 1] first slot of each slice
    int* col;      // [slots] column, -1 for padding
    double* val;   // [slots]
};

struct Args {
    int n, nlev, stop, maxiter, gmax;
    double rtol, atol;
    const int* lev;
    Sell A, L, U;
    const double* dinv;
    const double* ldi;
    double *x, *b, *r, *rh, *p, *v, *t, *ph, *sh;
    St* st;
    double* part;       // [kSlotsG][8][gmax]
    unsigned* cnt;      // [kSlotsG]
    int* out_iters;
    double* out_relres;
    int* out_status;
    cudaGraphConditionalHandle cond;
    int eager;          // 1: launched from a host loop (no graph, no condition to set)
    const void* amg;    // KCFD_PREC_AMG: the multigrid handle (host-side, for the cycle's launches)
};

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
template <int K>
__device__ __forceinline__ bool last_block_sum(const Args& a, int slot, double (&v)[K]) {
    __shared__ double sm[32 * 8];
    __shared__ int is_last;
    block_sum<K>(v, sm);
    double* part = a.part + (size_t)slot * 8 * a.gmax;
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
template <int NRHS>
__device__ void top_of_iteration(const Args& a, St& S) {
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

__device__ __forceinline__ void level_range(const Args& a, int l, int& r0, int& r1) {
    r0 = (a.nlev == 1) ? 0 : a.lev[l];
    r1 = (a.nlev == 1) ? a.n : a.lev[l + 1];
}

// Slot of entry 0 of row i and the width of its slice.
__device__ __forceinline__ void sell_row(const Sell& m, int i, int& base, int& w) {
    const int sl = i >> 5;
    const int o0 = __ldg(m.off + sl), o1 = __ldg(m.off + sl + 1);
    base = o0 + (i & 31);
    w = (o1 - o0) >> 5;
}

// acc += sum_k val x[col] over the row's entries (SUB: acc -= ...), in row order;
// columns and values are loaded in batches of B before the gathers of x.
template <int NRHS, bool SUB = false>
__device__ __forceinline__ void sell_gather(const Sell& m, int base, int w, const double* x, double (&acc)[NRHS]) {
    constexpr int B = NRHS == 1 ? 8 : 4;
    for (int k0 = 0; k0 < w; k0 += B) {
        int jj[B];
        double vv[B];
#pragma unroll
        for (int u = 0; u < B; ++u) {
            const bool in = k0 + u < w;
            const int slot = base + (k0 + u) * 32;
            jj[u] = in ? __ldg(m.col + slot) : -1;
            vv[u] = in ? __ldg(m.val + slot) : 0.0;
        }
        double xv[B][NRHS];
#pragma unroll
        for (int u = 0; u < B; ++u)
#pragma unroll
            for (int c = 0; c < NRHS; ++c) xv[u][c] = jj[u] >= 0 ? x[(size_t)jj[u] * NRHS + c] : 0.0;
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

// The forward sweep's gather: acc -= sum_k val y[col], where y = q on the level-0
// rows (col < n0: the sweep's input, never copied) and z elsewhere; row order kept.
template <int NRHS>
__device__ __forceinline__ void sell_gather_fwd(const Sell& m, int base, int w, const double* z, const double* q,
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
            vv[u] = in ? __ldg(m.val + slot) : 0.0;
        }
        double xv[B][NRHS];
#pragma unroll
        for (int u = 0; u < B; ++u) {
            const double* y = jj[u] < n0 ? q : z;
#pragma unroll
            for (int c = 0; c < NRHS; ++c) xv[u][c] = jj[u] >= 0 ? y[(size_t)jj[u] * NRHS + c] : 0.0;
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
__global__ void g_fill(int64_t m, const int* __restrict__ src, const double* __restrict__ in, double* __restrict__ out) {
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < m; k += (int64_t)gridDim.x * blockDim.x) {
        const int j = src[k];
        out[k] = j >= 0 ? in[j] : 0.0;
    }
}

// y = A M^-1 q on the rows of ILU level 0 is q itself: level-0 rows have no lower
// entries, so their factor rows are A's rows (u_ij = a_ij, u_ii = a_ii), and the
// backward sweep sets z_i = (q_i - sum_j a_ij z_j) / a_ii, so that
// a_ii z_i + sum_j a_ij z_j = q_i whatever the other levels hold. The SpMV kernels
// therefore take q there and multiply only the rows of the later levels (read from
// the first slice boundary at or below the level-1 start, so warps stay on slices).
// Nothing is stored for those rows: v = p and t = s there, so g_p and g_s read p and
// g_xr reads s in their place (the same values, bit for bit).
// Returns the first row the SpMV loop must treat (0 without the identity).
template <int PREC>
__device__ __forceinline__ int level0_rows(const Args& a) {
    return (PREC == KCFD_PREC_ILU0 && a.nlev >= 2) ? a.lev[1] : 0;
}

template <int NRHS>
__global__ void __launch_bounds__(kBlock) g_init(Args a) {
    St& S = *a.st;
    double red[2 * NRHS];
#pragma unroll
    for (int k = 0; k < 2 * NRHS; ++k) red[k] = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += gridDim.x * blockDim.x) {
        double acc[NRHS];
#pragma unroll
        for (int c = 0; c < NRHS; ++c) acc[c] = 0.0;
        int base, w;
        sell_row(a.A, i, base, w);
        sell_gather<NRHS>(a.A, base, w, a.x, acc);
#pragma unroll
        for (int c = 0; c < NRHS; ++c) {
            const size_t q = (size_t)i * NRHS + c;
            const double bb = a.b[q], rr = bb - acc[c];
            a.r[q] = rr;
            a.rh[q] = rr;
            a.p[q] = 0.0;
            a.v[q] = 0.0;
            red[c] += bb * bb;
            red[NRHS + c] += rr * rr;
        }
    }
    if (last_block_sum<2 * NRHS>(a, 0, red) && threadIdx.x == 0) {
        const bool gpu = a.stop == KCFD_STOP_GPU;
        for (int c = 0; c < NRHS; ++c) {
            S.bnorm[c] = sqrt(red[c]);
            S.rnorm[c] = sqrt(red[NRHS + c]);
            S.rho[c] = red[NRHS + c];
            S.rho_prev[c] = S.alpha[c] = S.omega[c] = 1.0;
            S.iters[c] = 0;
            S.status[c] = KCFD_OK;
            S.sconv[c] = 0;
            S.zero_x[c] = 0;
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
        top_of_iteration<NRHS>(a, S);
        if (!a.eager) cudaGraphSetConditional(a.cond, S.active ? 1u : 0u);
    }
}

// p = r + beta (p - omega v) (scipy / GPU-path forms); phat = M^-1 p for Jacobi, or
// phat = p for a single-level ILU (with more levels the sweeps read p itself on
// level 0).
template <int NRHS, int PREC>
__global__ void __launch_bounds__(kBlock) g_p(Args a) {
    pdl_enter();
    const St& S = *a.st;
    if (blockIdx.x == 0 && threadIdx.x == 0) a.st->trips += 1;
    if (!S.active) return;
    constexpr int U = Ilp<NRHS>::U;
    const bool gpu = a.stop == KCFD_STOP_GPU;
    const int it = S.it;
    const int n0 = level0_rows<PREC>(a);
    double om[NRHS], be[NRHS];
    int dn[NRHS];
#pragma unroll
    for (int c = 0; c < NRHS; ++c) {
        om[c] = S.omega[c];
        be[c] = S.beta[c];
        dn[c] = S.done[c];
    }
    const int stride = gridDim.x * blockDim.x;
    for (int i0 = blockIdx.x * blockDim.x + threadIdx.x; i0 < a.n; i0 += U * stride) {
        double R[U][NRHS], P[U][NRHS], V[U][NRHS], D[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int i = i0 + u * stride;
            if (i < a.n) {
                if (PREC == KCFD_PREC_JACOBI) D[u] = __ldg(a.dinv + i);
#pragma unroll
                for (int c = 0; c < NRHS; ++c) {
                    const size_t q = (size_t)i * NRHS + c;
                    R[u][c] = a.r[q];
                    P[u][c] = a.p[q];
                    // level-0 rows: v = A M^-1 p = p (never stored there)
                    V[u][c] = (i < n0) ? P[u][c] : a.v[q];
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
                else if (it == 0) pn = R[u][c];
                else pn = (P[u][c] - om[c] * V[u][c]) * be[c] + R[u][c];
                a.p[q] = pn;
                if (PREC == KCFD_PREC_JACOBI) a.ph[q] = D[u] * pn;
                if (PREC == KCFD_PREC_ILU0 && a.nlev == 1) a.ph[q] = pn;  // more levels: the sweeps read p
            }
        }
    }
}

// ILU forward sweep over level l (>= 1): z = q - L z. On the last level the backward
// scaling (no upper entries there) is applied too.
template <int NRHS>
__global__ void __launch_bounds__(kBlock) g_fwd(Args a, int l, int which) {
    pdl_enter();
    const St& S = *a.st;
    if (!S.active) return;
    const double* q = which ? a.r : a.p;
    double* z = which ? a.sh : a.ph;
    const int n0 = level0_rows<KCFD_PREC_ILU0>(a);  // y = q there (not copied into z)
    int dn[NRHS];
#pragma unroll
    for (int c = 0; c < NRHS; ++c) dn[c] = which ? (S.done[c] || S.sconv[c]) : S.done[c];
    int r0, r1;
    level_range(a, l, r0, r1);
    const bool last = (l == a.nlev - 1);
    // rows from r0 rounded down to a slice boundary, so that warps and slices align
    for (int i = (r0 & ~31) + blockIdx.x * blockDim.x + threadIdx.x; i < r1; i += gridDim.x * blockDim.x) {
        if (i < r0) continue;
        const double di = last ? __ldg(a.ldi + i) : 1.0;
        double acc[NRHS];
#pragma unroll
        for (int c = 0; c < NRHS; ++c) acc[c] = q[(size_t)i * NRHS + c];
        int base, w;
        sell_row(a.L, i, base, w);
        sell_gather_fwd<NRHS>(a.L, base, w, z, q, n0, acc);
#pragma unroll
        for (int c = 0; c < NRHS; ++c)
            if (!dn[c]) z[(size_t)i * NRHS + c] = acc[c] * di;
    }
}

// ILU backward sweep over level l: z = (z - U z) / u_ii. With a single level this is
// the whole preconditioner after the level-0 copy.
template <int NRHS>
__global__ void __launch_bounds__(kBlock) g_bwd(Args a, int l, int which) {
    pdl_enter();
    const St& S = *a.st;
    if (!S.active) return;
    double* z = which ? a.sh : a.ph;
    // level 0 of a multi-level factor starts from q (y = q there, not copied into z)
    const double* y = (l == 0 && a.nlev >= 2) ? (which ? a.r : a.p) : z;
    int dn[NRHS];
#pragma unroll
    for (int c = 0; c < NRHS; ++c) dn[c] = which ? (S.done[c] || S.sconv[c]) : S.done[c];
    int r0, r1;
    level_range(a, l, r0, r1);
    for (int i = (r0 & ~31) + blockIdx.x * blockDim.x + threadIdx.x; i < r1; i += gridDim.x * blockDim.x) {
        if (i < r0) continue;
        const double di = __ldg(a.ldi + i);
        double acc[NRHS];
#pragma unroll
        for (int c = 0; c < NRHS; ++c) acc[c] = y[(size_t)i * NRHS + c];
        int base, w;
        sell_row(a.U, i, base, w);
        sell_gather<NRHS, true>(a.U, base, w, z, acc);
#pragma unroll
        for (int c = 0; c < NRHS; ++c)
            if (!dn[c]) z[(size_t)i * NRHS + c] = acc[c] * di;
    }
}

template <int NRHS, int PREC>
__global__ void __launch_bounds__(kBlock) g_spmv_v(Args a) {
    pdl_enter();
    St& S = *a.st;
    if (!S.active) return;
    const double* ph = (PREC == KCFD_PREC_NONE) ? a.p : a.ph;
    double red[NRHS];
#pragma unroll
    for (int c = 0; c < NRHS; ++c) red[c] = 0.0;
    const int n0 = level0_rows<PREC>(a);
    const int stride = gridDim.x * blockDim.x;
    for (int q0 = blockIdx.x * blockDim.x + threadIdx.x; q0 < n0 * NRHS; q0 += stride) {
        // v = p on level 0: only its dot with rhat; readers take p there
        red[q0 % NRHS] += a.rh[q0] * a.p[q0];
    }
    for (int i = (n0 & ~31) + blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += stride) {
        if (i < n0) continue;
        int base, w;
        sell_row(a.A, i, base, w);
        double rhv[NRHS], acc[NRHS];
#pragma unroll
        for (int c = 0; c < NRHS; ++c) {
            rhv[c] = a.rh[(size_t)i * NRHS + c];
            acc[c] = 0.0;
        }
        sell_gather<NRHS>(a.A, base, w, ph, acc);
#pragma unroll
        for (int c = 0; c < NRHS; ++c) {
            a.v[(size_t)i * NRHS + c] = acc[c];
            red[c] += rhv[c] * acc[c];
        }
    }
    if (last_block_sum<NRHS>(a, 1, red) && threadIdx.x == 0) {
        const bool gpu = a.stop == KCFD_STOP_GPU;
        for (int c = 0; c < NRHS; ++c) {
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
template <int NRHS, int PREC>
__global__ void __launch_bounds__(kBlock) g_s(Args a) {
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
                if (PREC == KCFD_PREC_JACOBI) D[u] = __ldg(a.dinv + i);
#pragma unroll
                for (int c = 0; c < NRHS; ++c) {
                    const size_t q = (size_t)i * NRHS + c;
                    R[u][c] = a.r[q];
                    V[u][c] = (i < n0) ? a.p[q] : a.v[q];  // v = p on level 0
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
                a.r[q] = sv;
                if (PREC == KCFD_PREC_JACOBI) a.sh[q] = D[u] * sv;
                if (PREC == KCFD_PREC_ILU0 && a.nlev == 1) a.sh[q] = sv;  // more levels: the sweeps read s
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
            const bool conv = gpu ? (sn / S.bnorm[c] < S.thr[c]) : (sn < S.thr[c]);
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
template <int NRHS, int PREC>
__global__ void __launch_bounds__(kBlock) g_spmv_t(Args a) {
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
    const double* ph = (PREC == KCFD_PREC_NONE) ? a.p : a.ph;
    const double* sh = (PREC == KCFD_PREC_NONE) ? a.r : a.sh;
    double red[2 * NRHS];
#pragma unroll
    for (int k = 0; k < 2 * NRHS; ++k) red[k] = 0.0;
    const int stride = gridDim.x * blockDim.x;
    if (any_sc) {
        for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += stride) {
#pragma unroll
            for (int c = 0; c < NRHS; ++c)
                if (sc[c]) a.x[(size_t)i * NRHS + c] += al[c] * ph[(size_t)i * NRHS + c];
        }
    }
    const int n0 = active ? level0_rows<PREC>(a) : 0;
    if (active) {
        for (int q0 = blockIdx.x * blockDim.x + threadIdx.x; q0 < n0 * NRHS; q0 += stride) {
            const int c = q0 % NRHS;
            if (dn[c]) continue;
            const double tv = a.r[q0];  // t = s on level 0 (not stored; g_xr takes s there)
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
            sv[c] = a.r[(size_t)i * NRHS + c];
            acc[c] = 0.0;
        }
        sell_gather<NRHS>(a.A, base, w, sh, acc);
#pragma unroll
        for (int c = 0; c < NRHS; ++c) {
            if (dn[c]) continue;
            a.t[(size_t)i * NRHS + c] = acc[c];
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
// and the loop condition.
template <int NRHS, int PREC>
__global__ void __launch_bounds__(kBlock) g_xr(Args a) {
    pdl_enter();
    St& S = *a.st;
    // unconditional bound on the loop, whatever the state logic does
    if (!a.eager && blockIdx.x == 0 && threadIdx.x == 0 && S.trips > a.maxiter + 2) cudaGraphSetConditional(a.cond, 0u);
    if (!S.active) return;
    // two rows per thread for one right-hand side: 48 registers, 5 resident CTAs per SM
    // (four rows: 77 registers, 3 CTAs; measured 194.5 against 191.2 us per p' iteration)
    constexpr int U = NRHS == 1 ? 2 : Ilp<NRHS>::U;
    const bool gpu = a.stop == KCFD_STOP_GPU;
    const double* ph = (PREC == KCFD_PREC_NONE) ? a.p : a.ph;
    const double* sh = (PREC == KCFD_PREC_NONE) ? a.r : a.sh;
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
        double X[U][NRHS], HP[U][NRHS], HS[U][NRHS], R[U][NRHS], T[U][NRHS], RH[U][NRHS];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int i = i0 + u * stride;
            if (i < a.n) {
#pragma unroll
                for (int c = 0; c < NRHS; ++c) {
                    const size_t q = (size_t)i * NRHS + c;
                    X[u][c] = a.x[q];
                    HP[u][c] = ph[q];
                    HS[u][c] = sh[q];
                    R[u][c] = a.r[q];
                    T[u][c] = (i < n0) ? R[u][c] : a.t[q];  // t = s on level 0
                    RH[u][c] = a.rh[q];
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
                const double rn = R[u][c] - om[c] * T[u][c];
                a.r[q] = rn;
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
        top_of_iteration<NRHS>(a, S);
        if (!a.eager) cudaGraphSetConditional(a.cond, (S.active && S.trips <= a.maxiter + 2) ? 1u : 0u);
    }
}

// Results; x = 0 for right-hand sides with b == 0 (scipy returns b), over the grid.
template <int NRHS>
__global__ void g_final(Args a) {
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
