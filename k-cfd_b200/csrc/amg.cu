// Smoothed-aggregation algebraic multigrid on the device: the 'amg' preconditioner of
// core/preconditioner.py:63-74 (pyamg's smoothed_aggregation_solver(A).aspreconditioner()
// in the reference; pyamg is an optional dependency of the reference and absent here).
// The method is Vanek, Mandel and Brezina, "Algebraic multigrid by smoothed aggregation
// for second and fourth order elliptic problems", Computing 56 (1996):
//
//   aggregates  three greedy passes in row order over the matrix graph (every stored
//               off-diagonal entry is a link): (1) a row whose neighbours are all free
//               starts an aggregate with them; (2) a free row joins the pass-1
//               aggregate holding most of its neighbours (first met on a tie); (3) a row
//               still free starts an aggregate with its free neighbours;
//   P           (I - omega D^-1 A) T, T the aggregates' 0/1 indicator; omega = 4 / (3 rho),
//               rho = max_i sum_j |a_ij| / |a_ii| on level 0 (Gershgorin), a power
//               iteration on D^-1 A on the coarser levels;
//   A_c         P^T (A P) (Galerkin);
//   cycle       V(1,1), damped Jacobi with the level's omega, from a zero guess:
//               x = omega D^-1 b; r = b - A x; x += P V(P^T r); y = x + omega D^-1 (b - A x);
//               the coarsest level (at most kDenseMax rows) is solved by its dense inverse.
//
// The aggregates and every sparsity pattern (P, P^T, A P, P^T A P) depend on the
// pattern only; they are built once on the host (kcfd_amg_create), with, for every
// entry of a product, the list of its elementary products (index pairs into the two
// factors' values, in row-major order of the factors). A set-up (kcfd_amg_setup, every
// outer iteration of a SIMPLE solve) only refreshes values on the device: one thread
// sums one entry's list in that fixed order, so the hierarchy is deterministic, has
// the parallelism of the output (thousands of threads even on the coarsest products)
// and uses no atomics but one max (order-free).
//
// Layout: each level's operator A_l and its smoother matrix W_l = omega A_l D^-1 are kept
// in sliced ELL with 32-row slices (a warp reads 32 consecutive values per load), P and
// P^T in CSR. MIXED mode stores the V-cycle's values and vectors in FP32 and does its
// arithmetic in FP64 (loads widened, sums in double); the set-up is FP64 throughout.
#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "amg.h"
#include "kcfd_common.h"
#include "team.cuh"

namespace kcfd {
namespace amg {

constexpr int kMaxLevels = 16;
constexpr int kDenseMax = 256;   // largest coarsest level solved by its dense inverse
constexpr int kRedGrid = 1024;   // blocks of the power-iteration reductions (at most)
constexpr int kGjSmemMax = 200 * 1024;  // dynamic shared memory of the Gauss-Jordan kernel (at most)

struct Level {
    int n = 0, nnz = 0, nc = 0;                 // rows, entries, rows of the next level
    int *ip = nullptr, *ix = nullptr, *dslot = nullptr;
    double* a64 = nullptr;                      // level >= 1: Galerkin values (level 0: the caller's)
    double* dinv = nullptr;
    // sliced ELL of A_l: slot -> CSR entry (-1 padding)
    int *soff = nullptr, *scol = nullptr, *ssrc = nullptr;
    int64_t slots = 0;
    void *sA = nullptr, *sW = nullptr, *sd = nullptr;
    // transfer to level + 1
    int pnnz = 0;
    int *pip = nullptr, *pix = nullptr, *pdiag = nullptr;
    int *prow = nullptr, *plp = nullptr, *pla = nullptr;  // P entry -> its row; its A entries [plp, plp+1) in pla
    int rlanes = 1;                                        // lanes per coarse row of the restriction
    int slanes = 1;                                        // lanes per row of the smoothing kernels
    double* p64 = nullptr;
    void* pV = nullptr;
    int *rip = nullptr, *rix = nullptr, *rsrc = nullptr;
    double* r64 = nullptr;
    void* rV = nullptr;
    int* bip = nullptr;
    int64_t bnnz = 0;
    double* b64 = nullptr;
    int64_t* bptr = nullptr;                    // B entry -> its products [bptr, bptr+1) in (bx, bp)
    int *bx = nullptr, *bp = nullptr;           // A-entry, P-entry index of each product
    int64_t* cptr = nullptr;                    // C entry -> its products in (cr, cb)
    int *cr = nullptr, *cb = nullptr;           // R-entry, B-entry index of each product
    // cycle vectors (value type of the mode)
    void *x = nullptr, *r = nullptr, *y = nullptr, *b = nullptr;
    std::vector<int> agg;                       // host copy, for export
};

}  // namespace amg
}  // namespace kcfd

struct kcfd_amg {
    kcfd_amg_opts_t o;
    int mixed = 0;
    int sm_count = 0;
    int nlev = 0;
    kcfd::amg::Level lv[kcfd::amg::kMaxLevels];
    double* omega = nullptr;                    // [kMaxLevels]
    unsigned long long* rmax = nullptr;         // [kMaxLevels] Gershgorin ratio bits
    double* nrm2 = nullptr;                     // [2] power-iteration norms (ping-pong)
    double* part = nullptr;                     // [kRedGrid] block partials
    unsigned* cnt = nullptr;                    // arrival counter of the reductions
    double* powv[2] = {nullptr, nullptr};
    double* dense = nullptr;                    // coarsest: [nc][nc] FP64 work
    double* dinvm = nullptr;                    // coarsest: [nc][nc] FP64 inverse
    void* cinv = nullptr;                       // coarsest inverse in the cycle's value type
    int gj_smem = 0;                            // dynamic shared bytes of the Gauss-Jordan kernel (0: global)
    int64_t bytes = 0;
};

namespace kcfd {
namespace amg {
namespace {

__device__ __forceinline__ void pdl_enter() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

__device__ __forceinline__ bool inactive(const int* active) { return active && *(volatile const int*)active == 0; }

// acc = sum_k val[k] x[col[k]] over row i of a sliced-ELL matrix (row order), with the
// row's columns and values loaded in batches of 8 before the gathers of x.
template <typename V, typename T>
__device__ __forceinline__ double sell_row_dot(const int* __restrict__ off, const int* __restrict__ col,
                                               const V* __restrict__ val, int i, const T* x) {
    const int sl = i >> 5;
    const int o0 = __ldg(off + sl), o1 = __ldg(off + sl + 1);
    const int base = o0 + (i & 31), w = (o1 - o0) >> 5;
    constexpr int B = 8;
    double acc = 0.0;
    for (int k0 = 0; k0 < w; k0 += B) {
        int jj[B];
        double vv[B];
#pragma unroll
        for (int u = 0; u < B; ++u) {
            const bool in = k0 + u < w;
            const int slot = base + (k0 + u) * 32;
            jj[u] = in ? __ldg(col + slot) : -1;
            vv[u] = in ? (double)__ldg(val + slot) : 0.0;
        }
        double xv[B];
#pragma unroll
        for (int u = 0; u < B; ++u) xv[u] = jj[u] >= 0 ? (double)x[jj[u]] : 0.0;
#pragma unroll
        for (int u = 0; u < B; ++u)
            if (jj[u] >= 0) acc += vv[u] * xv[u];
    }
    return acc;
}

// acc = sum over CSR row [k0, k1) of val[k] x[col[k]], entries loaded in batches of 8.
template <typename V, typename T>
__device__ __forceinline__ double csr_row_dot(int k0, int k1, const int* __restrict__ col, const V* __restrict__ val,
                                              const T* x) {
    constexpr int B = 8;
    double acc = 0.0;
    for (int k = k0; k < k1; k += B) {
        int jj[B];
        double vv[B];
#pragma unroll
        for (int u = 0; u < B; ++u) {
            const bool in = k + u < k1;
            jj[u] = in ? __ldg(col + k + u) : -1;
            vv[u] = in ? (double)__ldg(val + k + u) : 0.0;
        }
        double xv[B];
#pragma unroll
        for (int u = 0; u < B; ++u) xv[u] = jj[u] >= 0 ? (double)x[jj[u]] : 0.0;
#pragma unroll
        for (int u = 0; u < B; ++u)
            if (jj[u] >= 0) acc += vv[u] * xv[u];
    }
    return acc;
}

// Lane q of the L lanes sharing row i of a sliced-ELL matrix: the partial sum over the
// row's entries q, q + L, ... (L = 1: the whole row, entries loaded in batches of 8).
template <int L, typename V, typename T>
__device__ __forceinline__ double sell_row_part(const int* __restrict__ off, const int* __restrict__ col,
                                                const V* __restrict__ val, int i, const T* x, int q) {
    if (L == 1) return sell_row_dot(off, col, val, i, x);
    const int sl = i >> 5;
    const int o0 = __ldg(off + sl), o1 = __ldg(off + sl + 1);
    const int base = o0 + (i & 31), w = (o1 - o0) >> 5;
    double acc = 0.0;
    for (int k = q; k < w; k += L) {
        const int j = __ldg(col + base + 32 * k);
        if (j >= 0) acc += (double)__ldg(val + base + 32 * k) * (double)x[j];
    }
    return acc;
}

// Rows of a level handled by groups of L lanes (the small coarse levels, whose rows are
// long and few, take several lanes per row so that more loads are in flight): f(i,
// partial sum of row i) for each row, called on every lane with i < n after the L
// partials are combined by a fixed xor-shuffle tree (lane q == 0 writes). The trip
// count depends on the warp's first group only, so every lane of a warp runs it.
template <int L, typename F>
__device__ __forceinline__ void rows_by_lanes(int n, F f) {
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    const int q = tid & (L - 1);
    const int groups = (gridDim.x * blockDim.x) / L;
    const int g = tid / L, g0 = (tid & ~31) / L;
    for (int t = 0; g0 + t * groups < n; ++t) {
        const int i = g + t * groups;
        f(i, q);
    }
}

// ------------------------------------------------------------------ cycle kernels --
// Pre-smoothing from a zero guess and the residual: x = sd b, r = b - W b (W = omega A D^-1).
template <typename V, typename TI, int L = 1>
__global__ void __launch_bounds__(256) k_pre(int n, const int* __restrict__ off, const int* __restrict__ col,
                                             const V* __restrict__ W, const V* __restrict__ sd, const TI* b, V* x,
                                             V* r, const int* active) {
    pdl_enter();
    if (inactive(active)) return;
    rows_by_lanes<L>(n, [&](int i, int q) {
        double wb = i < n ? sell_row_part<L>(off, col, W, i, b, q) : 0.0;
#pragma unroll
        for (int o = L / 2; o > 0; o >>= 1) wb += __shfl_xor_sync(0xffffffffu, wb, o);
        if (i < n && q == 0) {
            const double bi = (double)b[i];
            x[i] = (V)((double)__ldg(sd + i) * bi);
            r[i] = (V)(bi - wb);
        }
    });
}

// Restriction bc = P^T r (P^T in CSR). A coarse row gathers the fine rows of its
// smoothed aggregate (about 24 on 3D hexes), so L lanes share a row: lane q takes the
// entries q, q + L, ... (the lanes of a row read consecutive entries), then a fixed
// xor-shuffle tree sums the L partials.
template <typename V, int L>
__global__ void __launch_bounds__(256) k_restrict(int nc, const int* __restrict__ rip, const int* __restrict__ rix,
                                                  const V* __restrict__ R, const V* r, V* bc, const int* active) {
    pdl_enter();
    if (inactive(active)) return;
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    const int q = threadIdx.x & (L - 1);
    const int groups = (gridDim.x * blockDim.x) / L;
    const int g = tid / L, g0 = (tid & ~31) / L;  // this lane's row group, the warp's first
    // the trip count depends on the warp's first group only, so every lane of a warp
    // runs every trip (the shuffles need them all)
    for (int t = 0; g0 + t * groups < nc; ++t) {
        const int I = g + t * groups;
        const bool row = I < nc;
        double acc = 0.0;
        if (row) {
            // four entries per lane in flight: columns and values first, then the gathers
            const int k0 = __ldg(rip + I), k1 = __ldg(rip + I + 1);
            for (int k = k0 + q; k < k1; k += 4 * L) {
                int jj[4];
                double vv[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const bool in = k + u * L < k1;
                    jj[u] = in ? __ldg(rix + k + u * L) : -1;
                    vv[u] = in ? (double)__ldg(R + k + u * L) : 0.0;
                }
                double xv[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) xv[u] = jj[u] >= 0 ? (double)r[jj[u]] : 0.0;
#pragma unroll
                for (int u = 0; u < 4; ++u)
                    if (jj[u] >= 0) acc += vv[u] * xv[u];
            }
        }
#pragma unroll
        for (int o = L / 2; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (row && q == 0) bc[I] = (V)acc;
    }
}

// Coarsest level: y = C b with C the dense inverse, one warp per row.
template <typename V, typename TI, typename TO>
__global__ void __launch_bounds__(256) k_coarse(int nc, const V* __restrict__ C, const TI* b, TO* y,
                                                const int* active) {
    pdl_enter();
    if (inactive(active)) return;
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < nc; i += warps) {
        double acc = 0.0;
        for (int j = lane; j < nc; j += 32) acc += (double)__ldg(C + (size_t)i * nc + j) * (double)b[j];
        acc = warp_sum(acc);
        if (lane == 0) y[i] = (TO)acc;
    }
}

// Prolongation x += P y (P in CSR, one thread per fine row).
template <typename V>
__global__ void __launch_bounds__(256) k_prolong(int n, const int* __restrict__ pip, const int* __restrict__ pix,
                                                 const V* __restrict__ P, const V* yc, V* x, const int* active) {
    pdl_enter();
    if (inactive(active)) return;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        x[i] = (V)((double)x[i] + csr_row_dot(__ldg(pip + i), __ldg(pip + i + 1), pix, P, yc));
}

// Post-smoothing: y = x + sd (b - A x).
template <typename V, typename TI, typename TO, int L = 1>
__global__ void __launch_bounds__(256) k_post(int n, const int* __restrict__ off, const int* __restrict__ col,
                                              const V* __restrict__ A, const V* __restrict__ sd, const TI* b,
                                              const V* x, TO* y, const int* active) {
    pdl_enter();
    if (inactive(active)) return;
    rows_by_lanes<L>(n, [&](int i, int q) {
        double ax = i < n ? sell_row_part<L>(off, col, A, i, x, q) : 0.0;
#pragma unroll
        for (int o = L / 2; o > 0; o >>= 1) ax += __shfl_xor_sync(0xffffffffu, ax, o);
        if (i < n && q == 0) y[i] = (TO)((double)x[i] + (double)__ldg(sd + i) * ((double)b[i] - ax));
    });
}

// ------------------------------------------------------------------ set-up kernels --
// dinv (0 where |a_ii| <= 1e-30, as the Jacobi preconditioner) and, when rmax is given,
// the largest Gershgorin ratio sum_j |a_ij| |dinv_i| (a max: the order does not matter).
__global__ void k_diag(int n, const int* __restrict__ ip, const double* __restrict__ a, const int* __restrict__ dslot,
                       double* __restrict__ dinv, unsigned long long* rmax) {
    double m = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double d = a[dslot[i]];
        const double di = fabs(d) > 1e-30 ? 1.0 / d : 0.0;
        dinv[i] = di;
        if (rmax) {
            double s = 0.0;
            for (int k = ip[i]; k < ip[i + 1]; ++k) s += fabs(a[k]);
            m = fmax(m, s * fabs(di));
        }
    }
    if (rmax) {
        for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
        if ((threadIdx.x & 31) == 0) atomicMax(rmax, (unsigned long long)__double_as_longlong(m));
    }
}

__global__ void k_omega_gersh(const unsigned long long* rmax, double* omega) {
    const double r = __longlong_as_double((long long)*rmax);
    *omega = r > 1e-300 ? (4.0 / 3.0) / r : 4.0 / 3.0;
}

// Fixed-order sum of one value per thread over the grid: block partial, the last block
// to arrive sums the partials in index order and writes *out.
__device__ __forceinline__ void grid_sum_to(double v, double* part, unsigned* cnt, double* out) {
    __shared__ double sm[32];
    __shared__ int last;
    double a[1] = {v};
    block_sum<1>(a, sm);
    if (threadIdx.x == 0) {
        part[blockIdx.x] = a[0];
        __threadfence();
        last = atomicAdd(cnt, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    double t = 0.0;
    for (int j = threadIdx.x; j < (int)gridDim.x; j += blockDim.x) t += __ldcg(part + j);
    a[0] = t;
    block_sum<1>(a, sm);
    if (threadIdx.x == 0) {
        *out = a[0];
        *cnt = 0u;
    }
}

// Start vector of the power iteration: v_i = 0.5 + ((i * 2654435761) mod 2^32 >> 22) / 1024.
__global__ void k_pow_init(int n, double* v, double* part, unsigned* cnt, double* nrm2) {
    double s = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const unsigned h = (unsigned)i * 2654435761u;
        const double x = 0.5 + (double)(h >> 22) / 1024.0;
        v[i] = x;
        s += x * x;
    }
    grid_sum_to(s, part, cnt, nrm2);
}

// w = D^-1 A v / ||v||, ||w||^2 (A from the level's sliced-ELL copy).
template <typename V>
__global__ void k_pow_step(int n, const int* __restrict__ off, const int* __restrict__ col, const V* __restrict__ sA,
                           const double* __restrict__ dinv, const double* vin, const double* nrm2_in, double* vout,
                           double* part, unsigned* cnt, double* nrm2_out) {
    const double sc = 1.0 / sqrt(*nrm2_in);
    double s = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double acc = sell_row_dot(off, col, sA, i, vin);
        const double w = dinv[i] * (acc * sc);
        vout[i] = w;
        s += w * w;
    }
    grid_sum_to(s, part, cnt, nrm2_out);
}

__global__ void k_omega_pow(const double* nrm2, double* omega) {
    const double lam = sqrt(*nrm2);
    *omega = lam > 1e-300 ? (4.0 / 3.0) / lam : 4.0 / 3.0;
}

// The level's operator A in sliced ELL (0 in the padding).
template <typename V>
__global__ void k_sell_a(int64_t slots, const int* __restrict__ src, const double* __restrict__ a, V* sA) {
    for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < slots; s += (int64_t)gridDim.x * blockDim.x) {
        const int k = src[s];
        sA[s] = k >= 0 ? (V)a[k] : (V)0;
    }
}

// The smoother's W = omega A D^-1 in sliced ELL.
template <typename V>
__global__ void k_sell_w(int64_t slots, const int* __restrict__ src, const int* __restrict__ scol,
                         const double* __restrict__ a, const double* __restrict__ dinv, const double* __restrict__ omega,
                         V* sW) {
    const double w = *omega;
    for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < slots; s += (int64_t)gridDim.x * blockDim.x) {
        const int k = src[s];
        sW[s] = k >= 0 ? (V)(w * a[k] * dinv[scol[s]]) : (V)0;
    }
}

template <typename V>
__global__ void k_sd(int n, const double* __restrict__ dinv, const double* __restrict__ omega, V* sd) {
    const double w = *omega;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) sd[i] = (V)(w * dinv[i]);
}

// P = T - omega D^-1 (A T), one thread per entry (i, J) of P: s = the sum of row i's
// entries whose column lies in aggregate J (the entry's list, in row order), then
// P_iJ = [J = agg(i)] - omega dinv_i s.
template <typename V>
__global__ void k_pvals(int pnnz, const int* __restrict__ prow, const int* __restrict__ pdiag,
                        const int* __restrict__ plp, const int* __restrict__ pla, const double* __restrict__ a,
                        const double* __restrict__ dinv, const double* __restrict__ omega, double* p64, V* pV) {
    const double w = *omega;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < pnnz; e += gridDim.x * blockDim.x) {
        const int i = prow[e];
        double sum = 0.0;
        for (int t = plp[e]; t < plp[e + 1]; ++t) sum += a[pla[t]];
        const double p = (e == pdiag[i] ? 1.0 : 0.0) - (w * dinv[i]) * sum;
        p64[e] = p;
        pV[e] = (V)p;
    }
}

template <typename V>
__global__ void k_gather(int m, const int* __restrict__ src, const double* __restrict__ in, double* out64, V* outV) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < m; k += gridDim.x * blockDim.x) {
        const double v = in[src[k]];
        out64[k] = v;
        outV[k] = (V)v;
    }
}

// One entry of a sparse product per thread: out[s] = sum over its products t of
// x[xi[t]] y[yi[t]], in list order (B = A P: x = A, y = P; A_c = P^T B: x = R, y = B).
__global__ void k_product(int64_t m, const int64_t* __restrict__ ptr, const int* __restrict__ xi,
                          const int* __restrict__ yi, const double* __restrict__ x, const double* __restrict__ y,
                          double* __restrict__ out) {
    for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < m; s += (int64_t)gridDim.x * blockDim.x) {
        const int64_t t0 = ptr[s], t1 = ptr[s + 1];
        double acc = 0.0;
        int64_t t = t0;
        for (; t + 4 <= t1; t += 4) {
            int xa[4], ya[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                xa[u] = __ldg(xi + t + u);
                ya[u] = __ldg(yi + t + u);
            }
            double xv[4], yv[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                xv[u] = __ldg(x + xa[u]);
                yv[u] = __ldg(y + ya[u]);
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) acc += xv[u] * yv[u];
        }
        for (; t < t1; ++t) acc += __ldg(x + __ldg(xi + t)) * __ldg(y + __ldg(yi + t));
        out[s] = acc;
    }
}

// Coarsest level: the dense matrix, then its inverse by Gauss-Jordan elimination with
// partial pivoting in one CTA. A pivot below 1e-13 of the largest entry of its column
// (in the matrix before elimination) drops its unknown (row and column of the inverse
// set to zero), so a singular coarsest operator still gives a bounded cycle; the
// tolerance is per column so that one huge entry (a row pinned by a large diagonal)
// does not drop every other unknown.
__global__ void k_dense(int nc, const int* __restrict__ ip, const int* __restrict__ ix, const double* __restrict__ a,
                        double* M) {
    for (int t = threadIdx.x; t < nc * nc; t += blockDim.x) M[t] = 0.0;
    __syncthreads();
    for (int i = threadIdx.x; i < nc; i += blockDim.x)
        for (int k = ip[i]; k < ip[i + 1]; ++k) M[(size_t)i * nc + ix[k]] += a[k];
}

// When `smem` is set the matrix and its inverse live in dynamic shared memory (2 nc^2
// doubles): every elimination step then stays on the SM. Warp w of the block owns rows
// w, w + 32, ... and lane l columns l, l + 32, ... of [M | Inv], so no thread divides
// an index; warp 0 alone finds the pivot. A step is the pivot search, the row swap,
// the staging of the scaled pivot row and the pivot column, and the elimination.
template <typename V>
__global__ void __launch_bounds__(1024) k_gj(int nc, double* Mg, double* Invg, V* C, int smem) {
    extern __shared__ double dyn[];
    double* M = smem ? dyn : Mg;
    double* Inv = smem ? dyn + (size_t)nc * nc : Invg;
    __shared__ double prow[2 * kDenseMax];   // the scaled pivot row of [M | Inv]
    __shared__ double fcol[kDenseMax];       // the pivot column before the step
    __shared__ int drop[kDenseMax];
    __shared__ double ctol[kDenseMax];       // drop tolerance of each column
    __shared__ int piv_s;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5, nty = blockDim.x >> 5;
    const int W = 2 * nc;
    for (int i = ty; i < nc; i += nty)
        for (int j = tx; j < nc; j += 32) {
            const double v = Mg[(size_t)i * nc + j];
            if (smem) M[(size_t)i * nc + j] = v;
            Inv[(size_t)i * nc + j] = (i == j) ? 1.0 : 0.0;
        }
    for (int t = threadIdx.x; t < nc; t += blockDim.x) {
        drop[t] = 0;
        double cm = 0.0;
        for (int i = 0; i < nc; ++i) cm = fmax(cm, fabs(Mg[(size_t)i * nc + t]));
        ctol[t] = 1e-13 * cm;
    }
    __syncthreads();
    for (int k = 0; k < nc; ++k) {
        if (ty == 0) {
            // pivot: the largest |M[i][k]| over i >= k, the smallest i on ties
            double bv = -1.0;
            int bi = nc;
            for (int i = k + tx; i < nc; i += 32) {
                const double v = fabs(M[(size_t)i * nc + k]);
                if (v > bv) {
                    bv = v;
                    bi = i;
                }
            }
            for (int o = 16; o > 0; o >>= 1) {
                const double ov = __shfl_xor_sync(0xffffffffu, bv, o);
                const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
                if (ov > bv || (ov == bv && oi < bi)) {
                    bv = ov;
                    bi = oi;
                }
            }
            if (tx == 0) {
                piv_s = (bv > ctol[k]) ? bi : -1;
                if (piv_s < 0) drop[k] = 1;
            }
        }
        __syncthreads();
        const int p = piv_s;
        if (p < 0) continue;  // a dropped unknown: its inverse row and column are cleared below
        if (p != k)
            for (int j = threadIdx.x; j < W; j += blockDim.x) {
                double* A = j < nc ? M : Inv;
                const int c = j < nc ? j : j - nc;
                const double t = A[(size_t)k * nc + c];
                A[(size_t)k * nc + c] = A[(size_t)p * nc + c];
                A[(size_t)p * nc + c] = t;
            }
        __syncthreads();
        const double inv_p = 1.0 / M[(size_t)k * nc + k];
        for (int j = threadIdx.x; j < W; j += blockDim.x)
            prow[j] = (j < nc ? M[(size_t)k * nc + j] : Inv[(size_t)k * nc + j - nc]) * inv_p;
        for (int i = threadIdx.x; i < nc; i += blockDim.x) fcol[i] = M[(size_t)i * nc + k];
        __syncthreads();
        // entries whose pivot-row factor is zero are left alone: the eliminated columns of M
        // (j < k) and the columns of Inv that no step has touched yet, about half of [M | Inv]
        for (int i = ty; i < nc; i += nty) {
            const double f = fcol[i];
            if (i != k && f == 0.0) continue;
            for (int j = tx; j < W; j += 32) {
                double* A = j < nc ? M : Inv;
                const size_t q = (size_t)i * nc + (j < nc ? j : j - nc);
                const double pj = prow[j];
                if (i == k) A[q] = pj;
                else if (pj != 0.0) A[q] -= f * pj;
            }
        }
        __syncthreads();
    }
    for (int i = ty; i < nc; i += nty)
        for (int j = tx; j < nc; j += 32) {
            const size_t q = (size_t)i * nc + j;
            const double v = (drop[i] || drop[j]) ? 0.0 : Inv[q];
            Invg[q] = v;
            C[q] = (V)v;
        }
}

// ---------------------------------------------------------------- host: patterns --
// Host threads for the per-row passes of the set-up: KCFD_HOST_THREADS when set (a
// positive count), else the hardware's, at most 16.
int host_threads() {
    static const int t = [] {
        unsigned h = std::thread::hardware_concurrency();
        if (const char* e = std::getenv("KCFD_HOST_THREADS")) {
            const long v = std::strtol(e, nullptr, 10);
            if (v > 0) h = (unsigned)std::min(v, 1024L);
        }
        return (int)std::min(16u, std::max(1u, h));
    }();
    return t;
}

// fn(chunk, begin, end) over contiguous row ranges of [0, n) (at least 4096 rows each,
// one per host thread at most). Every row is computed by the same code whatever thread
// runs it, so the results do not depend on the thread count.
template <class Fn>
void for_row_chunks(int n, Fn&& fn) {
    const int chunks = (int)std::max<int64_t>(1, std::min<int64_t>(host_threads(), n / 4096));
    auto run = [&](int t) { fn(t, (int)((int64_t)n * t / chunks), (int)((int64_t)n * (t + 1) / chunks)); };
    std::vector<std::thread> pool;
    int t = 1;
    try {
        for (; t < chunks; ++t) pool.emplace_back(run, t);
    } catch (...) {
    }
    for (int u = t; u < chunks; ++u) run(u);
    run(0);
    for (auto& th : pool) th.join();
}

struct HostCsr {
    int n = 0, m = 0;
    std::vector<int> ip, ix;
};

// Aggregates of the rows of A (three greedy passes; every off-diagonal entry is a link).
int aggregate(const HostCsr& A, std::vector<int>& agg) {
    const int n = A.n;
    agg.assign(n, -1);
    int na = 0;
    for (int i = 0; i < n; ++i) {
        if (agg[i] >= 0) continue;
        bool has = false, free = true;
        for (int k = A.ip[i]; k < A.ip[i + 1]; ++k) {
            const int j = A.ix[k];
            if (j == i) continue;
            has = true;
            if (agg[j] >= 0) {
                free = false;
                break;
            }
        }
        if (!has || !free) continue;
        agg[i] = na;
        for (int k = A.ip[i]; k < A.ip[i + 1]; ++k)
            if (A.ix[k] != i) agg[A.ix[k]] = na;
        ++na;
    }
    const std::vector<int> p1 = agg;
    std::vector<int> cand, cnt;
    for (int i = 0; i < n; ++i) {
        if (agg[i] >= 0) continue;
        cand.clear();
        cnt.clear();
        for (int k = A.ip[i]; k < A.ip[i + 1]; ++k) {
            const int j = A.ix[k];
            if (j == i || p1[j] < 0) continue;
            const auto it = std::find(cand.begin(), cand.end(), p1[j]);
            if (it == cand.end()) {
                cand.push_back(p1[j]);
                cnt.push_back(1);
            } else {
                cnt[it - cand.begin()]++;
            }
        }
        if (cand.empty()) continue;
        size_t best = 0;
        for (size_t q = 1; q < cand.size(); ++q)
            if (cnt[q] > cnt[best]) best = q;
        agg[i] = cand[best];
    }
    for (int i = 0; i < n; ++i) {
        if (agg[i] >= 0) continue;
        agg[i] = na;
        for (int k = A.ip[i]; k < A.ip[i + 1]; ++k) {
            const int j = A.ix[k];
            if (j != i && agg[j] < 0) agg[j] = na;
        }
        ++na;
    }
    return na;
}

inline int pos_in(const int* b, const int* e, int v) { return (int)(std::lower_bound(b, e, v) - b); }

struct Transfer {
    HostCsr P, R, B, C;
    std::vector<int> pdiag, pmap, rsrc, bx, bp, cr, cb;
    std::vector<int64_t> bptr, cptr;
};

// Product lists of Z = X Y for a given pattern of Z: for each entry of Z, the (X entry,
// Y entry) pairs that add into it, in row-major order of X then Y. Two passes (count,
// fill), so nothing of the size of the list is held twice.
bool product_lists(const HostCsr& X, const HostCsr& Y, const HostCsr& Z, std::vector<int64_t>& ptr,
                   std::vector<int>& xi, std::vector<int>& yi) {
    const int64_t zn = Z.ip[Z.n];
    ptr.assign(zn + 1, 0);
    std::vector<int64_t> fill;
    for (int pass = 0; pass < 2; ++pass) {
        if (pass == 1) {
            for (int64_t s = 0; s < zn; ++s) ptr[s + 1] += ptr[s];
            if (ptr[zn] > INT32_MAX) return false;
            xi.assign(ptr[zn], 0);
            yi.assign(ptr[zn], 0);
            fill.assign(ptr.begin(), ptr.end() - 1);
        }
        // a row of Z only touches its own entries: rows in parallel
        for_row_chunks(X.n, [&](int, int r0, int r1) {
            for (int i = r0; i < r1; ++i) {
                const int* rb = Z.ix.data() + Z.ip[i];
                const int* re = Z.ix.data() + Z.ip[i + 1];
                for (int k = X.ip[i]; k < X.ip[i + 1]; ++k) {
                    const int j = X.ix[k];
                    for (int e = Y.ip[j]; e < Y.ip[j + 1]; ++e) {
                        const int64_t s = Z.ip[i] + pos_in(rb, re, Y.ix[e]);
                        if (pass == 0) {
                            ptr[s + 1]++;
                        } else {
                            const int64_t t = fill[s]++;
                            xi[t] = k;
                            yi[t] = e;
                        }
                    }
                }
            }
        });
    }
    return true;
}

// Patterns of P, R = P^T, B = A P and C = R B, with the slot maps of the value kernels.
bool build_transfer(const HostCsr& A, const std::vector<int>& agg, int na, Transfer& t) {
    const int n = A.n;
    HostCsr& P = t.P;
    P.n = n;
    P.m = na;
    P.ip.assign(n + 1, 0);
    P.ix.clear();
    t.pdiag.assign(n, -1);
    t.pmap.assign(A.ip[n], -1);
    std::vector<int> row;
    for (int i = 0; i < n; ++i) {
        row.clear();
        for (int k = A.ip[i]; k < A.ip[i + 1]; ++k) row.push_back(agg[A.ix[k]]);
        std::sort(row.begin(), row.end());
        row.erase(std::unique(row.begin(), row.end()), row.end());
        const int base = (int)P.ix.size();
        P.ix.insert(P.ix.end(), row.begin(), row.end());
        P.ip[i + 1] = (int)P.ix.size();
        const int* rb = P.ix.data() + base;
        const int* re = P.ix.data() + P.ix.size();
        for (int k = A.ip[i]; k < A.ip[i + 1]; ++k) t.pmap[k] = base + pos_in(rb, re, agg[A.ix[k]]);
        const int d = pos_in(rb, re, agg[i]);
        if (d >= (int)row.size() || row[d] != agg[i]) return false;  // no diagonal entry
        t.pdiag[i] = base + d;
    }
    // R = P^T (rows of each column in ascending fine-row order)
    HostCsr& R = t.R;
    R.n = na;
    R.m = n;
    R.ip.assign(na + 1, 0);
    for (int e = 0; e < P.ip[n]; ++e) R.ip[P.ix[e] + 1]++;
    for (int I = 0; I < na; ++I) R.ip[I + 1] += R.ip[I];
    R.ix.assign(P.ip[n], 0);
    t.rsrc.assign(P.ip[n], 0);
    {
        std::vector<int> fill(R.ip.begin(), R.ip.end() - 1);
        for (int i = 0; i < n; ++i)
            for (int e = P.ip[i]; e < P.ip[i + 1]; ++e) {
                const int s = fill[P.ix[e]]++;
                R.ix[s] = i;
                t.rsrc[s] = e;
            }
    }
    // patterns of B = A P and C = R B (row i: the union of the rows it combines)
    auto product_pattern = [&](const HostCsr& X, const HostCsr& Y, HostCsr& Z) {
        Z.n = X.n;
        Z.m = Y.m;
        Z.ip.assign(X.n + 1, 0);
        // rows in parallel into per-chunk buffers, then concatenated in chunk order
        std::vector<std::vector<int>> part(host_threads());
        for_row_chunks(X.n, [&](int c, int r0, int r1) {
            std::vector<int> rw;
            std::vector<int>& out = part[c];
            for (int i = r0; i < r1; ++i) {
                rw.clear();
                for (int k = X.ip[i]; k < X.ip[i + 1]; ++k) {
                    const int j = X.ix[k];
                    rw.insert(rw.end(), Y.ix.begin() + Y.ip[j], Y.ix.begin() + Y.ip[j + 1]);
                }
                std::sort(rw.begin(), rw.end());
                rw.erase(std::unique(rw.begin(), rw.end()), rw.end());
                Z.ip[i + 1] = (int)rw.size();
                out.insert(out.end(), rw.begin(), rw.end());
            }
        });
        int64_t tot = 0;
        for (int i = 0; i < X.n; ++i) {
            tot += Z.ip[i + 1];
            if (tot > INT32_MAX) return false;
            Z.ip[i + 1] = (int)tot;
        }
        Z.ix.clear();
        Z.ix.reserve(tot);
        for (auto& v : part) {
            Z.ix.insert(Z.ix.end(), v.begin(), v.end());
            std::vector<int>().swap(v);
        }
        return true;
    };
    return product_pattern(A, P, t.B) && product_lists(A, P, t.B, t.bptr, t.bx, t.bp) &&
           product_pattern(R, t.B, t.C) && product_lists(R, t.B, t.C, t.cptr, t.cr, t.cb);
}

// Sliced ELL (32-row slices) of a CSR pattern: off[slice], col[slot], src[slot] (the CSR
// entry of the slot, -1 for padding); entries keep their row order.
bool make_sell(const HostCsr& A, std::vector<int>& off, std::vector<int>& col, std::vector<int>& src) {
    const int n = A.n, ns = (n + 31) / 32;
    off.assign(ns + 1, 0);
    int64_t tot = 0;
    for (int s = 0; s < ns; ++s) {
        int w = 0;
        for (int i = 32 * s; i < std::min(n, 32 * s + 32); ++i) w = std::max(w, A.ip[i + 1] - A.ip[i]);
        off[s] = (int)tot;
        tot += 32LL * w;
        if (tot > INT32_MAX) return false;
    }
    off[ns] = (int)tot;
    col.assign(tot, -1);
    src.assign(tot, -1);
    for (int i = 0; i < n; ++i)
        for (int k = A.ip[i]; k < A.ip[i + 1]; ++k) {
            const int64_t slot = off[i >> 5] + 32LL * (k - A.ip[i]) + (i & 31);
            col[slot] = A.ix[k];
            src[slot] = k;
        }
    return true;
}

template <typename T>
bool up(kcfd_amg* h, T** dst, const std::vector<T>& v) {
    const size_t bytes = std::max<size_t>(v.size(), 1) * sizeof(T);
    if (cudaMalloc(dst, bytes) != cudaSuccess) return false;
    h->bytes += (int64_t)bytes;
    return v.empty() || cudaMemcpy(*dst, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice) == cudaSuccess;
}

bool alloc(kcfd_amg* h, void** dst, size_t bytes) {
    bytes = std::max<size_t>(bytes, 8);
    if (cudaMalloc(dst, bytes) != cudaSuccess) return false;
    h->bytes += (int64_t)bytes;
    return true;
}

void free_amg(kcfd_amg* h) {
    if (!h) return;
    for (int l = 0; l < kMaxLevels; ++l) {
        Level& L = h->lv[l];
        void* ps[] = {L.ip, L.ix, L.dslot, L.a64, L.dinv, L.soff, L.scol, L.ssrc, L.sA, L.sW, L.sd, L.pip, L.pix,
                      L.pdiag, L.prow, L.plp, L.pla, L.p64, L.pV, L.rip, L.rix, L.rsrc, L.r64, L.rV, L.bip, L.b64, L.bptr,
                      L.bx, L.bp, L.cptr, L.cr, L.cb, L.x, L.r, L.y, L.b};
        for (void* p : ps)
            if (p) cudaFree(p);
    }
    void* ps[] = {h->omega, h->rmax, h->nrm2, h->part, h->cnt, h->powv[0], h->powv[1], h->dense, h->dinvm, h->cinv};
    for (void* p : ps)
        if (p) cudaFree(p);
    delete h;
}

int grid_for(const kcfd_amg* h, int64_t n) {
    return (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)h->sm_count * 8));
}

// A grid-stride kernel's grid capped at the blocks that can be resident at once: a
// grid above that runs a second, partial wave (the level-0 FP64 smoothing and
// prolongation kernels take 40 registers, so 6 blocks of 256 threads per SM, where the
// default grid is 8 per SM: a third of the rows ran in a tail at a quarter of the
// occupancy). Occupancy per kernel function, looked up once.
int resident_grid(const void* f, int grid, int block) {
    static std::mutex mu;
    static std::vector<std::pair<const void*, int>> cache;  // (function, blocks resident on the device)
    int res = 0;
    {
        std::lock_guard<std::mutex> lk(mu);
        for (const auto& e : cache)
            if (e.first == f) res = e.second;
    }
    if (res == 0) {
        int dev = 0, sms = 0, occ = 0;
        if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, f, block, 0) != cudaSuccess || occ < 1) {
            (void)cudaGetLastError();
            return grid;
        }
        res = occ * sms;
        std::lock_guard<std::mutex> lk(mu);
        cache.emplace_back(f, res);
    }
    return std::max(1, std::min(grid, res));
}

template <typename K, typename... Act>
void launch(K k, int grid, int block, cudaStream_t st, bool pdl, Act... args) {
    cudaLaunchConfig_t cfg;
    std::memset(&cfg, 0, sizeof(cfg));
    cfg.gridDim = dim3(resident_grid((const void*)k, grid, block));
    cfg.blockDim = dim3(block);
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = pdl ? at : nullptr;
    cfg.numAttrs = pdl ? 1 : 0;
    cudaLaunchKernelEx(&cfg, k, args...);
}

template <typename V>
int setup_t(kcfd_amg* h, const double* vals, cudaStream_t st) {
    const int L = h->nlev;
    for (int l = 0; l < L - 1; ++l) {
        Level& lv = h->lv[l];
        Level& nx = h->lv[l + 1];
        const double* a = l == 0 ? vals : lv.a64;
        const int g = grid_for(h, lv.n);
        const int gs = grid_for(h, lv.slots);
        k_sell_a<V><<<gs, 256, 0, st>>>(lv.slots, lv.ssrc, a, (V*)lv.sA);
        if (l == 0) {
            KCFD_CUDA(cudaMemsetAsync(h->rmax, 0, sizeof(unsigned long long), st));
            k_diag<<<g, 256, 0, st>>>(lv.n, lv.ip, a, lv.dslot, lv.dinv, h->rmax);
            k_omega_gersh<<<1, 1, 0, st>>>(h->rmax, h->omega);
        } else {
            k_diag<<<g, 256, 0, st>>>(lv.n, lv.ip, a, lv.dslot, lv.dinv, nullptr);
            const int gr = std::min(kRedGrid, g);
            k_pow_init<<<gr, 256, 0, st>>>(lv.n, h->powv[0], h->part, h->cnt, h->nrm2);
            const int gp = resident_grid((const void*)k_pow_step<V>, gr, 256);
            for (int t = 0; t < h->o.power_iters; ++t) {
                const int a_ = t & 1, b_ = a_ ^ 1;
                k_pow_step<V><<<gp, 256, 0, st>>>(lv.n, lv.soff, lv.scol, (const V*)lv.sA, lv.dinv, h->powv[a_],
                                                  h->nrm2 + a_, h->powv[b_], h->part, h->cnt, h->nrm2 + b_);
            }
            k_omega_pow<<<1, 1, 0, st>>>(h->nrm2 + (h->o.power_iters & 1), h->omega + l);
        }
        const double* om = h->omega + l;
        k_sd<V><<<g, 256, 0, st>>>(lv.n, lv.dinv, om, (V*)lv.sd);
        k_sell_w<V><<<gs, 256, 0, st>>>(lv.slots, lv.ssrc, lv.scol, a, lv.dinv, om, (V*)lv.sW);
        k_pvals<V><<<grid_for(h, lv.pnnz), 256, 0, st>>>(lv.pnnz, lv.prow, lv.pdiag, lv.plp, lv.pla, a, lv.dinv, om,
                                                         lv.p64, (V*)lv.pV);
        k_gather<V><<<grid_for(h, lv.pnnz), 256, 0, st>>>(lv.pnnz, lv.rsrc, lv.p64, lv.r64, (V*)lv.rV);
        k_product<<<grid_for(h, lv.bnnz), 256, 0, st>>>(lv.bnnz, lv.bptr, lv.bx, lv.bp, a, lv.p64, lv.b64);
        k_product<<<grid_for(h, nx.nnz), 256, 0, st>>>(nx.nnz, lv.cptr, lv.cr, lv.cb, lv.r64, lv.b64, nx.a64);
        KCFD_CUDA(cudaGetLastError());
    }
    Level& c = h->lv[L - 1];
    const double* a = L == 1 ? vals : c.a64;
    k_dense<<<1, 1024, 0, st>>>(c.n, c.ip, c.ix, a, h->dense);
    k_gj<V><<<1, 1024, h->gj_smem, st>>>(c.n, h->dense, h->dinvm, (V*)h->cinv, h->gj_smem > 0 ? 1 : 0);
    KCFD_CUDA(cudaGetLastError());
    return KCFD_OK;
}

template <typename V>
int vcycle_t(const kcfd_amg* h, const double* in, double* out, const int* active, cudaStream_t st, bool pdl) {
    const int L = h->nlev;
    if (L == 1) {
        const int nc = h->lv[0].n;
        launch(k_coarse<V, double, double>, std::max(1, (nc + 7) / 8), 256, st, pdl, nc, (const V*)h->cinv, in, out,
               active);
        return KCFD_OK;
    }
    for (int l = 0; l < L - 1; ++l) {
        const Level& lv = h->lv[l];
        const Level& nx = h->lv[l + 1];
        const int g = grid_for(h, lv.n);
        if (l == 0) {
            launch(k_pre<V, double>, g, 256, st, pdl, lv.n, (const int*)lv.soff, (const int*)lv.scol, (const V*)lv.sW,
                   (const V*)lv.sd, in, (V*)lv.x, (V*)lv.r, active);
        } else {
            const int L_ = lv.slanes;
            auto pk = L_ >= 32 ? k_pre<V, V, 32> : L_ == 16 ? k_pre<V, V, 16> : L_ == 8 ? k_pre<V, V, 8>
                    : L_ == 4 ? k_pre<V, V, 4> : L_ == 2 ? k_pre<V, V, 2> : k_pre<V, V, 1>;
            launch(pk, grid_for(h, (int64_t)lv.n * L_), 256, st, pdl, lv.n, (const int*)lv.soff, (const int*)lv.scol,
                   (const V*)lv.sW, (const V*)lv.sd, (const V*)lv.b, (V*)lv.x, (V*)lv.r, active);
        }
        const int gr = grid_for(h, (int64_t)nx.n * lv.rlanes);
        auto rk = lv.rlanes >= 32 ? k_restrict<V, 32> : lv.rlanes == 16 ? k_restrict<V, 16> : lv.rlanes == 8 ? k_restrict<V, 8>
                : lv.rlanes == 4 ? k_restrict<V, 4> : lv.rlanes == 2 ? k_restrict<V, 2> : k_restrict<V, 1>;
        launch(rk, gr, 256, st, pdl, nx.n, (const int*)lv.rip, (const int*)lv.rix, (const V*)lv.rV, (const V*)lv.r,
               (V*)nx.b, active);
    }
    const Level& c = h->lv[L - 1];
    launch(k_coarse<V, V, V>, std::max(1, (c.n + 7) / 8), 256, st, pdl, c.n, (const V*)h->cinv, (const V*)c.b,
           (V*)c.y, active);
    for (int l = L - 2; l >= 0; --l) {
        const Level& lv = h->lv[l];
        const Level& nx = h->lv[l + 1];
        const int g = grid_for(h, lv.n);
        launch(k_prolong<V>, g, 256, st, pdl, lv.n, (const int*)lv.pip, (const int*)lv.pix, (const V*)lv.pV,
               (const V*)nx.y, (V*)lv.x, active);
        if (l == 0) {
            launch(k_post<V, double, double>, g, 256, st, pdl, lv.n, (const int*)lv.soff, (const int*)lv.scol,
                   (const V*)lv.sA, (const V*)lv.sd, in, (const V*)lv.x, out, active);
        } else {
            const int L_ = lv.slanes;
            auto qk = L_ >= 32 ? k_post<V, V, V, 32> : L_ == 16 ? k_post<V, V, V, 16> : L_ == 8 ? k_post<V, V, V, 8>
                    : L_ == 4 ? k_post<V, V, V, 4> : L_ == 2 ? k_post<V, V, V, 2> : k_post<V, V, V, 1>;
            launch(qk, grid_for(h, (int64_t)lv.n * L_), 256, st, pdl, lv.n, (const int*)lv.soff, (const int*)lv.scol,
                   (const V*)lv.sA, (const V*)lv.sd, (const V*)lv.b, (const V*)lv.x, (V*)lv.y, active);
        }
    }
    KCFD_CUDA(cudaGetLastError());
    return KCFD_OK;
}

}  // namespace

int setup(kcfd_amg* h, const double* vals64, cudaStream_t st) {
    return h->mixed ? setup_t<float>(h, vals64, st) : setup_t<double>(h, vals64, st);
}

int vcycle(const kcfd_amg* h, const double* in, double* out, const int* active, cudaStream_t st, bool pdl) {
    return h->mixed ? vcycle_t<float>(h, in, out, active, st, pdl) : vcycle_t<double>(h, in, out, active, st, pdl);
}

int levels(const kcfd_amg* h) { return h->nlev; }

}  // namespace amg
}  // namespace kcfd

using namespace kcfd;
using namespace kcfd::amg;

extern "C" {

int kcfd_amg_create(const kcfd_csr_t* A, const kcfd_amg_opts_t* opts, kcfd_amg** out) {
    KCFD_REQUIRE(A && out, "kcfd_amg_create: NULL argument");
    *out = nullptr;
    KCFD_REQUIRE(A->n > 0 && A->nnz >= A->n && A->indptr && A->indices, "kcfd_amg_create: bad CSR (n=%d nnz=%d)",
                 A->n, A->nnz);
    kcfd_amg_opts_t o;
    std::memset(&o, 0, sizeof(o));
    if (opts) o = *opts;
    KCFD_REQUIRE(o.mode == KCFD_MODE_FP64 || o.mode == KCFD_MODE_MIXED, "kcfd_amg_create: bad mode");
    if (o.coarse_max <= 0) o.coarse_max = 128;
    if (o.max_levels <= 0) o.max_levels = 12;
    if (o.power_iters <= 0) o.power_iters = 8;
    KCFD_REQUIRE(o.coarse_max <= kDenseMax, "kcfd_amg_create: coarse_max above %d", kDenseMax);
    KCFD_REQUIRE(o.max_levels <= kMaxLevels, "kcfd_amg_create: max_levels above %d", kMaxLevels);
    KCFD_REQUIRE(o.power_iters <= 100, "kcfd_amg_create: power_iters above 100");
    const int n = A->n, nnz = A->nnz;
    HostCsr cur;
    cur.n = cur.m = n;
    cur.ip.resize(n + 1);
    cur.ix.resize(nnz);
    if (cudaMemcpy(cur.ip.data(), A->indptr, (n + 1) * 4, cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(cur.ix.data(), A->indices, (size_t)nnz * 4, cudaMemcpyDeviceToHost) != cudaSuccess) {
        set_error("kcfd_amg_create: cannot read the CSR pattern (device pointers expected)");
        return KCFD_BAD_INPUT;
    }
    KCFD_REQUIRE(cur.ip[0] == 0 && cur.ip[n] == nnz, "kcfd_amg_create: indptr[0] != 0 or indptr[n] != nnz");
    for (int i = 0; i < n; ++i) KCFD_REQUIRE(cur.ip[i + 1] >= cur.ip[i], "kcfd_amg_create: indptr not monotone at %d", i);
    for (int k = 0; k < nnz; ++k)
        KCFD_REQUIRE(cur.ix[k] >= 0 && cur.ix[k] < n, "kcfd_amg_create: column %d out of range at %d", cur.ix[k], k);
    int dev = 0;
    cudaDeviceProp prop;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaGetDeviceProperties(&prop, dev) != cudaSuccess) {
        set_error("kcfd_amg_create: no CUDA device");
        return KCFD_CUDA_ERROR;
    }
    auto* h = new kcfd_amg();
    h->o = o;
    h->mixed = o.mode == KCFD_MODE_MIXED;
    h->sm_count = prop.multiProcessorCount;
    const size_t vs = h->mixed ? sizeof(float) : sizeof(double);
    auto fail = [&](int code, const char* msg, int a1 = 0, int a2 = 0) {
        free_amg(h);
        set_error(msg, a1, a2);
        return code;
    };
    bool ok = alloc(h, (void**)&h->omega, kMaxLevels * sizeof(double)) &&
              alloc(h, (void**)&h->rmax, kMaxLevels * sizeof(unsigned long long)) &&
              alloc(h, (void**)&h->nrm2, 2 * sizeof(double)) && alloc(h, (void**)&h->part, kRedGrid * sizeof(double)) &&
              alloc(h, (void**)&h->cnt, sizeof(unsigned));
    if (!ok || cudaMemset(h->cnt, 0, sizeof(unsigned)) != cudaSuccess)
        return fail(KCFD_CUDA_ERROR, "kcfd_amg_create: device allocation failed");
    int L = 0;
    while (true) {
        Level& lv = h->lv[L];
        lv.n = cur.n;
        lv.nnz = cur.ip[cur.n];
        // diagonal slot of every row
        std::vector<int> dslot(cur.n, -1);
        for (int i = 0; i < cur.n; ++i)
            for (int k = cur.ip[i]; k < cur.ip[i + 1]; ++k)
                if (cur.ix[k] == i) {
                    dslot[i] = k;
                    break;
                }
        for (int i = 0; i < cur.n; ++i)
            if (dslot[i] < 0) return fail(KCFD_BAD_INPUT, "kcfd_amg_create: row %d of level %d has no diagonal entry", i, L);
        ok = up(h, &lv.ip, cur.ip) && up(h, &lv.ix, cur.ix) && up(h, &lv.dslot, dslot) &&
             alloc(h, (void**)&lv.dinv, (size_t)cur.n * sizeof(double)) &&
             alloc(h, &lv.b, (size_t)cur.n * vs) && alloc(h, &lv.y, (size_t)cur.n * vs);
        if (ok && L > 0) ok = alloc(h, (void**)&lv.a64, (size_t)lv.nnz * sizeof(double));
        if (!ok) return fail(KCFD_CUDA_ERROR, "kcfd_amg_create: device allocation failed (level %d)", L);
        ++L;
        h->nlev = L;
        if (cur.n <= o.coarse_max || L >= o.max_levels) break;
        std::vector<int> agg;
        const int na = aggregate(cur, agg);
        if ((double)na > 0.8 * cur.n) break;  // coarsening stalled: this level is the coarsest
        Transfer t;
        if (!build_transfer(cur, agg, na, t))
            return fail(KCFD_BAD_INPUT, "kcfd_amg_create: level %d products too large for 32-bit slots", L - 1);
        std::vector<int> off, col, src;
        if (!make_sell(cur, off, col, src))
            return fail(KCFD_BAD_INPUT, "kcfd_amg_create: level %d sliced-ELL copy too large", L - 1);
        // P entry -> its row, and its A entries (a counting sort of A's entries by P entry)
        const int pn = t.P.ip[cur.n];
        std::vector<int> prow(pn), plp(pn + 1, 0), pla(cur.ip[cur.n]);
        for (int i = 0; i < cur.n; ++i)
            for (int e = t.P.ip[i]; e < t.P.ip[i + 1]; ++e) prow[e] = i;
        for (int k = 0; k < cur.ip[cur.n]; ++k) plp[t.pmap[k] + 1]++;
        for (int e = 0; e < pn; ++e) plp[e + 1] += plp[e];
        {
            std::vector<int> fill(plp.begin(), plp.end() - 1);
            for (int k = 0; k < cur.ip[cur.n]; ++k) pla[fill[t.pmap[k]]++] = k;
        }
        // restriction lanes: about three entries per lane of a coarse row
        const double ravg = (double)pn / std::max(1, na);
        lv.rlanes = 1;
        while (lv.rlanes < 32 && 3.0 * lv.rlanes < ravg) lv.rlanes <<= 1;
        // smoothing lanes: a level of few long rows shares each row between lanes until
        // about 64k threads are busy (at least two entries per lane)
        const double savg = (double)cur.ip[cur.n] / std::max(1, cur.n);
        lv.slanes = 1;
        while (lv.slanes < 32 && (int64_t)cur.n * lv.slanes < 65536 && 2.0 * 2 * lv.slanes <= savg) lv.slanes <<= 1;
        lv.agg = agg;
        lv.nc = na;
        lv.pnnz = t.P.ip[cur.n];
        lv.bnnz = t.B.ip[cur.n];
        lv.slots = (int64_t)col.size();
        ok = up(h, &lv.soff, off) && up(h, &lv.scol, col) && up(h, &lv.ssrc, src) &&
             alloc(h, &lv.sA, lv.slots * vs) && alloc(h, &lv.sW, lv.slots * vs) && alloc(h, &lv.sd, (size_t)cur.n * vs) &&
             up(h, &lv.pip, t.P.ip) && up(h, &lv.pix, t.P.ix) && up(h, &lv.pdiag, t.pdiag) && up(h, &lv.prow, prow) &&
             up(h, &lv.plp, plp) && up(h, &lv.pla, pla) &&
             alloc(h, (void**)&lv.p64, (size_t)lv.pnnz * sizeof(double)) && alloc(h, &lv.pV, (size_t)lv.pnnz * vs) &&
             up(h, &lv.rip, t.R.ip) && up(h, &lv.rix, t.R.ix) && up(h, &lv.rsrc, t.rsrc) &&
             alloc(h, (void**)&lv.r64, (size_t)lv.pnnz * sizeof(double)) && alloc(h, &lv.rV, (size_t)lv.pnnz * vs) &&
             up(h, &lv.bip, t.B.ip) && alloc(h, (void**)&lv.b64, (size_t)lv.bnnz * sizeof(double)) &&
             up(h, &lv.bptr, t.bptr) && up(h, &lv.bx, t.bx) && up(h, &lv.bp, t.bp) && up(h, &lv.cptr, t.cptr) &&
             up(h, &lv.cr, t.cr) && up(h, &lv.cb, t.cb) && alloc(h, &lv.x, (size_t)cur.n * vs) &&
             alloc(h, &lv.r, (size_t)cur.n * vs);
        if (!ok) return fail(KCFD_CUDA_ERROR, "kcfd_amg_create: device allocation failed (level %d)", L - 1);
        cur = std::move(t.C);
    }
    const Level& c = h->lv[L - 1];
    if (c.n > kDenseMax)
        return fail(KCFD_BAD_INPUT, "kcfd_amg_create: coarsening stopped at %d rows (the dense coarse solve takes at most %d)",
                    c.n, kDenseMax);
    const size_t nc2 = (size_t)c.n * c.n;
    ok = alloc(h, (void**)&h->dense, nc2 * sizeof(double)) && alloc(h, (void**)&h->dinvm, nc2 * sizeof(double)) &&
         alloc(h, &h->cinv, nc2 * vs);
    // the elimination in shared memory when the matrix and its inverse fit (nc <= 113).
    // The launch limit is an attribute of the kernel, shared by every handle in the
    // process, so it is always set to the same bound (a handle with a smaller coarsest
    // level must not lower it under another's)
    if (ok && 2 * nc2 * sizeof(double) <= (size_t)kGjSmemMax) {
        h->gj_smem = (int)(2 * nc2 * sizeof(double));
        const void* kf = h->mixed ? (const void*)k_gj<float> : (const void*)k_gj<double>;
        if (cudaFuncSetAttribute(kf, cudaFuncAttributeMaxDynamicSharedMemorySize, kGjSmemMax) != cudaSuccess) {
            (void)cudaGetLastError();
            h->gj_smem = 0;
        }
    }
    if (ok && L > 1) {
        const size_t pv = (size_t)h->lv[1].n;
        ok = alloc(h, (void**)&h->powv[0], pv * sizeof(double)) && alloc(h, (void**)&h->powv[1], pv * sizeof(double));
    }
    if (!ok) return fail(KCFD_CUDA_ERROR, "kcfd_amg_create: device allocation failed (coarsest level)");
    *out = h;
    return KCFD_OK;
}

int kcfd_amg_setup(kcfd_amg* h, const kcfd_csr_t* A, void* stream) {
    KCFD_REQUIRE(h && A, "kcfd_amg_setup: NULL argument");
    KCFD_REQUIRE(A->n == h->lv[0].n && A->nnz == h->lv[0].nnz, "kcfd_amg_setup: matrix size differs from the pattern");
    KCFD_REQUIRE(A->vals64, "kcfd_amg_setup: FP64 values required");
    return amg::setup(h, A->vals64, (cudaStream_t)stream);
}

int kcfd_amg_apply(kcfd_amg* h, const double* b, double* x, void* stream) {
    KCFD_REQUIRE(h && b && x, "kcfd_amg_apply: NULL argument");
    return amg::vcycle(h, b, x, nullptr, (cudaStream_t)stream, false);
}

int kcfd_amg_info(const kcfd_amg* h, int32_t* nlevels, int64_t* rows_nnz, int64_t* device_bytes) {
    KCFD_REQUIRE(h && nlevels, "kcfd_amg_info: NULL argument");
    *nlevels = h->nlev;
    if (rows_nnz)
        for (int l = 0; l < h->nlev; ++l) {
            rows_nnz[2 * l] = h->lv[l].n;
            rows_nnz[2 * l + 1] = h->lv[l].nnz;
        }
    if (device_bytes) *device_bytes = h->bytes;
    return KCFD_OK;
}

int kcfd_amg_export(const kcfd_amg* h, int32_t level, int32_t what, void* out_host) {
    KCFD_REQUIRE(h && out_host, "kcfd_amg_export: NULL argument");
    KCFD_REQUIRE(level >= 0 && level < h->nlev, "kcfd_amg_export: level %d out of range", level);
    const Level& L = h->lv[level];
    const bool last = level == h->nlev - 1;
    auto copy = [&](const void* src, size_t bytes) {
        KCFD_CUDA(cudaDeviceSynchronize());
        KCFD_CUDA(cudaMemcpy(out_host, src, bytes, cudaMemcpyDeviceToHost));
        return KCFD_OK;
    };
    switch (what) {
        case KCFD_AMG_AGGREGATES:
            KCFD_REQUIRE(!last, "kcfd_amg_export: the coarsest level has no aggregates");
            std::memcpy(out_host, L.agg.data(), L.agg.size() * sizeof(int));
            return KCFD_OK;
        case KCFD_AMG_INDPTR: return copy(L.ip, (size_t)(L.n + 1) * sizeof(int));
        case KCFD_AMG_INDICES: return copy(L.ix, (size_t)L.nnz * sizeof(int));
        case KCFD_AMG_VALUES:
            KCFD_REQUIRE(level > 0, "kcfd_amg_export: level 0 values are the caller's");
            return copy(L.a64, (size_t)L.nnz * sizeof(double));
        case KCFD_AMG_P_INDPTR:
            KCFD_REQUIRE(!last, "kcfd_amg_export: the coarsest level has no prolongator");
            return copy(L.pip, (size_t)(L.n + 1) * sizeof(int));
        case KCFD_AMG_P_INDICES:
            KCFD_REQUIRE(!last, "kcfd_amg_export: the coarsest level has no prolongator");
            return copy(L.pix, (size_t)L.pnnz * sizeof(int));
        case KCFD_AMG_P_VALUES:
            KCFD_REQUIRE(!last, "kcfd_amg_export: the coarsest level has no prolongator");
            return copy(L.p64, (size_t)L.pnnz * sizeof(double));
        case KCFD_AMG_OMEGA:
            KCFD_REQUIRE(!last, "kcfd_amg_export: the coarsest level has no smoother");
            return copy(h->omega + level, sizeof(double));
        case KCFD_AMG_COARSE_INVERSE:
            KCFD_REQUIRE(last, "kcfd_amg_export: the dense inverse belongs to the coarsest level");
            return copy(h->dinvm, (size_t)L.n * L.n * sizeof(double));
        default: break;
    }
    set_error("kcfd_amg_export: unknown item %d", what);
    return KCFD_BAD_INPUT;
}

void kcfd_amg_destroy(kcfd_amg* h) {
    free_amg(h);
    (void)cudaGetLastError();
}

}  // extern "C"
