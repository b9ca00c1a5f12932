// Teams of CTAs that run one Krylov solve together, and their deterministic
// reductions.
//
//  * CtaTeam  -- one CTA owns a whole system; phases are separated by __syncthreads.
//  * GridTeam -- every CTA of a cooperative launch owns a contiguous row range of one
//                system; phases are separated by a software grid barrier whose wait
//                is bounded by a clock64 budget (on expiry the kernel records
//                KCFD_TIMEOUT and returns; nothing spins forever). The same team
//                over the CTAs of one thread-block cluster (ranks from cluster_ids()) gives a
//                group whose members the hardware schedules together, with its own
//                barrier counter and partials.
//
// Reductions are fixed-order: a fixed xor-shuffle tree inside each warp, a fixed
// tree over warps, and (GridTeam) a fixed strided sum over CTA partials followed by
// the same warp tree. Every CTA therefore computes bit-identical scalars and takes
// the same branch, and a system gives the same result whatever runs beside it.
#pragma once
#include <cstdint>

namespace kcfd {

constexpr int kWarp = 32;

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Sum K values over the block; result returned to every thread. smem must hold
// 32*K doubles. Deterministic for a fixed blockDim.
template <int K>
__device__ __forceinline__ void block_sum(double (&v)[K], double* smem) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int k = 0; k < K; ++k) v[k] = warp_sum(v[k]);
    __syncthreads();
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < K; ++k) smem[k * 32 + wid] = v[k];
    }
    __syncthreads();
    if (wid == 0) {
#pragma unroll
        for (int k = 0; k < K; ++k) {
            double t = (lane < nw) ? smem[k * 32 + lane] : 0.0;
            t = warp_sum(t);
            if (lane == 0) smem[k * 32] = t;
        }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < K; ++k) v[k] = smem[k * 32];
    __syncthreads();
}

struct TeamCtl {
    unsigned int* bar;     // barrier counter (see GridTeam::sync)
    double* partials;      // [slots * kMaxK * size]
    int* err;              // KCFD_TIMEOUT when a barrier wait expired
    long long budget;      // clock64 cycles a barrier may wait
};

constexpr int kMaxK = 8;   // values per reduction
constexpr int kSlots = 8;  // reduction points per iteration

struct CtaTeam {
    int rank = 0, size = 1;
    __device__ __forceinline__ bool sync() {
        __syncthreads();
        return true;
    }
    template <int K>
    __device__ __forceinline__ bool allreduce(double (&v)[K], int /*slot*/, double* smem) {
        block_sum<K>(v, smem);
        return true;
    }
};

struct GridTeam {
    int rank, size;
    TeamCtl ctl;
    __device__ GridTeam(const TeamCtl& c) : rank(blockIdx.x), size(gridDim.x), ctl(c) {}
    __device__ GridTeam(const TeamCtl& c, int r, int n) : rank(r), size(n), ctl(c) {}

    // Grid barrier on one 32-bit counter (zeroed before the launch): CTA 0 adds
    // 2^31 - (size - 1), every other CTA adds 1, so the top bit flips exactly when the
    // last CTA arrives; a waiter polls until the top bit differs from the value it saw
    // on arrival. A CTA cannot arrive at the next barrier before this one completed,
    // so the flip cannot be undone under a waiter. Waits are bounded by a clock64
    // budget; on expiry the CTA records KCFD_TIMEOUT and every later wait fails fast.
    __device__ bool sync() {
        __shared__ int ok_s;
        __syncthreads();
        if (threadIdx.x == 0) {
            volatile unsigned int* vbar = ctl.bar;
            volatile int* verr = ctl.err;
            int ok = (*verr == 0);
            const unsigned int add = (rank == 0) ? (0x80000000u - (unsigned)(size - 1)) : 1u;
            __threadfence();
            const unsigned int old = atomicAdd(ctl.bar, add);
            long long t0 = clock64();
            while (ok && (((old ^ *vbar) & 0x80000000u) == 0)) {
                if (*verr != 0) {
                    ok = 0;
                    break;
                }
                if (clock64() - t0 > ctl.budget) {
                    atomicCAS(ctl.err, 0, 5 /*KCFD_TIMEOUT*/);
                    ok = 0;
                    break;
                }
            }
            __threadfence();
            ok_s = ok;
        }
        __syncthreads();
        return ok_s != 0;
    }

    template <int K>
    __device__ bool allreduce(double (&v)[K], int slot, double* smem) {
        block_sum<K>(v, smem);
        double* base = ctl.partials + (size_t)slot * kMaxK * size;
#pragma unroll
        for (int k = 0; k < K; ++k)
            if (threadIdx.x == k) base[(size_t)k * size + rank] = v[k];
        if (!sync()) return false;
        const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
        if (wid == 0) {
#pragma unroll
            for (int k = 0; k < K; ++k) {
                // after the barrier's fence: L2 loads (.cg), all issued before the sums
                const double* src = base + (size_t)k * size;
                double t = 0.0;
#pragma unroll 8
                for (int j = lane; j < size; j += 32) t += __ldcg(src + j);
                t = warp_sum(t);
                if (lane == 0) smem[k * 32] = t;
            }
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < K; ++k) v[k] = smem[k * 32];
        __syncthreads();
        return true;
    }
};

// This CTA's rank in its thread-block cluster, the cluster's CTA count and its index
// in the grid.
__device__ __forceinline__ void cluster_ids(int& rank, int& size, int& id) {
    unsigned r, n, c;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    asm volatile("mov.u32 %0, %%cluster_nctarank;" : "=r"(n));
    asm volatile("mov.u32 %0, %%clusterid.x;" : "=r"(c));
    rank = (int)r;
    size = (int)n;
    id = (int)c;
}

}  // namespace kcfd
