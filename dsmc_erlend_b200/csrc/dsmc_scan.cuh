// dsmc_scan.cuh - block scans and the decoupled look-back chain used by the
// single-pass kernels (Merrill and Garland, "Single-pass parallel prefix scan
// with decoupled look-back", 2016).
#pragma once

#include <cstdint>

#include "dsmc_device.cuh"

namespace dsmc {

// Status word of one tile of a chain: flag in bits 62-63, value below.
constexpr uint64_t LB_AGG = 1ull << 62;  // tile aggregate published
constexpr uint64_t LB_INC = 2ull << 62;  // inclusive prefix published
constexpr uint64_t LB_FLAGS = 3ull << 62;
constexpr uint64_t LB_VALUE = ~LB_FLAGS;

// Two 31-bit counts packed into one value (for the pair scan of cells).
__device__ __forceinline__ uint64_t pack2(uint32_t a, uint32_t b)
{
    return (static_cast<uint64_t>(a) << 31) | b;
}
__device__ __forceinline__ uint32_t pack2_a(uint64_t v) { return static_cast<uint32_t>(v >> 31); }
__device__ __forceinline__ uint32_t pack2_b(uint64_t v)
{
    return static_cast<uint32_t>(v & 0x7FFFFFFFull);
}

__device__ __forceinline__ void report_error(int *err, int code) { atomicCAS(err, 0, code); }

// Exclusive prefix of `agg` over the earlier tiles of one chain.  Tile
// `t` is the chain's first when `first` is set.  Called by one thread.  Every
// wait is bounded: after SPIN_LIMIT polls the chain is abandoned, the error
// word gets DSMC_ERR_TIMEOUT and the prefix is returned as 0.
__device__ __forceinline__ uint64_t lookback(uint64_t *status, int t, bool first, uint64_t agg,
                                            int *err)
{
    volatile uint64_t *vs = status;
    if (first) {
        __threadfence();
        vs[t] = LB_INC | agg;
        return 0;
    }
    vs[t] = LB_AGG | agg;
    __threadfence();
    uint64_t excl = 0;
    int j = t - 1;
    for (;;) {
        uint64_t w = vs[j];
        uint32_t spins = 0;
        while ((w & LB_FLAGS) == 0) {
            if (++spins > SPIN_LIMIT) {
                report_error(err, DSMC_ERR_TIMEOUT);
                vs[t] = LB_INC | agg;
                return 0;
            }
            __nanosleep(64);
            w = vs[j];
        }
        excl += (w & LB_VALUE);
        if ((w & LB_FLAGS) == LB_INC)
            break;
        --j;
    }
    __threadfence();
    vs[t] = LB_INC | (excl + agg);
    return excl;
}

__device__ __forceinline__ uint64_t warp_sum_u64(uint64_t v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Warp-wide form of lookback(): called by all 32 lanes of one warp.  Each
// poll reads the 32 predecessors t-1 .. t-32 at once, so the walk over tiles
// that have published only their aggregate advances 32 tiles per poll
// instead of one.  `chain0` is the chain's first tile: predecessors before
// it belong to another case and count as zero.  Returns the exclusive prefix
// in every lane.
__device__ __forceinline__ uint64_t lookback_warp(uint64_t *status, int t, int chain0,
                                                  uint64_t agg, int *err)
{
    volatile uint64_t *vs = status;
    const int lane = threadIdx.x & 31;
    if (t == chain0) {
        if (lane == 0) {
            __threadfence();
            vs[t] = LB_INC | agg;
        }
        __syncwarp();
        return 0;
    }
    if (lane == 0)
        vs[t] = LB_AGG | agg;
    __threadfence();
    __syncwarp();
    uint64_t excl = 0;
    int base = t - 1;
    uint32_t spins = 0;
    for (;;) {
        const int j = base - lane;
        uint64_t w = 2ull << 62; // LB_INC with value 0 before the chain
        if (j >= chain0)
            w = vs[j];
        if (!__all_sync(0xffffffffu, (w & LB_FLAGS) != 0)) {
            if (++spins > SPIN_LIMIT) {
                if (lane == 0) {
                    report_error(err, DSMC_ERR_TIMEOUT);
                    vs[t] = LB_INC | agg;
                }
                __syncwarp();
                return 0;
            }
            __nanosleep(32);
            continue;
        }
        const unsigned inc = __ballot_sync(0xffffffffu, (w & LB_FLAGS) == LB_INC);
        if (inc) {
            const int closest = __ffs(inc) - 1; // lowest lane = nearest tile
            excl += warp_sum_u64(lane <= closest ? (w & LB_VALUE) : 0ull);
            break;
        }
        excl += warp_sum_u64(w & LB_VALUE);
        base -= 32;
    }
    if (lane == 0) {
        __threadfence();
        vs[t] = LB_INC | (excl + agg);
    }
    __syncwarp();
    return excl;
}

// Block-wide form of lookback(): called by all NT threads of a CTA.  Each
// poll reads the NT predecessors t-1 .. t-NT at once (one per thread), so a
// chain whose tiles all run in one wave, and have published only their
// aggregates, is crossed NT tiles per poll.  Same contract as lookback_warp.
template <int NT>
__device__ __forceinline__ uint64_t lookback_block(uint64_t *status, int t, int chain0,
                                                   uint64_t agg, int *err)
{
    static_assert(NT % 32 == 0 && NT <= 1024, "block of whole warps");
    constexpr int NW = NT / 32;
    __shared__ uint64_t s_part[NW];
    __shared__ int s_near[NW]; // lowest lane holding an inclusive prefix, 32 if none
    volatile uint64_t *vs = status;
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    if (t == chain0) {
        if (threadIdx.x == 0) {
            __threadfence();
            vs[t] = LB_INC | agg;
        }
        return 0;
    }
    if (threadIdx.x == 0)
        vs[t] = LB_AGG | agg;
    __threadfence();
    uint64_t excl = 0;
    int base = t - 1;
    uint32_t spins = 0;
    for (;;) {
        const int j = base - static_cast<int>(threadIdx.x);
        uint64_t w = LB_INC; // value 0 before the chain
        if (j >= chain0)
            w = vs[j];
        if (!__syncthreads_and((w & LB_FLAGS) != 0)) {
            if (++spins > SPIN_LIMIT) { // uniform: every thread counts the same polls
                if (threadIdx.x == 0) {
                    report_error(err, DSMC_ERR_TIMEOUT);
                    vs[t] = LB_INC | agg;
                }
                return 0;
            }
            __nanosleep(32);
            continue;
        }
        const unsigned inc = __ballot_sync(0xffffffffu, (w & LB_FLAGS) == LB_INC);
        const int near = inc ? __ffs(inc) - 1 : 32;
        const uint64_t part = warp_sum_u64(lane <= near ? (w & LB_VALUE) : 0ull);
        if (lane == 0) {
            s_part[warp] = part;
            s_near[warp] = near;
        }
        __syncthreads();
        // Windows nearer than the first one holding an inclusive prefix are
        // summed whole; that one up to its prefix.
        bool done = false;
        for (int i = 0; i < NW && !done; ++i) {
            excl += s_part[i];
            done = s_near[i] < 32;
        }
        __syncthreads(); // s_part is rewritten by the next poll
        if (done)
            break;
        base -= NT;
    }
    if (threadIdx.x == 0) {
        __threadfence();
        vs[t] = LB_INC | (excl + agg);
    }
    return excl;
}

// Block-wide exclusive sum over NT threads; also returns the total.
template <class V, int NT = TILE_THREADS>
__device__ __forceinline__ V block_exclusive(V v, V &total)
{
    static_assert(NT % 32 == 0 && NT <= 1024, "block of whole warps");
    constexpr int NW = NT / 32;
    __shared__ V warp_tot[NW];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    V inc = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const V n = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o)
            inc += n;
    }
    if (lane == 31)
        warp_tot[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        V w = lane < NW ? warp_tot[lane] : V(0);
#pragma unroll
        for (int o = 1; o < NW; o <<= 1) {
            const V n = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o)
                w += n;
        }
        if (lane < NW)
            warp_tot[lane] = w;
    }
    __syncthreads();
    const V warp_excl = warp == 0 ? V(0) : warp_tot[warp - 1];
    total = warp_tot[NW - 1];
    __syncthreads();
    return warp_excl + inc - v;
}

// Index of the case that owns tile `t`: the last i with tile0[i] <= t.
__device__ __forceinline__ int case_of_tile(const int32_t *tile0, int stride, int ncase, int t)
{
    int lo = 0, hi = ncase - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (tile0[mid * stride] <= t)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

} // namespace dsmc
