// cpb_reduce.cuh -- deterministic grid-wide reductions ("last block done").
//
// Every block writes its partial to partials[blockIdx.x]; the last block to
// arrive sums all partials in a fixed order, so the result is bitwise
// reproducible run to run (no floating-point atomics).
#pragma once

#include <cuda_runtime.h>

namespace cpb {

struct Reducer {
    double* partials;    // >= gridDim.x entries
    unsigned* counter;   // zero before the launch; reset to zero by the last block
};

// Block-wide sum of `v` (all threads participate).  Result valid in thread 0.
template <int NT>
__device__ __forceinline__ double block_sum(double v, double* sh) {
    v = warp_sum(v);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    double r = 0;
    if (threadIdx.x < 32) {
        r = (threadIdx.x < NT / 32) ? sh[threadIdx.x] : 0.0;
        r = warp_sum(r);
    }
    return r;
}

template <int NT>
__device__ __forceinline__ double block_max(double v, double* sh) {
    v = warp_max(v);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    double r = 0;
    if (threadIdx.x < 32) {
        r = (threadIdx.x < NT / 32) ? sh[threadIdx.x] : 0.0;
        r = warp_max(r);
    }
    return r;
}

// Grid-wide sum (or max when IS_MAX).  Returns true in every thread of the
// last block, where *total holds the grid result (also in sh_total[0]).  The
// block's partial goes to slot `slot` (default: blockIdx.x); the partials are
// summed in slot order, so blocks that work on permuted units keep the sum's
// order by passing their unit's index.
template <int NT, bool IS_MAX = false>
__device__ __forceinline__ bool grid_reduce(double v, Reducer red, double* sh, double* result, int slot = -1) {
    double b = IS_MAX ? block_max<NT>(v, sh) : block_sum<NT>(v, sh);
    __shared__ bool is_last;
    if (threadIdx.x == 0) {
        red.partials[slot < 0 ? blockIdx.x : (unsigned)slot] = b;
        __threadfence();
        unsigned prev = atomicAdd(red.counter, 1u);
        is_last = (prev == gridDim.x - 1);
    }
    __syncthreads();
    if (!is_last) return false;
    __threadfence();
    // L2 reads (ld.global.cg: L1 is not coherent across blocks), eight in flight per thread
    double acc = 0.0;
    const unsigned G = gridDim.x;
    for (unsigned i0 = threadIdx.x; i0 < G; i0 += 8 * NT) {
        double pv[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const unsigned i = i0 + k * NT;
            pv[k] = i < G ? __ldcg(red.partials + i) : 0.0;
        }
#pragma unroll
        for (int k = 0; k < 8; ++k) acc = IS_MAX ? nan_max(acc, pv[k]) : acc + pv[k];
    }
    double tot = IS_MAX ? block_max<NT>(acc, sh) : block_sum<NT>(acc, sh);
    __shared__ double tot_sh;
    if (threadIdx.x == 0) {
        tot_sh = tot;
        *red.counter = 0u;
    }
    __syncthreads();
    *result = tot_sh;
    return true;
}

}  // namespace cpb
