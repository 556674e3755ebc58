// reduce.cuh -- deterministic block and grid reductions.
//
// A block reduces with warp shuffles and one shared-memory pass; a grid
// reduction writes one partial record per block and the last block to
// arrive (found with one atomic counter, no waiting) reduces all records in
// index order, so the result does not depend on block scheduling.
#pragma once
#include "common.cuh"

namespace ptc {

template <int NV>
__device__ __forceinline__ void block_sum_store(double (&v)[NV], double* __restrict__ out_block) {
    __shared__ double sh[32][NV];
    const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
    const int nthr = blockDim.x * blockDim.y * blockDim.z;
    const int lane = tid & 31, wid = tid >> 5, nw = (nthr + 31) >> 5;
#pragma unroll
    for (int q = 0; q < NV; q++)
        for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_down_sync(0xffffffffu, v[q], o);
    if (lane == 0)
#pragma unroll
        for (int q = 0; q < NV; q++) sh[wid][q] = v[q];
    __syncthreads();
    if (wid == 0) {
#pragma unroll
        for (int q = 0; q < NV; q++) {
            double x = lane < nw ? sh[lane][q] : 0.0;
            for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
            if (lane == 0) out_block[q] = x;
        }
    }
}

template <int NV>
__device__ __forceinline__ void block_max_store(double (&v)[NV], double* __restrict__ out_block) {
    __shared__ double sh[32][NV];
    const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
    const int nthr = blockDim.x * blockDim.y * blockDim.z;
    const int lane = tid & 31, wid = tid >> 5, nw = (nthr + 31) >> 5;
#pragma unroll
    for (int q = 0; q < NV; q++)
        for (int o = 16; o > 0; o >>= 1) v[q] = nmax(v[q], __shfl_down_sync(0xffffffffu, v[q], o));
    if (lane == 0)
#pragma unroll
        for (int q = 0; q < NV; q++) sh[wid][q] = v[q];
    __syncthreads();
    if (wid == 0) {
#pragma unroll
        for (int q = 0; q < NV; q++) {
            double x = lane < nw ? sh[lane][q] : 0.0;
            for (int o = 16; o > 0; o >>= 1) x = nmax(x, __shfl_down_sync(0xffffffffu, x, o));
            if (lane == 0) out_block[q] = x;
        }
    }
}

// single-block reduction of nparts partial records of NV values, fixed order
template <int NV, bool MAX>
__device__ void reduce_parts(const double* __restrict__ parts, int nparts, double (&out)[NV]) {
    __shared__ double sh[32][NV];
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5, nw = (blockDim.x + 31) >> 5;
    double v[NV];
#pragma unroll
    for (int q = 0; q < NV; q++) v[q] = 0.0;
    for (int b = tid; b < nparts; b += blockDim.x)
#pragma unroll
        for (int q = 0; q < NV; q++) v[q] = MAX ? nmax(v[q], parts[(size_t)b * NV + q]) : v[q] + parts[(size_t)b * NV + q];
#pragma unroll
    for (int q = 0; q < NV; q++)
        for (int o = 16; o > 0; o >>= 1) {
            double y = __shfl_down_sync(0xffffffffu, v[q], o);
            v[q] = MAX ? nmax(v[q], y) : v[q] + y;
        }
    if (lane == 0)
#pragma unroll
        for (int q = 0; q < NV; q++) sh[wid][q] = v[q];
    __syncthreads();
#pragma unroll
    for (int q = 0; q < NV; q++) {
        double x = 0.0;
        if (wid == 0) {
            x = lane < nw ? sh[lane][q] : 0.0;
            for (int o = 16; o > 0; o >>= 1) {
                double y = __shfl_down_sync(0xffffffffu, x, o);
                x = MAX ? nmax(x, y) : x + y;
            }
        }
        out[q] = x;  // valid in thread 0
    }
}


// grid completion: every block calls this after writing its partial record;
// returns true in exactly one block (the last one), which may then read all
// records.  The counter is reset by that block for the next launch.
__device__ __forceinline__ bool last_block_arrive(unsigned int* counter, unsigned int nblocks) {
    __shared__ bool is_last;
    __threadfence();
    __syncthreads();
    const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
    if (tid == 0) {
        const unsigned int prev = atomicAdd(counter, 1u);
        is_last = (prev == nblocks - 1);
        if (is_last) *counter = 0u;
    }
    __syncthreads();
    if (is_last) __threadfence();
    return is_last;
}

// block-wide reduction of nparts records of NV values (fixed order), result
// valid in every thread; bypasses L1 so records of other blocks are current
template <int NV, bool MAX>
__device__ void reduce_records(const double* parts, int nparts, double (&out)[NV]) {
    __shared__ double sh[32][NV];
    const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
    const int nthr = blockDim.x * blockDim.y * blockDim.z;
    const int lane = tid & 31, wid = tid >> 5, nw = (nthr + 31) >> 5;
    double v[NV];
#pragma unroll
    for (int q = 0; q < NV; q++) v[q] = 0.0;
    for (int b = tid; b < nparts; b += nthr)
#pragma unroll
        for (int q = 0; q < NV; q++) {
            const double x = __ldcg(&parts[(size_t)b * NV + q]);
            v[q] = MAX ? nmax(v[q], x) : v[q] + x;
        }
#pragma unroll
    for (int q = 0; q < NV; q++)
        for (int o = 16; o > 0; o >>= 1) {
            const double y = __shfl_down_sync(0xffffffffu, v[q], o);
            v[q] = MAX ? nmax(v[q], y) : v[q] + y;
        }
    __syncthreads();
    if (lane == 0)
#pragma unroll
        for (int q = 0; q < NV; q++) sh[wid][q] = v[q];
    __syncthreads();
#pragma unroll
    for (int q = 0; q < NV; q++) {
        double x = 0.0;
        for (int ww = 0; ww < nw; ww++) x = MAX ? nmax(x, sh[ww][q]) : x + sh[ww][q];
        out[q] = x;
    }
    __syncthreads();
}

}  // namespace ptc
