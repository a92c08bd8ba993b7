// gd_common.cuh -- shared device/host helpers for the sm_100a decoders.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/gd.h"

#define GD_FULL_MASK 0xffffffffu

namespace gd {

// Per-chunk status values written by kernels (same numbering as gd_status_t).
enum : uint32_t {
    ST_OK = GD_OK,
    ST_INVALID = GD_ERR_INVALID_ARG,
    ST_CORRUPT = GD_ERR_CORRUPT,
    ST_OVERRUN = GD_ERR_OVERRUN,
    ST_TIMEOUT = GD_ERR_TIMEOUT,
    ST_UNSUPPORTED = GD_ERR_UNSUPPORTED,
};

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }

__device__ __forceinline__ void put_status(uint32_t* st, uint64_t i, uint32_t v) {
    if (st) st[i] = v;
}

// Warp-wide inclusive prefix sum.
__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t v) {
    const uint32_t l = lane_id();
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t n = __shfl_up_sync(GD_FULL_MASK, v, o);
        if (l >= (uint32_t)o) v += n;
    }
    return v;
}

__device__ __forceinline__ uint64_t warp_incl_scan64(uint64_t v) {
    const uint32_t l = lane_id();
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint64_t n = __shfl_up_sync(GD_FULL_MASK, v, o);
        if (l >= (uint32_t)o) v += n;
    }
    return v;
}

// Block-wide exclusive scan of one uint32 per thread (NT threads, NT % 32 == 0).
// `tmp` must hold NT/32 + 1 words.  Returns the exclusive prefix; *total gets
// the block sum.  Contains __syncthreads.
template <int NT>
__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t* tmp, uint32_t* total) {
    const uint32_t l = lane_id(), w = threadIdx.x >> 5;
    uint32_t inc = warp_incl_scan(v);
    if (l == 31) tmp[w] = inc;
    __syncthreads();
    if (w == 0) {
        uint32_t x = (l < NT / 32) ? tmp[l] : 0;
        uint32_t xi = warp_incl_scan(x);
        if (l < NT / 32) tmp[l] = xi - x;
        if (l == NT / 32 - 1) tmp[NT / 32] = xi;
    }
    __syncthreads();
    uint32_t r = tmp[w] + inc - v;
    *total = tmp[NT / 32];
    return r;
}

// Block-wide exclusive scan of one uint64 per thread; as block_excl_scan.
// `tmp` must hold NT/32 + 1 words.  Contains __syncthreads.
template <int NT>
__device__ __forceinline__ uint64_t block_excl_scan64(uint64_t v, uint64_t* tmp, uint64_t* total) {
    const uint32_t l = lane_id(), w = threadIdx.x >> 5;
    uint64_t inc = warp_incl_scan64(v);
    if (l == 31) tmp[w] = inc;
    __syncthreads();
    if (w == 0) {
        uint64_t x = (l < NT / 32) ? tmp[l] : 0;
        uint64_t xi = warp_incl_scan64(x);
        if (l < NT / 32) tmp[l] = xi - x;
        if (l == NT / 32 - 1) tmp[NT / 32] = xi;
    }
    __syncthreads();
    uint64_t r = tmp[w] + inc - v;
    *total = tmp[NT / 32];
    return r;
}

}  // namespace gd
