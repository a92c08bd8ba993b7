// host_cuda.h -- runs the reference's CUDA kernels on host threads, to
// produce golden outputs of its GPU-only writers.  Oracle tooling only.
//
// A kernel launch is emulated block by block: one std::thread per CUDA
// thread of the block, with threadIdx / blockIdx thread-local, __syncthreads
// a barrier of the block's threads, and the warp collectives the writers use
// (__syncwarp, __shfl_down_sync with a full mask) an exchange among the
// 32 threads of the warp.  Blocks run one after another, so a kernel's
// `static __shared__` arrays (plain statics here) are the block's shared
// memory.  Force-included (-include) before the reference's headers.
#pragma once
#include <algorithm>
#include <atomic>
#include <barrier>
#include <cmath>
#include <math.h>
#include <cstring>
#include <cstdint>
#include <cstdio>
#include <functional>
#include <memory>
#include <thread>
#include <type_traits>
#include <vector>

#define __host__
#define __device__
#define __global__
#define __inline__ inline
#define __forceinline__ inline
#define __launch_bounds__(...)
#ifndef __shared__
#define __shared__
#endif

typedef int cudaError_t;
constexpr cudaError_t cudaSuccess = 0;
inline const char* cudaGetErrorString(cudaError_t) { return "host emulation"; }

// threadIdx.x is a lane number whose `32 - x` keeps a mark, so that the
// reference's `mask >> (32 - threadIdx.x)` shifts as the GPU does: a shift by
// 32 or more gives 0 (PTX shr clamps; on the host it would be undefined).
struct hc_shift {
    unsigned v;
    operator unsigned() const { return v; }
};
struct hc_lane {
    unsigned v = 0;
    hc_lane() = default;
    hc_lane(unsigned x) : v(x) {}
    operator unsigned() const { return v; }
};
inline hc_shift operator-(int a, hc_lane l) { return {(unsigned)a - l.v}; }
inline hc_shift operator-(unsigned a, hc_lane l) { return {a - l.v}; }
inline unsigned operator>>(unsigned a, hc_shift s) { return s.v >= 32 ? 0u : a >> s.v; }
inline unsigned operator<<(unsigned a, hc_shift s) { return s.v >= 32 ? 0u : a << s.v; }

struct hc_tid {
    hc_lane x;
    unsigned y = 0, z = 0;
};
struct hc_dim3 {
    unsigned x = 0, y = 0, z = 0;
};
inline thread_local hc_tid threadIdx;
inline thread_local hc_dim3 blockIdx;
inline hc_dim3 blockDim, gridDim;

namespace hc {
struct Block {
    std::unique_ptr<std::barrier<>> all;
    std::vector<std::unique_ptr<std::barrier<>>> warp;
    std::vector<uint64_t> xchg;  // one slot per thread, for warp exchanges
};
inline Block* g_block = nullptr;
inline unsigned flat() { return threadIdx.x.v + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z); }

// Launch `kern` over grid g of blocks of b threads, one block at a time.
inline void launch(hc_dim3 g, hc_dim3 b, const std::function<void()>& kern) {
    const unsigned nt = std::max(1u, b.x) * std::max(1u, b.y) * std::max(1u, b.z);
    gridDim = g;
    blockDim = b;
    for (unsigned bz = 0; bz < std::max(1u, g.z); ++bz)
        for (unsigned by = 0; by < std::max(1u, g.y); ++by)
            for (unsigned bx = 0; bx < std::max(1u, g.x); ++bx) {
                Block blk;
                blk.all = std::make_unique<std::barrier<>>(nt);
                for (unsigned w = 0; w < (nt + 31) / 32; ++w)
                    blk.warp.push_back(std::make_unique<std::barrier<>>(std::min(32u, nt - 32 * w)));
                blk.xchg.assign(nt, 0);
                g_block = &blk;
                std::vector<std::thread> th;
                for (unsigned t = 0; t < nt; ++t)
                    th.emplace_back([&, t]() {
                        threadIdx.x = hc_lane(t % std::max(1u, b.x));
                        threadIdx.y = (t / std::max(1u, b.x)) % std::max(1u, b.y);
                        threadIdx.z = t / (std::max(1u, b.x) * std::max(1u, b.y));
                        blockIdx = {bx, by, bz};
                        kern();
                    });
                for (auto& x : th) x.join();
                g_block = nullptr;
            }
}
}  // namespace hc

inline void __syncthreads() { hc::g_block->all->arrive_and_wait(); }
inline void __syncwarp(unsigned = 0xffffffffu) { hc::g_block->warp[hc::flat() / 32]->arrive_and_wait(); }
inline void __nanosleep(unsigned) { std::this_thread::yield(); }

template <typename T>
inline T __shfl_down_sync(unsigned, T v, int delta) {
    const unsigned me = hc::flat(), w = me / 32, lane = me % 32;
    uint64_t bits = 0;
    static_assert(sizeof(T) <= 8, "");
    std::memcpy(&bits, &v, sizeof(T));
    hc::g_block->xchg[me] = bits;
    __syncwarp();
    const unsigned src = lane + (unsigned)delta < 32 ? me + (unsigned)delta : me;
    T r;
    bits = hc::g_block->xchg[src];
    std::memcpy(&r, &bits, sizeof(T));
    __syncwarp();
    (void)w;
    return r;
}

// every lane of the warp takes part (the writers only use full masks)
inline unsigned __ballot_sync(unsigned, int pred) {
    const unsigned me = hc::flat(), w = me / 32;
    hc::g_block->xchg[me] = pred ? 1u : 0u;
    __syncwarp();
    unsigned r = 0;
    const unsigned n = std::min(32u, (unsigned)hc::g_block->xchg.size() - 32 * w);
    for (unsigned l = 0; l < n; ++l) r |= (hc::g_block->xchg[32 * w + l] ? 1u : 0u) << l;
    __syncwarp();
    return r;
}
inline int __popc(unsigned x) { return __builtin_popcount(x); }
// funnel shifts of the 64-bit hi:lo (the CUDA documentation's semantics):
// _c clamps the shift to 32, the plain forms take it modulo 32
inline unsigned __funnelshift_rc(unsigned lo, unsigned hi, unsigned s) {
    const uint64_t x = ((uint64_t)hi << 32) | lo;
    return (unsigned)(x >> (s < 32 ? s : 32));
}
inline unsigned __funnelshift_r(unsigned lo, unsigned hi, unsigned s) {
    return (unsigned)((((uint64_t)hi << 32) | lo) >> (s & 31));
}
inline unsigned __funnelshift_lc(unsigned lo, unsigned hi, unsigned s) {
    const uint64_t x = ((uint64_t)hi << 32) | lo;
    return (unsigned)((x << (s < 32 ? s : 32)) >> 32);
}
inline unsigned __funnelshift_l(unsigned lo, unsigned hi, unsigned s) {
    return (unsigned)(((((uint64_t)hi << 32) | lo) << (s & 31)) >> 32);
}

inline unsigned long long atomicAdd(unsigned long long* p, unsigned long long v) {
    return std::atomic_ref<unsigned long long>(*p).fetch_add(v);
}

// CUDA's integer min / max: the value, in the arguments' common type
template <typename A, typename B>
inline std::common_type_t<A, B> min(A a, B b) { return a < b ? a : b; }
template <typename A, typename B>
inline std::common_type_t<A, B> max(A a, B b) { return a < b ? b : a; }
