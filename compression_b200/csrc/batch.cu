// batch.cu -- batched mixed-codec decoding: one persistent launch over a
// list of warp-sized tasks of any codec, fed from a device work queue.
//
// No counterpart in the reference (its decoders are one launch per column
// and codec).  A task is one brle chunk, one RLE v1 / RLE v2 lane stream,
// one LZSS chunk or one Deflate stream; every codec has a warp-level decoder
// (brle_warp.cuh, rlev1.cuh, rlev2.cuh, lzss.cuh, inflate.cuh), so a single
// kernel can run them all.  Each warp repeatedly takes the next task either
// from a global atomic counter over an order array (dynamic: with tasks
// sorted longest-first this is LPT list scheduling) or by the static mapping
// task i -> warp i mod W.  Per-task %globaltimer start/end stamps (optional)
// are the measurements the learned cost model trains on.
#include "brle_warp.cuh"
#include "inflate.cuh"
#include "lzss.cuh"
#include "rlev1.cuh"
#include "rlev2.cuh"

namespace gd {
namespace batch {

constexpr int WPB = 4;  // warps per block
// Deflate workspace of a batch warp: a 4 KiB output window (nearer copies
// from shared memory, farther ones from the output), a 1 KiB input ring, an
// 8-bit distance table and batches of 512 literals / 64 commands (the
// standalone kernels use up to 32 KiB, 8 KiB, 10 bits, 2048 / 256); the
// largest codec workspace sets every warp's, so it is kept small.
using BatchInflSmem = infl::WarpSmemT<4096, 1, 1024, 8, 512, 64>;

__host__ __device__ constexpr uint32_t warp_smem_bytes(uint32_t max_lane) {
    // union of the per-codec warp workspaces
    uint32_t a = (uint32_t)sizeof(BatchInflSmem);
    uint32_t b = lzss::WARP_SMEM;
    uint32_t c = (uint32_t)sizeof(SegTable) + ((max_lane + 15u) & ~15u) + 160u + (uint32_t)sizeof(rlev2::WarpRuns);
    uint32_t d = brlew::WARP_SMEM;
    uint32_t m = a > b ? a : b;
    m = m > c ? m : c;
    m = m > d ? m : d;
    return (m + 15u) & ~15u;
}

__device__ __forceinline__ uint64_t globaltimer() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Copy lane stream `slot` (nw words) of an interleaved block into dst with
// the calling warp (asynchronous 4-byte copies), then zero 16 tail bytes.
__device__ __forceinline__ void load_slot_warp(const SegTable* T, const uint8_t* block, uint32_t slot, uint32_t nw,
                                               uint8_t* dst) {
    const uint32_t lane = lane_id();
    const uint32_t ltmask = (1u << slot) - 1u;
    for (uint32_t k = lane; k < nw; k += 32) {
        uint32_t j = 0;
#pragma unroll
        for (uint32_t step = 16; step; step >>= 1)
            if (j + step <= 31 && T->hi[j + step - 1] <= k) j += step;
        const uint32_t lo = j ? T->hi[j - 1] : 0u;
        const uint32_t off = T->base[j] + (k - lo) * 4u * (32u - j) + 4u * __popc(T->mask[j] & ltmask);
        const uint32_t sa = (uint32_t)__cvta_generic_to_shared(dst + 4 * k);
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa), "l"(block + off) : "memory");
    }
    asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
    if (lane < 4) reinterpret_cast<uint32_t*>(dst)[nw + lane] = 0;
    __syncwarp();
}

// One RLE v1 / v2 lane-stream task.
__device__ uint32_t rle_task(const gd_task& t, uint32_t max_lane, uint8_t* ws) {
    const uint32_t lane = lane_id();
    SegTable* T = reinterpret_cast<SegTable*>(ws);
    uint8_t* sbuf = ws + sizeof(SegTable);
    uint32_t bad = (t.lane >= 32 || (reinterpret_cast<uintptr_t>(t.src) & 3u)) ? 1u : 0u;
    const uint64_t l64 = t.col_len[lane];
    if (l64 > max_lane) bad = 1;
    const uint32_t len = bad ? 0u : (uint32_t)l64;
    const uint32_t nw = (len + 3) >> 2;
    uint32_t tot = warp_incl_scan(nw);
    tot = __shfl_sync(GD_FULL_MASK, tot, 31);
    if ((uint64_t)tot * 4 > t.src_len) bad = 1;
    if (__any_sync(GD_FULL_MASK, bad)) return ST_CORRUPT;
    seg_build(T, nw);
    const uint32_t slot = t.lane;
    const uint32_t my_len = __shfl_sync(GD_FULL_MASK, len, (int)slot);
    load_slot_warp(T, t.src, slot, (my_len + 3) >> 2, sbuf);
    if (t.codec == GD_CODEC_RLEV2) {
        const uint32_t ru = t.param;
        if (ru == 0 || t.chunk_size % (256ull * ru) || (reinterpret_cast<uintptr_t>(t.dst) & 7u)) return ST_INVALID;
        const uint32_t nv = (uint32_t)(t.chunk_size / 256u);
        // the run table sits past the stream's slot and its 160-byte tail
        auto* runs = reinterpret_cast<rlev2::WarpRuns*>(sbuf + ((max_lane + 15u) & ~15u) + 160u);
        return rlev2::decode_stream(sbuf, my_len, nv, slot, ru, reinterpret_cast<uint64_t*>(t.dst), t.dst_len / 8,
                                    *runs);
    }
    const uint32_t eb = t.param >> 16, wil = t.param & 0xffffu;
    if (!(eb == 4 || eb == 8) || wil == 0 || t.chunk_size % (32ull * wil * eb) ||
        (reinterpret_cast<uintptr_t>(t.dst) % eb))
        return ST_INVALID;
    const uint32_t nv = (uint32_t)(t.chunk_size / 32u / eb);
    if (eb == 4)
        return rlev1::lane_warp<uint32_t>(sbuf, my_len, nv, slot, wil, reinterpret_cast<uint32_t*>(t.dst),
                                          t.dst_len / 4);
    return rlev1::lane_warp<uint64_t>(sbuf, my_len, nv, slot, wil, reinterpret_cast<uint64_t*>(t.dst),
                                      t.dst_len / 8);
}

__device__ uint32_t run_task(const gd_task& t, uint32_t max_lane, uint8_t* ws) {
    switch (t.codec) {
        case GD_CODEC_BRLE:
            if (t.src_len > 0x7fffffffull || t.dst_len > 0x7fffffffull) return ST_INVALID;
            return brlew::chunk_warp(t.src, (uint32_t)t.src_len, t.dst, (uint32_t)t.dst_len, ws);
        case GD_CODEC_RLEV1:
        case GD_CODEC_RLEV2:
            return rle_task(t, max_lane, ws);
        case GD_CODEC_LZSS:
            if (t.dst_len != t.chunk_size || (reinterpret_cast<uintptr_t>(t.dst) & 3u)) return ST_INVALID;
            return lzss::chunk_warp(t.src, t.src_len, t.col_len, t.col_map, t.chunk_size, t.dst, ws);
        case GD_CODEC_DEFLATE: {
            if (t.src_len > 0xffffffffull || t.dst_len > 0xffffffffull) return ST_INVALID;
            uint32_t fin = 0;
            const uint32_t e = infl::stream_warp<4096, 1024, 8, 512, 64>(t.src, (uint32_t)t.src_len, t.dst,
                                                                     (uint32_t)t.dst_len, (int)t.param,
                                                                     *reinterpret_cast<BatchInflSmem*>(ws), &fin);
            return (e == ST_OK && fin != (uint32_t)t.dst_len) ? (uint32_t)ST_CORRUPT : e;
        }
        default:
            return ST_UNSUPPORTED;
    }
}

__global__ void __launch_bounds__(WPB * 32) batch_kernel(const gd_task* __restrict__ tasks, uint32_t n,
                                                        const uint32_t* __restrict__ order, uint32_t* counter,
                                                        int dynamic, uint32_t max_lane, uint32_t ws_bytes,
                                                        uint32_t* __restrict__ status,
                                                        uint64_t* __restrict__ timing) {
    extern __shared__ __align__(16) uint8_t smem[];
    const uint32_t lane = lane_id(), wid = threadIdx.x >> 5;
    uint8_t* ws = smem + wid * ws_bytes;
    const uint32_t gw = blockIdx.x * WPB + wid, W = gridDim.x * WPB;
    for (uint32_t k = 0;; ++k) {
        uint32_t i;
        if (dynamic) {
            uint32_t v = 0;
            if (lane == 0) v = atomicAdd(counter, 1u);
            i = __shfl_sync(GD_FULL_MASK, v, 0);
        } else {
            i = gw + k * W;
        }
        if (i >= n) break;
        const uint32_t ti = order ? order[i] : i;
        if (ti >= n) break;  // a malformed order array ends this worker
        const uint64_t t0 = globaltimer();
        const gd_task t = tasks[ti];
        const uint32_t e = run_task(t, max_lane, ws);
        __syncwarp();
        const uint64_t t1 = globaltimer();
        if (lane == 0) {
            put_status(status, ti, e);
            if (timing) {
                timing[2ull * ti] = t0;
                timing[2ull * ti + 1] = t1;
            }
        }
    }
}

}  // namespace batch
}  // namespace gd

extern "C" gd_status_t gd_batch_decode(const gd_task* d_tasks, uint32_t n_tasks, const uint32_t* d_order,
                                       int dynamic, uint32_t max_lane_bytes, uint32_t blocks_per_sm,
                                       uint32_t* d_counter, uint32_t* d_status, uint64_t* d_timing,
                                       gd_stream_t stream) {
    using namespace gd::batch;
    if (n_tasks == 0) return GD_OK;
    if (!d_tasks || (dynamic && !d_counter)) return GD_ERR_INVALID_ARG;
    const uint32_t ws = warp_smem_bytes(max_lane_bytes);
    const uint32_t smem = WPB * ws;
    if (smem > 220 * 1024) return GD_ERR_UNSUPPORTED;
    cudaStream_t s = (cudaStream_t)stream;
    cudaFuncSetAttribute(batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    int dev = 0, sms = 148, occ = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, batch_kernel, WPB * 32, smem);
    if (occ < 1) occ = 1;
    const uint32_t bps = blocks_per_sm ? (blocks_per_sm < (uint32_t)occ ? blocks_per_sm : (uint32_t)occ) : (uint32_t)occ;
    if (dynamic && cudaMemsetAsync(d_counter, 0, sizeof(uint32_t), s) != cudaSuccess) return GD_ERR_CUDA;
    batch_kernel<<<bps * (uint32_t)sms, WPB * 32, smem, s>>>(d_tasks, n_tasks, d_order, d_counter, dynamic,
                                                            max_lane_bytes, ws, d_status, d_timing);
    return cudaGetLastError() == cudaSuccess ? GD_OK : GD_ERR_CUDA;
}

extern "C" uint32_t gd_batch_warps(uint32_t max_lane_bytes, uint32_t blocks_per_sm) {
    using namespace gd::batch;
    const uint32_t smem = WPB * warp_smem_bytes(max_lane_bytes);
    cudaFuncSetAttribute(batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    int dev = 0, sms = 148, occ = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, batch_kernel, WPB * 32, smem);
    if (occ < 1) occ = 1;
    const uint32_t bps = blocks_per_sm ? (blocks_per_sm < (uint32_t)occ ? blocks_per_sm : (uint32_t)occ) : (uint32_t)occ;
    return bps * (uint32_t)sms * WPB;
}

// ---------------------------------------------------------------------------
// Batch decode with longest-first placement and no allocation at all.
//
// For callers that may not allocate device memory at decode time: hosts that
// hand the decoder a fixed memory budget up front (a query engine's
// pre-reserved pool, an embedded service with a hard memory cap) and treat
// any further allocation as a failure, and decode paths that must not pay
// cudaMalloc / cudaFree's implicit device-wide synchronisation while other
// streams of the process are busy.  gd_batch_decode needs a work-queue
// counter and an order array from its caller; here both live in the
// file-scope array below, together with the buckets of the sort that makes
// the order, so the only memory touched is the caller's tasks, costs,
// outputs and statuses plus this fixed array.
//
// Limits: at most NOALLOC_MAX_TASKS tasks per call (larger batches are
// rejected with GD_ERR_INVALID_ARG).  Nothing has to start at zero: the sort
// kernel clears the buckets and the counter at the start of every call.
// Calls that overlap in time on one device (two streams, or two host
// threads) share the array and race; the caller serialises them.  The
// array's device address is looked up once per device and kept for the life
// of the process; a cudaDeviceReset() of that device invalidates it, so the
// entry point is not for use after such a reset.
// ---------------------------------------------------------------------------
#include <mutex>

namespace gd {
namespace batch {

constexpr uint32_t NOALLOC_MAX_TASKS = GD_BATCH_NOALLOC_MAX_TASKS;
constexpr uint32_t NBUCKET = 1024;  // cost buckets of the order sort
constexpr uint32_t SORT_NT = 1024;  // threads of the single sort block
// [0, MAX): order; [MAX, MAX + NBUCKET): bucket cursors; [MAX + NBUCKET]: counter
static __device__ __align__(256) uint32_t g_noalloc_scratch[NOALLOC_MAX_TASKS + NBUCKET + 64];

// Bucket of cost c, with mn / mx the smallest and largest FINITE costs and
// scale = (NBUCKET - 1) / (mx - mn) (0 when all finite costs are equal).
// The highest cost goes to bucket 0, so the bucket order is longest first;
// costs equal to mn (all of them when scale is 0) go to the last bucket.
// Non-finite costs are placed explicitly: +inf first (bucket 0), -inf and
// NaN last (bucket NBUCKET - 1).
__device__ __forceinline__ uint32_t cost_bucket(float c, float mn, float scale) {
    if (c == INFINITY) return 0;
    if (!(c > -INFINITY && c < INFINITY)) return NBUCKET - 1;  // NaN or -inf
    const float q = (c - mn) * scale;                          // finite, >= 0
    const uint32_t b = q >= (float)(NBUCKET - 1) ? NBUCKET - 1 : (uint32_t)q;
    return NBUCKET - 1 - b;
}

// One block: counting sort of task indices by descending cost (bucketed, so
// tasks within a bucket are in arbitrary order) into scratch order[0..n),
// and the work-queue counter reset to zero.
__global__ void __launch_bounds__(SORT_NT) lpt_sort_kernel(const float* __restrict__ cost, uint32_t n,
                                                            uint32_t* __restrict__ scratch) {
    __shared__ uint32_t hist[NBUCKET];
    __shared__ float red_mn[SORT_NT / 32], red_mx[SORT_NT / 32];
    uint32_t* order = scratch;
    uint32_t* cursor = scratch + NOALLOC_MAX_TASKS;
    const uint32_t tid = threadIdx.x;
    float mn = INFINITY, mx = -INFINITY;
    for (uint32_t i = tid; i < n; i += SORT_NT) {
        const float c = cost[i];
        if (c > -INFINITY && c < INFINITY) {  // finite costs set the bucket range
            mn = fminf(mn, c);
            mx = fmaxf(mx, c);
        }
    }
    for (int s = 16; s; s >>= 1) {
        mn = fminf(mn, __shfl_xor_sync(GD_FULL_MASK, mn, s));
        mx = fmaxf(mx, __shfl_xor_sync(GD_FULL_MASK, mx, s));
    }
    if ((tid & 31) == 0) {
        red_mn[tid >> 5] = mn;
        red_mx[tid >> 5] = mx;
    }
    for (uint32_t b = tid; b < NBUCKET; b += SORT_NT) hist[b] = 0;
    if (tid == 0) scratch[NOALLOC_MAX_TASKS + NBUCKET] = 0;  // work-queue counter
    __syncthreads();
    mn = INFINITY;
    mx = -INFINITY;
    for (int w = 0; w < SORT_NT / 32; ++w) {
        mn = fminf(mn, red_mn[w]);
        mx = fmaxf(mx, red_mx[w]);
    }
    // no finite cost at all: mn = +inf, mx = -inf, span < 0, scale 0 (every
    // cost is non-finite and placed by cost_bucket without the range); a
    // span that overflows float gives scale 0 too
    const float span = mx - mn;
    const float scale = (span > 0.f && span < INFINITY) ? (float)(NBUCKET - 1) / span : 0.f;
    for (uint32_t i = tid; i < n; i += SORT_NT) atomicAdd(&hist[cost_bucket(cost[i], mn, scale)], 1u);
    __syncthreads();
    if (tid < 32) {  // exclusive scan of the buckets by warp 0, 32 buckets per lane
        uint32_t loc[NBUCKET / 32], s = 0;
#pragma unroll
        for (int k = 0; k < NBUCKET / 32; ++k) {
            loc[k] = s;
            s += hist[tid * (NBUCKET / 32) + k];
        }
        uint32_t inc = warp_incl_scan(s);
        const uint32_t base = inc - s;
#pragma unroll
        for (int k = 0; k < NBUCKET / 32; ++k) cursor[tid * (NBUCKET / 32) + k] = base + loc[k];
    }
    __syncthreads();
    for (uint32_t i = tid; i < n; i += SORT_NT) {
        const uint32_t p = atomicAdd(&cursor[cost_bucket(cost[i], mn, scale)], 1u);
        order[p] = i;
    }
}

}  // namespace batch
}  // namespace gd

extern "C" gd_status_t gd_batch_decode_lpt_noalloc(const gd_task* d_tasks, uint32_t n_tasks, const float* d_cost,
                                                   uint32_t max_lane_bytes, uint32_t blocks_per_sm,
                                                   uint32_t* d_status, gd_stream_t stream) {
    using namespace gd::batch;
    if (n_tasks == 0) return GD_OK;
    if (!d_tasks || !d_cost || n_tasks > NOALLOC_MAX_TASKS) return GD_ERR_INVALID_ARG;
    // Set-up, once per device with that device current: the device address
    // of the scratch array.  The first call on a device therefore makes a
    // runtime query and should come before any stream capture.
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return GD_ERR_CUDA;
    static std::mutex mu;
    static uint32_t* scratch_of[64] = {};
    static int sms_of[64] = {};
    uint32_t* scratch;
    int sms;
    {
        std::lock_guard<std::mutex> g(mu);
        if (!scratch_of[dev]) {
            void* p = nullptr;
            if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return GD_ERR_CUDA;
            int m = 0;
            if (cudaDeviceGetAttribute(&m, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || m <= 0)
                return GD_ERR_CUDA;
            sms_of[dev] = m;
            scratch_of[dev] = static_cast<uint32_t*>(p);
        }
        scratch = scratch_of[dev];
        sms = sms_of[dev];
    }
    const uint32_t ws = warp_smem_bytes(max_lane_bytes);
    const uint32_t smem = WPB * ws;
    if (smem > 220 * 1024) return GD_ERR_UNSUPPORTED;
    cudaStream_t s = (cudaStream_t)stream;
    if (cudaFuncSetAttribute(batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess)
        return GD_ERR_CUDA;
    int occ = 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, batch_kernel, WPB * 32, smem);
    if (occ < 1) occ = 1;
    const uint32_t bps = blocks_per_sm ? (blocks_per_sm < (uint32_t)occ ? blocks_per_sm : (uint32_t)occ) : (uint32_t)occ;
    lpt_sort_kernel<<<1, SORT_NT, 0, s>>>(d_cost, n_tasks, scratch);
    if (cudaGetLastError() != cudaSuccess) return GD_ERR_CUDA;
    batch_kernel<<<bps * (uint32_t)sms, WPB * 32, smem, s>>>(d_tasks, n_tasks, scratch,
                                                            scratch + NOALLOC_MAX_TASKS + NBUCKET, 1,
                                                            max_lane_bytes, ws, d_status, nullptr);
    return cudaGetLastError() == cudaSuccess ? GD_OK : GD_ERR_CUDA;
}
