// rlev1.cu -- RLE v1 (32-lane interleaved container) decoder for sm_100a: a
// block of 8 (or 4) warps owns as many adjacent lane streams of one chunk,
// copies them into shared memory, and each warp decodes one (warp-level
// decoder in rlev1.cuh).
#include "rlev1.cuh"

namespace gd {
namespace rlev1 {

// LANES_PER_BLOCK (8 default, 4 by GD_TUNE_RLEV1_LANES_PER_BLOCK): warps per
// block = lane streams per block
template <typename T, int LANES_PER_BLOCK>
__global__ void __launch_bounds__(LANES_PER_BLOCK * 32) decode_kernel(
    const uint8_t* __restrict__ data, const uint64_t* __restrict__ col_len, const uint64_t* __restrict__ blk_off,
    uint32_t n_chunks, uint64_t chunk_size, uint32_t wil, uint8_t* __restrict__ out, uint64_t out_n, uint32_t cap,
    uint32_t* __restrict__ status) {
    extern __shared__ __align__(16) uint8_t smem[];
    __shared__ SegTable T_;
    __shared__ uint32_t s_len[32];
    __shared__ uint32_t s_bad;

    const uint32_t lane = lane_id(), wid = threadIdx.x >> 5, tid = threadIdx.x;
    const uint32_t chunk = blockIdx.x / (32 / LANES_PER_BLOCK);
    const uint32_t L0 = (blockIdx.x % (32 / LANES_PER_BLOCK)) * LANES_PER_BLOCK;
    if (chunk >= n_chunks) return;
    const uint32_t nv = (uint32_t)(chunk_size / 32u / sizeof(T));
    const uint8_t* sbuf = smem + wid * cap;
    const uint64_t b0 = blk_off[chunk], b1 = blk_off[chunk + 1];
    const uint8_t* block = data + b0;

    if (wid == 0) {
        const uint64_t l64 = col_len[32ull * chunk + lane];
        uint32_t bad = (l64 > cap - 144) ? 1u : 0u;
        const uint32_t len = bad ? 0u : (uint32_t)l64;
        const uint32_t nw = (len + 3) >> 2;
        uint32_t tot = warp_incl_scan(nw);
        tot = __shfl_sync(GD_FULL_MASK, tot, 31);
        if (b1 < b0 || (uint64_t)tot * 4 > b1 - b0) bad = 1;
        if ((reinterpret_cast<uintptr_t>(block) & 3u) != 0) bad = 1;
        bad = __any_sync(GD_FULL_MASK, bad);
        seg_build(&T_, nw);
        s_len[lane] = len;
        if (lane == 0) s_bad = bad;
    }
    __syncthreads();
    if (s_bad) {
        if (tid == 0 && status) atomicMax(status + chunk, (uint32_t)ST_CORRUPT);
        return;
    }
    load_lane_streams<LANES_PER_BLOCK>(T_, s_len, block, smem, cap, L0);

    const uint32_t t = L0 + wid;
    const uint32_t len = s_len[t];
    const uint64_t obase = (uint64_t)chunk * chunk_size;
    const uint64_t want = out_n > obase ? min(chunk_size, out_n - obase) / sizeof(T) : 0;
    const uint32_t err = lane_warp<T>(sbuf, len, nv, t, wil, reinterpret_cast<T*>(out + obase), want);
    if (lane == 0 && err != ST_OK && status) atomicMax(status + chunk, err);
}

}  // namespace rlev1
}  // namespace gd

extern "C" gd_status_t gd_rlev1_decode(const uint8_t* d_data, const uint64_t* d_col_len, const uint64_t* d_blk_off,
                                       uint32_t n_chunks, uint64_t chunk_size, uint32_t comp_col_len,
                                       uint32_t elem_bytes, uint8_t* d_out, uint64_t out_n_bytes,
                                       uint32_t max_lane_bytes, uint32_t* d_status, gd_stream_t stream) {
    if (n_chunks == 0) return GD_OK;
    if (!d_data || !d_col_len || !d_blk_off || !d_out) return GD_ERR_INVALID_ARG;
    if (!(elem_bytes == 4 || elem_bytes == 8)) return GD_ERR_UNSUPPORTED;
    if (comp_col_len == 0 || comp_col_len % elem_bytes) return GD_ERR_INVALID_ARG;
    if (chunk_size == 0 || chunk_size % (32ull * comp_col_len) || chunk_size > (1ull << 31)) return GD_ERR_INVALID_ARG;
    if (out_n_bytes > chunk_size * (uint64_t)n_chunks || out_n_bytes <= chunk_size * (uint64_t)(n_chunks - 1))
        return GD_ERR_INVALID_ARG;
    if ((reinterpret_cast<uintptr_t>(d_out) % elem_bytes) != 0 || out_n_bytes % elem_bytes) return GD_ERR_INVALID_ARG;
    using namespace gd::rlev1;
    const uint32_t wil = comp_col_len / elem_bytes;
    const uint32_t nv = (uint32_t)(chunk_size / 32u / elem_bytes);
    // shared memory per lane stream: the caller's bound on the longest lane
    // stream if given, else the longest a valid stream of nv values can be
    // (a bound above the longest valid stream is clamped: longer lanes are corrupt)
    const uint32_t cap =
        max_lane_bytes ? min(lane_cap(max_lane_bytes), stream_cap(nv, elem_bytes)) : stream_cap(nv, elem_bytes);
    const int lpb = gd_tune_get(GD_TUNE_RLEV1_LANES_PER_BLOCK) == 4 ? 4 : 8;
    const uint32_t smem = (uint32_t)lpb * cap;
    if (smem > 200 * 1024) return GD_ERR_UNSUPPORTED;
    cudaStream_t s = (cudaStream_t)stream;
    if (d_status && cudaMemsetAsync(d_status, 0, 4ull * n_chunks, s) != cudaSuccess) return GD_ERR_CUDA;
    auto go = [&](auto kern, int lanes) {
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        kern<<<n_chunks * (32 / lanes), lanes * 32, smem, s>>>(d_data, d_col_len, d_blk_off, n_chunks, chunk_size, wil,
                                                            d_out, out_n_bytes, cap, d_status);
    };
    if (elem_bytes == 4) {
        if (lpb == 4) go(decode_kernel<uint32_t, 4>, 4);
        else go(decode_kernel<uint32_t, 8>, 8);
    } else {
        if (lpb == 4) go(decode_kernel<uint64_t, 4>, 4);
        else go(decode_kernel<uint64_t, 8>, 8);
    }
    return cudaGetLastError() == cudaSuccess ? GD_OK : GD_ERR_CUDA;
}
