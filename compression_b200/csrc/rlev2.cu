// rlev2.cu -- RLE v2 (transposed container) decoder for sm_100a.
//
// A block of 8 (or 4) warps owns as many adjacent lane streams of one chunk
// and copies them from the interleaved block into shared memory; then each
// warp decodes its stream with decode_stream (rlev2.cuh): lane 0 walks the
// run boundaries in batches, the lanes decode the headers and produce 32
// values per round.  After the copy the warps of a block never wait on each
// other, so one warp's walk overlaps the others' expansion.
// The grammar and its corrections to the reference are in rlev2.cuh.
#include "rlev2.cuh"

namespace gd {
namespace rlev2 {

template <int LANES_PER_BLOCK>
__global__ void __launch_bounds__(LANES_PER_BLOCK * 32) decode_kernel(
    const uint8_t* __restrict__ data, const uint64_t* __restrict__ col_len, const uint64_t* __restrict__ blk_off,
    uint32_t n_chunks, uint64_t chunk_size, uint32_t ru, uint8_t* __restrict__ out, uint64_t out_n, uint32_t cap,
    uint32_t* __restrict__ status) {
    extern __shared__ __align__(16) uint8_t smem[];
    __shared__ SegTable T_;
    __shared__ uint32_t s_len[32];
    __shared__ uint32_t s_bad;
    __shared__ WarpRuns R[LANES_PER_BLOCK];

    const uint32_t lane = lane_id(), wid = threadIdx.x >> 5, tid = threadIdx.x;
    const uint32_t chunk = blockIdx.x / (32 / LANES_PER_BLOCK);
    const uint32_t L0 = (blockIdx.x % (32 / LANES_PER_BLOCK)) * LANES_PER_BLOCK;
    if (chunk >= n_chunks) return;  // block-uniform
    const uint32_t nv = (uint32_t)(chunk_size / 256u);  // values per lane stream
    const uint64_t b0 = blk_off[chunk], b1 = blk_off[chunk + 1];
    const uint8_t* block = data + b0;

    // ---- segment table of the chunk (warp 0) ----
    if (wid == 0) {
        const uint64_t l64 = col_len[32ull * chunk + lane];
        uint32_t bad = (l64 > cap - 32) ? 1u : 0u;  // 16 zeroed + 16 readable bytes follow a stream
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

    // ---- copy this block's 8 lane streams into shared memory ----
    load_lane_streams<LANES_PER_BLOCK>(T_, s_len, block, smem, cap, L0);

    const uint32_t t = L0 + wid;  // the lane stream this warp expands
    const uint8_t* sbuf = smem + wid * cap;
    const uint64_t obase = (uint64_t)chunk * chunk_size;
    const uint64_t want_vals = out_n > obase ? min(chunk_size, out_n - obase) / 8 : 0;  // values of this chunk kept
    uint64_t* outv = reinterpret_cast<uint64_t*>(out + obase);
    const uint32_t plen = s_len[t];
    const uint32_t werr = decode_stream(sbuf, plen, nv, t, ru, outv, want_vals, R[wid]);
    if (lane == 0 && werr != ST_OK && status) atomicMax(status + chunk, werr);
}

}  // namespace rlev2
}  // namespace gd

extern "C" gd_status_t gd_rlev2_decode(const uint8_t* d_data, const uint64_t* d_col_len, const uint64_t* d_blk_off,
                                       uint32_t n_chunks, uint64_t chunk_size, uint32_t read_unit,
                                       uint8_t* d_out, uint64_t out_n_bytes, uint32_t max_lane_bytes,
                                       uint32_t* d_status, gd_stream_t stream) {
    if (n_chunks == 0) return GD_OK;
    if (!d_data || !d_col_len || !d_blk_off || !d_out) return GD_ERR_INVALID_ARG;
    if (read_unit == 0) return GD_ERR_UNSUPPORTED;
    if (chunk_size == 0 || chunk_size % (256ull * read_unit) || chunk_size > (1ull << 31)) return GD_ERR_INVALID_ARG;
    if (out_n_bytes > chunk_size * (uint64_t)n_chunks || out_n_bytes <= chunk_size * (uint64_t)(n_chunks - 1))
        return GD_ERR_INVALID_ARG;
    if ((reinterpret_cast<uintptr_t>(d_out) & 7u) != 0 || out_n_bytes % 8) return GD_ERR_INVALID_ARG;
    using namespace gd::rlev2;
    const uint32_t nv = (uint32_t)(chunk_size / 256u);
    // shared memory per lane stream: the caller's bound on the longest lane
    // stream if given, else the longest a valid stream of nv values can be
    // (a bound above the longest valid stream is clamped: longer lanes are
    // corrupt), plus 16 bytes for the header parser's 24-byte window reads
    const uint32_t cap = (max_lane_bytes ? min(lane_cap(max_lane_bytes), stream_cap(nv)) : stream_cap(nv)) + 16u;
    // 8 lane streams per block by default (a row's 8 words are one full
    // 32-byte sector, and 0.297 -> 0.288 ms on 256 MiB), 4 when 8 streams do
    // not fit in shared memory
    const int knob = gd_tune_get(GD_TUNE_RLEV2_LANES_PER_BLOCK);
    const int lpb = knob == 4 ? 4 : (knob == 8 || 8u * cap <= 200u * 1024u) ? 8 : 4;
    const uint32_t smem = (uint32_t)lpb * cap;
    if (smem > 200 * 1024) return GD_ERR_UNSUPPORTED;  // lane streams must fit in shared memory
    cudaStream_t s = (cudaStream_t)stream;
    // per-chunk status is the max over the chunk's lane streams
    if (d_status && cudaMemsetAsync(d_status, 0, 4ull * n_chunks, s) != cudaSuccess) return GD_ERR_CUDA;
    auto go = [&](auto kern, int lanes) {
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        kern<<<n_chunks * (32 / lanes), lanes * 32, smem, s>>>(d_data, d_col_len, d_blk_off, n_chunks, chunk_size,
                                                            read_unit, d_out, out_n_bytes, cap, d_status);
    };
    if (lpb == 8) go(decode_kernel<8>, 8);
    else go(decode_kernel<4>, 4);
    return cudaGetLastError() == cudaSuccess ? GD_OK : GD_ERR_CUDA;
}
