// lzss.cu -- LZSS (32-column interleaved container) decoder for sm_100a.
// The decoders are in lzss.cuh; GD_TUNE_LZSS_WARPS_PER_BLOCK selects one.
#include "lzss.cuh"

namespace gd {
namespace lzss {

// One warp per block and chunk; the chunk's output is staged in shared memory
// (chunk_warp_staged), so blocks per SM = shared memory / staged_smem(chunk).
__global__ void __launch_bounds__(32) decode_staged_kernel(const uint8_t* __restrict__ data,
                                                           const uint64_t* __restrict__ blk_off,
                                                           const uint64_t* __restrict__ col_len,
                                                           const uint8_t* __restrict__ col_map, uint32_t n_chunks,
                                                           uint64_t chunk_size, uint8_t* out,
                                                           uint32_t* __restrict__ status) {
    extern __shared__ __align__(16) uint8_t smem[];
    const uint32_t chunk = blockIdx.x;
    if (chunk >= n_chunks) return;
    const uint64_t b0 = blk_off[chunk], b1 = blk_off[chunk + 1];
    uint32_t err;
    if (b1 < b0) {
        err = ST_CORRUPT;
    } else {
        err = chunk_warp_staged(data + b0, b1 - b0, col_len + 32ull * chunk, col_map + 32ull * chunk, chunk_size,
                                out + (uint64_t)chunk * chunk_size, smem);
    }
    if (lane_id() == 0) put_status(status, chunk, err);
}

// WPB warps per block, one chunk per warp, one lane per column, output in
// rounds of RB column bytes (chunk_warp_groups).
template <int WPB, uint32_t RB, uint32_t GR>
__global__ void __launch_bounds__(WPB * 32) decode_groups_kernel(const uint8_t* __restrict__ data,
                                                                const uint64_t* __restrict__ blk_off,
                                                                const uint64_t* __restrict__ col_len,
                                                                const uint8_t* __restrict__ col_map,
                                                                uint32_t n_chunks, uint64_t chunk_size, uint8_t* out,
                                                                uint32_t* __restrict__ status) {
    extern __shared__ __align__(16) uint8_t smem[];
    const uint32_t wid = threadIdx.x >> 5;
    const uint32_t chunk = blockIdx.x * WPB + wid;
    if (chunk >= n_chunks) return;  // warp-uniform
    const uint64_t b0 = blk_off[chunk], b1 = blk_off[chunk + 1];
    uint32_t err;
    if (b1 < b0) {
        err = ST_CORRUPT;
    } else {
        err = chunk_warp_groups<RB, GR>(data + b0, b1 - b0, col_len + 32ull * chunk, col_map + 32ull * chunk,
                                        chunk_size, out + (uint64_t)chunk * chunk_size,
                                        smem + wid * group_warp_smem(RB, GR));
    }
    if (lane_id() == 0) put_status(status, chunk, err);
}

// One block of 32*G threads per chunk, G lanes per column (chunk_block_cols).
template <uint32_t G>
__global__ void __launch_bounds__(32 * G) decode_cols_kernel(const uint8_t* __restrict__ data,
                                                             const uint64_t* __restrict__ blk_off,
                                                             const uint64_t* __restrict__ col_len,
                                                             const uint8_t* __restrict__ col_map, uint32_t n_chunks,
                                                             uint64_t chunk_size, uint8_t* out,
                                                             uint32_t* __restrict__ status) {
    extern __shared__ __align__(16) uint8_t smem[];
    const uint32_t chunk = blockIdx.x;
    if (chunk >= n_chunks) return;  // block-uniform
    const uint64_t b0 = blk_off[chunk], b1 = blk_off[chunk + 1];
    uint32_t err;
    if (b1 < b0) {
        err = ST_CORRUPT;
    } else {
        err = chunk_block_cols<G>(data + b0, b1 - b0, col_len + 32ull * chunk, col_map + 32ull * chunk, chunk_size,
                                  out + (uint64_t)chunk * chunk_size, smem);
    }
    if (threadIdx.x == 0) put_status(status, chunk, err);
}

}  // namespace lzss
}  // namespace gd

extern "C" gd_status_t gd_lzss_decode(const uint8_t* d_data, const uint64_t* d_blk_off, const uint64_t* d_col_len,
                                      const uint8_t* d_col_map, uint32_t n_chunks, uint64_t chunk_size,
                                      uint8_t* d_out, uint64_t out_n_bytes, uint32_t* d_status,
                                      gd_stream_t stream) {
    if (n_chunks == 0) return GD_OK;
    if (!d_data || !d_blk_off || !d_col_len || !d_col_map || !d_out) return GD_ERR_INVALID_ARG;
    if (chunk_size == 0 || chunk_size % 128 || chunk_size > (1ull << 31)) return GD_ERR_INVALID_ARG;
    // whole chunks are written: match sources may lie in the zero padding of
    // a short final chunk, so the output must hold n_chunks * chunk_size
    if (out_n_bytes != chunk_size * (uint64_t)n_chunks) return GD_ERR_INVALID_ARG;
    if ((reinterpret_cast<uintptr_t>(d_out) & 3u) != 0) return GD_ERR_INVALID_ARG;
    using namespace gd::lzss;
    const int k = gd_tune_get(GD_TUNE_LZSS_WARPS_PER_BLOCK);
    const uint32_t cs = cols_smem(chunk_size);
    if ((k == 256 || k == 512) && cs <= 227u * 1024u) {
        auto go = [&](auto kern, uint32_t threads) {
            cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, cs);
            cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared);
            kern<<<n_chunks, threads, cs, (cudaStream_t)stream>>>(d_data, d_blk_off, d_col_len, d_col_map, n_chunks,
                                                                 chunk_size, d_out, d_status);
        };
        if (k == 256) go(decode_cols_kernel<8>, 256);
        else go(decode_cols_kernel<16>, 512);
        return cudaGetLastError() == cudaSuccess ? GD_OK : GD_ERR_CUDA;
    }
    // the staged decoder holds a whole chunk in shared memory; it needs
    // 16-byte aligned output for its row stores
    const uint32_t staged = staged_smem(chunk_size);
    if (k == 1 && staged <= 227u * 1024u && (reinterpret_cast<uintptr_t>(d_out) & 15u) == 0) {
        cudaFuncSetAttribute(decode_staged_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, staged);
        cudaFuncSetAttribute(decode_staged_kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                             cudaSharedmemCarveoutMaxShared);
        decode_staged_kernel<<<n_chunks, 32, staged, (cudaStream_t)stream>>>(d_data, d_blk_off, d_col_len, d_col_map,
                                                                            n_chunks, chunk_size, d_out, d_status);
        return cudaGetLastError() == cudaSuccess ? GD_OK : GD_ERR_CUDA;
    }
    // group decoder (any chunk size): one chunk per 32-thread block with
    // 320-byte rounds, or (k == 4) four per block with 256-byte rounds (the
    // batch decoder's shape)
    auto go = [&](auto kern, uint32_t wpb, uint32_t rb) {
        const uint32_t smem = wpb * group_warp_smem(rb, 64);
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared);
        kern<<<(n_chunks + wpb - 1) / wpb, wpb * 32, smem, (cudaStream_t)stream>>>(d_data, d_blk_off, d_col_len,
                                                                                d_col_map, n_chunks, chunk_size,
                                                                                d_out, d_status);
    };
    if (k == 4) go(decode_groups_kernel<4, 256, 64>, 4, 256);
    else go(decode_groups_kernel<1, 320, 64>, 1, 320);
    return cudaGetLastError() == cudaSuccess ? GD_OK : GD_ERR_CUDA;
}
