// lzss.cu -- LZSS (32-column interleaved container) decoder for sm_100a:
// one warp per chunk (the warp-level decoder is in lzss.cuh).
#include "lzss.cuh"

namespace gd {
namespace lzss {

// WPB: warps (chunks) per block (GD_TUNE_LZSS_WARPS_PER_BLOCK 2 / 4 / 8; also
// the path for chunks too large to stage in shared memory)
template <int WPB>
__global__ void __launch_bounds__(WPB * 32) decode_kernel(const uint8_t* __restrict__ data,
                                                         const uint64_t* __restrict__ blk_off,
                                                         const uint64_t* __restrict__ col_len,
                                                         const uint8_t* __restrict__ col_map, uint32_t n_chunks,
                                                         uint64_t chunk_size, uint8_t* out,
                                                         uint32_t* __restrict__ status) {
    extern __shared__ __align__(16) uint8_t smem[];
    const uint32_t wid = threadIdx.x >> 5;
    const uint32_t chunk = blockIdx.x * WPB + wid;
    if (chunk >= n_chunks) return;
    const uint64_t b0 = blk_off[chunk], b1 = blk_off[chunk + 1];
    uint32_t err;
    if (b1 < b0) {
        err = ST_CORRUPT;
    } else {
        err = chunk_warp(data + b0, b1 - b0, col_len + 32ull * chunk, col_map + 32ull * chunk, chunk_size,
                         out + (uint64_t)chunk * chunk_size, smem + wid * WARP_SMEM);
    }
    if (lane_id() == 0) put_status(status, chunk, err);
}

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
    // the staged decoder holds a whole chunk in shared memory; it needs
    // 16-byte aligned output for its row stores
    const uint32_t staged = staged_smem(chunk_size);
    const int k = gd_tune_get(GD_TUNE_LZSS_WARPS_PER_BLOCK);
    const uint32_t cs = cols_smem(chunk_size);
    if ((k == 0 || k == 256 || k == 512) && cs <= 227u * 1024u) {
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
    if (k <= 1 && staged <= 227u * 1024u && (reinterpret_cast<uintptr_t>(d_out) & 15u) == 0) {
        cudaFuncSetAttribute(decode_staged_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, staged);
        cudaFuncSetAttribute(decode_staged_kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                             cudaSharedmemCarveoutMaxShared);
        decode_staged_kernel<<<n_chunks, 32, staged, (cudaStream_t)stream>>>(d_data, d_blk_off, d_col_len, d_col_map,
                                                                            n_chunks, chunk_size, d_out, d_status);
        return cudaGetLastError() == cudaSuccess ? GD_OK : GD_ERR_CUDA;
    }
    const int wpb = (k == 2 || k == 8) ? k : 4;
    auto go = [&](auto kern) {
        const uint32_t smem = (uint32_t)wpb * WARP_SMEM;
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        kern<<<(n_chunks + wpb - 1) / wpb, wpb * 32, smem, (cudaStream_t)stream>>>(d_data, d_blk_off, d_col_len,
                                                                                d_col_map, n_chunks, chunk_size,
                                                                                d_out, d_status);
    };
    if (wpb == 2) go(decode_kernel<2>);
    else if (wpb == 8) go(decode_kernel<8>);
    else go(decode_kernel<4>);
    return cudaGetLastError() == cudaSuccess ? GD_OK : GD_ERR_CUDA;
}
