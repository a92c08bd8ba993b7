// brle_trans.cu -- byte-RLE flag-byte interleaved container decoder for sm_100a
// (1-byte symbols, and the 4-byte-symbol variant of brle_gpu_4B.h).
//
// Container (brle_trans::compress_gpu / decompress_gpu, include/brle/
// brle_trans.h:563-791): a chunk (4 KiB in the reference) is 32 columns,
// column q = bytes 4q + 128k .. +3.  Each column is one stream: a flag byte,
// then 8 items, flag bits LSB first; bit 1 = one literal byte, bit 0 = a count
// byte then a value byte written count times; after the 8th item the next
// byte is a flag byte again.  The streams are ranked by descending length
// (col_len sorted, col_map = rank -> column) and interleaved in 4-byte words
// over the ranks still active in each row; blocks start 128-byte aligned.
//
// The reference gives each stream one thread that reads its bytes one at a
// time from global memory.  Here one warp decodes a chunk: the chunk's block
// is staged in shared memory with 16-byte loads, lane r decodes rank r from
// shared memory (its words located incrementally, row by row), writes its
// column into a shared-memory copy of the chunk, and the warp stores the
// chunk with coalesced 16-byte stores.
#include "gd_common.cuh"

namespace gd {
namespace brlet {

constexpr int WPB = 4;                 // warps (chunks in flight) per block
constexpr uint32_t MAX_CHUNK = 8192;   // chunk_size <= 8192, multiple of 128

// Longest valid column stream for L output bytes: every byte a literal, plus
// the flag bytes and a reserved trailing one.
__host__ __device__ constexpr uint32_t col_max(uint32_t L) { return 2u + L + (L + 7u) / 8u; }
__host__ __device__ constexpr uint32_t in_cap(uint32_t L) { return 32u * ((col_max(L) + 3u) & ~3u); }
__host__ __device__ constexpr uint32_t warp_smem(uint32_t chunk) {
    return ((in_cap(chunk / 32u) + 15u) & ~15u) + chunk;
}

// SYM = 1: brle_trans; SYM = 4: the 4-byte-symbol variant (brle::
// decompress_func, include/brle/brle_gpu_4B.h:75-223): literals are 4-byte
// symbols and a run item is a count byte followed by the symbol.
template <int SYM>
__global__ void __launch_bounds__(WPB * 32) decode_kernel(const uint8_t* __restrict__ data,
                                                         const uint64_t* __restrict__ blk_off,
                                                         const uint64_t* __restrict__ col_len,
                                                         const uint8_t* __restrict__ col_map, uint32_t n_chunks,
                                                         uint32_t chunk_size, uint8_t* __restrict__ out,
                                                         uint64_t out_n, uint32_t* __restrict__ status) {
    extern __shared__ __align__(16) uint8_t smem[];
    __shared__ uint32_t s_len[WPB][32];
    const uint32_t lane = lane_id(), wid = threadIdx.x >> 5;
    const uint32_t L = chunk_size / 32u;
    const uint32_t icap = (in_cap(L) + 15u) & ~15u;
    uint8_t* sin = smem + wid * warp_smem(chunk_size);
    uint8_t* tile = sin + icap;
    uint32_t* slen = s_len[wid];
    for (uint32_t c = blockIdx.x * WPB + wid; c < n_chunks; c += gridDim.x * WPB) {
        const uint64_t b0 = blk_off[c], b1 = blk_off[c + 1];
        const uint64_t obase = (uint64_t)c * chunk_size;
        const uint64_t l64 = col_len[32ull * c + lane];
        const uint32_t col = col_map[32ull * c + lane];
        uint32_t bad = (l64 > col_max(L) || col >= 32u || b1 < b0 || obase >= out_n) ? 1u : 0u;
        const uint32_t len = bad ? 0u : (uint32_t)l64;
        // ranks must be sorted by descending length and col_map a permutation
        const uint32_t prev = __shfl_up_sync(GD_FULL_MASK, len, 1);
        if (lane > 0 && prev < len) bad = 1;
        if (__reduce_or_sync(GD_FULL_MASK, col < 32u ? 1u << col : 0u) != GD_FULL_MASK) bad = 1;
        const uint32_t words = (len + 3u) >> 2;
        const uint32_t tot = __shfl_sync(GD_FULL_MASK, warp_incl_scan(words), 31) * 4u;
        if (!bad && (uint64_t)tot > b1 - b0) bad = 1;
        const uint8_t* blk = data + b0;
        if ((reinterpret_cast<uintptr_t>(blk) & 3u) != 0) bad = 1;
        if (__any_sync(GD_FULL_MASK, bad)) {
            if (lane == 0) put_status(status, c, ST_CORRUPT);
            continue;
        }
        slen[lane] = len;
        // ---- stage the block ----
        if ((reinterpret_cast<uintptr_t>(blk) & 15u) == 0) {
            for (uint32_t i = lane; i < tot / 16u; i += 32) reinterpret_cast<uint4*>(sin)[i] = reinterpret_cast<const uint4*>(blk)[i];
            for (uint32_t i = (tot & ~15u) / 4u + lane; i < tot / 4u; i += 32)
                reinterpret_cast<uint32_t*>(sin)[i] = reinterpret_cast<const uint32_t*>(blk)[i];
        } else {
            for (uint32_t i = lane; i < tot / 4u; i += 32)
                reinterpret_cast<uint32_t*>(sin)[i] = reinterpret_cast<const uint32_t*>(blk)[i];
        }
        __syncwarp();
        // ---- decode rank `lane` into column `col` of the tile ----
        uint32_t err = ST_OK;
        {
            uint32_t act = 32;  // ranks active in the current row (lengths > 4*row)
            while (act > 0 && slen[act - 1] == 0) --act;
            uint32_t row_base = 0, row = 0;  // byte offset of the current row
            uint32_t o = 0, block = 0, head = 0, cnt = 0;
            bool pend = false;  // a count byte waits for its value byte
            uint32_t nb = 0, symv = 0;  // SYM 4: symbol bytes still to come, the symbol so far
            for (uint32_t j = 0; j < len; ++j) {
                if (j && (j & 3u) == 0) {  // next row
                    row_base += 4u * act;
                    ++row;
                    while (act > 0 && slen[act - 1] <= 4u * row) --act;
                }
                const uint32_t v = sin[row_base + 4u * lane + (j & 3u)];
                if constexpr (SYM == 4) {
                    if (nb) {  // a symbol byte
                        symv |= v << (8u * (4u - nb));
                        if (--nb == 0) {
                            if (o + 4u * cnt > L) {
                                err = ST_OVERRUN;
                                break;
                            }
                            for (uint32_t k = 0; k < cnt; ++k, o += 4)
                                *reinterpret_cast<uint32_t*>(tile + (o >> 2) * 128u + col * 4u) = symv;
                        }
                        continue;
                    }
                    if (block == 0) {
                        head = v;
                        block = 1;
                        continue;
                    }
                    const uint32_t lit = head & 1u;
                    head >>= 1;
                    if (++block == 9) block = 0;
                    if (lit) {  // v is the symbol's first byte
                        cnt = 1;
                        symv = v;
                        nb = 3;
                    } else {  // v is the count
                        cnt = v;
                        symv = 0;
                        nb = 4;
                    }
                    continue;
                }
                if (pend) {
                    pend = false;
                    if (o + cnt > L) {
                        err = ST_OVERRUN;
                        break;
                    }
                    for (uint32_t k = 0; k < cnt; ++k, ++o) tile[(o >> 2) * 128u + col * 4u + (o & 3u)] = (uint8_t)v;
                    continue;
                }
                if (block == 0) {
                    head = v;
                    block = 1;
                    continue;
                }
                const uint32_t lit = head & 1u;
                head >>= 1;
                if (++block == 9) block = 0;
                if (lit) {
                    if (o >= L) {
                        err = ST_OVERRUN;
                        break;
                    }
                    tile[(o >> 2) * 128u + col * 4u + (o & 3u)] = (uint8_t)v;
                    ++o;
                } else {
                    cnt = v;
                    pend = true;
                }
            }
            if (err == ST_OK && (pend || nb || o != L)) err = ST_CORRUPT;
        }
        const uint32_t e = __reduce_max_sync(GD_FULL_MASK, err);
        __syncwarp();
        // ---- store the chunk ----
        if (e == ST_OK) {
            const uint32_t want = (uint32_t)(out_n - obase < chunk_size ? out_n - obase : chunk_size);
            uint8_t* dst = out + obase;
            if ((reinterpret_cast<uintptr_t>(dst) & 15u) == 0) {
                for (uint32_t i = lane; i < want / 16u; i += 32)
                    reinterpret_cast<uint4*>(dst)[i] = reinterpret_cast<const uint4*>(tile)[i];
                for (uint32_t i = (want & ~15u) + lane; i < want; i += 32) dst[i] = tile[i];
            } else {
                for (uint32_t i = lane; i < want; i += 32) dst[i] = tile[i];
            }
        }
        if (lane == 0) put_status(status, c, e);
        __syncwarp();
    }
}

}  // namespace brlet
}  // namespace gd

template <int SYM>
static gd_status_t flag_decode(const uint8_t* d_data, const uint64_t* d_blk_off, const uint64_t* d_col_len,
                               const uint8_t* d_col_map, uint32_t n_chunks, uint64_t chunk_size, uint8_t* d_out,
                               uint64_t out_n_bytes, uint32_t* d_status, gd_stream_t stream) {
    using namespace gd::brlet;
    if (n_chunks == 0) return GD_OK;
    if (!d_data || !d_blk_off || !d_col_len || !d_col_map || !d_out) return GD_ERR_INVALID_ARG;
    if (chunk_size == 0 || chunk_size % 128 || chunk_size > MAX_CHUNK) return GD_ERR_INVALID_ARG;
    if (out_n_bytes > chunk_size * (uint64_t)n_chunks || out_n_bytes <= chunk_size * (uint64_t)(n_chunks - 1))
        return GD_ERR_INVALID_ARG;
    const uint32_t smem = WPB * warp_smem((uint32_t)chunk_size);
    if (cudaFuncSetAttribute(decode_kernel<SYM>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess)
        return GD_ERR_CUDA;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    uint32_t grid = (n_chunks + WPB - 1) / WPB;
    const uint32_t cap = (uint32_t)sms * 16;
    if (grid > cap) grid = cap;
    decode_kernel<SYM><<<grid, WPB * 32, smem, (cudaStream_t)stream>>>(d_data, d_blk_off, d_col_len, d_col_map,
                                                                      n_chunks, (uint32_t)chunk_size, d_out,
                                                                      out_n_bytes, d_status);
    return cudaGetLastError() == cudaSuccess ? GD_OK : GD_ERR_CUDA;
}

extern "C" gd_status_t gd_brle_trans_decode(const uint8_t* d_data, const uint64_t* d_blk_off, const uint64_t* d_col_len,
                                            const uint8_t* d_col_map, uint32_t n_chunks, uint64_t chunk_size,
                                            uint8_t* d_out, uint64_t out_n_bytes, uint32_t* d_status,
                                            gd_stream_t stream) {
    return flag_decode<1>(d_data, d_blk_off, d_col_len, d_col_map, n_chunks, chunk_size, d_out, out_n_bytes,
                          d_status, stream);
}

extern "C" gd_status_t gd_brle_trans4_decode(const uint8_t* d_data, const uint64_t* d_blk_off,
                                             const uint64_t* d_col_len, const uint8_t* d_col_map, uint32_t n_chunks,
                                             uint64_t chunk_size, uint8_t* d_out, uint64_t out_n_bytes,
                                             uint32_t* d_status, gd_stream_t stream) {
    return flag_decode<4>(d_data, d_blk_off, d_col_len, d_col_map, n_chunks, chunk_size, d_out, out_n_bytes,
                          d_status, stream);
}
