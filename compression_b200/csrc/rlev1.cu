// rlev1.cu -- RLE v1 (ORC-style integer RLE v1) decoder for sm_100a.
//
// Grammar (restated from decoder_warp, include/rle_v1/decoder.h:278-423):
// int8 header h; h < 0: -h literal values, each an unsigned LEB128 varint;
// h >= 0: a run of h+3 values, int8 delta then varint base, v_i = base+i*delta.
// Lane t of a chunk owns elements (i / wil)*32*wil + t*wil + i % wil,
// wil = COMP_COL_LEN / sizeof(T); a lane stream ends once it has produced
// chunk_size/32 bytes (decoder.h:283,291).
//
// The reference pairs a reader warp and a decoder warp per chunk (spin
// queues, one byte fetched per funnel-shift call, one scalar store per
// value).  Here every lane stream gets a whole warp (same block loader as
// RLE v2: 8 adjacent lane streams per block, copied with fully used 32-byte
// row sectors):
//   * runs are closed form: lane i writes base + i*delta;
//   * a literal group is decoded 32 values at a time: the lanes load a
//     128-byte window, ballot the varint terminators (bytes < 0x80), and lane
//     j finds the j-th terminator with a select over the 128-bit mask, so
//     every lane knows where its varint starts and ends and decodes it alone.
#include "interleave.cuh"

namespace gd {
namespace rlev1 {

constexpr int LANES_PER_BLOCK = 8;

// Largest lane stream for nv values: literal varints of up to 10 bytes plus
// one header per 127 values; +128 tail for terminator windows.
__host__ __device__ constexpr uint32_t stream_cap(uint32_t nv, uint32_t eb) {
    return (((eb == 8 ? 10u : 5u) * nv + nv / 127u + 64u + 15u) & ~15u) + 144u;
}

// Shared-memory bytes reserved for a lane stream of at most `n` bytes.
__host__ __device__ constexpr uint32_t lane_cap(uint32_t n) { return ((n + 15u) & ~15u) + 144u; }

// index (0-based) of the n-th set bit of the 128-bit mask m[0..3] (n < popc)
__device__ __forceinline__ uint32_t select128(const uint32_t m[4], uint32_t n) {
    uint32_t base = 0;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const uint32_t c = __popc(m[q]);
        if (n < c) return base + __fns(m[q], 0, (int)n + 1);
        n -= c;
        base += 32;
    }
    return 0xffffffffu;
}

template <typename T>
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
    T* outv = reinterpret_cast<T*>(out + obase);
    auto put = [&](uint32_t e, uint64_t v) {
        const uint64_t oe = (uint64_t)(e / wil) * 32u * wil + (uint64_t)t * wil + (e % wil);
        if (oe < want) outv[oe] = (T)v;
    };

    uint32_t err = ST_OK, pos = 0, g = 0;
    while (g < nv) {
        // ---- header (lane 0) ----
        uint32_t kind = 0, cnt = 0, next = 0, e = ST_OK;
        uint64_t base = 0, delta = 0;
        if (lane == 0) {
            uint32_t p = pos;
            if (p >= len) {
                e = ST_CORRUPT;
            } else {
                const uint32_t h = sbuf[p++];
                if (h & 0x80u) {
                    kind = 1;
                    cnt = 256u - h;
                } else if (p >= len) {
                    e = ST_CORRUPT;
                } else {
                    kind = 0;
                    cnt = h + 3u;
                    delta = (uint64_t)(int64_t)(int8_t)sbuf[p++];
                    uint32_t sh = 0, b;
                    do {
                        if (p >= len || sh > 63) {
                            e = ST_CORRUPT;
                            break;
                        }
                        b = sbuf[p++];
                        base |= (uint64_t)(b & 0x7fu) << sh;
                        sh += 7;
                    } while (b & 0x80u);
                    if (sizeof(T) == 4) base &= 0xffffffffull;
                }
            }
            next = p;
        }
        kind = __shfl_sync(GD_FULL_MASK, kind, 0);
        cnt = __shfl_sync(GD_FULL_MASK, cnt, 0);
        next = __shfl_sync(GD_FULL_MASK, next, 0);
        e = __shfl_sync(GD_FULL_MASK, e, 0);
        if (e != ST_OK) {
            err = e;
            break;
        }
        if (g + cnt > nv) {
            err = ST_OVERRUN;
            break;
        }
        if (kind == 0) {  // run: closed form
            base = ((uint64_t)__shfl_sync(GD_FULL_MASK, (uint32_t)(base >> 32), 0) << 32) |
                   __shfl_sync(GD_FULL_MASK, (uint32_t)base, 0);
            delta = ((uint64_t)__shfl_sync(GD_FULL_MASK, (uint32_t)(delta >> 32), 0) << 32) |
                    __shfl_sync(GD_FULL_MASK, (uint32_t)delta, 0);
            for (uint32_t i = lane; i < cnt; i += 32) put(g + i, base + (uint64_t)i * delta);
            g += cnt;
            pos = next;
            continue;
        }
        // literal group: cnt varints starting at `next`
        uint32_t p = next, rem = cnt;
        while (rem) {
            uint32_t m[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const uint32_t bpos = p + 32u * q + lane;
                const bool term = (bpos < len) && !(sbuf[bpos] & 0x80u);
                m[q] = __ballot_sync(GD_FULL_MASK, term);
            }
            const uint32_t nterm = __popc(m[0]) + __popc(m[1]) + __popc(m[2]) + __popc(m[3]);
            if (nterm == 0) {  // no varint ends within 128 bytes (or the stream ran out)
                err = ST_CORRUPT;
                break;
            }
            const uint32_t take = min(min(rem, nterm), 32u);
            if (lane < take) {
                const uint32_t end = select128(m, lane);
                const uint32_t beg = lane ? select128(m, lane - 1) + 1 : 0;
                uint64_t v = 0;
                uint32_t sh = 0;
                for (uint32_t k = beg; k <= end; ++k, sh += 7)
                    if (sh < 64) v |= (uint64_t)(sbuf[p + k] & 0x7fu) << sh;
                put(g + lane, v);
            }
            p += select128(m, take - 1) + 1;
            g += take;
            rem -= take;
        }
        if (err != ST_OK) break;
        pos = p;
    }
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
    const uint32_t cap = max_lane_bytes ? lane_cap(max_lane_bytes) : stream_cap(nv, elem_bytes);
    const uint32_t smem = LANES_PER_BLOCK * cap;
    if (smem > 200 * 1024) return GD_ERR_UNSUPPORTED;
    cudaStream_t s = (cudaStream_t)stream;
    if (d_status && cudaMemsetAsync(d_status, 0, 4ull * n_chunks, s) != cudaSuccess) return GD_ERR_CUDA;
    const uint32_t grid = n_chunks * (32 / LANES_PER_BLOCK);
    if (elem_bytes == 4) {
        cudaFuncSetAttribute(decode_kernel<uint32_t>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        decode_kernel<uint32_t><<<grid, LANES_PER_BLOCK * 32, smem, s>>>(d_data, d_col_len, d_blk_off, n_chunks,
                                                                        chunk_size, wil, d_out, out_n_bytes, cap, d_status);
    } else {
        cudaFuncSetAttribute(decode_kernel<uint64_t>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        decode_kernel<uint64_t><<<grid, LANES_PER_BLOCK * 32, smem, s>>>(d_data, d_col_len, d_blk_off, n_chunks,
                                                                        chunk_size, wil, d_out, out_n_bytes, cap, d_status);
    }
    return cudaGetLastError() == cudaSuccess ? GD_OK : GD_ERR_CUDA;
}
