// rlev1.cu -- RLE v1 (ORC-style integer RLE v1) decoder for sm_100a.
//
// Grammar (restated from decoder_warp, include/rle_v1/decoder.h:278-423):
// int8 header h; h < 0: -h literal values, each an unsigned LEB128 varint;
// h >= 0: a run of h+3 values, int8 delta then varint base, v_i = base+i*delta.
// Lane t of a chunk owns elements (i / wil)*32*wil + t*wil + i % wil,
// wil = COMP_COL_LEN / sizeof(T).
//
// One warp decodes one chunk, lane t decoding lane stream t (the reference's
// decoder warp), but: the lane streams are read straight out of the
// interleaved block through the segment table into per-lane shared-memory
// rings (no separate reader warp or spin queues); every round each lane
// produces exactly its wil-element slice of one output row into shared
// memory, and the warp writes the 32*COMP_COL_LEN-byte row with coalesced
// stores.  Every byte read is checked against the lane's stream length and
// malformed input ends the chunk with an error status.
#include "interleave.cuh"

namespace gd {
namespace rlev1 {

constexpr int WPB = 4;  // chunks (warps) per block

// per-lane stage stride: an odd number of elements past a 16-byte multiple,
// so lanes storing element i at the same time hit different banks
__host__ __device__ constexpr uint32_t stage_stride(uint32_t slice_bytes, uint32_t eb) {
    return ((slice_bytes + 15u) & ~15u) + eb;
}
__host__ __device__ constexpr uint32_t warp_smem(uint32_t slice_bytes, uint32_t eb) {
    return (uint32_t)sizeof(SegTable) + 32u * RING_STRIDE + 32u * stage_stride(slice_bytes, eb);
}

template <typename T>
__global__ void __launch_bounds__(WPB * 32) decode_kernel(const uint8_t* __restrict__ data,
                                                         const uint64_t* __restrict__ col_len,
                                                         const uint64_t* __restrict__ blk_off, uint32_t n_chunks,
                                                         uint64_t chunk_size, uint32_t wil,
                                                         uint8_t* __restrict__ out, uint64_t out_n,
                                                         uint32_t* __restrict__ status) {
    extern __shared__ __align__(16) uint8_t smem[];
    const uint32_t lane = lane_id(), wid = threadIdx.x >> 5;
    const uint32_t chunk = blockIdx.x * WPB + wid;
    if (chunk >= n_chunks) return;
    const uint32_t slice = wil * (uint32_t)sizeof(T);
    const uint32_t sstride = stage_stride(slice, (uint32_t)sizeof(T));
    uint8_t* wbase = smem + wid * warp_smem(slice, (uint32_t)sizeof(T));
    SegTable* T_ = reinterpret_cast<SegTable*>(wbase);
    uint8_t* ring = wbase + sizeof(SegTable);
    uint8_t* stage = ring + 32 * RING_STRIDE;

    uint32_t err = ST_OK;
    const uint64_t b0 = blk_off[chunk], b1 = blk_off[chunk + 1];
    const uint64_t len64 = col_len[32ull * chunk + lane];
    uint32_t len = len64 > 0x3fffffffull ? 0u : (uint32_t)len64;
    if (len64 > 0x3fffffffull) err = ST_CORRUPT;
    uint32_t nw = (len + 3) >> 2;
    // the block must hold every lane's padded stream
    uint32_t tot = warp_incl_scan(nw);
    tot = __shfl_sync(GD_FULL_MASK, tot, 31);
    if (b1 < b0 || (uint64_t)tot * 4 > b1 - b0) err = ST_CORRUPT;
    if ((reinterpret_cast<uintptr_t>(data + b0) & 3u) != 0) err = ST_CORRUPT;  // words are 4-byte loads
    if (__any_sync(GD_FULL_MASK, err != ST_OK)) {
        if (lane == 0) put_status(status, chunk, ST_CORRUPT);
        return;
    }
    const uint8_t* block = data + b0;
    seg_build(T_, nw);
    LaneWords lw;
    lw_init(lw, T_, nw);
    LaneRing r{ring + lane * RING_STRIDE, 0, 0, len};

    const uint64_t obase = (uint64_t)chunk * chunk_size;
    const uint64_t want = out_n > obase ? min(chunk_size, out_n - obase) : 0;
    const uint32_t rounds = (uint32_t)(chunk_size / 32 / sizeof(T) / wil);
    const uint32_t row_bytes = 32u * slice;
    T* my_stage = reinterpret_cast<T*>(stage + lane * sstride);
    const bool aligned4 = ((reinterpret_cast<uintptr_t>(out + obase) & 3u) == 0) && (slice % 4 == 0);

    // lane state: mode 0 = header next, 1 = literals, 2 = run
    uint32_t mode = 0, rem = 0;
    T val = 0;
    int64_t delta = 0;

    auto rd_byte = [&](uint32_t& b) -> bool {
        if (r.rd >= r.len) return false;
        b = ring_byte(r, r.rd);
        ++r.rd;
        return true;
    };
    auto rd_varint = [&](T& v) -> bool {
        uint64_t acc = 0;
        uint32_t sh = 0, b;
        do {
            if (!rd_byte(b)) return false;
            if (sh < 64) acc |= (uint64_t)(b & 0x7fu) << sh;
            sh += 7;
            if (sh > 70) return false;
        } while (b & 0x80u);
        v = (T)acc;
        return true;
    };

    for (uint32_t rnd = 0; rnd < rounds; ++rnd) {
        uint32_t produced = 0;
        for (;;) {
            const bool act = (produced < wil) && (err == ST_OK);
            const bool need = act && (r.fl - r.rd < (uint32_t)RING_LOW) && (lw.k < lw.nw);
            if (__any_sync(GD_FULL_MASK, need)) ring_refill(r, lw, T_, block);
            if (!__any_sync(GD_FULL_MASK, act)) break;
            if (act) {
                if (mode == 0) {
                    uint32_t hb;
                    if (!rd_byte(hb)) {
                        err = ST_CORRUPT;
                    } else if (hb & 0x80u) {
                        mode = 1;
                        rem = 256u - hb;  // -(int8)hb
                    } else {
                        uint32_t db;
                        T base;
                        if (!rd_byte(db) || !rd_varint(base)) {
                            err = ST_CORRUPT;
                        } else {
                            mode = 2;
                            rem = hb + 3u;
                            delta = (int8_t)db;
                            val = base;
                        }
                    }
                }
                if (err == ST_OK) {
                    T v;
                    if (mode == 1) {
                        if (!rd_varint(v)) err = ST_CORRUPT;
                    } else {
                        v = val;
                        val = (T)((uint64_t)val + (uint64_t)delta);
                    }
                    if (err == ST_OK) {
                        my_stage[produced++] = v;
                        if (--rem == 0) mode = 0;
                    }
                }
            }
        }
        __syncwarp();
        // write row rnd: bytes [rnd*row_bytes, +row_bytes) of the chunk, clipped
        const uint64_t roff = (uint64_t)rnd * row_bytes;
        if (roff < want) {
            const uint32_t n = (uint32_t)min((uint64_t)row_bytes, want - roff);
            uint8_t* dst = out + obase + roff;
            if (aligned4) {
                const uint32_t nwd = n >> 2;
                for (uint32_t i = lane; i < nwd; i += 32) {
                    const uint32_t byte = 4 * i, sl = byte / slice, o = byte - sl * slice;
                    reinterpret_cast<uint32_t*>(dst)[i] = *reinterpret_cast<const uint32_t*>(stage + sl * sstride + o);
                }
                for (uint32_t i = (nwd << 2) + lane; i < n; i += 32) {
                    const uint32_t sl = i / slice;
                    dst[i] = stage[sl * sstride + (i - sl * slice)];
                }
            } else {
                for (uint32_t i = lane; i < n; i += 32) {
                    const uint32_t sl = i / slice;
                    dst[i] = stage[sl * sstride + (i - sl * slice)];
                }
            }
        }
        __syncwarp();
        if (__any_sync(GD_FULL_MASK, err != ST_OK)) break;
    }
    err = __reduce_max_sync(GD_FULL_MASK, err);
    if (lane == 0) put_status(status, chunk, err);
}

}  // namespace rlev1
}  // namespace gd

extern "C" gd_status_t gd_rlev1_decode(const uint8_t* d_data, const uint64_t* d_col_len, const uint64_t* d_blk_off,
                                       uint32_t n_chunks, uint64_t chunk_size, uint32_t comp_col_len,
                                       uint32_t elem_bytes, uint8_t* d_out, uint64_t out_n_bytes,
                                       uint32_t* d_status, gd_stream_t stream) {
    if (n_chunks == 0) return GD_OK;
    if (!d_data || !d_col_len || !d_blk_off || !d_out) return GD_ERR_INVALID_ARG;
    if (!(elem_bytes == 4 || elem_bytes == 8)) return GD_ERR_UNSUPPORTED;
    if (comp_col_len == 0 || comp_col_len % elem_bytes || comp_col_len > 512) return GD_ERR_INVALID_ARG;
    if (chunk_size == 0 || chunk_size % (32ull * comp_col_len) || chunk_size > (1ull << 31)) return GD_ERR_INVALID_ARG;
    if (out_n_bytes > chunk_size * (uint64_t)n_chunks || out_n_bytes <= chunk_size * (uint64_t)(n_chunks - 1))
        return GD_ERR_INVALID_ARG;
    using namespace gd::rlev1;
    const uint32_t wil = comp_col_len / elem_bytes;
    const uint32_t smem = WPB * warp_smem(comp_col_len, elem_bytes);
    const uint32_t grid = (n_chunks + WPB - 1) / WPB;
    cudaStream_t s = (cudaStream_t)stream;
    if (elem_bytes == 4) {
        cudaFuncSetAttribute(decode_kernel<uint32_t>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        decode_kernel<uint32_t><<<grid, WPB * 32, smem, s>>>(d_data, d_col_len, d_blk_off, n_chunks, chunk_size, wil,
                                                            d_out, out_n_bytes, d_status);
    } else {
        cudaFuncSetAttribute(decode_kernel<uint64_t>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        decode_kernel<uint64_t><<<grid, WPB * 32, smem, s>>>(d_data, d_col_len, d_blk_off, n_chunks, chunk_size, wil,
                                                            d_out, out_n_bytes, d_status);
    }
    return cudaGetLastError() == cudaSuccess ? GD_OK : GD_ERR_CUDA;
}
