// rlev2.cu -- RLE v2 (ORC-style integer RLE v2, transposed container)
// decoder for sm_100a.  8-byte values.
//
// Grammar (restated from rlev2::decode_{short_repeat,direct,patched_base,
// delta}, include/rlev2/decoder.h:28-188; the GPU decoder_warp,
// decoder_new.h:360-611, decodes the same bytes): the top two header bits
// select SHORT_REPEAT, DIRECT, PATCHED_BASE or DELTA.  Lane t of a chunk owns
// the values t*RU + k*32*RU + j, j < RU.  Corrections to the reference (the
// oracle applies the same): 64-bit patch mask (decoder.h:174 keeps 16 bits),
// the delta accumulation runs len-2 times (decoder.h:117-123 runs len), and
// a PATCHED_BASE base with its top bit set is negative.
//
// Organisation as rlev1.cu: one warp per chunk, lane = lane stream, per-lane
// shared-memory input rings fed through the segment table, one output row
// (32 lanes x RU values) per round written with coalesced stores.  Each
// iteration a lane emits one value, so the four sub-encodings stay in step
// across the warp.  PATCHED_BASE patches are applied as the values stream
// out: the patch list (which follows the values in the stream) is read
// entry by entry straight from the block, so nothing is written back.
#include "interleave.cuh"

namespace gd {
namespace rlev2 {

constexpr int WPB = 4;

__host__ __device__ constexpr uint32_t stage_stride(uint32_t slice_bytes) { return ((slice_bytes + 15u) & ~15u) + 8u; }
__host__ __device__ constexpr uint32_t warp_smem(uint32_t slice_bytes) {
    return (uint32_t)sizeof(SegTable) + 32u * RING_STRIDE + 32u * stage_stride(slice_bytes);
}

__device__ __constant__ uint8_t W_DECODE[32] = {1,  2,  3,  4,  5,  6,  7,  8,  9,  10, 11, 12, 13, 14, 15, 16,
                                                17, 18, 19, 20, 21, 22, 23, 24, 26, 28, 30, 32, 40, 48, 56, 64};

__device__ __forceinline__ uint32_t closest_fixed(uint32_t b) {
    if (b <= 1) return 1;
    if (b <= 24) return b;
    if (b <= 26) return 26;
    if (b <= 28) return 28;
    if (b <= 30) return 30;
    if (b <= 32) return 32;
    if (b <= 40) return 40;
    if (b <= 48) return 48;
    if (b <= 56) return 56;
    return 64;
}

enum : uint32_t { M_HDR = 0, M_SR = 1, M_DIRECT = 2, M_PATCH = 3, M_DELTA = 4 };

__global__ void __launch_bounds__(WPB * 32) decode_kernel(const uint8_t* __restrict__ data,
                                                         const uint64_t* __restrict__ col_len,
                                                         const uint64_t* __restrict__ blk_off, uint32_t n_chunks,
                                                         uint64_t chunk_size, uint32_t ru,
                                                         uint8_t* __restrict__ out, uint64_t out_n,
                                                         uint32_t* __restrict__ status) {
    extern __shared__ __align__(16) uint8_t smem[];
    const uint32_t lane = lane_id(), wid = threadIdx.x >> 5;
    const uint32_t chunk = blockIdx.x * WPB + wid;
    if (chunk >= n_chunks) return;
    const uint32_t slice = ru * 8u;
    const uint32_t sstride = stage_stride(slice);
    uint8_t* wbase = smem + wid * warp_smem(slice);
    SegTable* T_ = reinterpret_cast<SegTable*>(wbase);
    uint8_t* ring = wbase + sizeof(SegTable);
    uint8_t* stage = ring + 32 * RING_STRIDE;

    uint32_t err = ST_OK;
    const uint64_t b0 = blk_off[chunk], b1 = blk_off[chunk + 1];
    const uint64_t len64 = col_len[32ull * chunk + lane];
    const uint32_t len = len64 > 0x3fffffffull ? 0u : (uint32_t)len64;
    if (len64 > 0x3fffffffull) err = ST_CORRUPT;
    const uint32_t nw = (len + 3) >> 2;
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
    const uint32_t rounds = (uint32_t)(chunk_size / 256u / ru);
    const uint32_t row_bytes = 32u * slice;
    uint64_t* my_stage = reinterpret_cast<uint64_t*>(stage + lane * sstride);
    const bool aligned16 = ((reinterpret_cast<uintptr_t>(out + obase) & 15u) == 0) && (slice % 16 == 0);

    // ---- lane state ----
    uint32_t mode = M_HDR, rem = 0, idx = 0;
    uint32_t fbw = 0, bits_left = 0, cur = 0;
    uint64_t val = 0, base = 0, delta = 0;
    bool dec_neg = false, dfixed = false;
    // patched-base state
    uint32_t pw = 0, cfb = 0, p_left = 0, p_bit = 0, p_start = 0, p_end = 0;
    uint32_t p_next = 0xffffffffu;
    uint64_t p_val = 0;

    auto rd_byte = [&](uint32_t& b) -> bool {
        if (r.rd >= r.len) return false;
        b = ring_byte(r, r.rd);
        ++r.rd;
        return true;
    };
    auto rd_uvarint = [&](uint64_t& v) -> bool {
        uint64_t acc = 0;
        uint32_t sh = 0, b;
        do {
            if (!rd_byte(b)) return false;
            if (sh < 64) acc |= (uint64_t)(b & 0x7fu) << sh;
            sh += 7;
            if (sh > 70) return false;
        } while (b & 0x80u);
        v = acc;
        return true;
    };
    // next fb-bit MSB-first value of the current packed run (readLongs)
    auto rd_bits = [&](uint32_t fb, uint64_t& v) -> bool {
        uint64_t res = 0;
        uint32_t need = fb;
        while (need > bits_left) {
            res = (bits_left ? (res << bits_left) : res) | (cur & ((1u << bits_left) - 1u));
            need -= bits_left;
            if (!rd_byte(cur)) return false;
            bits_left = 8;
        }
        if (need) {
            res = (res << need);
            bits_left -= need;
            res |= (cur >> bits_left) & ((1u << need) - 1u);
        }
        v = res;
        return true;
    };
    // random-access byte q of this lane's stream, straight from the block
    auto g_byte = [&](uint32_t q, uint32_t& b) -> bool {
        if (q >= r.len) return false;
        const uint32_t off = word_offset_at(T_, q >> 2) + (q & 3u);
        b = block[off];
        return true;
    };
    // decode the next patch entry (gap << pw | patch), cfb bits at p_bit
    auto next_patch = [&]() -> bool {
        if (p_left == 0) {
            p_next = 0xffffffffu;
            return true;
        }
        uint64_t e = 0;
        uint32_t bit = p_bit, need = cfb;
        while (need) {
            uint32_t b;
            if (!g_byte(p_start + (bit >> 3), b)) return false;
            const uint32_t avail = 8u - (bit & 7u);
            const uint32_t take = min(avail, need);
            const uint32_t v = (b >> (avail - take)) & ((1u << take) - 1u);
            e = (e << take) | v;
            need -= take;
            bit += take;
        }
        p_bit = bit;
        --p_left;
        const uint64_t pmask = (pw >= 64) ? ~0ull : ((1ull << pw) - 1ull);
        const uint32_t gap = (uint32_t)(pw >= 64 ? 0ull : (e >> pw));
        p_next = (p_next == 0xffffffffu ? 0u : p_next) + gap;
        p_val = (e & pmask) << fbw;
        return true;
    };
    // move the read position to byte `pos` (>= rd), discarding ring contents
    auto skip_to = [&](uint32_t pos) {
        if (pos <= r.fl) {
            r.rd = pos;
        } else {
            r.rd = pos;
            r.fl = pos & ~3u;
            lw.k = r.fl >> 2;
        }
    };

    for (uint32_t rnd = 0; rnd < rounds; ++rnd) {
        uint32_t produced = 0;
        for (;;) {
            const bool act = (produced < ru) && (err == ST_OK);
            const bool need = act && (r.fl - r.rd < (uint32_t)RING_LOW) && (lw.k < lw.nw);
            if (__any_sync(GD_FULL_MASK, need)) ring_refill(r, lw, T_, block);
            if (!__any_sync(GD_FULL_MASK, act)) break;
            if (!act) continue;
            if (mode == M_HDR) {
                uint32_t first, b;
                if (!rd_byte(first)) {
                    err = ST_CORRUPT;
                    continue;
                }
                const uint32_t enc = first >> 6;
                if (enc == 0) {  // SHORT_REPEAT
                    const uint32_t nb = ((first >> 3) & 7u) + 1u;
                    uint64_t v = 0;
                    for (uint32_t i = 0; i < nb && err == ST_OK; ++i) {
                        if (!rd_byte(b)) err = ST_CORRUPT;
                        v = (v << 8) | b;
                    }
                    val = v;
                    rem = (first & 7u) + 3u;
                    mode = M_SR;
                } else {
                    fbw = W_DECODE[(first >> 1) & 31u];
                    if (!rd_byte(b)) {
                        err = ST_CORRUPT;
                        continue;
                    }
                    const uint32_t rl = (((first & 1u) << 8) | b) + 1u;
                    rem = rl;
                    idx = 0;
                    bits_left = 0;
                    if (enc == 1) {
                        mode = M_DIRECT;
                    } else if (enc == 2) {  // PATCHED_BASE
                        uint32_t b3, b4;
                        if (!rd_byte(b3) || !rd_byte(b4)) {
                            err = ST_CORRUPT;
                            continue;
                        }
                        const uint32_t bw = ((b3 >> 5) & 7u) + 1u;
                        pw = W_DECODE[b3 & 31u];
                        const uint32_t pgw = ((b4 >> 5) & 7u) + 1u;
                        p_left = b4 & 31u;
                        uint64_t bv = 0;
                        for (uint32_t i = 0; i < bw && err == ST_OK; ++i) {
                            if (!rd_byte(b)) err = ST_CORRUPT;
                            bv = (bv << 8) | b;
                        }
                        const uint64_t msb = 1ull << (8 * bw - 1);
                        base = (bv & msb) ? (uint64_t)(-(int64_t)(bv & ~msb)) : bv;
                        cfb = closest_fixed(pw + pgw);
                        // the patch list starts after ceil(rl*fbw/8) value bytes
                        p_start = r.rd + (uint32_t)(((uint64_t)rl * fbw + 7) >> 3);
                        p_end = p_start + (uint32_t)(((uint64_t)p_left * cfb + 7) >> 3);
                        if (p_end > r.len) err = ST_CORRUPT;
                        p_bit = 0;
                        p_next = 0xffffffffu;
                        if (err == ST_OK && !next_patch()) err = ST_CORRUPT;
                        mode = M_PATCH;
                    } else {  // DELTA
                        uint64_t ub, zz;
                        if (!rd_uvarint(ub) || !rd_uvarint(zz) || rl < 2) {
                            err = ST_CORRUPT;
                            continue;
                        }
                        base = ub;
                        delta = (zz >> 1) ^ (0ull - (zz & 1ull));
                        dec_neg = !((int64_t)delta > 0);
                        dfixed = ((first >> 1) & 31u) == 0;
                        mode = M_DELTA;
                    }
                }
                if (err != ST_OK) continue;
            }
            // ---- emit one value ----
            uint64_t v = 0;
            if (mode == M_SR) {
                v = val;
            } else if (mode == M_DIRECT) {
                if (!rd_bits(fbw, v)) err = ST_CORRUPT;
            } else if (mode == M_PATCH) {
                if (!rd_bits(fbw, v)) err = ST_CORRUPT;
                // every patch entry whose accumulated gap lands here (entries
                // that only carry a 255 gap have a zero patch)
                while (idx == p_next && err == ST_OK) {
                    v |= p_val;
                    if (!next_patch()) err = ST_CORRUPT;
                }
                v += base;
            } else {  // M_DELTA (decoder.h:106-131)
                if (idx == 0) {
                    v = base;
                } else if (idx == 1) {
                    v = base + delta;
                } else if (dfixed) {
                    v = val + delta;
                } else {
                    uint64_t d = 0;
                    if (!rd_bits(fbw, d)) err = ST_CORRUPT;
                    v = dec_neg ? val - d : val + d;
                }
                val = v;
            }
            if (err != ST_OK) continue;
            my_stage[produced++] = v;
            ++idx;
            if (--rem == 0) {
                if (mode == M_PATCH) {
                    if (p_next != 0xffffffffu) err = ST_CORRUPT;  // patch beyond the run
                    skip_to(p_end);
                }
                mode = M_HDR;
            }
        }
        __syncwarp();
        const uint64_t roff = (uint64_t)rnd * row_bytes;
        if (roff < want) {
            const uint32_t n = (uint32_t)min((uint64_t)row_bytes, want - roff);
            uint8_t* dst = out + obase + roff;
            if (aligned16) {
                const uint32_t nq = n >> 4;
                for (uint32_t i = lane; i < nq; i += 32) {
                    const uint32_t byte = 16 * i, sl = byte / slice, o = byte - sl * slice;
                    const uint64_t* s8 = reinterpret_cast<const uint64_t*>(stage + sl * sstride + o);
                    uint4 q;
                    q.x = (uint32_t)s8[0];
                    q.y = (uint32_t)(s8[0] >> 32);
                    q.z = (uint32_t)s8[1];
                    q.w = (uint32_t)(s8[1] >> 32);
                    reinterpret_cast<uint4*>(dst)[i] = q;
                }
                for (uint32_t i = (nq << 4) + lane; i < n; i += 32) {
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
    // a lane must end exactly at the end of its stream
    if (err == ST_OK && (mode != M_HDR || r.rd != r.len)) err = ST_CORRUPT;
    err = __reduce_max_sync(GD_FULL_MASK, err);
    if (lane == 0) put_status(status, chunk, err);
}

}  // namespace rlev2
}  // namespace gd

extern "C" gd_status_t gd_rlev2_decode(const uint8_t* d_data, const uint64_t* d_col_len, const uint64_t* d_blk_off,
                                       uint32_t n_chunks, uint64_t chunk_size, uint32_t read_unit,
                                       uint8_t* d_out, uint64_t out_n_bytes, uint32_t* d_status,
                                       gd_stream_t stream) {
    if (n_chunks == 0) return GD_OK;
    if (!d_data || !d_col_len || !d_blk_off || !d_out) return GD_ERR_INVALID_ARG;
    if (read_unit == 0 || read_unit > 64) return GD_ERR_UNSUPPORTED;
    if (chunk_size == 0 || chunk_size % (256ull * read_unit) || chunk_size > (1ull << 31)) return GD_ERR_INVALID_ARG;
    if (out_n_bytes > chunk_size * (uint64_t)n_chunks || out_n_bytes <= chunk_size * (uint64_t)(n_chunks - 1))
        return GD_ERR_INVALID_ARG;
    using namespace gd::rlev2;
    const uint32_t smem = WPB * warp_smem(read_unit * 8u);
    const uint32_t grid = (n_chunks + WPB - 1) / WPB;
    cudaFuncSetAttribute(decode_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    decode_kernel<<<grid, WPB * 32, smem, (cudaStream_t)stream>>>(d_data, d_col_len, d_blk_off, n_chunks, chunk_size,
                                                                   read_unit, d_out, out_n_bytes, d_status);
    return cudaGetLastError() == cudaSuccess ? GD_OK : GD_ERR_CUDA;
}
