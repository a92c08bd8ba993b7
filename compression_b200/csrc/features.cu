// features.cu -- per-task header features for the learned cost model.
//
// No counterpart in the reference (its decoders have no scheduler).  One warp
// per batch task reads only the task's container headers -- never the values
// a decoder produces -- and reports what the decode cost depends on beyond
// the sizes the host already knows:
//   RLE v1 lane stream  run headers and literal groups (rle_v1 grammar:
//                       header byte, -h literal varints or delta + base);
//   RLE v2 lane stream  run headers, and the share of DIRECT / PATCHED_BASE
//                       runs (the bit-unpacking kinds);
//   byte-RLE chunk      tokens, and the share of literal tokens;
//   LZSS chunk          tokens over the 32 columns, and the share of literals
//                       (1 - match density), from the flag bytes;
//   Deflate stream      the first block's type and, for a dynamic block, its
//                       literal/length code count (HLIT + 257): a stream's
//                       later block headers are only found by decoding it.
// Each walk is bounded by the stream's length; a malformed stream sets the
// task's error feature instead of faulting.
#include "interleave.cuh"
#include "rlev2.cuh"

namespace gd {
namespace feat {

// Block offset of word k of `slot` in an interleaved block (segment table T).
__device__ __forceinline__ uint32_t word_off(const SegTable* T, uint32_t slot, uint32_t k) {
    uint32_t j = 0;
#pragma unroll
    for (uint32_t step = 16; step; step >>= 1)
        if (j + step <= 31 && T->hi[j + step - 1] <= k) j += step;
    const uint32_t lo = j ? T->hi[j - 1] : 0u;
    return T->base[j] + (k - lo) * 4u * (32u - j) + 4u * __popc(T->mask[j] & ((1u << slot) - 1u));
}

// Sequential byte reader over one slot's stream of an interleaved block.
struct SlotReader {
    const SegTable* T;
    const uint8_t* block;
    uint32_t slot, len, kw, w;
    __device__ uint32_t at(uint32_t pos) {  // pos < len
        const uint32_t k = pos >> 2;
        if (k != kw) {
            kw = k;
            w = __ldg(reinterpret_cast<const uint32_t*>(block + word_off(T, slot, k)));
        }
        return (w >> (8u * (pos & 3u))) & 0xffu;
    }
};

struct Out {
    float units, lit_share, density, bad;
};

// rle_v1 lane stream (decoder.h:278-423 grammar): h < 0: -h literal
// varints; else a run: delta byte, base varint.
__device__ Out rlev1_walk(SlotReader& r, uint32_t out_bytes) {
    uint32_t pos = 0, runs = 0, groups = 0, lit_vals = 0, run_vals = 0, bad = 0;
    while (pos < r.len) {
        const int32_t h = (int8_t)r.at(pos++);
        uint32_t nvar = 1;
        if (h < 0) {
            ++groups;
            nvar = (uint32_t)(-h);
            lit_vals += nvar;
        } else {
            ++runs;
            run_vals += (uint32_t)h + 3u;
            ++pos;  // delta byte
        }
        for (uint32_t i = 0; i < nvar && pos < r.len; ++i) {
            uint32_t n = 0;
            while (pos < r.len && (r.at(pos) & 0x80u) && n < 10u) ++pos, ++n;
            ++pos;
        }
        if (pos > r.len) bad = 1;
    }
    const uint32_t hdr = runs + groups, vals = lit_vals + run_vals;
    return {log2f(1.0f + hdr), vals ? (float)lit_vals / vals : 0.f, hdr * 1024.f / max(out_bytes, 1u), (float)bad};
}

// RLE v2 lane stream: the byte length of the run at pos from its header
// (decoder.h:28-188 grammar); 0 when it runs past the stream.
__device__ Out rlev2_walk(SlotReader& r, uint32_t out_bytes) {
    uint32_t pos = 0, runs = 0, unpack = 0, bad = 0;
    while (pos < r.len && !bad) {
        const uint32_t h = r.at(pos), kind = h >> 6;
        ++runs;
        if (kind == 0u) {
            pos += 2u + ((h >> 3) & 7u);
            continue;
        }
        if (pos + 2u > r.len) {
            bad = 1;
            break;
        }
        const uint32_t len = (((h & 1u) << 8) | r.at(pos + 1)) + 1u;
        const uint32_t fbw = rlev2::w_decode((h >> 1) & 31u);
        if (kind == 1u) {
            ++unpack;
            pos += 2u + (len * fbw + 7u) / 8u;
        } else if (kind == 2u) {
            ++unpack;
            if (pos + 4u > r.len) {
                bad = 1;
                break;
            }
            const uint32_t b2 = r.at(pos + 2), b3 = r.at(pos + 3);
            const uint32_t cfb = rlev2::closest_fixed(rlev2::w_decode(b2 & 31u) + (b3 >> 5) + 1u);
            pos += 4u + (b2 >> 5) + 1u + (len * fbw + 7u) / 8u + ((b3 & 31u) * cfb + 7u) / 8u;
        } else {
            uint32_t q = pos + 2u;
            for (int v = 0; v < 2; ++v) {  // base uvarint, delta svarint
                uint32_t n = 0;
                while (q < r.len && (r.at(q) & 0x80u) && n < 10u) ++q, ++n;
                ++q;
            }
            pos = q + (((h >> 1) & 31u) ? ((len - 2u) * fbw + 7u) / 8u : 0u);
        }
    }
    if (pos > r.len) bad = 1;
    return {log2f(1.0f + runs), runs ? (float)unpack / runs : 0.f, runs * 1024.f / max(out_bytes, 1u), (float)bad};
}

__global__ void __launch_bounds__(128) features_kernel(const gd_task* __restrict__ tasks, uint32_t n,
                                                      float4* __restrict__ feat) {
    __shared__ SegTable Ts[4];
    const uint32_t lane = lane_id(), wid = threadIdx.x >> 5;
    SegTable* T = &Ts[wid];
    for (uint32_t ti = blockIdx.x * 4 + wid; ti < n; ti += gridDim.x * 4) {
        const gd_task t = tasks[ti];
        Out o{0.f, 0.f, 0.f, 0.f};
        const uint32_t out_bytes = (uint32_t)min(t.dst_len, (uint64_t)0xffffffffu);
        if (t.codec == GD_CODEC_RLEV1 || t.codec == GD_CODEC_RLEV2 || t.codec == GD_CODEC_LZSS) {
            const uint64_t l64 = t.col_len[lane];
            const uint32_t len = l64 > 0xffffu ? 0u : (uint32_t)l64;
            uint32_t bad = l64 > 0xffffu ? 1u : 0u;
            const uint32_t nw = (len + 3u) >> 2;
            uint32_t tot = warp_incl_scan(nw);
            tot = __shfl_sync(GD_FULL_MASK, tot, 31);
            if ((uint64_t)tot * 4u > t.src_len) bad = 1;
            if (__any_sync(GD_FULL_MASK, bad)) {
                o.bad = 1.f;
            } else {
                seg_build(T, nw);
                if (t.codec == GD_CODEC_LZSS) {
                    // every lane walks its rank's column: a flag byte, then 8
                    // tokens, flag bit 1 = literal byte, 0 = 2-byte match
                    SlotReader r{T, t.src, lane, len, 0xffffffffu, 0};
                    uint32_t pos = 0, toks = 0, lits = 0, head = 0, k = 8;
                    while (pos < len) {
                        if (k == 8u) {
                            head = r.at(pos++);
                            k = 0;
                            continue;
                        }
                        const uint32_t lit = (head >> k) & 1u;
                        ++k;
                        ++toks;
                        lits += lit;
                        pos += lit ? 1u : 2u;
                    }
                    const uint32_t T_ = __reduce_add_sync(GD_FULL_MASK, toks);
                    const uint32_t L_ = __reduce_add_sync(GD_FULL_MASK, lits);
                    o = {log2f(1.0f + T_), T_ ? (float)L_ / T_ : 0.f, T_ * 1024.f / max(out_bytes, 1u), 0.f};
                } else {
                    const uint32_t slot = t.lane & 31u;
                    const uint32_t slen = __shfl_sync(GD_FULL_MASK, len, (int)slot);
                    if (lane == 0) {
                        SlotReader r{T, t.src, slot, slen, 0xffffffffu, 0};
                        o = t.codec == GD_CODEC_RLEV1 ? rlev1_walk(r, out_bytes / 32u)
                                                      : rlev2_walk(r, out_bytes / 32u);
                    }
                }
                __syncwarp();
            }
        } else if (t.codec == GD_CODEC_BRLE) {
            if (lane == 0) {
                // tokens: c <= 127 a run (2 bytes), else c - 127 literal bytes
                uint32_t pos = 0, toks = 0, lits = 0;
                const uint32_t clen = (uint32_t)min(t.src_len, (uint64_t)0x7fffffffu);
                while (pos < clen) {
                    const uint32_t c = __ldg(t.src + pos);
                    ++toks;
                    if (c > 127u) {
                        ++lits;
                        pos += c - 126u;
                    } else {
                        pos += 2u;
                    }
                }
                o = {log2f(1.0f + toks), toks ? (float)lits / toks : 0.f, toks * 1024.f / max(out_bytes, 1u),
                     pos > clen ? 1.f : 0.f};
            }
        } else if (t.codec == GD_CODEC_DEFLATE) {
            if (lane == 0) {
                const uint32_t skip = t.param == 1 ? 2u : 0u;  // the zlib header
                if (t.src_len >= skip + 3u && t.param != 2) {
                    const uint32_t b0 = __ldg(t.src + skip), b1 = __ldg(t.src + skip + 1);
                    const uint32_t btype = (b0 >> 1) & 3u;
                    const uint32_t hlit = ((b0 >> 3) & 31u) + 257u;
                    (void)b1;
                    o = {0.f, btype == 3u ? 0.f : (float)btype * 0.5f, btype == 2u ? hlit / 286.f : 0.f,
                         btype == 3u ? 1.f : 0.f};
                } else {
                    o.bad = t.param == 2 ? 0.f : 1.f;
                }
            }
        }
        if (lane == 0) feat[ti] = make_float4(o.units, o.lit_share, o.density, o.bad);
        __syncwarp();
    }
}

}  // namespace feat
}  // namespace gd

extern "C" gd_status_t gd_task_features(const gd_task* d_tasks, uint32_t n_tasks, float* d_features,
                                        gd_stream_t stream) {
    if (n_tasks == 0) return GD_OK;
    if (!d_tasks || !d_features || (reinterpret_cast<uintptr_t>(d_features) & 15u)) return GD_ERR_INVALID_ARG;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const uint32_t want = (n_tasks + 3u) / 4u, cap = (uint32_t)sms * 16u;
    gd::feat::features_kernel<<<want < cap ? want : cap, 128, 0, (cudaStream_t)stream>>>(
        d_tasks, n_tasks, reinterpret_cast<float4*>(d_features));
    return cudaGetLastError() == cudaSuccess ? GD_OK : GD_ERR_CUDA;
}
