// brle_warp.cuh -- warp-level byte-RLE chunk decoder (the batched decoder's
// unit of work; the plain brle kernel uses a 256-thread block per chunk).
//
// Same method as brle.cu at warp scale: 1 KiB tiles of compressed bytes,
// 32-byte segments with backward-pass exit tables, one lane following the
// token chain across the 32 segments, a warp scan placing tokens, and a
// merge-path expansion (64 output bytes per lane per round, 16-byte stores).
// Grammar: brle::decode, include/brle/brle.h:76-97.
#pragma once
#include "gd_common.cuh"

namespace gd {
namespace brlew {

constexpr uint32_t SEG = 32;
constexpr uint32_t TILE = 32 * SEG;
constexpr uint32_t HALO = 160;
constexpr uint32_t TPW = TILE / 2;  // most tokens one tile can hold
constexpr uint32_t NONE = 0xffffffffu;
// tile | exit tables | token output offsets | token positions | entries
constexpr uint32_t WARP_SMEM = TILE + HALO + 16 + 32 * SEG + TPW * 4 + TPW * 2 + 32 * 4 + 16;

__device__ __forceinline__ uint32_t tok_in(uint32_t c) { return c > 127u ? c - 126u : 2u; }
__device__ __forceinline__ uint32_t tok_out(uint32_t c) { return c > 127u ? c - 127u : c + 3u; }

// Decode one chunk (clen compressed bytes at src) into dst[0..want) with the
// calling warp; ws = WARP_SMEM bytes of shared memory (16-byte aligned).
// Returns a gd status (same on every lane).
static __device__ __noinline__ uint32_t chunk_warp(const uint8_t* __restrict__ src, uint32_t clen,
                                            uint8_t* __restrict__ dst, uint32_t want, uint8_t* ws) {
    const uint32_t lane = lane_id();
    uint8_t* s_tile = ws;
    uint8_t* s_tbl = ws + TILE + HALO + 16;
    uint32_t* tl_out = reinterpret_cast<uint32_t*>(s_tbl + 32 * SEG);
    uint16_t* tl_pos = reinterpret_cast<uint16_t*>(tl_out + TPW);
    uint32_t* s_entry = reinterpret_cast<uint32_t*>(tl_pos + TPW);
    const bool aligned16 = ((reinterpret_cast<uintptr_t>(dst) & 15u) == 0);
    uint32_t carry = 0, opos = 0, err = ST_OK;

    for (uint32_t t0 = 0; t0 < clen; t0 += TILE) {
        const uint32_t n_ld = min(clen - t0, TILE + HALO);
        const uint8_t* g = src + t0;
        const uint32_t sh = (uint32_t)(reinterpret_cast<uintptr_t>(g) & 15u);
        const uint8_t* tb = s_tile + sh;
        {
            uint32_t head = (16u - sh) & 15u;
            if (head > n_ld) head = n_ld;
            if (lane < head) s_tile[sh + lane] = g[lane];
            const uint32_t nv = (n_ld - head) >> 4;
            const uint4* gv = reinterpret_cast<const uint4*>(g + head);
            uint4* sv = reinterpret_cast<uint4*>(s_tile + sh + head);
            for (uint32_t i = lane; i < nv; i += 32) sv[i] = __ldg(gv + i);
            for (uint32_t i = head + 16 * nv + lane; i < n_ld; i += 32) s_tile[sh + i] = g[i];
        }
        __syncwarp();
        const uint32_t S = t0 + SEG * lane;
        const uint32_t lim = min(S + SEG, clen);
        uint8_t* tbl = s_tbl + lane * SEG;
        if (S < clen) {
            for (int32_t p = (int32_t)lim - 1; p >= (int32_t)S; --p) {
                const uint32_t n = (uint32_t)p + tok_in(tb[(uint32_t)p - t0]);
                tbl[(uint32_t)p - S] = (n >= lim) ? (uint8_t)(n - S) : tbl[n - S];
            }
        }
        __syncwarp();
        if (lane == 0) {
            uint32_t e = carry;
            for (uint32_t t = 0; t < 32; ++t) {
                const uint32_t St = t0 + SEG * t;
                if (St >= clen || e >= min(St + SEG, clen)) {
                    s_entry[t] = NONE;
                    continue;
                }
                s_entry[t] = e;
                e = St + s_tbl[t * SEG + (e - St)];
            }
            carry = e;
        }
        __syncwarp();
        carry = __shfl_sync(GD_FULL_MASK, carry, 0);
        uint32_t mask = 0, cnt = 0;
        bool bad = false;
        {
            const uint32_t e = s_entry[lane];
            if (e != NONE) {
                uint32_t p = e;
                while (p < lim) {
                    mask |= 1u << (p - S);
                    const uint32_t c = tb[p - t0];
                    if (p + tok_in(c) > clen) bad = true;
                    cnt += tok_out(c);
                    p += tok_in(c);
                }
            }
        }
        if (__any_sync(GD_FULL_MASK, bad)) {
            err = ST_CORRUPT;
            break;
        }
        const uint32_t inc = warp_incl_scan(cnt);
        const uint32_t total = __shfl_sync(GD_FULL_MASK, inc, 31);
        if ((uint64_t)opos + total > want) {
            err = ST_OVERRUN;
            break;
        }
        const uint32_t excl = inc - cnt;
        const uint32_t ntok = __popc(mask);
        const uint32_t tinc = warp_incl_scan(ntok);
        const uint32_t n_w = __shfl_sync(GD_FULL_MASK, tinc, 31);
        {
            uint32_t j = tinc - ntok, o = opos + excl;
            uint32_t m = mask;
            while (m) {
                const uint32_t tp = S + (__ffs(m) - 1) - t0;
                tl_out[j] = o;
                tl_pos[j] = (uint16_t)tp;
                o += tok_out(tb[tp]);
                ++j;
                m &= m - 1;
            }
        }
        __syncwarp();
        if (n_w) {
            const uint32_t wbeg = opos, wend = opos + total;
            for (uint32_t r = wbeg & ~15u; r < wend; r += 32 * 64) {
                const uint32_t lo = max(r + 64 * lane, wbeg);
                const uint32_t hi = min(r + 64 * lane + 64, wend);
                if (lo >= hi) continue;
                uint32_t a = 0, b = n_w;
                while (b - a > 1) {
                    const uint32_t m = (a + b) >> 1;
                    if (tl_out[m] <= lo) a = m;
                    else b = m;
                }
                uint32_t k = a;
                uint32_t ks = tl_out[k], kp = tl_pos[k];
                uint32_t kc = tb[kp];
                uint32_t ke = ks + tok_out(kc);
                for (uint32_t v0 = lo & ~15u; v0 < hi; v0 += 16) {
                    const uint32_t x0 = max(v0, lo), x1 = min(v0 + 16, hi);
                    while (ke <= x0) {
                        ++k;
                        ks = ke;
                        kp = tl_pos[k];
                        kc = tb[kp];
                        ke = ks + tok_out(kc);
                    }
                    if (aligned16 && x0 == v0 && x1 == v0 + 16 && kc <= 127u && ke >= x1) {
                        const uint32_t rep = 0x01010101u * tb[kp + 1];
                        *reinterpret_cast<uint4*>(dst + v0) = make_uint4(rep, rep, rep, rep);
                        continue;
                    }
                    uint32_t w[4] = {0, 0, 0, 0};
                    uint32_t x = x0;
                    for (;;) {
                        const uint32_t n = min(ke, x1) - x;
                        if (kc <= 127u) {
                            const uint32_t rep = 0x01010101u * tb[kp + 1];
#pragma unroll
                            for (uint32_t q = 0; q < 4; ++q) {
                                const uint32_t ql = v0 + 4 * q;
                                const uint32_t a0 = max(x, ql), a1 = min(x + n, ql + 4);
                                if (a0 < a1) {
                                    const uint32_t nb = a1 - a0;
                                    const uint32_t msk = (nb == 4 ? 0xffffffffu : ((1u << (8 * nb)) - 1u)) << (8 * (a0 - ql));
                                    w[q] = (w[q] & ~msk) | (rep & msk);
                                }
                            }
                        } else {
                            const uint8_t* lit = tb + kp + 1 + (x - ks);
                            for (uint32_t i = 0; i < n; ++i) {
                                const uint32_t bo = x - v0 + i;
                                w[bo >> 2] |= (uint32_t)lit[i] << (8 * (bo & 3u));
                            }
                        }
                        x += n;
                        if (x >= x1) break;
                        ++k;
                        ks = ke;
                        kp = tl_pos[k];
                        kc = tb[kp];
                        ke = ks + tok_out(kc);
                    }
                    if (aligned16 && x0 == v0 && x1 == v0 + 16) {
                        *reinterpret_cast<uint4*>(dst + v0) = make_uint4(w[0], w[1], w[2], w[3]);
                    } else {
                        for (uint32_t y = x0; y < x1; ++y) dst[y] = (uint8_t)(w[(y - v0) >> 2] >> (8 * ((y - v0) & 3u)));
                    }
                }
            }
        }
        opos += total;
        __syncwarp();
    }
    if (err == ST_OK && (opos != want || carry != clen)) err = ST_CORRUPT;
    return err;
}

}  // namespace brlew
}  // namespace gd
