/*
 * gd_oracle.c -- CPU oracle for the decode hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is a plain-C restatement of the
 * reference decoders (ZaidQureshi/compression).  It is the checker that the
 * CUDA kernels are compared against; nothing in the shipped library links or
 * calls it.  Only tests/, __graft_entry__.smoke() and the CPU-baseline leg of
 * bench.py load liboracle.so.
 *
 * Each routine cites the reference file:line whose behaviour it restates.
 * Deliberate deviations (documented quirk fixes) are marked "FIX Qn".
 *
 * Return codes follow gd_status_t in include/gd.h:
 *   0 OK, 2 CORRUPT (stream grammar violated / truncated), 3 OVERRUN
 *   (stream would write past the chunk), 5 UNSUPPORTED.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <zlib.h>

#define GDO_OK 0
#define GDO_INVALID 1
#define GDO_CORRUPT 2
#define GDO_OVERRUN 3
#define GDO_UNSUPPORTED 5

/* ------------------------------------------------------------------------ */
/* Byte-RLE, contiguous chunk format                                         */
/* ------------------------------------------------------------------------ */

/*
 * Decode one chunk of the brle container.
 * Restates brle::decode, include/brle/brle.h:76-97 (the non-lookahead path,
 * which is the live one because of the USE_LOOKAHEADd typo at brle.h:23).
 * Control byte c: c > 127 -> (c-127) literal bytes follow;
 *                 c <= 127 -> next byte repeated c+3 times.
 */
static int brle_decode_chunk(const uint8_t* in, uint64_t in_len, uint8_t* out, uint64_t out_cap,
                             uint64_t* out_len) {
    uint64_t used = 0, o = 0;
    while (used < in_len) {
        uint8_t ch = in[used++];
        uint64_t count;
        if (ch > 127) {
            count = (uint64_t)ch - 127;
            if (used + count > in_len) return GDO_CORRUPT;
            if (o + count > out_cap) return GDO_OVERRUN;
            memcpy(out + o, in + used, count);
            used += count;
        } else {
            count = (uint64_t)ch + 3;
            if (used >= in_len) return GDO_CORRUPT;
            if (o + count > out_cap) return GDO_OVERRUN;
            memset(out + o, in[used++], count);
        }
        o += count;
    }
    *out_len = o;
    return GDO_OK;
}

/*
 * Whole-container decode: chunk i occupies data[ptr[i] .. ptr[i+1]) and
 * decodes to out[i*chunk_size ..].  The final chunk may be short; every other
 * chunk must decode to exactly chunk_size bytes (brle.h:26-29,150).
 */
int gdo_brle_decode(const uint8_t* data, const uint64_t* ptr, uint32_t n_chunks,
                    uint64_t chunk_size, uint8_t* out, uint64_t out_total) {
    for (uint32_t c = 0; c < n_chunks; ++c) {
        uint64_t base = (uint64_t)c * chunk_size;
        if (base >= out_total) return GDO_INVALID;
        uint64_t want = out_total - base < chunk_size ? out_total - base : chunk_size;
        if (ptr[c + 1] < ptr[c]) return GDO_CORRUPT;
        uint64_t got = 0;
        int rc = brle_decode_chunk(data + ptr[c], ptr[c + 1] - ptr[c], out + base, want, &got);
        if (rc) return rc;
        if (got != want) return GDO_CORRUPT;
    }
    return GDO_OK;
}

/* ------------------------------------------------------------------------ */
/* 4-byte-word lane interleave shared by RLE v1, RLE v2 and LZSS              */
/* ------------------------------------------------------------------------ */

/*
 * Split one interleaved block into its 32 lane streams.
 * Row k of the block holds, in slot order s = 0..31, one 4-byte word from
 * every slot whose stream length exceeds 4k.  Slot s is a lane for RLE v1/v2
 * (reader ballot order, rle_v1/decoder.h:72-95; writer
 * rlev2/encoder_trans.h:291-349) and a length-sorted rank for LZSS
 * (lzss/lzss_gpu2.h:162-199 reader, :497-509 writer).
 * lane_buf[s] receives ceil(len[s]/4)*4 bytes.
 */
static int deinterleave(const uint8_t* block, uint64_t block_cap, const uint64_t* len,
                        uint8_t* lane_buf[32]) {
    uint64_t rows = 0;
    for (int s = 0; s < 32; ++s) {
        uint64_t w = (len[s] + 3) / 4;
        if (w > rows) rows = w;
    }
    uint64_t pos = 0;
    for (uint64_t k = 0; k < rows; ++k) {
        for (int s = 0; s < 32; ++s) {
            if (len[s] > 4 * k) {
                if (pos + 4 > block_cap) return GDO_CORRUPT;
                memcpy(lane_buf[s] + 4 * k, block + pos, 4);
                pos += 4;
            }
        }
    }
    return GDO_OK;
}

/* ------------------------------------------------------------------------ */
/* RLE v1 (ORC-style integer RLE v1, interleaved container)                  */
/* ------------------------------------------------------------------------ */

/*
 * Decode one lane stream of RLE v1.
 * Restates decoder_warp, include/rle_v1/decoder.h:278-423:
 *   h = int8 header.  h < 0: -h literals, each an unsigned LEB128 varint of
 *   the element type (:301-350).  h >= 0: run of h+3 values; delta = int8,
 *   base = unsigned varint; v_i = (int64)base + i*delta truncated to the
 *   element type (:354-411).  The lane stops once it has produced
 *   chunk_size/32 bytes (:283,291).
 * Element i of the lane lands at (i / wil) * 32 * wil + lane * wil + i % wil,
 * wil = comp_col_len / elem_bytes (:286-288,332-340).
 */
static int rlev1_decode_lane(const uint8_t* s, uint64_t s_len, int lane, uint64_t n_elems,
                             uint32_t wil, uint32_t eb, uint8_t* chunk_out) {
    uint64_t p = 0, e = 0;
    const uint64_t emask = (eb == 8) ? ~0ull : ((1ull << (8 * eb)) - 1);
#define RD(b)                                     \
    do {                                          \
        if (p >= s_len) return GDO_CORRUPT;       \
        (b) = s[p++];                             \
    } while (0)
#define PUT(val)                                                                      \
    do {                                                                              \
        if (e >= n_elems) return GDO_OVERRUN;                                         \
        uint64_t idx_ = (e / wil) * 32ull * wil + (uint64_t)lane * wil + (e % wil);   \
        uint64_t v_ = (uint64_t)(val) & emask;                                        \
        memcpy(chunk_out + idx_ * eb, &v_, eb);                                       \
        ++e;                                                                          \
    } while (0)
    while (e < n_elems) {
        uint8_t hb;
        RD(hb);
        int8_t h = (int8_t)hb;
        if (h < 0) {
            int cnt = -(int)h;
            for (int i = 0; i < cnt; ++i) {
                uint64_t v = 0;
                int off = 0;
                for (;;) {
                    uint8_t b;
                    RD(b);
                    if (off < 64) v |= (uint64_t)(b & 0x7f) << off;
                    if (!(b & 0x80)) break;
                    off += 7;
                    if (off > 70) return GDO_CORRUPT;
                }
                PUT(v);
            }
        } else {
            uint8_t db;
            RD(db);
            int8_t delta = (int8_t)db;
            uint64_t base = 0;
            int off = 0;
            for (;;) {
                uint8_t b;
                RD(b);
                if (off < 64) base |= (uint64_t)(b & 0x7f) << off;
                if (!(b & 0x80)) break;
                off += 7;
                if (off > 70) return GDO_CORRUPT;
            }
            /* the reference accumulates the varint in the element type */
            base &= emask;
            for (int i = 0; i < (int)h + 3; ++i) {
                int64_t v = (int64_t)base + (int64_t)i * (int64_t)delta;
                PUT(v);
            }
        }
    }
#undef RD
#undef PUT
    return GDO_OK;
}

/*
 * Whole-container RLE v1 decode (rle_v1::decompress_gpu, rlev1.h:100-199;
 * kernel inflate, decoder.h:426-470).  Block c starts at blk_off[c] in data;
 * col_len[32c+t] is lane t's unpadded stream length.  Chunk c decodes to
 * out[c*chunk_size ..], truncated to out_total.
 */
int gdo_rlev1_decode(const uint8_t* data, uint64_t data_len, const uint64_t* blk_off,
                     const uint64_t* col_len, uint32_t n_chunks, uint64_t chunk_size,
                     uint32_t comp_col_len, uint32_t elem_bytes, uint8_t* out, uint64_t out_total) {
    if (!(elem_bytes == 1 || elem_bytes == 2 || elem_bytes == 4 || elem_bytes == 8)) return GDO_INVALID;
    if (comp_col_len == 0 || comp_col_len % elem_bytes) return GDO_INVALID;
    if (chunk_size % (32ull * comp_col_len)) return GDO_INVALID;
    uint32_t wil = comp_col_len / elem_bytes;
    uint64_t n_elems = chunk_size / 32 / elem_bytes;
    uint8_t* tmp = (uint8_t*)malloc(chunk_size);
    uint8_t* lanes[32];
    uint64_t cap = 0;
    for (uint32_t c = 0; c < n_chunks; ++c)
        for (int t = 0; t < 32; ++t)
            if (col_len[32ull * c + t] + 8 > cap) cap = col_len[32ull * c + t] + 8;
    for (int t = 0; t < 32; ++t) lanes[t] = (uint8_t*)calloc(cap ? cap : 8, 1);
    int rc = GDO_OK;
    for (uint32_t c = 0; c < n_chunks && rc == GDO_OK; ++c) {
        if (blk_off[c] > data_len) { rc = GDO_CORRUPT; break; }
        rc = deinterleave(data + blk_off[c], data_len - blk_off[c], col_len + 32ull * c, lanes);
        for (int t = 0; t < 32 && rc == GDO_OK; ++t)
            rc = rlev1_decode_lane(lanes[t], col_len[32ull * c + t], t, n_elems, wil, elem_bytes, tmp);
        if (rc) break;
        uint64_t base = (uint64_t)c * chunk_size;
        if (base < out_total) {
            uint64_t n = out_total - base < chunk_size ? out_total - base : chunk_size;
            memcpy(out + base, tmp, n);
        }
    }
    for (int t = 0; t < 32; ++t) free(lanes[t]);
    free(tmp);
    return rc;
}

/* ------------------------------------------------------------------------ */
/* RLE v2 (ORC-style integer RLE v2, transposed container)                   */
/* ------------------------------------------------------------------------ */

/* include/rlev2/utils.h:38 */
static const uint8_t RLEV2_WIDTH_DECODE[32] = {1,  2,  3,  4,  5,  6,  7,  8,  9,  10, 11,
                                               12, 13, 14, 15, 16, 17, 18, 19, 20, 21, 22,
                                               23, 24, 26, 28, 30, 32, 40, 48, 56, 64};
/* include/rlev2/utils.h:53-60 (closest fixed width) */
static uint8_t rlev2_closest_fixed(uint32_t b) {
    if (b <= 1) return 1;
    if (b <= 24) return (uint8_t)b;
    if (b <= 26) return 26;
    if (b <= 28) return 28;
    if (b <= 30) return 30;
    if (b <= 32) return 32;
    if (b <= 40) return 40;
    if (b <= 48) return 48;
    if (b <= 56) return 56;
    return 64;
}

typedef struct {
    const uint8_t* s;
    uint64_t len, p;
} rd_t;

static int rd_byte(rd_t* r, uint8_t* b) {
    if (r->p >= r->len) return GDO_CORRUPT;
    *b = r->s[r->p++];
    return GDO_OK;
}

/* rlev2::readVulong, include/rlev2/decoder.h:74-83 */
static int rd_uvarint(rd_t* r, uint64_t* v) {
    uint64_t ret = 0;
    int off = 0;
    uint8_t b;
    do {
        if (rd_byte(r, &b)) return GDO_CORRUPT;
        if (off < 64) ret |= (uint64_t)(b & 0x7f) << off;
        off += 7;
        if (off > 70) return GDO_CORRUPT;
    } while (b >= 0x80);
    *v = ret;
    return GDO_OK;
}

/* rlev2::readLongs, include/rlev2/decoder.h:41-72: MSB-first bit unpack */
static int rd_longs(rd_t* r, int64_t* dst, uint32_t n, uint32_t fb, uint32_t* bits_left,
                    uint32_t* cur) {
    for (uint32_t i = 0; i < n; ++i) {
        uint64_t result = 0;
        uint32_t need = fb;
        while (need > *bits_left) {
            result <<= *bits_left;
            result |= *cur & ((1u << *bits_left) - 1);
            need -= *bits_left;
            uint8_t b;
            if (rd_byte(r, &b)) return GDO_CORRUPT;
            *cur = b;
            *bits_left = 8;
        }
        if (need > 0) {
            result <<= need;
            *bits_left -= need;
            result |= (*cur >> *bits_left) & ((1u << need) - 1);
        }
        dst[i] = (int64_t)result;
    }
    return GDO_OK;
}

/*
 * Decode one RLE v2 lane stream into vals[0..n_vals).
 * Restates rlev2::block_decode and decode_{short_repeat,direct,
 * patched_base,delta}, include/rlev2/decoder.h:28-222.
 *  FIX Q1: the patch mask is 64-bit (decoder.h:174 uses uint16_t and drops
 *          the high bits of patches wider than 16 bits).
 *  FIX Q2: the variable-delta accumulation runs len-2 times (decoder.h:117-123
 *          runs len times and writes two values past the run).
 *  FIX Q4: a PATCHED_BASE base whose top bit is set is negative (ORC
 *          semantics); the reference ignores the sign (decoder.h:160).  All
 *          streams the reference encoder emits for non-negative data decode
 *          identically either way.
 */
static int rlev2_decode_lane(const uint8_t* s, uint64_t s_len, int64_t* vals, uint64_t n_vals,
                             uint64_t* produced) {
    rd_t r = {s, s_len, 0};
    uint64_t o = 0;
    while (r.p < s_len) {
        uint8_t first;
        rd_byte(&r, &first);
        uint8_t enc = first & 0xC0;
        if (enc == 0x00) { /* SHORT_REPEAT, decoder.h:28-39 */
            uint32_t nb = ((first >> 3) & 7) + 1, cnt = (first & 7) + 3;
            uint64_t v = 0;
            for (uint32_t i = 0; i < nb; ++i) {
                uint8_t b;
                if (rd_byte(&r, &b)) return GDO_CORRUPT;
                v = (v << 8) | b;
            }
            if (o + cnt > n_vals) return GDO_OVERRUN;
            for (uint32_t i = 0; i < cnt; ++i) vals[o++] = (int64_t)v;
        } else if (enc == 0x40) { /* DIRECT, decoder.h:135-142 */
            uint32_t fbw = RLEV2_WIDTH_DECODE[(first >> 1) & 0x1f];
            uint8_t b;
            if (rd_byte(&r, &b)) return GDO_CORRUPT;
            uint32_t len = (((uint32_t)(first & 1) << 8) | b) + 1;
            if (o + len > n_vals) return GDO_OVERRUN;
            uint32_t bl = 0, cur = 0;
            if (rd_longs(&r, vals + o, len, fbw, &bl, &cur)) return GDO_CORRUPT;
            o += len;
        } else if (enc == 0x80) { /* PATCHED_BASE, decoder.h:144-188 */
            uint32_t fbw = RLEV2_WIDTH_DECODE[(first >> 1) & 0x1f];
            uint8_t b2, b3, b4;
            if (rd_byte(&r, &b2) || rd_byte(&r, &b3) || rd_byte(&r, &b4)) return GDO_CORRUPT;
            uint32_t len = (((uint32_t)(first & 1) << 8) | b2) + 1;
            uint32_t bw = ((b3 >> 5) & 7) + 1;
            uint32_t pw = RLEV2_WIDTH_DECODE[b3 & 0x1f];
            uint32_t pgw = ((b4 >> 5) & 7) + 1;
            uint32_t pll = b4 & 0x1f;
            uint64_t base = 0;
            for (uint32_t i = 0; i < bw; ++i) {
                uint8_t b;
                if (rd_byte(&r, &b)) return GDO_CORRUPT;
                base = (base << 8) | b;
            }
            int64_t sbase;
            uint64_t msb = 1ull << (8 * bw - 1);
            if (base & msb) sbase = -(int64_t)(base & ~msb); /* FIX Q4 */
            else sbase = (int64_t)base;
            if (o + len > n_vals) return GDO_OVERRUN;
            uint32_t bl = 0, cur = 0;
            if (rd_longs(&r, vals + o, len, fbw, &bl, &cur)) return GDO_CORRUPT;
            int64_t plist[32];
            uint32_t cfb = rlev2_closest_fixed(pw + pgw);
            /* the patch list continues in the same bit stream position as the
               reference: readLongs starts a fresh byte (bitsLeft = 0) */
            bl = 0;
            cur = 0;
            if (rd_longs(&r, plist, pll, cfb, &bl, &cur)) return GDO_CORRUPT;
            uint64_t pmask = (pw >= 64) ? ~0ull : ((1ull << pw) - 1); /* FIX Q1 */
            uint64_t gap = 0;
            for (uint32_t p = 0; p < pll; ++p) {
                gap += (uint64_t)plist[p] >> pw;
                if (gap >= len) return GDO_CORRUPT;
                vals[o + gap] = (int64_t)((uint64_t)vals[o + gap] |
                                          (((uint64_t)plist[p] & pmask) << fbw));
            }
            for (uint32_t i = 0; i < len; ++i) vals[o + i] = (int64_t)((uint64_t)vals[o + i] + (uint64_t)sbase);
            o += len;
        } else { /* DELTA, decoder.h:93-133 */
            uint32_t efbw = (first >> 1) & 0x1f;
            uint32_t fbw = RLEV2_WIDTH_DECODE[efbw];
            uint8_t b;
            if (rd_byte(&r, &b)) return GDO_CORRUPT;
            uint32_t len = (((uint32_t)(first & 1) << 8) | b) + 1;
            uint64_t ubase, zz;
            if (rd_uvarint(&r, &ubase) || rd_uvarint(&r, &zz)) return GDO_CORRUPT;
            int64_t bv = (int64_t)ubase;
            int64_t bd = (int64_t)(zz >> 1) ^ -(int64_t)(zz & 1);
            if (len < 2 || o + len > n_vals) return (len < 2) ? GDO_CORRUPT : GDO_OVERRUN;
            vals[o++] = bv;
            bv = (int64_t)((uint64_t)bv + (uint64_t)bd);
            vals[o++] = bv;
            if (efbw != 0) {
                uint32_t bl = 0, cur = 0;
                if (rd_longs(&r, vals + o, len - 2, fbw, &bl, &cur)) return GDO_CORRUPT;
                for (uint32_t i = 0; i < len - 2; ++i) { /* FIX Q2 */
                    if (bd > 0) bv = (int64_t)((uint64_t)bv + (uint64_t)vals[o + i]);
                    else bv = (int64_t)((uint64_t)bv - (uint64_t)vals[o + i]);
                    vals[o + i] = bv;
                }
            } else {
                for (uint32_t i = 0; i < len - 2; ++i) {
                    bv = (int64_t)((uint64_t)bv + (uint64_t)bd);
                    vals[o + i] = bv;
                }
            }
            o += len - 2;
        }
    }
    *produced = o;
    return GDO_OK;
}

/*
 * Whole-container RLE v2 decode (rlev2::decompress_gpu,
 * include/rlev2/decoder_trans.h:615-681; inflate decoder_new.h:618-657).
 * Lane t of chunk c owns the 8-byte values at chunk-local index
 * t*RU + k*32*RU + j, j < RU (encoder_trans.h:40-108, decoder_new.h:366,395-400).
 * A lane stops when its stream bytes are consumed; it must have produced
 * exactly chunk_size/256 values.
 */
int gdo_rlev2_decode(const uint8_t* data, uint64_t data_len, const uint64_t* blk_off,
                     const uint64_t* col_len, uint32_t n_chunks, uint64_t chunk_size,
                     uint32_t read_unit, uint8_t* out, uint64_t out_total) {
    if (read_unit == 0 || chunk_size % (256ull * read_unit)) return GDO_INVALID;
    uint64_t n_vals = chunk_size / 8 / 32;
    int64_t* vals = (int64_t*)malloc(n_vals * 8);
    int64_t* tmp = (int64_t*)malloc(chunk_size);
    uint8_t* lanes[32];
    uint64_t cap = 0;
    for (uint64_t i = 0; i < 32ull * n_chunks; ++i)
        if (col_len[i] + 8 > cap) cap = col_len[i] + 8;
    for (int t = 0; t < 32; ++t) lanes[t] = (uint8_t*)calloc(cap, 1);
    int rc = GDO_OK;
    for (uint32_t c = 0; c < n_chunks && rc == GDO_OK; ++c) {
        if (blk_off[c] > data_len) { rc = GDO_CORRUPT; break; }
        rc = deinterleave(data + blk_off[c], data_len - blk_off[c], col_len + 32ull * c, lanes);
        for (int t = 0; t < 32 && rc == GDO_OK; ++t) {
            uint64_t got = 0;
            rc = rlev2_decode_lane(lanes[t], col_len[32ull * c + t], vals, n_vals, &got);
            if (rc == GDO_OK && got != n_vals) rc = GDO_CORRUPT;
            for (uint64_t i = 0; i < n_vals && rc == GDO_OK; ++i) {
                uint64_t k = i / read_unit, j = i % read_unit;
                tmp[(uint64_t)t * read_unit + k * 32 * read_unit + j] = vals[i];
            }
        }
        if (rc) break;
        uint64_t base = (uint64_t)c * chunk_size;
        if (base < out_total) {
            uint64_t n = out_total - base < chunk_size ? out_total - base : chunk_size;
            memcpy(out + base, tmp, n);
        }
    }
    for (int t = 0; t < 32; ++t) free(lanes[t]);
    free(vals);
    free(tmp);
    return rc;
}

/* ------------------------------------------------------------------------ */
/* LZSS, interleaved container                                               */
/* ------------------------------------------------------------------------ */

/*
 * Decode one LZSS column stream of col_bytes output bytes.
 * Restates lzss::decompress_func (interleaved variant),
 * include/lzss/lzss_gpu2.h:112-325, with the contiguous form
 * lzss_gpu2.h:718-792 / lzss_cpu.h:110 as the grammar reference:
 *   a flag byte, then 8 tokens LSB-first; bit 1 = one literal byte;
 *   bit 0 = 2-byte little-endian v, length = (v & 31) + 3, offset = v >> 5,
 *   copied from this column's own history (offset bytes back).
 * The column stops when its output is complete; a trailing flag byte that
 * the encoder reserves after a full group of 8 tokens carries no tokens.
 */
static int lzss_decode_column(const uint8_t* s, uint64_t s_len, uint8_t* col, uint64_t col_bytes) {
    uint64_t p = 0, o = 0;
    while (o < col_bytes) {
        if (p >= s_len) return GDO_CORRUPT;
        uint8_t flags = s[p++];
        for (int i = 0; i < 8 && o < col_bytes; ++i, flags >>= 1) {
            if (flags & 1) {
                if (p >= s_len) return GDO_CORRUPT;
                col[o++] = s[p++];
            } else {
                if (p + 2 > s_len) return GDO_CORRUPT;
                uint32_t v = (uint32_t)s[p] | ((uint32_t)s[p + 1] << 8);
                p += 2;
                uint32_t len = (v & 31) + 3, off = v >> 5;
                if (off == 0 || off > o) return GDO_CORRUPT;
                if (o + len > col_bytes) return GDO_OVERRUN;
                for (uint32_t j = 0; j < len; ++j, ++o) col[o] = col[o - off];
            }
        }
    }
    if (p > s_len) return GDO_CORRUPT;
    return GDO_OK;
}

/*
 * Whole-container LZSS decode (lzss::decompress_gpu(in,len,meta,...),
 * include/lzss/lzss_gpu2.h:2129-2314).  Metadata: blk_off[n+1], col_len
 * (32 per chunk, sorted descending, the stream length of rank r), col_map
 * (rank -> output column).  Column q of chunk c owns output bytes
 * c*chunk_size + 4q + 128k .. +3 (lzss_gpu2.h:152,239-248).
 */
int gdo_lzss_decode(const uint8_t* data, uint64_t data_len, const uint64_t* blk_off,
                    const uint64_t* col_len, const uint8_t* col_map, uint32_t n_chunks,
                    uint64_t chunk_size, uint8_t* out, uint64_t out_total) {
    if (chunk_size == 0 || chunk_size % 128) return GDO_INVALID;
    uint64_t col_bytes = chunk_size / 32;
    uint8_t* col = (uint8_t*)malloc(col_bytes);
    uint8_t* tmp = (uint8_t*)malloc(chunk_size);
    uint8_t* ranks[32];
    uint64_t cap = 0;
    for (uint64_t i = 0; i < 32ull * n_chunks; ++i)
        if (col_len[i] + 8 > cap) cap = col_len[i] + 8;
    for (int t = 0; t < 32; ++t) ranks[t] = (uint8_t*)calloc(cap, 1);
    int rc = GDO_OK;
    for (uint32_t c = 0; c < n_chunks && rc == GDO_OK; ++c) {
        if (blk_off[c] > data_len) { rc = GDO_CORRUPT; break; }
        rc = deinterleave(data + blk_off[c], data_len - blk_off[c], col_len + 32ull * c, ranks);
        for (int r = 0; r < 32 && rc == GDO_OK; ++r) {
            uint32_t q = col_map[32ull * c + r];
            if (q >= 32) { rc = GDO_CORRUPT; break; }
            rc = lzss_decode_column(ranks[r], col_len[32ull * c + r], col, col_bytes);
            for (uint64_t k = 0; k < col_bytes / 4 && rc == GDO_OK; ++k)
                memcpy(tmp + 128 * k + 4 * q, col + 4 * k, 4);
        }
        if (rc) break;
        uint64_t base = (uint64_t)c * chunk_size;
        if (base < out_total) {
            uint64_t n = out_total - base < chunk_size ? out_total - base : chunk_size;
            memcpy(out + base, tmp, n);
        }
    }
    for (int t = 0; t < 32; ++t) free(ranks[t]);
    free(col);
    free(tmp);
    return rc;
}

/* ------------------------------------------------------------------------ */
/* LZSS, contiguous container                                                */
/* ------------------------------------------------------------------------ */

/*
 * lzss::decompress_gpu_base container (include/lzss/lzss.h:1126-1188):
 * [u64 in_n_bytes][u32 chunk_size][u32 n_chunks][u32 hist][u32 min][u32 max]
 * [u64 end of every chunk's stream][data].  Each chunk is decoded as
 * lzss::decompress_func (lzss.h:234-305) does: flag byte, then up to 8 tokens
 * while compressed bytes remain (literal = 1 byte, match = 2-byte v with
 * length (v & 31) + 3 and offset v >> 5 back in the chunk's own output).
 * Chunk c's output is bytes [c*chunk_size, ..) (the last chunk may be short).
 */
int gdo_lzss_contig_decode(const uint8_t* in, uint64_t in_len, uint8_t* out, uint64_t out_cap) {
    if (in_len < 28) return GDO_CORRUPT;
    uint64_t n;
    uint32_t h[5];
    memcpy(&n, in, 8);
    memcpy(h, in + 8, 20);
    const uint64_t chunk = h[0], nc = h[1];
    if (chunk == 0 || n > out_cap || nc != (n ? (n - 1) / chunk + 1 : 0)) return GDO_CORRUPT;
    if (in_len < 28 + 8 * nc) return GDO_CORRUPT;
    const uint8_t* data = in + 28 + 8 * nc;
    const uint64_t dlen = in_len - 28 - 8 * nc;
    uint64_t beg = 0;
    for (uint64_t c = 0; c < nc; ++c) {
        uint64_t end;
        memcpy(&end, in + 28 + 8 * c, 8);
        if (end < beg || end > dlen) return GDO_CORRUPT;
        const uint8_t* s = data + beg;
        const uint64_t sl = end - beg;
        uint8_t* o = out + c * chunk;
        const uint64_t want = n - c * chunk < chunk ? n - c * chunk : chunk;
        uint64_t p = 0, q = 0;
        while (p < sl) {
            uint8_t flags = s[p++];
            for (int i = 0; i < 8 && p < sl; ++i, flags >>= 1) {
                if (flags & 1) {
                    if (q >= want) return GDO_OVERRUN;
                    o[q++] = s[p++];
                } else {
                    if (p + 2 > sl) return GDO_CORRUPT;
                    uint32_t v = (uint32_t)s[p] | ((uint32_t)s[p + 1] << 8);
                    p += 2;
                    uint32_t len = (v & 31) + 3, off = v >> 5;
                    if (off == 0 || off > q) return GDO_CORRUPT;
                    if (q + len > want) return GDO_OVERRUN;
                    for (uint32_t j = 0; j < len; ++j, ++q) o[q] = o[q - off];
                }
            }
        }
        if (q != want) return GDO_CORRUPT;
        beg = end;
    }
    return GDO_OK;
}

/* ------------------------------------------------------------------------ */
/* Byte-RLE, flag-byte interleaved container                                 */
/* ------------------------------------------------------------------------ */

/*
 * One column stream of brle_trans (restates brle_trans::decompress_func,
 * include/brle/brle_trans.h:72-202): a flag byte, then 8 items, flag bits
 * LSB first; bit 1 = one literal byte, bit 0 = a count byte then a value
 * byte written count times.  After the 8th item the next byte is a flag
 * byte again (a reserved trailing one carries no items).  The column must
 * produce exactly col_bytes bytes.
 */
static int brle_trans_decode_column(const uint8_t* s, uint64_t s_len, uint8_t* col, uint64_t col_bytes) {
    uint64_t p = 0, o = 0;
    uint32_t block = 0, head = 0;
    while (p < s_len) {
        uint8_t v = s[p++];
        if (block == 0) {
            head = v;
            block = 1;
            continue;
        }
        const uint32_t lit = head & 1;
        head >>= 1;
        if (++block == 9) block = 0;
        if (lit) {
            if (o >= col_bytes) return GDO_OVERRUN;
            col[o++] = v;
        } else {
            if (p >= s_len) return GDO_CORRUPT;  /* a count without its value byte */
            const uint8_t x = s[p++];
            if (o + v > col_bytes) return GDO_OVERRUN;
            for (uint32_t k = 0; k < v; ++k) col[o++] = x;
        }
    }
    return o == col_bytes ? GDO_OK : GDO_CORRUPT;
}

/*
 * Whole-container decode (brle_trans::decompress_gpu, brle_trans.h:661-791):
 * blk_off[n+1], col_len[32n] (sorted descending), col_map[32n] (rank ->
 * column); column q of chunk c owns output bytes c*chunk_size + 4q + 128k
 * .. +3 (brle_trans.h:107-119,146-159).
 */
int gdo_brle_trans_decode(const uint8_t* data, uint64_t data_len, const uint64_t* blk_off,
                          const uint64_t* col_len, const uint8_t* col_map, uint32_t n_chunks,
                          uint64_t chunk_size, uint8_t* out, uint64_t out_total) {
    if (chunk_size == 0 || chunk_size % 128) return GDO_INVALID;
    uint64_t col_bytes = chunk_size / 32;
    uint8_t* col = (uint8_t*)malloc(col_bytes);
    uint8_t* tmp = (uint8_t*)malloc(chunk_size);
    uint8_t* ranks[32];
    uint64_t cap = 0;
    for (uint64_t i = 0; i < 32ull * n_chunks; ++i)
        if (col_len[i] + 8 > cap) cap = col_len[i] + 8;
    for (int t = 0; t < 32; ++t) ranks[t] = (uint8_t*)calloc(cap, 1);
    int rc = GDO_OK;
    for (uint32_t c = 0; c < n_chunks && rc == GDO_OK; ++c) {
        if (blk_off[c] > data_len) { rc = GDO_CORRUPT; break; }
        rc = deinterleave(data + blk_off[c], data_len - blk_off[c], col_len + 32ull * c, ranks);
        for (int r = 0; r < 32 && rc == GDO_OK; ++r) {
            uint32_t q = col_map[32ull * c + r];
            if (q >= 32) { rc = GDO_CORRUPT; break; }
            rc = brle_trans_decode_column(ranks[r], col_len[32ull * c + r], col, col_bytes);
            for (uint64_t k = 0; k < col_bytes / 4 && rc == GDO_OK; ++k)
                memcpy(tmp + 128 * k + 4 * q, col + 4 * k, 4);
        }
        if (rc) break;
        uint64_t base = (uint64_t)c * chunk_size;
        if (base < out_total) {
            uint64_t n = out_total - base < chunk_size ? out_total - base : chunk_size;
            memcpy(out + base, tmp, n);
        }
    }
    for (int t = 0; t < 32; ++t) free(ranks[t]);
    free(col);
    free(tmp);
    return rc;
}

/*
 * One column stream of the 4-byte-symbol variant (restates
 * brle::decompress_func of include/brle/brle_gpu_4B.h:75-223): the same
 * flag-byte grammar over 4-byte symbols -- bit 1 = one literal symbol (4
 * bytes), bit 0 = a count byte then a symbol written count times.
 */
static int brle_trans4_decode_column(const uint8_t* s, uint64_t s_len, uint8_t* col, uint64_t col_bytes) {
    uint64_t p = 0, o = 0;
    uint32_t block = 0, head = 0;
    while (p < s_len) {
        uint8_t v = s[p];
        if (block == 0) {
            head = v;
            block = 1;
            ++p;
            continue;
        }
        const uint32_t lit = head & 1;
        head >>= 1;
        if (++block == 9) block = 0;
        uint32_t cnt = 1;
        if (!lit) {
            cnt = v;
            ++p;
        }
        if (p + 4 > s_len) return GDO_CORRUPT;  /* an item cut short */
        if (o + 4ull * cnt > col_bytes) return GDO_OVERRUN;
        for (uint32_t k = 0; k < cnt; ++k, o += 4) memcpy(col + o, s + p, 4);
        p += 4;
    }
    return o == col_bytes ? GDO_OK : GDO_CORRUPT;
}

/*
 * Whole-container decode of brle_trans (sym 1) or its 4-byte-symbol variant
 * (sym 4, brle::decompress_gpu in brle_gpu_4B.h:717-897, 8 KiB chunks in the
 * reference): the same ranked 32-column container.
 */
static int brle_flag_container_decode(const uint8_t* data, uint64_t data_len, const uint64_t* blk_off,
                                      const uint64_t* col_len, const uint8_t* col_map, uint32_t n_chunks,
                                      uint64_t chunk_size, uint8_t* out, uint64_t out_total, int sym) {
    if (chunk_size == 0 || chunk_size % 128) return GDO_INVALID;
    uint64_t col_bytes = chunk_size / 32;
    uint8_t* col = (uint8_t*)malloc(col_bytes);
    uint8_t* tmp = (uint8_t*)malloc(chunk_size);
    uint8_t* ranks[32];
    uint64_t cap = 0;
    for (uint64_t i = 0; i < 32ull * n_chunks; ++i)
        if (col_len[i] + 8 > cap) cap = col_len[i] + 8;
    for (int t = 0; t < 32; ++t) ranks[t] = (uint8_t*)calloc(cap, 1);
    int rc = GDO_OK;
    for (uint32_t c = 0; c < n_chunks && rc == GDO_OK; ++c) {
        if (blk_off[c] > data_len) { rc = GDO_CORRUPT; break; }
        rc = deinterleave(data + blk_off[c], data_len - blk_off[c], col_len + 32ull * c, ranks);
        for (int r = 0; r < 32 && rc == GDO_OK; ++r) {
            uint32_t q = col_map[32ull * c + r];
            if (q >= 32) { rc = GDO_CORRUPT; break; }
            rc = sym == 4 ? brle_trans4_decode_column(ranks[r], col_len[32ull * c + r], col, col_bytes)
                          : brle_trans_decode_column(ranks[r], col_len[32ull * c + r], col, col_bytes);
            for (uint64_t k = 0; k < col_bytes / 4 && rc == GDO_OK; ++k)
                memcpy(tmp + 128 * k + 4 * q, col + 4 * k, 4);
        }
        if (rc) break;
        uint64_t base = (uint64_t)c * chunk_size;
        if (base < out_total) {
            uint64_t n = out_total - base < chunk_size ? out_total - base : chunk_size;
            memcpy(out + base, tmp, n);
        }
    }
    for (int t = 0; t < 32; ++t) free(ranks[t]);
    free(col);
    free(tmp);
    return rc;
}

int gdo_brle_trans4_decode(const uint8_t* data, uint64_t data_len, const uint64_t* blk_off,
                           const uint64_t* col_len, const uint8_t* col_map, uint32_t n_chunks,
                           uint64_t chunk_size, uint8_t* out, uint64_t out_total) {
    return brle_flag_container_decode(data, data_len, blk_off, col_len, col_map, n_chunks, chunk_size, out,
                                      out_total, 4);
}

/* ------------------------------------------------------------------------ */
/* Deflate / zlib                                                           */
/* ------------------------------------------------------------------------ */

/*
 * Inflate each chunk with system zlib (the algorithm the reference's
 * Deflate container is produced with: zlib.compress in
 * orig_compressor.py:87, consumed by deflate::decompress_gpu,
 * include/zlib/zlib.h:966-1082, which skips the 2-byte zlib header,
 * zlib.h:580).  zlib_header 1: each stream is a zlib stream (RFC 1950);
 * 2: a gzip member (RFC 1952; the header cudf::io::gpuinflate parses with
 * parse_hdr, cudf_deflate.cuh:1180-1216); 0: raw deflate (RFC 1951).  Chunk i: compressed bytes
 * data[comp_off[i] .. comp_off[i]+comp_len[i]), output
 * out[out_off[i] .. out_off[i+1]).
 */
int gdo_inflate(const uint8_t* data, const uint64_t* comp_off, const uint64_t* comp_len,
                const uint64_t* out_off, uint32_t n_chunks, int zlib_header, uint8_t* out) {
    for (uint32_t c = 0; c < n_chunks; ++c) {
        z_stream zs;
        memset(&zs, 0, sizeof(zs));
        /* 0 raw deflate, 1 zlib (RFC 1950), 2 gzip member (RFC 1952) */
        const int wbits = zlib_header == 2 ? 15 + 16 : (zlib_header ? 15 : -15);
        if (inflateInit2(&zs, wbits) != Z_OK) return GDO_INVALID;
        zs.next_in = (Bytef*)(data + comp_off[c]);
        zs.avail_in = (uInt)comp_len[c];
        uint64_t want = out_off[c + 1] - out_off[c];
        zs.next_out = out + out_off[c];
        zs.avail_out = (uInt)want;
        int zr = inflate(&zs, Z_FINISH);
        uint64_t got = zs.total_out;
        inflateEnd(&zs);
        if (zr != Z_STREAM_END) return (zr == Z_BUF_ERROR && got == want) ? GDO_OVERRUN : GDO_CORRUPT;
        if (got != want) return GDO_CORRUPT;
    }
    return GDO_OK;
}

/* Version tag so tests can check they loaded this file's build. */
const char* gdo_version(void) { return "gd-oracle-1"; }

/* Single-stream entry points (the per-lane / per-column grammars above), for
 * checking against the reference's contiguous codecs. */
int gdo_rlev2_decode_stream(const uint8_t* s, uint64_t len, int64_t* vals, uint64_t n_vals) {
    uint64_t got = 0;
    int rc = rlev2_decode_lane(s, len, vals, n_vals, &got);
    if (rc == GDO_OK && got != n_vals) rc = GDO_CORRUPT;
    return rc;
}

int gdo_lzss_decode_stream(const uint8_t* s, uint64_t len, uint8_t* out, uint64_t n_out) {
    return lzss_decode_column(s, len, out, n_out);
}

/*
 * Lane / column streams of an interleaved container (RLE v1, RLE v2, LZSS,
 * byte-RLE transposed), written back to back in slot order: stream 32c+s is
 * col_len[32c+s] bytes at out + out_off[32c+s], so that the reference's
 * contiguous per-stream decoders (rlev2::block_decode, decoder.h:190;
 * lzss::decompress_func, lzss_cpu.h:110) can be run on each one.
 * out_off has 32*n_chunks + 1 entries.
 */
int gdo_export_lanes(const uint8_t* data, uint64_t data_len, const uint64_t* blk_off,
                     const uint64_t* col_len, uint32_t n_chunks, uint8_t* out, uint64_t* out_off) {
    uint8_t* lanes[32];
    uint64_t cap = 0;
    for (uint64_t i = 0; i < 32ull * n_chunks; ++i)
        if (col_len[i] + 8 > cap) cap = col_len[i] + 8;
    for (int t = 0; t < 32; ++t) lanes[t] = (uint8_t*)calloc(cap ? cap : 8, 1);
    int rc = GDO_OK;
    uint64_t pos = 0;
    out_off[0] = 0;
    for (uint32_t c = 0; c < n_chunks && rc == GDO_OK; ++c) {
        if (blk_off[c] > data_len) { rc = GDO_CORRUPT; break; }
        rc = deinterleave(data + blk_off[c], data_len - blk_off[c], col_len + 32ull * c, lanes);
        for (int s = 0; s < 32 && rc == GDO_OK; ++s) {
            uint64_t n = col_len[32ull * c + s];
            memcpy(out + pos, lanes[s], n);
            pos += n;
            out_off[32ull * c + s + 1] = pos;
        }
    }
    for (int t = 0; t < 32; ++t) free(lanes[t]);
    return rc;
}
