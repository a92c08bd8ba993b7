// gd_encode.cpp -- host encoders for every container the decoders read.
//
// These produce the compressed inputs (the "compress" half of each codec
// pair).  Each encoder restates the reference encoder's choices exactly so
// that the byte streams match what the reference writes for the same input;
// the citations name the reference routine restated.  Encoders run on the
// host, one std::thread per core, over independent chunks.
#include <algorithm>
#include <atomic>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <vector>
#include <zlib.h>

#include "../../../include/gd.h"

namespace {

template <typename F>
void parallel_for(uint64_t n, F&& f) {
    unsigned nt = std::thread::hardware_concurrency();
    if (nt == 0) nt = 1;
    if (nt > n) nt = (unsigned)n;
    if (nt <= 1) {
        for (uint64_t i = 0; i < n; ++i) f(i);
        return;
    }
    std::atomic<uint64_t> next{0};
    std::vector<std::thread> th;
    for (unsigned t = 0; t < nt; ++t)
        th.emplace_back([&]() {
            for (;;) {
                uint64_t i = next.fetch_add(1);
                if (i >= n) break;
                f(i);
            }
        });
    for (auto& x : th) x.join();
}

// Interleave 32 slot streams in 4-byte words: row k holds one word of every
// slot whose length exceeds 4k, in slot order.  Pad bytes are zero.
// rle_v1/encoder.h:564-588 (write_byte_op), rlev2/encoder_trans.h:291-349
// (tranpose_col_len_single), lzss/lzss_gpu2.h:497-509 (writeupdate).
void interleave(const std::vector<uint8_t>* slot[32], const uint64_t len[32], uint8_t* dst) {
    uint64_t rows = 0;
    for (int s = 0; s < 32; ++s) rows = std::max<uint64_t>(rows, (len[s] + 3) / 4);
    uint64_t pos = 0;
    for (uint64_t k = 0; k < rows; ++k)
        for (int s = 0; s < 32; ++s)
            if (len[s] > 4 * k) {
                for (int b = 0; b < 4; ++b) {
                    uint64_t i = 4 * k + b;
                    dst[pos + b] = i < len[s] ? (*slot[s])[i] : 0;
                }
                pos += 4;
            }
}

// Size of an interleaved block: 4-byte padded lanes, rounded to 128 bytes
// (rle_v1/encoder.h:504-520, rlev2/encoder_trans.h:240-251,
// lzss/lzss_gpu2.h:485-493).
uint64_t block_bytes(const uint64_t len[32]) {
    uint64_t s = 0;
    for (int t = 0; t < 32; ++t) s += (len[t] + 3) / 4 * 4;
    return (s + 127) / 128 * 128;
}

// ---------------------------------------------------------------------------
// Byte-RLE (brle.h format)
// ---------------------------------------------------------------------------

// brle::encode, include/brle/brle.h:129-230 (non-lookahead path).
void brle_encode_chunk(const uint8_t* in, uint64_t n, std::vector<uint8_t>& out) {
    uint8_t lit[128];
    uint32_t num = 0, tail = 0;
    bool rep = false;
    auto flush = [&]() {
        if (num == 0) return;
        if (rep) {
            out.push_back((uint8_t)(num - 3));
            out.push_back(lit[0]);
        } else {
            out.push_back((uint8_t)(num + 127));
            out.insert(out.end(), lit, lit + num);
        }
        rep = false;
        tail = 0;
        num = 0;
    };
    for (uint64_t i = 0; i < n; ++i) {
        uint8_t c = in[i];
        if (num == 0) {
            lit[num++] = c;
            tail = 1;
        } else if (rep) {
            if (c == lit[0]) {
                if (++num == 130) flush();
            } else {
                flush();
                lit[num++] = c;
                tail = 1;
            }
        } else {
            tail = (c == lit[num - 1]) ? tail + 1 : 1;
            if (tail == 3) {
                if (num + 1 == 3) {
                    num += 1;
                    rep = true;
                } else {
                    num -= 2;
                    flush();
                    lit[0] = c;
                    num = 3;
                    rep = true;
                }
            } else {
                lit[num++] = c;
                if (num == 128) flush();
            }
        }
    }
    flush();
}

// ---------------------------------------------------------------------------
// RLE v1 (per-lane stream)
// ---------------------------------------------------------------------------

template <typename T>
void put_varint(std::vector<uint8_t>& o, T v) {
    do {
        uint8_t b = v & 0x7f;
        if ((v & ~(T)0x7f) != 0) b |= 0x80;
        o.push_back(b);
        v = v >> 7;
    } while (v != 0);
}

// compression_warp, include/rle_v1/encoder.h:607-1018, with write_byte_op's
// interleave factored out: this emits lane `vals`' byte stream.
template <typename T>
void rlev1_encode_lane(const T* vals, uint64_t n, std::vector<uint8_t>& o) {
    T buf[2] = {0, 0};
    uint8_t head = 0, count = 0;
    T first_val = 0;
    uint16_t dcount = 0;
    int8_t cur_delta = 0;
    bool dflag = false;
    uint64_t lit_idx = 0;
    uint16_t lcount = 0;
    T prev = 0;
    uint64_t i = 0;
    auto diff = [](T a, T b) -> int64_t { return (int64_t)(T)(a - b); };
    auto push = [&](T v) {
        buf[head] = v;
        head = (head + 1) % 2;
    };
    auto start_lit = [&]() {
        lit_idx = o.size();
        o.push_back(1);
    };
    auto write_run = [&](int hdr) {
        o.push_back((uint8_t)(int8_t)hdr);
        o.push_back((uint8_t)cur_delta);
        put_varint<T>(o, first_val);
    };
    // first value (:688-697)
    T rd = vals[i++];
    dcount = 1;
    prev = rd;
    push(rd);
    count++;
    // second value (:699-739)
    rd = vals[i++];
    int64_t td = diff(rd, prev);
    if (td > 127 || td < -128) {
        dflag = false;
        start_lit();
        lcount = 1;
        put_varint<T>(o, buf[0]);
        count--;
    } else {
        dflag = true;
        cur_delta = (int8_t)td;
        dcount++;
    }
    prev = rd;
    push(rd);
    count++;
    while (i < n) {
        if (lcount == 127) {  // :745-754
            o[lit_idx] = (uint8_t)(int8_t)(-(int)lcount);
            lcount = 0;
        }
        rd = vals[i++];
        if (dcount == 1) {  // :787-822
            td = diff(rd, prev);
            if (td > 127 || td < -128) {
                dflag = false;
                if (lcount == 0) start_lit();
                uint8_t tail = (head == 0) ? 1 : 0;
                put_varint<T>(o, buf[tail]);
                lcount++;
                count--;
            } else {
                dflag = true;
                cur_delta = (int8_t)td;
                dcount++;
            }
            prev = rd;
            push(rd);
            count++;
            continue;
        }
        if ((T)(prev + (T)cur_delta) == rd && dflag) {  // :825-865
            dcount++;
            if (dcount == 3) {
                first_val = buf[head];
                if (lcount != 0) {
                    o[lit_idx] = (uint8_t)(int8_t)(-(int)lcount);
                    lcount = 0;
                }
            } else if (dcount == 130) {
                write_run(dcount - 4);
                dcount = 1;
                count = 0;
                lcount = 0;
            }
            push(rd);
            count = std::min<uint8_t>(count + 1, 2);
            prev = rd;
        } else {
            if (dcount >= 3) {  // :872-903
                write_run(dcount - 3);
                dcount = 1;
                count = 0;
                lcount = 0;
                push(rd);
                count = std::min<uint8_t>(count + 1, 2);
                prev = rd;
            } else {  // :905-969
                if (lcount == 0) {
                    lit_idx = o.size();
                    o.push_back(3);
                }
                lcount++;
                put_varint<T>(o, buf[head]);
                if (lcount == 127) {
                    o[lit_idx] = (uint8_t)(int8_t)(-(int)lcount);
                    lcount = 0;
                }
                td = diff(rd, prev);
                if (td > 127 || td < -128) {
                    if (lcount == 0) {
                        lit_idx = o.size();
                        o.push_back(3);
                    }
                    dflag = false;
                    count = 0;
                    uint8_t tail = (head == 0) ? 1 : 0;
                    put_varint<T>(o, buf[tail]);
                    lcount++;
                    dcount = 1;
                } else {
                    count = 1;
                    dflag = true;
                    cur_delta = (int8_t)td;
                    dcount = 2;
                }
                prev = rd;
                push(rd);
                count = std::min<uint8_t>(count + 1, 2);
            }
        }
    }
    // tail (:975-1052)
    if (dcount >= 3 && dflag) {
        write_run(dcount - 3);
    } else {
        if (count == 1) {
            if (lcount == 127) {
                o[lit_idx] = (uint8_t)(int8_t)(-(int)lcount);
                lcount = 0;
            }
            if (lcount == 0) start_lit();
            uint8_t tail = (head == 0) ? 1 : 0;
            put_varint<T>(o, buf[tail]);
            lcount++;
        }
        if (count == 2) {
            if (lcount == 127) {
                o[lit_idx] = (uint8_t)(int8_t)(-(int)lcount);
                lcount = 0;
            }
            if (lcount == 0) start_lit();
            put_varint<T>(o, buf[head]);
            lcount++;
            if (lcount == 127) {
                o[lit_idx] = (uint8_t)(int8_t)(-(int)lcount);
                lcount = 0;
            }
            if (lcount == 0) start_lit();
            head = (head + 1) % 2;
            put_varint<T>(o, buf[head]);
            lcount++;
        }
        o[lit_idx] = (uint8_t)(int8_t)(-(int)lcount);
    }
}

// ---------------------------------------------------------------------------
// RLE v2 (per-lane stream, HEAD-side semantics of include/rlev2/encoder.h)
// ---------------------------------------------------------------------------

const uint8_t W_DECODE[32] = {1,  2,  3,  4,  5,  6,  7,  8,  9,  10, 11, 12, 13, 14, 15, 16,
                              17, 18, 19, 20, 21, 22, 23, 24, 26, 28, 30, 32, 40, 48, 56, 64};
// utils.h:40-51
uint8_t w_encode(uint32_t w) {
    if (w <= 1) return 0;
    if (w <= 24) return (uint8_t)(w - 1);
    if (w <= 26) return 24;
    if (w <= 28) return 25;
    if (w <= 30) return 26;
    if (w <= 32) return 27;
    if (w <= 40) return 28;
    if (w <= 48) return 29;
    if (w <= 56) return 30;
    return 31;
}
// utils.h:53-60
uint8_t w_closest(uint32_t b) {
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
// utils.h:62-69
uint8_t w_closest_aligned(uint32_t b) {
    if (b <= 1) return 1;
    if (b <= 2) return 2;
    if (b <= 4) return 4;
    if (b <= 8) return 8;
    if (b <= 16) return 16;
    if (b <= 24) return 24;
    if (b <= 32) return 32;
    if (b <= 40) return 40;
    if (b <= 48) return 48;
    if (b <= 56) return 56;
    return 64;
}

struct V2Info {
    int64_t deltas[128];
    int64_t literals[128];
    uint32_t num_literals = 0, fix_runlen = 0, var_runlen = 0;
    uint8_t delta_bits = 0;
    bool is_fixed_delta = false;
    std::vector<uint8_t>* out;
    void w(uint8_t b) { out->push_back(b); }
};

// encoder.h:109-122
uint8_t closest_num_bits(int64_t v) {
    if (v < 0) return w_closest(64);
    uint8_t c = 0;
    uint64_t u = (uint64_t)v;
    while (u) {
        u >>= 1;
        ++c;
    }
    return w_closest(c);
}

// encoder.h:126-165
void write_aligned(const int64_t* in, uint32_t len, uint8_t bits, V2Info& info) {
    if (bits < 8) {
        uint8_t mask = (uint8_t)((1 << bits) - 1);
        uint32_t hops = 8 / bits, rem = len % hops, end = len - rem;
        for (uint32_t i = 0; i < end; i += hops) {
            uint8_t tw = 0;
            for (uint32_t j = 0; j < hops; ++j) tw |= (uint8_t)((in[i + j] & mask) << (8 - (j + 1) * bits));
            info.w(tw);
        }
        if (rem > 0) {
            int shift = 8 - bits;
            uint8_t tw = 0;
            for (uint32_t i = end; i < len; ++i) {
                tw |= (uint8_t)((in[i] & mask) << shift);
                shift -= bits;
            }
            info.w(tw);
        }
    } else {
        int bytes = bits / 8;
        for (uint32_t i = 0; i < len; ++i)
            for (int j = bytes - 1; j >= 0; --j) info.w((uint8_t)(((uint64_t)in[i] >> (j * 8)) & 0xff));
    }
}

// encoder.h:169-216
void write_unaligned(const int64_t* in, uint32_t len, uint8_t bits, V2Info& info) {
    uint32_t left = 8;
    uint8_t cur = 0;
    for (uint32_t i = 0; i < len; ++i) {
        uint64_t value = (uint64_t)in[i];
        uint32_t tw = bits;
        while (tw > left) {
            cur |= (uint8_t)(value >> (tw - left));
            tw -= left;
            value &= (tw >= 64) ? ~0ull : ((1ull << tw) - 1);
            info.w(cur);
            cur = 0;
            left = 8;
        }
        left -= tw;
        cur |= (uint8_t)(value << left);
        if (left == 0) {
            info.w(cur);
            cur = 0;
            left = 8;
        }
    }
    if (left != 8) info.w(cur);
}

// encoder.h:220-228
void bit_hist(const int64_t* d, uint32_t n, uint8_t* hist) {
    for (int i = 0; i < 32; ++i) hist[i] = 0;
    for (uint32_t i = 0; i < n; ++i) hist[w_encode(closest_num_bits(d[i]))]++;
}
// encoder.h:231-242
uint8_t percentile_bits(const uint8_t* hist, uint32_t len, int p) {
    p = std::min(100 - p, 100);
    int32_t plen = (p == 0 ? 0 : (int32_t)((len * p - 1) / 100 + 1));
    for (int i = 31; i >= 0; --i) {
        plen -= hist[i];
        if (plen < 0) return W_DECODE[i];
    }
    return 0;
}

void write_direct(V2Info& info);
void write_delta(V2Info& info);

// encoder.h:538-569
void write_short_repeat(V2Info& info) {
    int64_t val = info.literals[0];
    uint8_t vb = closest_num_bits(val);
    uint8_t nbytes = (uint8_t)((vb - 1) / 8 + 1);
    info.w((uint8_t)(((nbytes - 1) << 3) | (info.fix_runlen - 3)));
    for (int i = nbytes - 1; i >= 0; --i) info.w((uint8_t)(((uint64_t)val >> (i * 8)) & 0xff));
    info.fix_runlen = 0;
    info.num_literals = 0;
}

// encoder.h:580-598
void write_direct(V2Info& info) {
    uint8_t hist[32];
    bit_hist(info.literals, info.num_literals, hist);
    uint8_t nb = percentile_bits(hist, info.num_literals, 100);
    nb = w_closest_aligned(nb);
    uint8_t enc = w_encode(nb);
    uint16_t vl = (uint16_t)(info.var_runlen - 1);
    info.w((uint8_t)(0x40 | (enc << 1) | ((vl & 0x100) >> 8)));
    info.w((uint8_t)(vl & 0xff));
    write_aligned(info.literals, info.num_literals, nb, info);
    info.var_runlen = 0;
    info.num_literals = 0;
}

// encoder.h:600-620
void write_vulong(int64_t v, V2Info& info) {
    uint64_t u = (uint64_t)v;
    for (;;) {
        if ((u & ~0x7full) == 0) {
            info.w((uint8_t)u);
            return;
        }
        info.w((uint8_t)(0x80 | (u & 0x7f)));
        u >>= 7;
    }
}
void write_vslong(int64_t v, V2Info& info) { write_vulong((int64_t)(((uint64_t)v << 1) ^ (uint64_t)(v >> 63)), info); }

// encoder.h:631-697 (HEAD side)
void write_delta(V2Info& info) {
    uint16_t len = 0;
    uint8_t enc = 0;
    uint8_t nb = w_closest_aligned(info.delta_bits);
    if (info.is_fixed_delta) {
        if (info.fix_runlen > 3) {
            len = (uint16_t)(info.fix_runlen - 1);
            info.fix_runlen = 0;
        } else {
            len = (uint16_t)(info.var_runlen - 1);
            info.var_runlen = 0;
        }
    } else {
        if (nb == 1) nb = 2;
        enc = w_encode(nb);
        len = (uint16_t)(info.var_runlen - 1);
        info.var_runlen = 0;
    }
    info.w((uint8_t)(0xC0 | (enc << 1) | ((len & 0x100) >> 8)));
    info.w((uint8_t)(len & 0xff));
    write_vulong(info.literals[0], info);
    write_vslong(info.deltas[0], info);
    if (!info.is_fixed_delta) write_aligned(info.deltas + 1, info.num_literals - 2, nb, info);
    for (int i = 0; i < 128; ++i) info.deltas[i] = 0;
    info.num_literals = 0;
}

struct PatchBlob {
    uint32_t patch_len, patch_width, patch_gap_width;
    uint8_t bits95p, bits100p;
    int64_t literal_min;
    int64_t reduced[128];
    int64_t gap_patch[128];
};

// encoder.h:244-364
void prepare_patched(V2Info& info, PatchBlob& pb) {
    int64_t mask = (int64_t)((1ull << pb.bits95p) - 1);
    pb.patch_len = (info.num_literals + 19) / 20;
    pb.patch_width = w_closest(pb.bits100p - pb.bits95p);
    if (pb.patch_width == 64) {
        pb.patch_width = 56;
        pb.bits95p = 8;
        mask = (int64_t)((1ull << pb.bits95p) - 1);
    }
    uint32_t gi = 0, pi = 0;
    uint64_t prev = 0, max_gap = 0;
    int64_t gaps[128], patches[128];
    for (uint32_t i = 0; i < info.num_literals; ++i) {
        if (pb.reduced[i] > mask) {
            uint64_t gap = i - prev;
            if (gap > max_gap) max_gap = gap;
            prev = i;
            gaps[gi++] = (int64_t)gap;
            patches[pi++] = pb.reduced[i] >> pb.bits95p;
            pb.reduced[i] &= mask;
        }
    }
    pb.patch_len = gi;
    if (max_gap == 0 && pb.patch_len != 0) pb.patch_gap_width = 1;
    else pb.patch_gap_width = closest_num_bits((int64_t)max_gap);
    if (pb.patch_gap_width > 8) {
        pb.patch_gap_width = 8;
        pb.patch_len += (max_gap == 511) ? 2 : 1;
    }
    gi = 0;
    pi = 0;
    uint32_t pos = 0;
    for (uint32_t i = 0; i < pb.patch_len; ++i) {
        int64_t g = gaps[gi++];
        int64_t p = patches[pi++];
        while (g > 255) {
            pb.gap_patch[pos++] = (int64_t)(255ull << pb.patch_width);
            i++;
            g -= 255;
        }
        pb.gap_patch[pos++] = (int64_t)(((uint64_t)g << pb.patch_width) | (uint64_t)p);
    }
}

// encoder.h:700-785
void write_patched(V2Info& info, PatchBlob& pb) {
    uint32_t& vl = info.var_runlen;
    vl -= 1;
    uint8_t h1 = (uint8_t)(0x80 | (w_encode(pb.bits95p) << 1) | ((vl & 0x100) >> 8));
    uint8_t h2 = (uint8_t)(vl & 0xff);
    bool neg = pb.literal_min < 0;
    if (neg) pb.literal_min = -pb.literal_min;
    uint32_t vbits = closest_num_bits(pb.literal_min) + 1;
    uint32_t vbytes = (vbits - 1) / 8 + 1;
    if (neg) pb.literal_min |= (int64_t)(1ull << (vbytes * 8 - 1));
    uint8_t h3 = (uint8_t)(((vbytes - 1) << 5) | w_encode(pb.patch_width));
    uint8_t h4 = (uint8_t)(((pb.patch_gap_width - 1) << 5) | pb.patch_len);
    info.w(h1);
    info.w(h2);
    info.w(h3);
    info.w(h4);
    for (int i = (int)vbytes - 1; i >= 0; --i) info.w((uint8_t)(((uint64_t)pb.literal_min >> (i * 8)) & 0xff));
    write_unaligned(pb.reduced, info.num_literals, w_closest(pb.bits95p), info);
    write_unaligned(pb.gap_patch, pb.patch_len, w_closest(pb.patch_gap_width + pb.patch_width), info);
    info.var_runlen = 0;
    info.num_literals = 0;
}

// encoder.h:85-89 (HEAD): the subtraction safety test, with the reference's
// two's-complement wrap of `smaller - INT64_MIN` made explicit.
bool safe_subtract(int64_t larger, int64_t smaller) {
    if (smaller > 0) return true;
    int64_t t = (int64_t)((uint64_t)smaller - (uint64_t)INT64_MIN);
    return larger > t;
}

// encoder.h:367-535 (HEAD side)
void determine_encoding(V2Info& info) {
    int64_t* lit = info.literals;
    if (info.num_literals <= 3) {
        write_direct(info);
        return;
    }
    bool inc = true, dec = true;
    info.is_fixed_delta = true;
    int64_t lmin = lit[0], lmax = lit[0];
    int64_t init_delta = (int64_t)((uint64_t)lit[1] - (uint64_t)lit[0]);
    int64_t max_delta = 0;
    for (uint32_t i = 1; i < info.num_literals; ++i) {
        int64_t l1 = lit[i], l0 = lit[i - 1];
        int64_t cd = (int64_t)((uint64_t)l1 - (uint64_t)l0);
        lmin = std::min(lmin, l1);
        lmax = std::max(lmax, l1);
        inc &= (l0 <= l1);
        dec &= (l0 >= l1);
        info.is_fixed_delta &= (cd == init_delta);
        int64_t ad = cd < 0 ? (int64_t)(0 - (uint64_t)cd) : cd;
        info.deltas[i - 1] = ad;
        max_delta = std::max(max_delta, ad);
    }
    info.deltas[0] = init_delta;
    if (!safe_subtract(lmax, lmin)) {
        write_direct(info);
        return;
    }
    if (lmin == lmax || info.is_fixed_delta) {
        write_delta(info);
        return;
    }
    if (init_delta != 0) {
        info.delta_bits = closest_num_bits(max_delta);
        if (inc || dec) {
            write_delta(info);
            return;
        }
    }
    uint8_t hist[32];
    bit_hist(info.literals, info.num_literals, hist);
    uint8_t b100 = percentile_bits(hist, info.num_literals, 100);
    uint8_t b90 = percentile_bits(hist, info.num_literals, 90);
    if ((uint32_t)(b100 - b90) > 1) {
        PatchBlob pb;
        pb.literal_min = lmin;
        for (uint32_t i = 0; i < info.num_literals; ++i)
            pb.reduced[i] = (int64_t)((uint64_t)lit[i] - (uint64_t)lmin);
        bit_hist(pb.reduced, info.num_literals, hist);
        pb.bits95p = percentile_bits(hist, info.num_literals, 95);
        pb.bits100p = percentile_bits(hist, info.num_literals, 100);
        if ((pb.bits100p - pb.bits95p) != 0) {
            prepare_patched(info, pb);
            write_patched(info, pb);
        } else {
            write_direct(info);
        }
        return;
    }
    write_direct(info);
}

// block_encode's per-value state machine, encoder.h:840-961 (HEAD side),
// fed with one lane's values in the transposed order of
// rlev2/encoder_trans.h:40-108.
void rlev2_encode_lane(const int64_t* vals, uint64_t n, std::vector<uint8_t>& out) {
    V2Info info;
    for (int i = 0; i < 128; ++i) info.deltas[i] = 0;
    info.out = &out;
    int64_t prev_delta = 0;
    uint32_t& num = info.num_literals;
    int64_t* lit = info.literals;
    for (uint64_t k = 0; k < n; ++k) {
        int64_t val = vals[k];
        if (num == 0) {
            prev_delta = 0;
            lit[num++] = val;
            info.fix_runlen = 1;
            info.var_runlen = 1;
            continue;
        }
        if (num == 1) {
            lit[num++] = val;
            prev_delta = (int64_t)((uint64_t)val - (uint64_t)lit[0]);
            if (val == lit[0]) {
                info.fix_runlen = 2;
                info.var_runlen = 0;
            } else {
                info.fix_runlen = 0;
                info.var_runlen = 2;
            }
            continue;
        }
        int64_t cur_delta = (int64_t)((uint64_t)val - (uint64_t)lit[num - 1]);
        if (prev_delta == 0 && cur_delta == 0) {
            lit[num++] = val;
            if (info.var_runlen > 0) info.fix_runlen = 2;
            info.fix_runlen++;
            if (info.fix_runlen >= 3 && info.var_runlen > 0) {
                num -= 3;
                info.var_runlen -= 2;
                determine_encoding(info);
                for (uint32_t ii = 0; ii < 3; ++ii) lit[ii] = val;
                num = 3;
            }
            if (info.fix_runlen == 128) determine_encoding(info);
            continue;
        }
        if (info.fix_runlen >= 3) {
            if (info.fix_runlen <= 10) {
                write_short_repeat(info);
            } else {
                info.is_fixed_delta = true;
                write_delta(info);
            }
        }
        if (info.fix_runlen > 0 && info.fix_runlen < 3 && val != lit[num - 1]) {
            info.var_runlen = info.fix_runlen;
            info.fix_runlen = 0;
        }
        if (num == 0) {
            lit[num++] = val;
            info.fix_runlen = 1;
            info.var_runlen = 1;
        } else {
            prev_delta = (int64_t)((uint64_t)val - (uint64_t)lit[num - 1]);
            lit[num++] = val;
            info.var_runlen++;
            if (info.var_runlen == 128) determine_encoding(info);
        }
    }
    if (num != 0) {
        if (info.var_runlen != 0) {
            determine_encoding(info);
        } else if (info.fix_runlen != 0) {
            if (info.fix_runlen < 3) {
                info.var_runlen = info.fix_runlen;
                info.fix_runlen = 0;
                determine_encoding(info);
            } else if (info.fix_runlen <= 10) {
                write_short_repeat(info);
            } else {
                info.is_fixed_delta = true;
                write_delta(info);
            }
        }
    }
}

// ---------------------------------------------------------------------------
// LZSS (per-column stream)
// ---------------------------------------------------------------------------

// One column of the interleaved LZSS writer: compress_init_func /
// compress_func_new, include/lzss/lzss_gpu2.h:330-707 (identical token
// grammar to the contiguous compress_func, lzss_cpu.h:540-655).
//
// find_match (lzss_gpu2.h:70-108) scans the 2048-byte history ring from its
// oldest entry (hist_offset 1; offset 0 is never a source), keeps the first
// longest match, stops at 34 bytes, and limits a match to the history
// (source end <= current position) and to the 512-byte lookahead.  The scan
// here visits the same candidates in the same order -- only positions whose
// next three bytes agree with the lookahead, since shorter matches are
// discarded -- so it returns the same (offset, length).
void lzss_encode_column(const uint8_t* d, uint32_t L, std::vector<uint8_t>& out) {
    const uint32_t HIST = 2048, LOOK = 512, MAXM = 34, MINM = 3;
    // forward chains over equal 3-byte keys, built back to front
    std::vector<int32_t> nxt(L, -1);
    std::vector<uint32_t> key_of(L, 0);
    // open-addressed table: key -> first position (front of chain) and cursor
    uint32_t tsize = 1;
    while (tsize < 2 * L + 2) tsize <<= 1;
    std::vector<int64_t> tkey(tsize, -1);
    std::vector<int32_t> tfirst(tsize, -1), tcur(tsize, -1);
    auto slot = [&](uint32_t key) {
        uint32_t h = (key * 2654435761u) & (tsize - 1);
        while (tkey[h] != -1 && tkey[h] != (int64_t)key) h = (h + 1) & (tsize - 1);
        return h;
    };
    for (int64_t p = (int64_t)L - 3; p >= 0; --p) {
        uint32_t key = ((uint32_t)d[p] << 16) | ((uint32_t)d[p + 1] << 8) | d[p + 2];
        key_of[p] = key;
        uint32_t h = slot(key);
        if (tkey[h] == -1) tkey[h] = key;
        nxt[p] = tfirst[h];
        tfirst[h] = (int32_t)p;
    }
    for (uint32_t h = 0; h < tsize; ++h) tcur[h] = tfirst[h];

    out.clear();
    out.push_back(0);  // first flag byte
    uint64_t flag_pos = 0;
    uint8_t flags = 0;
    int blocks = 0;
    uint32_t cur = 0;
    while (cur < L) {
        uint32_t hist_count = std::min(cur, HIST);
        uint32_t look = std::min(LOOK, L - cur);
        uint32_t best_len = 0, best_pos = 0;
        if (look >= MINM && cur >= 3 && cur + 2 < L) {
            uint32_t lo = cur - hist_count + 1;  // oldest candidate (hist_offset 1)
            uint32_t h = slot(key_of[cur]);
            int32_t p = tcur[h];
            while (p != -1 && (uint32_t)p < lo) p = nxt[p];
            tcur[h] = p;  // lo never decreases
            for (; p != -1 && (uint32_t)p + MINM <= cur; p = nxt[p]) {
                uint32_t lim = std::min(std::min(MAXM, look), cur - (uint32_t)p);
                uint32_t f = 3;
                while (f < lim && d[p + f] == d[cur + f]) ++f;
                if (f > best_len) {
                    best_len = f;
                    best_pos = (uint32_t)p;
                }
                if (f >= MAXM) break;
            }
        }
        if (best_len < MINM) {
            out.push_back(d[cur]);
            flags |= (uint8_t)(1u << blocks);
            cur += 1;
        } else {
            uint32_t off = cur - best_pos;
            uint32_t v = (off << 5) | (best_len - MINM);
            out.push_back((uint8_t)(v & 0xff));
            out.push_back((uint8_t)(v >> 8));
            cur += best_len;
        }
        if (++blocks == 8) {
            out[flag_pos] = flags;
            flags = 0;
            blocks = 0;
            flag_pos = out.size();
            out.push_back(0);  // reserved flag byte (kept even if no token follows)
        }
    }
    if (blocks != 0) out[flag_pos] = flags;
}


// Byte-RLE flag-byte column stream (restated from brle_trans::compress_func,
// include/brle/brle_trans.h:437-562): maximal runs of equal bytes; a run of
// 3 or more becomes a run item (count byte, value byte; flag bit 0), a
// shorter run becomes that many literal items (one byte each; flag bit 1).
// A flag byte precedes every 8 items, bits LSB first; after the 8th item of a
// group the next flag byte is reserved even if no item follows (it stays 0).
void brle_trans_encode_column(const uint8_t* d, uint32_t L, std::vector<uint8_t>& out) {
    out.assign(1, 0);
    size_t hpos = 0;
    uint32_t items = 0;
    uint8_t flags = 0;
    auto item_done = [&]() {
        out[hpos] = flags;
        if (++items == 8) {
            flags = 0;
            items = 0;
            hpos = out.size();
            out.push_back(0);
        }
    };
    uint32_t i = 0;
    while (i < L) {
        uint32_t j = i + 1;
        while (j < L && d[j] == d[i]) ++j;
        const uint32_t run = j - i;
        if (run >= 3) {
            out.push_back((uint8_t)run);
            out.push_back(d[i]);
            item_done();
        } else {
            for (uint32_t k = 0; k < run; ++k) {
                flags |= (uint8_t)(1u << items);
                out.push_back(d[i]);
                item_done();
            }
        }
        i = j;
    }
}

// Columns of a chunk (column q = bytes 4q + 128k .. +3), encoded by `enc`,
// ranked by descending length (ties by descending column), interleaved over
// the active ranks in 4-byte words; blocks 128-byte aligned.  Shared by the
// LZSS and byte-RLE flag containers.  chunk_size is a multiple of 128; a
// short final chunk is zero padded.
template <class Enc>
uint64_t ranked_container(const uint8_t* in, uint64_t n, uint64_t chunk_size, uint8_t* data, uint64_t* blk_off,
                          uint64_t* col_len, uint8_t* col_map, Enc enc) {
    if (n == 0 || chunk_size == 0 || chunk_size % 128) return 0;
    uint64_t nc = (n - 1) / chunk_size + 1;
    std::vector<std::vector<uint8_t>> cols(nc * 32);
    parallel_for(nc, [&](uint64_t c) {
        uint64_t len = std::min(chunk_size, n - c * chunk_size);
        std::vector<uint8_t> chunk(chunk_size, 0);
        memcpy(chunk.data(), in + c * chunk_size, len);
        uint32_t L = (uint32_t)(chunk_size / 32);
        std::vector<uint8_t> col(L);
        for (int q = 0; q < 32; ++q) {
            for (uint32_t k = 0; k < L / 4; ++k) memcpy(&col[4 * k], &chunk[128ull * k + 4 * q], 4);
            enc(col.data(), L, cols[c * 32 + q]);
        }
    });
    blk_off[0] = 0;
    for (uint64_t c = 0; c < nc; ++c) {
        int order[32];
        for (int q = 0; q < 32; ++q) order[q] = q;
        std::stable_sort(order, order + 32, [&](int a, int b) {
            return cols[c * 32 + a].size() < cols[c * 32 + b].size();
        });
        uint64_t len[32];
        for (int r = 0; r < 32; ++r) {
            int q = order[31 - r];
            col_map[c * 32 + r] = (uint8_t)q;
            len[r] = col_len[c * 32 + r] = cols[c * 32 + q].size();
        }
        blk_off[c + 1] = blk_off[c] + block_bytes(len);
    }
    parallel_for(nc, [&](uint64_t c) {
        uint64_t len[32];
        const std::vector<uint8_t>* sl[32];
        for (int r = 0; r < 32; ++r) {
            len[r] = col_len[c * 32 + r];
            sl[r] = &cols[c * 32 + col_map[c * 32 + r]];
        }
        memset(data + blk_off[c], 0, blk_off[c + 1] - blk_off[c]);
        interleave(sl, len, data + blk_off[c]);
    });
    return blk_off[nc];
}

}  // namespace

extern "C" {

// ---------------------------------------------------------------------------
// Byte-RLE container: [u32 n_ptr][u64 ptr[n_ptr]][u64 total][data]
// (brle::compress_gpu, include/brle/brle.h:251-303).  Returns the number of
// bytes written to `out` (caller sizes it with gd_brle_max_encoded_bytes), or 0.
// ---------------------------------------------------------------------------
uint64_t gd_brle_max_encoded_bytes(uint64_t n, uint64_t chunk_size) {
    uint64_t nc = n ? (n - 1) / chunk_size + 1 : 0;
    return 4 + 8 * (nc + 1) + 8 + n + (n / 128 + 1) * 2 + nc * 2 + 64;
}

uint64_t gd_brle_encode(const uint8_t* in, uint64_t n, uint64_t chunk_size, uint8_t* out) {
    if (n == 0 || chunk_size == 0) return 0;
    uint64_t nc = (n - 1) / chunk_size + 1;
    std::vector<std::vector<uint8_t>> parts(nc);
    parallel_for(nc, [&](uint64_t c) {
        uint64_t len = std::min(chunk_size, n - c * chunk_size);
        parts[c].reserve(len / 4);
        brle_encode_chunk(in + c * chunk_size, len, parts[c]);
    });
    uint32_t n_ptr = (uint32_t)(nc + 1);
    memcpy(out, &n_ptr, 4);
    uint64_t hdr = 4 + 8 * (nc + 1) + 8, acc = 0;
    for (uint64_t c = 0; c <= nc; ++c) {
        memcpy(out + 4 + 8 * c, &acc, 8);
        if (c < nc) acc += parts[c].size();
    }
    memcpy(out + 4 + 8 * (nc + 1), &n, 8);
    uint64_t o = hdr;
    for (uint64_t c = 0; c < nc; ++c) {
        memcpy(out + o, parts[c].data(), parts[c].size());
        o += parts[c].size();
    }
    return o;
}

// ---------------------------------------------------------------------------
// RLE v1 container (rle_v1::compress_gpu, include/rle_v1/rlev1.h:25-97).
// Input is padded with zeros to whole chunks (rlev1.h:38-44).  Writes
// blk_off[n_chunks+1], col_len[32*n_chunks]; returns data bytes written to
// `data` (sized by gd_rlev1_max_encoded_bytes), 0 on bad arguments.
// ---------------------------------------------------------------------------
uint64_t gd_rlev1_max_encoded_bytes(uint64_t n, uint64_t chunk_size) {
    uint64_t nc = n ? (n - 1) / chunk_size + 1 : 0;
    // worst case: 1 header byte per 127 literals + 10-byte varints
    return nc * (chunk_size / 4 * 11 + 32 * 64 + 256);
}

uint64_t gd_rlev1_encode(const uint8_t* in, uint64_t n, uint64_t chunk_size, uint32_t comp_col_len,
                         uint32_t elem_bytes, uint8_t* data, uint64_t* blk_off, uint64_t* col_len) {
    if (n == 0 || chunk_size == 0 || !(elem_bytes == 4 || elem_bytes == 8)) return 0;
    if (comp_col_len == 0 || comp_col_len % elem_bytes || chunk_size % (32ull * comp_col_len)) return 0;
    uint64_t nc = (n - 1) / chunk_size + 1;
    uint64_t ne = chunk_size / 32 / elem_bytes;  // values per lane
    uint32_t wil = comp_col_len / elem_bytes;
    std::vector<std::vector<uint8_t>> lanes(nc * 32);
    parallel_for(nc, [&](uint64_t c) {
        std::vector<uint8_t> chunk(chunk_size, 0);
        uint64_t len = std::min(chunk_size, n - c * chunk_size);
        memcpy(chunk.data(), in + c * chunk_size, len);
        for (int t = 0; t < 32; ++t) {
            if (elem_bytes == 4) {
                std::vector<uint32_t> v(ne);
                const uint32_t* src = (const uint32_t*)chunk.data();
                for (uint64_t e = 0; e < ne; ++e) v[e] = src[(e / wil) * 32 * wil + (uint64_t)t * wil + e % wil];
                rlev1_encode_lane<uint32_t>(v.data(), ne, lanes[c * 32 + t]);
            } else {
                std::vector<uint64_t> v(ne);
                const uint64_t* src = (const uint64_t*)chunk.data();
                for (uint64_t e = 0; e < ne; ++e) v[e] = src[(e / wil) * 32 * wil + (uint64_t)t * wil + e % wil];
                rlev1_encode_lane<uint64_t>(v.data(), ne, lanes[c * 32 + t]);
            }
        }
    });
    blk_off[0] = 0;
    for (uint64_t c = 0; c < nc; ++c) {
        uint64_t len[32];
        for (int t = 0; t < 32; ++t) len[t] = col_len[c * 32 + t] = lanes[c * 32 + t].size();
        blk_off[c + 1] = blk_off[c] + block_bytes(len);
    }
    parallel_for(nc, [&](uint64_t c) {
        uint64_t len[32];
        const std::vector<uint8_t>* sl[32];
        for (int t = 0; t < 32; ++t) {
            len[t] = col_len[c * 32 + t];
            sl[t] = &lanes[c * 32 + t];
        }
        memset(data + blk_off[c], 0, blk_off[c + 1] - blk_off[c]);
        interleave(sl, len, data + blk_off[c]);
    });
    return blk_off[nc];
}

// ---------------------------------------------------------------------------
// RLE v2 transposed container (rlev2::compress_gpu_transpose,
// include/rlev2/encoder_trans.h:428-537).  8-byte values.  Input padded with
// zeros to whole chunks.  blk_off[n_chunks] holds the data byte count here;
// the reference overwrites it with the input size (encoder_trans.h:490-492),
// which the caller can do when writing that container.
// ---------------------------------------------------------------------------
uint64_t gd_rlev2_max_encoded_bytes(uint64_t n, uint64_t chunk_size) {
    uint64_t nc = n ? (n - 1) / chunk_size + 1 : 0;
    return nc * (chunk_size + chunk_size / 8 + 32 * 128 + 256);
}

uint64_t gd_rlev2_encode(const uint8_t* in, uint64_t n, uint64_t chunk_size, uint32_t read_unit, uint8_t* data,
                         uint64_t* blk_off, uint64_t* col_len) {
    if (n == 0 || chunk_size == 0 || read_unit == 0 || chunk_size % (256ull * read_unit)) return 0;
    uint64_t nc = (n - 1) / chunk_size + 1;
    uint64_t nv = chunk_size / 8 / 32;
    std::vector<std::vector<uint8_t>> lanes(nc * 32);
    parallel_for(nc, [&](uint64_t c) {
        std::vector<int64_t> chunk(chunk_size / 8, 0);
        uint64_t len = std::min(chunk_size, n - c * chunk_size);
        memcpy(chunk.data(), in + c * chunk_size, len);
        std::vector<int64_t> v(nv);
        for (int t = 0; t < 32; ++t) {
            for (uint64_t i = 0; i < nv; ++i)
                v[i] = chunk[(uint64_t)t * read_unit + (i / read_unit) * 32 * read_unit + i % read_unit];
            lanes[c * 32 + t].reserve(nv * 4);
            rlev2_encode_lane(v.data(), nv, lanes[c * 32 + t]);
        }
    });
    blk_off[0] = 0;
    for (uint64_t c = 0; c < nc; ++c) {
        uint64_t len[32];
        for (int t = 0; t < 32; ++t) len[t] = col_len[c * 32 + t] = lanes[c * 32 + t].size();
        blk_off[c + 1] = blk_off[c] + block_bytes(len);
    }
    parallel_for(nc, [&](uint64_t c) {
        uint64_t len[32];
        const std::vector<uint8_t>* sl[32];
        for (int t = 0; t < 32; ++t) {
            len[t] = col_len[c * 32 + t];
            sl[t] = &lanes[c * 32 + t];
        }
        memset(data + blk_off[c], 0, blk_off[c + 1] - blk_off[c]);
        interleave(sl, len, data + blk_off[c]);
    });
    return blk_off[nc];
}

// Encode one RLE v2 lane stream (exposed for pinning against the reference's
// contiguous block_encode).
uint64_t gd_rlev2_encode_stream(const int64_t* vals, uint64_t n, uint8_t* out, uint64_t cap) {
    std::vector<uint8_t> o;
    rlev2_encode_lane(vals, n, o);
    if (o.size() > cap) return 0;
    memcpy(out, o.data(), o.size());
    return o.size();
}

// Encode one RLE v1 lane stream of 4- or 8-byte values.
uint64_t gd_rlev1_encode_stream(const void* vals, uint64_t n, uint32_t elem_bytes, uint8_t* out, uint64_t cap) {
    std::vector<uint8_t> o;
    if (n < 2) return 0;
    if (elem_bytes == 4) rlev1_encode_lane<uint32_t>((const uint32_t*)vals, n, o);
    else if (elem_bytes == 8) rlev1_encode_lane<uint64_t>((const uint64_t*)vals, n, o);
    else return 0;
    if (o.size() > cap) return 0;
    memcpy(out, o.data(), o.size());
    return o.size();
}

// Encode one LZSS column stream (exposed for pinning against the
// reference's contiguous compress_func).
uint64_t gd_lzss_encode_stream(const uint8_t* in, uint32_t n, uint8_t* out, uint64_t cap) {
    std::vector<uint8_t> o;
    lzss_encode_column(in, n, o);
    if (o.size() > cap) return 0;
    memcpy(out, o.data(), o.size());
    return o.size();
}

// ---------------------------------------------------------------------------
// LZSS interleaved container (lzss::compress_gpu, lzss_gpu2.h:1915-2127).
// chunk_size must be a multiple of 128; a short final chunk is zero padded
// to a whole chunk (the reference drops it, lzss_gpu2.h:1959), so every
// column of every chunk holds chunk_size/32 bytes.
// Column q of a chunk is bytes 4q+128k..+3.  Lanes are ranked by descending
// stream length, ties by descending column (the reversed stable ascending
// radix sort, lzss_gpu2.h:1063-1086).  Writes blk_off[n+1], col_len[32n]
// (sorted), col_map[32n] (rank -> column).
// ---------------------------------------------------------------------------
uint64_t gd_lzss_max_encoded_bytes(uint64_t n, uint64_t chunk_size) {
    uint64_t nc = n ? (n - 1) / chunk_size + 1 : 0;
    return nc * (chunk_size + chunk_size / 8 + 32 * 8 + 256);
}

uint64_t gd_lzss_encode(const uint8_t* in, uint64_t n, uint64_t chunk_size, uint8_t* data, uint64_t* blk_off,
                        uint64_t* col_len, uint8_t* col_map) {
    return ranked_container(in, n, chunk_size, data, blk_off, col_len, col_map, lzss_encode_column);
}

// ---------------------------------------------------------------------------
// Deflate container: each chunk a zlib (or raw deflate) stream, zero padded
// to 8 bytes and concatenated (orig_compressor.py:44-126).  Chunk c covers
// input bytes [out_off[c], out_off[c+1]).  mode[c]: 0 default strategy at
// `level`, 1 fixed Huffman (Z_FIXED), 2 stored (level 0).  Writes
// comp_off[n+1] (8-byte aligned) and comp_len[n] (padded length).  Returns
// total bytes, or 0 on failure.
// ---------------------------------------------------------------------------
uint64_t gd_deflate_max_encoded_bytes(const uint64_t* out_off, uint32_t n) {
    uint64_t s = 0;
    for (uint32_t c = 0; c < n; ++c) s += compressBound((uLong)(out_off[c + 1] - out_off[c])) + 64;
    return s;
}

uint64_t gd_deflate_encode(const uint8_t* in, const uint64_t* out_off, uint32_t n, int level, const uint8_t* mode,
                           int zlib_header, uint8_t* data, uint64_t* comp_off, uint64_t* comp_len) {
    std::vector<std::vector<uint8_t>> parts(n);
    std::atomic<int> fail{0};
    parallel_for(n, [&](uint64_t c) {
        uint64_t len = out_off[c + 1] - out_off[c];
        z_stream zs;
        memset(&zs, 0, sizeof(zs));
        int m = mode ? mode[c] : 0;
        int lv = (m == 2) ? 0 : level;
        int strat = (m == 1) ? Z_FIXED : Z_DEFAULT_STRATEGY;
        if (deflateInit2(&zs, lv, Z_DEFLATED, zlib_header ? 15 : -15, 8, strat) != Z_OK) {
            fail = 1;
            return;
        }
        parts[c].resize(deflateBound(&zs, (uLong)len) + 16);
        zs.next_in = (Bytef*)(in + out_off[c]);
        zs.avail_in = (uInt)len;
        zs.next_out = parts[c].data();
        zs.avail_out = (uInt)parts[c].size();
        if (deflate(&zs, Z_FINISH) != Z_STREAM_END) fail = 1;
        parts[c].resize(zs.total_out);
        deflateEnd(&zs);
    });
    if (fail) return 0;
    uint64_t o = 0;
    for (uint32_t c = 0; c < n; ++c) {
        comp_off[c] = o;
        uint64_t pl = (parts[c].size() + 7) / 8 * 8;
        comp_len[c] = pl;
        memcpy(data + o, parts[c].data(), parts[c].size());
        memset(data + o + parts[c].size(), 0, pl - parts[c].size());
        o += pl;
    }
    comp_off[n] = o;
    return o;
}


// ---------------------------------------------------------------------------
// Byte-RLE flag-byte interleaved container (brle_trans::compress_gpu,
// include/brle/brle_trans.h:563-660): the column streams of
// brle_trans_encode_column in the ranked 32-column layout.  The reference
// fixes the chunk at 4 KiB; any multiple of 128 is accepted here.  Writes
// blk_off[n+1], col_len[32n] (sorted), col_map[32n] (rank -> column).
// ---------------------------------------------------------------------------
uint64_t gd_brle_trans_max_encoded_bytes(uint64_t n, uint64_t chunk_size) {
    uint64_t nc = n ? (n - 1) / chunk_size + 1 : 0;
    return nc * (chunk_size + chunk_size / 8 + 32 * 8 + 256);
}

uint64_t gd_brle_trans_encode(const uint8_t* in, uint64_t n, uint64_t chunk_size, uint8_t* data, uint64_t* blk_off,
                              uint64_t* col_len, uint8_t* col_map) {
    return ranked_container(in, n, chunk_size, data, blk_off, col_len, col_map, brle_trans_encode_column);
}

// ---------------------------------------------------------------------------
// LZSS contiguous container (lzss::compress_gpu, include/lzss/lzss.h:1060-1124):
//   [u64 in_n_bytes][u32 chunk_size][u32 n_chunks][u32 2048][u32 3][u32 34]
//   [u64 end offset of every chunk's stream in the data][data]
// chunk c = input bytes [c*chunk_size, ..) (the last may be short) tokenised
// by the same find_match grammar as one LZSS column.
// ---------------------------------------------------------------------------
uint64_t gd_lzss_contig_max_encoded_bytes(uint64_t n, uint64_t chunk_size) {
    uint64_t nc = n ? (n - 1) / chunk_size + 1 : 0;
    return 28 + 8 * nc + nc * (chunk_size + chunk_size / 8 + 16);
}

uint64_t gd_lzss_contig_encode(const uint8_t* in, uint64_t n, uint64_t chunk_size, uint8_t* out) {
    if (n == 0 || chunk_size == 0 || chunk_size > 0xffffffffull) return 0;
    const uint64_t nc = (n - 1) / chunk_size + 1;
    if (nc > 0xffffffffull) return 0;
    std::vector<std::vector<uint8_t>> parts(nc);
    parallel_for(nc, [&](uint64_t c) {
        const uint64_t len = std::min(chunk_size, n - c * chunk_size);
        lzss_encode_column(in + c * chunk_size, (uint32_t)len, parts[c]);
    });
    const uint32_t head[5] = {(uint32_t)chunk_size, (uint32_t)nc, 2048u, 3u, 34u};
    memcpy(out, &n, 8);
    memcpy(out + 8, head, 20);
    uint64_t* lens = reinterpret_cast<uint64_t*>(out + 28);
    uint8_t* data = out + 28 + 8 * nc;
    uint64_t pos = 0;
    for (uint64_t c = 0; c < nc; ++c) {
        memcpy(data + pos, parts[c].data(), parts[c].size());
        pos += parts[c].size();
        memcpy(&lens[c], &pos, 8);  // the header is 28 bytes: lens are not 8-byte aligned
    }
    return 28 + 8 * nc + pos;
}

}  // extern "C"
