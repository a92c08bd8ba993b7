// lane_enc.h -- RLE v1 and RLE v2 lane-stream encoders, compiled for both
// the host (gd_encode.cpp, g++) and the device (encode.cu, nvcc).
//
// A lane stream is the byte stream of one of the 32 lanes of a chunk; the
// container interleaves the 32 streams afterwards.  The encoders are state
// machines over the lane's values in order, written against two small
// concepts so that one source serves both sides:
//   Vals: operator[](uint64_t i) -> the lane's i-th value (read in order);
//   Sink: put(byte), size(), set(index, byte) (a retroactive header write).
// Restated from the reference's writers: RLE v1 compression_warp
// (include/rle_v1/encoder.h:607-1018, write_byte_op's interleave factored
// out) and RLE v2 block_encode / determineEncoding and its writers
// (include/rlev2/encoder.h:109-969, HEAD-side semantics).
#pragma once
#include <cstdint>

#ifdef __CUDACC__
#define GD_HD __host__ __device__ __forceinline__
#else
#define GD_HD inline
#endif

namespace gd {
namespace enc {

template <typename T>
GD_HD T min_(T a, T b) { return a < b ? a : b; }
template <typename T>
GD_HD T max_(T a, T b) { return a > b ? a : b; }

// ---------------------------------------------------------------------------
// RLE v1
// ---------------------------------------------------------------------------

// unsigned LEB128 of a value of the lane's element type (decoder.h:301-350)
template <typename T, class Sink>
GD_HD void put_varint(Sink& o, T v) {
    do {
        uint8_t b = (uint8_t)(v & 0x7f);
        if ((v & ~(T)0x7f) != 0) b |= 0x80;
        o.put(b);
        v = v >> 7;
    } while (v != 0);
}

// compression_warp, include/rle_v1/encoder.h:607-1018: lane `vals` (n >= 2
// values of type T) as an RLE v1 byte stream.
template <typename T, class Vals, class Sink>
GD_HD void rlev1_encode_lane(const Vals& vals, uint64_t n, Sink& o) {
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
        o.put(1);
    };
    auto write_run = [&](int hdr) {
        o.put((uint8_t)(int8_t)hdr);
        o.put((uint8_t)cur_delta);
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
            o.set(lit_idx, (uint8_t)(int8_t)(-(int)lcount));
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
                    o.set(lit_idx, (uint8_t)(int8_t)(-(int)lcount));
                    lcount = 0;
                }
            } else if (dcount == 130) {
                write_run(dcount - 4);
                dcount = 1;
                count = 0;
                lcount = 0;
            }
            push(rd);
            count = min_<uint8_t>(count + 1, 2);
            prev = rd;
        } else {
            if (dcount >= 3) {  // :872-903
                write_run(dcount - 3);
                dcount = 1;
                count = 0;
                lcount = 0;
                push(rd);
                count = min_<uint8_t>(count + 1, 2);
                prev = rd;
            } else {  // :905-969
                if (lcount == 0) {
                    lit_idx = o.size();
                    o.put(3);
                }
                lcount++;
                put_varint<T>(o, buf[head]);
                if (lcount == 127) {
                    o.set(lit_idx, (uint8_t)(int8_t)(-(int)lcount));
                    lcount = 0;
                }
                td = diff(rd, prev);
                if (td > 127 || td < -128) {
                    if (lcount == 0) {
                        lit_idx = o.size();
                        o.put(3);
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
                count = min_<uint8_t>(count + 1, 2);
            }
        }
    }
    // tail (:975-1052)
    if (dcount >= 3 && dflag) {
        write_run(dcount - 3);
    } else {
        if (count == 1) {
            if (lcount == 127) {
                o.set(lit_idx, (uint8_t)(int8_t)(-(int)lcount));
                lcount = 0;
            }
            if (lcount == 0) start_lit();
            uint8_t tail = (head == 0) ? 1 : 0;
            put_varint<T>(o, buf[tail]);
            lcount++;
        }
        if (count == 2) {
            if (lcount == 127) {
                o.set(lit_idx, (uint8_t)(int8_t)(-(int)lcount));
                lcount = 0;
            }
            if (lcount == 0) start_lit();
            put_varint<T>(o, buf[head]);
            lcount++;
            if (lcount == 127) {
                o.set(lit_idx, (uint8_t)(int8_t)(-(int)lcount));
                lcount = 0;
            }
            if (lcount == 0) start_lit();
            head = (head + 1) % 2;
            put_varint<T>(o, buf[head]);
            lcount++;
        }
        o.set(lit_idx, (uint8_t)(int8_t)(-(int)lcount));
    }
}

// ---------------------------------------------------------------------------
// RLE v2 (HEAD-side semantics of include/rlev2/encoder.h)
// ---------------------------------------------------------------------------

// __BIT_WIDTH_DECODE_MAP (utils.h:38-39) as arithmetic
GD_HD uint8_t w_decode(uint32_t c) {
    return (uint8_t)(c < 24u ? c + 1u : (c < 28u ? 26u + 2u * (c - 24u) : 40u + 8u * (c - 28u)));
}
// utils.h:40-51
GD_HD uint8_t w_encode(uint32_t w) {
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
GD_HD uint8_t w_closest(uint32_t b) {
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
GD_HD uint8_t w_closest_aligned(uint32_t b) {
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

// the writer's literal buffer (runs are at most 128 values, utils.h:78)
template <class Sink>
struct V2Info {
    int64_t deltas[128];
    int64_t literals[128];
    uint32_t num_literals, fix_runlen, var_runlen;
    uint8_t delta_bits;
    bool is_fixed_delta;
    Sink* out;
    GD_HD void w(uint8_t b) { out->put(b); }
};

// encoder.h:109-122
GD_HD uint8_t closest_num_bits(int64_t v) {
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
template <class Info>
GD_HD void write_aligned(const int64_t* in, uint32_t len, uint8_t bits, Info& info) {
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
template <class Info>
GD_HD void write_unaligned(const int64_t* in, uint32_t len, uint8_t bits, Info& info) {
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
GD_HD void bit_hist(const int64_t* d, uint32_t n, uint8_t* hist) {
    for (int i = 0; i < 32; ++i) hist[i] = 0;
    for (uint32_t i = 0; i < n; ++i) hist[w_encode(closest_num_bits(d[i]))]++;
}
// encoder.h:231-242
GD_HD uint8_t percentile_bits(const uint8_t* hist, uint32_t len, int p) {
    p = min_(100 - p, 100);
    int32_t plen = (p == 0 ? 0 : (int32_t)((len * p - 1) / 100 + 1));
    for (int i = 31; i >= 0; --i) {
        plen -= hist[i];
        if (plen < 0) return w_decode((uint32_t)i);
    }
    return 0;
}

// encoder.h:538-569
template <class Info>
GD_HD void write_short_repeat(Info& info) {
    int64_t val = info.literals[0];
    uint8_t vb = closest_num_bits(val);
    uint8_t nbytes = (uint8_t)((vb - 1) / 8 + 1);
    info.w((uint8_t)(((nbytes - 1) << 3) | (info.fix_runlen - 3)));
    for (int i = nbytes - 1; i >= 0; --i) info.w((uint8_t)(((uint64_t)val >> (i * 8)) & 0xff));
    info.fix_runlen = 0;
    info.num_literals = 0;
}

// encoder.h:580-598
template <class Info>
GD_HD void write_direct(Info& info) {
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
template <class Info>
GD_HD void write_vulong(int64_t v, Info& info) {
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
template <class Info>
GD_HD void write_vslong(int64_t v, Info& info) {
    write_vulong((int64_t)(((uint64_t)v << 1) ^ (uint64_t)(v >> 63)), info);
}

// encoder.h:631-697 (HEAD side)
template <class Info>
GD_HD void write_delta(Info& info) {
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
template <class Info>
GD_HD void prepare_patched(Info& info, PatchBlob& pb) {
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
template <class Info>
GD_HD void write_patched(Info& info, PatchBlob& pb) {
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
GD_HD bool safe_subtract(int64_t larger, int64_t smaller) {
    if (smaller > 0) return true;
    int64_t t = (int64_t)((uint64_t)smaller - (uint64_t)(-9223372036854775807ll - 1));
    return larger > t;
}

// encoder.h:367-535 (HEAD side)
template <class Info>
GD_HD void determine_encoding(Info& info) {
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
        lmin = min_(lmin, l1);
        lmax = max_(lmax, l1);
        inc &= (l0 <= l1);
        dec &= (l0 >= l1);
        info.is_fixed_delta &= (cd == init_delta);
        int64_t ad = cd < 0 ? (int64_t)(0 - (uint64_t)cd) : cd;
        info.deltas[i - 1] = ad;
        max_delta = max_(max_delta, ad);
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
// over one lane's n values in the order `vals` gives them (the transposed
// order of rlev2/encoder_trans.h:40-108 for a container lane).
template <class Vals, class Sink>
GD_HD void rlev2_encode_lane(const Vals& vals, uint64_t n, Sink& out) {
    V2Info<Sink> info;
    for (int i = 0; i < 128; ++i) info.deltas[i] = 0;
    info.num_literals = info.fix_runlen = info.var_runlen = 0;
    info.delta_bits = 0;
    info.is_fixed_delta = false;
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

}  // namespace enc
}  // namespace gd
