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
#include "../lane_enc.h"

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
// RLE v1 and RLE v2 lane streams: the encoders live in lane_enc.h, shared
// with the device encoders (encode.cu); here they write into a vector.
// ---------------------------------------------------------------------------

struct VecSink {
    std::vector<uint8_t>& v;
    void put(uint8_t b) { v.push_back(b); }
    uint64_t size() const { return v.size(); }
    void set(uint64_t i, uint8_t b) { v[i] = b; }
};

template <typename T>
void rlev1_encode_lane(const T* vals, uint64_t n, std::vector<uint8_t>& o) {
    VecSink s{o};
    gd::enc::rlev1_encode_lane<T>(vals, n, s);
}

void rlev2_encode_lane(const int64_t* vals, uint64_t n, std::vector<uint8_t>& o) {
    VecSink s{o};
    gd::enc::rlev2_encode_lane(vals, n, s);
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
// group the next flag byte is reserved even if no item follows (it stays 0) --
// except after the column's last item when that is a run: the reference
// writes that run without counting it (compress_func, brle_trans.h:529-536;
// compress_init_func sizes it the same way, :354-357), so no flag byte is
// reserved after it even when it fills slot 8.
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
            if (j < L) item_done();  // the column's last run is not counted
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

// The 4-byte-symbol variant of the flag-byte column (restated from
// brle::compress_func, include/brle/brle_gpu_4B.h:321-638): the column's
// 4-byte words are its symbols; a maximal run of 3 or more equal symbols is
// a run item (count byte, symbol; flag bit 0), a shorter one that many
// literal items (the symbol; flag bit 1).  A flag byte precedes every 8
// items and after the 8th item of a group the next one is reserved -- except
// after the column's last item when that is a run, which the reference
// writes without counting it (brle_gpu_4B.h:604-616).  A reserved flag byte
// that no item follows is 0 here; the reference leaves it unwritten.
void brle_trans4_encode_column(const uint8_t* d, uint32_t L, std::vector<uint8_t>& out) {
    out.assign(1, 0);
    size_t hpos = 0;
    uint32_t items = 0;
    uint8_t flags = 0;
    auto put_sym = [&](uint32_t k) { out.insert(out.end(), d + 4 * k, d + 4 * k + 4); };
    auto item_done = [&]() {
        if (++items == 8) {
            out[hpos] = flags;
            flags = 0;
            items = 0;
            hpos = out.size();
            out.push_back(0);
        }
        if (items != 0) out[hpos] = flags;
    };
    const uint32_t ns = L / 4;
    uint32_t i = 0;
    while (i < ns) {
        uint32_t j = i + 1;
        while (j < ns && memcmp(d + 4 * j, d + 4 * i, 4) == 0) ++j;
        const uint32_t run = j - i;
        const bool last = j == ns;
        if (run >= 3) {
            out.push_back((uint8_t)run);
            put_sym(i);
            if (!last) item_done();
        } else {
            for (uint32_t k = 0; k < run; ++k) {
                flags |= (uint8_t)(1u << items);
                put_sym(i);
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

// The 4-byte-symbol flag container (brle::compress_gpu,
// include/brle/brle_gpu_4B.h:640-715): brle_trans4_encode_column in the same
// ranked 32-column layout.  The reference fixes the chunk at 8 KiB and drops
// a partial last chunk; here any multiple of 128 up to 8 KiB is accepted and
// the last chunk is zero padded.
uint64_t gd_brle_trans4_max_encoded_bytes(uint64_t n, uint64_t chunk_size) {
    uint64_t nc = n ? (n - 1) / chunk_size + 1 : 0;
    return nc * (chunk_size + chunk_size / 16 + 32 * 8 + 256);
}

uint64_t gd_brle_trans4_encode(const uint8_t* in, uint64_t n, uint64_t chunk_size, uint8_t* data, uint64_t* blk_off,
                               uint64_t* col_len, uint8_t* col_map) {
    if (chunk_size > 8192) return 0;
    return ranked_container(in, n, chunk_size, data, blk_off, col_len, col_map, brle_trans4_encode_column);
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
