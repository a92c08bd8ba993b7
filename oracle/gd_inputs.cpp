// gd_inputs.cpp -- input builders for the CPU baselines -- TEST
// INFRASTRUCTURE ONLY (linked into liboracle.so with gd_oracle.c and the
// seeded column generators of compression_b200/csrc/host/gd_gen.cpp).
//
// bench.py's reference arm times the reference's own CPU decoders on the
// host cores and must not load the product library, so it builds its inputs
// here: the generators (the same source as the product's, so a seed gives the
// same column) and, for RLE v1 -- whose only reference encoder is the GPU
// writer compression_warp (include/rle_v1/encoder.h:607-1018), with no CPU
// counterpart -- the lane-stream state machine of lane_enc.h (pinned byte for
// byte to that writer by tests/golden/rlev1_golden.npz) plus the 32-lane
// 4-byte interleave of write_byte_op (encoder.h:564-588): word row k holds
// the k-th word of every lane longer than 4k bytes, in lane order, and a
// block is the sum of its 4-byte-padded lanes rounded up to 128 bytes
// (encoder.h:504-520).
#include <cstdint>
#include <cstring>
#include <thread>
#include <atomic>
#include <vector>

#include "../compression_b200/csrc/lane_enc.h"

namespace {

struct Sink {
    std::vector<uint8_t>& v;
    void put(uint8_t b) { v.push_back(b); }
    uint64_t size() const { return v.size(); }
    void set(uint64_t i, uint8_t b) { v[i] = b; }
};

template <typename F>
void each(uint64_t n, F&& f) {
    unsigned nt = std::thread::hardware_concurrency();
    if (nt == 0) nt = 1;
    if (nt > n) nt = (unsigned)n;
    std::atomic<uint64_t> next{0};
    std::vector<std::thread> th;
    for (unsigned t = 0; t < nt; ++t)
        th.emplace_back([&]() {
            for (uint64_t i; (i = next.fetch_add(1)) < n;) f(i);
        });
    for (auto& x : th) x.join();
}

template <typename T>
void lanes_of_chunk(const uint8_t* in, uint64_t n, uint64_t c, uint64_t chunk, uint32_t ccl,
                    std::vector<uint8_t>* lanes) {
    std::vector<uint8_t> buf(chunk, 0);
    const uint64_t len = n - c * chunk < chunk ? n - c * chunk : chunk;
    memcpy(buf.data(), in + c * chunk, len);
    const T* src = reinterpret_cast<const T*>(buf.data());
    const uint64_t ne = chunk / 32 / sizeof(T), wil = ccl / sizeof(T);
    std::vector<T> v(ne);
    for (int t = 0; t < 32; ++t) {
        // lane t owns COMP_COL_LEN-byte slices at line stride 32 * COMP_COL_LEN
        for (uint64_t e = 0; e < ne; ++e) v[e] = src[(e / wil) * 32 * wil + (uint64_t)t * wil + e % wil];
        lanes[t].clear();
        Sink s{lanes[t]};
        gd::enc::rlev1_encode_lane<T>(v.data(), ne, s);
    }
}

}  // namespace

extern "C" {

uint64_t gdo_rlev1_max_encoded_bytes(uint64_t n, uint64_t chunk) {
    const uint64_t nc = n ? (n - 1) / chunk + 1 : 0;
    return nc * (chunk + chunk / 4 + 32 * 8 + 256);
}

// The RLE v1 container of `in` (n bytes): data, blk_off[nc + 1], col_len[32 nc].
// Returns the data size, 0 for bad arguments.
uint64_t gdo_rlev1_encode(const uint8_t* in, uint64_t n, uint64_t chunk, uint32_t ccl, uint32_t elem_bytes,
                          uint8_t* data, uint64_t* blk_off, uint64_t* col_len) {
    if (n == 0 || chunk == 0 || !(elem_bytes == 4 || elem_bytes == 8)) return 0;
    if (ccl == 0 || ccl % elem_bytes || chunk % (32ull * ccl)) return 0;
    const uint64_t nc = (n - 1) / chunk + 1;
    std::vector<std::vector<uint8_t>> lanes(nc * 32);
    each(nc, [&](uint64_t c) {
        if (elem_bytes == 4) lanes_of_chunk<uint32_t>(in, n, c, chunk, ccl, &lanes[c * 32]);
        else lanes_of_chunk<uint64_t>(in, n, c, chunk, ccl, &lanes[c * 32]);
    });
    blk_off[0] = 0;
    for (uint64_t c = 0; c < nc; ++c) {
        uint64_t s = 0;
        for (int t = 0; t < 32; ++t) {
            col_len[c * 32 + t] = lanes[c * 32 + t].size();
            s += (col_len[c * 32 + t] + 3) / 4 * 4;
        }
        blk_off[c + 1] = blk_off[c] + (s + 127) / 128 * 128;
    }
    each(nc, [&](uint64_t c) {
        uint8_t* dst = data + blk_off[c];
        memset(dst, 0, blk_off[c + 1] - blk_off[c]);
        uint64_t rows = 0;
        for (int t = 0; t < 32; ++t) rows = rows > (col_len[c * 32 + t] + 3) / 4 ? rows : (col_len[c * 32 + t] + 3) / 4;
        uint64_t pos = 0;
        for (uint64_t k = 0; k < rows; ++k)
            for (int t = 0; t < 32; ++t) {
                const std::vector<uint8_t>& l = lanes[c * 32 + t];
                if (l.size() <= 4 * k) continue;
                for (int b = 0; b < 4; ++b) dst[pos + b] = 4 * k + b < l.size() ? l[4 * k + b] : 0;
                pos += 4;
            }
    });
    return blk_off[nc];
}

}  // extern "C"
