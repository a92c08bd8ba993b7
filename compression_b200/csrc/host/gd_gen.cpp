// gd_gen.cpp -- seeded synthetic column generators.
//
// The reference benchmarks read external datasets that are not available
// (mortgage and taxi columns); these generators produce stand-ins with the
// shapes, sizes and value distributions the benchmark workloads name.  All
// randomness comes from std::mt19937_64 turned into numbers by the explicit
// transforms below, so a (seed, size) pair gives the same bytes everywhere.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <random>
#include <thread>
#include <vector>

#include "../../../include/gd.h"

namespace {

struct Rng {
    std::mt19937_64 g;
    explicit Rng(uint64_t s) : g(s) {}
    uint64_t u64() { return g(); }
    double unit() { return (double)(g() >> 11) * (1.0 / 9007199254740992.0); }  // [0,1)
    // uniform integer in [lo, hi]
    int64_t range(int64_t lo, int64_t hi) { return lo + (int64_t)(g() % (uint64_t)(hi - lo + 1)); }
    // geometric on {1,2,...} with the given mean
    uint64_t geometric(double mean) {
        double p = 1.0 / mean;
        double u = 1.0 - unit();  // (0,1]
        return 1 + (uint64_t)std::floor(std::log(u) / std::log(1.0 - p));
    }
};

uint64_t mix(uint64_t seed, uint64_t k) {
    uint64_t z = seed + 0x9E3779B97F4A7C15ull * (k + 1);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

template <typename F>
void parallel_for(uint64_t n, F&& f) {
    unsigned nt = std::thread::hardware_concurrency();
    if (nt == 0) nt = 1;
    if (nt > n) nt = (unsigned)n;
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

// Markov source: order-2 contexts over a 64-symbol alphabet, each context a
// random permutation with Zipf(1.0) weights.
struct Markov {
    std::vector<uint8_t> sym;   // 4096 contexts x 64 ranked symbols
    std::vector<double> cdf;    // 64
    explicit Markov(uint64_t seed) : sym(4096 * 64), cdf(64) {
        Rng r(mix(seed, 0x4d41524b));
        double s = 0;
        for (int k = 0; k < 64; ++k) s += 1.0 / (k + 1);
        double acc = 0;
        for (int k = 0; k < 64; ++k) {
            acc += 1.0 / (k + 1) / s;
            cdf[k] = acc;
        }
        cdf[63] = 1.0;
        for (int c = 0; c < 4096; ++c) {
            uint8_t* p = &sym[c * 64];
            for (int k = 0; k < 64; ++k) p[k] = (uint8_t)k;
            for (int k = 63; k > 0; --k) std::swap(p[k], p[r.u64() % (k + 1)]);
        }
    }
    uint8_t next(Rng& r, uint8_t a, uint8_t b) const {
        double u = r.unit();
        int k = (int)(std::lower_bound(cdf.begin(), cdf.end(), u) - cdf.begin());
        if (k > 63) k = 63;
        return sym[((a & 63) * 64 + (b & 63)) * 64 + k];
    }
};

}  // namespace

extern "C" {

// RLE v1 workload: int32 column of alternating segments.  A run segment has
// length geometric(mean 12) clamped to 3..130, base uniform in [0,2^20) and
// delta uniform in [-128,127]; a literal group has 1..128 values uniform in
// [0,2^20).  Generated in independent 1 Mi-value blocks.
void gd_gen_rlev1_ints(uint64_t seed, uint64_t n, int32_t* out) {
    const uint64_t B = 1 << 20;
    uint64_t nb = (n + B - 1) / B;
    parallel_for(nb, [&](uint64_t b) {
        Rng r(mix(seed, b));
        uint64_t i = b * B, end = std::min(n, i + B);
        bool run = true;
        while (i < end) {
            if (run) {
                uint64_t L = std::min<uint64_t>(130, std::max<uint64_t>(3, r.geometric(12.0)));
                int64_t base = r.range(0, (1 << 20) - 1), d = r.range(-128, 127);
                for (uint64_t k = 0; k < L && i < end; ++k) out[i++] = (int32_t)(base + (int64_t)k * d);
            } else {
                uint64_t L = (uint64_t)r.range(1, 128);
                for (uint64_t k = 0; k < L && i < end; ++k) out[i++] = (int32_t)r.range(0, (1 << 20) - 1);
            }
            run = !run;
        }
    });
}

// Byte-RLE workload: runs with length geometric(mean 20) of a byte drawn
// from 16 distinct values with Zipf(s=1.2) frequencies.
void gd_gen_brle_bytes(uint64_t seed, uint64_t n, uint8_t* out) {
    uint8_t vals[16];
    {
        Rng r(mix(seed, 0xB11E));
        uint8_t perm[256];
        for (int k = 0; k < 256; ++k) perm[k] = (uint8_t)k;
        for (int k = 255; k > 0; --k) std::swap(perm[k], perm[r.u64() % (k + 1)]);
        memcpy(vals, perm, 16);
    }
    double cdf[16], s = 0, acc = 0;
    for (int k = 0; k < 16; ++k) s += std::pow(k + 1.0, -1.2);
    for (int k = 0; k < 16; ++k) {
        acc += std::pow(k + 1.0, -1.2) / s;
        cdf[k] = acc;
    }
    cdf[15] = 1.0;
    const uint64_t B = 1 << 22;
    uint64_t nb = (n + B - 1) / B;
    parallel_for(nb, [&](uint64_t b) {
        Rng r(mix(seed, b));
        uint64_t i = b * B, end = std::min(n, i + B);
        while (i < end) {
            uint64_t L = r.geometric(20.0);
            double u = r.unit();
            int k = 0;
            while (k < 15 && cdf[k] < u) ++k;
            uint64_t m = std::min(L, end - i);
            memset(out + i, vals[k], m);
            i += m;
        }
    });
}

// RLE v2 workload: int64 column; each 512-value segment is one of
// DELTA (sorted timestamps, deltas uniform in [1,1000]), SHORT_REPEAT
// (constant runs of 3..10), DIRECT (uniform 17-bit) or PATCHED_BASE
// (uniform 12-bit with 2% outliers uniform below 2^40).
void gd_gen_rlev2_ints(uint64_t seed, uint64_t n, int64_t* out) {
    const uint64_t S = 512;
    uint64_t ns = (n + S - 1) / S;
    const uint64_t G = 1024;  // segments per independent block
    uint64_t nb = (ns + G - 1) / G;
    parallel_for(nb, [&](uint64_t b) {
        Rng r(mix(seed, b));
        int64_t ts = 1600000000000ll + (int64_t)b * 1000000000ll;
        for (uint64_t sg = b * G; sg < std::min(ns, (b + 1) * G); ++sg) {
            uint64_t i = sg * S, end = std::min(n, i + S);
            int kind = (int)(r.u64() % 4);
            while (i < end) {
                if (kind == 0) {
                    ts += r.range(1, 1000);
                    out[i++] = ts;
                } else if (kind == 1) {
                    uint64_t L = (uint64_t)r.range(3, 10);
                    int64_t v = r.range(0, (1 << 20) - 1);
                    for (uint64_t k = 0; k < L && i < end; ++k) out[i++] = v;
                } else if (kind == 2) {
                    out[i++] = r.range(0, (1 << 17) - 1);
                } else {
                    out[i++] = (r.unit() < 0.02) ? r.range(0, (1ll << 40) - 1) : r.range(0, (1 << 12) - 1);
                }
            }
        }
    });
}

// LZ workload: order-2 Markov bytes over 64 symbols; at each generator step,
// with probability 0.4 a copy of length uniform in [3,258] from a distance
// uniform in [1,max_dist] (capped at the position) is emitted instead of one
// symbol.  Generated in independent 4 MiB blocks.
void gd_gen_markov_copy(uint64_t seed, uint64_t n, uint32_t max_dist, uint8_t* out) {
    Markov mk(seed);
    const uint64_t B = 4ull << 20;
    uint64_t nb = (n + B - 1) / B;
    parallel_for(nb, [&](uint64_t b) {
        Rng r(mix(seed, b + 77));
        uint64_t start = b * B, end = std::min(n, start + B), i = start;
        while (i < end) {
            uint64_t pos = i - start;
            if (pos > 0 && r.unit() < 0.4) {
                uint64_t L = (uint64_t)r.range(3, 258);
                uint64_t d = (uint64_t)r.range(1, max_dist);
                if (d > pos) d = pos;
                for (uint64_t k = 0; k < L && i < end; ++k, ++i) out[i] = out[i - d];
            } else {
                uint8_t a = pos >= 2 ? out[i - 2] : 0, c = pos >= 1 ? out[i - 1] : 0;
                out[i] = mk.next(r, a, c);
                ++i;
            }
        }
    });
}

// n sizes drawn log-uniform in [lo, hi], scaled so they sum to `total`,
// each a multiple of `granule` (>= granule).  Returns 0 on success.
int gd_gen_loguniform_sizes(uint64_t seed, uint32_t n, uint64_t lo, uint64_t hi, uint64_t total, uint64_t granule,
                            uint64_t* out) {
    if (n == 0 || granule == 0 || total < (uint64_t)n * granule) return 1;
    Rng r(mix(seed, 0x51E5));
    std::vector<double> x(n);
    double s = 0, llo = std::log((double)lo), lhi = std::log((double)hi);
    for (uint32_t i = 0; i < n; ++i) {
        x[i] = std::exp(llo + (lhi - llo) * r.unit());
        s += x[i];
    }
    uint64_t units = total / granule, acc = 0;
    for (uint32_t i = 0; i < n; ++i) {
        uint64_t u = (uint64_t)std::llround(x[i] / s * (double)units);
        if (u < 1) u = 1;
        out[i] = u;
        acc += u;
    }
    // fix the rounding drift on the largest entries / smallest entries
    int64_t drift = (int64_t)units - (int64_t)acc;
    uint32_t k = 0;
    while (drift != 0) {
        uint32_t i = (uint32_t)(mix(seed, k++) % n);
        if (drift > 0) {
            out[i]++;
            drift--;
        } else if (out[i] > 1) {
            out[i]--;
            drift++;
        }
    }
    for (uint32_t i = 0; i < n; ++i) out[i] *= granule;
    return 0;
}

}  // extern "C"
