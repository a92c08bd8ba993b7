// ref_rlev2 -- runs the reference's own contiguous RLE v2 codec
// (include/rlev2/encoder.h block_encode, include/rlev2/decoder.h
// block_decode; HEAD side of the unresolved merge, patch mask widened to 64
// bits -- see oracle/ref/Makefile) on one stream of int64 values.  The
// transposed container applies the same per-lane encoder to each lane's
// values (encoder_trans.h:9-289).  Oracle tooling only.
//   ref_rlev2 encode <int64 raw> <stream>           block_encode, one chunk (<= 4096 values)
//   ref_rlev2 decode <stream> <n_values> <int64 raw> block_decode
//   ref_rlev2 encode_lanes <int64 raw> <values per stream> <threads> <streams>
//       block_encode of every consecutive group of <values per stream> values
//       on <threads> host threads, written in the bench format below
//   ref_rlev2 bench <streams> <threads> <seconds>   block_decode of every stream
//       of a [u64 n][u64 values per stream][u64 offsets[n+1]][bytes] file on
//       <threads> host threads, repeated for about <seconds>; prints
//       "<bytes decoded> <seconds taken>"
#include <common.h>
#include <rlev2/encoder.h>
#include <rlev2/decoder.h>

#include <atomic>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <algorithm>
#include <thread>
#include <vector>

static std::vector<uint8_t> slurp(const char* p) {
    FILE* f = fopen(p, "rb");
    if (!f) exit(2);
    std::vector<uint8_t> v;
    uint8_t buf[1 << 16];
    size_t n;
    while ((n = fread(buf, 1, sizeof buf, f)) > 0) v.insert(v.end(), buf, buf + n);
    fclose(f);
    return v;
}
static void spit(const char* p, const void* d, size_t n) {
    FILE* f = fopen(p, "wb");
    if (!f || fwrite(d, 1, n, f) != n) exit(3);
    fclose(f);
}

static int bench(std::vector<uint8_t>& in, int threads, double budget) {
    uint64_t n, nv;
    memcpy(&n, in.data(), 8);
    memcpy(&nv, in.data() + 8, 8);
    std::vector<uint64_t> off(n + 1);
    memcpy(off.data(), in.data() + 16, 8 * (n + 1));
    uint8_t* data = in.data() + 16 + 8 * (n + 1);
    uint64_t bytes = 0;
    const auto t0 = std::chrono::steady_clock::now();
    double dt = 0;
    do {
        std::atomic<uint64_t> next{0};
        std::vector<std::thread> th;
        for (int t = 0; t < threads; ++t)
            th.emplace_back([&]() {
                // decode_delta writes two values past a run (decoder.h:117-123): slack
                std::vector<int64_t> out(CHUNK_SIZE / 8 + 16);
                for (uint64_t i; (i = next.fetch_add(1)) < n;) rlev2::block_decode(0, data, off.data() + i, out.data());
            });
        for (auto& x : th) x.join();
        bytes += n * nv * 8;
        dt = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    } while (dt < budget);
    printf("%llu %.6f\n", (unsigned long long)bytes, dt);
    return 0;
}

int main(int argc, char** argv) {
    if (argc < 4) return 1;
    std::vector<uint8_t> in = slurp(argv[2]);
    if (!strcmp(argv[1], "bench")) return bench(in, atoi(argv[3]), argc > 4 ? atof(argv[4]) : 5.0);
    if (!strcmp(argv[1], "encode_lanes")) {
        if (argc < 6) return 1;
        const uint64_t nv = strtoull(argv[3], nullptr, 10);
        const int threads = atoi(argv[4]);
        if (nv == 0 || nv * 8 > CHUNK_SIZE || in.size() % (nv * 8)) return 4;
        const uint64_t n = in.size() / (nv * 8);
        std::vector<std::vector<uint8_t>> enc(n);
        std::atomic<uint64_t> next{0};
        std::vector<std::thread> th;
        for (int t = 0; t < threads; ++t)
            th.emplace_back([&]() {
                std::vector<uint8_t> buf(OUTPUT_CHUNK_SIZE * 2);
                for (uint64_t i; (i = next.fetch_add(1)) < n;) {
                    uint64_t len = 0;
                    std::fill(buf.begin(), buf.end(), 0);
                    rlev2::block_encode(0, reinterpret_cast<int64_t*>(in.data() + i * nv * 8), nv * 8, buf.data(), &len);
                    enc[i].assign(buf.begin(), buf.begin() + len);
                }
            });
        for (auto& x : th) x.join();
        std::vector<uint64_t> head(2 + n + 1);
        head[0] = n;
        head[1] = nv;
        for (uint64_t i = 0; i < n; ++i) head[3 + i] = head[2 + i] + enc[i].size();
        std::vector<uint8_t> out(8 * head.size() + head[2 + n] + 64, 0);
        memcpy(out.data(), head.data(), 8 * head.size());
        for (uint64_t i = 0; i < n; ++i) memcpy(out.data() + 8 * head.size() + head[2 + i], enc[i].data(), enc[i].size());
        spit(argv[5], out.data(), out.size());
        return 0;
    }
    if (!strcmp(argv[1], "encode")) {
        if (in.size() > CHUNK_SIZE) return 4;
        std::vector<uint8_t> out(OUTPUT_CHUNK_SIZE * 2, 0);
        uint64_t len = 0;
        rlev2::block_encode(0, reinterpret_cast<int64_t*>(in.data()), in.size(), out.data(), &len);
        spit(argv[3], out.data(), len);
    } else {
        const uint64_t nv = strtoull(argv[3], nullptr, 10);
        // decode_delta writes two values past a run (decoder.h:117-123): slack
        std::vector<int64_t> out(CHUNK_SIZE / 8 + 16, 0);
        uint64_t off[2] = {0, in.size()};
        rlev2::block_decode(0, in.data(), off, out.data());
        spit(argv[4], out.data(), nv * 8);
    }
    return 0;
}
