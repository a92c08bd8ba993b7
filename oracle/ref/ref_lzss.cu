// ref_lzss -- runs the reference's own contiguous LZSS codec
// (include/lzss/lzss_cpu.h, compiled from the reference sources) on one
// stream.  The 32-column container applies this token grammar to each column
// (lzss_gpu2.h:330-707), so one column = one call here.  Oracle tooling only.
//   ref_lzss encode <raw> <stream>           lzss::compress_func, one chunk
//   ref_lzss decode <stream> <n_out> <raw>    lzss::decompress_func
//   ref_lzss encode_lanes <raw> <bytes per stream> <threads> <streams>
//       lzss::compress_func of every consecutive <bytes per stream> bytes on
//       <threads> host threads, written in the bench format below
//   ref_lzss bench <streams> <threads> <seconds>   lzss::decompress_func on every
//       stream of a [u64 n][u64 bytes per stream][u64 offsets[n+1]][bytes] file
//       on <threads> host threads, repeated for about <seconds>; prints
//       "<bytes decoded> <seconds taken>"
#include <lzss/lzss_cpu.h>

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

static int bench(const std::vector<uint8_t>& in, int threads, double budget) {
    uint64_t n, nb;
    memcpy(&n, in.data(), 8);
    memcpy(&nb, in.data() + 8, 8);
    std::vector<uint64_t> off(n + 1);
    memcpy(off.data(), in.data() + 16, 8 * (n + 1));
    const uint8_t* data = in.data() + 16 + 8 * (n + 1);
    uint64_t bytes = 0;
    const auto t0 = std::chrono::steady_clock::now();
    double dt = 0;
    do {
        std::atomic<uint64_t> next{0};
        std::vector<std::thread> th;
        for (int t = 0; t < threads; ++t)
            th.emplace_back([&]() {
                std::vector<uint8_t> out(nb + 64);
                for (uint64_t i; (i = next.fetch_add(1)) < n;) {
                    const uint64_t lens[1] = {off[i + 1] - off[i]};
                    lzss::decompress_func(data + off[i], out.data(), lens[0], nb, nb, 1, lens, 0);
                }
            });
        for (auto& x : th) x.join();
        bytes += n * nb;
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
        const uint64_t nb = strtoull(argv[3], nullptr, 10);
        const int threads = atoi(argv[4]);
        if (nb == 0 || in.size() % nb) return 4;
        const uint64_t n = in.size() / nb;
        const uint64_t oc = nb + OVERHEAD_PER_CHUNK_((uint32_t)nb) + 16;
        std::vector<std::vector<uint8_t>> enc(n);
        std::atomic<uint64_t> next{0};
        std::vector<std::thread> th;
        for (int t = 0; t < threads; ++t)
            th.emplace_back([&]() {
                std::vector<uint8_t> buf(oc);
                for (uint64_t i; (i = next.fetch_add(1)) < n;) {
                    uint64_t len = 0;
                    std::fill(buf.begin(), buf.end(), 0);  // the trailing reserved flag byte stays 0
                    lzss::compress_func(in.data() + i * nb, buf.data(), nb, oc, nb, oc, 1, &len, 0);
                    enc[i].assign(buf.begin(), buf.begin() + len);
                }
            });
        for (auto& x : th) x.join();
        std::vector<uint64_t> head(2 + n + 1);
        head[0] = n;
        head[1] = nb;
        for (uint64_t i = 0; i < n; ++i) head[3 + i] = head[2 + i] + enc[i].size();
        std::vector<uint8_t> out(8 * head.size() + head[2 + n] + 64, 0);
        memcpy(out.data(), head.data(), 8 * head.size());
        for (uint64_t i = 0; i < n; ++i) memcpy(out.data() + 8 * head.size() + head[2 + i], enc[i].data(), enc[i].size());
        spit(argv[5], out.data(), out.size());
        return 0;
    }
    if (!strcmp(argv[1], "encode")) {
        const uint64_t n = in.size();
        const uint64_t oc = n + OVERHEAD_PER_CHUNK_((uint32_t)n) + 16;
        std::vector<uint8_t> out(oc, 0);  // the trailing reserved flag byte stays 0
        uint64_t len = 0;
        lzss::compress_func(in.data(), out.data(), n, oc, n, oc, 1, &len, 0);
        spit(argv[3], out.data(), len);
    } else {
        const uint64_t n_out = strtoull(argv[3], nullptr, 10);
        std::vector<uint8_t> out(n_out + 64, 0);
        uint64_t lens[1] = {in.size()};
        lzss::decompress_func(in.data(), out.data(), in.size(), n_out, n_out, 1, lens, 0);
        spit(argv[4], out.data(), n_out);
    }
    return 0;
}
