// ref_lzss -- runs the reference's own contiguous LZSS codec
// (include/lzss/lzss_cpu.h, compiled from the reference sources) on one
// stream.  The 32-column container applies this token grammar to each column
// (lzss_gpu2.h:330-707), so one column = one call here.  Oracle tooling only.
//   ref_lzss encode <raw> <stream>           lzss::compress_func, one chunk
//   ref_lzss decode <stream> <n_out> <raw>    lzss::decompress_func
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
