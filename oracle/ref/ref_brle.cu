// ref_brle -- runs the reference's own byte-RLE codec (include/brle/brle.h,
// compiled from the reference sources) on a file.  Oracle tooling only.
//   ref_brle encode <raw> <container>   brle::encode per 256 KiB chunk, laid out
//                                       as brle::compress_gpu does (brle.h:278-292)
//   ref_brle decode <container> <raw>   brle::decode per chunk (brle.h:26-100)
//   ref_brle bench <container> <threads> <seconds>
//                                       brle::decode of every chunk on <threads>
//                                       host threads, repeated for about <seconds>;
//                                       prints "<bytes decoded> <seconds taken>"
#include <brle/brle.h>

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
    uint32_t n_ptr;
    memcpy(&n_ptr, in.data(), 4);
    std::vector<uint64_t> ptr(n_ptr);
    memcpy(ptr.data(), in.data() + 4, 8 * n_ptr);
    uint64_t total;
    memcpy(&total, in.data() + 4 + 8 * n_ptr, 8);
    const uint8_t* data = in.data() + 4 + 8 * n_ptr + 8;
    const uint64_t nc = n_ptr - 1;
    std::vector<uint8_t> out(nc * CHUNK_SIZE);
    uint64_t bytes = 0;
    const auto t0 = std::chrono::steady_clock::now();
    double dt = 0;
    do {
        std::atomic<uint64_t> next{0};
        std::vector<std::thread> th;
        for (int t = 0; t < threads; ++t)
            th.emplace_back([&]() {
                for (uint64_t c; (c = next.fetch_add(1)) < nc;) brle::decode(data, out.data(), ptr.data(), c);
            });
        for (auto& x : th) x.join();
        bytes += total;
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
        const uint64_t nc = (n - 1) / CHUNK_SIZE + 1;
        in.resize(nc * CHUNK_SIZE, 0);  // encode reads only min(n - c*CHUNK, CHUNK) bytes
        std::vector<uint8_t> enc(nc * OUTPUT_CHUNK_SIZE);
        std::vector<uint64_t> ptr(nc + 1, 0);
        for (uint64_t c = 0; c < nc; ++c)
            ptr[c + 1] = ptr[c] + brle::encode(in.data() + c * CHUNK_SIZE, enc.data() + c * OUTPUT_CHUNK_SIZE, n, c);
        std::vector<uint8_t> out(4 + 8 * (nc + 1) + 8 + ptr[nc]);
        const uint32_t n_ptr = (uint32_t)(nc + 1);
        memcpy(out.data(), &n_ptr, 4);
        memcpy(out.data() + 4, ptr.data(), 8 * (nc + 1));
        memcpy(out.data() + 4 + 8 * (nc + 1), &n, 8);
        for (uint64_t c = 0; c < nc; ++c)
            memcpy(out.data() + 4 + 8 * (nc + 1) + 8 + ptr[c], enc.data() + c * OUTPUT_CHUNK_SIZE, ptr[c + 1] - ptr[c]);
        spit(argv[3], out.data(), out.size());
    } else {
        uint32_t n_ptr;
        memcpy(&n_ptr, in.data(), 4);
        std::vector<uint64_t> ptr(n_ptr);
        memcpy(ptr.data(), in.data() + 4, 8 * n_ptr);
        uint64_t total;
        memcpy(&total, in.data() + 4 + 8 * n_ptr, 8);
        const uint8_t* data = in.data() + 4 + 8 * n_ptr + 8;
        std::vector<uint8_t> out((uint64_t)(n_ptr - 1) * CHUNK_SIZE);
        for (uint64_t c = 0; c + 1 < n_ptr; ++c) brle::decode(data, out.data(), ptr.data(), c);
        spit(argv[3], out.data(), total);
    }
    return 0;
}
