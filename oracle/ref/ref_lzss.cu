// ref_lzss -- runs the reference's own contiguous LZSS codec
// (include/lzss/lzss_cpu.h, compiled from the reference sources) on one
// stream.  The 32-column container applies this token grammar to each column
// (lzss_gpu2.h:330-707), so one column = one call here.  Oracle tooling only.
//   ref_lzss encode <raw> <stream>           lzss::compress_func, one chunk
//   ref_lzss decode <stream> <n_out> <raw>    lzss::decompress_func
#include <lzss/lzss_cpu.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
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

int main(int argc, char** argv) {
    if (argc < 4) return 1;
    std::vector<uint8_t> in = slurp(argv[2]);
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
