// ref_brle_trans_host -- the reference's own byte-RLE flag-container GPU
// writer (brle_trans::compress_init_func, writeupdate and compress_func of
// include/brle/brle_trans.h, extracted by extract_fns.awk into
// _ref/inc/brle_trans_writer.h) run on host threads through host_cuda.h, as
// brle_trans::compress_gpu launches it (brle_trans.h:563-660), to produce
// golden containers, and its reader (brle_trans::decompress_func, :72-202,
// launched as decompress_gpu does, :758: n/2 blocks of 64 threads, two
// chunks per block).  Built with REF_SYM4 it runs the 4-byte-symbol writer
// and reader instead (brle::compress_init_func, check_f, writeupdate,
// compress_func, parallel_scan and decompress_func of
// include/brle/brle_gpu_4B.h, as its compress_gpu and decompress_gpu launch
// them, :640-735, :860).  The reference has no CPU code for these
// containers.  Oracle tooling only.
//   ref_brle_trans_host encode <raw, a multiple of CHUNK_SIZE bytes> <out prefix>
//       writes <out prefix>.data (blk_off[n] bytes; bytes the writer never
//       stores are 0), .col_len (u64 x 32n, sorted), .col_map (u8 x 32n) and
//       .blk_off (u64 x n+1)
//   ref_brle_trans_host decode <prefix> <out bytes> <raw out>
#ifdef REF_SYM4
#include "brle_gpu_4B_writer.h"
namespace wr = brle;
#else
#include "brle_trans_writer.h"
namespace wr = brle_trans;
#endif

#include <cstdlib>
#include <cstring>
#include <string>
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
static void spit(const std::string& p, const void* d, size_t n) {
    FILE* f = fopen(p.c_str(), "wb");
    if (!f || fwrite(d, 1, n, f) != n) exit(3);
    fclose(f);
}

static int decode(const std::string& pre, uint64_t n_out, const char* dst) {
    std::vector<uint8_t> data = slurp((pre + ".data").c_str()), cm = slurp((pre + ".col_map").c_str());
    std::vector<uint8_t> clb = slurp((pre + ".col_len").c_str()), bob = slurp((pre + ".blk_off").c_str());
    const uint32_t nb = (uint32_t)(bob.size() / 8 - 1);
    std::vector<uint64_t> col_len(clb.size() / 8), blk(nb + 1);
    memcpy(col_len.data(), clb.data(), clb.size());
    memcpy(blk.data(), bob.data(), bob.size());
    data.resize(data.size() + 256, 0);
    std::vector<uint8_t> out((uint64_t)nb * CHUNK_SIZE, 0);
#ifdef REF_SYM4
    hc::launch({nb, 1, 1}, {BLK_SIZE, 1, 1}, [&]() {
        wr::decompress_func(data.data(), out.data(), nb, col_len.data(), cm.data(), blk.data());
    });
#else
    hc::launch({nb / 2, 1, 1}, {64, 1, 1}, [&]() {
        wr::decompress_func(data.data(), out.data(), nb, col_len.data(), cm.data(), blk.data());
    });
#endif
    spit(dst, out.data(), n_out < out.size() ? n_out : out.size());
    return 0;
}

int main(int argc, char** argv) {
    if (argc >= 5 && !strcmp(argv[1], "decode")) return decode(argv[2], strtoull(argv[3], nullptr, 10), argv[4]);
    if (argc < 4 || strcmp(argv[1], "encode")) return 1;
    std::vector<uint8_t> in = slurp(argv[2]);
    const std::string pre = argv[3];
    const uint64_t n = in.size();
    if (n == 0 || n % CHUNK_SIZE) return 4;
    // compress_gpu: n_chunks = in / CHUNK_SIZE, chunk_size = in / n_chunks
    const uint32_t nc = (uint32_t)(n / CHUNK_SIZE);
    const uint64_t chunk = n / nc;
    const uint64_t exp_out = chunk + OVERHEAD_PER_CHUNK_(chunk);
    std::vector<uint64_t> col_len(32ull * nc, 0), blk(nc + 1, 0), sorted(32ull * nc, 0);
    std::vector<uint8_t> col_map(32ull * nc, 0);
    hc::launch({nc, 1, 1}, {BLK_SIZE, 1, 1}, [&]() {
        wr::compress_init_func(in.data(), n, chunk, exp_out, nc, col_len.data(), blk.data());
    });
#ifdef REF_SYM4
    wr::parallel_scan(blk.data(), nc);  // brle_gpu_4B.h:710
#else
    // cub::DeviceScan::InclusiveSum over blk_offset[0..n] (brle_trans.h:612-619)
    for (uint32_t c = 1; c <= nc; ++c) blk[c] += blk[c - 1];
#endif
    // ExampleKernel (brle_trans.h:202-221, brle_gpu_4B.h:225-244): cub::BlockRadixSort of the 32
    // (col_len, column) pairs, ascending and stable, stored back to front
    for (uint32_t c = 0; c < nc; ++c) {
        std::vector<std::pair<uint64_t, int>> kv(32);
        for (int t = 0; t < 32; ++t) kv[t] = {col_len[32ull * c + t], t};
        std::stable_sort(kv.begin(), kv.end(), [](auto& a, auto& b) { return a.first < b.first; });
        for (int i = 0; i < 32; ++i) {
            col_map[32ull * c + 31 - i] = (uint8_t)kv[i].second;
            sorted[32ull * c + 31 - i] = kv[i].first;
        }
    }
    std::vector<uint8_t> out(blk[nc] + 256, 0);
    uint64_t out_n = 0;
    hc::launch({nc, 1, 1}, {BLK_SIZE, 1, 1}, [&]() {
        wr::compress_func(in.data(), out.data(), n, &out_n, chunk, nc, sorted.data(), col_map.data(),
                                  blk.data());
    });
    spit(pre + ".data", out.data(), blk[nc]);
    spit(pre + ".col_len", sorted.data(), 8 * sorted.size());
    spit(pre + ".col_map", col_map.data(), col_map.size());
    spit(pre + ".blk_off", blk.data(), 8 * blk.size());
    return 0;
}
