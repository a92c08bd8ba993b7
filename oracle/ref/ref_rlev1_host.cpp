// ref_rlev1_host -- the reference's own RLE v1 GPU writer and reader
// (include/rle_v1/encoder.h: setup_deflate, reduction_scan, deflate, as
// rle_v1::compress_gpu launches them, rlev1.h:25-97; include/rle_v1/
// decoder.h: inflate with its reader and decoder warps, as
// rle_v1::decompress_gpu launches it, rlev1.h:100-199) run on host threads
// through host_cuda.h, to produce golden containers and decoded outputs.  The
// reference has no CPU RLE v1 code.  Oracle tooling only.
//   ref_rlev1_host encode <raw> <elem bytes 4|8> <chunk size> <COMP_COL_LEN> <out prefix>
//       writes <out prefix>.data (the blocks, blk_off[n] bytes; bytes the
//       writer never stores are 0), .col_len (u64 x 32n) and .blk_off (u64 x n+1)
//   ref_rlev1_host decode <prefix> <elem bytes 4|8> <chunk size> <COMP_COL_LEN> <out bytes> <raw out>
//       decodes <prefix>.data / .col_len / .blk_off
#include <rle_v1/encoder.h>
#include <rle_v1/decoder.h>

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
static void spit(const std::string& p, const void* d, size_t n) {
    FILE* f = fopen(p.c_str(), "wb");
    if (!f || fwrite(d, 1, n, f) != n) exit(3);
    fclose(f);
}

template <typename T>
static int encode(std::vector<uint8_t>& in, uint64_t chunk, int ccl, const std::string& pre) {
    const uint64_t n = in.size();
    const uint32_t num_blk = (uint32_t)((n + chunk - 1) / chunk);
    in.resize((uint64_t)num_blk * chunk, 0);  // compress_gpu zeroes d_in past the input (rlev1.h:41-43)
    std::vector<uint64_t> col_len(32ull * num_blk, 0), blk_off(num_blk + 1, 0);
    hc::launch({num_blk, 1, 1}, {32, 2, 1}, [&]() {
        setup_deflate<uint64_t, T, uint32_t, 8>(in.data(), col_len.data(), blk_off.data(), chunk, ccl);
    });
    reduction_scan(blk_off.data(), num_blk);
    std::vector<uint8_t> out(blk_off[num_blk] + 256, 0);
    hc::launch({num_blk, 1, 1}, {32, 2, 1}, [&]() {
        deflate<uint64_t, T, uint32_t, 8>(in.data(), out.data(), col_len.data(), blk_off.data(), chunk, ccl);
    });
    spit(pre + ".data", out.data(), blk_off[num_blk]);
    spit(pre + ".col_len", col_len.data(), 8 * col_len.size());
    spit(pre + ".blk_off", blk_off.data(), 8 * blk_off.size());
    return 0;
}

template <typename T>
static int decode(const std::string& pre, uint64_t chunk, int ccl, uint64_t n_out, const char* dst) {
    std::vector<uint8_t> data = slurp((pre + ".data").c_str());
    std::vector<uint8_t> clb = slurp((pre + ".col_len").c_str()), bob = slurp((pre + ".blk_off").c_str());
    const uint32_t num_blk = (uint32_t)(bob.size() / 8 - 1);
    std::vector<uint64_t> col_len(clb.size() / 8), blk_off(num_blk + 1);
    memcpy(col_len.data(), clb.data(), clb.size());
    memcpy(blk_off.data(), bob.data(), bob.size());
    data.resize(data.size() + 256, 0);
    std::vector<uint8_t> out((uint64_t)num_blk * chunk, 0);
    hc::launch({num_blk, 1, 1}, {32, 2, 1}, [&]() {
        inflate<uint32_t, T, uint32_t, 8>(data.data(), out.data(), col_len.data(), blk_off.data(), chunk, ccl);
    });
    spit(dst, out.data(), n_out < out.size() ? n_out : out.size());
    return 0;
}

int main(int argc, char** argv) {
    if (argc >= 8 && !strcmp(argv[1], "decode")) {
        const int eb = atoi(argv[3]);
        const uint64_t chunk = strtoull(argv[4], nullptr, 10), n_out = strtoull(argv[6], nullptr, 10);
        const int ccl = atoi(argv[5]);
        if (eb == 4) return decode<uint32_t>(argv[2], chunk, ccl, n_out, argv[7]);
        if (eb == 8) return decode<uint64_t>(argv[2], chunk, ccl, n_out, argv[7]);
        return 4;
    }
    if (argc < 7 || strcmp(argv[1], "encode")) return 1;
    std::vector<uint8_t> in = slurp(argv[2]);
    const int eb = atoi(argv[3]);
    const uint64_t chunk = strtoull(argv[4], nullptr, 10);
    const int ccl = atoi(argv[5]);
    if (chunk == 0 || ccl <= 0 || chunk % (32ull * ccl) || in.empty()) return 4;
    if (eb == 4) return encode<uint32_t>(in, chunk, ccl, argv[6]);
    if (eb == 8) return encode<uint64_t>(in, chunk, ccl, argv[6]);
    return 4;
}
