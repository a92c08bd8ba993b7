// gd_compat.hpp -- the reference's namespaced host entry points, forwarded to
// the C ABI of libgd.so (include/gd.h).
//
// A program written against ZaidQureshi/compression's decompress calls can
// swap its codec headers for this one and link -lgd: the names, template
// parameters, argument meanings, side files and output ownership (new[]) are
// the reference's.  Template parameters that only tuned the reference's
// kernels (queue depths, read/write unit types) are accepted and ignored.
#pragma once

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

#include "gd.h"

namespace gd_compat_detail {

// Move a library-owned result into a new[] buffer (the reference's ownership).
inline uint8_t* adopt(uint8_t* p, uint64_t n) {
    uint8_t* q = new uint8_t[n ? n : 1];
    if (n) std::memcpy(q, p, n);
    gd_free(p);
    return q;
}

inline bool read_file(const std::string& path, std::vector<uint64_t>& v) {
    std::ifstream f(path, std::ios::binary | std::ios::ate);
    if (!f) return false;
    const std::streamsize n = f.tellg();
    f.seekg(0);
    v.resize((size_t)n / 8);
    return (bool)f.read(reinterpret_cast<char*>(v.data()), (std::streamsize)(v.size() * 8));
}

inline void report(int rc, const char* where) {
    if (rc != GD_OK) std::fprintf(stderr, "gd: %s: %s\n", where, gd_status_string(rc));
}

}  // namespace gd_compat_detail

// include/brle/brle.h:305-342
namespace brle {
inline void decompress_gpu(const uint8_t* const in, uint8_t** out, const uint64_t in_n_bytes, uint64_t* out_n_bytes) {
    uint8_t* p = nullptr;
    uint64_t n = 0;
    const gd_status_t rc = gd_brle_decompress(in, in_n_bytes, &p, &n);
    gd_compat_detail::report(rc, "brle::decompress_gpu");
    *out = rc == GD_OK ? gd_compat_detail::adopt(p, n) : nullptr;
    *out_n_bytes = rc == GD_OK ? n : 0;
}
}  // namespace brle

// include/rle_v1/rlev1.h:100-199: metadata from the side files the
// reference's compress_gpu writes (./input_data/rle_v1_{col_len,blk_offset}.bin).
namespace rle_v1 {
template <typename READ_COL_TYPE, typename DATA_TYPE, typename OUT_COL_TYPE, int QUEUE_SIZE = 8>
void decompress_gpu(const uint8_t* const in, uint8_t** out, const uint64_t in_n_bytes, uint64_t* out_n_bytes,
                    int COMP_COL_LEN, uint64_t chunk_size) {
    std::vector<uint64_t> col, blk;
    *out = nullptr;
    *out_n_bytes = 0;
    if (!gd_compat_detail::read_file("./input_data/rle_v1_col_len.bin", col) ||
        !gd_compat_detail::read_file("./input_data/rle_v1_blk_offset.bin", blk)) {
        std::fprintf(stderr, "Fatal Error: Col Len read error\n");
        return;
    }
    uint8_t* p = nullptr;
    uint64_t n = 0;
    const gd_status_t rc = gd_rlev1_decompress(in, in_n_bytes, col.data(), col.size() * 8, blk.data(),
                                               blk.size() * 8, (uint32_t)COMP_COL_LEN, (uint32_t)sizeof(DATA_TYPE),
                                               chunk_size, &p, &n);
    gd_compat_detail::report(rc, "rle_v1::decompress_gpu");
    if (rc == GD_OK) {
        *out = gd_compat_detail::adopt(p, n);
        *out_n_bytes = n;
    }
}
}  // namespace rle_v1

// include/rlev2/decoder_trans.h:615-681 (8-byte values; blk_off[n_chunks]
// holds the decompressed size, as compress_gpu_transpose leaves it).
namespace rlev2 {
template <int READ_UNIT, int queue_size, typename COMP_TYPE>
void decompress_gpu(const uint8_t* in, const uint64_t in_n_bytes, const uint64_t n_chunks, uint64_t* blk_off,
                    uint64_t* col_len, uint64_t*& out, uint64_t& out_n_bytes, uint64_t CHUNK_SIZE) {
    uint8_t* p = nullptr;
    uint64_t n = 0;
    const gd_status_t rc =
        gd_rlev2_decompress(in, in_n_bytes, n_chunks, blk_off, col_len, (uint32_t)READ_UNIT, CHUNK_SIZE, &p, &n);
    gd_compat_detail::report(rc, "rlev2::decompress_gpu");
    out = nullptr;
    out_n_bytes = 0;
    if (rc == GD_OK) {
        out = new uint64_t[n / 8 ? n / 8 : 1];
        std::memcpy(out, p, n);
        gd_free(p);
        out_n_bytes = n;
    }
}
}  // namespace rlev2

// include/lzss/lzss_gpu2.h:2129-2314 (metadata as the .meta sidecar holds it)
namespace lzss {
inline int decompress_gpu(const uint8_t* const in, const uint64_t in_n_bytes, const uint8_t** const in_metadata,
                          const uint64_t* const in_metadata_lens, const uint64_t in_metadata_num, uint8_t** out,
                          uint64_t* out_n_bytes) {
    uint8_t* p = nullptr;
    uint64_t n = 0;
    const int rc = gd_lzss_decompress(in, in_n_bytes, in_metadata, in_metadata_lens, in_metadata_num, &p, &n);
    if (rc != 0) {
        if (rc > 0) gd_compat_detail::report(rc, "lzss::decompress_gpu");
        *out = nullptr;
        *out_n_bytes = 0;
        return rc;
    }
    *out = gd_compat_detail::adopt(p, n);
    *out_n_bytes = n;
    return 0;
}
}  // namespace lzss

// include/lzss/lzss.h:1126-1188 (contiguous container)
namespace lzss {
inline void decompress_gpu_base(const uint8_t* const in, uint8_t** out, const uint64_t in_n_bytes,
                                uint64_t* out_n_bytes) {
    uint8_t* p = nullptr;
    uint64_t n = 0;
    const gd_status_t rc = gd_lzss_contig_decompress(in, in_n_bytes, &p, &n);
    gd_compat_detail::report(rc, "lzss::decompress_gpu_base");
    *out = rc == GD_OK ? gd_compat_detail::adopt(p, n) : nullptr;
    *out_n_bytes = rc == GD_OK ? n : 0;
}
}  // namespace lzss

// include/brle/brle_trans.h:661-791: metadata from the side files the
// reference's compress_gpu writes (./input_data/{col_len,col_map,blk_offset}.bin),
// 4 KiB chunks.
namespace brle_trans {
inline void decompress_gpu(const uint8_t* const in, uint8_t** out, const uint64_t in_n_bytes, uint64_t* out_n_bytes) {
    std::vector<uint64_t> col, blk;
    *out = nullptr;
    *out_n_bytes = 0;
    std::ifstream fm("./input_data/col_map.bin", std::ios::binary | std::ios::ate);
    if (!gd_compat_detail::read_file("./input_data/col_len.bin", col) ||
        !gd_compat_detail::read_file("./input_data/blk_offset.bin", blk) || !fm) {
        std::fprintf(stderr, "Fatal Error: Col Len read error\n");
        return;
    }
    std::vector<uint8_t> map((size_t)fm.tellg());
    fm.seekg(0);
    fm.read(reinterpret_cast<char*>(map.data()), (std::streamsize)map.size());
    uint8_t* p = nullptr;
    uint64_t n = 0;
    const gd_status_t rc = gd_brle_trans_decompress(in, in_n_bytes, col.data(), col.size() * 8, map.data(),
                                                    map.size(), blk.data(), blk.size() * 8, 4096, &p, &n);
    gd_compat_detail::report(rc, "brle_trans::decompress_gpu");
    if (rc == GD_OK) {
        *out = gd_compat_detail::adopt(p, n);
        *out_n_bytes = n;
    }
}
}  // namespace brle_trans

// include/zlib/zlib.h:966-1082
namespace deflate {
template <typename READ_COL_TYPE, size_t WRITE_COL_LEN, uint16_t queue_depth, uint8_t NUM_SUBCHUNKS,
          bool shared_tree_flag = false>
void decompress_gpu(const uint8_t* const in, uint8_t** out, const uint64_t in_n_bytes, uint64_t* out_n_bytes,
                    uint64_t* col_len_f, const uint64_t col_n_bytes, uint64_t* blk_offset_f, const uint64_t blk_n_bytes,
                    uint64_t chunk_size) {
    uint8_t* p = nullptr;
    uint64_t n = 0;
    const gd_status_t rc =
        gd_deflate_decompress(in, in_n_bytes, col_len_f, col_n_bytes, blk_offset_f, blk_n_bytes, chunk_size, &p, &n);
    gd_compat_detail::report(rc, "deflate::decompress_gpu");
    *out = rc == GD_OK ? gd_compat_detail::adopt(p, n) : nullptr;
    *out_n_bytes = rc == GD_OK ? n : 0;
}
}  // namespace deflate

// include/cudf_deflate.cuh:236-250, 1399-1415 (device-side descriptor API)
namespace cudf {
namespace io {
using gpu_inflate_input_s = ::gd_inflate_input;
using gpu_inflate_status_s = ::gd_inflate_status;
inline int gpuinflate(gpu_inflate_input_s* inputs, gpu_inflate_status_s* outputs, int count, int parse_hdr,
                      void* stream = nullptr) {
    return gd_gpuinflate(inputs, outputs, count, parse_hdr, stream) == GD_OK ? 0 : 1;
}
inline int gpu_copy_uncompressed_blocks(gpu_inflate_input_s* inputs, int count, void* stream = nullptr) {
    return gd_copy_uncompressed_blocks(inputs, count, stream) == GD_OK ? 0 : 1;
}
}  // namespace io
}  // namespace cudf

// ---------------------------------------------------------------------------
// Writers: the reference's compress calls on the device encoders.  Outputs
// are new[] buffers (the LZSS metadata malloc'd), as the reference hands
// them out; rle_v1 writes its side files as the reference does.

namespace gd_compat_detail {
inline bool write_file(const char* path, const void* p, uint64_t n) {
    std::ofstream f(path, std::ios::binary);
    return f && f.write(static_cast<const char*>(p), (std::streamsize)n);
}
}  // namespace gd_compat_detail

// include/brle/brle.h:251-303
namespace brle {
inline void compress_gpu(const uint8_t* in, uint8_t** out, const uint64_t in_n_bytes, uint64_t* out_n_bytes) {
    uint8_t* p = nullptr;
    uint64_t n = 0;
    const gd_status_t rc = gd_brle_compress(in, in_n_bytes, &p, &n);
    gd_compat_detail::report(rc, "brle::compress_gpu");
    *out = rc == GD_OK ? gd_compat_detail::adopt(p, n) : nullptr;
    *out_n_bytes = rc == GD_OK ? n : 0;
}
}  // namespace brle

// include/rle_v1/rlev1.h:22-97: [u64 in_n_bytes][data], with col_len and
// blk_offset written to ./input_data/rle_v1_{col_len,blk_offset}.bin.
namespace rle_v1 {
template <typename READ_COL_TYPE, typename DATA_TYPE, typename OUT_COL_TYPE>
void compress_gpu(const uint8_t* const in, uint8_t** out, const uint64_t in_n_bytes, uint64_t* out_n_bytes,
                  int COMP_COL_LEN, uint64_t CHUNK_SIZE) {
    uint8_t* p = nullptr;
    uint64_t n = 0, nc = 0, *col = nullptr, *blk = nullptr;
    const gd_status_t rc = gd_rlev1_compress(in, in_n_bytes, (uint32_t)COMP_COL_LEN, (uint32_t)sizeof(DATA_TYPE),
                                             CHUNK_SIZE, &p, &n, &col, &blk, &nc);
    gd_compat_detail::report(rc, "rle_v1::compress_gpu");
    *out = nullptr;
    *out_n_bytes = 0;
    if (rc != GD_OK) return;
    if (!gd_compat_detail::write_file("./input_data/rle_v1_col_len.bin", col, 8 * 32 * nc) ||
        !gd_compat_detail::write_file("./input_data/rle_v1_blk_offset.bin", blk, 8 * (nc + 1)))
        std::fprintf(stderr, "gd: rle_v1::compress_gpu: cannot write ./input_data side files\n");
    gd_free(col);
    gd_free(blk);
    *out = gd_compat_detail::adopt(p, n);
    *out_n_bytes = n;
}
}  // namespace rle_v1

// include/rlev2/encoder_trans.h:428-537 (8-byte values; blk_off[n_chunks]
// holds in_n_bytes, as decompress_gpu expects).
namespace rlev2 {
template <int READ_UNIT, typename COMP_TYPE, typename IN_T>
void compress_gpu_transpose(const IN_T* const in, const uint64_t in_n_bytes, uint8_t*& out, uint64_t& out_n_bytes,
                            uint64_t& meta_data_size, uint64_t& out_n_chunks, uint64_t*& blk_off,
                            uint64_t*& col_len, uint64_t CHUNK_SIZE) {
    static_assert(sizeof(IN_T) == 8, "the RLE v2 encoder takes 8-byte values");
    uint8_t* p = nullptr;
    uint64_t n = 0, nc = 0, *bo = nullptr, *cl = nullptr;
    const gd_status_t rc = gd_rlev2_compress(reinterpret_cast<const uint8_t*>(in), in_n_bytes, (uint32_t)READ_UNIT,
                                             CHUNK_SIZE, &p, &n, &bo, &cl, &nc);
    gd_compat_detail::report(rc, "rlev2::compress_gpu_transpose");
    out = nullptr;
    out_n_bytes = meta_data_size = out_n_chunks = 0;
    blk_off = col_len = nullptr;
    if (rc != GD_OK) return;
    blk_off = new uint64_t[nc + 1];
    col_len = new uint64_t[32 * nc];
    std::memcpy(blk_off, bo, 8 * (nc + 1));
    std::memcpy(col_len, cl, 8 * 32 * nc);
    gd_free(bo);
    gd_free(cl);
    out = gd_compat_detail::adopt(p, n);
    out_n_bytes = n;
    out_n_chunks = nc;
    meta_data_size = 8 * 32 * nc + 8 * (nc + 1);  // encoder_trans.h:443
}
}  // namespace rlev2

// include/lzss/lzss_gpu2.h:1952-2127 (128 KiB chunks; the four metadata
// blobs and their arrays are malloc'd, as the reference's are)
namespace lzss {
inline void compress_gpu(const uint8_t* const in, const uint64_t in_n_bytes, uint8_t** out, uint64_t* out_n_bytes,
                         uint8_t*** out_metadata, uint64_t** out_metadata_lens, uint64_t* out_metadata_num) {
    uint8_t* p = nullptr;
    uint64_t n = 0;
    const int rc = gd_lzss_compress(in, in_n_bytes, &p, &n, out_metadata, out_metadata_lens, out_metadata_num);
    gd_compat_detail::report(rc, "lzss::compress_gpu");
    *out = rc == GD_OK ? gd_compat_detail::adopt(p, n) : nullptr;
    *out_n_bytes = rc == GD_OK ? n : 0;
    if (rc != GD_OK) *out_metadata_num = 0;
}
}  // namespace lzss
