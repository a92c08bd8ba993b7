// encode.cu -- RLE v1 and RLE v2 container encoders for sm_100a.
//
// The writer side of the two interleaved integer containers
// (rle_v1::compress_gpu, include/rle_v1/rlev1.h:25-97;
// rlev2::compress_gpu_transpose, include/rlev2/encoder_trans.h:428-537),
// producing the same bytes as the host encoders (both run the lane encoders
// of lane_enc.h).  Three launches on one stream:
//   1. lane_encode_kernel: a warp per chunk, a thread per lane stream.  Each
//      thread gathers its lane's values straight from the column (RLE v1:
//      COMP_COL_LEN-byte slices at a 32-slice stride; RLE v2: READ_UNIT-value
//      slices) and runs the lane encoder into its own scratch slot, buffering
//      4 bytes in a register so the scratch is written in whole words (the
//      literal-count byte written back later is a byte store or a register
//      edit).  The warp sums its lanes' padded word counts into the chunk's
//      block size;
//   2. offsets_kernel: one block turns the block sizes into blk_off;
//   3. interleave_kernel: a block per chunk writes row k = one word of every
//      lane longer than 4k bytes, in lane order, through the same segment
//      table the decoders read with (interleave.cuh), then zeroes the block's
//      pad to 128 bytes.
// The encoders are serial per lane, so the first launch has one thread per
// lane stream (32 x chunks); the column is read once and the scratch and the
// container written once each.
#include "gd_common.cuh"
#include "interleave.cuh"
#include "lane_enc.h"

namespace gd {
namespace encd {

constexpr int NT = 128;  // threads per block (4 chunks per block in launch 1)

// Byte sink over one lane's scratch slot (cap bytes, a multiple of 4).
struct DevSink {
    uint32_t* w;
    uint32_t n, cap, cur;  // bytes put; capacity; bytes [n & ~3, n) not yet stored
    __device__ __forceinline__ void put(uint8_t b) {
        cur |= (uint32_t)b << (8u * (n & 3u));
        ++n;
        if ((n & 3u) == 0) {
            if (n <= cap) w[(n >> 2) - 1] = cur;
            cur = 0;
        }
    }
    __device__ __forceinline__ uint32_t size() const { return n; }
    __device__ __forceinline__ void set(uint64_t i, uint8_t b) {
        if (i >= (n & ~3u)) {
            const uint32_t sh = 8u * ((uint32_t)i & 3u);
            cur = (cur & ~(0xffu << sh)) | ((uint32_t)b << sh);
        } else if (i < cap) {
            reinterpret_cast<uint8_t*>(w)[i] = b;
        }
    }
    // store the last partial word (its unused bytes are zero)
    __device__ __forceinline__ void flush() {
        if ((n & 3u) && n < cap) w[n >> 2] = cur;
    }
};

// RLE v1 lane t: value e is element (e / wil) * 32 * wil + t * wil + e % wil
// of the chunk (encoder.h:139-153); elements past the input are zero.
template <typename T>
struct V1Vals {
    const T* base;
    uint64_t avail;
    uint32_t t, wil;
    __device__ __forceinline__ T operator[](uint64_t e) const {
        const uint32_t q = (uint32_t)e / wil, r = (uint32_t)e - q * wil;
        const uint64_t idx = (uint64_t)q * 32u * wil + (uint64_t)t * wil + r;
        return idx < avail ? base[idx] : (T)0;
    }
};

// RLE v2 lane t: value i is chunk value t * ru + (i / ru) * 32 * ru + i % ru
// (encoder_trans.h:40-108); values past the input are zero.
struct V2Vals {
    const int64_t* base;
    uint64_t avail;
    uint32_t t, ru;
    __device__ __forceinline__ int64_t operator[](uint64_t i) const {
        const uint32_t q = (uint32_t)i / ru, r = (uint32_t)i - q * ru;
        const uint64_t idx = (uint64_t)t * ru + (uint64_t)q * 32u * ru + r;
        return idx < avail ? base[idx] : 0;
    }
};

// CODEC: GD_CODEC_RLEV1 (T = uint32_t / uint64_t, param = wil) or
// GD_CODEC_RLEV2 (T = int64_t, param = read unit).  blk_size[c] gets chunk
// c's block size (the launch passes blk_off + 1).
template <int CODEC, typename T>
__global__ void __launch_bounds__(NT) lane_encode_kernel(const uint8_t* __restrict__ in, uint64_t n_bytes,
                                                         uint32_t n_chunks, uint64_t chunk_size, uint32_t param,
                                                         uint8_t* __restrict__ scratch, uint32_t lane_cap,
                                                         uint64_t* __restrict__ col_len,
                                                         uint64_t* __restrict__ blk_size,
                                                         uint32_t* __restrict__ status) {
    const uint32_t c = (blockIdx.x * NT + threadIdx.x) >> 5;
    const uint32_t t = lane_id();
    if (c >= n_chunks) return;  // warp-uniform
    const uint64_t cb = (uint64_t)c * chunk_size;
    const uint64_t have = n_bytes > cb ? (n_bytes - cb < chunk_size ? n_bytes - cb : chunk_size) : 0;
    DevSink s{reinterpret_cast<uint32_t*>(scratch + ((uint64_t)c * 32u + t) * lane_cap), 0u, lane_cap, 0u};
    if constexpr (CODEC == GD_CODEC_RLEV1) {
        const V1Vals<T> v{reinterpret_cast<const T*>(in + cb), have / sizeof(T), t, param};
        enc::rlev1_encode_lane<T>(v, chunk_size / 32u / sizeof(T), s);
    } else {
        const V2Vals v{reinterpret_cast<const int64_t*>(in + cb), have / 8u, t, param};
        enc::rlev2_encode_lane(v, chunk_size / 256u, s);
    }
    s.flush();
    const bool over = s.n > lane_cap;
    const uint32_t len = over ? 0u : s.n;
    col_len[(uint64_t)c * 32u + t] = len;
    const uint32_t words = __reduce_add_sync(GD_FULL_MASK, (len + 3u) >> 2);
    const bool bad = __any_sync(GD_FULL_MASK, over);
    if (t == 0) {
        blk_size[c] = ((uint64_t)words * 4u + 127u) & ~127ull;
        put_status(status, c, bad ? (uint32_t)ST_OVERRUN : (uint32_t)ST_OK);
    }
}

// blk_off[1..n] hold block sizes on entry and their inclusive prefix sums on
// exit; blk_off[0] = 0.  One block of 1024 threads, each over a contiguous
// range of chunks.
__global__ void __launch_bounds__(1024) offsets_kernel(uint64_t* __restrict__ blk_off, uint32_t n) {
    __shared__ uint64_t tmp[1024 / 32 + 1];
    const uint64_t per = ((uint64_t)n + 1023u) / 1024u;
    const uint64_t b = min((uint64_t)n, threadIdx.x * per), e = min((uint64_t)n, b + per);
    uint64_t sum = 0;
    for (uint64_t i = b; i < e; ++i) sum += blk_off[1 + i];
    uint64_t tot;
    uint64_t acc = block_excl_scan64<1024>(sum, tmp, &tot);
    for (uint64_t i = b; i < e; ++i) {
        acc += blk_off[1 + i];
        blk_off[1 + i] = acc;
    }
    if (threadIdx.x == 0) blk_off[0] = 0;
}

// Block c = lanes' words in rows; a block of NT threads per chunk.
__global__ void __launch_bounds__(NT) interleave_kernel(const uint8_t* __restrict__ scratch, uint32_t lane_cap,
                                                        const uint64_t* __restrict__ col_len,
                                                        const uint64_t* __restrict__ blk_off, uint32_t n_chunks,
                                                        uint8_t* __restrict__ data) {
    __shared__ SegTable T;
    __shared__ uint32_t s_nw[32];
    __shared__ uint32_t s_tot;
    const uint32_t lane = lane_id(), wid = threadIdx.x >> 5;
    for (uint32_t c = blockIdx.x; c < n_chunks; c += gridDim.x) {
        if (wid == 0) {
            const uint32_t nw = (uint32_t)((col_len[(uint64_t)c * 32u + lane] + 3u) >> 2);
            seg_build(&T, nw);
            s_nw[lane] = nw;
            const uint32_t tot = __reduce_add_sync(GD_FULL_MASK, nw);
            if (lane == 0) s_tot = tot;
        }
        __syncthreads();
        const uint64_t b0 = blk_off[c];
        uint32_t* dst = reinterpret_cast<uint32_t*>(data + b0);
        const uint32_t* src0 = reinterpret_cast<const uint32_t*>(scratch + (uint64_t)c * 32u * lane_cap);
        for (uint32_t t = wid; t < 32; t += NT / 32) {
            const uint32_t nw = s_nw[t], ltmask = (1u << t) - 1u;
            const uint32_t* src = src0 + (uint64_t)t * (lane_cap / 4u);
            for (uint32_t k = lane; k < nw; k += 32) {
                uint32_t j = 0;  // segment of row k: the number of lanes with at most k words
#pragma unroll
                for (uint32_t step = 16; step; step >>= 1)
                    if (j + step <= 31 && T.hi[j + step - 1] <= k) j += step;
                const uint32_t lo = j ? T.hi[j - 1] : 0u;
                const uint32_t off = T.base[j] + (k - lo) * 4u * (32u - j) + 4u * __popc(T.mask[j] & ltmask);
                dst[off >> 2] = src[k];
            }
        }
        const uint32_t bw = (uint32_t)((blk_off[c + 1] - b0) >> 2);
        for (uint32_t w = s_tot + threadIdx.x; w < bw; w += NT) dst[w] = 0;
        __syncthreads();  // T and s_nw are rebuilt for the next chunk
    }
}

// Longest lane stream the encoders can write for nv values, rounded to 4:
// RLE v1 -- every value a literal varint (5 / 10 bytes) plus a header byte
// per 127 literals; RLE v2 -- at most 10 bytes per value for a one-value
// DIRECT run (2 header bytes + 8), less for every other run.
inline uint64_t rlev1_lane_cap(uint64_t chunk_size, uint32_t eb) {
    const uint64_t ne = chunk_size / 32u / eb;
    return (ne * (eb == 4 ? 5u : 10u) + ne / 64u + 16u + 3u) & ~3ull;
}
inline uint64_t rlev2_lane_cap(uint64_t chunk_size) {
    const uint64_t nv = chunk_size / 256u;
    return (nv * 11u + 64u + 3u) & ~3ull;
}

template <typename Kern>
gd_status_t run(Kern k1, const uint8_t* d_in, uint64_t n_bytes, uint64_t chunk_size, uint32_t param,
                uint64_t lane_cap, uint8_t* d_scratch, uint8_t* d_data, uint64_t* d_blk_off, uint64_t* d_col_len,
                uint32_t* d_status, cudaStream_t s) {
    const uint64_t nc = (n_bytes + chunk_size - 1) / chunk_size;
    const uint32_t grid1 = (uint32_t)((nc + NT / 32 - 1) / (NT / 32));
    k1<<<grid1, NT, 0, s>>>(d_in, n_bytes, (uint32_t)nc, chunk_size, param, d_scratch, (uint32_t)lane_cap,
                            d_col_len, d_blk_off + 1, d_status);
    offsets_kernel<<<1, 1024, 0, s>>>(d_blk_off, (uint32_t)nc);
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const uint64_t g3 = nc < (uint64_t)sms * 16u ? nc : (uint64_t)sms * 16u;
    interleave_kernel<<<(uint32_t)g3, NT, 0, s>>>(d_scratch, (uint32_t)lane_cap, d_col_len, d_blk_off,
                                                  (uint32_t)nc, d_data);
    return cudaGetLastError() == cudaSuccess ? GD_OK : GD_ERR_CUDA;
}

}  // namespace encd
}  // namespace gd

using namespace gd::encd;

extern "C" uint64_t gd_rlev1_encode_bound(uint64_t n_bytes, uint64_t chunk_size, uint32_t elem_bytes) {
    if (n_bytes == 0 || chunk_size == 0 || !(elem_bytes == 4 || elem_bytes == 8)) return 0;
    return (n_bytes + chunk_size - 1) / chunk_size * 32u * rlev1_lane_cap(chunk_size, elem_bytes);
}

extern "C" gd_status_t gd_rlev1_encode_device(const uint8_t* d_in, uint64_t n_bytes, uint64_t chunk_size,
                                              uint32_t comp_col_len, uint32_t elem_bytes, uint8_t* d_scratch,
                                              uint8_t* d_data, uint64_t* d_blk_off, uint64_t* d_col_len,
                                              uint32_t* d_status, gd_stream_t stream) {
    if (n_bytes == 0) return GD_OK;
    if (!d_in || !d_scratch || !d_data || !d_blk_off || !d_col_len) return GD_ERR_INVALID_ARG;
    if (!(elem_bytes == 4 || elem_bytes == 8) || n_bytes % elem_bytes) return GD_ERR_INVALID_ARG;
    if (comp_col_len == 0 || comp_col_len % elem_bytes) return GD_ERR_INVALID_ARG;
    if (chunk_size == 0 || chunk_size % (32ull * comp_col_len) || chunk_size > (1ull << 30))
        return GD_ERR_INVALID_ARG;
    if ((reinterpret_cast<uintptr_t>(d_in) % elem_bytes) || (reinterpret_cast<uintptr_t>(d_scratch) & 3u) ||
        (reinterpret_cast<uintptr_t>(d_data) & 3u))
        return GD_ERR_INVALID_ARG;
    if ((n_bytes + chunk_size - 1) / chunk_size > 0xffffffffull) return GD_ERR_UNSUPPORTED;
    // a lane of one value cannot be encoded (the writer starts from two)
    if (chunk_size / 32u / elem_bytes < 2) return GD_ERR_UNSUPPORTED;
    const uint64_t cap = rlev1_lane_cap(chunk_size, elem_bytes);
    const uint32_t wil = comp_col_len / elem_bytes;
    cudaStream_t s = (cudaStream_t)stream;
    if (elem_bytes == 4)
        return run(lane_encode_kernel<GD_CODEC_RLEV1, uint32_t>, d_in, n_bytes, chunk_size, wil, cap, d_scratch,
                   d_data, d_blk_off, d_col_len, d_status, s);
    return run(lane_encode_kernel<GD_CODEC_RLEV1, uint64_t>, d_in, n_bytes, chunk_size, wil, cap, d_scratch, d_data,
               d_blk_off, d_col_len, d_status, s);
}

extern "C" uint64_t gd_rlev2_encode_bound(uint64_t n_bytes, uint64_t chunk_size) {
    if (n_bytes == 0 || chunk_size == 0) return 0;
    return (n_bytes + chunk_size - 1) / chunk_size * 32u * rlev2_lane_cap(chunk_size);
}

extern "C" gd_status_t gd_rlev2_encode_device(const uint8_t* d_in, uint64_t n_bytes, uint64_t chunk_size,
                                              uint32_t read_unit, uint8_t* d_scratch, uint8_t* d_data,
                                              uint64_t* d_blk_off, uint64_t* d_col_len, uint32_t* d_status,
                                              gd_stream_t stream) {
    if (n_bytes == 0) return GD_OK;
    if (!d_in || !d_scratch || !d_data || !d_blk_off || !d_col_len) return GD_ERR_INVALID_ARG;
    if (read_unit == 0 || n_bytes % 8) return GD_ERR_INVALID_ARG;
    if (chunk_size == 0 || chunk_size % (256ull * read_unit) || chunk_size > (1ull << 30)) return GD_ERR_INVALID_ARG;
    if ((reinterpret_cast<uintptr_t>(d_in) & 7u) || (reinterpret_cast<uintptr_t>(d_scratch) & 3u) ||
        (reinterpret_cast<uintptr_t>(d_data) & 3u))
        return GD_ERR_INVALID_ARG;
    if ((n_bytes + chunk_size - 1) / chunk_size > 0xffffffffull) return GD_ERR_UNSUPPORTED;
    return run(lane_encode_kernel<GD_CODEC_RLEV2, int64_t>, d_in, n_bytes, chunk_size, read_unit,
               rlev2_lane_cap(chunk_size), d_scratch, d_data, d_blk_off, d_col_len, d_status, (cudaStream_t)stream);
}
