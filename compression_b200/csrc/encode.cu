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

// Block c = slots' words in rows; a block of NT threads per chunk.  Slot t's
// stream is scratch slot col_map[32c + t] of the chunk (LZSS: slots are
// length ranks) or slot t (col_map null).
__global__ void __launch_bounds__(NT) interleave_kernel(const uint8_t* __restrict__ scratch, uint32_t lane_cap,
                                                        const uint64_t* __restrict__ col_len,
                                                        const uint64_t* __restrict__ blk_off, uint32_t n_chunks,
                                                        uint8_t* __restrict__ data,
                                                        const uint8_t* __restrict__ col_map = nullptr) {
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
            const uint32_t st = col_map ? (col_map[(uint64_t)c * 32u + t] & 31u) : t;
            const uint32_t* src = src0 + (uint64_t)st * (lane_cap / 4u);
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

// ---------------------------------------------------------------------------
// LZSS interleaved container (lzss::compress_gpu, include/lzss/lzss_gpu2.h:
// 1915-2127; columns by compress_init_func / compress_func_new :330-707)
// ---------------------------------------------------------------------------
//
// Column q of a chunk is the chunk's bytes [128k + 4q, 128k + 4q + 4) for
// every k; each column is one token stream: a flag byte before every 8
// tokens (bit set = literal byte, clear = 2-byte match v = offset << 5 |
// (length - 3), offsets 1..2047 back into the column, lengths 3..34).  The
// greedy writer takes at every position the oldest of the longest matches in
// the 2048-byte history (find_match, lzss_gpu2.h:70-108), so a position's
// match depends only on the position: a warp per column stages the column in
// shared memory, indexes its 3-byte keys by hash bucket (positions ascending
// inside a bucket), and at each token checks the bucket's candidates 32 at a
// time, oldest first (one lane per candidate, the longest with the oldest
// winning ties), stopping at a 34-byte match.  A per-bucket cursor drops
// candidates older than the history as the walk advances.  Lane 0 writes the
// tokens into the column's scratch slot.  (Finding every position's match
// with a lane per position instead was 2.4x slower on Markov columns: their
// candidate lists are long, and serial per lane.)

constexpr uint32_t LZ_WPB = 4;      // columns (warps) per block
constexpr uint32_t LZ_NB = 512;     // hash buckets of 3-byte keys
constexpr uint32_t LZ_HIST = 2048, LZ_LOOK = 512, LZ_MAXM = 34, LZ_MINM = 3;

__host__ __device__ constexpr uint32_t a16(uint32_t x) { return (x + 15u) & ~15u; }
// column bytes (+64 zero pad) | positions by bucket | bucket starts | cursors
__host__ __device__ constexpr uint32_t lz_warp_smem(uint32_t L) {
    return a16(L + 64u) + a16(2u * L) + a16(2u * (LZ_NB + 1u)) + a16(2u * LZ_NB);
}
__device__ __forceinline__ uint32_t lz_key(const uint8_t* d, uint32_t p) {
    return ((uint32_t)d[p] << 16) | ((uint32_t)d[p + 1] << 8) | d[p + 2];
}
__device__ __forceinline__ uint32_t lz_hash(uint32_t key) { return (key * 2654435761u) >> 23; }  // 9 bits

__global__ void __launch_bounds__(LZ_WPB * 32) lzss_column_kernel(const uint8_t* __restrict__ in, uint64_t n_bytes,
                                                                  uint64_t chunk_size, uint32_t n_cols,
                                                                  uint8_t* __restrict__ scratch, uint32_t cap,
                                                                  uint32_t* __restrict__ raw_len, uint32_t wsm) {
    extern __shared__ __align__(16) uint8_t smem[];
    const uint32_t lane = lane_id(), wid = threadIdx.x >> 5;
    const uint32_t col = blockIdx.x * LZ_WPB + wid;  // 32 * chunk + column
    if (col >= n_cols) return;                        // warp-uniform
    const uint32_t q = col & 31u;
    const uint32_t L = (uint32_t)(chunk_size / 32u);
    uint8_t* d = smem + wid * wsm;
    uint16_t* pos = reinterpret_cast<uint16_t*>(d + a16(L + 64u));
    uint16_t* start = reinterpret_cast<uint16_t*>(reinterpret_cast<uint8_t*>(pos) + a16(2u * L));
    uint16_t* cursor = reinterpret_cast<uint16_t*>(reinterpret_cast<uint8_t*>(start) + a16(2u * (LZ_NB + 1u)));

    // ---- the column: word k = chunk bytes [128k + 4q, +4); zero past the input ----
    const uint64_t cb = (uint64_t)(col >> 5) * chunk_size;
    for (uint32_t k = lane; k < L / 4u; k += 32) {
        const uint64_t g = cb + 128ull * k + 4u * q;
        uint32_t w = 0;
        if (g + 4 <= n_bytes) {
            w = __ldg(reinterpret_cast<const uint32_t*>(in + g));
        } else {
            for (uint32_t b = 0; b < 4; ++b)
                if (g + b < n_bytes) w |= (uint32_t)__ldg(in + g + b) << (8u * b);
        }
        reinterpret_cast<uint32_t*>(d)[k] = w;
    }
    for (uint32_t i = L + lane; i < L + 64u; i += 32) d[i] = 0;
    for (uint32_t b = lane; b < LZ_NB; b += 32) cursor[b] = 0;
    __syncwarp();

    // ---- bucket index of the positions with a full key (p + 2 < L) ----
    const uint32_t np = L - 2u;
    for (uint32_t p0 = 0; p0 < np; p0 += 32) {  // counts (one leader per distinct bucket)
        const uint32_t p = p0 + lane;
        const uint32_t h = p < np ? lz_hash(lz_key(d, p)) : LZ_NB + lane;
        const uint32_t peers = __match_any_sync(GD_FULL_MASK, h);
        if (p < np && (peers & ((1u << lane) - 1u)) == 0) cursor[h] += __popc(peers);
        __syncwarp();
    }
    {
        constexpr uint32_t PER = LZ_NB / 32u;
        uint32_t v[PER], sum = 0;
#pragma unroll
        for (uint32_t i = 0; i < PER; ++i) {
            v[i] = cursor[lane * PER + i];
            sum += v[i];
        }
        uint32_t run = warp_incl_scan(sum) - sum;
#pragma unroll
        for (uint32_t i = 0; i < PER; ++i) {
            start[lane * PER + i] = (uint16_t)run;
            run += v[i];
        }
        if (lane == 31) start[LZ_NB] = (uint16_t)run;
    }
    __syncwarp();
    for (uint32_t b = lane; b < LZ_NB; b += 32) cursor[b] = 0;
    __syncwarp();
    for (uint32_t p0 = 0; p0 < np; p0 += 32) {  // scatter, ascending inside each bucket
        const uint32_t p = p0 + lane;
        const uint32_t h = p < np ? lz_hash(lz_key(d, p)) : LZ_NB + lane;
        const uint32_t peers = __match_any_sync(GD_FULL_MASK, h);
        if (p < np) pos[start[h] + cursor[h] + __popc(peers & ((1u << lane) - 1u))] = (uint16_t)p;
        __syncwarp();
        if (p < np && (peers & ((1u << lane) - 1u)) == 0) cursor[h] += __popc(peers);
        __syncwarp();
    }
    for (uint32_t b = lane; b < LZ_NB; b += 32) cursor[b] = start[b];
    __syncwarp();

    // ---- greedy token walk (warp-uniform), tokens written by lane 0 ----
    DevSink o{reinterpret_cast<uint32_t*>(scratch + (uint64_t)col * cap), 0u, cap, 0u};
    if (lane == 0) o.put(0);  // first flag byte
    uint32_t flag_pos = 0, flags = 0, blocks = 0, cur = 0;
    while (cur < L) {
        const uint32_t hist_count = cur < LZ_HIST ? cur : LZ_HIST;
        const uint32_t look = (L - cur) < LZ_LOOK ? (L - cur) : LZ_LOOK;
        uint32_t best_len = 0, best_pos = 0;
        if (look >= LZ_MINM && cur >= 3 && cur + 2 < L) {
            const uint32_t lo = cur - hist_count + 1;  // the oldest history entry (offset 0 is never a source)
            const uint32_t key = lz_key(d, cur), b = lz_hash(key);
            const uint32_t end = start[b + 1];
            uint32_t idx = cursor[b];
            while (idx < end && pos[idx] < lo) ++idx;
            __syncwarp();
            if (lane == 0) cursor[b] = (uint16_t)idx;
            for (uint32_t base = idx; base < end; base += 32) {
                const uint32_t j = base + lane;
                const uint32_t p = j < end ? pos[j] : 0xffffu;
                const bool valid = j < end && p + LZ_MINM <= cur;
                uint32_t f = 0;
                if (valid && lz_key(d, p) == key) {
                    uint32_t lim = cur - p;
                    lim = lim < look ? lim : look;
                    lim = lim < LZ_MAXM ? lim : LZ_MAXM;
                    f = 3;
                    while (f < lim && d[p + f] == d[cur + f]) ++f;
                }
                const uint32_t best = __reduce_max_sync(GD_FULL_MASK, f ? (f << 6) | (63u - lane) : 0u);
                if ((best >> 6) > best_len) {
                    best_len = best >> 6;
                    best_pos = pos[base + 63u - (best & 63u)];
                }
                if (best_len >= LZ_MAXM || __any_sync(GD_FULL_MASK, !valid)) break;
            }
        }
        if (best_len < LZ_MINM) {
            if (lane == 0) o.put(d[cur]);
            flags |= 1u << blocks;
            cur += 1;
        } else {
            const uint32_t v = ((cur - best_pos) << 5) | (best_len - LZ_MINM);
            if (lane == 0) {
                o.put((uint8_t)(v & 0xffu));
                o.put((uint8_t)(v >> 8));
            }
            cur += best_len;
        }
        if (++blocks == 8) {
            if (lane == 0) {
                o.set(flag_pos, (uint8_t)flags);
                flag_pos = o.n;
                o.put(0);  // the next flag byte is reserved even if no token follows
            }
            flags = 0;
            blocks = 0;
        }
    }
    if (lane == 0) {
        if (blocks != 0) o.set(flag_pos, (uint8_t)flags);
        o.flush();
        raw_len[col] = o.n <= cap ? o.n : 0xffffffffu;
    }
}

// A warp per chunk: slots are the columns by descending stream length (equal
// lengths: the higher column first, as the reference's stable ascending sort
// read backwards); col_map[32c + slot] = column, col_len in slot order, and
// the chunk's block size into blk_size[c].
__global__ void __launch_bounds__(NT) lzss_rank_kernel(const uint32_t* __restrict__ raw_len, uint32_t n_chunks,
                                                       uint64_t* __restrict__ col_len, uint8_t* __restrict__ col_map,
                                                       uint64_t* __restrict__ blk_size, uint32_t* __restrict__ status) {
    const uint32_t c = (blockIdx.x * NT + threadIdx.x) >> 5;
    const uint32_t q = lane_id();
    if (c >= n_chunks) return;  // warp-uniform
    const uint32_t r0 = raw_len[(uint64_t)c * 32u + q];
    const bool over = r0 == 0xffffffffu;
    const uint32_t len = over ? 0u : r0;
    uint32_t rank = 0;
#pragma unroll 8
    for (uint32_t o = 0; o < 32; ++o) {
        const uint32_t lo = __shfl_sync(GD_FULL_MASK, len, o);
        rank += (lo > len) || (lo == len && o > q);
    }
    col_map[(uint64_t)c * 32u + rank] = (uint8_t)q;
    col_len[(uint64_t)c * 32u + rank] = len;
    const uint32_t words = __reduce_add_sync(GD_FULL_MASK, (len + 3u) >> 2);
    const bool bad = __any_sync(GD_FULL_MASK, over);
    if (q == 0) {
        blk_size[c] = ((uint64_t)words * 4u + 127u) & ~127ull;
        put_status(status, c, bad ? (uint32_t)ST_OVERRUN : (uint32_t)ST_OK);
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
// LZSS column of L bytes: all literals, a flag byte per 8 tokens and the
// reserved one after the last group
inline uint64_t lzss_col_cap(uint64_t chunk_size) {
    const uint64_t L = chunk_size / 32u;
    return (L + L / 8u + 8u + 3u) & ~3ull;
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

extern "C" uint64_t gd_lzss_encode_bound(uint64_t n_bytes, uint64_t chunk_size) {
    if (n_bytes == 0 || chunk_size == 0) return 0;
    return (n_bytes + chunk_size - 1) / chunk_size * 32u * (lzss_col_cap(chunk_size) + 4u) + 16u;
}

extern "C" gd_status_t gd_lzss_encode_device(const uint8_t* d_in, uint64_t n_bytes, uint64_t chunk_size,
                                             uint8_t* d_scratch, uint8_t* d_data, uint64_t* d_blk_off,
                                             uint64_t* d_col_len, uint8_t* d_col_map, uint32_t* d_status,
                                             gd_stream_t stream) {
    if (n_bytes == 0) return GD_OK;
    if (!d_in || !d_scratch || !d_data || !d_blk_off || !d_col_len || !d_col_map) return GD_ERR_INVALID_ARG;
    if (chunk_size == 0 || chunk_size % 128u || chunk_size > 128u * 1024u) return GD_ERR_INVALID_ARG;
    if ((reinterpret_cast<uintptr_t>(d_in) & 3u) || (reinterpret_cast<uintptr_t>(d_scratch) & 3u) ||
        (reinterpret_cast<uintptr_t>(d_data) & 3u))
        return GD_ERR_INVALID_ARG;
    const uint64_t nc = (n_bytes + chunk_size - 1) / chunk_size;
    if (nc * 32u > 0xffffffffull) return GD_ERR_UNSUPPORTED;
    const uint64_t cap = lzss_col_cap(chunk_size);
    uint32_t* raw_len = reinterpret_cast<uint32_t*>(d_scratch + nc * 32u * cap);
    const uint32_t L = (uint32_t)(chunk_size / 32u);
    const uint32_t wsm = lz_warp_smem(L);
    cudaStream_t s = (cudaStream_t)stream;
    cudaFuncSetAttribute(lzss_column_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, LZ_WPB * wsm);
    const uint32_t ncol = (uint32_t)(nc * 32u);
    lzss_column_kernel<<<(ncol + LZ_WPB - 1) / LZ_WPB, LZ_WPB * 32, LZ_WPB * wsm, s>>>(
        d_in, n_bytes, chunk_size, ncol, d_scratch, (uint32_t)cap, raw_len, wsm);
    lzss_rank_kernel<<<(uint32_t)((nc + NT / 32 - 1) / (NT / 32)), NT, 0, s>>>(raw_len, (uint32_t)nc, d_col_len,
                                                                              d_col_map, d_blk_off + 1, d_status);
    offsets_kernel<<<1, 1024, 0, s>>>(d_blk_off, (uint32_t)nc);
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const uint64_t g3 = nc < (uint64_t)sms * 16u ? nc : (uint64_t)sms * 16u;
    interleave_kernel<<<(uint32_t)g3, NT, 0, s>>>(d_scratch, (uint32_t)cap, d_col_len, d_blk_off, (uint32_t)nc, d_data,
                                                  d_col_map);
    return cudaGetLastError() == cudaSuccess ? GD_OK : GD_ERR_CUDA;
}

// ---------------------------------------------------------------------------
// Byte-RLE flag container (brle_trans::compress_gpu, include/brle/brle_trans.h:
// 563-660; column streams by compress_func :437-562)
// ---------------------------------------------------------------------------
//
// Same column split, ranking and interleave as the LZSS container; only the
// column stream differs: maximal runs of equal bytes, a run of 3 or more as a
// run item (count byte, value byte; flag bit 0), a shorter one as that many
// literal items (flag bit 1), a flag byte before every 8 items (LSB first)
// and, after the 8th item of a group, the next flag byte reserved (0 if no
// item follows) -- except after the column's last item when that is a run,
// which the reference writes without counting it (brle_trans.h:529-536).  A thread per column: the warp's 32 lanes are one chunk's
// 32 columns, so each step reads 128 contiguous input bytes.  Output bytes
// gather in a word register; a group's flag byte goes into that register when
// its word is still open, else it is stored over the 0 already written.
// Run counts fit the count byte because a column holds at most 252 bytes.

__global__ void __launch_bounds__(NT) brle_trans_column_kernel(const uint8_t* __restrict__ in, uint64_t n_bytes,
                                                               uint64_t chunk_size, uint32_t n_cols,
                                                               uint8_t* __restrict__ scratch, uint32_t cap,
                                                               uint32_t* __restrict__ raw_len) {
    const uint32_t col = blockIdx.x * NT + threadIdx.x;
    if (col >= n_cols) return;
    const uint64_t c = col >> 5;
    const uint32_t q = col & 31u;
    const uint32_t L = (uint32_t)(chunk_size / 32u);
    const uint64_t base = c * chunk_size + 4u * q;
    uint8_t* slot = scratch + (uint64_t)col * cap;
    uint32_t* wslot = reinterpret_cast<uint32_t*>(slot);
    uint32_t pos = 1, hpos = 0, items = 0, flags = 0, wbuf = 0;  // byte 0: the first flag byte
    auto put = [&](uint32_t b) {
        wbuf |= b << (8u * (pos & 3u));
        if ((++pos & 3u) == 0) {
            wslot[(pos >> 2) - 1u] = wbuf;
            wbuf = 0;
        }
    };
    auto set_flag = [&]() {
        if (hpos >= (pos & ~3u))
            wbuf |= flags << (8u * (hpos & 3u));
        else
            slot[hpos] = (uint8_t)flags;
    };
    auto item_done = [&]() {
        if (++items == 8u) {
            set_flag();
            flags = 0;
            items = 0;
            hpos = pos;
            put(0u);
        }
    };
    auto emit = [&](uint32_t v, uint32_t run, bool last) {
        if (run >= 3u) {
            put(run);
            put(v);
            if (!last) item_done();  // the column's last run is written uncounted
        } else {
            for (uint32_t k = 0; k < run; ++k) {
                flags |= 1u << items;
                put(v);
                item_done();
            }
        }
    };
    uint32_t cur = 0, run = 0;
    for (uint32_t k = 0; k < L / 4u; ++k) {
        const uint64_t at = base + 128ull * k;
        uint32_t w = 0;
        if (at + 4u <= n_bytes) {
            w = *reinterpret_cast<const uint32_t*>(in + at);
        } else {
            for (uint32_t b = 0; b < 4u; ++b)
                if (at + b < n_bytes) w |= (uint32_t)in[at + b] << (8u * b);
        }
#pragma unroll
        for (uint32_t b = 0; b < 4u; ++b) {
            const uint32_t x = (w >> (8u * b)) & 0xffu;
            if (run && x == cur) {
                ++run;
            } else {
                if (run) emit(cur, run, false);
                cur = x;
                run = 1;
            }
        }
    }
    if (run) emit(cur, run, true);
    if (items) set_flag();
    if (pos & 3u) wslot[pos >> 2] = wbuf;
    raw_len[col] = pos;
}

extern "C" uint64_t gd_brle_trans_encode_bound(uint64_t n_bytes, uint64_t chunk_size) {
    if (n_bytes == 0 || chunk_size == 0) return 0;
    return (n_bytes + chunk_size - 1) / chunk_size * 32u * (lzss_col_cap(chunk_size) + 4u) + 16u;
}

extern "C" gd_status_t gd_brle_trans_encode_device(const uint8_t* d_in, uint64_t n_bytes, uint64_t chunk_size,
                                                   uint8_t* d_scratch, uint8_t* d_data, uint64_t* d_blk_off,
                                                   uint64_t* d_col_len, uint8_t* d_col_map, uint32_t* d_status,
                                                   gd_stream_t stream) {
    if (n_bytes == 0) return GD_OK;
    if (!d_in || !d_scratch || !d_data || !d_blk_off || !d_col_len || !d_col_map) return GD_ERR_INVALID_ARG;
    if (chunk_size == 0 || chunk_size % 128u || chunk_size / 32u > 252u) return GD_ERR_INVALID_ARG;
    if ((reinterpret_cast<uintptr_t>(d_in) & 3u) || (reinterpret_cast<uintptr_t>(d_scratch) & 3u) ||
        (reinterpret_cast<uintptr_t>(d_data) & 3u))
        return GD_ERR_INVALID_ARG;
    const uint64_t nc = (n_bytes + chunk_size - 1) / chunk_size;
    if (nc * 32u > 0xffffffffull) return GD_ERR_UNSUPPORTED;
    const uint64_t cap = lzss_col_cap(chunk_size);
    uint32_t* raw_len = reinterpret_cast<uint32_t*>(d_scratch + nc * 32u * cap);
    cudaStream_t s = (cudaStream_t)stream;
    const uint32_t ncol = (uint32_t)(nc * 32u);
    brle_trans_column_kernel<<<(ncol + NT - 1) / NT, NT, 0, s>>>(d_in, n_bytes, chunk_size, ncol, d_scratch,
                                                                 (uint32_t)cap, raw_len);
    lzss_rank_kernel<<<(uint32_t)((nc + NT / 32 - 1) / (NT / 32)), NT, 0, s>>>(raw_len, (uint32_t)nc, d_col_len,
                                                                              d_col_map, d_blk_off + 1, d_status);
    offsets_kernel<<<1, 1024, 0, s>>>(d_blk_off, (uint32_t)nc);
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const uint64_t g3 = nc < (uint64_t)sms * 16u ? nc : (uint64_t)sms * 16u;
    interleave_kernel<<<(uint32_t)g3, NT, 0, s>>>(d_scratch, (uint32_t)cap, d_col_len, d_blk_off, (uint32_t)nc, d_data,
                                                  d_col_map);
    return cudaGetLastError() == cudaSuccess ? GD_OK : GD_ERR_CUDA;
}
