// brle_enc.cu -- byte-RLE (brle.h container) encoder for sm_100a.
//
// The writer of the container the brle decoder reads:
// [u32 n_ptr][u64 ptr[n_ptr]][u64 total][chunk token streams], chunk c's
// tokens encoding input bytes [c*chunk_size, ...) with the greedy encoder of
// brle::encode (include/brle/brle.h:129-230, non-lookahead path): a literal
// token (c - 127 bytes, c > 127) holds up to 128 bytes and is cut where three
// equal bytes start a run token (c <= 127: c + 3 copies, up to 130).  The
// reference runs one thread per chunk (brle.h:242-248).
//
// Here a block of 256 threads encodes a chunk.  The greedy encoder
// resynchronises: after a maximal run of L >= 5 equal bytes with
// L mod 130 not in {1,2,3,4}, the encoder's state before the next (different)
// byte is "run token pending" or "nothing pending", whatever came before the
// run -- a run token starts at offset 0, 1 or 2 of the run (1 or 2 when a
// 128-byte literal is cut inside it) and the run then leaves (L - offset) mod
// 130 bytes, never 1 or 2, which would be a pending literal.  So the next
// byte always starts a fresh literal, and encoding from there with an empty
// state gives the serial encoder's tokens.  Thread k finds the first such
// point in its 1/256 of the chunk (scanning only runs that start in its
// range), owns the region up to the next thread's point, and encodes it
// serially into its own slot of a scratch area; a block scan of the region
// sizes places the regions, and two more launches turn the chunk sizes into
// ptr[] and copy the tokens into place.  Incompressible chunks have no such
// points and fall back to one thread, as in the reference.
#include "gd_common.cuh"

namespace gd {
namespace brlee {

constexpr int NT = 256;
constexpr uint32_t NONE = 0xffffffffu;

// Scratch area of a chunk: region k starts at
//   off(P_k) = (P_k + P_k / 128 + 8k + 3) & ~3,
// and a region of R bytes encodes into at most R + R/128 + 2 bytes, so the
// slots of consecutive owners never overlap.
__host__ __device__ constexpr uint64_t area_bytes(uint64_t chunk) { return (chunk + chunk / 128 + 8ull * NT + 31) & ~15ull; }

struct WordSink {
    uint32_t* w;
    uint32_t n, cur;
    __device__ __forceinline__ void put(uint32_t b) {
        cur |= (b & 0xffu) << (8u * (n & 3u));
        ++n;
        if ((n & 3u) == 0) {
            w[(n >> 2) - 1] = cur;
            cur = 0;
        }
    }
    __device__ __forceinline__ void flush() {
        if (n & 3u) w[n >> 2] = cur;
    }
};

// The greedy encoder (brle.h:129-230) over x[P, Pn) from an empty state; the
// literal buffer is always the input bytes [start, i), so it is not copied.
__device__ uint32_t encode_region(const uint8_t* __restrict__ x, uint32_t P, uint32_t Pn, WordSink& o) {
    uint32_t num = 0, tail = 0, start = 0, val = 0, prev = 0;
    bool rep = false;
    auto lit = [&](uint32_t s, uint32_t n) {
        o.put(n + 127u);
        for (uint32_t j = s; j < s + n; ++j) o.put(__ldg(x + j));
    };
    for (uint32_t i = P; i < Pn; ++i) {
        const uint32_t c = __ldg(x + i);
        if (num == 0) {
            start = i;
            num = 1;
            tail = 1;
            rep = false;
        } else if (rep) {
            if (c == val) {
                if (++num == 130u) {
                    o.put(127u);
                    o.put(val);
                    num = 0;
                    rep = false;
                }
            } else {
                o.put(num - 3u);
                o.put(val);
                rep = false;
                start = i;
                num = 1;
                tail = 1;
            }
        } else {
            tail = (c == prev) ? tail + 1 : 1;
            if (tail == 3) {
                if (num + 1 != 3) lit(start, num - 2);
                start = i - 2;
                num = 3;
                rep = true;
                val = c;
            } else if (++num == 128u) {
                lit(start, 128u);
                num = 0;
            }
        }
        prev = c;
    }
    if (num) {
        if (rep) {
            o.put(num - 3u);
            o.put(val);
        } else {
            lit(start, num);
        }
    }
    return o.n;
}

// Launch 1: a block per chunk.  tab[c*NT + k] = (slot offset, bytes, output
// offset in the chunk) of thread k's region; csize[c + 1] = chunk c's bytes.
__global__ void __launch_bounds__(NT) regions_kernel(const uint8_t* __restrict__ in, uint64_t n_bytes,
                                                     uint64_t chunk_size, uint32_t n_chunks,
                                                     uint8_t* __restrict__ area, uint64_t area_stride,
                                                     uint4* __restrict__ tab, uint64_t* __restrict__ csize) {
    __shared__ uint32_t s_P[NT];
    __shared__ uint32_t s_tmp[NT / 32 + 1];
    const uint32_t k = threadIdx.x;
    for (uint32_t c = blockIdx.x; c < n_chunks; c += gridDim.x) {
        const uint64_t cb = (uint64_t)c * chunk_size;
        const uint32_t len = (uint32_t)(n_bytes - cb < chunk_size ? n_bytes - cb : chunk_size);
        const uint8_t* x = in + cb;
        // ---- this thread's resynchronisation point ----
        uint32_t P = NONE;
        if (k == 0) {
            P = 0;
        } else {
            const uint32_t a = (uint32_t)((uint64_t)k * len / NT), b = (uint32_t)((uint64_t)(k + 1) * len / NT);
            uint32_t s = a ? a : 1u;  // position 0 is thread 0's
            while (s < b && __ldg(x + s) == __ldg(x + s - 1)) ++s;  // the run that began before a
            while (s < b) {                                            // runs that begin in [a, b)
                const uint32_t v = __ldg(x + s);
                uint32_t e = s + 1;
                while (e < len && __ldg(x + e) == v) ++e;
                if (e >= len) break;  // the chunk's last run: nothing follows it
                const uint32_t L = e - s, r = L % 130u;
                if (L >= 5 && (r == 0 || r >= 5)) {
                    P = e;
                    break;
                }
                s = e;
            }
        }
        s_P[k] = P;
        __syncthreads();
        // ---- encode the owned region [P, next owner's point) ----
        uint32_t bytes = 0, off = 0;
        if (P != NONE) {
            uint32_t Pn = len;
            for (uint32_t j = k + 1; j < (uint32_t)NT; ++j)
                if (s_P[j] != NONE) {
                    Pn = s_P[j];
                    break;
                }
            off = (P + P / 128u + 8u * k + 3u) & ~3u;
            WordSink o{reinterpret_cast<uint32_t*>(area + (uint64_t)c * area_stride + off), 0u, 0u};
            bytes = encode_region(x, P, Pn, o);
            o.flush();
        }
        uint32_t total;
        const uint32_t dst = block_excl_scan<NT>(bytes, s_tmp, &total);
        tab[(uint64_t)c * NT + k] = make_uint4(off, bytes, dst, 0u);
        if (k == 0) csize[c + 1] = total;
        __syncthreads();  // s_P and s_tmp are reused by the next chunk
    }
}

// Launch 2: ptr[] = prefix sums of the chunk sizes (csize[1..n] in place),
// and the container header: n_ptr, ptr[], the input size; *out_bytes = the
// container's length.  One block of 1024 threads.
__global__ void __launch_bounds__(1024) header_kernel(uint64_t* __restrict__ csize, uint32_t n, uint64_t n_bytes,
                                                      uint8_t* __restrict__ out, uint64_t* __restrict__ out_bytes) {
    __shared__ uint64_t tmp[1024 / 32 + 1];
    const uint64_t per = ((uint64_t)n + 1023u) / 1024u;
    const uint64_t b = min((uint64_t)n, threadIdx.x * per), e = min((uint64_t)n, b + per);
    uint64_t sum = 0;
    for (uint64_t i = b; i < e; ++i) sum += csize[1 + i];
    uint64_t tot;
    uint64_t acc = block_excl_scan64<1024>(sum, tmp, &tot);
    // ptr values sit at out + 4 + 8i: 4-byte aligned, so two 32-bit stores each
    uint32_t* o32 = reinterpret_cast<uint32_t*>(out + 4);
    for (uint64_t i = b; i < e; ++i) {
        acc += csize[1 + i];
        csize[1 + i] = acc;
        o32[2 * (i + 1)] = (uint32_t)acc;
        o32[2 * (i + 1) + 1] = (uint32_t)(acc >> 32);
    }
    if (threadIdx.x == 0) {
        csize[0] = 0;
        reinterpret_cast<uint32_t*>(out)[0] = n + 1;
        o32[0] = 0;
        o32[1] = 0;
        o32[2 * (n + 1)] = (uint32_t)n_bytes;
        o32[2 * (n + 1) + 1] = (uint32_t)(n_bytes >> 32);
        *out_bytes = 4ull + 8ull * (n + 1) + 8ull + tot;
    }
}

// Launch 3: a block per chunk copies its regions' tokens to the container.
__global__ void __launch_bounds__(NT) place_kernel(const uint8_t* __restrict__ area, uint64_t area_stride,
                                                   const uint4* __restrict__ tab,
                                                   const uint64_t* __restrict__ ptr, uint32_t n_chunks,
                                                   uint8_t* __restrict__ data) {
    __shared__ uint32_t s_dst[NT], s_src[NT];
    for (uint32_t c = blockIdx.x; c < n_chunks; c += gridDim.x) {
        const uint4 t = tab[(uint64_t)c * NT + threadIdx.x];
        s_dst[threadIdx.x] = t.z;
        s_src[threadIdx.x] = t.x;
        __syncthreads();
        const uint64_t p0 = ptr[c];
        const uint32_t total = (uint32_t)(ptr[c + 1] - p0);
        const uint8_t* a = area + (uint64_t)c * area_stride;
        uint8_t* d = data + p0;
        for (uint32_t i = threadIdx.x; i < total; i += NT) {
            // the last region whose output starts at or before i (empty
            // regions start where the next one does, so this one holds i)
            uint32_t r = 0;
#pragma unroll
            for (uint32_t step = NT / 2; step; step >>= 1)
                if (s_dst[r + step] <= i) r += step;
            d[i] = a[s_src[r] + (i - s_dst[r])];
        }
        __syncthreads();
    }
}

}  // namespace brlee
}  // namespace gd

using namespace gd::brlee;

extern "C" uint64_t gd_brle_encode_scratch_bytes(uint64_t n_bytes, uint64_t chunk_size) {
    if (n_bytes == 0 || chunk_size == 0) return 0;
    const uint64_t nc = (n_bytes - 1) / chunk_size + 1;
    const uint64_t cs = chunk_size < n_bytes ? chunk_size : n_bytes;
    return nc * area_bytes(cs) + nc * NT * 16ull + 8ull * (nc + 1) + 64;
}

extern "C" gd_status_t gd_brle_encode_device(const uint8_t* d_in, uint64_t n_bytes, uint64_t chunk_size,
                                             uint8_t* d_scratch, uint8_t* d_out, uint64_t* d_out_bytes,
                                             gd_stream_t stream) {
    if (n_bytes == 0 || chunk_size == 0) return GD_ERR_INVALID_ARG;
    if (!d_in || !d_scratch || !d_out || !d_out_bytes) return GD_ERR_INVALID_ARG;
    if (chunk_size > (1ull << 30) || (reinterpret_cast<uintptr_t>(d_scratch) & 15u) ||
        (reinterpret_cast<uintptr_t>(d_out) & 3u))
        return GD_ERR_INVALID_ARG;
    const uint64_t nc = (n_bytes - 1) / chunk_size + 1;
    if (nc >= 0xffffffffull) return GD_ERR_UNSUPPORTED;
    const uint64_t cs = chunk_size < n_bytes ? chunk_size : n_bytes;
    const uint64_t stride = area_bytes(cs);
    uint8_t* area = d_scratch;
    uint4* tab = reinterpret_cast<uint4*>(d_scratch + nc * stride);
    uint64_t* csize = reinterpret_cast<uint64_t*>(d_scratch + nc * stride + nc * NT * 16ull);
    cudaStream_t s = (cudaStream_t)stream;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const uint32_t grid = (uint32_t)(nc < (uint64_t)sms * 8u ? nc : (uint64_t)sms * 8u);
    regions_kernel<<<grid, NT, 0, s>>>(d_in, n_bytes, chunk_size, (uint32_t)nc, area, stride, tab, csize);
    header_kernel<<<1, 1024, 0, s>>>(csize, (uint32_t)nc, n_bytes, d_out, d_out_bytes);
    place_kernel<<<grid, NT, 0, s>>>(area, stride, tab, csize, (uint32_t)nc, d_out + 4 + 8 * (nc + 1) + 8);
    return cudaGetLastError() == cudaSuccess ? GD_OK : GD_ERR_CUDA;
}
