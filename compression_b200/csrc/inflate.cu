// inflate.cu -- Deflate / zlib inflate kernels for sm_100a: one warp per
// stream (the warp-level decoder is in inflate.cuh), with offset-array and
// cuDF-descriptor front ends.
#include "inflate.cuh"

namespace gd {
namespace infl {

// Chunk sources: offset arrays (gd_inflate) or cuDF-style descriptors.
struct OffsetChunks {
    const uint8_t* data;
    const uint64_t* comp_off;
    const uint64_t* comp_len;
    const uint64_t* out_off;
    uint8_t* out;
    uint32_t* status;
    static constexpr bool exact = true;  // output size is known exactly
    __device__ bool get(uint32_t c, const uint8_t*& src, uint64_t& slen, uint8_t*& dst, uint64_t& dlen) const {
        src = data + comp_off[c];
        slen = comp_len[c];
        const uint64_t o0 = out_off[c], o1 = out_off[c + 1];
        dst = out + o0;
        dlen = o1 - o0;
        return o1 >= o0;
    }
    __device__ void put(uint32_t c, uint32_t err, uint64_t) const { put_status(status, c, err); }
};

struct CudfChunks {
    const gd_inflate_input* in;
    gd_inflate_status* st;
    static constexpr bool exact = false;  // dstSize is a capacity
    __device__ bool get(uint32_t c, const uint8_t*& src, uint64_t& slen, uint8_t*& dst, uint64_t& dlen) const {
        src = static_cast<const uint8_t*>(in[c].srcDevice);
        slen = in[c].srcSize;
        dst = static_cast<uint8_t*>(in[c].dstDevice);
        dlen = in[c].dstSize;
        return true;
    }
    __device__ void put(uint32_t c, uint32_t err, uint64_t written) const {
        st[c].bytes_written = written;
        st[c].status = err ? 1u : 0u;
        st[c].reserved = 0;
    }
};

// NW warps per block, one stream per warp; WIN: output window (see
// WarpSmemT).  Blocks are handed out by the hardware in launch order, so
// `order` (longest first, say) is also the order streams start in.
template <class Chunks, uint32_t WIN, int NW>
__global__ void __launch_bounds__(NW * 32) inflate_kernel(Chunks ch, uint32_t n_chunks, int zlib_hdr,
                                                         const uint32_t* __restrict__ order) {
    extern __shared__ __align__(16) uint8_t smem_raw[];
    const uint32_t wid = threadIdx.x >> 5;
    const uint32_t slot = blockIdx.x * NW + wid;
    if (slot >= n_chunks) return;
    const uint32_t chunk = order ? order[slot] : slot;
    WarpSmemT<WIN>& S = *reinterpret_cast<WarpSmemT<WIN>*>(smem_raw + wid * sizeof(WarpSmemT<WIN>));
    const uint8_t* src;
    uint8_t* dst;
    uint64_t clen64, olen64;
    uint32_t err = ch.get(chunk, src, clen64, dst, olen64) ? ST_OK : ST_CORRUPT;
    if (olen64 > 0xffffffffull || clen64 > 0xffffffffull) err = ST_CORRUPT;
    uint32_t fin = 0;
    if (err == ST_OK) err = stream_warp_impl<WIN>(src, (uint32_t)clen64, dst, (uint32_t)olen64, zlib_hdr, S, &fin);
    if (err == ST_OK && Chunks::exact && fin != (uint32_t)olen64) err = ST_CORRUPT;
    if (lane_id() == 0) ch.put(chunk, err, err == ST_OK ? fin : 0);
}

// Reader/writer pairs: NP pairs per block, warps 2i (decoder) and 2i+1
// (writer) share stream i's state and hand batches over through it.
template <class Chunks, uint32_t WIN, int NP, uint32_t RB = IRING, uint32_t DB = LBITS, uint32_t NL = NLIT,
          uint32_t NC = NCMD>
__global__ void __launch_bounds__(NP * 64) inflate_pair_kernel(Chunks ch, uint32_t n_chunks, int zlib_hdr,
                                                              const uint32_t* __restrict__ order,
                                                              uint32_t spin_limit, uint32_t writer_stop) {
    using SmemT = WarpSmemT<WIN, 2, RB, DB, NL, NC>;
    extern __shared__ __align__(16) uint8_t smem_raw[];
    const uint32_t wid = threadIdx.x >> 5, pair = wid >> 1;
    const uint32_t slot = blockIdx.x * NP + pair;
    if (slot >= n_chunks) return;  // both warps of the pair leave together
    const uint32_t chunk = order ? order[slot] : slot;
    SmemT& S = *reinterpret_cast<SmemT*>(smem_raw + pair * sizeof(SmemT));
    const uint8_t* src;
    uint8_t* dst;
    uint64_t clen64, olen64;
    uint32_t err = ch.get(chunk, src, clen64, dst, olen64) ? ST_OK : ST_CORRUPT;
    if (olen64 > 0xffffffffull || clen64 > 0xffffffffull) err = ST_CORRUPT;
    if (err != ST_OK) {  // decided identically by both warps: neither enters the hand-off
        if ((wid & 1u) == 0 && lane_id() == 0) ch.put(chunk, err, 0);
        return;
    }
    if (threadIdx.x == 64 * pair) {
        S.produced = 0;
        S.consumed = 0;
    }
    // counters cleared before either warp of the pair uses them: a barrier of
    // the pair's 64 threads, reached unconditionally by both warps
    asm volatile("bar.sync %0, 64;" ::"r"(1u + pair) : "memory");
    if (wid & 1u) {
        const uint32_t werr = stream_pair_writer<WIN, RB, DB, NL, NC>(S, src, dst, spin_limit, writer_stop);
        if (werr != ST_OK && lane_id() == 0) ch.put(chunk, werr, 0);
        return;
    }
    uint32_t fin = 0;
    err = stream_warp_impl<WIN, 2, RB, DB, NL, NC>(src, (uint32_t)clen64, dst, (uint32_t)olen64, zlib_hdr, S, &fin,
                                                   spin_limit);
    if (err == ST_OK && Chunks::exact && fin != (uint32_t)olen64) err = ST_CORRUPT;
    if (lane_id() == 0) ch.put(chunk, err, err == ST_OK ? fin : 0);
}

}  // namespace infl
}  // namespace gd

namespace {
__global__ void copy_uncompressed_kernel(const gd_inflate_input* in, int count) {
    const int c = blockIdx.x;
    if (c >= count) return;
    const uint8_t* s = static_cast<const uint8_t*>(in[c].srcDevice);
    uint8_t* d = static_cast<uint8_t*>(in[c].dstDevice);
    const uint64_t n = min(in[c].srcSize, in[c].dstSize);
    for (uint64_t i = threadIdx.x; i < n; i += blockDim.x) d[i] = s[i];
}

template <class Chunks, uint32_t WIN, int NW>
gd_status_t launch_cfg(const Chunks& ch, uint32_t n, int zlib_hdr, const uint32_t* order, cudaStream_t s) {
    using namespace gd::infl;
    const uint32_t smem = NW * (uint32_t)sizeof(WarpSmemT<WIN>);
    static bool attr_set = false;  // benign race: the attribute call is idempotent
    if (!attr_set) {
        if (cudaFuncSetAttribute(inflate_kernel<Chunks, WIN, NW>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 smem) != cudaSuccess)
            return GD_ERR_CUDA;
        attr_set = true;
    }
    const uint32_t grid = (n + NW - 1) / NW;
    inflate_kernel<Chunks, WIN, NW><<<grid, NW * 32, smem, s>>>(ch, n, zlib_hdr, order);
    return cudaGetLastError() == cudaSuccess ? GD_OK : GD_ERR_CUDA;
}

template <class Chunks, uint32_t WIN, int NP, uint32_t RB = gd::infl::IRING, uint32_t DB = gd::infl::LBITS,
          uint32_t NL = gd::infl::NLIT, uint32_t NC = gd::infl::NCMD>
gd_status_t launch_pair(const Chunks& ch, uint32_t n, int zlib_hdr, const uint32_t* order, cudaStream_t s) {
    using namespace gd::infl;
    const uint32_t smem = NP * (uint32_t)sizeof(WarpSmemT<WIN, 2, RB, DB, NL, NC>);
    auto kern = inflate_pair_kernel<Chunks, WIN, NP, RB, DB, NL, NC>;
    static bool attr_set = false;  // benign race: the attribute call is idempotent
    if (!attr_set) {
        if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess)
            return GD_ERR_CUDA;
        attr_set = true;
    }
    const uint32_t grid = (n + NP - 1) / NP;
    const int spin = gd_tune_get(GD_TUNE_INFLATE_PAIR_SPIN);
    const int stop = gd_tune_get(GD_TUNE_INFLATE_WRITER_STOP);
    kern<<<grid, NP * 64, smem, s>>>(ch, n, zlib_hdr, order, spin > 0 ? (uint32_t)spin : PAIR_SPIN_LIMIT,
                                     stop > 0 ? (uint32_t)stop : 0u);
    return cudaGetLastError() == cudaSuccess ? GD_OK : GD_ERR_CUDA;
}

// Launch configuration (GD_TUNE_INFLATE_VARIANT): 1 / 2 = one warp per
// stream without a window, 2 / 4 warps per block; 3 = one warp per stream
// with a window; 4 / 5 = decoder/writer warp pairs without a window (copies
// read the output), 2 / 4 pairs per block; 6 = one decoder/writer pair per
// block with a 32 KiB shared window; 7 - 13 = pairs with a 16 / 8 / 4 KiB
// window (nearer copies from shared memory, farther ones from the output)
// and smaller rings, distance tables and batches, so that 7 to 15 pairs fit
// on an SM; 0 (default) = 12 for at least 4 streams per SM, else 6.
template <class Chunks>
gd_status_t launch_inflate(const Chunks& ch, uint32_t n, int zlib_hdr, const uint32_t* order, cudaStream_t s) {
    int v = gd_tune_get(GD_TUNE_INFLATE_VARIANT);
    if (v == 0) {
        // many streams: throughput, i.e. more pairs per SM (no window); few:
        // the fastest single stream (window)
        int dev = 0, sms = 148;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        v = n >= 4u * (uint32_t)sms ? 12 : 6;
    }
    switch (v) {
        case 1: return launch_cfg<Chunks, 0, 2>(ch, n, zlib_hdr, order, s);
        case 2: return launch_cfg<Chunks, 0, 4>(ch, n, zlib_hdr, order, s);
        case 3: return launch_cfg<Chunks, 32768, 1>(ch, n, zlib_hdr, order, s);
        case 4: return launch_pair<Chunks, 0, 2>(ch, n, zlib_hdr, order, s);
        case 5: return launch_pair<Chunks, 0, 4>(ch, n, zlib_hdr, order, s);
        case 7: return launch_pair<Chunks, 16384, 1, 2048, 8, 1024, 128>(ch, n, zlib_hdr, order, s);
        case 8: return launch_pair<Chunks, 16384, 2, 2048, 8, 1024, 128>(ch, n, zlib_hdr, order, s);
        case 9: return launch_pair<Chunks, 8192, 1, 2048, 8, 1024, 128>(ch, n, zlib_hdr, order, s);
        case 10: return launch_pair<Chunks, 4096, 1, 2048, 8, 1024, 128>(ch, n, zlib_hdr, order, s);
        case 11: return launch_pair<Chunks, 8192, 1, 1024, 8, 512, 64>(ch, n, zlib_hdr, order, s);
        case 12: return launch_pair<Chunks, 4096, 1, 1024, 8, 512, 64>(ch, n, zlib_hdr, order, s);
        case 13: return launch_pair<Chunks, 4096, 2, 1024, 8, 512, 64>(ch, n, zlib_hdr, order, s);
        case 14: return launch_pair<Chunks, 2048, 1, 1024, 8, 512, 64>(ch, n, zlib_hdr, order, s);
        default: return launch_pair<Chunks, 32768, 1>(ch, n, zlib_hdr, order, s);
    }
}
}  // namespace

extern "C" gd_status_t gd_inflate(const uint8_t* d_data, const uint64_t* d_comp_off, const uint64_t* d_comp_len,
                                  const uint64_t* d_out_off, uint32_t n_chunks, int zlib_header, uint8_t* d_out,
                                  uint32_t* d_status, gd_stream_t stream) {
    if (n_chunks == 0) return GD_OK;
    if (!d_data || !d_comp_off || !d_comp_len || !d_out_off || !d_out) return GD_ERR_INVALID_ARG;
    // compressed words are fetched as aligned 16-byte loads from the data base
    if (reinterpret_cast<uintptr_t>(d_data) & 15u) return GD_ERR_INVALID_ARG;
    gd::infl::OffsetChunks ch{d_data, d_comp_off, d_comp_len, d_out_off, d_out, d_status};
    return launch_inflate(ch, n_chunks, zlib_header, nullptr, (cudaStream_t)stream);
}

// Same, with chunks visited in the order given by d_order (a permutation of
// 0..n_chunks-1); used by the scheduler to start long chunks first.
extern "C" gd_status_t gd_inflate_ordered(const uint8_t* d_data, const uint64_t* d_comp_off,
                                          const uint64_t* d_comp_len, const uint64_t* d_out_off, uint32_t n_chunks,
                                          int zlib_header, uint8_t* d_out, uint32_t* d_status,
                                          const uint32_t* d_order, gd_stream_t stream) {
    if (n_chunks == 0) return GD_OK;
    if (!d_data || !d_comp_off || !d_comp_len || !d_out_off || !d_out) return GD_ERR_INVALID_ARG;
    if (reinterpret_cast<uintptr_t>(d_data) & 15u) return GD_ERR_INVALID_ARG;
    gd::infl::OffsetChunks ch{d_data, d_comp_off, d_comp_len, d_out_off, d_out, d_status};
    return launch_inflate(ch, n_chunks, zlib_header, d_order, (cudaStream_t)stream);
}

extern "C" gd_status_t gd_gpuinflate(const gd_inflate_input* d_inputs, gd_inflate_status* d_outputs, int count,
                                     int parse_hdr, gd_stream_t stream) {
    if (count <= 0) return GD_OK;
    if (!d_inputs || !d_outputs) return GD_ERR_INVALID_ARG;
    gd::infl::CudfChunks ch{d_inputs, d_outputs};
    return launch_inflate(ch, (uint32_t)count, parse_hdr ? 2 : 0, nullptr, (cudaStream_t)stream);
}

extern "C" gd_status_t gd_copy_uncompressed_blocks(const gd_inflate_input* d_inputs, int count, gd_stream_t stream) {
    if (count <= 0) return GD_OK;
    if (!d_inputs) return GD_ERR_INVALID_ARG;
    copy_uncompressed_kernel<<<count, 256, 0, (cudaStream_t)stream>>>(d_inputs, count);
    return cudaGetLastError() == cudaSuccess ? GD_OK : GD_ERR_CUDA;
}
