// gd_api.cpp -- host side of the C ABI: status strings, the reference-shaped
// synchronous host API (H2D copy, device decode, D2H copy, malloc'd output),
// and the per-thread device staging pool behind it.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <unordered_map>
#include <vector>

#include "../../../include/gd.h"

namespace {

// Grow-only device buffers, one set per host thread.  Slots are reused
// across calls so the host API does not pay cudaMalloc on every call.
struct Pool {
    struct Slot {
        void* p = nullptr;
        size_t cap = 0;
        int dev = -1;
    };
    Slot s[8];
    ~Pool() {
        for (auto& x : s)
            if (x.p) cudaFree(x.p);  // may fail harmlessly at process teardown
    }
    void* get(int i, size_t n) {
        int dev = 0;
        cudaGetDevice(&dev);
        Slot& x = s[i];
        if (n == 0) n = 16;
        if (x.p && x.cap >= n && x.dev == dev) return x.p;
        if (x.p) {
            int cur = dev;
            cudaSetDevice(x.dev);
            cudaFree(x.p);
            cudaSetDevice(cur);
        }
        x.p = nullptr;
        x.cap = 0;
        size_t cap = (n + (2u << 20) - 1) & ~(size_t)((2u << 20) - 1);
        if (cudaMalloc(&x.p, cap) != cudaSuccess) {
            cudaGetLastError();
            x.p = nullptr;
            return nullptr;
        }
        x.cap = cap;
        x.dev = dev;
        return x.p;
    }
};
thread_local Pool g_pool;

// Output buffers of the host API are page-locked so the device-to-host copy
// runs at full link speed.  They are recycled: gd_free() returns a buffer to
// this cache instead of unpinning it (pinning is expensive).
struct PinnedCache {
    std::mutex m;
    std::unordered_map<void*, size_t> live;      // handed out -> capacity
    std::vector<std::pair<void*, size_t>> idle;  // free for reuse
    void* get(size_t n) {
        std::lock_guard<std::mutex> g(m);
        size_t best = (size_t)-1;
        int bi = -1;
        for (size_t i = 0; i < idle.size(); ++i)
            if (idle[i].second >= n && idle[i].second < best) {
                best = idle[i].second;
                bi = (int)i;
            }
        if (bi >= 0) {
            auto e = idle[bi];
            idle.erase(idle.begin() + bi);
            live[e.first] = e.second;
            return e.first;
        }
        void* p = nullptr;
        const size_t cap = n ? n : 1;
        if (cudaHostAlloc(&p, cap, cudaHostAllocDefault) != cudaSuccess) {
            cudaGetLastError();
            p = malloc(cap);  // pageable fallback for the host buffer only
            return p;
        }
        live[p] = cap;
        return p;
    }
    bool put(void* p) {
        std::lock_guard<std::mutex> g(m);
        auto it = live.find(p);
        if (it == live.end()) return false;
        idle.emplace_back(it->first, it->second);
        live.erase(it);
        // keep at most 8 idle buffers pinned
        while (idle.size() > 8) {
            cudaFreeHost(idle.front().first);
            idle.erase(idle.begin());
        }
        return true;
    }
};
PinnedCache& pinned() {
    static PinnedCache* c = new PinnedCache();  // never destroyed: outlives CUDA teardown
    return *c;
}

gd_status_t collect(const uint32_t* d_status, uint32_t n, cudaStream_t s) {
    std::vector<uint32_t> st(n);
    if (cudaMemcpyAsync(st.data(), d_status, 4ull * n, cudaMemcpyDeviceToHost, s) != cudaSuccess) return GD_ERR_CUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess) return GD_ERR_CUDA;
    uint32_t worst = GD_OK;
    for (uint32_t v : st)
        if (v > worst) worst = v;
    return (gd_status_t)worst;
}

// Three non-blocking streams (host->device copies, decoding, device->host
// copies) and their events, per host thread and device.
constexpr int kMaxPieces = 32;
struct Pipe {
    int dev = -1;
    cudaStream_t st[3] = {nullptr, nullptr, nullptr};
    cudaEvent_t in_done[kMaxPieces], dec_done[kMaxPieces];
    bool init() {
        int d = 0;
        cudaGetDevice(&d);
        if (dev == d) return true;
        if (dev >= 0) return false;  // one device per host thread for the pipelined path
        for (auto& x : st)
            if (cudaStreamCreateWithFlags(&x, cudaStreamNonBlocking) != cudaSuccess) return false;
        for (int i = 0; i < kMaxPieces; ++i)
            if (cudaEventCreateWithFlags(&in_done[i], cudaEventDisableTiming) != cudaSuccess ||
                cudaEventCreateWithFlags(&dec_done[i], cudaEventDisableTiming) != cudaSuccess)
                return false;
        dev = d;
        return true;
    }
};
thread_local Pipe g_pipe;

// Host buffers in, host buffer out, in pieces of whole chunks: piece i's
// host->device copy, its decode and its device->host copy run on three
// streams, so copies in both directions (separate copy engines) overlap
// decoding of the neighbouring pieces.  Chunk c's input is
// h_in[in_at(c) .. in_at(c+1)) (copied to the same offset of d_in), its
// output d_out[out_at(c) .. out_at(c+1)); both must be non-decreasing in c.
// prologue(stream) issues the metadata copies (on the decode stream, before
// the first decode); launch(a, b, stream) decodes chunks [a, b).  Decoders
// read no input byte past their own chunks' streams that affects the
// result, so a piece may decode while the next piece is still arriving.
// Piece bounds: whole chunks, about total/pieces output bytes (at least
// 4 MiB) each, at most kMaxPieces pieces.
template <class OutAt>
std::vector<uint64_t> piece_cuts(uint64_t n, OutAt out_at, uint64_t pieces) {
    const uint64_t total = out_at(n);
    const uint64_t want = total / pieces > (4ull << 20) ? total / pieces : (4ull << 20);
    std::vector<uint64_t> cut{0};
    for (uint64_t c = 0; c < n && cut.size() < (size_t)kMaxPieces;) {
        uint64_t e = c + 1;
        while (e < n && out_at(e) - out_at(c) < want) ++e;
        cut.push_back(e);
        c = e;
    }
    if (cut.back() != n) cut.push_back(n);
    return cut;
}

template <class InAt, class OutAt, class Prologue, class Launch>
gd_status_t run_piped(uint64_t n, const uint8_t* h_in, uint8_t* d_in, InAt in_at, uint8_t* d_out, uint8_t* h_out,
                      OutAt out_at, uint32_t* d_st, Prologue prologue, Launch launch, uint64_t pieces = 16) {
    if (!g_pipe.init()) return GD_ERR_CUDA;
    cudaStream_t si = g_pipe.st[0], sk = g_pipe.st[1], so = g_pipe.st[2];
    const std::vector<uint64_t> cut = piece_cuts(n, out_at, pieces);
    const int np = (int)cut.size() - 1;
    gd_status_t r = prologue(sk);
    if (r != GD_OK) return r;
    for (int i = 0; i < np; ++i) {
        const uint64_t a = cut[i], b = cut[i + 1];
        const uint64_t i0 = in_at(a), i1 = in_at(b);
        if (i1 > i0 && cudaMemcpyAsync(d_in + i0, h_in + i0, i1 - i0, cudaMemcpyHostToDevice, si) != cudaSuccess)
            return GD_ERR_CUDA;
        cudaEventRecord(g_pipe.in_done[i], si);
        cudaStreamWaitEvent(sk, g_pipe.in_done[i], 0);
        r = launch(a, b, sk);
        if (r != GD_OK) {
            for (auto x : g_pipe.st) cudaStreamSynchronize(x);
            return r;
        }
        cudaEventRecord(g_pipe.dec_done[i], sk);
        cudaStreamWaitEvent(so, g_pipe.dec_done[i], 0);
        const uint64_t o0 = out_at(a), o1 = out_at(b);
        if (o1 > o0 && cudaMemcpyAsync(h_out + o0, d_out + o0, o1 - o0, cudaMemcpyDeviceToHost, so) != cudaSuccess)
            return GD_ERR_CUDA;
    }
    if (cudaStreamSynchronize(so) != cudaSuccess) return GD_ERR_CUDA;
    return collect(d_st, (uint32_t)n, sk);
}

template <typename T>
T rd(const uint8_t* p) {
    T v;
    memcpy(&v, p, sizeof(T));
    return v;
}

// Deflate streams of chunk c: in[comp_off[c] .. + comp_len[c]), output
// out[out_off[c] .. out_off[c+1]).  Pieced as run_piped when the streams lie
// in chunk order; otherwise the whole input is copied with the first piece.
// Fewer pieces than the other codecs: a piece ends with its longest stream.
gd_status_t inflate_piped(const uint8_t* in, uint64_t in_n, const uint64_t* comp_off, const uint64_t* comp_len,
                          const uint64_t* out_off, uint64_t n, int zlib_header, uint8_t* d_data, uint64_t* d_meta,
                          uint8_t* d_out, uint8_t* h, uint32_t* d_st);

}  // namespace

extern "C" {

const char* gd_version(void) { return "gd-b200 0.1 (sm_100a)"; }

const char* gd_status_string(int s) {
    switch (s) {
        case GD_OK: return "ok";
        case GD_ERR_INVALID_ARG: return "invalid argument";
        case GD_ERR_CORRUPT: return "corrupt stream";
        case GD_ERR_OVERRUN: return "output overrun";
        case GD_ERR_TIMEOUT: return "device wait timed out";
        case GD_ERR_UNSUPPORTED: return "unsupported";
        case GD_ERR_CUDA: return "cuda error";
        case GD_ERR_NOMEM: return "out of memory";
        default: return "unknown";
    }
}

void gd_free(void* p) {
    if (p && !pinned().put(p)) free(p);
}

// ---------------------------------------------------------------------------
gd_status_t gd_brle_decompress(const uint8_t* in, uint64_t in_n_bytes, uint8_t** out, uint64_t* out_n_bytes) {
    if (!in || !out || !out_n_bytes || in_n_bytes < 4) return GD_ERR_INVALID_ARG;
    const uint32_t n_ptr = rd<uint32_t>(in);
    if (n_ptr < 1) return GD_ERR_INVALID_ARG;
    const uint64_t hdr = 4ull + 8ull * n_ptr;
    if (in_n_bytes < hdr + 8) return GD_ERR_INVALID_ARG;
    const uint32_t n_chunks = n_ptr - 1;
    const uint64_t total = rd<uint64_t>(in + hdr);
    const uint8_t* data = in + hdr + 8;
    const uint64_t data_n = in_n_bytes - hdr - 8;
    const uint64_t chunk = 256 * 1024;  // CHUNK_SIZE, include/brle/brle.h:8
    std::vector<uint64_t> ptr(n_ptr);
    memcpy(ptr.data(), in + 4, 8ull * n_ptr);
    if (ptr[n_chunks] > data_n) return GD_ERR_CORRUPT;
    *out = nullptr;
    *out_n_bytes = 0;
    if (n_chunks == 0 || total == 0) {
        *out = (uint8_t*)malloc(1);
        return total == 0 ? GD_OK : GD_ERR_CORRUPT;
    }
    for (uint32_t c = 0; c < n_chunks; ++c)
        if (ptr[c + 1] < ptr[c]) return GD_ERR_CORRUPT;
    uint8_t* d_data = (uint8_t*)g_pool.get(0, data_n);
    uint64_t* d_ptr = (uint64_t*)g_pool.get(1, 8ull * n_ptr);
    uint8_t* d_out = (uint8_t*)g_pool.get(2, total);
    uint32_t* d_st = (uint32_t*)g_pool.get(3, 4ull * n_chunks);
    if (!d_data || !d_ptr || !d_out || !d_st) return GD_ERR_NOMEM;
    uint8_t* h = (uint8_t*)pinned().get(total);
    if (!h) return GD_ERR_NOMEM;
    auto out_at = [&](uint64_t c) { return c * chunk < total ? c * chunk : total; };
    gd_status_t r = run_piped(
        n_chunks, data, d_data, [&](uint64_t c) { return ptr[c]; }, d_out, h, out_at, d_st,
        [&](cudaStream_t st) {
            return cudaMemcpyAsync(d_ptr, ptr.data(), 8ull * n_ptr, cudaMemcpyHostToDevice, st) == cudaSuccess
                       ? GD_OK : GD_ERR_CUDA;
        },
        [&](uint64_t a, uint64_t b, cudaStream_t st) {
            return gd_brle_decode(d_data, d_ptr + a, (uint32_t)(b - a), chunk, d_out + a * chunk,
                                  out_at(b) - out_at(a), d_st + a, st);
        });
    if (r != GD_OK) {
        gd_free(h);
        return r;
    }
    *out = h;
    *out_n_bytes = total;
    return GD_OK;
}

// ---------------------------------------------------------------------------
gd_status_t gd_rlev1_decompress(const uint8_t* in, uint64_t in_n_bytes, const uint64_t* col_len,
                                uint64_t col_n_bytes, const uint64_t* blk_off, uint64_t blk_n_bytes,
                                uint32_t comp_col_len, uint32_t elem_bytes, uint64_t chunk_size, uint8_t** out,
                                uint64_t* out_n_bytes) {
    if (!in || !col_len || !blk_off || !out || !out_n_bytes || in_n_bytes < 8 || blk_n_bytes < 16)
        return GD_ERR_INVALID_ARG;
    const uint64_t n = blk_n_bytes / 8 - 1;
    if (col_n_bytes < 8 * 32 * n) return GD_ERR_INVALID_ARG;
    const uint64_t total = rd<uint64_t>(in);
    const uint8_t* data = in + 8;
    const uint64_t data_n = in_n_bytes - 8;
    if (blk_off[n] > data_n || total > n * chunk_size) return GD_ERR_CORRUPT;
    *out = nullptr;
    *out_n_bytes = 0;
    uint8_t* d_data = (uint8_t*)g_pool.get(0, data_n);
    uint64_t* d_cl = (uint64_t*)g_pool.get(1, 8 * 32 * n);
    uint64_t* d_bo = (uint64_t*)g_pool.get(4, 8 * (n + 1));
    uint8_t* d_out = (uint8_t*)g_pool.get(2, total);
    uint32_t* d_st = (uint32_t*)g_pool.get(3, 4 * n);
    if (!d_data || !d_cl || !d_bo || !d_out || !d_st) return GD_ERR_NOMEM;
    uint64_t mx = 0;
    for (uint64_t i = 0; i < 32 * n; ++i) mx = col_len[i] > mx ? col_len[i] : mx;
    const bool mono = std::is_sorted(blk_off, blk_off + n + 1);
    uint8_t* h = (uint8_t*)pinned().get(total ? total : 1);
    if (!h) return GD_ERR_NOMEM;
    auto out_at = [&](uint64_t c) { return c * chunk_size < total ? c * chunk_size : total; };
    gd_status_t r = run_piped(
        n, data, d_data, [&](uint64_t c) { return mono ? blk_off[c] : (c ? data_n : 0); }, d_out, h, out_at, d_st,
        [&](cudaStream_t st) {
            bool ok = cudaMemcpyAsync(d_cl, col_len, 8 * 32 * n, cudaMemcpyHostToDevice, st) == cudaSuccess;
            ok = ok && cudaMemcpyAsync(d_bo, blk_off, 8 * (n + 1), cudaMemcpyHostToDevice, st) == cudaSuccess;
            return ok ? GD_OK : GD_ERR_CUDA;
        },
        [&](uint64_t a, uint64_t b, cudaStream_t st) {
            return gd_rlev1_decode(d_data, d_cl + 32 * a, d_bo + a, (uint32_t)(b - a), chunk_size, comp_col_len,
                                   elem_bytes, d_out + a * chunk_size, out_at(b) - out_at(a),
                                   (uint32_t)(mx < 0xffffffffull ? mx : 0), d_st + a, st);
        });
    if (r != GD_OK) {
        gd_free(h);
        return r;
    }
    *out = h;
    *out_n_bytes = total;
    return GD_OK;
}

// ---------------------------------------------------------------------------
gd_status_t gd_rlev2_decompress(const uint8_t* in, uint64_t in_n_bytes, uint64_t n_chunks, const uint64_t* blk_off,
                                const uint64_t* col_len, uint32_t read_unit, uint64_t chunk_size, uint8_t** out,
                                uint64_t* out_n_bytes) {
    if (!in || !blk_off || !col_len || !out || !out_n_bytes || n_chunks == 0) return GD_ERR_INVALID_ARG;
    const uint64_t total = blk_off[n_chunks];  // the decompressed size (encoder_trans.h:490-492)
    if (total > n_chunks * chunk_size || total <= (n_chunks - 1) * chunk_size) return GD_ERR_CORRUPT;
    std::vector<uint64_t> bo(blk_off, blk_off + n_chunks + 1);
    bo[n_chunks] = in_n_bytes;  // device API: last entry bounds the data
    *out = nullptr;
    *out_n_bytes = 0;
    uint8_t* d_data = (uint8_t*)g_pool.get(0, in_n_bytes);
    uint64_t* d_cl = (uint64_t*)g_pool.get(1, 8 * 32 * n_chunks);
    uint64_t* d_bo = (uint64_t*)g_pool.get(4, 8 * (n_chunks + 1));
    uint8_t* d_out = (uint8_t*)g_pool.get(2, total);
    uint32_t* d_st = (uint32_t*)g_pool.get(3, 4 * n_chunks);
    if (!d_data || !d_cl || !d_bo || !d_out || !d_st) return GD_ERR_NOMEM;
    uint64_t mx = 0;
    for (uint64_t i = 0; i < 32 * n_chunks; ++i) mx = col_len[i] > mx ? col_len[i] : mx;
    const bool mono = std::is_sorted(bo.begin(), bo.end());
    uint8_t* h = (uint8_t*)pinned().get(total);
    if (!h) return GD_ERR_NOMEM;
    auto out_at = [&](uint64_t c) { return c * chunk_size < total ? c * chunk_size : total; };
    gd_status_t r = run_piped(
        n_chunks, in, d_data, [&](uint64_t c) { return mono ? bo[c] : (c ? in_n_bytes : 0); }, d_out, h, out_at,
        d_st,
        [&](cudaStream_t st) {
            bool ok = cudaMemcpyAsync(d_cl, col_len, 8 * 32 * n_chunks, cudaMemcpyHostToDevice, st) == cudaSuccess;
            ok = ok && cudaMemcpyAsync(d_bo, bo.data(), 8 * (n_chunks + 1), cudaMemcpyHostToDevice, st) == cudaSuccess;
            return ok ? GD_OK : GD_ERR_CUDA;
        },
        [&](uint64_t a, uint64_t b, cudaStream_t st) {
            return gd_rlev2_decode(d_data, d_cl + 32 * a, d_bo + a, (uint32_t)(b - a), chunk_size, read_unit,
                                   d_out + a * chunk_size, out_at(b) - out_at(a),
                                   (uint32_t)(mx < 0xffffffffull ? mx : 0), d_st + a, st);
        });
    if (r != GD_OK) {
        gd_free(h);
        return r;
    }
    *out = h;
    *out_n_bytes = total;
    return GD_OK;
}

// ---------------------------------------------------------------------------
int gd_lzss_decompress(const uint8_t* in, uint64_t in_n_bytes, const uint8_t* const* meta, const uint64_t* meta_lens,
                       uint64_t meta_num, uint8_t** out, uint64_t* out_n_bytes) {
    if (meta_num < 4 || !meta || !meta_lens) return -1;  // as lzss_gpu2.h:2212-2213
    if (!in || !out || !out_n_bytes || meta_lens[0] < 8) return GD_ERR_INVALID_ARG;
    const uint64_t chunk = rd<uint64_t>(meta[0]);
    const uint64_t n = meta_lens[1] / 8 - 1;
    if (n == 0 || meta_lens[2] < 8 * 32 * n || meta_lens[3] < 32 * n) return GD_ERR_INVALID_ARG;
    std::vector<uint64_t> bo(n + 1);
    memcpy(bo.data(), meta[1], 8 * (n + 1));
    if (bo[n] > in_n_bytes) return GD_ERR_CORRUPT;
    const uint64_t total = n * chunk;
    *out = nullptr;
    *out_n_bytes = 0;
    uint8_t* d_data = (uint8_t*)g_pool.get(0, in_n_bytes);
    uint64_t* d_cl = (uint64_t*)g_pool.get(1, 8 * 32 * n);
    uint64_t* d_bo = (uint64_t*)g_pool.get(4, 8 * (n + 1));
    uint8_t* d_map = (uint8_t*)g_pool.get(5, 32 * n);
    uint8_t* d_out = (uint8_t*)g_pool.get(2, total);
    uint32_t* d_st = (uint32_t*)g_pool.get(3, 4 * n);
    if (!d_data || !d_cl || !d_bo || !d_map || !d_out || !d_st) return GD_ERR_NOMEM;
    const bool mono = std::is_sorted(bo.begin(), bo.end());
    uint8_t* h = (uint8_t*)pinned().get(total);
    if (!h) return GD_ERR_NOMEM;
    int r = run_piped(
        n, in, d_data, [&](uint64_t c) { return mono ? bo[c] : (c ? in_n_bytes : 0); }, d_out, h,
        [&](uint64_t c) { return c * chunk; }, d_st,
        [&](cudaStream_t st) {
            bool ok = cudaMemcpyAsync(d_cl, meta[2], 8 * 32 * n, cudaMemcpyHostToDevice, st) == cudaSuccess;
            ok = ok && cudaMemcpyAsync(d_bo, bo.data(), 8 * (n + 1), cudaMemcpyHostToDevice, st) == cudaSuccess;
            ok = ok && cudaMemcpyAsync(d_map, meta[3], 32 * n, cudaMemcpyHostToDevice, st) == cudaSuccess;
            return ok ? GD_OK : GD_ERR_CUDA;
        },
        [&](uint64_t a, uint64_t b, cudaStream_t st) {
            return gd_lzss_decode(d_data, d_bo + a, d_cl + 32 * a, d_map + 32 * a, (uint32_t)(b - a), chunk,
                                  d_out + a * chunk, (b - a) * chunk, d_st + a, st);
        });
    if (r != GD_OK) {
        gd_free(h);
        return r;
    }
    *out = h;
    *out_n_bytes = total;
    return 0;
}

// ---------------------------------------------------------------------------
gd_status_t gd_deflate_decompress(const uint8_t* in, uint64_t in_n_bytes, const uint64_t* col_len,
                                  uint64_t col_n_bytes, const uint64_t* blk_offset, uint64_t blk_n_bytes,
                                  uint64_t chunk_size, uint8_t** out, uint64_t* out_n_bytes) {
    if (!in || !col_len || !blk_offset || !out || !out_n_bytes || blk_n_bytes < 24 || chunk_size == 0)
        return GD_ERR_INVALID_ARG;
    const uint64_t n = blk_n_bytes / 8 - 2;  // zlib.h:970
    if (col_n_bytes < 8 * n) return GD_ERR_INVALID_ARG;
    const uint64_t total = blk_offset[0];
    if (total > n * chunk_size || total <= (n - 1) * chunk_size) return GD_ERR_CORRUPT;
    std::vector<uint64_t> coff(n + 1), clen(n), ooff(n + 1);
    for (uint64_t i = 0; i <= n; ++i) coff[i] = blk_offset[1 + i];
    for (uint64_t i = 0; i < n; ++i) {
        clen[i] = col_len[i];
        ooff[i] = i * chunk_size;
        if (coff[i] + clen[i] > in_n_bytes) return GD_ERR_CORRUPT;
    }
    ooff[n] = total;
    *out = nullptr;
    *out_n_bytes = 0;
    uint8_t* d_data = (uint8_t*)g_pool.get(0, in_n_bytes);
    uint64_t* d_meta = (uint64_t*)g_pool.get(1, 8 * (3 * n + 2));
    uint8_t* d_out = (uint8_t*)g_pool.get(2, total);
    uint32_t* d_st = (uint32_t*)g_pool.get(3, 4 * n);
    if (!d_data || !d_meta || !d_out || !d_st) return GD_ERR_NOMEM;
    uint8_t* h = (uint8_t*)pinned().get(total);
    if (!h) return GD_ERR_NOMEM;
    gd_status_t r = inflate_piped(in, in_n_bytes, coff.data(), clen.data(), ooff.data(), n, 1, d_data, d_meta, d_out,
                                  h, d_st);
    if (r != GD_OK) {
        gd_free(h);
        return r;
    }
    *out = h;
    *out_n_bytes = total;
    return GD_OK;
}


// ---------------------------------------------------------------------------
// LZSS contiguous container (replaces lzss::decompress_gpu_base,
// include/lzss/lzss.h:1126-1188): [u64 in_n_bytes][u32 chunk_size]
// [u32 n_chunks][u32 hist][u32 min][u32 max][u64 stream end per chunk][data].
// ---------------------------------------------------------------------------
gd_status_t gd_lzss_contig_decompress(const uint8_t* in, uint64_t in_n_bytes, uint8_t** out, uint64_t* out_n_bytes) {
    if (!in || !out || !out_n_bytes || in_n_bytes < 28) return GD_ERR_INVALID_ARG;
    uint64_t total;
    uint32_t head[5];
    memcpy(&total, in, 8);
    memcpy(head, in + 8, 20);
    const uint64_t chunk = head[0], n = head[1];
    if (chunk == 0 || n == 0 || n != (total ? (total - 1) / chunk + 1 : 0)) return GD_ERR_CORRUPT;
    if (head[2] != 2048 || head[3] != 3 || head[4] != 34) return GD_ERR_UNSUPPORTED;  // lzss.h:24-32
    if (in_n_bytes < 28 + 8 * n) return GD_ERR_CORRUPT;
    std::vector<uint64_t> ends(n);
    memcpy(ends.data(), in + 28, 8 * n);  // not 8-byte aligned in the container
    const uint64_t dlen = in_n_bytes - 28 - 8 * n;
    if (ends[n - 1] > dlen) return GD_ERR_CORRUPT;
    *out = nullptr;
    *out_n_bytes = 0;
    uint8_t* d_data = (uint8_t*)g_pool.get(0, dlen + 16);
    uint64_t* d_ends = (uint64_t*)g_pool.get(1, 8 * n);
    uint8_t* d_out = (uint8_t*)g_pool.get(2, total);
    uint32_t* d_st = (uint32_t*)g_pool.get(3, 4 * n);
    if (!d_data || !d_ends || !d_out || !d_st) return GD_ERR_NOMEM;
    uint8_t* h = (uint8_t*)pinned().get(total);
    if (!h) return GD_ERR_NOMEM;
    // one piece: a chunk's stream starts where the previous chunk's ends
    gd_status_t r = run_piped(
        n, in + 28 + 8 * n, d_data, [&](uint64_t c) { return c ? dlen : 0; }, d_out, h,
        [&](uint64_t c) { return c * chunk < total ? c * chunk : total; }, d_st,
        [&](cudaStream_t st) {
            return cudaMemcpyAsync(d_ends, ends.data(), 8 * n, cudaMemcpyHostToDevice, st) == cudaSuccess
                       ? GD_OK : GD_ERR_CUDA;
        },
        [&](uint64_t, uint64_t, cudaStream_t st) {
            return gd_lzss_contig_decode(d_data, d_ends, (uint32_t)n, chunk, d_out, total, d_st, st);
        },
        1);
    if (r != GD_OK) {
        gd_free(h);
        return r;
    }
    *out = h;
    *out_n_bytes = total;
    return GD_OK;
}

// ---------------------------------------------------------------------------
// Byte-RLE flag-byte interleaved container (replaces
// brle_trans::decompress_gpu, include/brle/brle_trans.h:661-791, which reads
// col_len / col_map / blk_offset from ./input_data side files): the output is
// n_chunks * chunk_size bytes, n_chunks = blk_n_bytes/8 - 1.
// ---------------------------------------------------------------------------
using FlagDecode = gd_status_t (*)(const uint8_t*, const uint64_t*, const uint64_t*, const uint8_t*, uint32_t,
                                   uint64_t, uint8_t*, uint64_t, uint32_t*, gd_stream_t);

static gd_status_t flag_decompress(FlagDecode decode, const uint8_t* in, uint64_t in_n_bytes,
                                   const uint64_t* col_len, uint64_t col_n_bytes, const uint8_t* col_map,
                                   uint64_t map_n_bytes, const uint64_t* blk_off, uint64_t blk_n_bytes,
                                   uint64_t chunk_size, uint8_t** out, uint64_t* out_n_bytes) {
    if (!in || !col_len || !col_map || !blk_off || !out || !out_n_bytes || blk_n_bytes < 16) return GD_ERR_INVALID_ARG;
    const uint64_t n = blk_n_bytes / 8 - 1;
    if (col_n_bytes < 8 * 32 * n || map_n_bytes < 32 * n) return GD_ERR_INVALID_ARG;
    if (blk_off[n] > in_n_bytes) return GD_ERR_CORRUPT;
    const uint64_t total = n * chunk_size;
    *out = nullptr;
    *out_n_bytes = 0;
    uint8_t* d_data = (uint8_t*)g_pool.get(0, in_n_bytes + 16);
    uint64_t* d_cl = (uint64_t*)g_pool.get(1, 8 * 32 * n);
    uint64_t* d_bo = (uint64_t*)g_pool.get(4, 8 * (n + 1));
    uint8_t* d_map = (uint8_t*)g_pool.get(5, 32 * n);
    uint8_t* d_out = (uint8_t*)g_pool.get(2, total);
    uint32_t* d_st = (uint32_t*)g_pool.get(3, 4 * n);
    if (!d_data || !d_cl || !d_bo || !d_map || !d_out || !d_st) return GD_ERR_NOMEM;
    const bool mono = std::is_sorted(blk_off, blk_off + n + 1);
    uint8_t* h = (uint8_t*)pinned().get(total);
    if (!h) return GD_ERR_NOMEM;
    gd_status_t r = run_piped(
        n, in, d_data, [&](uint64_t c) { return mono ? blk_off[c] : (c ? in_n_bytes : 0); }, d_out, h,
        [&](uint64_t c) { return c * chunk_size; }, d_st,
        [&](cudaStream_t st) {
            bool ok = cudaMemcpyAsync(d_cl, col_len, 8 * 32 * n, cudaMemcpyHostToDevice, st) == cudaSuccess;
            ok = ok && cudaMemcpyAsync(d_bo, blk_off, 8 * (n + 1), cudaMemcpyHostToDevice, st) == cudaSuccess;
            ok = ok && cudaMemcpyAsync(d_map, col_map, 32 * n, cudaMemcpyHostToDevice, st) == cudaSuccess;
            return ok ? GD_OK : GD_ERR_CUDA;
        },
        [&](uint64_t a, uint64_t b, cudaStream_t st) {
            return decode(d_data, d_bo + a, d_cl + 32 * a, d_map + 32 * a, (uint32_t)(b - a), chunk_size,
                          d_out + a * chunk_size, (b - a) * chunk_size, d_st + a, st);
        });
    if (r != GD_OK) {
        gd_free(h);
        return r;
    }
    *out = h;
    *out_n_bytes = total;
    return GD_OK;
}

gd_status_t gd_brle_trans_decompress(const uint8_t* in, uint64_t in_n_bytes, const uint64_t* col_len,
                                     uint64_t col_n_bytes, const uint8_t* col_map, uint64_t map_n_bytes,
                                     const uint64_t* blk_off, uint64_t blk_n_bytes, uint64_t chunk_size,
                                     uint8_t** out, uint64_t* out_n_bytes) {
    return flag_decompress(gd_brle_trans_decode, in, in_n_bytes, col_len, col_n_bytes, col_map, map_n_bytes, blk_off,
                           blk_n_bytes, chunk_size, out, out_n_bytes);
}

// brle::decompress_gpu of include/brle/brle_gpu_4B.h:717-897 (4-byte
// symbols, 8 KiB chunks there), with its side files' arrays passed in.
gd_status_t gd_brle_trans4_decompress(const uint8_t* in, uint64_t in_n_bytes, const uint64_t* col_len,
                                      uint64_t col_n_bytes, const uint8_t* col_map, uint64_t map_n_bytes,
                                      const uint64_t* blk_off, uint64_t blk_n_bytes, uint64_t chunk_size,
                                      uint8_t** out, uint64_t* out_n_bytes) {
    return flag_decompress(gd_brle_trans4_decode, in, in_n_bytes, col_len, col_n_bytes, col_map, map_n_bytes,
                           blk_off, blk_n_bytes, chunk_size, out, out_n_bytes);
}


// ---------------------------------------------------------------------------
// Deflate chunks of any size (extension of deflate::decompress_gpu, which
// assumes one uniform chunk size: zlib.h:966-1082).
// ---------------------------------------------------------------------------
gd_status_t gd_inflate_decompress(const uint8_t* in, uint64_t in_n_bytes, const uint64_t* comp_off,
                                  const uint64_t* comp_len, const uint64_t* out_off, uint32_t n_chunks,
                                  int zlib_header, uint8_t** out, uint64_t* out_n_bytes) {
    if (!in || !comp_off || !comp_len || !out_off || !out || !out_n_bytes || n_chunks == 0) return GD_ERR_INVALID_ARG;
    const uint64_t n = n_chunks;
    for (uint64_t i = 0; i < n; ++i) {
        if (comp_off[i] + comp_len[i] > in_n_bytes || out_off[i + 1] < out_off[i]) return GD_ERR_CORRUPT;
    }
    const uint64_t total = out_off[n];
    *out = nullptr;
    *out_n_bytes = 0;
    uint8_t* d_data = (uint8_t*)g_pool.get(0, in_n_bytes + 16);
    uint64_t* d_meta = (uint64_t*)g_pool.get(1, 8 * (3 * n + 2));
    uint8_t* d_out = (uint8_t*)g_pool.get(2, total ? total : 1);
    uint32_t* d_st = (uint32_t*)g_pool.get(3, 4 * n);
    if (!d_data || !d_meta || !d_out || !d_st) return GD_ERR_NOMEM;
    uint8_t* h = (uint8_t*)pinned().get(total ? total : 1);
    if (!h) return GD_ERR_NOMEM;
    gd_status_t r = inflate_piped(in, in_n_bytes, comp_off, comp_len, out_off, n, zlib_header, d_data, d_meta, d_out,
                                  h, d_st);
    if (r != GD_OK) {
        gd_free(h);
        return r;
    }
    *out = h;
    *out_n_bytes = total;
    return GD_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Host compress calls on the device encoders: the column is copied in,
// encoded on the device and the container and its metadata copied back.
// Their own grow-only pool, so interleaved compress and decompress calls do
// not resize each other's staging buffers.
namespace {
thread_local Pool g_epool;

struct EncBufs {
    uint8_t* in;
    uint8_t* scratch;
    uint8_t* data;
    uint64_t* blk_off;
    uint64_t* col_len;
    uint8_t* col_map;
    uint32_t* st;
};

// Stage the column and size the interleaved encoders' buffers for nc chunks.
gd_status_t enc_stage(const uint8_t* in, uint64_t n, uint64_t nc, uint64_t bound, EncBufs& b, cudaStream_t s) {
    b.in = (uint8_t*)g_epool.get(0, n);
    b.scratch = (uint8_t*)g_epool.get(1, bound);
    b.data = (uint8_t*)g_epool.get(2, bound);
    b.blk_off = (uint64_t*)g_epool.get(3, 8 * (nc + 1));
    b.col_len = (uint64_t*)g_epool.get(4, 8 * 32 * nc);
    b.col_map = (uint8_t*)g_epool.get(5, 32 * nc);
    b.st = (uint32_t*)g_epool.get(6, 4 * nc);
    if (!b.in || !b.scratch || !b.data || !b.blk_off || !b.col_len || !b.col_map || !b.st) return GD_ERR_NOMEM;
    return cudaMemcpyAsync(b.in, in, n, cudaMemcpyHostToDevice, s) == cudaSuccess ? GD_OK : GD_ERR_CUDA;
}

// After the encoder: its status, then blk_off and col_len (and col_map) into
// malloc'd arrays and the blk_off[nc] data bytes into a pinned buffer at
// offset `at` (the caller fills the first `at` bytes).
gd_status_t enc_fetch(const EncBufs& b, uint64_t nc, uint64_t at, cudaStream_t s, uint8_t** data, uint64_t* data_n,
                      uint64_t** blk_off, uint64_t** col_len, uint8_t** col_map) {
    gd_status_t r = collect(b.st, (uint32_t)nc, s);
    if (r != GD_OK) return r;
    uint64_t* bo = (uint64_t*)malloc(8 * (nc + 1));
    uint64_t* cl = (uint64_t*)malloc(8 * 32 * nc);
    uint8_t* cm = col_map ? (uint8_t*)malloc(32 * nc) : nullptr;
    uint8_t* h = nullptr;
    auto fail = [&](gd_status_t why) {
        free(bo);
        free(cl);
        free(cm);
        if (h) gd_free(h);
        return why;
    };
    if (!bo || !cl || (col_map && !cm)) return fail(GD_ERR_NOMEM);
    bool ok = cudaMemcpyAsync(bo, b.blk_off, 8 * (nc + 1), cudaMemcpyDeviceToHost, s) == cudaSuccess;
    ok = ok && cudaMemcpyAsync(cl, b.col_len, 8 * 32 * nc, cudaMemcpyDeviceToHost, s) == cudaSuccess;
    ok = ok && (!cm || cudaMemcpyAsync(cm, b.col_map, 32 * nc, cudaMemcpyDeviceToHost, s) == cudaSuccess);
    ok = ok && cudaStreamSynchronize(s) == cudaSuccess;
    if (!ok) return fail(GD_ERR_CUDA);
    h = (uint8_t*)pinned().get(at + bo[nc]);
    if (!h) return fail(GD_ERR_NOMEM);  // no pinned host buffer for the container
    ok = cudaMemcpyAsync(h + at, b.data, bo[nc], cudaMemcpyDeviceToHost, s) == cudaSuccess &&
         cudaStreamSynchronize(s) == cudaSuccess;
    if (!ok) return fail(GD_ERR_CUDA);
    *data = h;
    *data_n = at + bo[nc];
    *blk_off = bo;
    *col_len = cl;
    if (col_map) *col_map = cm;
    return GD_OK;
}
}  // namespace

extern "C" {

gd_status_t gd_brle_compress(const uint8_t* in, uint64_t in_n_bytes, uint8_t** out, uint64_t* out_n_bytes) {
    if (!in || !out || !out_n_bytes || in_n_bytes == 0) return GD_ERR_INVALID_ARG;
    *out = nullptr;
    *out_n_bytes = 0;
    const uint64_t chunk = 256 * 1024;  // CHUNK_SIZE, include/brle/brle.h:8
    const uint64_t cap = gd_brle_max_encoded_bytes(in_n_bytes, chunk);
    const uint64_t sb = gd_brle_encode_scratch_bytes(in_n_bytes, chunk);
    if (!cap || !sb) return GD_ERR_INVALID_ARG;
    if (!g_pipe.init()) return GD_ERR_CUDA;
    cudaStream_t s = g_pipe.st[1];
    uint8_t* d_in = (uint8_t*)g_epool.get(0, in_n_bytes);
    uint8_t* d_sc = (uint8_t*)g_epool.get(1, sb);
    uint8_t* d_out = (uint8_t*)g_epool.get(2, cap);
    uint64_t* d_len = (uint64_t*)g_epool.get(3, 8);
    if (!d_in || !d_sc || !d_out || !d_len) return GD_ERR_NOMEM;
    if (cudaMemcpyAsync(d_in, in, in_n_bytes, cudaMemcpyHostToDevice, s) != cudaSuccess) return GD_ERR_CUDA;
    gd_status_t r = gd_brle_encode_device(d_in, in_n_bytes, chunk, d_sc, d_out, d_len, s);
    if (r != GD_OK) {
        cudaStreamSynchronize(s);  // the input copy may still be reading `in`
        return r;
    }
    uint64_t len = 0;
    if (cudaMemcpyAsync(&len, d_len, 8, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return GD_ERR_CUDA;
    if (len > cap) return GD_ERR_OVERRUN;
    uint8_t* h = (uint8_t*)pinned().get(len);
    if (!h) return GD_ERR_NOMEM;
    if (cudaMemcpyAsync(h, d_out, len, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess) {
        gd_free(h);
        return GD_ERR_CUDA;
    }
    *out = h;
    *out_n_bytes = len;
    return GD_OK;
}

gd_status_t gd_rlev1_compress(const uint8_t* in, uint64_t in_n_bytes, uint32_t comp_col_len, uint32_t elem_bytes,
                              uint64_t chunk_size, uint8_t** out, uint64_t* out_n_bytes, uint64_t** col_len,
                              uint64_t** blk_off, uint64_t* n_chunks) {
    if (!in || !out || !out_n_bytes || !col_len || !blk_off || !n_chunks || in_n_bytes == 0 || chunk_size == 0)
        return GD_ERR_INVALID_ARG;
    *out = nullptr;
    *out_n_bytes = 0;
    const uint64_t bound = gd_rlev1_encode_bound(in_n_bytes, chunk_size, elem_bytes);
    if (!bound) return GD_ERR_INVALID_ARG;
    if (!g_pipe.init()) return GD_ERR_CUDA;
    cudaStream_t s = g_pipe.st[1];
    const uint64_t nc = (in_n_bytes + chunk_size - 1) / chunk_size;
    EncBufs b;
    gd_status_t r = enc_stage(in, in_n_bytes, nc, bound, b, s);
    if (r == GD_OK)
        r = gd_rlev1_encode_device(b.in, in_n_bytes, chunk_size, comp_col_len, elem_bytes, b.scratch, b.data,
                                   b.blk_off, b.col_len, b.st, s);
    if (r == GD_OK) r = enc_fetch(b, nc, 8, s, out, out_n_bytes, blk_off, col_len, nullptr);
    if (r != GD_OK) {
        cudaStreamSynchronize(s);  // the input copy may still be reading `in`
        return r;
    }
    memcpy(*out, &in_n_bytes, 8);  // [u64 in_n_bytes][data], include/rle_v1/rlev1.h:67-70
    *n_chunks = nc;
    return GD_OK;
}

gd_status_t gd_rlev2_compress(const uint8_t* in, uint64_t in_n_bytes, uint32_t read_unit, uint64_t chunk_size,
                              uint8_t** out, uint64_t* out_n_bytes, uint64_t** blk_off, uint64_t** col_len,
                              uint64_t* n_chunks) {
    if (!in || !out || !out_n_bytes || !blk_off || !col_len || !n_chunks || in_n_bytes == 0 || chunk_size == 0)
        return GD_ERR_INVALID_ARG;
    *out = nullptr;
    *out_n_bytes = 0;
    const uint64_t bound = gd_rlev2_encode_bound(in_n_bytes, chunk_size);
    if (!bound) return GD_ERR_INVALID_ARG;
    if (!g_pipe.init()) return GD_ERR_CUDA;
    cudaStream_t s = g_pipe.st[1];
    const uint64_t nc = (in_n_bytes + chunk_size - 1) / chunk_size;
    EncBufs b;
    gd_status_t r = enc_stage(in, in_n_bytes, nc, bound, b, s);
    if (r == GD_OK)
        r = gd_rlev2_encode_device(b.in, in_n_bytes, chunk_size, read_unit, b.scratch, b.data, b.blk_off, b.col_len,
                                   b.st, s);
    if (r == GD_OK) r = enc_fetch(b, nc, 0, s, out, out_n_bytes, blk_off, col_len, nullptr);
    if (r != GD_OK) {
        cudaStreamSynchronize(s);  // the input copy may still be reading `in`
        return r;
    }
    (*blk_off)[nc] = in_n_bytes;  // the column's size in the last entry, include/rlev2/encoder_trans.h:492
    *n_chunks = nc;
    return GD_OK;
}

int gd_lzss_compress(const uint8_t* in, uint64_t in_n_bytes, uint8_t** out, uint64_t* out_n_bytes,
                     uint8_t*** out_meta, uint64_t** out_meta_lens, uint64_t* out_meta_num) {
    if (!in || !out || !out_n_bytes || !out_meta || !out_meta_lens || !out_meta_num || in_n_bytes == 0)
        return GD_ERR_INVALID_ARG;
    *out = nullptr;
    *out_n_bytes = 0;
    const uint64_t chunk = 128 * 1024;  // CHUNK_SIZE_(), include/lzss/lzss_gpu2.h:25
    const uint64_t bound = gd_lzss_encode_bound(in_n_bytes, chunk);
    if (!bound) return GD_ERR_INVALID_ARG;
    if (!g_pipe.init()) return GD_ERR_CUDA;
    cudaStream_t s = g_pipe.st[1];
    const uint64_t nc = (in_n_bytes + chunk - 1) / chunk;
    EncBufs b;
    uint64_t *bo = nullptr, *cl = nullptr;
    uint8_t* cm = nullptr;
    gd_status_t r = enc_stage(in, in_n_bytes, nc, bound, b, s);
    if (r == GD_OK)
        r = gd_lzss_encode_device(b.in, in_n_bytes, chunk, b.scratch, b.data, b.blk_off, b.col_len, b.col_map, b.st,
                                  s);
    if (r == GD_OK) r = enc_fetch(b, nc, 0, s, out, out_n_bytes, &bo, &cl, &cm);
    if (r != GD_OK) {
        cudaStreamSynchronize(s);  // the input copy may still be reading `in`
        return r;
    }
    // Four blobs as include/lzss/lzss_gpu2.h:2090-2108 hands them out:
    // chunk size, blk_offset, col_len, col_map.
    uint8_t** meta = (uint8_t**)malloc(4 * sizeof(uint8_t*));
    uint64_t* lens = (uint64_t*)malloc(4 * sizeof(uint64_t));
    uint64_t* cs = (uint64_t*)malloc(8);
    if (!meta || !lens || !cs) {
        free(meta);
        free(lens);
        free(cs);
        free(bo);
        free(cl);
        free(cm);
        gd_free(*out);
        *out = nullptr;
        *out_n_bytes = 0;
        return GD_ERR_NOMEM;
    }
    *cs = chunk;
    meta[0] = (uint8_t*)cs;
    meta[1] = (uint8_t*)bo;
    meta[2] = (uint8_t*)cl;
    meta[3] = cm;
    lens[0] = 8;
    lens[1] = 8 * (nc + 1);
    lens[2] = 8 * 32 * nc;
    lens[3] = 32 * nc;
    *out_meta = meta;
    *out_meta_lens = lens;
    *out_meta_num = 4;
    return GD_OK;
}

}  // extern "C"

namespace {
gd_status_t inflate_piped(const uint8_t* in, uint64_t in_n, const uint64_t* comp_off, const uint64_t* comp_len,
                          const uint64_t* out_off, uint64_t n, int zlib_header, uint8_t* d_data, uint64_t* d_meta,
                          uint8_t* d_out, uint8_t* h, uint32_t* d_st) {
    bool mono = true;
    for (uint64_t i = 0; i + 1 < n && mono; ++i) mono = comp_off[i] + comp_len[i] <= comp_off[i + 1];
    auto in_at = [&](uint64_t c) -> uint64_t {
        if (!mono) return c ? in_n : 0;
        return c < n ? comp_off[c] : in_n;
    };
    // inside every piece the streams start longest first: the piece ends
    // with its longest stream, so that one must not start last
    constexpr uint64_t kPieces = 4;
    uint32_t* d_order = (uint32_t*)g_pool.get(6, 4 * n);
    if (!d_order) return GD_ERR_NOMEM;
    std::vector<uint32_t> order(n);
    for (uint64_t i = 0; i < n; ++i) order[i] = (uint32_t)i;
    auto out_at = [&](uint64_t c) { return out_off[c]; };
    {
        const std::vector<uint64_t> cuts = piece_cuts(n, out_at, kPieces);  // as run_piped cuts them
        for (size_t i = 0; i + 1 < cuts.size(); ++i)
            std::stable_sort(order.begin() + cuts[i], order.begin() + cuts[i + 1], [&](uint32_t x, uint32_t y) {
                return out_off[x + 1] - out_off[x] > out_off[y + 1] - out_off[y];
            });
    }
    return run_piped(
        n, in, d_data, in_at, d_out, h, out_at, d_st,
        [&](cudaStream_t st) {
            bool ok = cudaMemcpyAsync(d_meta, comp_off, 8 * n, cudaMemcpyHostToDevice, st) == cudaSuccess;
            ok = ok && cudaMemcpyAsync(d_meta + n + 1, comp_len, 8 * n, cudaMemcpyHostToDevice, st) == cudaSuccess;
            ok = ok && cudaMemcpyAsync(d_meta + 2 * n + 1, out_off, 8 * (n + 1), cudaMemcpyHostToDevice, st) ==
                           cudaSuccess;
            ok = ok && cudaMemcpyAsync(d_order, order.data(), 4 * n, cudaMemcpyHostToDevice, st) == cudaSuccess;
            return ok ? GD_OK : GD_ERR_CUDA;
        },
        [&](uint64_t a, uint64_t b, cudaStream_t st) {
            return gd_inflate_ordered(d_data, d_meta, d_meta + n + 1, d_meta + 2 * n + 1, (uint32_t)(b - a),
                                      zlib_header, d_out, d_st, d_order + a, st);
        },
        kPieces);
}
}  // namespace
