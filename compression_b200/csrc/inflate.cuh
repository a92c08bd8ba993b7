// inflate.cuh -- warp-level Deflate / zlib / gzip inflate for sm_100a
// (shared by the plain kernels in inflate.cu and the batched decoder).
//
// Replaces the reference's deflate::inflate / inflate_shared
// (include/zlib/zlib.h:832-962): there one lane per chunk decodes codes
// bit-serially from global-memory trees (zlib.h:233-266) and a writer warp
// copies back-references; stored blocks are dropped (zlib.h:532-543).
//
// Here one warp owns a chunk and alternates two phases:
//   decode  -- lane 0 reads the bit stream from a shared-memory input ring and
//              decodes symbols with 10-bit lookup tables (longer codes fall
//              back to a canonical count/symbol walk), appending commands
//              (literal runs, (length, distance) copies, stored blocks) to a
//              shared command buffer;
//   execute -- all 32 lanes write the commands to the output: literal runs
//              and stored data as coalesced byte stores, copies in 32-byte
//              waves (distance >= 32: each wave reads bytes written by earlier
//              waves; distance < 32: the period-`distance` pattern is read
//              from before the copy).  The warp also refills the input ring.
//              With a window (WIN > 0) the last 32 KiB of output are kept in
//              shared memory and copies read only there.
// Dynamic tables are rebuilt per block; table fills are spread over the warp.
// Every read is bounded by the chunk's compressed size and every write by its
// output size; malformed input yields GD_ERR_CORRUPT / GD_ERR_OVERRUN.
#pragma once
#include "gd_common.cuh"

namespace gd {
namespace infl {

constexpr int WPB = 2;             // warps (chunks) per block
constexpr uint32_t IRING = 8192;   // input ring bytes per warp
constexpr uint32_t LBITS = 10;     // primary lookup bits
constexpr uint32_t NCMD = 256;     // commands per batch
constexpr uint32_t NLIT = 2048;    // literal bytes per batch

// length codes 257..285 and distance codes 0..29 (RFC 1951 3.2.5)
__device__ __constant__ uint16_t LBASE[29] = {3,  4,  5,  6,  7,  8,  9,  10, 11,  13,  15,  17,  19,  23, 27,
                                              31, 35, 43, 51, 59, 67, 83, 99, 115, 131, 163, 195, 227, 258};
__device__ __constant__ uint8_t LEXT[29] = {0, 0, 0, 0, 0, 0, 0, 0, 1, 1, 1, 1, 2, 2, 2,
                                            2, 3, 3, 3, 3, 4, 4, 4, 4, 5, 5, 5, 5, 0};
__device__ __constant__ uint16_t DBASE[30] = {1,   2,   3,   4,   5,   7,    9,    13,   17,   25,
                                              33,  49,  65,  97,  129, 193,  257,  385,  513,  769,
                                              1025, 1537, 2049, 3073, 4097, 6145, 8193, 12289, 16385, 24577};
__device__ __constant__ uint8_t DEXT[30] = {0, 0, 0, 0, 1, 1, 2, 2,  3,  3,  4,  4,  5,  5,  6,
                                            6, 7, 7, 8, 8, 9, 9, 10, 10, 11, 11, 12, 12, 13, 13};
__device__ __constant__ uint8_t CLORDER[19] = {16, 17, 18, 0, 8, 7, 9, 6, 10, 5, 11, 4, 12, 3, 13, 2, 14, 1, 15};

// A canonical Huffman code: primary table + count/symbol arrays for the walk.
template <uint32_t BITS>
struct HuffT {
    uint32_t lut[1u << BITS];  // (sym << 8) | len, len 0 = longer than LBITS, 0xffffffff = invalid
    uint16_t count[16];
    uint16_t sym[320];
};
using Huff = HuffT<LBITS>;

enum : uint32_t { C_LIT = 0, C_COPY = 1, C_STORED = 2 };

// One batch of decoded commands: literal bytes, commands, and the output
// position of its first byte.  last = no batch follows (pair hand-off).
template <uint32_t NL, uint32_t NC>
struct BatchT {
    static constexpr uint32_t kLits = NL, kCmds = NC;
    uint8_t lits[NL];
    uint32_t cmd_a[NC];  // C_LIT: literal buffer offset | C_COPY: distance | C_STORED: input offset
    uint32_t cmd_b[NC];  // length
    uint8_t cmd_t[NC];
    uint32_t n_cmd, n_lit, pos0, last;
};
using Batch = BatchT<NLIT, NCMD>;

// Per-stream shared state.  WIN > 0: the last WIN output bytes are kept in a
// shared-memory window (a power of two; with 32768, the Deflate window, no
// back-reference reads global memory, with less only the farther ones do);
// WIN = 0: copies read the output already written to global memory (a
// smaller footprint, for kernels that run other decoders beside this one).  NB = 1: one warp decodes and
// executes; NB = 2: a decoder warp fills batch k+1 while a writer warp
// executes batch k.
// RB: input ring bytes; DB: distance lookup bits; NL / NC: literal bytes and
// commands per batch (smaller values for kernels that run many warps).
template <uint32_t WIN, int NB = 1, uint32_t RB = IRING, uint32_t DB = LBITS, uint32_t NL = NLIT, uint32_t NC = NCMD>
struct alignas(16) WarpSmemT {
    uint8_t win[WIN ? WIN : 16];
    uint8_t ring[RB];
    HuffT<LBITS> lit;
    HuffT<DB> dist;
    uint8_t lens[320];
    uint8_t cl_tmp[320];   // code lengths while a dynamic header is read
    uint16_t offs[16];     // canonical code offsets (build_huff)
    BatchT<NL, NC> bt[NB];
    // decoder state shared between lane 0 and the warp
    uint32_t status, done;
    uint32_t produced, consumed;  // pair hand-off counters
};
using WarpSmem = WarpSmemT<0, 1>;

// Windowless form: copies read the output already written (global memory).
// Up to 4 consecutive commands whose sources all lie before the first of
// them -- literal runs, and copies of at most 128 bytes whose distance
// exceeds their offset into the group plus their length -- are executed
// together: every lane issues all of its loads (4 bytes per command) before
// any store, so the group pays one memory latency instead of one per
// command.  Other commands run one at a time.
template <class BatchType>
static __device__ __forceinline__ void execute_batch_out(const BatchType& B, uint32_t pos,
                                                         const uint8_t* __restrict__ src,
                                                         uint8_t* __restrict__ dst) {
    const uint32_t lane = lane_id();
    const uint32_t nc = B.n_cmd;
    uint32_t c = 0;
    while (c < nc) {
        uint32_t tg[4], ag[4], ng[4];
#pragma unroll
        for (uint32_t i = 0; i < 4; ++i) {
            const bool ok = c + i < nc;
            tg[i] = ok ? B.cmd_t[c + i] : (uint32_t)C_STORED;
            ag[i] = ok ? B.cmd_a[c + i] : 0u;
            ng[i] = ok ? B.cmd_b[c + i] : 0u;
        }
        uint32_t g = 0, off = 0;
#pragma unroll
        for (uint32_t i = 0; i < 4; ++i) {
            const bool fits = ng[i] <= 128u && (tg[i] == C_LIT || (tg[i] == C_COPY && ag[i] >= off + ng[i]));
            if (g == i && fits) {
                g = i + 1;
                off += ng[i];
            }
        }
        if (g >= 2) {
            uint8_t v[4][4];
            uint32_t o = 0;
#pragma unroll
            for (uint32_t i = 0; i < 4; ++i) {
#pragma unroll
                for (uint32_t w = 0; w < 4; ++w) {
                    const uint32_t k = lane + 32u * w;
                    v[i][w] = 0;
                    if (i < g && k < ng[i])
                        v[i][w] = tg[i] == C_LIT ? B.lits[ag[i] + k] : dst[pos + o - ag[i] + k];
                }
                o += i < g ? ng[i] : 0u;
            }
            o = 0;
#pragma unroll
            for (uint32_t i = 0; i < 4; ++i) {
#pragma unroll
                for (uint32_t w = 0; w < 4; ++w) {
                    const uint32_t k = lane + 32u * w;
                    if (i < g && k < ng[i]) dst[pos + o + k] = v[i][w];
                }
                o += i < g ? ng[i] : 0u;
            }
            pos += o;
            c += g;
            __syncwarp();
            continue;
        }
        const uint32_t t = tg[0], a = ag[0], n = ng[0];
        uint8_t* d = dst + pos;
        if (t == C_LIT) {
            for (uint32_t k = lane; k < n; k += 32) d[k] = B.lits[a + k];
        } else if (t == C_STORED) {
            const uint8_t* s = src + a;
            for (uint32_t k = lane; k < n; k += 32) d[k] = s[k];
        } else {
            const uint8_t* s = d - a;
            if (a >= 128) {  // 128-byte waves: one latency per 128 bytes
                for (uint32_t k0 = 0; k0 < n; k0 += 128) {
                    uint8_t v[4];
#pragma unroll
                    for (uint32_t w = 0; w < 4; ++w) {
                        const uint32_t k = k0 + lane + 32u * w;
                        v[w] = k < n ? s[k] : (uint8_t)0;
                    }
                    __syncwarp();
#pragma unroll
                    for (uint32_t w = 0; w < 4; ++w) {
                        const uint32_t k = k0 + lane + 32u * w;
                        if (k < n) d[k] = v[w];
                    }
                    __syncwarp();
                }
            } else if (a >= 32) {
                for (uint32_t k0 = 0; k0 < n; k0 += 32) {
                    const uint32_t k = k0 + lane;
                    uint8_t v = 0;
                    if (k < n) v = s[k];
                    __syncwarp();
                    if (k < n) d[k] = v;
                    __syncwarp();
                }
            } else {
                for (uint32_t k = lane; k < n; k += 32) d[k] = s[k % a];
            }
        }
        pos += n;
        ++c;
        __syncwarp();
    }
}

// Write batch B (output starting at pos) with the calling warp.
template <uint32_t WIN, class BatchType>
static __device__ __forceinline__ void execute_batch(const BatchType& B, uint32_t pos, uint8_t* win,
                                                     const uint8_t* __restrict__ src, uint8_t* __restrict__ dst) {
    const uint32_t lane = lane_id();
    const uint32_t nc = B.n_cmd;
    if constexpr (WIN == 0) {
        execute_batch_out(B, pos, src, dst);
        return;
    }
    // the next command's fields are loaded before the current one is written
    uint32_t tn = nc ? B.cmd_t[0] : 0u, an = nc ? B.cmd_a[0] : 0u, nn = nc ? B.cmd_b[0] : 0u;
    for (uint32_t c = 0; c < nc; ++c) {
        const uint32_t t = tn, a = an, n = nn;
        if (c + 1 < nc) {
            tn = B.cmd_t[c + 1];
            an = B.cmd_a[c + 1];
            nn = B.cmd_b[c + 1];
        }
        uint8_t* d = dst + pos;
        if constexpr (WIN != 0) {
            // every output byte also goes to the window; copies read it there
            constexpr uint32_t M = WIN - 1;
            if (t == C_LIT) {
                for (uint32_t k = lane; k < n; k += 32) {
                    const uint8_t v = B.lits[a + k];
                    d[k] = v;
                    win[(pos + k) & M] = v;
                }
            } else if (t == C_STORED) {
                const uint8_t* s = src + a;
                for (uint32_t k = lane; k < n; k += 32) {
                    const uint8_t v = s[k];
                    d[k] = v;
                    win[(pos + k) & M] = v;
                }
            } else if (WIN < 32768u && a > WIN) {
                // a window smaller than the Deflate window: farther sources
                // are read from the output (written long before this wave)
                const uint8_t* s = d - a;
                for (uint32_t k0 = 0; k0 < n; k0 += 128) {
                    uint8_t v[4];
#pragma unroll
                    for (uint32_t i = 0; i < 4; ++i) {
                        const uint32_t k = k0 + lane + 32u * i;
                        v[i] = k < n ? s[k] : (uint8_t)0;
                    }
                    __syncwarp();
#pragma unroll
                    for (uint32_t i = 0; i < 4; ++i) {
                        const uint32_t k = k0 + lane + 32u * i;
                        if (k < n) {
                            d[k] = v[i];
                            win[(pos + k) & M] = v[i];
                        }
                    }
                    __syncwarp();
                }
            } else if (a >= 128) {
                // 128-byte waves (four bytes a lane): with distance >= 128 a
                // wave reads only bytes written before it
                const uint32_t sp = pos - a;
                for (uint32_t k0 = 0; k0 < n; k0 += 128) {
                    uint8_t v[4];
#pragma unroll
                    for (uint32_t i = 0; i < 4; ++i) {
                        const uint32_t k = k0 + lane + 32u * i;
                        v[i] = k < n ? win[(sp + k) & M] : (uint8_t)0;
                    }
                    __syncwarp();
#pragma unroll
                    for (uint32_t i = 0; i < 4; ++i) {
                        const uint32_t k = k0 + lane + 32u * i;
                        if (k < n) {
                            d[k] = v[i];
                            win[(pos + k) & M] = v[i];
                        }
                    }
                    __syncwarp();
                }
            } else if (a >= 32) {
                // 32-byte waves: a wave reads bytes written before it (earlier
                // waves or earlier commands) and writes after every lane has read
                const uint32_t sp = pos - a;
                for (uint32_t k0 = 0; k0 < n; k0 += 32) {
                    const uint32_t k = k0 + lane;
                    uint8_t v = 0;
                    if (k < n) v = win[(sp + k) & M];
                    __syncwarp();
                    if (k < n) {
                        d[k] = v;
                        win[(pos + k) & M] = v;
                    }
                    __syncwarp();
                }
            } else {
                // distance < 32: the copy repeats the a bytes before it
                const uint32_t sp = pos - a;
                for (uint32_t k = lane; k < n; k += 32) {
                    const uint8_t v = win[(sp + k % a) & M];
                    d[k] = v;
                    win[(pos + k) & M] = v;
                }
            }
        }
        pos += n;
        __syncwarp();
    }
}

// Hand-off between the two warps of a pair: counters in shared memory.
// produced = batches the decoder has filled, consumed = batches the writer
// has executed.  Every wait is bounded (by default 2^25 polls, about a
// second; GD_TUNE_INFLATE_PAIR_SPIN sets it): on expiry the waiter reports
// GD_ERR_TIMEOUT and both warps still leave.
constexpr uint32_t PAIR_SPIN_LIMIT = 1u << 25;

// Wait (lane 0 spins, the warp follows) until *ctr >= target, polling at
// most `limit` times; false on expiry.
__device__ __forceinline__ bool pair_wait(const uint32_t* ctr, uint32_t target, uint32_t limit) {
    uint32_t ok = 1;
    if (lane_id() == 0) {
        uint32_t it = 0;
        while (*reinterpret_cast<const volatile uint32_t*>(ctr) < target) {
            if (++it > limit) {
                ok = 0;
                break;
            }
            __nanosleep(32);
        }
        __threadfence_block();  // the batch written before the counter is visible
    }
    return __shfl_sync(GD_FULL_MASK, ok, 0) != 0;
}

// Publish *ctr = value after this warp's earlier shared-memory writes.
__device__ __forceinline__ void pair_post(uint32_t* ctr, uint32_t value) {
    __syncwarp();
    if (lane_id() == 0) {
        __threadfence_block();
        *reinterpret_cast<volatile uint32_t*>(ctr) = value;
    }
    __syncwarp();
}

// Lookup-table entries carry what the decoder needs next, so a length or
// distance needs no second table lookup:
//   bits 0-3 code length (0 = longer than LBITS: canonical walk), 4-7 extra
//   bits, 8-23 value, 24-31 kind.
// Table kinds: TK_PLAIN (code-length code: value = symbol), TK_LIT
// (literal/length: E_LIT value = byte, E_LEN value = length base, E_EOB,
// E_BAD), TK_DIST (E_DIST value = distance base, E_BAD).
enum : uint32_t { TK_PLAIN = 0, TK_LIT = 1, TK_DIST = 2 };
enum : uint32_t { E_LIT = 0, E_LEN = 1, E_EOB = 2, E_DIST = 3, E_BAD = 4 };

__device__ __forceinline__ uint32_t make_entry(uint32_t tk, uint32_t sym, uint32_t L) {
    uint32_t kind = E_LIT, value = sym, extra = 0;
    if (tk == TK_LIT) {
        if (sym == 256) {
            kind = E_EOB;
        } else if (sym > 256) {
            if (sym > 285) {
                kind = E_BAD;
            } else {
                kind = E_LEN;
                value = LBASE[sym - 257];
                extra = LEXT[sym - 257];
            }
        }
    } else if (tk == TK_DIST) {
        if (sym > 29) {
            kind = E_BAD;
        } else {
            kind = E_DIST;
            value = DBASE[sym];
            extra = DEXT[sym];
        }
    }
    return L | (extra << 4) | (value << 8) | (kind << 24);
}

// Build `h` from code lengths lens[0..n) for table kind tk.  Counting /
// offsets on lane 0, the primary table fill spread over the warp.  Returns
// false (on every lane) for an over-subscribed or otherwise unusable code.
template <uint32_t BITS>
static __device__ bool build_huff(HuffT<BITS>* h, const uint8_t* lens, uint32_t n, uint32_t* sh_flag, uint16_t* offs,
                                  uint32_t tk) {
    const uint32_t lane = lane_id();
    for (uint32_t i = lane; i < (1u << BITS); i += 32) h->lut[i] = 0xffffffffu;
    if (lane == 0) {
        for (int i = 0; i < 16; ++i) h->count[i] = 0;
        for (uint32_t s = 0; s < n; ++s) h->count[lens[s]]++;
        int left = 1;
        bool ok = true;
        for (int L = 1; L < 16; ++L) {
            left <<= 1;
            left -= h->count[L];
            if (left < 0) ok = false;
        }
        offs[1] = 0;
        for (int L = 1; L < 15; ++L) offs[L + 1] = offs[L] + h->count[L];
        for (uint32_t s = 0; s < n; ++s)
            if (lens[s]) h->sym[offs[lens[s]]++] = (uint16_t)s;
        *sh_flag = ok ? 1u : 0u;
    }
    __syncwarp();
    if (!*sh_flag) return false;
    // canonical codes in symbol order: code(s) = first(len) + rank among equal lengths
    // lane-parallel: every lane walks the sorted symbol list for a subset of lengths
    for (uint32_t L = 1 + lane; L <= BITS; L += 32) {
        uint32_t first = 0, idx = 0;
        uint32_t code = 0;
        for (uint32_t l = 1; l < L; ++l) {
            code = (code + h->count[l]) << 1;
            idx += h->count[l];
        }
        first = code;
        for (uint32_t k = 0; k < h->count[L]; ++k) {
            const uint32_t c = first + k;
            // deflate sends codes MSB first into an LSB-first stream: reverse
            const uint32_t rev = __brev(c) >> (32 - L);
            const uint32_t entry = make_entry(tk, h->sym[idx + k], L);
            for (uint32_t f = rev; f < (1u << BITS); f += (1u << L)) h->lut[f] = entry;
        }
    }
    __syncwarp();
    // prefixes of codes longer than BITS: mark for the canonical walk
    for (uint32_t L = BITS + 1 + lane; L < 16; L += 32) {
        uint32_t code = 0, idx = 0;
        for (uint32_t l = 1; l < L; ++l) {
            code = (code + h->count[l]) << 1;
            idx += h->count[l];
        }
        for (uint32_t k = 0; k < h->count[L]; ++k) {
            const uint32_t c = code + k;
            const uint32_t pre = __brev(c >> (L - BITS)) >> (32 - BITS);
            atomicExch(&h->lut[pre], 0u);  // len 0: walk
        }
    }
    __syncwarp();
    return true;
}

// Inflate one stream with the calling warp.  src: clen compressed bytes
// (the 16-byte-aligned span around them must be readable); dst: room for
// olen bytes; hdr: 0 raw deflate, 1 zlib, 2 gzip; S: this warp's shared
// state.  Returns a gd status (same on every lane); *written = bytes output.
// stream_warp_impl is inlined into the caller, so the compiler sees that S is
// shared memory and uses shared-memory loads and stores throughout;
// stream_warp is the out-of-line form for kernels that run several decoders.
// NB = 2 (decoder of a pair): instead of executing a batch, hand it to the
// writer warp (see stream_pair_writer); S.produced / S.consumed must be 0.
template <uint32_t WIN, int NB = 1, uint32_t RB = IRING, uint32_t DB = LBITS, uint32_t NL = NLIT, uint32_t NC = NCMD>
static __device__ __forceinline__ uint32_t stream_warp_impl(const uint8_t* __restrict__ src, uint32_t clen,
                                                            uint8_t* __restrict__ dst, uint32_t olen, int zlib_hdr,
                                                            WarpSmemT<WIN, NB, RB, DB, NL, NC>& S, uint32_t* written,
                                                            uint32_t spin_limit = PAIR_SPIN_LIMIT) {
    static_assert(RB >= 1024 && (RB & (RB - 1)) == 0, "input ring: a power of two >= 1 KiB");
    // a window below the Deflate window's 32 KiB serves the nearer copies;
    // the executor reads farther ones from the output
    static_assert(WIN == 0 || (WIN >= 2048 && (WIN & (WIN - 1)) == 0), "window: 0 or a power of two >= 2 KiB");
    const uint32_t lane = lane_id();
    uint32_t err = ST_OK;
    // input ring: compressed byte i (chunk-relative) at ring[(i + sh) % RB];
    // fills are 16-byte aligned global loads.
    const uint32_t sh = (uint32_t)(reinterpret_cast<uintptr_t>(src) & 15u);
    const uint8_t* src_al = src - sh;
    const uint32_t span = clen + sh;  // bytes of the aligned view we may touch
    uint32_t fill = 0;                // aligned-view bytes loaded so far
    auto refill = [&](uint32_t consumed_al) {
        // load the aligned view up to consumed_al + RB (whole 16-byte words,
        // plus the ragged end of the chunk once it is reached)
        uint32_t target = min(consumed_al + RB, span);
        if (target < span) target &= ~15u;
        if (target > fill) {
            const uint32_t a = fill, b = target & ~15u;
            for (uint32_t i = a + 16 * lane; i + 16 <= b; i += 512) {
                const uint4 v = *reinterpret_cast<const uint4*>(src_al + i);
                *reinterpret_cast<uint4*>(S.ring + (i & (RB - 1))) = v;
            }
            for (uint32_t i = max(a, b) + lane; i < target; i += 32)
                if (i >= sh) S.ring[i & (RB - 1)] = src_al[i];
            fill = target;
        }
        __syncwarp();
    };

    // ---- lane-0 decoder state ----
    uint64_t bitbuf = 0;
    uint32_t bitcnt = 0;
    uint32_t inpos = sh;     // next aligned-view byte to move into bitbuf
    uint32_t opos = 0;       // output bytes committed by decoded commands
    uint32_t bfinal = 0, btype = 0xff, in_block = 0;

    if (lane == 0) {
        S.status = err;
        S.done = 0;
    }
    __syncwarp();
    refill(0);
    if (lane == 0 && err == ST_OK && zlib_hdr == 1) {
        // zlib (RFC 1950): CMF, FLG; no preset dictionary
        if (clen < 2) err = ST_CORRUPT;
        else {
            const uint32_t cmf = S.ring[(sh + 0) & (RB - 1)], flg = S.ring[(sh + 1) & (RB - 1)];
            if ((cmf & 15u) != 8u || ((cmf << 8) | flg) % 31u != 0 || (flg & 32u)) err = ST_CORRUPT;
            inpos += 2;
        }
        S.status = err;
    } else if (lane == 0 && err == ST_OK && zlib_hdr == 2) {
        // gzip (RFC 1952) member header; the 8-byte trailer is not read
        auto at = [&](uint32_t i) -> uint32_t { return i < clen && sh + i < fill ? S.ring[(sh + i) & (RB - 1)] : 0x100u; };
        uint32_t p = 10;
        if (at(0) != 0x1fu || at(1) != 0x8bu || at(2) != 8u || clen < 18) err = ST_CORRUPT;
        const uint32_t flg = at(3);
        if (err == ST_OK && (flg & 4u)) {  // FEXTRA
            const uint32_t xl = at(p) | (at(p + 1) << 8);
            p += 2 + xl;
        }
        if (err == ST_OK && (flg & 8u)) {  // FNAME
            while (p < clen && at(p) != 0) { if (at(p) > 0xffu) { err = ST_CORRUPT; break; } ++p; }
            ++p;
        }
        if (err == ST_OK && (flg & 16u)) {  // FCOMMENT
            while (p < clen && at(p) != 0) { if (at(p) > 0xffu) { err = ST_CORRUPT; break; } ++p; }
            ++p;
        }
        if (err == ST_OK && (flg & 2u)) p += 2;  // FHCRC
        if (err == ST_OK && p + 8 > clen) err = ST_CORRUPT;
        inpos += p;
        S.status = err;
    }
    __syncwarp();
    err = S.status;

    // lane-0 helpers ------------------------------------------------------
    auto need_bits = [&](uint32_t n) -> bool {
        while (bitcnt < n) {
            if (inpos >= fill) return false;
            bitbuf |= (uint64_t)S.ring[inpos & (RB - 1)] << bitcnt;
            ++inpos;
            bitcnt += 8;
        }
        return true;
    };
    // top up bitbuf: single bytes up to a 4-byte boundary of the stream,
    // then one aligned 32-bit word per call (the ring is word aligned and
    // RB a multiple of 4), single bytes again at the end of the input
    auto fill_bits = [&]() {
        while (bitcnt <= 56 && inpos < fill && (inpos & 3u)) {
            bitbuf |= (uint64_t)S.ring[inpos & (RB - 1)] << bitcnt;
            ++inpos;
            bitcnt += 8;
        }
        if (bitcnt <= 32 && (inpos & 3u) == 0 && inpos + 4 <= fill) {
            const uint32_t w = *reinterpret_cast<const uint32_t*>(S.ring + (inpos & (RB - 1)));
            bitbuf |= (uint64_t)w << bitcnt;
            inpos += 4;
            bitcnt += 32;
        }
        while (bitcnt <= 56 && inpos < fill && inpos + 4 > fill) {
            bitbuf |= (uint64_t)S.ring[inpos & (RB - 1)] << bitcnt;
            ++inpos;
            bitcnt += 8;
        }
    };
    auto get_bits = [&](uint32_t n, uint32_t& v) -> bool {
        if (!need_bits(n)) return false;
        v = (uint32_t)(bitbuf & ((1ull << n) - 1ull));
        bitbuf >>= n;
        bitcnt -= n;
        return true;
    };
    // decode one symbol of code h; returns false on exhausted input / bad code
    // canonical walk (puff-style) for codes longer than LBITS
    auto walk = [&](const auto* h, uint32_t& sym) -> bool {
        int code = 0, first = 0, index = 0;
        uint64_t bb = bitbuf;
        for (uint32_t L = 1; L < 16; ++L) {
            if (L > bitcnt) return false;
            code |= (int)(bb & 1u);
            bb >>= 1;
            const int cnt = h->count[L];
            if (code - cnt < first) {
                sym = h->sym[index + (code - first)];
                bitbuf >>= L;
                bitcnt -= L;
                return true;
            }
            index += cnt;
            first += cnt;
            first <<= 1;
            code <<= 1;
        }
        return false;
    };
    // decode one entry of table h (kind tk); false on exhausted input / bad code
    auto decode_ent = [&](const auto* h, uint32_t tk, uint32_t& e) -> bool {
        fill_bits();
        e = h->lut[bitbuf & (uint64_t)(sizeof(h->lut) / 4 - 1)];
        const uint32_t L = e & 15u;
        if (e != 0xffffffffu && L != 0) {
            if (L > bitcnt) return false;
            bitbuf >>= L;
            bitcnt -= L;
            return true;
        }
        if (e == 0xffffffffu) return false;
        uint32_t sym;
        if (!walk(h, sym)) return false;
        e = make_entry(tk, sym, 0);
        return true;
    };
    // one symbol of a plain table (the code-length code)
    auto decode_sym = [&](const auto* h, uint32_t& sym) -> bool {
        uint32_t e;
        if (!decode_ent(h, TK_PLAIN, e)) return false;
        sym = (e >> 8) & 0xffffu;
        return true;
    };

    uint32_t* sflag = &S.done;  // scratch word for build_huff's broadcast (restored below)
    // main loop ------------------------------------------------------------
    uint32_t kb = 0;  // batches handed off (pairs: the buffer is bt[kb & 1])
    while (err == ST_OK) {
        auto& BT = S.bt[NB == 2 ? (kb & 1u) : 0u];
        // pairs: the buffer's previous batch (kb - 2) must have been executed
        if constexpr (NB == 2) {
            if (kb >= 2 && !pair_wait(&S.consumed, kb - 1, spin_limit)) {
                err = ST_TIMEOUT;
                break;
            }
        }
        // ---- refill input for the decoder (warp) ----
        uint32_t inpos_b = __shfl_sync(GD_FULL_MASK, inpos, 0);
        refill(inpos_b > 64 ? inpos_b - 64 : 0);

        // ---- block header (table builds need the warp) ----
        uint32_t hdr_state = 0;  // 0 = none, 1 = fixed, 2 = dynamic lens ready, 3 = stored, 4 = end
        if (lane == 0) {
            BT.n_cmd = 0;
            BT.n_lit = 0;
            if (!in_block) {
                if (bfinal) {
                    hdr_state = 4;
                } else {
                    uint32_t bf, bt;
                    if (!get_bits(1, bf) || !get_bits(2, bt)) err = ST_CORRUPT;
                    bfinal = bf;
                    btype = bt;
                    if (err == ST_OK) {
                        if (bt == 0) {
                            hdr_state = 3;
                        } else if (bt == 1) {
                            for (int i = 0; i < 144; ++i) S.lens[i] = 8;
                            for (int i = 144; i < 256; ++i) S.lens[i] = 9;
                            for (int i = 256; i < 280; ++i) S.lens[i] = 7;
                            for (int i = 280; i < 288; ++i) S.lens[i] = 8;
                            for (int i = 0; i < 30; ++i) S.lens[288 + i] = 5;
                            hdr_state = 1;
                        } else if (bt == 2) {
                            hdr_state = 2;
                        } else {
                            err = ST_CORRUPT;
                        }
                    }
                }
            }
            S.status = err | (hdr_state << 8);
        }
        __syncwarp();
        {
            const uint32_t w = S.status;
            err = w & 0xffu;
            hdr_state = w >> 8;
        }
        if (err != ST_OK || hdr_state == 4) break;

        if (hdr_state == 2) {
            // dynamic: code-length code, then literal/length + distance lengths
            uint32_t nlen = 0, ndist = 0;
            if (lane == 0) {
                uint32_t hlit, hdist, hclen;
                if (!get_bits(5, hlit) || !get_bits(5, hdist) || !get_bits(4, hclen)) err = ST_CORRUPT;
                nlen = hlit + 257;
                ndist = hdist + 1;
                if (nlen > 286 || ndist > 30) err = ST_CORRUPT;
                for (int i = 0; i < 19; ++i) S.lens[i] = 0;
                for (uint32_t i = 0; i < hclen + 4 && err == ST_OK; ++i) {
                    uint32_t v;
                    if (!get_bits(3, v)) err = ST_CORRUPT;
                    S.lens[CLORDER[i]] = (uint8_t)v;
                }
                S.status = err;
            }
            __syncwarp();
            err = S.status;
            if (err != ST_OK) break;
            if (!build_huff(&S.lit, S.lens, 19, sflag, S.offs, TK_PLAIN)) {
                err = ST_CORRUPT;
                break;
            }
            if (lane == 0) {
                // read nlen + ndist code lengths (lens[0..nlen) lit, [288..288+ndist) dist)
                uint8_t* tmp = S.cl_tmp;
                uint32_t i = 0;
                const uint32_t tot = nlen + ndist;
                while (i < tot && err == ST_OK) {
                    uint32_t sym;
                    if (!decode_sym(&S.lit, sym)) {
                        err = ST_CORRUPT;
                        break;
                    }
                    if (sym < 16) {
                        tmp[i++] = (uint8_t)sym;
                    } else {
                        uint32_t rep = 0, v = 0, x;
                        if (sym == 16) {
                            if (i == 0) {
                                err = ST_CORRUPT;
                                break;
                            }
                            v = tmp[i - 1];
                            if (!get_bits(2, x)) err = ST_CORRUPT;
                            rep = 3 + x;
                        } else if (sym == 17) {
                            if (!get_bits(3, x)) err = ST_CORRUPT;
                            rep = 3 + x;
                        } else {
                            if (!get_bits(7, x)) err = ST_CORRUPT;
                            rep = 11 + x;
                        }
                        if (i + rep > tot) err = ST_CORRUPT;
                        for (uint32_t k = 0; k < rep && err == ST_OK; ++k) tmp[i++] = (uint8_t)v;
                    }
                }
                if (err == ST_OK && tmp[256] == 0) err = ST_CORRUPT;  // no end-of-block code
                for (uint32_t k = 0; k < 288; ++k) S.lens[k] = (k < nlen) ? tmp[k] : 0;
                for (uint32_t k = 0; k < 30; ++k) S.lens[288 + k] = (k < ndist) ? tmp[nlen + k] : 0;
                S.status = err;
            }
            __syncwarp();
            err = S.status;
            if (err != ST_OK) break;
        }
        if (hdr_state == 1 || hdr_state == 2) {
            const bool ok1 = build_huff(&S.lit, S.lens, 288, sflag, S.offs, TK_LIT);
            // a distance code with a single used symbol is allowed (incomplete)
            const bool ok2 = ok1 && build_huff(&S.dist, S.lens + 288, 30, sflag, S.offs, TK_DIST);
            if (!ok1 || !ok2) {
                err = ST_CORRUPT;
                break;
            }
            if (lane == 0) in_block = 1;
        }

        // ---- decode a batch of commands (lane 0) ----
        if (lane == 0) {
            uint32_t nc = 0, nl = 0;
            if (hdr_state == 3) {
                // stored block: align to a byte, LEN / NLEN
                const uint32_t drop = bitcnt & 7u;
                bitbuf >>= drop;
                bitcnt -= drop;
                uint32_t ln, nln;
                if (!get_bits(16, ln) || !get_bits(16, nln) || (ln ^ 0xffffu) != nln) err = ST_CORRUPT;
                // the bytes still in bitbuf come first
                uint32_t avail_bytes = bitcnt >> 3;
                if (err == ST_OK) {
                    if (opos + ln > olen) err = ST_OVERRUN;
                    const uint32_t from_buf = min(avail_bytes, ln);
                    for (uint32_t k = 0; k < from_buf && err == ST_OK; ++k) {
                        BT.lits[nl++] = (uint8_t)(bitbuf & 0xffu);
                        bitbuf >>= 8;
                        bitcnt -= 8;
                    }
                    if (from_buf && err == ST_OK) {
                        BT.cmd_t[nc] = C_LIT;
                        BT.cmd_a[nc] = 0;
                        BT.cmd_b[nc] = from_buf;
                        ++nc;
                    }
                    const uint32_t rest = ln - from_buf;
                    if (err == ST_OK && rest) {
                        // remaining bytes straight from global (aligned-view offset inpos)
                        if (inpos + rest > span) err = ST_CORRUPT;
                        // the stored bytes are read from global: skip them in the ring
                        if (fill < inpos + rest) fill = max(fill, (inpos + rest) & ~15u);
                        BT.cmd_t[nc] = C_STORED;
                        BT.cmd_a[nc] = inpos - sh;
                        BT.cmd_b[nc] = rest;
                        ++nc;
                        inpos += rest;
                    }
                    opos += ln;
                }
            } else {
                // Huffman-coded symbols until the batch is full or the block ends.
                // Literals accumulate in a run that becomes one command when a
                // copy or the end of the batch closes it.
                uint32_t run = 0, run_start = nl;
                // fast loop while enough input is buffered: the bit buffer is
                // topped up from one aligned ring word at a time, codes of
                // <= LBITS bits decode with one lookup (a literal entry is any
                // nonzero value below 2^24), rounds of symbols run without
                // per-symbol capacity checks (a symbol reads <= 6 input bytes
                // and adds <= 2 commands and <= 1 literal), the output bound
                // is checked once per batch (below), and anything else --
                // long codes, end of block, invalid entries -- falls to the
                // checked loop with the bit state untouched
                {
                    const uint32_t* r32 = reinterpret_cast<const uint32_t*>(S.ring);
                    constexpr uint32_t RW = RB / 4 - 1;
                    // align the next ring load to a word
                    while ((inpos & 3u) && bitcnt <= 56 && fill - inpos >= 16) {
                        bitbuf |= (uint64_t)S.ring[inpos & (RB - 1)] << bitcnt;
                        ++inpos;
                        bitcnt += 8;
                    }
                    bool fall = (inpos & 3u) != 0;
                    while (!fall && err == ST_OK) {
                        uint32_t budget = min((NC - 2 - nc) / 2, NL - nl);
                        budget = min(budget, fill - inpos >= 24 ? (fill - inpos - 16) / 6 : 0u);
                        if (budget == 0) break;
                        for (; budget; --budget) {
                            if (bitcnt <= 32) {
                                bitbuf |= (uint64_t)r32[(inpos >> 2) & RW] << bitcnt;
                                bitcnt += 32;
                                inpos += 4;
                            }
                            const uint32_t e = S.lit.lut[(uint32_t)bitbuf & ((1u << LBITS) - 1u)];
                            if (e - 1u < 0xffffffu) {  // literal
                                const uint32_t L = e & 15u;
                                bitbuf >>= L;
                                bitcnt -= L;
                                BT.lits[nl++] = (uint8_t)(e >> 8);
                                ++run;
                                ++opos;
                                continue;
                            }
                            const uint32_t L = e & 15u;
                            if ((e >> 24) != E_LEN || L == 0) {  // walk / end of block / bad: checked loop
                                fall = true;
                                break;
                            }
                            // length: its extra bits are in the buffer (>= 33 - 10 bits left)
                            const uint32_t ex = (e >> 4) & 15u;
                            const uint64_t b1 = bitbuf >> L;
                            const uint32_t len = ((e >> 8) & 0xffffu) + ((uint32_t)b1 & ((1u << ex) - 1u));
                            uint64_t b2 = b1 >> ex;
                            uint32_t c2 = bitcnt - L - ex;
                            const bool top = c2 <= 32;
                            if (top) {
                                b2 |= (uint64_t)r32[(inpos >> 2) & RW] << c2;
                                c2 += 32;
                            }
                            const uint32_t ed = S.dist.lut[(uint32_t)b2 & ((1u << DB) - 1u)];
                            const uint32_t Ld = ed & 15u;
                            if (Ld == 0 || (ed >> 24) != E_DIST) {  // long / bad distance code: checked loop
                                fall = true;
                                break;
                            }
                            if (top) inpos += 4;
                            const uint32_t exd = (ed >> 4) & 15u;
                            const uint64_t b3 = b2 >> Ld;
                            const uint32_t dist = ((ed >> 8) & 0xffffu) + ((uint32_t)b3 & ((1u << exd) - 1u));
                            if (dist > opos) {
                                err = ST_CORRUPT;
                                break;
                            }
                            bitbuf = b3 >> exd;
                            bitcnt = c2 - Ld - exd;
                            if (run) {
                                BT.cmd_t[nc] = C_LIT;
                                BT.cmd_a[nc] = nl - run;
                                BT.cmd_b[nc] = run;
                                ++nc;
                                run = 0;
                            }
                            BT.cmd_t[nc] = C_COPY;
                            BT.cmd_a[nc] = dist;
                            BT.cmd_b[nc] = len;
                            ++nc;
                            opos += len;
                        }
                    }
                    run_start = nl - run;  // the open literal run, for the checked loop
                }
                while (err == ST_OK && nc < NC - 2 && nl < NL && (fill - inpos >= 32 || fill >= span)) {
                    uint32_t e;
                    if (!decode_ent(&S.lit, TK_LIT, e)) {
                        err = ST_CORRUPT;
                        break;
                    }
                    const uint32_t kind = e >> 24;
                    if (kind == E_LIT) {
                        if (opos >= olen) {
                            err = ST_OVERRUN;
                            break;
                        }
                        if (run == 0) run_start = nl;
                        BT.lits[nl++] = (uint8_t)(e >> 8);
                        ++run;
                        ++opos;
                        continue;
                    }
                    if (run) {
                        BT.cmd_t[nc] = C_LIT;
                        BT.cmd_a[nc] = run_start;
                        BT.cmd_b[nc] = run;
                        ++nc;
                        run = 0;
                    }
                    if (kind == E_EOB) {
                        in_block = 0;
                        break;
                    }
                    if (kind != E_LEN) {
                        err = ST_CORRUPT;
                        break;
                    }
                    uint32_t x, ed;
                    if (!get_bits((e >> 4) & 15u, x)) {
                        err = ST_CORRUPT;
                        break;
                    }
                    const uint32_t len = ((e >> 8) & 0xffffu) + x;
                    if (!decode_ent(&S.dist, TK_DIST, ed) || (ed >> 24) != E_DIST || !get_bits((ed >> 4) & 15u, x)) {
                        err = ST_CORRUPT;
                        break;
                    }
                    const uint32_t dist = ((ed >> 8) & 0xffffu) + x;
                    if (dist > opos) {
                        err = ST_CORRUPT;
                        break;
                    }
                    if (opos + len > olen) {
                        err = ST_OVERRUN;
                        break;
                    }
                    BT.cmd_t[nc] = C_COPY;
                    BT.cmd_a[nc] = dist;
                    BT.cmd_b[nc] = len;
                    ++nc;
                    opos += len;
                }
                if (run) {
                    BT.cmd_t[nc] = C_LIT;
                    BT.cmd_a[nc] = run_start;
                    BT.cmd_b[nc] = run;
                    ++nc;
                }
                // the fast loop does not bound the output per symbol: a batch
                // that would write past the end is not executed
                if (err == ST_OK && opos > olen) err = ST_OVERRUN;
            }
            BT.n_cmd = nc;
            BT.n_lit = nl;
            S.status = err;
        }
        __syncwarp();
        err = S.status;
        fill = __shfl_sync(GD_FULL_MASK, fill, 0);
        if (err != ST_OK) break;

        // ---- execute the batch (all lanes), or hand it to the writer ----
        const uint32_t nc = BT.n_cmd;
        uint32_t pos = __shfl_sync(GD_FULL_MASK, opos, 0);
        // pos is the end position after the batch; walk back to its start
        {
            uint32_t tot = 0;
            for (uint32_t c = lane; c < nc; c += 32) tot += BT.cmd_b[c];
            for (int o = 16; o; o >>= 1) tot += __shfl_xor_sync(GD_FULL_MASK, tot, o);
            pos -= tot;
        }
        if constexpr (NB == 2) {
            if (lane == 0) {
                BT.pos0 = pos;
                BT.last = 0;
            }
            pair_post(&S.produced, kb + 1);
            ++kb;
        } else {
            execute_batch<WIN>(BT, pos, S.win, src, dst);
        }
    }
    if constexpr (NB == 2) {  // the final (empty) hand-off
        if (err != ST_TIMEOUT && kb >= 2 && !pair_wait(&S.consumed, kb - 1, spin_limit)) err = ST_TIMEOUT;
        auto& BT = S.bt[kb & 1u];
        if (lane == 0) {
            BT.n_cmd = 0;
            BT.last = 1;
        }
        pair_post(&S.produced, kb + 1);
    }
    const uint32_t fin = __shfl_sync(GD_FULL_MASK, opos, 0);
    *written = fin;
    return __shfl_sync(GD_FULL_MASK, err, 0);
}

template <uint32_t WIN, uint32_t RB = IRING, uint32_t DB = LBITS, uint32_t NL = NLIT, uint32_t NC = NCMD>
static __device__ __noinline__ uint32_t stream_warp(const uint8_t* __restrict__ src, uint32_t clen,
                                                    uint8_t* __restrict__ dst, uint32_t olen, int zlib_hdr,
                                                    WarpSmemT<WIN, 1, RB, DB, NL, NC>& S, uint32_t* written) {
    return stream_warp_impl<WIN, 1, RB, DB, NL, NC>(src, clen, dst, olen, zlib_hdr, S, written);
}

// Writer warp of a pair: executes batch k while the decoder warp (running
// stream_warp_impl<WIN, 2> on the same S) decodes batch k+1.  The decoder's
// last hand-off is an empty batch marked last (also after an error).
// Returns GD_ERR_TIMEOUT if a wait expired, else OK.  stop_after > 0 (a test
// setting) makes the writer leave after that many batches without posting
// more, so that the decoder's bounded wait is exercised.
template <uint32_t WIN, uint32_t RB = IRING, uint32_t DB = LBITS, uint32_t NL = NLIT, uint32_t NC = NCMD>
static __device__ __forceinline__ uint32_t stream_pair_writer(WarpSmemT<WIN, 2, RB, DB, NL, NC>& S,
                                                              const uint8_t* __restrict__ src,
                                                              uint8_t* __restrict__ dst, uint32_t spin_limit,
                                                              uint32_t stop_after) {
    for (uint32_t kb = 0;; ++kb) {
        if (stop_after && kb >= stop_after) return ST_OK;  // the decoder's wait will run out
        if (!pair_wait(&S.produced, kb + 1, spin_limit)) return ST_TIMEOUT;
        auto& BT = S.bt[kb & 1u];
        if (BT.last) return ST_OK;
        execute_batch<WIN>(BT, BT.pos0, S.win, src, dst);
        pair_post(&S.consumed, kb + 1);
    }
}

}  // namespace infl
}  // namespace gd
