// interleave.cuh -- warp-level reader for the 32-slot, 4-byte-word
// interleaved block layout shared by the RLE v1, RLE v2 and LZSS containers.
//
// Layout (rle_v1/encoder.h:564-588, rlev2/encoder_trans.h:291-349,
// lzss/lzss_gpu2.h:497-509): row k of a block holds one 4-byte word of every
// slot whose stream is longer than 4k bytes, in slot order.  A slot is a lane
// (RLE v1/v2) or a length rank (LZSS).
//
// The rows fall into at most 32 segments with a constant active set: sort the
// slots' word counts nw; rows [sorted[j-1], sorted[j]) have exactly the slots
// of rank >= j active (32-j words per row).  With that table a lane computes
// the block offset of any of its words in O(1), so each lane streams its own
// words into a private shared-memory ring; all 32 lanes issue their loads
// together (row-local, hence mostly coalesced) in a warp-wide refill.
#pragma once
#include "gd_common.cuh"

namespace gd {

constexpr int RING = 256;          // bytes of input ring per lane
constexpr int RING_STRIDE = 260;   // padded so lanes at equal offsets hit distinct banks
constexpr int RING_LOW = 64;       // refill when fewer bytes than this are buffered

struct SegTable {
    uint32_t hi[32];    // rows of segment j end at hi[j] (= sorted word count j)
    uint32_t base[32];  // byte offset of row hi[j-1] (segment start) in the block
    uint32_t mask[32];  // active slots in segment j
};

// Build the segment table for a block.  nw = this lane's word count.
// Every lane of the warp must call it.
__device__ __forceinline__ void seg_build(SegTable* T, uint32_t nw) {
    const uint32_t l = lane_id();
    uint32_t rank = 0;
#pragma unroll 8
    for (int s = 0; s < 32; ++s) {
        uint32_t o = __shfl_sync(GD_FULL_MASK, nw, s);
        rank += (o < nw) || (o == nw && (uint32_t)s < l);
    }
    T->hi[rank] = nw;
    __syncwarp();
    uint32_t my_mask = 0;
#pragma unroll 8
    for (int j = 0; j < 32; ++j) {
        uint32_t m = __ballot_sync(GD_FULL_MASK, rank >= (uint32_t)j);
        if ((uint32_t)j == l) my_mask = m;
    }
    const uint32_t hi = T->hi[l];
    const uint32_t lo = l ? T->hi[l - 1] : 0u;
    const uint32_t bytes = (hi - lo) * 4u * (32u - l);
    const uint32_t inc = warp_incl_scan(bytes);
    T->base[l] = inc - bytes;
    T->mask[l] = my_mask;
    __syncwarp();
}

// Per-lane cursor over the lane's words in the block.
struct LaneWords {
    uint32_t k;      // next word to load
    uint32_t nw;     // words in this lane's stream
    uint32_t j;      // current segment
    uint32_t lo, hi; // rows of segment j
    uint32_t row_bytes, pre, base;
};

__device__ __forceinline__ void lw_seek_seg_to(LaneWords& w, const SegTable* T, uint32_t ltmask, uint32_t k) {
    while (w.j < 31 && k >= T->hi[w.j]) ++w.j;
    w.lo = w.j ? T->hi[w.j - 1] : 0u;
    w.hi = T->hi[w.j];
    w.row_bytes = 4u * (32u - w.j);
    w.pre = 4u * __popc(T->mask[w.j] & ltmask);
    w.base = T->base[w.j];
}

__device__ __forceinline__ void lw_seek_seg(LaneWords& w, const SegTable* T, uint32_t ltmask) {
    lw_seek_seg_to(w, T, ltmask, w.k);
}

// Block offset of word kk (kk >= every word asked for before).
__device__ __forceinline__ uint32_t lw_addr(LaneWords& w, const SegTable* T, uint32_t ltmask, uint32_t kk) {
    if (kk >= w.hi) lw_seek_seg_to(w, T, ltmask, kk);
    return w.base + (kk - w.lo) * w.row_bytes + w.pre;
}

__device__ __forceinline__ void lw_init(LaneWords& w, const SegTable* T, uint32_t nw) {
    w.k = 0;
    w.nw = nw;
    w.j = 0;
    lw_seek_seg(w, T, (1u << lane_id()) - 1u);
}

// Block offset of word k of this lane (random access; binary search).
__device__ __forceinline__ uint32_t word_offset_at(const SegTable* T, uint32_t k) {
    uint32_t j = 0;
#pragma unroll
    for (uint32_t step = 16; step; step >>= 1)
        if (j + step <= 31 && T->hi[j + step - 1] <= k) j += step;
    const uint32_t lo = j ? T->hi[j - 1] : 0u;
    return T->base[j] + (k - lo) * 4u * (32u - j) + 4u * __popc(T->mask[j] & ((1u << lane_id()) - 1u));
}

// Input ring of one lane: bytes [rd, fl) of the lane stream are buffered at
// ring[pos % RING].
struct LaneRing {
    uint8_t* buf;   // this lane's ring (RING bytes, 4-byte aligned)
    uint32_t rd;    // next byte to consume
    uint32_t fl;    // bytes loaded
    uint32_t len;   // stream length in bytes
};

__device__ __forceinline__ uint32_t ring_byte(const LaneRing& r, uint32_t pos) { return r.buf[pos & (RING - 1)]; }

// Warp-wide refill: every lane tops up its ring.  Must be called by all lanes.
__device__ __forceinline__ void ring_refill(LaneRing& r, LaneWords& w, const SegTable* T, const uint8_t* block) {
    const uint32_t ltmask = (1u << lane_id()) - 1u;
    uint32_t room = (RING - (r.fl - r.rd)) >> 2;
    uint32_t n = min(room, w.nw - w.k);
    while (n) {
        // up to 4 independent loads in flight per lane
        const uint32_t m = min(n, 4u);
        uint32_t off[4], v[4];
#pragma unroll
        for (uint32_t i = 0; i < 4; ++i) off[i] = (i < m) ? lw_addr(w, T, ltmask, w.k + i) : 0u;
#pragma unroll
        for (uint32_t i = 0; i < 4; ++i)
            if (i < m) v[i] = __ldg(reinterpret_cast<const uint32_t*>(block + off[i]));
#pragma unroll
        for (uint32_t i = 0; i < 4; ++i)
            if (i < m) *reinterpret_cast<uint32_t*>(r.buf + ((r.fl + 4 * i) & (RING - 1))) = v[i];
        r.fl += 4 * m;
        w.k += m;
        n -= m;
    }
}

// Block-cooperative copy of `nlanes` adjacent lane streams (slots L0..) of
// an interleaved block into shared memory: stream i goes to dst + i*cap.
// For each row, the group's words are contiguous, so threads (row, slot)
// read whole 32-byte sectors.  Also zeroes 16 bytes after every stream.
// Must be called by every thread of the block; ends with __syncthreads().
template <int NLANES>
__device__ __forceinline__ void load_lane_streams(const SegTable& T, const uint32_t* s_len, const uint8_t* block,
                                                  uint8_t* dst, uint32_t cap, uint32_t L0) {
    const uint32_t tid = threadIdx.x;
    uint32_t maxw = 0;
#pragma unroll
    for (int i = 0; i < NLANES; ++i) maxw = max(maxw, (s_len[L0 + i] + 3) >> 2);
    // Rows every slot reaches (segment 0: [0, T.hi[0]), 128 bytes each) hold
    // the group's words contiguously at 4*L0: with the block 16-byte aligned
    // and NLANES, L0 multiples of 4, one 16-byte load fetches 4 lanes' words
    // (a quarter of the memory requests of word copies).
    uint32_t k0 = 0;
    if constexpr (NLANES % 4 == 0) {
        if ((reinterpret_cast<uintptr_t>(block) & 15u) == 0 && (L0 & 3u) == 0) {
            constexpr uint32_t Q = NLANES / 4;
            const uint32_t rows0 = min(T.hi[0], maxw);
            const uint32_t cw = cap >> 2;
#pragma unroll 4
            for (uint32_t x = tid; x < rows0 * Q; x += blockDim.x) {
                const uint32_t k = x / Q, q = x % Q;
                const uint4 v = __ldg(reinterpret_cast<const uint4*>(block + k * 128u + 16u * ((L0 >> 2) + q)));
                uint32_t* d0 = reinterpret_cast<uint32_t*>(dst + 4u * q * cap) + k;
                d0[0] = v.x;
                d0[cw] = v.y;
                d0[2 * cw] = v.z;
                d0[3 * cw] = v.w;
            }
            k0 = rows0;
        }
    }
    const uint32_t sub = tid % NLANES;
    const uint32_t l = L0 + sub;
    const uint32_t nwl = (s_len[l] + 3) >> 2;
    const uint32_t ltmask = (1u << l) - 1u;
    uint32_t* d = reinterpret_cast<uint32_t*>(dst + sub * cap);
    // a thread's rows only grow, so its segment index is tracked, not searched
    uint32_t j = 0;
    for (uint32_t k = k0 + tid / NLANES; k < maxw; k += blockDim.x / NLANES) {
        if (k < nwl) {
            while (j < 31 && T.hi[j] <= k) ++j;
            const uint32_t lo = j ? T.hi[j - 1] : 0u;
            const uint32_t off = T.base[j] + (k - lo) * 4u * (32u - j) + 4u * __popc(T.mask[j] & ltmask);
            // asynchronous 4-byte global->shared copy: all of a thread's
            // loads are in flight at once instead of one round trip each
            const uint32_t sa = (uint32_t)__cvta_generic_to_shared(d + k);
            asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa), "l"(block + off) : "memory");
        }
    }
    asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
    if (tid < NLANES * 4) {
        const uint32_t s2 = tid / 4;
        const uint32_t w = ((s_len[L0 + s2] + 3) >> 2) + (tid & 3u);
        reinterpret_cast<uint32_t*>(dst + s2 * cap)[w] = 0;
    }
    __syncthreads();
}

}  // namespace gd
