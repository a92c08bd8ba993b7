/*
 * gd.h -- C ABI of the B200 decode library (libgd.so).
 *
 * This is the drop-in boundary for the decompress calls of
 * ZaidQureshi/compression.  Each entry point names the reference interface
 * it replaces (file:line within that project).  The ABI uses plain pointers
 * and sizes only; a CUDA stream is passed as an opaque `gd_stream_t`
 * (a cudaStream_t, NULL = legacy default stream).
 *
 * Two tiers:
 *   - Device API (gd_*_decode): device pointers in and out, asynchronous on
 *     the given stream, caller owns every buffer, per-chunk status written to
 *     device memory.  Thread safe; never allocates.
 *   - Host API (gd_*_decompress): the reference's synchronous host-buffer
 *     signatures (H2D copy, decode, D2H copy, callee-allocated output that
 *     the caller releases with gd_free).  Device staging buffers come from a
 *     per-device pool owned by the library.
 *
 * Status codes are returned by every call and written per chunk by kernels.
 * No decoder traps, asserts or waits without a bound: a malformed stream
 * yields GD_ERR_CORRUPT / GD_ERR_OVERRUN for that chunk.
 */
#ifndef GD_H_
#define GD_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum gd_status {
    GD_OK = 0,
    GD_ERR_INVALID_ARG = 1, /* bad sizes / pointers / parameters */
    GD_ERR_CORRUPT = 2,     /* stream grammar violated or truncated */
    GD_ERR_OVERRUN = 3,     /* stream would write past its chunk */
    GD_ERR_TIMEOUT = 4,     /* a bounded device wait gave up */
    GD_ERR_UNSUPPORTED = 5, /* valid but unsupported feature */
    GD_ERR_CUDA = 6,        /* CUDA runtime error */
    GD_ERR_NOMEM = 7        /* allocation failed (host API only) */
} gd_status_t;

typedef void* gd_stream_t;

/* Library version string. */
const char* gd_version(void);
/* Human-readable name of a status code. */
const char* gd_status_string(int status);

/* ------------------------------------------------------------------------
 * Device API
 * ------------------------------------------------------------------------ */

/*
 * Byte-RLE, contiguous chunk container (brle.h format).
 * Replaces brle::kernel_decompress / brle::decompress_gpu
 * (include/brle/brle.h:102-109, :305-342).
 * d_data: compressed payload; d_ptr[n_chunks+1]: byte offsets of each chunk
 * in d_data; chunk c decodes to d_out[c*chunk_size ..], the last chunk to
 * out_n_bytes - c*chunk_size bytes.  d_status: n_chunks uint32 (may be NULL).
 */
gd_status_t gd_brle_decode(const uint8_t* d_data, const uint64_t* d_ptr, uint32_t n_chunks,
                           uint64_t chunk_size, uint8_t* d_out, uint64_t out_n_bytes,
                           uint32_t* d_status, gd_stream_t stream);

/*
 * RLE v1, 32-lane interleaved container.
 * Replaces rle_v1::inflate / rle_v1::decompress_gpu
 * (include/rle_v1/decoder.h:426-470, include/rle_v1/rlev1.h:100-199).
 * d_data: compressed blocks (the container after its 8-byte size header);
 * d_col_len[32*n_chunks]: per-lane stream bytes; d_blk_off[n_chunks+1]:
 * block start offsets.  elem_bytes 4 or 8; comp_col_len = COMP_COL_LEN.
 * max_lane_bytes: an upper bound on col_len (sizes the shared-memory copy
 * of each lane stream; 0 = the worst case for chunk_size).  A lane longer
 * than the bound fails its chunk with GD_ERR_CORRUPT.
 */
gd_status_t gd_rlev1_decode(const uint8_t* d_data, const uint64_t* d_col_len, const uint64_t* d_blk_off,
                            uint32_t n_chunks, uint64_t chunk_size, uint32_t comp_col_len,
                            uint32_t elem_bytes, uint8_t* d_out, uint64_t out_n_bytes,
                            uint32_t max_lane_bytes, uint32_t* d_status, gd_stream_t stream);

/*
 * RLE v2, 32-lane transposed container (8-byte values).
 * Replaces rlev2::inflate / rlev2::decompress_gpu<READ_UNIT,...>
 * (include/rlev2/decoder_new.h:618-657, include/rlev2/decoder_trans.h:615-681).
 * read_unit = READ_UNIT (values per lane slice); max_lane_bytes as for
 * gd_rlev1_decode.
 */
gd_status_t gd_rlev2_decode(const uint8_t* d_data, const uint64_t* d_col_len, const uint64_t* d_blk_off,
                            uint32_t n_chunks, uint64_t chunk_size, uint32_t read_unit,
                            uint8_t* d_out, uint64_t out_n_bytes, uint32_t max_lane_bytes,
                            uint32_t* d_status, gd_stream_t stream);

/*
 * LZSS, 32-column interleaved container.
 * Replaces lzss::kernel_decompress(blk_off,col_len,col_map)
 * (include/lzss/lzss_gpu2.h:1898-1907 -> decompress_func :112-325).
 * d_col_len: stream bytes per rank (sorted descending); d_col_map: rank ->
 * output column.  chunk_size multiple of 128 (runtime; the reference fixes
 * it at 128 KiB, lzss_gpu2.h:25).
 */
gd_status_t gd_lzss_decode(const uint8_t* d_data, const uint64_t* d_blk_off, const uint64_t* d_col_len,
                           const uint8_t* d_col_map, uint32_t n_chunks, uint64_t chunk_size,
                           uint8_t* d_out, uint64_t out_n_bytes, uint32_t* d_status,
                           gd_stream_t stream);

/*
 * Deflate / zlib inflate of independent chunks of any size.
 * Replaces deflate::inflate / inflate_shared / deflate::decompress_gpu
 * (include/zlib/zlib.h:832-962, :966-1082).  Chunk c: compressed bytes at
 * d_data + d_comp_off[c] (d_comp_len[c] bytes, trailing zero padding
 * allowed), output d_out[d_out_off[c] .. d_out_off[c+1]).  zlib_header: 1 =
 * zlib streams (2-byte header skipped and checked, as zlib.h:580), 0 = raw
 * deflate, 2 = gzip member (header parsed, trailer ignored).  Stored, fixed
 * and dynamic blocks are all decoded (the zlib/gzip checksums are not
 * verified).  d_data must be 16-byte aligned (compressed words are fetched
 * as aligned 16-byte loads; nothing outside a chunk's 16-byte-aligned span
 * is read).
 */
gd_status_t gd_inflate(const uint8_t* d_data, const uint64_t* d_comp_off, const uint64_t* d_comp_len,
                       const uint64_t* d_out_off, uint32_t n_chunks, int zlib_header, uint8_t* d_out,
                       uint32_t* d_status, gd_stream_t stream);

/* gd_inflate visiting chunks in the order d_order[0..n_chunks) (a
 * permutation), e.g. longest first.  No reference counterpart: the
 * reference maps chunk i to thread block i (zlib.h:1044-1057). */
gd_status_t gd_inflate_ordered(const uint8_t* d_data, const uint64_t* d_comp_off, const uint64_t* d_comp_len,
                               const uint64_t* d_out_off, uint32_t n_chunks, int zlib_header, uint8_t* d_out,
                               uint32_t* d_status, const uint32_t* d_order, gd_stream_t stream);

/*
 * LZSS, contiguous container (one token stream per chunk, not interleaved).
 * Replaces lzss::kernel_decompress(lens) / decompress_func
 * (include/lzss/lzss.h:234-305, :1014-1020).  Chunk c's stream is
 * d_data[d_ends[c-1] .. d_ends[c]) (d_ends = the container's cumulative
 * stream ends, d_ends[-1] = 0) and decodes to d_out[c*chunk_size ..]; the
 * last chunk to out_n_bytes - c*chunk_size bytes.
 */
gd_status_t gd_lzss_contig_decode(const uint8_t* d_data, const uint64_t* d_ends, uint32_t n_chunks,
                                  uint64_t chunk_size, uint8_t* d_out, uint64_t out_n_bytes,
                                  uint32_t* d_status, gd_stream_t stream);

/*
 * Byte-RLE flag-byte container, 32-column ranked interleave.
 * Replaces brle_trans::decompress_func (include/brle/brle_trans.h:72-202).
 * d_blk_off[n+1], d_col_len[32n] (stream bytes per rank, sorted
 * descending), d_col_map[32n] (rank -> column).  chunk_size: a multiple of
 * 128 up to 8192 (the reference fixes 4096, brle_trans.h:26).
 */
gd_status_t gd_brle_trans_decode(const uint8_t* d_data, const uint64_t* d_blk_off, const uint64_t* d_col_len,
                                 const uint8_t* d_col_map, uint32_t n_chunks, uint64_t chunk_size,
                                 uint8_t* d_out, uint64_t out_n_bytes, uint32_t* d_status,
                                 gd_stream_t stream);
/* The 4-byte-symbol variant (brle::decompress_func, include/brle/
 * brle_gpu_4B.h:75-223; 8 KiB chunks there): the same container, literals
 * are 4-byte symbols and a run item is a count byte and a symbol.
 * chunk_size a multiple of 128, at most 8192. */
gd_status_t gd_brle_trans4_decode(const uint8_t* d_data, const uint64_t* d_blk_off, const uint64_t* d_col_len,
                                  const uint8_t* d_col_map, uint32_t n_chunks, uint64_t chunk_size,
                                  uint8_t* d_out, uint64_t out_n_bytes, uint32_t* d_status, gd_stream_t stream);

/*
 * cuDF-compatible inflate interface (layouts of gpu_inflate_input_s and
 * gpu_inflate_status_s, include/cudf_deflate.cuh:236-250).
 * Replaces cudf::io::gpuinflate (include/cudf_deflate.cuh:1399-1407).
 * parse_hdr = 1: inputs are gzip members (as cuDF); 0: raw deflate.
 * status: 0 ok, 1 corrupt / overrun (cuDF's convention).
 */
typedef struct gd_inflate_input {
    const void* srcDevice;
    uint64_t srcSize;
    void* dstDevice;
    uint64_t dstSize;
} gd_inflate_input;

typedef struct gd_inflate_status {
    uint64_t bytes_written;
    uint32_t status;
    uint32_t reserved;
} gd_inflate_status;

gd_status_t gd_gpuinflate(const gd_inflate_input* d_inputs, gd_inflate_status* d_outputs, int count,
                          int parse_hdr, gd_stream_t stream);

/* Replaces cudf::io::gpu_copy_uncompressed_blocks (cudf_deflate.cuh:1409-1415). */
gd_status_t gd_copy_uncompressed_blocks(const gd_inflate_input* d_inputs, int count, gd_stream_t stream);

/* ------------------------------------------------------------------------
 * Batched mixed-codec decoding (no reference counterpart: the reference
 * launches one decoder per column and codec)
 * ------------------------------------------------------------------------ */

typedef enum gd_codec {
    GD_CODEC_BRLE = 0,
    GD_CODEC_RLEV1 = 1,
    GD_CODEC_RLEV2 = 2,
    GD_CODEC_LZSS = 3,
    GD_CODEC_DEFLATE = 4
} gd_codec_t;

/* One warp-sized unit of work.  All pointers are device pointers.
 *   BRLE:    src/src_len = one chunk's token stream; dst/dst_len = its output.
 *   RLEV1/2: src/src_len = the chunk's interleaved block; col_len = its 32
 *            lane lengths; lane = which lane stream; dst = the chunk's output
 *            base; dst_len = bytes of the chunk kept; chunk_size = the chunk
 *            size; param = RLE v1: (elem_bytes << 16) | values per lane slice,
 *            RLE v2: READ_UNIT.
 *   LZSS:    src/src_len = the chunk's block; col_len/col_map = its 32 ranks;
 *            dst_len = chunk_size (whole chunk written).
 *   DEFLATE: src/src_len = one stream; dst/dst_len = its exact output;
 *            param = 0 raw, 1 zlib, 2 gzip (src's 16-byte-aligned span readable). */
typedef struct gd_task {
    uint32_t codec;
    uint32_t param;
    uint32_t lane;
    uint32_t reserved;
    const uint8_t* src;
    uint64_t src_len;
    uint8_t* dst;
    uint64_t dst_len;
    uint64_t chunk_size;
    const uint64_t* col_len;
    const uint8_t* col_map;
} gd_task;

/*
 * Decode n_tasks tasks in one persistent launch (blocks_per_sm x SMs blocks
 * of 4 warps; 0 = as many as fit).  dynamic = 1: warps take tasks in the
 * order d_order[0..n) (NULL = identity) from a work queue whose counter is
 * d_counter (one uint32 of caller scratch, zeroed by this call); dynamic = 0:
 * task d_order[i] runs on warp i mod W.  max_lane_bytes bounds col_len of
 * RLE tasks.  d_status[n] (task index order) and optional d_timing[2n]
 * (%globaltimer ns at each task's start and end) are written per task.
 */
gd_status_t gd_batch_decode(const gd_task* d_tasks, uint32_t n_tasks, const uint32_t* d_order, int dynamic,
                            uint32_t max_lane_bytes, uint32_t blocks_per_sm, uint32_t* d_counter,
                            uint32_t* d_status, uint64_t* d_timing, gd_stream_t stream);

/*
 * No counterpart in the reference.  Header features of every task for the
 * learned cost model, computed on the device from the containers' headers
 * only: d_features[4n] (16-byte aligned) receives per task
 *   [0] log2(1 + units): run headers (RLE v1 / v2 lane), tokens (byte-RLE,
 *       LZSS chunk), 0 (Deflate);
 *   [1] literal share: literal values / values (RLE v1), DIRECT and
 *       PATCHED_BASE runs / runs (RLE v2), literal tokens / tokens (byte-RLE,
 *       LZSS: 1 - match density), first block type / 2 (Deflate: 0 stored,
 *       0.5 fixed, 1 dynamic);
 *   [2] units per KiB of output; Deflate: HLIT + 257 of a dynamic first
 *       block / 286;
 *   [3] 1 if the walk found the headers malformed, else 0.
 * Each walk is bounded by the stream's length.
 */
gd_status_t gd_task_features(const gd_task* d_tasks, uint32_t n_tasks, float* d_features, gd_stream_t stream);

/* Number of warps gd_batch_decode runs with for these parameters. */
uint32_t gd_batch_warps(uint32_t max_lane_bytes, uint32_t blocks_per_sm);

/*
 * No counterpart in the reference.  gd_batch_decode with longest-first
 * placement and no memory allocated or taken from the caller beyond the
 * listed arguments: the tasks are ordered by descending d_cost[n] (any cost
 * estimate, e.g. gd_mlp_predict output; bucketed, so near-equal costs run in
 * any order) and fed through the dynamic work queue.  The order array, sort
 * buckets and queue counter live in a fixed device array inside the library
 * (GD_BATCH_NOALLOC_MAX_TASKS tasks at most; more is GD_ERR_INVALID_ARG).
 * +inf costs run first, NaN and -inf costs last.  It serves callers that may
 * not allocate at decode time: hosts with a fixed, pre-reserved memory budget,
 * and decode paths that must not pay cudaMalloc / cudaFree's implicit
 * device-wide synchronisation.  Nothing needs zeroing beforehand.  The first call on a device looks up that
 * array's address (a runtime query, with the device current) and should come
 * before any stream capture.  Calls overlapping in time on one device share
 * the array and race: serialise them.  d_status[n] is written per task.
 */
#define GD_BATCH_NOALLOC_MAX_TASKS 65536u
gd_status_t gd_batch_decode_lpt_noalloc(const gd_task* d_tasks, uint32_t n_tasks, const float* d_cost,
                                        uint32_t max_lane_bytes, uint32_t blocks_per_sm, uint32_t* d_status,
                                        gd_stream_t stream);

/* ------------------------------------------------------------------------
 * Launch tuning knobs (no reference counterpart: its launch shapes are
 * compile-time constants).  Process-wide; each selects among compiled kernel
 * variants or sets a launch shape, 0 = the built-in default.  Set by the
 * autotuner, which times the choices on the device.
 * ------------------------------------------------------------------------ */
typedef enum gd_tune_key {
    GD_TUNE_INFLATE_VARIANT = 0, /* 1 / 2: one warp per stream, no window, 2 / 4 warps per block;
                                    3: one warp per stream with a 32 KiB shared output window;
                                    4 / 5: decoder + writer warp pair per stream, no window
                                    (copies read the output), 2 / 4 pairs per block;
                                    6: decoder + writer pair with the window, one per block;
                                    7 / 8: pairs with a 16 KiB window, 1 / 2 per block;
                                    9 / 10: 8 / 4 KiB window; 11 / 12: 8 / 4 KiB window with a
                                    1 KiB ring and batches of 512 literals / 64 commands;
                                    13: as 12, 2 pairs per block (copies beyond the window
                                    read the output); 14: as 12 with a 2 KiB window;
                                    0 (default): 12 for >= 4 streams per SM, else 6 */
    GD_TUNE_BRLE_BLOCKS_PER_SM = 1,   /* byte-RLE grid = value x SMs blocks (default 8) */
    GD_TUNE_RLEV1_LANES_PER_BLOCK = 2, /* 0/8: 8 lane streams per block; 4: 4 */
    GD_TUNE_RLEV2_LANES_PER_BLOCK = 3, /* 0: 8 lane streams per block (4 if 8 do not fit in shared
                                          memory); 8: 8; 4: 4 */
    GD_TUNE_LZSS_WARPS_PER_BLOCK = 4,  /* 0: one chunk per 32-thread block, one lane per column, a
                                          flag group per lane and step, output in 320-byte rounds
                                          per column (any chunk size); 4: the same with four chunks
                                          per block and 256-byte rounds (the batch decoder's shape);
                                          512 / 256: one chunk per block of 512 / 256 threads, 16 / 8
                                          lanes per column, output staged in shared memory; 1: one
                                          chunk per warp, one lane per column, output staged */
    GD_TUNE_INFLATE_PAIR_SPIN = 5,     /* polls of a decoder/writer hand-off wait before the stream
                                          gives up with GD_ERR_TIMEOUT (0: 2^25, about a second) */
    GD_TUNE_INFLATE_WRITER_STOP = 6,   /* test knob for the bounded hand-off wait: k > 0 makes each
                                          pair's writer warp leave after executing k batches, so the
                                          decoder warp's wait runs out and the stream reports
                                          GD_ERR_TIMEOUT (0: off) */
    GD_TUNE_COUNT = 7
} gd_tune_key_t;

/* Set a knob; returns its previous value, or -1 for an unknown key or a
 * negative value.  Takes effect for launches made afterwards. */
int gd_tune_set(int key, int value);
/* Current value of a knob, -1 for an unknown key. */
int gd_tune_get(int key);

/* ------------------------------------------------------------------------
 * Learned task-cost model: FP32 MLP 16 -> 64 -> 64 -> 1 (ReLU), parameters
 * W1[16][64] | b1[64] | W2[64][64] | b2[64] | W3[64] | b3 in one float array.
 * No reference counterpart.
 * ------------------------------------------------------------------------ */

uint32_t gd_mlp_num_params(void);
/* d_out[i] = MLP(d_x[i*16 .. i*16+16)) for i < n. */
gd_status_t gd_mlp_predict(const float* d_params, const float* d_x, uint32_t n, float* d_out, gd_stream_t stream);
/* One mini-batch step on rows d_idx[0..nb) (nb <= 256) of (d_x, d_y),
 * minimising the mean squared error.  d_grad != NULL: write the gradient and
 * leave the parameters; else an Adam step (step >= 1) updates d_params, d_m,
 * d_v.  d_loss (optional): the mini-batch loss. */
gd_status_t gd_mlp_train_step(float* d_params, float* d_m, float* d_v, const float* d_x, const float* d_y,
                              const uint32_t* d_idx, uint32_t nb, float lr, float beta1, float beta2, float eps,
                              uint32_t step, float* d_grad, float* d_loss, gd_stream_t stream);

/* ------------------------------------------------------------------------
 * Host API (reference signatures; synchronous; output from malloc)
 * ------------------------------------------------------------------------ */

/* Release a buffer returned by a gd_*_decompress call. */
void gd_free(void* p);

/* brle::decompress_gpu (include/brle/brle.h:305-342).
 * in: [u32 n_ptr][u64 ptr[n_ptr]][u64 total][data], chunk size 256 KiB. */
gd_status_t gd_brle_decompress(const uint8_t* in, uint64_t in_n_bytes, uint8_t** out,
                               uint64_t* out_n_bytes);

/* rle_v1::decompress_gpu (include/rle_v1/rlev1.h:100-199) with the side files
 * (col_len, blk_offset) passed in memory.  in: [u64 in_n_bytes][blocks]. */
gd_status_t gd_rlev1_decompress(const uint8_t* in, uint64_t in_n_bytes, const uint64_t* col_len,
                                uint64_t col_n_bytes, const uint64_t* blk_off, uint64_t blk_n_bytes,
                                uint32_t comp_col_len, uint32_t elem_bytes, uint64_t chunk_size,
                                uint8_t** out, uint64_t* out_n_bytes);

/* rlev2::decompress_gpu (include/rlev2/decoder_trans.h:615-681).
 * blk_off[n_chunks] holds the decompressed size (encoder_trans.h:490-492). */
gd_status_t gd_rlev2_decompress(const uint8_t* in, uint64_t in_n_bytes, uint64_t n_chunks,
                                const uint64_t* blk_off, const uint64_t* col_len, uint32_t read_unit,
                                uint64_t chunk_size, uint8_t** out, uint64_t* out_n_bytes);

/* lzss::decompress_gpu (include/lzss/lzss_gpu2.h:2129-2314).  meta:
 * [0] u64 chunk_size, [1] u64 blk_off[n+1], [2] u64 col_len[32n],
 * [3] u8 col_map[32n].  Returns 0 on success, -1 on bad metadata (as the
 * reference), or a positive gd_status_t. */
int gd_lzss_decompress(const uint8_t* in, uint64_t in_n_bytes, const uint8_t* const* meta,
                       const uint64_t* meta_lens, uint64_t meta_num, uint8_t** out,
                       uint64_t* out_n_bytes);

/* deflate::decompress_gpu (include/zlib/zlib.h:966-1082): in = concatenated
 * zlib streams padded to 8 bytes; col_len = padded stream lengths;
 * blk_offset = [u64 total][u64 0][u64 cumulative offsets]; chunk_size =
 * uniform uncompressed chunk size. */
gd_status_t gd_deflate_decompress(const uint8_t* in, uint64_t in_n_bytes, const uint64_t* col_len,
                                  uint64_t col_n_bytes, const uint64_t* blk_offset, uint64_t blk_n_bytes,
                                  uint64_t chunk_size, uint8_t** out, uint64_t* out_n_bytes);

/* Deflate chunks of any size (an extension: deflate::decompress_gpu,
 * include/zlib/zlib.h:966-1082, assumes one uniform chunk size).  in = the
 * streams; comp_off[n] / comp_len[n] locate each; out_off[n+1] are the output
 * offsets (out_off[n] = total); zlib_header as for gd_inflate. */
gd_status_t gd_inflate_decompress(const uint8_t* in, uint64_t in_n_bytes, const uint64_t* comp_off,
                                  const uint64_t* comp_len, const uint64_t* out_off, uint32_t n_chunks,
                                  int zlib_header, uint8_t** out, uint64_t* out_n_bytes);

/* lzss::decompress_gpu_base (include/lzss/lzss.h:1126-1188): in = the whole
 * contiguous container [u64 in_n_bytes][u32 chunk_size][u32 n_chunks]
 * [u32 2048][u32 3][u32 34][u64 stream end per chunk][data]. */
gd_status_t gd_lzss_contig_decompress(const uint8_t* in, uint64_t in_n_bytes, uint8_t** out, uint64_t* out_n_bytes);

/* brle_trans::decompress_gpu (include/brle/brle_trans.h:661-791), with the
 * arrays of its side files ./input_data/{col_len,col_map,blk_offset}.bin
 * passed in; the output is (blk_n_bytes/8 - 1) * chunk_size bytes. */
gd_status_t gd_brle_trans_decompress(const uint8_t* in, uint64_t in_n_bytes, const uint64_t* col_len,
                                     uint64_t col_n_bytes, const uint8_t* col_map, uint64_t map_n_bytes,
                                     const uint64_t* blk_off, uint64_t blk_n_bytes, uint64_t chunk_size,
                                     uint8_t** out, uint64_t* out_n_bytes);
/* brle::decompress_gpu of include/brle/brle_gpu_4B.h:717-897 (4-byte symbols),
 * with the arrays of its side files passed in. */
gd_status_t gd_brle_trans4_decompress(const uint8_t* in, uint64_t in_n_bytes, const uint64_t* col_len,
                                      uint64_t col_n_bytes, const uint8_t* col_map, uint64_t map_n_bytes,
                                      const uint64_t* blk_off, uint64_t blk_n_bytes, uint64_t chunk_size,
                                      uint8_t** out, uint64_t* out_n_bytes);

/* ------------------------------------------------------------------------
 * Encoders and generators (host; produce the containers above)
 * ------------------------------------------------------------------------ */

uint64_t gd_brle_max_encoded_bytes(uint64_t n, uint64_t chunk_size);
/* brle::compress_gpu (include/brle/brle.h:251-303). */
uint64_t gd_brle_encode(const uint8_t* in, uint64_t n, uint64_t chunk_size, uint8_t* out);

uint64_t gd_rlev1_max_encoded_bytes(uint64_t n, uint64_t chunk_size);
/* rle_v1::compress_gpu (include/rle_v1/rlev1.h:25-97). */
uint64_t gd_rlev1_encode(const uint8_t* in, uint64_t n, uint64_t chunk_size, uint32_t comp_col_len,
                         uint32_t elem_bytes, uint8_t* data, uint64_t* blk_off, uint64_t* col_len);
uint64_t gd_rlev1_encode_stream(const void* vals, uint64_t n, uint32_t elem_bytes, uint8_t* out,
                                uint64_t cap);

uint64_t gd_rlev2_max_encoded_bytes(uint64_t n, uint64_t chunk_size);
/* rlev2::compress_gpu_transpose (include/rlev2/encoder_trans.h:428-537). */
uint64_t gd_rlev2_encode(const uint8_t* in, uint64_t n, uint64_t chunk_size, uint32_t read_unit,
                         uint8_t* data, uint64_t* blk_off, uint64_t* col_len);
/* rlev2::block_encode on one stream (include/rlev2/encoder.h:795-969). */
uint64_t gd_rlev2_encode_stream(const int64_t* vals, uint64_t n, uint8_t* out, uint64_t cap);

/* ------------------------------------------------------------------------
 * Device encoders (sm_100a) for the byte-RLE, LZSS, RLE v1 and RLE v2
 * containers: the same bytes as the host encoders gd_*_encode,
 * written from a column already in device memory.  Asynchronous on `stream`.
 *
 * d_scratch and d_data each hold gd_*_encode_bound(n_bytes, ...) bytes (4-byte
 * aligned); d_blk_off holds n_chunks + 1 and d_col_len 32 * n_chunks values;
 * d_status (optional) n_chunks words (GD_ERR_OVERRUN if a lane outgrew its
 * scratch slot, which the bound rules out).  The encoded size is
 * d_blk_off[n_chunks].  n_bytes must be a multiple of the value size and
 * d_in aligned to it; the last chunk is zero-padded as the host encoders do.
 * ------------------------------------------------------------------------ */
/* brle::compress_gpu (include/brle/brle.h:242-303): the whole container
 * [u32 n_ptr][u64 ptr][u64 total][data] written to d_out (4-byte aligned,
 * gd_brle_max_encoded_bytes(n_bytes, chunk_size) bytes); its length goes to
 * the device word *d_out_bytes.  d_scratch: gd_brle_encode_scratch_bytes
 * bytes, 16-byte aligned. */
uint64_t gd_brle_encode_scratch_bytes(uint64_t n_bytes, uint64_t chunk_size);
gd_status_t gd_brle_encode_device(const uint8_t* d_in, uint64_t n_bytes, uint64_t chunk_size,
                                  uint8_t* d_scratch, uint8_t* d_out, uint64_t* d_out_bytes,
                                  gd_stream_t stream);
/* lzss::compress_gpu (include/lzss/lzss_gpu2.h:1915-2127): the interleaved
 * container with its .meta arrays -- d_blk_off (n_chunks + 1), d_col_len and
 * d_col_map (32 * n_chunks, slots by descending column length).  chunk_size
 * a multiple of 128, at most 128 KiB; d_in, d_scratch and d_data 4-byte
 * aligned, the latter two gd_lzss_encode_bound bytes each.  The last chunk
 * is zero-padded to a whole chunk. */
uint64_t gd_lzss_encode_bound(uint64_t n_bytes, uint64_t chunk_size);
gd_status_t gd_lzss_encode_device(const uint8_t* d_in, uint64_t n_bytes, uint64_t chunk_size,
                                  uint8_t* d_scratch, uint8_t* d_data, uint64_t* d_blk_off,
                                  uint64_t* d_col_len, uint8_t* d_col_map, uint32_t* d_status,
                                  gd_stream_t stream);
/* brle_trans::compress_gpu (include/brle/brle_trans.h:563-660): the
 * byte-RLE flag container with the arrays of its side files -- d_blk_off
 * (n_chunks + 1), d_col_len and d_col_map (32 * n_chunks, slots by
 * descending column length).  chunk_size a multiple of 128, at most 8064
 * (the reference's is 4096); buffers as for gd_lzss_encode_device, sized by
 * gd_brle_trans_encode_bound.  The last chunk is zero-padded. */
uint64_t gd_brle_trans_encode_bound(uint64_t n_bytes, uint64_t chunk_size);
gd_status_t gd_brle_trans_encode_device(const uint8_t* d_in, uint64_t n_bytes, uint64_t chunk_size,
                                        uint8_t* d_scratch, uint8_t* d_data, uint64_t* d_blk_off,
                                        uint64_t* d_col_len, uint8_t* d_col_map, uint32_t* d_status,
                                        gd_stream_t stream);
/* rle_v1::compress_gpu (include/rle_v1/rlev1.h:25-97); elem_bytes 4 or 8. */
uint64_t gd_rlev1_encode_bound(uint64_t n_bytes, uint64_t chunk_size, uint32_t elem_bytes);
gd_status_t gd_rlev1_encode_device(const uint8_t* d_in, uint64_t n_bytes, uint64_t chunk_size,
                                   uint32_t comp_col_len, uint32_t elem_bytes, uint8_t* d_scratch,
                                   uint8_t* d_data, uint64_t* d_blk_off, uint64_t* d_col_len,
                                   uint32_t* d_status, gd_stream_t stream);
/* rlev2::compress_gpu_transpose (include/rlev2/encoder_trans.h:428-537). */
uint64_t gd_rlev2_encode_bound(uint64_t n_bytes, uint64_t chunk_size);
gd_status_t gd_rlev2_encode_device(const uint8_t* d_in, uint64_t n_bytes, uint64_t chunk_size,
                                   uint32_t read_unit, uint8_t* d_scratch, uint8_t* d_data,
                                   uint64_t* d_blk_off, uint64_t* d_col_len, uint32_t* d_status,
                                   gd_stream_t stream);

/* ------------------------------------------------------------------------
 * Host compress calls on the device encoders (synchronous): the column is
 * copied from host memory, encoded on the current device and the container
 * and its metadata returned in buffers released with gd_free, each one
 * separately.  The same bytes as the host encoders gd_*_encode.
 * in_n_bytes == 0 is GD_ERR_INVALID_ARG.
 * ------------------------------------------------------------------------ */
/* brle::compress_gpu (include/brle/brle.h:242-303): the container
 * [u32 n_ptr][u64 ptr][u64 total][data] in 256 KiB chunks, the input of
 * gd_brle_decompress. */
gd_status_t gd_brle_compress(const uint8_t* in, uint64_t in_n_bytes, uint8_t** out, uint64_t* out_n_bytes);
/* rle_v1::compress_gpu (include/rle_v1/rlev1.h:25-97): *out is
 * [u64 in_n_bytes][data]; *col_len (32 * n_chunks values) and *blk_off
 * (n_chunks + 1) are the arrays the reference writes to its side files
 * ./input_data/rle_v1_{col_len,blk_offset}.bin.  elem_bytes 4 or 8. */
gd_status_t gd_rlev1_compress(const uint8_t* in, uint64_t in_n_bytes, uint32_t comp_col_len, uint32_t elem_bytes,
                              uint64_t chunk_size, uint8_t** out, uint64_t* out_n_bytes, uint64_t** col_len,
                              uint64_t** blk_off, uint64_t* n_chunks);
/* rlev2::compress_gpu_transpose (include/rlev2/encoder_trans.h:428-537) on
 * int64 values: *out is the data, *blk_off (n_chunks + 1) ends with
 * in_n_bytes (encoder_trans.h:492), *col_len holds 32 * n_chunks values. */
gd_status_t gd_rlev2_compress(const uint8_t* in, uint64_t in_n_bytes, uint32_t read_unit, uint64_t chunk_size,
                              uint8_t** out, uint64_t* out_n_bytes, uint64_t** blk_off, uint64_t** col_len,
                              uint64_t* n_chunks);
/* lzss::compress_gpu (include/lzss/lzss_gpu2.h:1915-2127), 128 KiB chunks:
 * *out is the data; *out_meta_num = 4 blobs in *out_meta (lengths in
 * *out_meta_lens): the u64 chunk size, blk_offset, col_len and col_map --
 * the metadata gd_lzss_decompress takes.  The last chunk is zero-padded to
 * a whole chunk (the reference drops a partial last chunk).  Release the
 * four blobs, *out_meta and *out_meta_lens with gd_free. */
int gd_lzss_compress(const uint8_t* in, uint64_t in_n_bytes, uint8_t** out, uint64_t* out_n_bytes,
                     uint8_t*** out_meta, uint64_t** out_meta_lens, uint64_t* out_meta_num);

uint64_t gd_lzss_max_encoded_bytes(uint64_t n, uint64_t chunk_size);
/* lzss::compress_gpu (include/lzss/lzss_gpu2.h:1915-2127). */
uint64_t gd_lzss_encode(const uint8_t* in, uint64_t n, uint64_t chunk_size, uint8_t* data,
                        uint64_t* blk_off, uint64_t* col_len, uint8_t* col_map);
/* lzss::compress_func on one stream (include/lzss/lzss_cpu.h:540-655). */
uint64_t gd_lzss_encode_stream(const uint8_t* in, uint32_t n, uint8_t* out, uint64_t cap);

uint64_t gd_lzss_contig_max_encoded_bytes(uint64_t n, uint64_t chunk_size);
/* lzss::compress_gpu, contiguous container (include/lzss/lzss.h:1060-1124). */
uint64_t gd_lzss_contig_encode(const uint8_t* in, uint64_t n, uint64_t chunk_size, uint8_t* out);

uint64_t gd_brle_trans_max_encoded_bytes(uint64_t n, uint64_t chunk_size);
/* brle_trans::compress_gpu (include/brle/brle_trans.h:563-660). */
uint64_t gd_brle_trans_encode(const uint8_t* in, uint64_t n, uint64_t chunk_size, uint8_t* data,
                              uint64_t* blk_off, uint64_t* col_len, uint8_t* col_map);

uint64_t gd_brle_trans4_max_encoded_bytes(uint64_t n, uint64_t chunk_size);
/* brle::compress_gpu of include/brle/brle_gpu_4B.h:640-715 (4-byte symbols). */
uint64_t gd_brle_trans4_encode(const uint8_t* in, uint64_t n, uint64_t chunk_size, uint8_t* data,
                               uint64_t* blk_off, uint64_t* col_len, uint8_t* col_map);

uint64_t gd_deflate_max_encoded_bytes(const uint64_t* out_off, uint32_t n);
/* zlib_chunk_compress (orig_compressor.py:44-126) with per-chunk sizes. */
uint64_t gd_deflate_encode(const uint8_t* in, const uint64_t* out_off, uint32_t n, int level,
                           const uint8_t* mode, int zlib_header, uint8_t* data, uint64_t* comp_off,
                           uint64_t* comp_len);

void gd_gen_rlev1_ints(uint64_t seed, uint64_t n, int32_t* out);
void gd_gen_brle_bytes(uint64_t seed, uint64_t n, uint8_t* out);
void gd_gen_rlev2_ints(uint64_t seed, uint64_t n, int64_t* out);
void gd_gen_markov_copy(uint64_t seed, uint64_t n, uint32_t max_dist, uint8_t* out);
int gd_gen_loguniform_sizes(uint64_t seed, uint32_t n, uint64_t lo, uint64_t hi, uint64_t total,
                            uint64_t granule, uint64_t* out);

#ifdef __cplusplus
}
#endif

#endif /* GD_H_ */
