// ref_cudf -- the reference's vendored cuDF inflate (include/cudf_deflate.cuh:
// cudf::io::gpuinflate, :1399-1407, block-per-stream inflate_kernel, :1229),
// compiled from the reference sources for sm_100a into a shared library: the
// GPU comparator the Deflate decoder is timed against.  Comparator / oracle
// tooling only; it runs on well-formed streams, as the reference's own driver
// passes them (base_deflate.h:66-72: each zlib stream past its 2-byte header).
#include <cudf_deflate.cuh>

extern "C" int ref_cudf_gpuinflate(void* inputs, void* outputs, int count, int parse_hdr, void* stream) {
    const cudaError_t e = cudf::io::gpuinflate(static_cast<cudf::io::gpu_inflate_input_s*>(inputs),
                                               static_cast<cudf::io::gpu_inflate_status_s*>(outputs), count,
                                               parse_hdr, static_cast<cudaStream_t>(stream));
    return e == cudaSuccess && cudaGetLastError() == cudaSuccess ? 0 : 6;
}
