// mlp.cu -- the batch scheduler's learned cost model: an FP32 MLP
// 16 -> 64 -> 64 -> 1 (ReLU) predicting a task's log decode time from its
// header features, with hand-written inference and training kernels.
//
// No counterpart in the reference.  Parameters are one flat float array:
//   W1[16][64] | b1[64] | W2[64][64] | b2[64] | W3[64] | b3
// (row-major [in][out]).  Training minimises the mean squared error between
// the prediction and the measured log time with Adam; one 256-thread block
// runs a whole step (forward, backward, update) for a mini-batch of up to 256
// rows with every activation in shared memory.  Gradients can be written out
// instead of applied, for checking against a CPU implementation.
#include "gd_common.cuh"

namespace gd {
namespace mlp {

constexpr int IN = 16, H = 64;
constexpr int O_W1 = 0, O_B1 = O_W1 + IN * H, O_W2 = O_B1 + H, O_B2 = O_W2 + H * H, O_W3 = O_B2 + H,
              O_B3 = O_W3 + H, NP = O_B3 + 1;  // 5313 parameters
constexpr int NT = 256;                        // threads per block = rows per block

// ---- inference: one thread per row, weights broadcast from shared memory ----
__global__ void __launch_bounds__(NT) predict_kernel(const float* __restrict__ P, const float* __restrict__ X,
                                                     uint32_t n, float* __restrict__ out) {
    __shared__ float w[NP];
    for (int i = threadIdx.x; i < NP; i += NT) w[i] = P[i];
    __syncthreads();
    const uint32_t r = blockIdx.x * NT + threadIdx.x;
    if (r >= n) return;
    float x[IN];
#pragma unroll
    for (int k = 0; k < IN; ++k) x[k] = X[(size_t)r * IN + k];
    float h1[H];
#pragma unroll
    for (int j = 0; j < H; ++j) {
        float z = w[O_B1 + j];
#pragma unroll
        for (int k = 0; k < IN; ++k) z = fmaf(x[k], w[O_W1 + k * H + j], z);
        h1[j] = fmaxf(z, 0.f);
    }
    float o = w[O_B3];
#pragma unroll 4
    for (int j = 0; j < H; ++j) {
        float z = w[O_B2 + j];
#pragma unroll
        for (int i = 0; i < H; ++i) z = fmaf(h1[i], w[O_W2 + i * H + j], z);
        o = fmaf(fmaxf(z, 0.f), w[O_W3 + j], o);
    }
    out[r] = o;
}

// ---- one training step (or one gradient evaluation) in one block ----
// Rows idx[0..nb) of (X, y); nb <= NT.  If grad != nullptr the gradient of
// the mean squared error is written there and P is left unchanged; otherwise
// an Adam step (lr, beta1, beta2, eps, step t >= 1) updates P, M, V.
// loss (optional) receives the mini-batch MSE before the update.
__global__ void __launch_bounds__(NT) train_kernel(float* __restrict__ P, float* __restrict__ M,
                                                   float* __restrict__ V, const float* __restrict__ X,
                                                   const float* __restrict__ y, const uint32_t* __restrict__ idx,
                                                   uint32_t nb, float lr, float beta1, float beta2, float eps,
                                                   uint32_t t, float* __restrict__ grad, float* __restrict__ loss) {
    extern __shared__ __align__(16) float sm[];
    float* w = sm;                // NP
    float* g = w + NP;            // NP gradients
    float* xs = g + NP;           // NT x IN
    float* a1 = xs + NT * IN;     // NT x H: h1, later dZ1
    float* a2 = a1 + NT * H;      // NT x H: h2, later dZ2
    float* dout = a2 + NT * H;    // NT
    __shared__ float red[NT / 32];
    const int tid = threadIdx.x;
    for (int i = tid; i < NP; i += NT) {
        w[i] = P[i];
        g[i] = 0.f;
    }
    const bool row = tid < (int)nb;
    const uint32_t r = row ? idx[tid] : 0u;
    for (int k = 0; k < IN; ++k) xs[tid * IN + k] = row ? X[(size_t)r * IN + k] : 0.f;
    __syncthreads();
    // forward
    for (int j = 0; j < H; ++j) {
        float z = w[O_B1 + j];
        for (int k = 0; k < IN; ++k) z = fmaf(xs[tid * IN + k], w[O_W1 + k * H + j], z);
        a1[tid * H + j] = fmaxf(z, 0.f);
    }
    float o = w[O_B3];
    for (int j = 0; j < H; ++j) {
        float z = w[O_B2 + j];
        for (int i = 0; i < H; ++i) z = fmaf(a1[tid * H + i], w[O_W2 + i * H + j], z);
        const float h = fmaxf(z, 0.f);
        a2[tid * H + j] = h;
        o = fmaf(h, w[O_W3 + j], o);
    }
    const float err = row ? (o - y[r]) : 0.f;
    dout[tid] = 2.f * err / (float)nb;
    // mini-batch loss
    float l2 = err * err;
    for (int s = 16; s; s >>= 1) l2 += __shfl_xor_sync(GD_FULL_MASK, l2, s);
    if ((tid & 31) == 0) red[tid >> 5] = l2;
    __syncthreads();
    if (tid == 0 && loss) {
        float s = 0.f;
        for (int i = 0; i < NT / 32; ++i) s += red[i];
        *loss = s / (float)nb;
    }
    // layer 3: dW3[j] = sum_r dout[r] h2[r][j], db3 = sum dout
    if (tid < H) {
        float s = 0.f;
        for (int q = 0; q < (int)nb; ++q) s = fmaf(dout[q], a2[q * H + tid], s);
        g[O_W3 + tid] = s;
    } else if (tid == H) {
        float s = 0.f;
        for (int q = 0; q < (int)nb; ++q) s += dout[q];
        g[O_B3] = s;
    }
    __syncthreads();
    // dZ2 = dout * W3 * relu'(z2)   (in place of h2)
    for (int j = 0; j < H; ++j) {
        const float h = a2[tid * H + j];
        a2[tid * H + j] = (row && h > 0.f) ? dout[tid] * w[O_W3 + j] : 0.f;
    }
    __syncthreads();
    // dW2[i][j] = sum_r h1[r][i] dZ2[r][j]; each thread 16 of the 4096 entries
    for (int e = tid; e < H * H; e += NT) {
        const int i = e / H, j = e % H;
        float s = 0.f;
        for (int q = 0; q < (int)nb; ++q) s = fmaf(a1[q * H + i], a2[q * H + j], s);
        g[O_W2 + e] = s;
    }
    if (tid < H) {
        float s = 0.f;
        for (int q = 0; q < (int)nb; ++q) s += a2[q * H + tid];
        g[O_B2 + tid] = s;
    }
    __syncthreads();
    // dZ1[r][i] = relu'(z1) * sum_j dZ2[r][j] W2[i][j]   (in place of h1)
    {
        float d1[H];
        for (int i = 0; i < H; ++i) {
            float s = 0.f;
            for (int j = 0; j < H; ++j) s = fmaf(a2[tid * H + j], w[O_W2 + i * H + j], s);
            d1[i] = (a1[tid * H + i] > 0.f) ? s : 0.f;
        }
        for (int i = 0; i < H; ++i) a1[tid * H + i] = d1[i];
    }
    __syncthreads();
    // dW1[k][i] = sum_r x[r][k] dZ1[r][i]; db1[i] = sum_r dZ1[r][i]
    for (int e = tid; e < IN * H; e += NT) {
        const int k = e / H, i = e % H;
        float s = 0.f;
        for (int q = 0; q < (int)nb; ++q) s = fmaf(xs[q * IN + k], a1[q * H + i], s);
        g[O_W1 + e] = s;
    }
    if (tid < H) {
        float s = 0.f;
        for (int q = 0; q < (int)nb; ++q) s += a1[q * H + tid];
        g[O_B1 + tid] = s;
    }
    __syncthreads();
    if (grad) {
        for (int i = tid; i < NP; i += NT) grad[i] = g[i];
        return;
    }
    // Adam (bias-corrected)
    const float c1 = 1.f - powf(beta1, (float)t), c2 = 1.f - powf(beta2, (float)t);
    for (int i = tid; i < NP; i += NT) {
        const float gi = g[i];
        const float m = beta1 * M[i] + (1.f - beta1) * gi;
        const float v = beta2 * V[i] + (1.f - beta2) * gi * gi;
        M[i] = m;
        V[i] = v;
        P[i] = w[i] - lr * (m / c1) / (sqrtf(v / c2) + eps);
    }
}

constexpr uint32_t TRAIN_SMEM = (uint32_t)((2 * NP + NT * IN + 2 * NT * H + NT) * sizeof(float));

}  // namespace mlp
}  // namespace gd

extern "C" uint32_t gd_mlp_num_params(void) { return gd::mlp::NP; }

extern "C" gd_status_t gd_mlp_predict(const float* d_params, const float* d_x, uint32_t n, float* d_out,
                                      gd_stream_t stream) {
    if (n == 0) return GD_OK;
    if (!d_params || !d_x || !d_out) return GD_ERR_INVALID_ARG;
    gd::mlp::predict_kernel<<<(n + gd::mlp::NT - 1) / gd::mlp::NT, gd::mlp::NT, 0, (cudaStream_t)stream>>>(
        d_params, d_x, n, d_out);
    return cudaGetLastError() == cudaSuccess ? GD_OK : GD_ERR_CUDA;
}

extern "C" gd_status_t gd_mlp_train_step(float* d_params, float* d_m, float* d_v, const float* d_x, const float* d_y,
                                         const uint32_t* d_idx, uint32_t nb, float lr, float beta1, float beta2,
                                         float eps, uint32_t step, float* d_grad, float* d_loss, gd_stream_t stream) {
    using namespace gd::mlp;
    if (nb == 0 || nb > (uint32_t)NT || !d_params || !d_x || !d_y || !d_idx) return GD_ERR_INVALID_ARG;
    if (!d_grad && (!d_m || !d_v || step == 0)) return GD_ERR_INVALID_ARG;
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(train_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, TRAIN_SMEM);
        attr = true;
    }
    train_kernel<<<1, NT, TRAIN_SMEM, (cudaStream_t)stream>>>(d_params, d_m, d_v, d_x, d_y, d_idx, nb, lr, beta1,
                                                             beta2, eps, step, d_grad, d_loss);
    return cudaGetLastError() == cudaSuccess ? GD_OK : GD_ERR_CUDA;
}
