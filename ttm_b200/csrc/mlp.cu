// Training and inference kernels of the schedule selector: a small multilayer perceptron
// (dense layers with ReLU) that predicts per-schedule run times from a TTM's shape features.
// Float32, row-major activations [batch][features], weights [out][in].
#include <cuda_runtime.h>

#include <cmath>

#include "tlibttm.h"

namespace {

// y[b][o] = act(sum_i x[b][i] * w[o][i] + bias[o])
__global__ void mlp_fwd_kernel(const float* __restrict__ x, const float* __restrict__ w, const float* __restrict__ bias,
                               float* __restrict__ y, int batch, int in, int out, int relu)
{
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= batch * out) return;
    const int b = idx / out, o = idx % out;
    const float* xr = x + (size_t)b * in;
    const float* wr = w + (size_t)o * in;
    float acc = bias ? bias[o] : 0.0f;
    for (int i = 0; i < in; ++i) acc = fmaf(xr[i], wr[i], acc);
    y[idx] = (relu && acc < 0.0f) ? 0.0f : acc;
}

// dz = dy * (y > 0) for a ReLU layer (y is the layer's output), dz = dy otherwise
__global__ void mlp_dz_kernel(const float* __restrict__ dy, const float* __restrict__ y, float* __restrict__ dz, int n,
                              int relu)
{
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= n) return;
    dz[idx] = (relu && !(y[idx] > 0.0f)) ? 0.0f : dy[idx];
}

// dw[o][i] = sum_b dz[b][o] x[b][i];  db[o] = sum_b dz[b][o] (computed by the i == 0 threads)
__global__ void mlp_dw_kernel(const float* __restrict__ dz, const float* __restrict__ x, float* __restrict__ dw,
                              float* __restrict__ db, int batch, int in, int out)
{
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= out * in) return;
    const int o = idx / in, i = idx % in;
    float acc = 0.0f, accb = 0.0f;
    for (int b = 0; b < batch; ++b) {
        const float d = dz[(size_t)b * out + o];
        acc = fmaf(d, x[(size_t)b * in + i], acc);
        accb += d;
    }
    dw[idx] = acc;
    if (i == 0 && db) db[o] = accb;
}

// dx[b][i] = sum_o dz[b][o] w[o][i]
__global__ void mlp_dx_kernel(const float* __restrict__ dz, const float* __restrict__ w, float* __restrict__ dx, int batch,
                              int in, int out)
{
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= batch * in) return;
    const int b = idx / in, i = idx % in;
    float acc = 0.0f;
    for (int o = 0; o < out; ++o) acc = fmaf(dz[(size_t)b * out + o], w[(size_t)o * in + i], acc);
    dx[idx] = acc;
}

// masked mean squared error: dy = 2 (y - t) mask * inv_count, loss += sum (y - t)^2 mask * inv_count
__global__ void mlp_mse_kernel(const float* __restrict__ y, const float* __restrict__ t, const float* __restrict__ mask,
                               float* __restrict__ dy, float* __restrict__ loss, int n, float inv_count)
{
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    float e2 = 0.0f;
    if (idx < n) {
        const float mk = mask ? mask[idx] : 1.0f;
        const float d = (y[idx] - t[idx]) * mk;
        dy[idx] = 2.0f * d * inv_count;
        e2 = d * d * inv_count;
    }
    if (loss) {
        for (int off = 16; off > 0; off >>= 1) e2 += __shfl_xor_sync(0xffffffffu, e2, off);
        if ((threadIdx.x & 31) == 0) atomicAdd(loss, e2);
    }
}

// Adam (Kingma & Ba, 2015) with bias correction
__global__ void mlp_adam_kernel(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                                float* __restrict__ v, int n, float lr, float b1, float b2, float eps, float bc1,
                                float bc2)
{
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= n) return;
    const float gi = g[idx];
    const float mi = b1 * m[idx] + (1.0f - b1) * gi;
    const float vi = b2 * v[idx] + (1.0f - b2) * gi * gi;
    m[idx] = mi;
    v[idx] = vi;
    p[idx] -= lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
}

inline unsigned blocks_for(long long n) { return (unsigned)((n + 255) / 256); }

int status(cudaError_t e) { return e == cudaSuccess ? TLIBTTM_OK : TLIBTTM_ERR_CUDA; }

}  // namespace

extern "C" {

int tlibttm_mlp_forward(const float* x, const float* w, const float* bias, float* y, int batch, int in, int out,
                        int relu, void* stream)
{
    if (batch <= 0 || in <= 0 || out <= 0 || !x || !w || !y) return TLIBTTM_ERR_ARG;
    mlp_fwd_kernel<<<blocks_for((long long)batch * out), 256, 0, static_cast<cudaStream_t>(stream)>>>(x, w, bias, y, batch,
                                                                                                    in, out, relu);
    return status(cudaGetLastError());
}

int tlibttm_mlp_backward(const float* x, const float* w, const float* y, const float* dy, float* dz, float* dx,
                         float* dw, float* db, int batch, int in, int out, int relu, void* stream)
{
    if (batch <= 0 || in <= 0 || out <= 0 || !x || !w || !y || !dy || !dz || !dw) return TLIBTTM_ERR_ARG;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    mlp_dz_kernel<<<blocks_for((long long)batch * out), 256, 0, s>>>(dy, y, dz, batch * out, relu);
    mlp_dw_kernel<<<blocks_for((long long)out * in), 256, 0, s>>>(dz, x, dw, db, batch, in, out);
    if (dx) mlp_dx_kernel<<<blocks_for((long long)batch * in), 256, 0, s>>>(dz, w, dx, batch, in, out);
    return status(cudaGetLastError());
}

int tlibttm_mlp_mse_grad(const float* y, const float* t, const float* mask, float* dy, float* loss, int n,
                         float inv_count, void* stream)
{
    if (n <= 0 || !y || !t || !dy) return TLIBTTM_ERR_ARG;
    mlp_mse_kernel<<<blocks_for(n), 256, 0, static_cast<cudaStream_t>(stream)>>>(y, t, mask, dy, loss, n, inv_count);
    return status(cudaGetLastError());
}

int tlibttm_mlp_adam(float* p, const float* g, float* m, float* v, int n, float lr, float beta1, float beta2, float eps,
                     int step, void* stream)
{
    if (n <= 0 || !p || !g || !m || !v || step < 1) return TLIBTTM_ERR_ARG;
    const float bc1 = 1.0f - std::pow(beta1, (float)step);
    const float bc2 = 1.0f - std::pow(beta2, (float)step);
    mlp_adam_kernel<<<blocks_for(n), 256, 0, static_cast<cudaStream_t>(stream)>>>(p, g, m, v, n, lr, beta1, beta2, eps,
                                                                                 bc1, bc2);
    return status(cudaGetLastError());
}

}  // extern "C"
