// fe_model.cu — the learned warm-start model object and its C ABI.
//
// A model holds the FP32 master parameters, their BF16 copy used by the
// tensor-core kernels, Adam moments, and the feature/target standardisation.
// Features enter as raw FP32 rows of 12; targets are the raw normalised
// pressures of the two solves (see the feature definition in fe_learned.cu).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <random>
#include <vector>

#include "../../include/fluid_step.h"
#include "fe_error.h"
#include "fe_mlp.h"
#include "fe_model.h"

using namespace fe;

namespace {

__global__ void k_prepare_x(const float* __restrict__ x, const float* __restrict__ norm,
                            __nv_bfloat16* __restrict__ xb, uint32_t n) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t packed[8];
#pragma unroll
    for (int f = 0; f < 16; f += 2) {
        float v0 = 0.0f, v1 = 0.0f;
        if (f < (int)mlp::kFeatures) v0 = (x[(size_t)i * mlp::kFeatures + f] - norm[f]) / norm[12 + f];
        if (f + 1 < (int)mlp::kFeatures)
            v1 = (x[(size_t)i * mlp::kFeatures + f + 1] - norm[f + 1]) / norm[13 + f];
        __nv_bfloat162 two = __floats2bfloat162_rn(v0, v1);  // .x = v0 (low half)
        packed[f / 2] = *reinterpret_cast<uint32_t*>(&two);
    }
    uint4* dst = reinterpret_cast<uint4*>(xb + (size_t)i * 16);
    dst[0] = make_uint4(packed[0], packed[1], packed[2], packed[3]);
    dst[1] = make_uint4(packed[4], packed[5], packed[6], packed[7]);
}

__global__ void k_standardize_y(const float* __restrict__ y, const float* __restrict__ norm,
                                float* __restrict__ ys, uint32_t n) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 2 * n) return;
    uint32_t c = i & 1u;
    ys[i] = (y[i] - norm[24 + c]) / norm[26 + c];
}

__global__ void k_destandardize_y(float* __restrict__ y, const float* __restrict__ norm, uint32_t n) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 2 * n) return;
    uint32_t c = i & 1u;
    y[i] = y[i] * norm[26 + c] + norm[24 + c];
}

__global__ void k_to_bf16(const float* __restrict__ src, __nv_bfloat16* __restrict__ dst, uint32_t n) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = __float2bfloat16_rn(src[i]);
}

#define M_CUDA(call)                                                                         \
    do {                                                                                     \
        cudaError_t e_ = (call);                                                             \
        if (e_ != cudaSuccess) {                                                             \
            fe_set_error_message("%s: %s", #call, cudaGetErrorString(e_));                   \
            return e_ == cudaErrorMemoryAllocation ? FE_ERR_OUT_OF_MEMORY : FE_ERR_CUDA;     \
        }                                                                                    \
    } while (0)

}  // namespace

fe_status fe_model::ensure_scratch(uint32_t n) {
    if (n <= scratch_rows) return FE_OK;
    cudaFree(xb);
    cudaFree(ys);
    xb = nullptr;
    ys = nullptr;
    uint32_t rows = n + 1024;
    M_CUDA(cudaMalloc(&xb, (size_t)rows * 16 * sizeof(__nv_bfloat16)));
    M_CUDA(cudaMalloc(&ys, (size_t)rows * 2 * sizeof(float)));
    scratch_rows = rows;
    return FE_OK;
}

mlp::Params fe_model::params() const { return mlp::params_from(wbf16, master); }

fe_status fe_model::refresh_bf16(cudaStream_t s) {
    k_to_bf16<<<(mlp::kWeights + 255) / 256, 256, 0, s>>>(master, wbf16, mlp::kWeights);
    M_CUDA(cudaGetLastError());
    return FE_OK;
}

fe_status fe_model::prepare_x(const float* x, uint32_t n, cudaStream_t s) {
    fe_status st = ensure_scratch(n);
    if (st != FE_OK) return st;
    k_prepare_x<<<(n + 255) / 256, 256, 0, s>>>(x, norm, xb, n);
    M_CUDA(cudaGetLastError());
    return FE_OK;
}

extern "C" {

FE_API fe_status fe_model_create(uint32_t seed, int device, fe_model** out) {
    if (!out) {
        fe_set_error_message("out is NULL");
        return FE_ERR_INVALID_ARGUMENT;
    }
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count) {
        fe_set_error_message("no CUDA device %d", device);
        return FE_ERR_NO_DEVICE;
    }
    M_CUDA(cudaSetDevice(device));
    fe_model* m = new fe_model();
    m->device = device;
    cudaDeviceGetAttribute(&m->num_sms, cudaDevAttrMultiProcessorCount, device);
    auto fail = [&](fe_status s) {
        fe_model_destroy(m);
        return s;
    };
    if (cudaMalloc(&m->master, mlp::kParams * 4) != cudaSuccess ||
        cudaMalloc(&m->grad, (mlp::kParams + 1) * 4) != cudaSuccess ||
        cudaMalloc(&m->grad_part, (size_t)m->num_sms * (mlp::kParams + 1) * 4) != cudaSuccess ||
        cudaMalloc(&m->adam_m, mlp::kParams * 4) != cudaSuccess ||
        cudaMalloc(&m->adam_v, mlp::kParams * 4) != cudaSuccess ||
        cudaMalloc(&m->wbf16, mlp::kWeights * 2) != cudaSuccess ||
        cudaMalloc(&m->norm, 32 * 4) != cudaSuccess ||
        cudaMalloc(&m->flags, 16) != cudaSuccess) {
        fe_set_error_message("cudaMalloc failed");
        return fail(FE_ERR_OUT_OF_MEMORY);
    }
    // He-style initialisation with a fixed seed; input columns 12..15 zero.
    std::vector<float> p(mlp::kParams, 0.0f);
    std::mt19937 rng(seed);
    std::normal_distribution<float> nd(0.0f, 1.0f);
    for (int o = 0; o < 64; ++o)
        for (int k = 0; k < 12; ++k) p[o * 16 + k] = nd(rng) * std::sqrt(2.0f / 12.0f);
    for (uint32_t i = 0; i < mlp::kW2; ++i) p[mlp::kW1 + i] = nd(rng) * std::sqrt(2.0f / 64.0f);
    for (uint32_t i = 0; i < mlp::kW3; ++i) p[mlp::kW1 + mlp::kW2 + i] = nd(rng) * std::sqrt(1.0f / 64.0f);
    std::vector<float> norm(32, 0.0f);
    for (int f = 0; f < 12; ++f) norm[12 + f] = 1.0f;  // x mean 0, std 1
    norm[26] = norm[27] = 1.0f;                         // y mean 0, std 1
    if (cudaMemcpy(m->master, p.data(), mlp::kParams * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemset(m->grad, 0, (mlp::kParams + 1) * 4) != cudaSuccess ||
        cudaMemset(m->adam_m, 0, mlp::kParams * 4) != cudaSuccess ||
        cudaMemset(m->adam_v, 0, mlp::kParams * 4) != cudaSuccess ||
        cudaMemset(m->flags, 0, 16) != cudaSuccess ||
        cudaMemcpy(m->norm, norm.data(), 32 * 4, cudaMemcpyHostToDevice) != cudaSuccess) {
        fe_set_error_message("initial upload failed");
        return fail(FE_ERR_CUDA);
    }
    fe_status s = m->refresh_bf16(nullptr);
    if (s != FE_OK) return fail(s);
    if (cudaDeviceSynchronize() != cudaSuccess) return fail(FE_ERR_CUDA);
    *out = m;
    return FE_OK;
}

FE_API fe_status fe_model_destroy(fe_model* m) {
    if (!m) return FE_OK;
    cudaSetDevice(m->device);
    cudaDeviceSynchronize();
    for (void* p : {(void*)m->master, (void*)m->grad, (void*)m->grad_part, (void*)m->adam_m,
                    (void*)m->adam_v,
                    (void*)m->wbf16, (void*)m->norm, (void*)m->flags, (void*)m->xb, (void*)m->ys})
        if (p) cudaFree(p);
    delete m;
    return FE_OK;
}

FE_API fe_status fe_model_set_parameters(fe_model* m, const float* params, size_t count) {
    if (!m || !params || count != mlp::kParams) {
        fe_set_error_message("expected %u parameters", mlp::kParams);
        return FE_ERR_INVALID_ARGUMENT;
    }
    M_CUDA(cudaSetDevice(m->device));
    std::vector<float> p(params, params + count);
    for (int o = 0; o < 64; ++o)
        for (int k = 12; k < 16; ++k) p[o * 16 + k] = 0.0f;
    M_CUDA(cudaMemcpy(m->master, p.data(), count * 4, cudaMemcpyHostToDevice));
    M_CUDA(cudaMemset(m->adam_m, 0, mlp::kParams * 4));
    M_CUDA(cudaMemset(m->adam_v, 0, mlp::kParams * 4));
    m->step = 0;
    fe_status s = m->refresh_bf16(nullptr);
    if (s != FE_OK) return s;
    M_CUDA(cudaDeviceSynchronize());
    return FE_OK;
}

FE_API fe_status fe_model_get_parameters(const fe_model* m, float* params, size_t count) {
    if (!m || !params || count != mlp::kParams) {
        fe_set_error_message("expected %u parameters", mlp::kParams);
        return FE_ERR_INVALID_ARGUMENT;
    }
    M_CUDA(cudaSetDevice(m->device));
    M_CUDA(cudaMemcpy(params, m->master, count * 4, cudaMemcpyDeviceToHost));
    return FE_OK;
}

FE_API fe_status fe_model_set_normalization(fe_model* m, const float* x_mean, const float* x_std,
                                            const float* y_mean, const float* y_std) {
    if (!m || !x_mean || !x_std || !y_mean || !y_std) {
        fe_set_error_message("NULL argument");
        return FE_ERR_INVALID_ARGUMENT;
    }
    float norm[32] = {0};
    for (int f = 0; f < 12; ++f) {
        if (!(x_std[f] > 0.0f) || !std::isfinite(x_mean[f])) {
            fe_set_error_message("feature %d: std must be > 0", f);
            return FE_ERR_INVALID_ARGUMENT;
        }
        norm[f] = x_mean[f];
        norm[12 + f] = x_std[f];
    }
    for (int c = 0; c < 2; ++c) {
        if (!(y_std[c] > 0.0f) || !std::isfinite(y_mean[c])) {
            fe_set_error_message("target %d: std must be > 0", c);
            return FE_ERR_INVALID_ARGUMENT;
        }
        norm[24 + c] = y_mean[c];
        norm[26 + c] = y_std[c];
    }
    M_CUDA(cudaSetDevice(m->device));
    M_CUDA(cudaMemcpy(m->norm, norm, sizeof norm, cudaMemcpyHostToDevice));
    std::memcpy(m->h_norm, norm, sizeof norm);
    return FE_OK;
}

FE_API fe_status fe_model_get_normalization(const fe_model* m, float* out32) {
    if (!m || !out32) {
        fe_set_error_message("NULL argument");
        return FE_ERR_INVALID_ARGUMENT;
    }
    M_CUDA(cudaSetDevice(m->device));
    M_CUDA(cudaMemcpy(out32, m->norm, 32 * 4, cudaMemcpyDeviceToHost));
    return FE_OK;
}

FE_API fe_status fe_model_forward(fe_model* m, const float* d_x, float* d_y, uint32_t n, void* stream) {
    if (!m || ((!d_x || !d_y) && n)) {
        fe_set_error_message("NULL argument");
        return FE_ERR_INVALID_ARGUMENT;
    }
    if (n == 0) return FE_OK;
    cudaStream_t s = (cudaStream_t)stream;
    M_CUDA(cudaSetDevice(m->device));
    fe_status st = m->prepare_x(d_x, n, s);
    if (st != FE_OK) return st;
    M_CUDA(mlp::infer(m->params(), m->xb, d_y, n, m->flags, s, m->num_sms));
    k_destandardize_y<<<(2 * n + 255) / 256, 256, 0, s>>>(d_y, m->norm, n);
    M_CUDA(cudaGetLastError());
    return FE_OK;
}

static fe_status model_grads(fe_model* m, const float* d_x, const float* d_y, uint32_t n,
                             cudaStream_t s) {
    fe_status st = m->prepare_x(d_x, n, s);
    if (st != FE_OK) return st;
    k_standardize_y<<<(2 * n + 255) / 256, 256, 0, s>>>(d_y, m->norm, m->ys, n);
    M_CUDA(cudaGetLastError());
    M_CUDA(mlp::train_grads(m->params(), m->xb, m->ys, n, m->grad, m->grad_part, m->flags, s,
                            m->num_sms));
    return FE_OK;
}

FE_API fe_status fe_model_gradients(fe_model* m, const float* d_x, const float* d_y, uint32_t n,
                                    float* h_grads, float* h_loss) {
    if (!m || !d_x || !d_y || n == 0) {
        fe_set_error_message("NULL argument or n == 0");
        return FE_ERR_INVALID_ARGUMENT;
    }
    M_CUDA(cudaSetDevice(m->device));
    M_CUDA(cudaMemset(m->grad, 0, (mlp::kParams + 1) * 4));
    fe_status st = model_grads(m, d_x, d_y, n, nullptr);
    if (st != FE_OK) return st;
    M_CUDA(cudaDeviceSynchronize());
    uint32_t flags = 0;
    M_CUDA(cudaMemcpy(&flags, m->flags, 4, cudaMemcpyDeviceToHost));
    if (flags) {
        fe_set_error_message("tensor-core wait timed out");
        return FE_ERR_TIMEOUT;
    }
    if (h_grads) M_CUDA(cudaMemcpy(h_grads, m->grad, mlp::kParams * 4, cudaMemcpyDeviceToHost));
    if (h_loss) M_CUDA(cudaMemcpy(h_loss, m->grad + mlp::kParams, 4, cudaMemcpyDeviceToHost));
    M_CUDA(cudaMemset(m->grad, 0, (mlp::kParams + 1) * 4));
    return FE_OK;
}

FE_API fe_status fe_model_train_step(fe_model* m, const float* d_x, const float* d_y, uint32_t n,
                                     float lr, float weight_decay, void* stream, float* h_loss) {
    if (!m || !d_x || !d_y || n == 0 || !(lr > 0.0f)) {
        fe_set_error_message("NULL argument, n == 0 or lr <= 0");
        return FE_ERR_INVALID_ARGUMENT;
    }
    cudaStream_t s = (cudaStream_t)stream;
    M_CUDA(cudaSetDevice(m->device));
    if (h_loss) M_CUDA(cudaMemsetAsync(m->grad + mlp::kParams, 0, 4, s));
    fe_status st = model_grads(m, d_x, d_y, n, s);
    if (st != FE_OK) return st;
    m->step += 1;
    M_CUDA(mlp::adam(m->master, m->grad, m->adam_m, m->adam_v, m->wbf16, mlp::kParams,
                     mlp::kWeights, lr, 0.9f, 0.999f, 1e-8f, m->step, weight_decay, s));
    if (h_loss) {
        M_CUDA(cudaMemcpyAsync(h_loss, m->grad + mlp::kParams, 4, cudaMemcpyDeviceToHost, s));
        M_CUDA(cudaStreamSynchronize(s));
        *h_loss /= (float)n;
    }
    return FE_OK;
}

FE_API fe_status fe_model_read_flags(fe_model* m, uint32_t* flags) {
    if (!m || !flags) {
        fe_set_error_message("NULL argument");
        return FE_ERR_INVALID_ARGUMENT;
    }
    M_CUDA(cudaSetDevice(m->device));
    M_CUDA(cudaMemcpy(flags, m->flags, 4, cudaMemcpyDeviceToHost));
    return FE_OK;
}

}  // extern "C"
