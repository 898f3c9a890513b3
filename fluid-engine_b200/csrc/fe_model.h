// fe_model.h — internal layout of fe_model (the learned warm-start model).
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/fluid_step.h"
#include "fe_mlp.h"

struct fe_model {
    int device = 0;
    int num_sms = 148;
    float* master = nullptr;          // FP32 parameters (fe::mlp layout)
    float* grad = nullptr;            // gradients + 1 loss accumulator
    float* grad_part = nullptr;       // per-block gradient slices [num_sms][kParams + 1]
    float* adam_m = nullptr;
    float* adam_v = nullptr;
    __nv_bfloat16* wbf16 = nullptr;   // BF16 weights for the tensor cores
    float* norm = nullptr;            // x mean[12], x std[12], y mean[2], y std[2]
    float h_norm[32] = {0};
    uint32_t* flags = nullptr;        // device error word
    __nv_bfloat16* xb = nullptr;      // scratch: standardised BF16 rows
    float* ys = nullptr;              // scratch: standardised targets
    uint32_t scratch_rows = 0;
    uint32_t step = 0;

    fe_status ensure_scratch(uint32_t n);
    fe_status refresh_bf16(cudaStream_t s);
    fe_status prepare_x(const float* x, uint32_t n, cudaStream_t s);
    fe::mlp::Params params() const;
};
