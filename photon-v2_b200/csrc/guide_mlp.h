// Guiding network kernels (tcgen05 BF16 forward pass; training in guide_train.cu).
#pragma once

#include "guide.cuh"

#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace pg
{
namespace guide
{

// Bytes of the packed BF16 weight image the forward kernel copies into shared memory.
int image_bytes();

// FP32 parameters (kNumParams, packed order of guide.cuh) -> weight image.
void pack_image(const float* d_params, unsigned char* d_image, cudaStream_t s);

// Forward pass of n queries. d_features: [n][8] FP32 (7 used). d_out_raw: [n][40] FP32 raw
// outputs (decode() turns them into a mixture). d_out_acts (optional): [n][4][64] BF16 post-ReLU
// hidden activations, for training. Errors are OR-ed into *d_error (PG_DEV_ERR_GUIDE_WAIT).
// With d_n set, the kernel reads the row count from device memory (at most n): graph-safe.
// d_out_raw may be null when d_out_mix ([n][kMixFloats], decoded mixture) is given.
void launch_forward(const unsigned char* d_image, const float* d_features, uint32_t n, float* d_out_raw,
                    __nv_bfloat16* d_out_acts, uint32_t* d_error, cudaStream_t s, const uint32_t* d_n = nullptr,
                    float* d_out_mix = nullptr);

// Loss and gradient of a batch (forward pass included): d_grads += d loss / d params, *d_loss +=
// loss; d_total receives sum of weights. d_dirw: [n] (direction xyz, weight). d_raw: [n][40] and
// d_acts: [n][4][64] scratch.
// With d_n set, at most n samples and the count is read from device memory (graph-safe). With
// clamp_factor > 0, sample weights are first capped (in place) at clamp_factor x their mean.
// tensor_cores: the backward pass as BF16 tcgen05 MMAs with FP32 accumulation in tensor memory
// (default); false: the FP32 CUDA-core backward, kept as a cross-check.
void launch_gradients(const float* d_params, const unsigned char* d_image, const float* d_features,
                      const float4* d_dirw, uint32_t n, float* d_raw, __nv_bfloat16* d_acts,
                      float* d_grads, float* d_loss, float* d_total, uint32_t* d_error, cudaStream_t s,
                      const uint32_t* d_n = nullptr, float clamp_factor = 0.0f, bool tensor_cores = true);

// One Adam step (beta 0.9 / 0.999, eps 1e-8) on the FP32 parameters; zeroes d_grads. The step
// number t is *d_step + 1, and *d_step is incremented afterwards (graph-safe).
void launch_adam(float* d_params, float* d_grads, float* d_m, float* d_v, uint32_t* d_step, float lr, cudaStream_t s);

}// end namespace guide
}// end namespace pg
