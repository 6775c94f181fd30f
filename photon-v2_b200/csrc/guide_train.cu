// Guiding network training: loss gradient, backward pass and Adam.
//
// A training batch is n samples (features, sampled direction, weight). The forward pass runs on
// the tensor cores (guide_mlp.cu) and keeps the BF16 hidden activations; this file computes
//   loss = -sum_i w_i log q(d_i | x_i) / sum_i w_i
// (the KL divergence to the target density up to a constant, Mueller et al. 2019) and its gradient
// with respect to every parameter, then applies Adam to the FP32 master parameters.
//
// Backward pass: one block of 128 threads per 128 samples, thread = sample. Each thread turns its
// raw outputs into d loss / d raw (the analytic derivative of the vMF mixture's log density) and
// back-propagates through the layers with the same BF16-rounded weights the forward pass used.
// Per layer, the block stages the layer inputs and pre-activation gradients of its 128 samples in
// shared memory and reduces the weight gradient sum_t x[t][i] dz[t][o] over them (FP32), adding
// the block's partial to the global gradient with one atomic per weight.
#include "guide_mlp.h"

#include "pg_runtime.h"
#include "../../include/photon_gpu.h"

#include <cuda_bf16.h>

#include <cstring>
#include <vector>

namespace pg
{
namespace guide
{

namespace
{

constexpr int kBlock = 128;
constexpr int kPitch = kHidden + 1;   // shared-memory row pitch (floats), avoids bank conflicts

__device__ __forceinline__ float bf16r(float x)
{
	return __bfloat162float(__float2bfloat16_rn(x));
}

__global__ void weight_sum_kernel(const float4* __restrict__ dirw, uint32_t n_max, const uint32_t* __restrict__ d_n,
                                  float* __restrict__ total)
{
	const uint32_t n = d_n ? min(*d_n, n_max) : n_max;
	float s = 0.0f;
	for(uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
	{
		s += dirw[i].w;
	}
	for(int o = 16; o > 0; o >>= 1)
	{
		s += __shfl_xor_sync(0xFFFFFFFFu, s, o);
	}
	if((threadIdx.x & 31) == 0)
	{
		atomicAdd(total, s);
	}
}

// Caps every sample weight at factor x the batch's mean weight (the sum in *total), in place.
__global__ void clamp_weights_kernel(float4* __restrict__ dirw, uint32_t n_max, const uint32_t* __restrict__ d_n,
                                     const float* __restrict__ total, float factor)
{
	const uint32_t n = d_n ? min(*d_n, n_max) : n_max;
	if(n == 0u)
	{
		return;
	}
	const float cap = factor * *total / static_cast<float>(n);
	for(uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
	{
		dirw[i].w = fminf(dirw[i].w, cap);
	}
}

// d loss / d raw for one sample (40 values) and its loss term.
__device__ void output_gradient(const float* raw, V3 d, float scale, float* g, float* loss_term)
{
	Mixture m = decode(raw);
	float v[kLobes];
	float q = 0.0f;
	#pragma unroll
	for(int j = 0; j < kLobes; ++j)
	{
		v[j] = vmf_pdf(m.mu[j], m.kappa[j], d);
		q += m.w[j] * v[j];
	}
	q = fmaxf(q, 1e-30f);
	*loss_term = scale * logf(q);   // scale = -w / total
	#pragma unroll
	for(int j = 0; j < kLobes; ++j)
	{
		const float r = m.w[j] * v[j] / q;
		const float k = m.kappa[j];
		const float cosv = dot(m.mu[j], d);
		g[5 * j + 0] = scale * (r - m.w[j]);
		const float e = expf(-2.0f * k);
		const float dlogv_dk = 1.0f / k - 2.0f * e / (1.0f - e) + (cosv - 1.0f);
		const float k_raw = expf(raw[5 * j + 4]);
		const bool inside = k_raw > kMinKappa && k_raw < kMaxKappa;
		g[5 * j + 4] = inside ? scale * r * dlogv_dk * k : 0.0f;
		const V3 mraw = v3(raw[5 * j + 1], raw[5 * j + 2], raw[5 * j + 3]);
		const float norm = fmaxf(sqrtf(dot(mraw, mraw)), 1e-30f);
		const float c = scale * r * k / norm;
		g[5 * j + 1] = c * (d.x - cosv * m.mu[j].x);
		g[5 * j + 2] = c * (d.y - cosv * m.mu[j].y);
		g[5 * j + 3] = c * (d.z - cosv * m.mu[j].z);
	}
}

// Adds sum_t x[t][i] * dz[t][o] over the block's samples to grad[i * out_dim + o] (i < in_rows).
__device__ void reduce_weight_grad(const float* sx, const float* sd, int in_rows, int out_dim, float* grad)
{
	for(int e = threadIdx.x; e < in_rows * out_dim; e += kBlock)
	{
		const int i = e / out_dim, o = e % out_dim;
		float acc = 0.0f;
		for(int t = 0; t < kBlock; ++t)
		{
			acc += sx[t * kPitch + i] * sd[t * kPitch + o];
		}
		if(acc != 0.0f)
		{
			atomicAdd(grad + e, acc);
		}
	}
}

__device__ void reduce_bias_grad(const float* sd, int out_dim, float* grad)
{
	for(int o = threadIdx.x; o < out_dim; o += kBlock)
	{
		float acc = 0.0f;
		for(int t = 0; t < kBlock; ++t)
		{
			acc += sd[t * kPitch + o];
		}
		if(acc != 0.0f)
		{
			atomicAdd(grad + o, acc);
		}
	}
}

__global__ void __launch_bounds__(kBlock)
backward_kernel(const float* __restrict__ params, const float* __restrict__ features,
                const float4* __restrict__ dirw, const float* __restrict__ raw_out,
                const __nv_bfloat16* __restrict__ acts, uint32_t n_max, const uint32_t* __restrict__ d_n,
                const float* __restrict__ total_weight, float* __restrict__ grads, float* __restrict__ loss)
{
	const uint32_t n = d_n ? min(*d_n, n_max) : n_max;
	if(blockIdx.x * kBlock >= n)
	{
		return;   // whole block past the live samples (uniform exit before any barrier)
	}
	extern __shared__ float smem_f[];   // sx, sd: [kBlock][kPitch] each (dynamic, 66 KB)
	float* sx = smem_f;
	float* sd = smem_f + kBlock * kPitch;
	__shared__ float sloss[kBlock / 32];
	const int tid = threadIdx.x;
	const uint32_t row = blockIdx.x * kBlock + tid;
	const bool valid = row < n;

	// ---- d loss / d out
	float g[kOut];
	float loss_term = 0.0f;
	if(valid)
	{
		float raw[kOut];
		#pragma unroll
		for(int i = 0; i < kOut; ++i)
		{
			raw[i] = raw_out[static_cast<size_t>(row) * kOut + i];
		}
		const float4 dw = dirw[row];
		const float scale = -dw.w / fmaxf(*total_weight, 1e-30f);
		output_gradient(raw, v3(dw.x, dw.y, dw.z), scale, g, &loss_term);
	}
	else
	{
		#pragma unroll
		for(int i = 0; i < kOut; ++i)
		{
			g[i] = 0.0f;
		}
	}
	for(int o = 16; o > 0; o >>= 1)
	{
		loss_term += __shfl_xor_sync(0xFFFFFFFFu, loss_term, o);
	}
	if((tid & 31) == 0)
	{
		sloss[tid >> 5] = loss_term;
	}

	// layer inputs x_l of this sample (x_1..x_4: BF16 activations of the forward pass)
	auto load_act = [&](int layer, float* x)
	{
		#pragma unroll
		for(int c = 0; c < kHidden; ++c)
		{
			x[c] = valid ? __bfloat162float(acts[(static_cast<size_t>(row) * kHiddenLayers + layer) * kHidden + c]) : 0.0f;
		}
	};

	// ---- output layer: dW4 = x4^T g, db4 = sum g, dx4 = W4 g
	float x[kHidden], dz[kHidden];
	load_act(3, x);
	#pragma unroll
	for(int c = 0; c < kHidden; ++c)
	{
		sx[tid * kPitch + c] = x[c];
		sd[tid * kPitch + c] = c < kOut ? g[c] : 0.0f;
	}
	__syncthreads();
	if(tid == 0)
	{
		float s = 0.0f;
		for(int w = 0; w < kBlock / 32; ++w)
		{
			s += sloss[w];
		}
		atomicAdd(loss, s);
	}
	reduce_weight_grad(sx, sd, kHidden, kOut, grads + kOffW4);
	reduce_bias_grad(sd, kOut, grads + kOffB4);
	#pragma unroll 4
	for(int i = 0; i < kHidden; ++i)
	{
		float acc = 0.0f;
		#pragma unroll
		for(int o = 0; o < kOut; ++o)
		{
			acc += bf16r(__ldg(params + kOffW4 + i * kOut + o)) * g[o];
		}
		dz[i] = x[i] > 0.0f ? acc : 0.0f;   // through the ReLU that produced x4
	}

	// ---- hidden layers 3, 2, 1, then the input layer 0
	const int w_off[4] = {kOffW0, kOffW1, kOffW2, kOffW3};
	const int b_off[4] = {kOffB0, kOffB1, kOffB2, kOffB3};
	for(int l = 3; l >= 1; --l)
	{
		load_act(l - 1, x);   // x_l, the input of layer l
		__syncthreads();      // previous reductions are done with sx / sd
		#pragma unroll
		for(int c = 0; c < kHidden; ++c)
		{
			sx[tid * kPitch + c] = x[c];
			sd[tid * kPitch + c] = dz[c];
		}
		__syncthreads();
		reduce_weight_grad(sx, sd, kHidden, kHidden, grads + w_off[l]);
		reduce_bias_grad(sd, kHidden, grads + b_off[l]);
		// dz of the layer below, reading this layer's dz back from shared memory
		const float* my_dz = sd + tid * kPitch;
		#pragma unroll 4
		for(int i = 0; i < kHidden; ++i)
		{
			float acc = 0.0f;
			#pragma unroll 8
			for(int o = 0; o < kHidden; ++o)
			{
				acc += bf16r(__ldg(params + w_off[l] + i * kHidden + o)) * my_dz[o];
			}
			dz[i] = x[i] > 0.0f ? acc : 0.0f;
		}
	}

	// input layer: x_0 is the one-blob encoding, recomputed in 64-column chunks
	__syncthreads();
	#pragma unroll
	for(int c = 0; c < kHidden; ++c)
	{
		sd[tid * kPitch + c] = dz[c];
	}
	float f[kInputs];
	#pragma unroll
	for(int i = 0; i < kInputs; ++i)
	{
		f[i] = valid ? features[static_cast<size_t>(row) * 8 + i] : 0.0f;
	}
	for(int chunk = 0; chunk * kHidden < kIn; ++chunk)
	{
		const int cols = min(kHidden, kIn - chunk * kHidden);
		__syncthreads();
		for(int c = 0; c < cols; ++c)
		{
			const int k = chunk * kHidden + c;
			sx[tid * kPitch + c] = valid ? bf16r(one_blob(f[k / kBins], k % kBins)) : 0.0f;
		}
		__syncthreads();
		reduce_weight_grad(sx, sd, cols, kHidden, grads + kOffW0 + chunk * kHidden * kHidden);
		if(chunk == 0)
		{
			reduce_bias_grad(sd, kHidden, grads + kOffB0);
		}
	}
}

__global__ void adam_kernel(float* __restrict__ params, float* __restrict__ grads, float* __restrict__ m,
                            float* __restrict__ v, uint32_t count, float lr, float beta1, float beta2,
                            float eps, const uint32_t* __restrict__ step)
{
	const float t = static_cast<float>(*step + 1u);
	const float bias1 = 1.0f - powf(beta1, t);
	const float bias2 = 1.0f - powf(beta2, t);
	for(uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x)
	{
		const float g = grads[i];
		const float mi = beta1 * m[i] + (1.0f - beta1) * g;
		const float vi = beta2 * v[i] + (1.0f - beta2) * g * g;
		m[i] = mi;
		v[i] = vi;
		params[i] -= lr * (mi / bias1) / (sqrtf(vi / bias2) + eps);
		grads[i] = 0.0f;
	}
}

__global__ void step_kernel(uint32_t* step)
{
	++*step;
}

}// end anonymous namespace

void launch_gradients(const float* d_params, const unsigned char* d_image, const float* d_features,
                      const float4* d_dirw, uint32_t n, float* d_raw, __nv_bfloat16* d_acts,
                      float* d_grads, float* d_loss, float* d_total, uint32_t* d_error, cudaStream_t s,
                      const uint32_t* d_n, float clamp_factor)
{
	if(n == 0)
	{
		return;
	}
	PG_CUDA_CHECK(cudaMemsetAsync(d_total, 0, sizeof(float), s));
	weight_sum_kernel<<<64, 256, 0, s>>>(d_dirw, n, d_n, d_total);
	PG_CUDA_CHECK(cudaGetLastError());
	if(clamp_factor > 0.0f)
	{
		// rare, very bright samples would otherwise dominate single steps
		clamp_weights_kernel<<<64, 256, 0, s>>>(const_cast<float4*>(d_dirw), n, d_n, d_total, clamp_factor);
		PG_CUDA_CHECK(cudaMemsetAsync(d_total, 0, sizeof(float), s));
		weight_sum_kernel<<<64, 256, 0, s>>>(d_dirw, n, d_n, d_total);
		PG_CUDA_CHECK(cudaGetLastError());
	}
	launch_forward(d_image, d_features, n, d_raw, d_acts, d_error, s, d_n);
	constexpr int smem_bytes = 2 * kBlock * kPitch * sizeof(float);
	static const bool configured = []
	{
		PG_CUDA_CHECK(cudaFuncSetAttribute(backward_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_bytes));
		return true;
	}();
	(void)configured;
	backward_kernel<<<(n + kBlock - 1) / kBlock, kBlock, smem_bytes, s>>>(d_params, d_features, d_dirw, d_raw, d_acts,
	                                                                     n, d_n, d_total, d_grads, d_loss);
	PG_CUDA_CHECK(cudaGetLastError());
}

void launch_adam(float* d_params, float* d_grads, float* d_m, float* d_v, uint32_t* d_step, float lr, cudaStream_t s)
{
	adam_kernel<<<64, 256, 0, s>>>(d_params, d_grads, d_m, d_v, kNumParams, lr, 0.9f, 0.999f, 1e-8f, d_step);
	PG_CUDA_CHECK(cudaGetLastError());
	step_kernel<<<1, 1, 0, s>>>(d_step);
	PG_CUDA_CHECK(cudaGetLastError());
}

}// end namespace guide
}// end namespace pg

using namespace pg;

namespace
{

// Host [n][7] features, [n][3] directions, [n] weights -> device [n][8] and [n] float4.
void upload_batch(const float* features, const float* dirs, const float* weights, uint64_t n,
                  DeviceBuffer<float>& d_feat, DeviceBuffer<float4>& d_dirw, cudaStream_t s)
{
	std::vector<float> feat(n * 8, 0.0f);
	std::vector<float4> dw(n);
	for(uint64_t i = 0; i < n; ++i)
	{
		std::memcpy(&feat[i * 8], features + i * guide::kInputs, sizeof(float) * guide::kInputs);
		dw[i] = make_float4(dirs[3 * i], dirs[3 * i + 1], dirs[3 * i + 2], weights[i]);
	}
	PG_CUDA_CHECK(cudaMemcpyAsync(d_feat.get(), feat.data(), d_feat.bytes(), cudaMemcpyHostToDevice, s));
	PG_CUDA_CHECK(cudaMemcpyAsync(d_dirw.get(), dw.data(), d_dirw.bytes(), cudaMemcpyHostToDevice, s));
}

}// end anonymous namespace

extern "C" {

int pgpu_guide_gradients(const float* params, const float* features, const float* dirs, const float* weights,
                         uint64_t n, float* out_loss, float* out_grads)
{
	return guarded([&]
	{
		if(!params || !out_grads || n == 0 || !features || !dirs || !weights)
		{
			throw Error(PG_ERR_INVALID_ARGUMENT, "pgpu_guide_gradients: empty batch or null pointer");
		}
		if(n > (1u << 24))
		{
			throw Error(PG_ERR_INVALID_ARGUMENT, "pgpu_guide_gradients: batch too large");
		}
		require_device();
		cudaStream_t s = library_stream();
		DeviceBuffer<float> d_params(guide::kNumParams), d_grads(guide::kNumParams);
		DeviceBuffer<unsigned char> d_image(guide::image_bytes());
		DeviceBuffer<float> d_feat(n * 8), d_raw(n * guide::kOut), d_scalars(2);
		DeviceBuffer<float4> d_dirw(n);
		DeviceBuffer<__nv_bfloat16> d_acts(n * guide::kHiddenLayers * guide::kHidden);
		DeviceBuffer<uint32_t> d_err(1);
		PG_CUDA_CHECK(cudaMemsetAsync(d_err.get(), 0, sizeof(uint32_t), s));
		PG_CUDA_CHECK(cudaMemsetAsync(d_grads.get(), 0, d_grads.bytes(), s));
		PG_CUDA_CHECK(cudaMemsetAsync(d_scalars.get(), 0, d_scalars.bytes(), s));
		PG_CUDA_CHECK(cudaMemcpyAsync(d_params.get(), params, d_params.bytes(), cudaMemcpyHostToDevice, s));
		upload_batch(features, dirs, weights, n, d_feat, d_dirw, s);
		guide::pack_image(d_params.get(), d_image.get(), s);
		guide::launch_gradients(d_params.get(), d_image.get(), d_feat.get(), d_dirw.get(), static_cast<uint32_t>(n),
		                        d_raw.get(), d_acts.get(), d_grads.get(), d_scalars.get(), d_scalars.get() + 1,
		                        d_err.get(), s);
		float scalars[2] = {0.0f, 0.0f};
		uint32_t err = 0;
		PG_CUDA_CHECK(cudaMemcpyAsync(out_grads, d_grads.get(), d_grads.bytes(), cudaMemcpyDeviceToHost, s));
		PG_CUDA_CHECK(cudaMemcpyAsync(scalars, d_scalars.get(), sizeof(scalars), cudaMemcpyDeviceToHost, s));
		PG_CUDA_CHECK(cudaMemcpyAsync(&err, d_err.get(), sizeof(err), cudaMemcpyDeviceToHost, s));
		PG_CUDA_CHECK(cudaStreamSynchronize(s));
		if(err)
		{
			throw Error(PG_ERR_CUDA, "guiding network: tensor-core wait timed out");
		}
		if(out_loss) { *out_loss = scalars[0]; }
	});
}

int pgpu_guide_train(float* params, const float* features, const float* dirs, const float* weights,
                     uint64_t n, uint32_t steps, uint32_t batch, float lr, float* out_losses)
{
	return guarded([&]
	{
		if(!params || n == 0 || !features || !dirs || !weights || steps == 0 || batch == 0)
		{
			throw Error(PG_ERR_INVALID_ARGUMENT, "pgpu_guide_train: empty input");
		}
		if(n > (1u << 24))
		{
			throw Error(PG_ERR_INVALID_ARGUMENT, "pgpu_guide_train: data set too large");
		}
		require_device();
		cudaStream_t s = library_stream();
		const uint32_t b = static_cast<uint32_t>(std::min<uint64_t>(batch, n));
		DeviceBuffer<float> d_params(guide::kNumParams), d_grads(guide::kNumParams), d_m(guide::kNumParams),
			d_v(guide::kNumParams);
		DeviceBuffer<unsigned char> d_image(guide::image_bytes());
		DeviceBuffer<float> d_feat(n * 8), d_raw(b * guide::kOut), d_scalars(2 * steps);
		DeviceBuffer<float4> d_dirw(n);
		DeviceBuffer<__nv_bfloat16> d_acts(static_cast<size_t>(b) * guide::kHiddenLayers * guide::kHidden);
		DeviceBuffer<uint32_t> d_err(1), d_step(1);
		PG_CUDA_CHECK(cudaMemsetAsync(d_err.get(), 0, sizeof(uint32_t), s));
		PG_CUDA_CHECK(cudaMemsetAsync(d_step.get(), 0, sizeof(uint32_t), s));
		PG_CUDA_CHECK(cudaMemsetAsync(d_grads.get(), 0, d_grads.bytes(), s));
		PG_CUDA_CHECK(cudaMemsetAsync(d_m.get(), 0, d_m.bytes(), s));
		PG_CUDA_CHECK(cudaMemsetAsync(d_v.get(), 0, d_v.bytes(), s));
		PG_CUDA_CHECK(cudaMemsetAsync(d_scalars.get(), 0, d_scalars.bytes(), s));
		PG_CUDA_CHECK(cudaMemcpyAsync(d_params.get(), params, d_params.bytes(), cudaMemcpyHostToDevice, s));
		upload_batch(features, dirs, weights, n, d_feat, d_dirw, s);
		for(uint32_t step = 0; step < steps; ++step)
		{
			const uint32_t first = static_cast<uint32_t>((static_cast<uint64_t>(step) * b) % n);
			const uint32_t count = std::min<uint32_t>(b, static_cast<uint32_t>(n - first));
			guide::pack_image(d_params.get(), d_image.get(), s);
			guide::launch_gradients(d_params.get(), d_image.get(), d_feat.get() + static_cast<size_t>(first) * 8,
			                        d_dirw.get() + first, count, d_raw.get(), d_acts.get(), d_grads.get(),
			                        d_scalars.get() + 2 * step, d_scalars.get() + 2 * step + 1, d_err.get(), s);
			guide::launch_adam(d_params.get(), d_grads.get(), d_m.get(), d_v.get(), d_step.get(), lr, s);
		}
		std::vector<float> scalars(2 * steps);
		uint32_t err = 0;
		PG_CUDA_CHECK(cudaMemcpyAsync(params, d_params.get(), d_params.bytes(), cudaMemcpyDeviceToHost, s));
		PG_CUDA_CHECK(cudaMemcpyAsync(scalars.data(), d_scalars.get(), d_scalars.bytes(), cudaMemcpyDeviceToHost, s));
		PG_CUDA_CHECK(cudaMemcpyAsync(&err, d_err.get(), sizeof(err), cudaMemcpyDeviceToHost, s));
		PG_CUDA_CHECK(cudaStreamSynchronize(s));
		if(err)
		{
			throw Error(PG_ERR_CUDA, "guiding network: tensor-core wait timed out");
		}
		if(out_losses)
		{
			for(uint32_t i = 0; i < steps; ++i)
			{
				out_losses[i] = scalars[2 * i];
			}
		}
	});
}

}// extern "C"
