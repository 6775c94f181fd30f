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
#include "tcgen05.cuh"
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

// ---------------------------------------------------------------------------------------------
// Backward pass on the tensor cores (tcgen05, BF16 operands, FP32 accumulators in TMEM).
//
// Per 128-sample tile and layer l (4 down to 0), with G_l = d loss / d z_l [128 x out_l] and
// X_l the layer's input [128 x in_l]:
//   dW_l += X_l^T G_l      MMA M = 128 (the layer's inputs, padded; one extra row of ones gives
//                           the bias gradient sum_t G_l[t]), N = out_l, K = 128 samples;
//   dX_l  = G_l W_l^T      MMA M = 128 samples, N = in_l = 64, K = out_l (layers 4..1);
//   G_l-1 = dX_l where X_l > 0 (the ReLU that produced X_l).
// The weight gradients stay in tensor memory across all tiles a CTA processes and reach global
// memory once per CTA. Operands: G_l as sample rows (K = out_l) for dX, and the transposed
// X_l^T / G_l^T (K = samples) for dW, written by each thread for its own sample; the transposed
// buffers' K-chunk stride carries 16 bytes of padding so that the 8 sample groups a warp writes
// land in different banks.

namespace tcb
{

using namespace tc;

constexpr int kThreads = 128;
constexpr uint32_t kLboG = kTile * 16u;                // G rows (samples) x K = outputs: 2048
constexpr uint32_t kLboXT = kTile * 16u + 16u;         // X^T: 128 rows x K = samples, padded: 2064
constexpr uint32_t kLboGT = kHidden * 16u + 16u;       // G^T: 64 rows x K = samples, padded: 1040
constexpr uint32_t kLboW = kHidden * 16u;              // W_l: 64 rows (inputs) x K = outputs: 1024

constexpr int kBwHidden = kHidden * kHidden * 2;       // 8,192
constexpr int kOffBw = 0;                              // W1, W2, W3, W4 (W4: K = 48)
constexpr int kOffG = kOffBw + 3 * kBwHidden + kHidden * kOutPad * 2;     // 30,720
constexpr int kOffXT = kOffG + kTile * kHidden * 2;                       // 47,104
constexpr int kOffGT = kOffXT + (kTile / 8) * static_cast<int>(kLboXT);   // 80,128
constexpr int kOffBar = kOffGT + (kTile / 8) * static_cast<int>(kLboGT);  // 96,768
constexpr int kOffSlot = kOffBar + 8;
// More than half an SM's shared memory: one CTA per SM, so that each CTA's 512 TMEM columns are free.
constexpr int kSmemBytes = 120 * 1024;
static_assert(kOffSlot + 8 <= kSmemBytes && kSmemBytes <= 227 * 1024, "shared memory");
static_assert(kOffG % 16 == 0 && kOffXT % 16 == 0 && kOffGT % 16 == 0 && kOffBar % 8 == 0, "alignment");

// TMEM columns: the dX accumulator, then the weight gradients of every layer (rows = the layer's
// inputs, columns = its outputs).
constexpr uint32_t kColAcc = 0;
constexpr uint32_t kColW0a = 64;    // inputs 0..127 of layer 0
constexpr uint32_t kColW0b = 128;   // inputs 128..223 of layer 0, bias in row 96
// layer l >= 1: 192, 256, 320, 384 (bias in row 64)
PG_HD constexpr uint32_t col_w(int l) { return l == 0 ? kColW0a : 128u + 64u * static_cast<uint32_t>(l); }
constexpr uint32_t kTmemColsB = 512;

__device__ __forceinline__ void st_bf16(unsigned char* base, uint32_t off, float v)
{
	*reinterpret_cast<__nv_bfloat16*>(base + off) = __float2bfloat16_rn(v);
}

__global__ void __launch_bounds__(kThreads, 1)
backward_tc_kernel(const float* __restrict__ params, const float* __restrict__ features,
                   const float4* __restrict__ dirw, const float* __restrict__ raw_out,
                   const __nv_bfloat16* __restrict__ acts, uint32_t n_max, const uint32_t* __restrict__ d_n,
                   const float* __restrict__ total_weight, float* __restrict__ grads, float* __restrict__ loss,
                   uint32_t* __restrict__ error)
{
	const uint32_t n = d_n ? min(*d_n, n_max) : n_max;
	const uint32_t num_tiles = (n + kTile - 1) / kTile;
	if(blockIdx.x >= num_tiles)
	{
		return;   // uniform per CTA, before any barrier or tensor-memory use
	}
	extern __shared__ __align__(128) unsigned char smem[];
	const uint32_t tid = threadIdx.x;
	const uint32_t warp = tid >> 5;

	// W_1..W_4 as B operands of dX: [64 rows = layer inputs][K = layer outputs], BF16 as the
	// forward pass rounds them
	for(uint32_t e = tid; e < 3u * kHidden * kHidden + kHidden * kOutPad; e += kThreads)
	{
		uint32_t l, i, o, out;
		if(e < 3u * kHidden * kHidden)
		{
			l = 1u + e / (kHidden * kHidden);
			i = (e % (kHidden * kHidden)) / kHidden;
			o = e % kHidden;
			out = kHidden;
		}
		else
		{
			l = 4u;
			i = (e - 3u * kHidden * kHidden) / kOutPad;
			o = (e - 3u * kHidden * kHidden) % kOutPad;
			out = kOut;
		}
		const int w_off[5] = {kOffW0, kOffW1, kOffW2, kOffW3, kOffW4};
		const float w = o < out ? params[w_off[l] + i * out + o] : 0.0f;
		st_bf16(smem + kOffBw + (l - 1u) * kBwHidden, core_offset_lbo(i, o, kLboW), w);
	}
	const uint32_t bar = smem_u32(smem + kOffBar);
	uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(smem + kOffSlot);
	if(tid == 0)
	{
		mbar_init(bar, 1);
		asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
	}
	if(warp == 0)
	{
		asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
		             :: "r"(smem_u32(tmem_slot)), "r"(kTmemColsB) : "memory");
		asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
	}
	fence_async_smem();
	fence_before_sync();
	__syncthreads();
	fence_after_sync();
	const uint32_t tmem = *tmem_slot;
	const uint32_t tmem_row = tmem + ((warp * 32u) << 16);

	unsigned char* gbuf = smem + kOffG;
	unsigned char* xt = smem + kOffXT;
	unsigned char* gt = smem + kOffGT;
	const uint32_t a_g = smem_u32(gbuf), a_xt = smem_u32(xt), a_gt = smem_u32(gt);

	uint32_t phase = 0;
	bool failed = false;
	// the staged operands -> one dW chain (and, for layers 4..1, one dX chain), committed and awaited
	auto run = [&](uint32_t col_w, uint32_t n_out, bool acc_w, int dx_layer) -> bool
	{
		fence_async_smem();
		fence_before_sync();
		__syncthreads();
		if(tid == 0)
		{
			fence_after_sync();
			const uint32_t idesc_w = instr_desc(kTile, n_out);
			for(uint32_t ks = 0; ks < kTile / 16u; ++ks)
			{
				const uint64_t ad = smem_desc(a_xt + ks * 2u * kLboXT, kLboXT, 128u);
				const uint64_t bd = smem_desc(a_gt + ks * 2u * kLboGT, kLboGT, 128u);
				mma_bf16(tmem + col_w, ad, bd, idesc_w, (acc_w || ks > 0) ? 1u : 0u);
			}
			if(dx_layer >= 1)
			{
				const uint32_t idesc_x = instr_desc(kTile, kHidden);
				const uint32_t w_base = smem_u32(smem + kOffBw + (dx_layer - 1) * kBwHidden);
				for(uint32_t ks = 0; ks < n_out / 16u; ++ks)
				{
					const uint64_t ad = smem_desc(a_g + ks * 2u * kLboG, kLboG, 128u);
					const uint64_t bd = smem_desc(w_base + ks * 2u * kLboW, kLboW, 128u);
					mma_bf16(tmem + kColAcc, ad, bd, idesc_x, ks > 0 ? 1u : 0u);
				}
			}
			mma_commit(bar);
		}
		// one thread polls the barrier; the others wait at the block barrier, which issues no
		// instructions while the MMAs run
		const bool ok = tid == 0 ? mbar_wait(bar, phase) : true;
		if(__syncthreads_or(ok ? 0 : 1))
		{
			if(!ok)
			{
				mbar_wait(bar, phase);   // bounded: do not free TMEM under running MMAs
			}
			return false;
		}
		phase ^= 1u;
		fence_after_sync();
		return true;
	};

	bool first = true;
	for(uint32_t tile = blockIdx.x; tile < num_tiles && !failed; tile += gridDim.x, first = false)
	{
		const uint32_t row = tile * kTile + tid;
		const bool valid = row < n;

		// ---- d loss / d raw outputs (48 columns, the last 8 zero)
		float g[kHidden];
		#pragma unroll
		for(int c = 0; c < kHidden; ++c)
		{
			g[c] = 0.0f;
		}
		float loss_term = 0.0f;
		if(valid)
		{
			float raw[kOut];
			#pragma unroll
			for(int c = 0; c < kOut; ++c)
			{
				raw[c] = raw_out[static_cast<size_t>(row) * kOut + c];
			}
			const float4 dw = dirw[row];
			const float scale = -dw.w / fmaxf(*total_weight, 1e-30f);
			output_gradient(raw, v3(dw.x, dw.y, dw.z), scale, g, &loss_term);
		}
		for(int o = 16; o > 0; o >>= 1)
		{
			loss_term += __shfl_xor_sync(0xFFFFFFFFu, loss_term, o);
		}
		if((tid & 31u) == 0u && loss_term != 0.0f)
		{
			atomicAdd(loss, loss_term);
		}

		// ---- layers 4..1: dW_l and dX_l together
		for(int l = 4; l >= 1 && !failed; --l)
		{
			const uint32_t n_out = l == 4 ? static_cast<uint32_t>(kOutPad) : static_cast<uint32_t>(kHidden);
			float x[kHidden];
			const uint4* src = reinterpret_cast<const uint4*>(acts + (static_cast<size_t>(row) * kHiddenLayers + (l - 1)) * kHidden);
			#pragma unroll
			for(int c = 0; c < kHidden / 8; ++c)
			{
				const uint4 q = valid ? src[c] : make_uint4(0u, 0u, 0u, 0u);
				const uint32_t w4[4] = {q.x, q.y, q.z, q.w};
				#pragma unroll
				for(int j = 0; j < 4; ++j)
				{
					x[8 * c + 2 * j] = __bfloat162float(__ushort_as_bfloat16(static_cast<unsigned short>(w4[j] & 0xFFFFu)));
					x[8 * c + 2 * j + 1] = __bfloat162float(__ushort_as_bfloat16(static_cast<unsigned short>(w4[j] >> 16)));
				}
			}
			// X_l^T (+ the ones row) and G_l^T, transposed; G_l as this sample's row
			#pragma unroll
			for(int f = 0; f < kHidden; ++f)
			{
				st_bf16(xt, core_offset_lbo(static_cast<uint32_t>(f), tid, kLboXT), x[f]);
			}
			st_bf16(xt, core_offset_lbo(kHidden, tid, kLboXT), 1.0f);
			#pragma unroll
			for(int o = 0; o < kHidden; ++o)
			{
				if(o < static_cast<int>(n_out))
				{
					st_bf16(gt, core_offset_lbo(static_cast<uint32_t>(o), tid, kLboGT), g[o]);
				}
			}
			#pragma unroll
			for(int c = 0; c < kHidden / 8; ++c)
			{
				if(c * 8 < static_cast<int>(n_out))
				{
					uint4 q;
					q.x = pack_bf16x2(g[8 * c + 0], g[8 * c + 1]);
					q.y = pack_bf16x2(g[8 * c + 2], g[8 * c + 3]);
					q.z = pack_bf16x2(g[8 * c + 4], g[8 * c + 5]);
					q.w = pack_bf16x2(g[8 * c + 6], g[8 * c + 7]);
					*reinterpret_cast<uint4*>(gbuf + core_offset_lbo(tid, static_cast<uint32_t>(8 * c), kLboG)) = q;
				}
			}
			if(!run(col_w(l), n_out, !first, l))
			{
				failed = true;
				break;
			}
			// G_l-1 = dX_l through the ReLU that produced X_l
			float acc[kHidden];
			#pragma unroll
			for(int c = 0; c < 4; ++c)
			{
				tmem_ld16(tmem_row + kColAcc + c * 16, acc + c * 16);
			}
			tmem_wait_ld();
			#pragma unroll
			for(int c = 0; c < kHidden; ++c)
			{
				g[c] = x[c] > 0.0f ? acc[c] : 0.0f;
			}
			fence_before_sync();
			__syncthreads();   // every thread's accumulator row is read before the next chain
		}
		if(failed)
		{
			break;
		}

		// ---- layer 0: dW_0 in two halves of its 224 one-blob inputs
		float f7[kInputs];
		#pragma unroll
		for(int i = 0; i < kInputs; ++i)
		{
			f7[i] = valid ? features[static_cast<size_t>(row) * 8 + i] : 0.0f;
		}
		#pragma unroll
		for(int o = 0; o < kHidden; ++o)
		{
			st_bf16(gt, core_offset_lbo(static_cast<uint32_t>(o), tid, kLboGT), g[o]);
		}
		// unrolled over the inputs so that f7 stays in registers (indexed at run time it went to
		// local memory)
		#pragma unroll
		for(int half = 0; half < 2; ++half)
		{
			const int k0 = half * 128;
			#pragma unroll
			for(int i = half * 4; i < (half == 0 ? 4 : kInputs); ++i)
			{
				#pragma unroll 8
				for(int b = 0; b < kBins; ++b)
				{
					st_bf16(xt, core_offset_lbo(static_cast<uint32_t>(i * kBins + b - k0), tid, kLboXT), one_blob(f7[i], b));
				}
			}
			if(half == 1)
			{
				st_bf16(xt, core_offset_lbo(static_cast<uint32_t>(kIn - 128), tid, kLboXT), 1.0f);
			}
			if(!run(half == 0 ? kColW0a : kColW0b, kHidden, !first, 0))
			{
				failed = true;
				break;
			}
			fence_before_sync();
			__syncthreads();
		}
	}

	if(!failed)
	{
		// ---- the CTA's weight gradients to global memory: thread t holds row t of each block
		auto flush = [&](uint32_t col, uint32_t n_out, int w_off, int b_off, uint32_t rows, uint32_t bias_row,
		                 uint32_t first_input, uint32_t out_stride)
		{
			float v[kHidden];
			for(uint32_t c = 0; c < n_out; c += 16)
			{
				tmem_ld16(tmem_row + col + c, v + c);
			}
			tmem_wait_ld();
			if(tid < rows)
			{
				float* dst = grads + w_off + (first_input + tid) * out_stride;
				for(uint32_t c = 0; c < out_stride; ++c)
				{
					if(v[c] != 0.0f) { atomicAdd(dst + c, v[c]); }
				}
			}
			else if(tid == bias_row)
			{
				for(uint32_t c = 0; c < out_stride; ++c)
				{
					if(v[c] != 0.0f) { atomicAdd(grads + b_off + c, v[c]); }
				}
			}
		};
		flush(kColW0a, kHidden, kOffW0, kOffB0, 128u, 0xFFFFFFFFu, 0u, kHidden);
		flush(kColW0b, kHidden, kOffW0, kOffB0, static_cast<uint32_t>(kIn - 128), static_cast<uint32_t>(kIn - 128),
		      128u, kHidden);
		flush(col_w(1), kHidden, kOffW1, kOffB1, kHidden, kHidden, 0u, kHidden);
		flush(col_w(2), kHidden, kOffW2, kOffB2, kHidden, kHidden, 0u, kHidden);
		flush(col_w(3), kHidden, kOffW3, kOffB3, kHidden, kHidden, 0u, kHidden);
		flush(col_w(4), kOutPad, kOffW4, kOffB4, kHidden, kHidden, 0u, kOut);
	}
	else if(tid == 0)
	{
		atomicOr(error, PG_DEV_ERR_GUIDE_WAIT);
	}
	fence_before_sync();
	__syncthreads();
	if(warp == 0)
	{
		asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(tmem), "r"(kTmemColsB) : "memory");
	}
}

}// end namespace tcb

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
                      const uint32_t* d_n, float clamp_factor, bool tensor_cores)
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
	if(tensor_cores)
	{
		static const bool configured_tc = []
		{
			PG_CUDA_CHECK(cudaFuncSetAttribute(tcb::backward_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
			                                   tcb::kSmemBytes));
			return true;
		}();
		(void)configured_tc;
		// one CTA per SM: a batch of up to one tile per SM runs in one round of tiles; larger
		// batches keep their weight gradients in TMEM across each CTA's tiles, and every CTA adds
		// them to global memory once
		const uint32_t tiles = (n + kTile - 1) / kTile;
		const uint32_t grid = std::max(1u, std::min(tiles, static_cast<uint32_t>(sm_count())));
		tcb::backward_tc_kernel<<<grid, tcb::kThreads, tcb::kSmemBytes, s>>>(d_params, d_features, d_dirw, d_raw, d_acts,
		                                                                     n, d_n, d_total, d_grads, d_loss, d_error);
		PG_CUDA_CHECK(cudaGetLastError());
		return;
	}
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
	return pgpu_guide_gradients_ex(params, features, dirs, weights, n, 0u, out_loss, out_grads);
}

int pgpu_guide_gradients_ex(const float* params, const float* features, const float* dirs, const float* weights,
                            uint64_t n, uint32_t flags, float* out_loss, float* out_grads)
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
		                        d_err.get(), s, nullptr, 0.0f, (flags & PG_GUIDE_BACKWARD_CUDA_CORES) == 0u);
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
