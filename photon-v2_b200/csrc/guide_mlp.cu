// Guiding network on the 5th-generation tensor cores: fused forward pass of the whole MLP with
// tcgen05.mma (BF16 operands in shared memory, FP32 accumulators in tensor memory).
//
// Two CTAs of 256 threads per SM walk 128-row tiles of queries; each row is owned by two threads
// (part 0: threads 0-127, part 1: threads 128-255, thread t and t + 128 on row t), so that the
// per-row work between the MMAs is split in two and each SM has 16 warps to hide its latency.
// Per tile:
//   1. the two threads of a row one-blob encode its inputs (alternating inputs) into the A
//      operand buffer (BF16, 224 columns, fed to the MMAs in two K halves);
//   2. per layer, one elected thread issues the K/16 MMAs (M = 128, N = 64 or 48, K = 16 each)
//      into tensor memory and commits them to an mbarrier;
//   3. after the barrier completes, each thread reads its half of its row of the accumulator
//      (tcgen05.ld from the TMEM lane of the row: warps w and w + 4 share lanes 32 (w % 4) ...),
//      adds the bias, applies ReLU, rounds to BF16 and writes it as the next layer's A operand;
//      after the last layer each thread decodes 4 of the row's 8 lobes (the softmax's maximum and
//      sum are exchanged through shared memory) or writes its 20 raw outputs.
// All weights (BF16, 59 KB) stay resident in shared memory for the kernel's lifetime.
//
// Operand layout: K-major, no swizzle. A core matrix is 8 rows x 16 bytes (8 BF16 along K); for a
// matrix of R rows, element (r, k) lives at
//   (k / 8) * (R * 16) + (r / 8) * 128 + (r % 8) * 16 + (k % 8) * 2,
// so the descriptor's leading byte offset (between K chunks) is R * 16 and its stride byte offset
// (between 8-row groups) is 128. Weights are stored transposed (W^T, [out][in]) so that both
// operands are K-major: D[M x N] = A[M x K] * B[N x K]^T.
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

using namespace tc;

constexpr int kThreads = 256;                 // two threads per tile row
constexpr int kParts = kThreads / kTile;
constexpr uint32_t kTmemCols = 128;   // power of two >= 64 accumulator columns
static_assert(kParts == 2 && kHidden == 64 && kLobes == 8 && kOut == 40 && kOutPad == 48,
              "the column split below assumes two parts, 64 hidden units and 8 lobes");

// ---- shared-memory image of the weights (also the device-side packed format)
constexpr int kW0Bytes = kHidden * kIn * 2;         // 28,672
constexpr int kWhBytes = kHidden * kHidden * 2;     //  8,192
constexpr int kW4Bytes = kOutPad * kHidden * 2;     //  6,144
constexpr int kOffImgW0 = 0;
constexpr int kOffImgW1 = kOffImgW0 + kW0Bytes;
constexpr int kOffImgW2 = kOffImgW1 + kWhBytes;
constexpr int kOffImgW3 = kOffImgW2 + kWhBytes;
constexpr int kOffImgW4 = kOffImgW3 + kWhBytes;
constexpr int kOffImgBias = kOffImgW4 + kW4Bytes;   // FP32 biases: 4 x 64 + 48
constexpr int kBiasCount = kHiddenLayers * kHidden + kOutPad;
constexpr int kImageBytes = kOffImgBias + kBiasCount * 4;   // 60,576

// ---- activation buffers
// The input layer is fed in two K halves (one-blob inputs 0-3, then 4-6) so that the A buffer is
// 32 KB and two CTAs fit on an SM.
constexpr int kInHalf0 = 4 * kBins;                 // 128 columns
constexpr int kInHalf1 = kIn - kInHalf0;            //  96 columns
constexpr int kActInBytes = kTile * kInHalf0 * 2;   // 32,768: input half, later hidden ping
constexpr int kActHBytes = kTile * kHidden * 2;     // 16,384: hidden pong
constexpr int kOffSmemImage = 0;
constexpr int kOffSmemActIn = (kImageBytes + 1023) / 1024 * 1024;
constexpr int kOffSmemActH = kOffSmemActIn + kActInBytes;
constexpr int kOffSmemXch = kOffSmemActH + kActHBytes;         // [part][row] float2: softmax max, sum
constexpr int kOffSmemBar = kOffSmemXch + kParts * kTile * 8;  // 8-byte aligned
constexpr int kOffSmemTmem = kOffSmemBar + 8;
constexpr int kSmemBytes = kOffSmemTmem + 8;
static_assert(kImageBytes % 16 == 0 && kOffSmemActH % 16 == 0 && kOffSmemBar % 8 == 0, "alignment");
static_assert(kSmemBytes <= 227 * 1024, "shared memory");

// Writes 8 consecutive K values of row r (k0 multiple of 8) of an A-layout buffer.
__device__ __forceinline__ void store_row8(unsigned char* buf, uint32_t r, uint32_t k0, const float* v)
{
	uint4 q;
	q.x = pack_bf16x2(v[0], v[1]);
	q.y = pack_bf16x2(v[2], v[3]);
	q.z = pack_bf16x2(v[4], v[5]);
	q.w = pack_bf16x2(v[6], v[7]);
	*reinterpret_cast<uint4*>(buf + core_offset(r, k0, kTile)) = q;
}

// ---- the fused forward kernel

__global__ void __launch_bounds__(kThreads, 2)
mlp_forward_kernel(const unsigned char* __restrict__ image, const float* __restrict__ features,
                   uint32_t n_max, const uint32_t* __restrict__ d_n, float* __restrict__ out_raw,
                   float* __restrict__ out_mix, __nv_bfloat16* __restrict__ out_acts, uint32_t* __restrict__ error)
{
	const uint32_t n = d_n ? min(*d_n, n_max) : n_max;
	extern __shared__ __align__(128) unsigned char smem[];
	const uint32_t tid = threadIdx.x;
	const uint32_t warp = tid >> 5;
	const uint32_t r = tid & (kTile - 1);   // the tile row this thread works on
	const uint32_t part = tid / kTile;      // which half of the row's columns / lobes

	// weights + biases into shared memory
	{
		const uint4* src = reinterpret_cast<const uint4*>(image);
		uint4* dst = reinterpret_cast<uint4*>(smem + kOffSmemImage);
		for(uint32_t i = tid; i < kImageBytes / 16; i += kThreads)
		{
			dst[i] = __ldg(src + i);
		}
	}
	const uint32_t bar = smem_u32(smem + kOffSmemBar);
	uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(smem + kOffSmemTmem);
	if(tid == 0)
	{
		mbar_init(bar, 1);
		asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
	}
	if(warp == 0)
	{
		asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
		             :: "r"(smem_u32(tmem_slot)), "r"(kTmemCols) : "memory");
		asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
	}
	fence_before_sync();
	__syncthreads();
	fence_after_sync();
	const uint32_t tmem = *tmem_slot;
	const uint32_t tmem_row = tmem + (((warp & 3u) * 32u) << 16);   // this warp's 32 lanes, column 0

	const float* bias = reinterpret_cast<const float*>(smem + kOffImgBias);
	unsigned char* act_in = smem + kOffSmemActIn;
	unsigned char* act_h = smem + kOffSmemActH;
	float2* xch = reinterpret_cast<float2*>(smem + kOffSmemXch);
	const uint32_t w_addr[5] = {smem_u32(smem + kOffImgW0), smem_u32(smem + kOffImgW1), smem_u32(smem + kOffImgW2),
	                            smem_u32(smem + kOffImgW3), smem_u32(smem + kOffImgW4)};

	uint32_t phase = 0;
	bool failed = false;
	const uint32_t num_tiles = (n + kTile - 1) / kTile;
	for(uint32_t tile = blockIdx.x; tile < num_tiles && !failed; tile += gridDim.x)
	{
		const uint32_t row = tile * kTile + r;
		const bool valid = row < n;

		float f[kInputs];
		#pragma unroll
		for(int i = 0; i < kInputs; ++i)
		{
			f[i] = valid ? __ldg(features + static_cast<size_t>(row) * 8 + i) : -1.0f;
		}

		// One MMA chain (k_steps x K = 16) from A buffer a_buf against weights w_base starting at
		// global K-step ks0, committed to the mbarrier; every thread then waits for it.
		auto run_mma = [&](const unsigned char* a_buf, uint32_t k_steps, uint32_t w_base, uint32_t n_dim,
		                   uint32_t ks0, bool accumulate) -> bool
		{
			if(tid == 0)
			{
				fence_after_sync();
				const uint32_t a_base = smem_u32(a_buf);
				const uint32_t idesc = instr_desc(kTile, n_dim);
				for(uint32_t ks = 0; ks < k_steps; ++ks)
				{
					const uint64_t ad = smem_desc(a_base + ks * 2u * (kTile * 16u), kTile * 16u, 128u);
					const uint64_t bd = smem_desc(w_base + (ks0 + ks) * 2u * (n_dim * 16u), n_dim * 16u, 128u);
					mma_bf16(tmem, ad, bd, idesc, (accumulate || ks > 0) ? 1u : 0u);
				}
				mma_commit(bar);
			}
			// one thread polls the barrier; the others wait at the block barrier, which issues no
			// instructions while the MMAs run
			const bool ok = tid == 0 ? mbar_wait(bar, phase) : true;
			if(__syncthreads_or(ok ? 0 : 1))
			{
				// the tensor cores did not report back: one more bounded wait for this phase so
				// that the accumulator is not freed under running MMAs, then give up
				if(!ok)
				{
					mbar_wait(bar, phase);
				}
				return false;
			}
			phase ^= 1u;
			fence_after_sync();
			return true;
		};

		// 1. input layer in two K halves: one-blob encode (the row's two threads take alternate
		//    inputs), then accumulate into TMEM
		bool tile_ok = true;
		for(int half = 0; half < 2 && tile_ok; ++half)
		{
			const int i0 = half == 0 ? 0 : 4, i1 = half == 0 ? 4 : kInputs;
			for(int i = i0 + static_cast<int>(part); i < i1; i += kParts)
			{
				// the input by selects, so that f stays in registers (a run-time index would put
				// it in local memory)
				float fi = f[0];
				#pragma unroll
				for(int q = 1; q < kInputs; ++q)
				{
					fi = i == q ? f[q] : fi;
				}
				// Its 32 bins g_b = exp(-z_b^2 / 2), z_b = 32 fi - (b + 1/2). Per 8-bin chunk one
				// exponential gives g at the chunk's first bin and one the ratio to the next bin,
				// g_{b+1} / g_b = exp(z_b - 1/2), which shrinks by e^-1 per bin: two multiplies per
				// further bin. Where the chunk's first bin underflows to 0, every bin of the chunk
				// is below 1e-8.
				const float s32 = fi * static_cast<float>(kBins) - 0.5f;
				#pragma unroll
				for(int c = 0; c < kBins / 8; ++c)
				{
					const float z0 = s32 - static_cast<float>(c * 8);
					float g = __expf(-0.5f * z0 * z0);
					float ratio = __expf(z0 - 0.5f);
					float v[8];
					#pragma unroll
					for(int j = 0; j < 8; ++j)
					{
						v[j] = valid ? g : 0.0f;
						g *= ratio;
						ratio *= 0.36787944117144233f;   // e^-1
					}
					store_row8(act_in, r, static_cast<uint32_t>((i - i0) * kBins + c * 8), v);
				}
			}
			fence_async_smem();
			fence_before_sync();
			__syncthreads();
			const uint32_t k_steps = (half == 0 ? kInHalf0 : kInHalf1) / 16;
			tile_ok = run_mma(act_in, k_steps, w_addr[0], kHidden, half == 0 ? 0u : kInHalf0 / 16, half == 1);
		}
		if(!tile_ok)
		{
			failed = true;
			break;
		}

		// 2./3. H1 (act_h) -> H2 (act_in) -> H3 (act_h) -> H4 (act_in) -> out
		#pragma unroll 1
		for(int layer = 0; layer < 5; ++layer)
		{
			const bool last = layer == 4;
			const uint32_t n_dim = last ? kOutPad : kHidden;
			unsigned char* o_buf = (layer & 1) ? act_in : act_h;
			if(layer > 0)
			{
				const unsigned char* a_buf = (layer & 1) ? act_h : act_in;
				if(!run_mma(a_buf, kHidden / 16, w_addr[layer], n_dim, 0u, false))
				{
					failed = true;
					break;
				}
			}

			if(!last)
			{
				// hidden units [32 part, 32 part + 32) of the row
				const uint32_t c0 = part * 32u;
				float acc[32];
				tmem_ld16(tmem_row + c0, acc);
				tmem_ld16(tmem_row + c0 + 16u, acc + 16);
				tmem_wait_ld();
				const float* b = bias + layer * kHidden + c0;
				#pragma unroll
				for(int j = 0; j < 32; ++j)
				{
					acc[j] = fmaxf(acc[j] + b[j], 0.0f);
				}
				#pragma unroll
				for(int c = 0; c < 4; ++c)
				{
					store_row8(o_buf, r, c0 + c * 8, acc + c * 8);
				}
				if(out_acts && valid)
				{
					uint4* dst = reinterpret_cast<uint4*>(out_acts + (static_cast<size_t>(row) * kHiddenLayers + layer) * kHidden + c0);
					#pragma unroll
					for(int c = 0; c < 4; ++c)
					{
						dst[c] = make_uint4(pack_bf16x2(acc[c * 8 + 0], acc[c * 8 + 1]), pack_bf16x2(acc[c * 8 + 2], acc[c * 8 + 3]),
						                    pack_bf16x2(acc[c * 8 + 4], acc[c * 8 + 5]), pack_bf16x2(acc[c * 8 + 6], acc[c * 8 + 7]));
					}
				}
			}
			else
			{
				// lobes [4 part, 4 part + 4): raw outputs [20 part, 20 part + 20), inside the
				// loaded accumulator columns [16 part, 16 part + 32)
				float acc[32];
				tmem_ld16(tmem_row + part * 16u, acc);
				tmem_ld16(tmem_row + part * 16u + 16u, acc + 16);
				tmem_wait_ld();
				const float* b = bias + kHiddenLayers * kHidden + part * 20u;
				float raw[20];
				#pragma unroll
				for(int q = 0; q < 20; ++q)
				{
					raw[q] = (part ? acc[q + 4] : acc[q]) + b[q];
				}
				if(out_raw && valid)
				{
					float4* dst = reinterpret_cast<float4*>(out_raw + static_cast<size_t>(row) * kOut + part * 20u);
					#pragma unroll
					for(int c = 0; c < 5; ++c)
					{
						dst[c] = make_float4(raw[4 * c + 0], raw[4 * c + 1], raw[4 * c + 2], raw[4 * c + 3]);
					}
				}
				if(out_mix)   // a kernel argument: the same for every thread, so the barriers are safe
				{
					// the mixture of decode(): softmax weights over all 8 lobes, unit means, clamped
					// concentrations, and each lobe's weight x vMF normalisation
					float mx = raw[0];
					#pragma unroll
					for(int j = 1; j < 4; ++j)
					{
						mx = fmaxf(mx, raw[5 * j]);
					}
					xch[part * kTile + r].x = mx;
					__syncthreads();
					mx = fmaxf(xch[r].x, xch[kTile + r].x);
					float e[4], sum = 0.0f;
					#pragma unroll
					for(int j = 0; j < 4; ++j)
					{
						e[j] = expf(raw[5 * j] - mx);
						sum += e[j];
					}
					xch[part * kTile + r].y = sum;
					__syncthreads();
					sum = xch[r].y + xch[kTile + r].y;
					if(valid)
					{
						float2* dst = reinterpret_cast<float2*>(out_mix + static_cast<size_t>(row) * kMixFloats) + 12u * part;
						#pragma unroll
						for(int j = 0; j < 4; ++j)
						{
							const float w = e[j] / sum;
							V3 d = v3(raw[5 * j + 1], raw[5 * j + 2], raw[5 * j + 3]);
							const float l2 = dot(d, d);
							const V3 mu = l2 > 1e-20f ? d * (1.0f / sqrtf(l2)) : v3(0.0f, 0.0f, 1.0f);
							const float k = fminf(fmaxf(expf(raw[5 * j + 4]), kMinKappa), kMaxKappa);
							const float c = w * k / (2.0f * kPi * (1.0f - expf(-2.0f * k)));
							dst[3 * j + 0] = make_float2(w, mu.x);
							dst[3 * j + 1] = make_float2(mu.y, mu.z);
							dst[3 * j + 2] = make_float2(k, c);
						}
					}
				}
			}
			fence_async_smem();
			fence_before_sync();
			__syncthreads();
			fence_after_sync();
		}
	}

	if(failed && tid == 0)
	{
		atomicOr(error, PG_DEV_ERR_GUIDE_WAIT);
	}
	fence_before_sync();
	__syncthreads();
	if(warp == 0)
	{
		asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(tmem), "r"(kTmemCols) : "memory");
	}
}

// FP32 parameters -> BF16 shared-memory image (W^T in the K-major core-matrix layout) + biases.
__global__ void pack_image_kernel(const float* __restrict__ params, unsigned char* __restrict__ image)
{
	const uint32_t total = kHidden * kIn + 3 * kHidden * kHidden + kOutPad * kHidden + kBiasCount;
	for(uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x)
	{
		uint32_t j = i;
		if(j < kHidden * kIn)
		{
			const uint32_t o = j / kIn, k = j % kIn;   // W0^T[o][k] = W0[k][o]
			*reinterpret_cast<__nv_bfloat16*>(image + kOffImgW0 + core_offset(o, k, kHidden)) =
				__float2bfloat16_rn(params[kOffW0 + k * kHidden + o]);
			continue;
		}
		j -= kHidden * kIn;
		if(j < 3u * kHidden * kHidden)
		{
			const uint32_t l = j / (kHidden * kHidden), e = j % (kHidden * kHidden);
			const uint32_t o = e / kHidden, k = e % kHidden;
			const int src = (l == 0 ? kOffW1 : (l == 1 ? kOffW2 : kOffW3)) + k * kHidden + o;
			*reinterpret_cast<__nv_bfloat16*>(image + kOffImgW1 + l * kWhBytes + core_offset(o, k, kHidden)) =
				__float2bfloat16_rn(params[src]);
			continue;
		}
		j -= 3u * kHidden * kHidden;
		if(j < static_cast<uint32_t>(kOutPad * kHidden))
		{
			const uint32_t o = j / kHidden, k = j % kHidden;
			const float w = o < static_cast<uint32_t>(kOut) ? params[kOffW4 + k * kOut + o] : 0.0f;
			*reinterpret_cast<__nv_bfloat16*>(image + kOffImgW4 + core_offset(o, k, kOutPad)) = __float2bfloat16_rn(w);
			continue;
		}
		j -= kOutPad * kHidden;
		float b = 0.0f;
		if(j < static_cast<uint32_t>(kHiddenLayers * kHidden))
		{
			const uint32_t l = j / kHidden, o = j % kHidden;
			const int off[4] = {kOffB0, kOffB1, kOffB2, kOffB3};
			b = params[off[l] + o];
		}
		else if(j - kHiddenLayers * kHidden < static_cast<uint32_t>(kOut))
		{
			b = params[kOffB4 + (j - kHiddenLayers * kHidden)];
		}
		reinterpret_cast<float*>(image + kOffImgBias)[j] = b;
	}
}

}// end anonymous namespace

int image_bytes() { return kImageBytes; }

void pack_image(const float* d_params, unsigned char* d_image, cudaStream_t s)
{
	pack_image_kernel<<<64, 256, 0, s>>>(d_params, d_image);
	PG_CUDA_CHECK(cudaGetLastError());
}

void launch_forward(const unsigned char* d_image, const float* d_features, uint32_t n, float* d_out_raw,
                    __nv_bfloat16* d_out_acts, uint32_t* d_error, cudaStream_t s, const uint32_t* d_n,
                    float* d_out_mix)
{
	if(n == 0)
	{
		return;
	}
	static const bool configured = []
	{
		PG_CUDA_CHECK(cudaFuncSetAttribute(mlp_forward_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes));
		return true;
	}();
	(void)configured;
	const uint32_t tiles = (n + kTile - 1) / kTile;
	const uint32_t grid = std::min<uint32_t>(tiles, 2u * static_cast<uint32_t>(sm_count()));
	mlp_forward_kernel<<<grid, kThreads, kSmemBytes, s>>>(d_image, d_features, n, d_n, d_out_raw, d_out_mix,
	                                                     d_out_acts, d_error);
	PG_CUDA_CHECK(cudaGetLastError());
}

}// end namespace guide
}// end namespace pg

using namespace pg;

namespace
{

// Host entry of the forward pass: copies the parameters and queries in, runs the tensor-core
// kernel, and copies back the raw outputs [n][40] and / or the decoded mixtures [n][48].
void forward_on_host(const char* what, const float* params, const float* features, uint64_t n, float* out_raw,
                     float* out_mix)
{
	if(!params || (n > 0 && (!features || (!out_raw && !out_mix))))
	{
		throw Error(PG_ERR_INVALID_ARGUMENT, std::string(what) + ": null pointer");
	}
	if(n > (1u << 30))
	{
		throw Error(PG_ERR_INVALID_ARGUMENT, std::string(what) + ": too many queries");
	}
	require_device();
	if(n == 0)
	{
		return;
	}
	cudaStream_t s = library_stream();
	DeviceBuffer<float> d_params(guide::kNumParams);
	DeviceBuffer<unsigned char> d_image(guide::image_bytes());
	DeviceBuffer<float> d_feat(n * 8);
	DeviceBuffer<float> d_raw(out_raw ? n * guide::kOut : 0);
	DeviceBuffer<float> d_mix(out_mix ? n * guide::kMixFloats : 0);
	DeviceBuffer<uint32_t> d_err(1);
	PG_CUDA_CHECK(cudaMemsetAsync(d_err.get(), 0, sizeof(uint32_t), s));
	PG_CUDA_CHECK(cudaMemcpyAsync(d_params.get(), params, d_params.bytes(), cudaMemcpyHostToDevice, s));
	// features: host [n][7] -> device [n][8]
	std::vector<float> feat(n * 8, 0.0f);
	for(uint64_t i = 0; i < n; ++i)
	{
		std::memcpy(&feat[i * 8], features + i * guide::kInputs, sizeof(float) * guide::kInputs);
	}
	PG_CUDA_CHECK(cudaMemcpyAsync(d_feat.get(), feat.data(), d_feat.bytes(), cudaMemcpyHostToDevice, s));
	guide::pack_image(d_params.get(), d_image.get(), s);
	guide::launch_forward(d_image.get(), d_feat.get(), static_cast<uint32_t>(n), out_raw ? d_raw.get() : nullptr,
	                      nullptr, d_err.get(), s, nullptr, out_mix ? d_mix.get() : nullptr);
	uint32_t err = 0;
	if(out_raw)
	{
		PG_CUDA_CHECK(cudaMemcpyAsync(out_raw, d_raw.get(), d_raw.bytes(), cudaMemcpyDeviceToHost, s));
	}
	if(out_mix)
	{
		PG_CUDA_CHECK(cudaMemcpyAsync(out_mix, d_mix.get(), d_mix.bytes(), cudaMemcpyDeviceToHost, s));
	}
	PG_CUDA_CHECK(cudaMemcpyAsync(&err, d_err.get(), sizeof(err), cudaMemcpyDeviceToHost, s));
	PG_CUDA_CHECK(cudaStreamSynchronize(s));
	if(err)
	{
		throw Error(PG_ERR_CUDA, "guiding network: tensor-core wait timed out");
	}
}

}// end anonymous namespace

extern "C" {

int pgpu_guide_forward(const float* params, const float* features, uint64_t n, float* out_raw)
{
	return guarded([&]
	{
		if(n > 0 && !out_raw)
		{
			throw Error(PG_ERR_INVALID_ARGUMENT, "pgpu_guide_forward: null pointer");
		}
		forward_on_host("pgpu_guide_forward", params, features, n, out_raw, nullptr);
	});
}

int pgpu_guide_mixture(const float* params, const float* features, uint64_t n, float* out_mix)
{
	return guarded([&]
	{
		if(n > 0 && !out_mix)
		{
			throw Error(PG_ERR_INVALID_ARGUMENT, "pgpu_guide_mixture: null pointer");
		}
		forward_on_host("pgpu_guide_mixture", params, features, n, nullptr, out_mix);
	});
}

}// extern "C"
