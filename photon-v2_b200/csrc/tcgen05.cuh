// Thin wrappers over the sm_100a tensor-core instructions the guiding network kernels use:
// tcgen05.mma (kind::f16, BF16 operands in shared memory, FP32 accumulator in tensor memory),
// tcgen05.ld, mbarrier completion tracking, and the no-swizzle K-major operand layout.
//
// Operand layout: K-major, no swizzle. A core matrix is 8 rows x 16 bytes (8 BF16 along K); for a
// matrix of R rows, element (r, k) lives at
//   (k / 8) * LBO + (r / 8) * 128 + (r % 8) * 16 + (k % 8) * 2,
// with LBO (the byte distance between K-adjacent core matrices) R * 16 in the dense layout; the
// descriptor's stride byte offset (between 8-row groups) is 128.
#pragma once

#include "pg_common.cuh"

#include <cuda_bf16.h>

namespace pg
{
namespace tc
{

constexpr uint32_t kWaitLimit = 1u << 22;   // bounded mbarrier wait: error flag instead of a hang

PG_HD uint32_t core_offset(uint32_t r, uint32_t k, uint32_t rows)
{
	return (k >> 3) * (rows * 16u) + (r >> 3) * 128u + (r & 7u) * 16u + (k & 7u) * 2u;
}

// The same layout with an explicit LBO (bytes between K-adjacent core matrices).
PG_HD uint32_t core_offset_lbo(uint32_t r, uint32_t k, uint32_t lbo)
{
	return (k >> 3) * lbo + (r >> 3) * 128u + (r & 7u) * 16u + (k & 7u) * 2u;
}

// ---- PTX wrappers (tcgen05 / mbarrier), sm_100a

__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
	return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
	uint64_t d = 0;
	d |= static_cast<uint64_t>((saddr >> 4) & 0x3FFFu);
	d |= static_cast<uint64_t>((lbo >> 4) & 0x3FFFu) << 16;
	d |= static_cast<uint64_t>((sbo >> 4) & 0x3FFFu) << 32;
	d |= static_cast<uint64_t>(1u) << 46;   // descriptor version 1 (sm_100); no swizzle, base offset 0
	return d;
}

// kind::f16 instruction descriptor: BF16 A and B (K-major), FP32 D, shape M x N.
constexpr uint32_t instr_desc(uint32_t m, uint32_t n)
{
	return (1u << 4) | (1u << 7) | (1u << 10) | ((n >> 3) << 17) | ((m >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t accumulate)
{
	asm volatile(
		"{\n\t.reg .pred p;\n\t"
		"setp.ne.b32 p, %4, 0;\n\t"
		"tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
		:
		: "r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate),
		  "r"(0u), "r"(0u), "r"(0u), "r"(0u)
		: "memory");
}

__device__ __forceinline__ void mma_commit(uint32_t bar)
{
	asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" :: "r"(bar) : "memory");
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count)
{
	asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity)
{
	for(uint32_t i = 0; i < kWaitLimit; ++i)
	{
		uint32_t done;
		asm volatile(
			"{\n\t.reg .pred P;\n\t"
			"mbarrier.try_wait.parity.shared::cta.b64 P, [%1], %2;\n\t"
			"selp.u32 %0, 1, 0, P;\n\t}\n"
			: "=r"(done) : "r"(bar), "r"(parity) : "memory");
		if(done)
		{
			return true;
		}
	}
	return false;
}

__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v)
{
	uint32_t r[16];
	asm volatile(
		"tcgen05.ld.sync.aligned.32x32b.x16.b32 "
		"{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
		: "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
		  "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
		: "r"(taddr));
	#pragma unroll
	for(int i = 0; i < 16; ++i)
	{
		v[i] = __uint_as_float(r[i]);
	}
}

__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

__device__ __forceinline__ uint32_t pack_bf16x2(float a, float b)
{
	const __nv_bfloat16 lo = __float2bfloat16_rn(a);
	const __nv_bfloat16 hi = __float2bfloat16_rn(b);
	return static_cast<uint32_t>(__bfloat16_as_ushort(lo)) | (static_cast<uint32_t>(__bfloat16_as_ushort(hi)) << 16);
}


}// end namespace tc
}// end namespace pg
