// BSDF test entry point of the C ABI: one case per thread through the device BSDF functions
// the path tracer uses (bsdf.cuh).
#include "bsdf.cuh"
#include "pg_runtime.h"

#include "../../include/photon_gpu.h"

namespace pg
{
namespace
{

constexpr int kCaseIn = 19;
constexpr int kCaseOut = 16;

__global__ void bsdf_cases_kernel(const float* __restrict__ cases, const float* __restrict__ normals,
                                  uint64_t n, float* __restrict__ out)
{
	const uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
	if(i >= n)
	{
		return;
	}
	const float* c = cases + kCaseIn * i;
	const float* nn = normals + 6 * i;
	Material m{};
	const int type = static_cast<int>(c[0]);
	if(type == 0)
	{
		m.type = PG_MAT_MATTE;
		m.cr = c[1]; m.cg = c[2]; m.cb = c[3];
	}
	else if(type == 1)
	{
		m.type = PG_MAT_CONDUCTOR;
		m.alpha = fmaxf(c[1] * c[1], 0.001f);
		m.cr = c[2]; m.cg = c[3]; m.cb = c[4];
	}
	else
	{
		m.type = PG_MAT_DIELECTRIC;
		m.alpha = fmaxf(c[1] * c[1], 0.001f);
		m.ior_outer = c[2];
		m.ior_inner = c[3];
	}
	const Frame f = make_frame(v3(nn[0], nn[1], nn[2]), v3(nn[3], nn[4], nn[5]));
	const V3 v = v3(c[10], c[11], c[12]);
	const V3 l = v3(c[13], c[14], c[15]);
	float* o = out + kCaseOut * i;
	for(int k = 0; k < kCaseOut; ++k)
	{
		o[k] = 0.0f;
	}
	RGB fval;
	if(bsdf_eval(m, f, l, v, &fval))
	{
		o[0] = 1.0f; o[1] = fval.r; o[2] = fval.g; o[3] = fval.b;
	}
	const float pdf = bsdf_pdf(m, f, l, v);
	if(pdf > 0.0f)
	{
		o[4] = 1.0f; o[5] = pdf;
	}
	const BsdfSample s = bsdf_sample(m, f, v, c[16], c[17], c[18]);
	if(s.ok)
	{
		o[6] = 1.0f;
		o[7] = s.l.x; o[8] = s.l.y; o[9] = s.l.z;
		o[10] = s.weight.r; o[11] = s.weight.g; o[12] = s.weight.b;
		o[13] = s.rel_ior;
		o[14] = s.cos;
	}
}

}// end anonymous namespace
}// end namespace pg

using namespace pg;

extern "C" int pgpu_bsdf_eval(const float* cases, const float* normals, uint64_t n, float* out)
{
	return guarded([&]
	{
		if(!cases || !normals || !out)
		{
			throw Error(PG_ERR_INVALID_ARGUMENT, "pgpu_bsdf_eval: null pointer");
		}
		require_device();
		if(n == 0)
		{
			return;
		}
		cudaStream_t s = library_stream();
		DeviceBuffer<float> d_cases(n * kCaseIn), d_normals(n * 6), d_out(n * kCaseOut);
		PG_CUDA_CHECK(cudaMemcpyAsync(d_cases.get(), cases, d_cases.bytes(), cudaMemcpyHostToDevice, s));
		PG_CUDA_CHECK(cudaMemcpyAsync(d_normals.get(), normals, d_normals.bytes(), cudaMemcpyHostToDevice, s));
		bsdf_cases_kernel<<<static_cast<unsigned>((n + 127) / 128), 128, 0, s>>>(
			d_cases.get(), d_normals.get(), n, d_out.get());
		PG_CUDA_CHECK(cudaGetLastError());
		PG_CUDA_CHECK(cudaMemcpyAsync(out, d_out.get(), d_out.bytes(), cudaMemcpyDeviceToHost, s));
		PG_CUDA_CHECK(cudaStreamSynchronize(s));
	});
}
