// Film test entry point of the C ABI: splats given samples through the device filter and
// deposit functions the renderer uses (film.cuh), so that the reference's film known answers
// can be checked without a render around them.
#include "film.cuh"
#include "pg_runtime.h"

#include "../../include/photon_gpu.h"

#include <string>

namespace pg
{
namespace
{

constexpr int kSampleFloats = 5;   // raster x, raster y, r, g, b

__global__ void film_splat_kernel(const FilmView f, const float* __restrict__ samples, uint64_t n)
{
	const uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
	if(i >= n)
	{
		return;
	}
	const float* s = samples + kSampleFloats * i;
	film_deposit(f, s[0], s[1], make_float4(s[2], s[3], s[4], 1.0f));
}

}// end anonymous namespace
}// end namespace pg

using namespace pg;

extern "C" int pgpu_film_splat(uint32_t filter, uint32_t width, uint32_t height, const float* samples,
                               uint64_t n, double* out_sums)
{
	return guarded([&]
	{
		if(filter != PG_FILTER_GAUSSIAN && filter != PG_FILTER_MITCHELL_NETRAVALI && filter != PG_FILTER_BLACKMAN_HARRIS)
		{
			throw Error(PG_ERR_INVALID_ARGUMENT, "pgpu_film_splat: filter " + std::to_string(filter) +
				" is not one of the 4 x 4 filters (1 gaussian, 2 mitchell-netravali, 3 blackman-harris)");
		}
		if(width == 0 || height == 0 || static_cast<uint64_t>(width) * height > (1ull << 24))
		{
			throw Error(PG_ERR_INVALID_ARGUMENT, "pgpu_film_splat: the film must have 1 to 2^24 pixels");
		}
		if(n > (1ull << 26))
		{
			throw Error(PG_ERR_INVALID_ARGUMENT, "pgpu_film_splat: more than 2^26 samples");
		}
		if((!samples && n > 0) || !out_sums)
		{
			throw Error(PG_ERR_INVALID_ARGUMENT, "pgpu_film_splat: null pointer");
		}
		require_device();
		cudaStream_t s = library_stream();
		DeviceBuffer<double> d_sums(static_cast<std::size_t>(width) * height * kFilmChannels);
		PG_CUDA_CHECK(cudaMemsetAsync(d_sums.get(), 0, d_sums.bytes(), s));
		if(n > 0)
		{
			DeviceBuffer<float> d_samples(n * kSampleFloats);
			PG_CUDA_CHECK(cudaMemcpyAsync(d_samples.get(), samples, d_samples.bytes(), cudaMemcpyHostToDevice, s));
			const FilmView f = make_film_view(d_sums.get(), width, height, filter);
			film_splat_kernel<<<static_cast<unsigned>((n + 127) / 128), 128, 0, s>>>(f, d_samples.get(), n);
			PG_CUDA_CHECK(cudaGetLastError());
			PG_CUDA_CHECK(cudaStreamSynchronize(s));
		}
		PG_CUDA_CHECK(cudaMemcpyAsync(out_sums, d_sums.get(), d_sums.bytes(), cudaMemcpyDeviceToHost, s));
		PG_CUDA_CHECK(cudaStreamSynchronize(s));
	});
}
