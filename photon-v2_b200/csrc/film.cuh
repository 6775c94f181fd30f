// The FP64 film and its sample filters.
//
// The film holds, per pixel, the reference's RadianceSensor (R, G, B, W) sums
// (Engine/Source/Core/Receiver/RadianceSensor.h:13-16); developing divides RGB by W
// (HdrRgbFilm::developRegion, Engine/Source/Core/Filmic/HdrRgbFilm.cpp:167-205).
//
// A sample at raster position (rx, ry) adds f(px + 0.5 - rx, py + 0.5 - ry) times its radiance to
// every pixel whose centre lies within the filter's half size, and the same weight to W
// (HdrRgbFilm::addRgbSample, HdrRgbFilm.cpp:82-123). With the 4 x 4 filters the renderer first
// collects every path's radiance in a per-path buffer (the shading kernel stores it when the path
// ends, the traversal kernel adds the NEE light found at its last vertex), and one pass in path
// order then splats all samples: consecutive paths are neighbouring pixels, so a warp's atomics
// land in a few adjacent cache lines instead of all over the film. Samples are spread over the film's sample
// window, the pixel-centre rectangle grown by the half size on every side, so that border pixels
// see the whole filter support (TSamplingFilm::updateSampleDimensions with soft edges,
// Engine/Source/Core/Filmic/TSamplingFilm.ipp:102-119). Here the window is cut into W x H equal
// cells and each pixel index owns one cell, which keeps the per-pixel stratification of the box
// filter (whose window is exactly the pixel grid) and the uniform sample density the reference
// has.
//
// Filters (SampleFilter.cpp:12-61; sizes in pixels):
//   box                 1 x 1, weight 1
//   gaussian            4 x 4, exp(-(x^2 + y^2) / (2 * 0.5^2)) minus its value at (2, 2), clamped at 0
//   mitchell-netravali  4 x 4, separable cubic with B = C = 1/3 (Mitchell and Netravali 1988)
//   blackman-harris     4 x 4, separable 4-term window of radius 2 with the last coefficient
//                       0.01174 so that it reaches 0 at the edge (TBlackmanHarris2D.h:42-62)
// The box filter's W is not accumulated per sample: every pixel receives exactly spp samples of
// weight 1, so the render adds spp to each pixel's W once per call.
#pragma once

#include <cstdint>

namespace pg
{

enum SampleFilterType : uint32_t
{
	PG_FILTER_BOX = 0,
	PG_FILTER_GAUSSIAN = 1,
	PG_FILTER_MITCHELL_NETRAVALI = 2,
	PG_FILTER_BLACKMAN_HARRIS = 3,
};

constexpr uint32_t kFilmChannels = 4;   // R, G, B, W

struct FilmView
{
	double*  sums = nullptr;   // [height][width][4]
	uint32_t width = 0, height = 0;
	uint32_t filter = PG_FILTER_BOX;
	float    half = 0.5f;      // filter half size (pixels)
	float    x0 = 0.0f, y0 = 0.0f;   // sample window corner
	float    sx = 1.0f, sy = 1.0f;   // sample window cell size (window extent / resolution)
	float4*  samples = nullptr;      // 4 x 4 filters: radiance of every path of the pass (by path index)
};

inline FilmView make_film_view(double* sums, uint32_t width, uint32_t height, uint32_t filter)
{
	FilmView f;
	f.sums = sums;
	f.width = width;
	f.height = height;
	f.filter = filter;
	f.half = filter == PG_FILTER_BOX ? 0.5f : 2.0f;
	// window [0.5 - half, size - 0.5 + half) over size cells; exactly [0, size) with cells of 1
	// for the box filter
	f.x0 = 0.5f - f.half;
	f.y0 = 0.5f - f.half;
	f.sx = static_cast<float>((static_cast<double>(width) - 1.0 + 2.0 * f.half) / width);
	f.sy = static_cast<float>((static_cast<double>(height) - 1.0 + 2.0 * f.half) / height);
	return f;
}

#ifdef __CUDACC__

// One axis of the separable filters (the Gaussian's axis factor; its edge value is removed from
// the product). Written with explicitly rounded operations so that every translation unit, with
// or without FMA contraction, computes the same weights for a sample: W and RGB must see equal
// weights.
__device__ __forceinline__ float filter_axis(uint32_t filter, float x)
{
	if(filter == PG_FILTER_GAUSSIAN)
	{
		return expf(__fmul_rn(-2.0f, __fmul_rn(x, x)));
	}
	if(filter == PG_FILTER_MITCHELL_NETRAVALI)
	{
		// B = C = 1/3: (7|x|^3 - 12|x|^2 + 16/3) / 6 and (-7/3|x|^3 + 12|x|^2 - 20|x| + 32/3) / 6
		constexpr float b = 1.0f / 3.0f, c = 1.0f / 3.0f;
		constexpr float p3 = 12.0f - 9.0f * b - 6.0f * c, p2 = -18.0f + 12.0f * b + 6.0f * c, p0 = 6.0f - 2.0f * b;
		constexpr float q3 = -b - 6.0f * c, q2 = 6.0f * b + 30.0f * c, q1 = -12.0f * b - 48.0f * c,
		                q0 = 8.0f * b + 24.0f * c;
		const float a = fabsf(x);
		const float a2 = __fmul_rn(a, a), a3 = __fmul_rn(a2, a);
		if(a < 1.0f)
		{
			return __fmul_rn(__fadd_rn(__fadd_rn(__fmul_rn(p3, a3), __fmul_rn(p2, a2)), p0), 1.0f / 6.0f);
		}
		if(a < 2.0f)
		{
			return __fmul_rn(__fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(q3, a3), __fmul_rn(q2, a2)), __fmul_rn(q1, a)), q0),
			                 1.0f / 6.0f);
		}
		return 0.0f;
	}
	// Blackman-Harris, radius 2: n = (x / 2 + 1) / 2 in [0, 1]
	const float n = __fmul_rn(__fadd_rn(__fmul_rn(x, 0.5f), 1.0f), 0.5f);
	constexpr float kTwoPi = 6.28318530717958647692f;
	const float t = __fmul_rn(kTwoPi, n);
	return __fadd_rn(__fadd_rn(__fsub_rn(0.35875f, __fmul_rn(0.48829f, cosf(t))), __fmul_rn(0.14128f, cosf(__fmul_rn(2.0f, t)))),
	                 -__fmul_rn(0.01174f, cosf(__fmul_rn(3.0f, t))));
}

// exp(-2 * 2^2) twice: the Gaussian's value at the corner (2, 2) of its support
constexpr float kGaussianEdge = 1.12535174719259114e-7f;

// Adds v.xyz * f and v.w * f to (R, G, B, W) of every pixel in the filter footprint of the sample
// at (rx, ry); zero components are skipped. Not used for the box filter.
static __device__ __noinline__ void film_deposit(const FilmView f, float rx, float ry, float4 v)
{
	const float cx = __fsub_rn(rx, 0.5f), cy = __fsub_rn(ry, 0.5f);
	const int x0 = max(0, static_cast<int>(ceilf(cx - f.half)));
	const int x1 = min(static_cast<int>(f.width) - 1, static_cast<int>(floorf(cx + f.half)));
	const int y0 = max(0, static_cast<int>(ceilf(cy - f.half)));
	const int y1 = min(static_cast<int>(f.height) - 1, static_cast<int>(floorf(cy + f.half)));
	if(x0 > x1 || y0 > y1)
	{
		return;
	}
	float wx[5];
	const int nx = min(x1 - x0 + 1, 5);
	for(int i = 0; i < nx; ++i)
	{
		wx[i] = filter_axis(f.filter, __fsub_rn(static_cast<float>(x0 + i), cx));
	}
	const int ny = min(y1 - y0 + 1, 5);
	for(int j = 0; j < ny; ++j)
	{
		const float wy = filter_axis(f.filter, __fsub_rn(static_cast<float>(y0 + j), cy));
		double* row = f.sums + (static_cast<size_t>(y0 + j) * f.width + x0) * kFilmChannels;
		for(int i = 0; i < nx; ++i)
		{
			float w = __fmul_rn(wx[i], wy);
			if(f.filter == PG_FILTER_GAUSSIAN)
			{
				w = fmaxf(__fsub_rn(w, kGaussianEdge), 0.0f);
			}
			if(w == 0.0f)
			{
				continue;
			}
			double* px = row + static_cast<size_t>(i) * kFilmChannels;
			const double dw = static_cast<double>(w);
			if(v.x != 0.0f) { atomicAdd(px + 0, static_cast<double>(v.x) * dw); }
			if(v.y != 0.0f) { atomicAdd(px + 1, static_cast<double>(v.y) * dw); }
			if(v.z != 0.0f) { atomicAdd(px + 2, static_cast<double>(v.z) * dw); }
			if(v.w != 0.0f) { atomicAdd(px + 3, static_cast<double>(v.w) * dw); }
		}
	}
}

// Box filter: the sample's radiance goes to the pixel that owns it.
__device__ __forceinline__ void film_add_box(const FilmView& f, uint32_t pixel, float r, float g, float b)
{
	double* px = f.sums + static_cast<size_t>(pixel) * kFilmChannels;
	if(r != 0.0f) { atomicAdd(px + 0, static_cast<double>(r)); }
	if(g != 0.0f) { atomicAdd(px + 1, static_cast<double>(g)); }
	if(b != 0.0f) { atomicAdd(px + 2, static_cast<double>(b)); }
}

#endif

}// end namespace pg
