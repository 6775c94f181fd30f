// Image (lat-long) environment: the dome of actor(image-dome) with a PFM of any size.
//
// Lookup (LatLongEnvEmitter::evalEmittedEnergy, LatLongEnvEmitter.cpp:83-91): the radiance of a
// direction is the dome image at the direction's lat-long coordinates (PLatLongEnvSphere's hit UV,
// PLatLongEnvSphere.cpp:60-110, TSphere::surfaceToLatLong01, Math/Geometry/TSphere.ipp:393-437):
//   phi = atan2(x, z) in [0, 2 pi), theta = acos(y);  u = phi / 2 pi,  v = (pi - theta) / pi
// in the dome's local frame (its actor rotation). The image is sampled bilinearly with texel
// centres at ((i + 0.5) / W, (j + 0.5) / H) and edges clamped (AImageDome.cpp:10-17,
// TPixelTexture2D::samplePixelBufferBilinear, Core/Texture/Pixel/TPixelTexture2D.ipp:127-172; its
// "flipped" wrap of u is applied twice, to the sample point and again to the texel corners, and
// cancels). Row j = 0 of the image is its bottom row (v small, looking down).
//
// Sampling (LatLongEnvEmitter.cpp:36-81, 93-150): texel (i, j) is chosen with probability
// proportional to max(luminance, 1e-6) * sin(theta_j), theta_j = (1 - (j + 0.5) / H) pi, then a
// uniform point (u, v) inside it, whose direction w is followed from the shading point x. The
// reference picks the texel by inverting a 2D piecewise-constant CDF (TPwcDistribution2D); an
// alias table over all texels picks from the same distribution. A constant environment is a
// 1 x 1 image.
//
// Densities. The reference's dome is a sphere of radius r around the scene (1.01 x the farthest
// scene-bound corner from the dome centre c, ADome.cpp:42-60). It converts the uv density to an
// area density on that sphere, pdf_uv / (2 pi^2 r^2 sin theta) (PLatLongEnvSphere.cpp:165-186),
// and then to solid angle at x with the squared distance d to the sphere along w and a cosine
// (lta::pdfA_to_pdfW). For NEE that cosine is taken at the point where the sampled observation
// ray of length r ends, projected onto the sphere, q = c + r (x + r w - c) / |x + r w - c|, and
// the shadow ray aims at q (PLatLongEnvSphere.cpp:125-160, TDirectLightEstimator.ipp:71-98);
// for a BSDF-sampled ray that leaves the scene it is taken at the ray's own hit p = x + d w
// (LatLongEnvEmitter::calcDirectPdf). Both coincide with the true solid-angle density
// pdf_uv / (2 pi^2 sin theta) only at the dome centre. By default the estimates below use the
// reference's densities, so that they converge to what the reference computes (which is biased
// away from the centre: a grey Lambertian sphere of albedo 0.5 under a unit dome renders 0.512 in
// the reference); `exact` uses the true density of the sampled direction and aims the shadow ray
// along it, which is unbiased.
#pragma once

#include "bsdf.cuh"

#include <cstdint>

namespace pg
{

struct EnvMap
{
	const float4* texels = nullptr;   // [h][w]: radiance rgb, uv-space sampling density of the texel
	const float2* alias = nullptr;    // per texel: accept probability, alias texel index bits
	uint32_t width = 0, height = 0;   // 0: no environment
	float rot[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};   // dome local -> world, row-major
	float center[3] = {0, 0, 0};      // dome sphere
	float radius = 1.0f;
	uint32_t exact = 0;               // 1: true densities instead of the reference's
};

#ifdef __CUDACC__

constexpr float kEnvPi = 3.14159265358979323846f;

// Lat-long coordinates of a world direction.
__device__ __forceinline__ float2 env_uv(const EnvMap& m, V3 d)
{
	// local = R^T d
	const float lx = m.rot[0] * d.x + m.rot[3] * d.y + m.rot[6] * d.z;
	const float ly = m.rot[1] * d.x + m.rot[4] * d.y + m.rot[7] * d.z;
	const float lz = m.rot[2] * d.x + m.rot[5] * d.y + m.rot[8] * d.z;
	const float len = sqrtf(lx * lx + ly * ly + lz * lz);
	const float cos_theta = fminf(fmaxf(len > 0.0f ? ly / len : 1.0f, -1.0f), 1.0f);
	const float theta = acosf(cos_theta);
	float phi = atan2f(lx, lz);
	if(phi < 0.0f)
	{
		phi += 2.0f * kEnvPi;
	}
	return make_float2(phi * (1.0f / (2.0f * kEnvPi)), (kEnvPi - theta) * (1.0f / kEnvPi));
}

__device__ __forceinline__ RGB env_texel(const EnvMap& m, int i, int j)
{
	const float4 t = __ldg(m.texels + static_cast<size_t>(j) * m.width + i);
	return RGB{t.x, t.y, t.z};
}

// Bilinear, clamped to the edges.
__device__ __forceinline__ RGB env_lookup(const EnvMap& m, float2 uv)
{
	const int w = static_cast<int>(m.width), h = static_cast<int>(m.height);
	const float x = fminf(fmaxf(uv.x, 0.0f), 1.0f) * static_cast<float>(w) - 0.5f;
	const float y = fminf(fmaxf(uv.y, 0.0f), 1.0f) * static_cast<float>(h) - 0.5f;
	const float fx0 = floorf(x), fy0 = floorf(y);
	const float ax = x - fx0, ay = y - fy0;
	const int i0 = min(max(static_cast<int>(fx0), 0), w - 1), i1 = min(max(static_cast<int>(fx0) + 1, 0), w - 1);
	const int j0 = min(max(static_cast<int>(fy0), 0), h - 1), j1 = min(max(static_cast<int>(fy0) + 1, 0), h - 1);
	const RGB c00 = env_texel(m, i0, j0), c01 = env_texel(m, i0, j1);
	const RGB c10 = env_texel(m, i1, j0), c11 = env_texel(m, i1, j1);
	return c00 * ((1.0f - ax) * (1.0f - ay)) + c01 * ((1.0f - ax) * ay) + c10 * (ax * (1.0f - ay)) + c11 * (ax * ay);
}

// Distance from x (inside the dome) along unit w to the dome sphere.
__device__ __forceinline__ float env_distance(const EnvMap& m, V3 x, V3 w)
{
	const V3 o = x - v3(m.center[0], m.center[1], m.center[2]);
	const float b = dot(o, w);
	const float c = dot(o, o) - m.radius * m.radius;
	return -b + sqrtf(fmaxf(b * b - c, 0.0f));
}

// uv-space density of the texel containing uv.
__device__ __forceinline__ float env_pdf_uv(const EnvMap& m, float2 uv)
{
	const int i = min(max(static_cast<int>(uv.x * static_cast<float>(m.width)), 0), static_cast<int>(m.width) - 1);
	const int j = min(max(static_cast<int>(uv.y * static_cast<float>(m.height)), 0), static_cast<int>(m.height) - 1);
	return __ldg(m.texels + static_cast<size_t>(j) * m.width + i).w;
}

// The reference's density for a BSDF-sampled ray from x along w that reaches the dome.
__device__ __forceinline__ float env_pdf_hit(const EnvMap& m, V3 x, V3 w)
{
	const float2 uv = env_uv(m, w);
	const float sin_theta = sinf(kEnvPi * (1.0f - uv.y));
	float pdf = env_pdf_uv(m, uv) / (2.0f * kEnvPi * kEnvPi * sin_theta);
	if(!m.exact)
	{
		const float d = env_distance(m, x, w);
		const V3 p = x + w * d;
		const float cos_p = fabsf(dot(w, p - v3(m.center[0], m.center[1], m.center[2]))) / m.radius;
		pdf = pdf * (d * d) / (m.radius * m.radius * cos_p);
	}
	return isfinite(pdf) && pdf > 0.0f ? pdf : 0.0f;
}

// A direction w from the image's distribution for NEE at x, with the reference's density, the
// radiance, and the direction of the shadow ray (towards q); false where the density is not finite.
__device__ __forceinline__ bool env_sample(const EnvMap& m, V3 x, float u_texel, float u_x, float u_y,
                                           V3* out_dir, float* out_pdf_w, RGB* out_radiance, V3* out_shadow_dir)
{
	const uint32_t n = m.width * m.height;
	const float scaled = u_texel * static_cast<float>(n);
	const uint32_t k0 = min(static_cast<uint32_t>(scaled), n - 1u);
	const float2 a = __ldg(m.alias + k0);
	const uint32_t k = (scaled - static_cast<float>(k0)) < a.x ? k0 : __float_as_uint(a.y);
	const uint32_t ti = k % m.width, tj = k / m.width;
	const float2 uv = make_float2((static_cast<float>(ti) + u_x) / static_cast<float>(m.width),
	                              (static_cast<float>(tj) + u_y) / static_cast<float>(m.height));
	const float theta = (1.0f - uv.y) * kEnvPi, phi = uv.x * (2.0f * kEnvPi);
	float st, ct, sp, cp;
	sincosf(theta, &st, &ct);
	sincosf(phi, &sp, &cp);
	const float lx = st * sp, ly = ct, lz = st * cp;
	const V3 w = v3(m.rot[0] * lx + m.rot[1] * ly + m.rot[2] * lz,
	                m.rot[3] * lx + m.rot[4] * ly + m.rot[5] * lz,
	                m.rot[6] * lx + m.rot[7] * ly + m.rot[8] * lz);
	float pdf = __ldg(m.texels + k).w / (2.0f * kEnvPi * kEnvPi * st);
	V3 shadow_dir = w;
	if(!m.exact)
	{
		const V3 c = v3(m.center[0], m.center[1], m.center[2]);
		const float d = env_distance(m, x, w);
		const V3 u = normalize(x + w * m.radius - c);   // direction of q from the dome centre
		pdf = pdf * (d * d) / (m.radius * m.radius * fabsf(dot(w, u)));
		shadow_dir = c + u * m.radius - x;
	}
	if(!(st > 0.0f) || !isfinite(pdf) || !(pdf > 0.0f))
	{
		return false;
	}
	*out_dir = w;
	*out_pdf_w = pdf;
	*out_radiance = env_lookup(m, uv);
	*out_shadow_dir = shadow_dir;
	return true;
}

#endif

}// end namespace pg
