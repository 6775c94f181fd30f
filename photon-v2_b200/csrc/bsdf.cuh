// Device BSDFs of the path-tracing core: Lambertian, GGX conductor and GGX dielectric.
//
// Each function follows the reference class it replaces, including its measurability rules,
// under the Strict sidedness policy the estimators use (BNEEPTEstimator.cpp:46,
// Engine/Source/Core/SurfaceBehavior/BsdfQueryContext.h:19) and radiance transport:
//   LambertianReflector    Engine/Source/Core/SurfaceBehavior/SurfaceOptics/LambertianReflector.cpp:39-99
//   OpaqueMicrofacet       .../SurfaceOptics/OpaqueMicrofacet.cpp:59-155
//   TranslucentMicrofacet  .../SurfaceOptics/TranslucentMicrofacet.cpp:62-370
//   IsoTrowbridgeReitz     .../Property/IsoTrowbridgeReitz.cpp:20-56 (alpha floor 0.001,
//                          IsoTrowbridgeReitzConstant.h:23-29), height-correlated Smith G
//                          (ShapeInvariantMicrofacet.cpp:20-70), VNDF sampling after Dupuy
//                          (TrowbridgeReitz.cpp:19-82)
//   Schlick conductor Fresnel  .../Property/SchlickApproxConductorFresnel.cpp:35-40
//   exact dielectric Fresnel   .../Property/ExactDielectricFresnel.cpp:12-40
//   refraction direction       .../Property/DielectricFresnel.cpp:18-42
// The SurfaceOptics wrapper checks (SurfaceOptics.cpp:14-66: V and L must agree in sidedness)
// are folded into each entry point.
#pragma once

#include "pg_common.cuh"

namespace pg
{

constexpr float kPi = 3.14159265358979323846f;
constexpr float kRcpPi = 0.318309886183790671538f;
constexpr float kTwoPi = 6.28318530717958647692f;

enum MaterialType : uint32_t
{
	PG_MAT_MATTE = 0,
	PG_MAT_CONDUCTOR = 1,
	PG_MAT_DIELECTRIC = 2,
	PG_MAT_ABSORBER = 3,     // IdealAbsorber: never measurable (the surface of an area light)
};

// 32-byte material record. For matte: c = albedo. Conductor: c = F0, alpha. Dielectric:
// alpha, ior_outer, ior_inner.
struct alignas(16) Material
{
	uint32_t type;
	float    cr, cg, cb;
	float    alpha;
	float    ior_outer;
	float    ior_inner;
	float    pad;
};

struct RGB
{
	float r, g, b;
};

PG_HD RGB rgb(float r, float g, float b) { return RGB{r, g, b}; }
PG_HD RGB operator * (RGB a, RGB b) { return RGB{a.r * b.r, a.g * b.g, a.b * b.b}; }
PG_HD RGB operator * (RGB a, float s) { return RGB{a.r * s, a.g * s, a.b * s}; }
PG_HD RGB operator + (RGB a, RGB b) { return RGB{a.r + b.r, a.g + b.g, a.b + b.b}; }
PG_HD bool is_finite(RGB a) { return isfinite(a.r) && isfinite(a.g) && isfinite(a.b); }
PG_HD bool is_zero(RGB a) { return a.r == 0.0f && a.g == 0.0f && a.b == 0.0f; }
PG_HD RGB safe_clamp(RGB a, float lo, float hi)
{
	return RGB{safe_clamp(a.r, lo, hi), safe_clamp(a.g, lo, hi), safe_clamp(a.b, lo, hi)};
}

// Surface frame at a hit: geometry normal, shading normal and the shading basis built from the
// shading normal alone (HitInfo::computeBases falls back to Basis3R::makeFromUnitY when dN/dU = 0,
// Engine/Source/Core/HitInfo.h:140-170, Engine/Source/Math/TOrthonormalBasis3.ipp:16-39).
struct Frame
{
	V3 ng;
	V3 ns;
	V3 bx, bz;   // shading basis x and z axes (y axis = ns)
};

__device__ __forceinline__ Frame make_frame(V3 ng, V3 ns)
{
	Frame f;
	f.ng = ng;
	f.ns = ns;
	V3 x;
	if(fabsf(ns.y) < 0.707106781186547524f)
	{
		x = v3(-ns.z, 0.0f, ns.x);
		x = x * (1.0f / sqrtf(x.x * x.x + x.z * x.z));
	}
	else
	{
		x = v3(ns.y, -ns.x, 0.0f);
		x = x * (1.0f / sqrtf(x.x * x.x + x.y * x.y));
	}
	f.bx = x;
	f.bz = cross(x, ns);
	return f;
}

__device__ __forceinline__ V3 local_to_world(const Frame& f, V3 v)
{
	return f.bx * v.x + f.ns * v.y + f.bz * v.z;
}

__device__ __forceinline__ V3 world_to_local(const Frame& f, V3 v)
{
	return v3(dot(f.bx, v), dot(f.ns, v), dot(f.bz, v));
}

// Strict sidedness (Engine/Source/Core/LTA/SidednessAgreement.h:119-280).
__device__ __forceinline__ bool sidedness_agreed(const Frame& f, V3 v)
{
	return dot(f.ng, v) * dot(f.ns, v) > 0.0f;
}
__device__ __forceinline__ bool same_hemisphere(const Frame& f, V3 a, V3 b)
{
	return sidedness_agreed(f, a) && sidedness_agreed(f, b) && dot(a, f.ng) * dot(b, f.ng) > 0.0f;
}
__device__ __forceinline__ bool opposite_hemisphere(const Frame& f, V3 a, V3 b)
{
	return sidedness_agreed(f, a) && sidedness_agreed(f, b) && dot(a, f.ng) * dot(b, f.ng) < 0.0f;
}

// ---------------------------------------------------------------------------------------------
// GGX (isotropic Trowbridge-Reitz), height-correlated masking-shadowing.

__device__ __forceinline__ float ggx_lambda(float alpha2, V3 n, V3 d)
{
	const float nod = dot(n, d);
	const float nod2 = fminf(nod * nod, 1.0f);
	return 0.5f * (-1.0f + sqrtf(1.0f + alpha2 * (1.0f / nod2 - 1.0f)));
}

__device__ __forceinline__ float ggx_d(float alpha, V3 n, V3 h)
{
	const float noh = dot(n, h);
	const float alpha2 = alpha * alpha;
	const float noh2 = noh * noh;
	const float inner = noh2 * (alpha2 - 1.0f) + 1.0f;
	return alpha2 / (kPi * inner * inner);
}

// Microfacet::isSidednessAgreed (Microfacet.h:131-144) then height-correlated G.
__device__ __forceinline__ float ggx_g(float alpha, V3 n, V3 h, V3 l, V3 v)
{
	const float nol = dot(n, l), nov = dot(n, v), hol = dot(h, l), hov = dot(h, v);
	if(!(hol * nol > 0.0f && hov * nov > 0.0f))
	{
		return 0.0f;
	}
	const float alpha2 = alpha * alpha;
	return 1.0f / (1.0f + ggx_lambda(alpha2, n, l) + ggx_lambda(alpha2, n, v));
}

// Visible normal density D_v(H) = G1(V) D(H) |H.V / N.V| (ShapeInvariantMicrofacet.h:124-138).
__device__ __forceinline__ float ggx_vndf(float alpha, V3 n, V3 h, V3 v)
{
	const float g1v = 1.0f / (1.0f + ggx_lambda(alpha * alpha, n, v));
	return g1v * ggx_d(alpha, n, h) * fabsf(dot(h, v) / dot(n, v));
}

// Dupuy's spherical-cap VNDF sampling in the stretched frame (TrowbridgeReitz.cpp:19-82).
__device__ __forceinline__ V3 ggx_sample_visible_h(const Frame& f, float alpha, V3 v, float u0, float u1)
{
	const V3 upper_v = dot(v, f.ns) >= 0.0f ? v : -v;
	const V3 lv = world_to_local(f, upper_v);
	const V3 sv = normalize(v3(lv.x * alpha, lv.y, lv.z * alpha));
	const float phi = kTwoPi * u0;
	const float y = fmaf(1.0f - u1, 1.0f + sv.y, -sv.y);
	const float sin_theta = sqrtf(clampf(1.0f - y * y, 0.0f, 1.0f));
	float sp, cp;
	sincosf(phi, &sp, &cp);
	const V3 hemi = v3(sin_theta * sp, y, sin_theta * cp) + sv;
	const V3 local_h = v3(hemi.x * alpha, hemi.y, hemi.z * alpha);
	const V3 world_h = local_to_world(f, local_h);
	const float len2 = length_sq(world_h);
	// safeNormalize(N): fall back to the normal if the direction cannot be normalised.
	const V3 h = world_h * (1.0f / sqrtf(len2));
	return (len2 > 0.0f && is_finite(h)) ? h : f.ns;
}

__device__ __forceinline__ bool half_vector_same_hemisphere(V3 l, V3 v, V3 n, V3* out_h)
{
	V3 h = l + v;
	if(is_zero(h))
	{
		return false;
	}
	h = normalize(h);
	const float nh = dot(n, h);
	const float s = nh > 0.0f ? 1.0f : (nh < 0.0f ? -1.0f : 0.0f);
	h = h * s;
	*out_h = h;
	return !is_zero(h);
}

__device__ __forceinline__ RGB schlick(RGB f0, float cos_i)
{
	// std::pow(float, int) promotes to double in the reference; x^5 in double then to float.
	const double x = static_cast<double>(1.0f - fabsf(cos_i));
	const double x2 = x * x;
	const float m = static_cast<float>(x2 * x2 * x);
	return RGB{(1.0f - f0.r) * m + f0.r, (1.0f - f0.g) * m + f0.g, (1.0f - f0.b) * m + f0.b};
}

__device__ __forceinline__ float dielectric_reflectance(float eta_outer, float eta_inner, float cos_i)
{
	float eta_i = eta_outer, eta_t = eta_inner;
	if(cos_i < 0.0f)
	{
		const float tmp = eta_i; eta_i = eta_t; eta_t = tmp;
		cos_i = fabsf(cos_i);
	}
	const float ratio = eta_i / eta_t;
	const float sin_t2 = (1.0f - cos_i * cos_i) * ratio * ratio;
	if(sin_t2 >= 1.0f)
	{
		return 1.0f;
	}
	const float cos_t = sqrtf(1.0f - sin_t2);
	const float rpar = (eta_t * cos_i - eta_i * cos_t) / (eta_t * cos_i + eta_i * cos_t);
	const float rper = (eta_i * cos_i - eta_t * cos_t) / (eta_i * cos_i + eta_t * cos_t);
	return 0.5f * (rpar * rpar + rper * rper);
}

__device__ __forceinline__ bool refract_dir(float eta_outer, float eta_inner, V3 i, V3 n, V3* out)
{
	const float ion = dot(i, n);
	const float sign_ion = ion < 0.0f ? -1.0f : 1.0f;
	const float ratio = sign_ion < 0.0f ? eta_inner / eta_outer : eta_outer / eta_inner;
	const float sq = 1.0f - ratio * ratio * (1.0f - ion * ion);
	if(sq <= 0.0f)
	{
		return false;
	}
	const float nf = ratio * ion - sign_ion * sqrtf(sq);
	*out = normalize(n * nf + i * (-ratio));
	return true;
}

__device__ __forceinline__ float reflection_probability(float f_avg)
{
	return clampf(f_avg, 0.0001f, 1.0f - 0.0001f);
}

// ---------------------------------------------------------------------------------------------
// Entry points. `mat` is the material record, f the surface frame.

struct BsdfSample
{
	V3    l;
	RGB   weight;      // pdf-applied BSDF * cos
	float rel_ior;
	float cos;
	bool  ok;
};

// bsdf_eval / bsdf_pdf / bsdf_sample are kept out of line: each holds all three surface optics,
// and the shade kernel calls pdf twice. Inlined copies made that kernel large enough to stall
// on instruction fetch.
//
// calcBsdf: returns false when not measurable.
static __device__ __noinline__ bool bsdf_eval(const Material& mat, const Frame& f, V3 l, V3 v, RGB* out)
{
	if(!sidedness_agreed(f, l) || !sidedness_agreed(f, v) || mat.type == PG_MAT_ABSORBER)
	{
		return false;
	}
	const V3 n = f.ns;
	if(mat.type == PG_MAT_MATTE)
	{
		if(!same_hemisphere(f, l, v))
		{
			return false;
		}
		*out = RGB{mat.cr * kRcpPi, mat.cg * kRcpPi, mat.cb * kRcpPi};
		return is_finite(*out);
	}
	if(mat.type == PG_MAT_CONDUCTOR)
	{
		const float nol = dot(n, l), nov = dot(n, v);
		if(!same_hemisphere(f, l, v))
		{
			return false;
		}
		V3 h;
		if(!half_vector_same_hemisphere(l, v, n, &h))
		{
			return false;
		}
		const RGB F = schlick(RGB{mat.cr, mat.cg, mat.cb}, dot(h, l));
		const float D = ggx_d(mat.alpha, n, h);
		const float G = ggx_g(mat.alpha, n, h, l, v);
		*out = F * (D * G / (4.0f * fabsf(nov * nol)));
		return is_finite(*out);
	}
	// dielectric
	const float nol = dot(n, l), nov = dot(n, v);
	const float nol_nov = nol * nov;
	if(nol_nov == 0.0f)
	{
		return false;
	}
	if(same_hemisphere(f, l, v))
	{
		V3 h;
		if(!half_vector_same_hemisphere(l, v, n, &h))
		{
			return false;
		}
		const float hol = dot(h, l);
		const float F = dielectric_reflectance(mat.ior_outer, mat.ior_inner, hol);
		const float D = ggx_d(mat.alpha, n, h);
		const float G = ggx_g(mat.alpha, n, h, l, v);
		const float val = F * (D * G / (4.0f * fabsf(nol_nov)));
		*out = RGB{val, val, val};
		return isfinite(val);
	}
	if(opposite_hemisphere(f, l, v))
	{
		float eta_i = mat.ior_outer, eta_t = mat.ior_inner;
		if(nol < 0.0f)
		{
			const float tmp = eta_i; eta_i = eta_t; eta_t = tmp;
		}
		V3 h = l * (-eta_i) + v * (-eta_t);
		if(is_zero(h))
		{
			return false;
		}
		h = normalize(h);
		if(dot(n, h) < 0.0f)
		{
			h = -h;
		}
		const float hov = dot(h, v);
		const float hol = dot(h, l);
		const float F = 1.0f - dielectric_reflectance(mat.ior_outer, mat.ior_inner, hol);
		const float D = ggx_d(mat.alpha, n, h);
		const float G = ggx_g(mat.alpha, n, h, l, v);
		const float transport = eta_t / eta_i;
		const float ior_term = transport * eta_i / (eta_i * hol + eta_t * hov);
		if(!isfinite(ior_term))
		{
			return false;
		}
		const float dot_term = fabsf(hol * hov / nol_nov);
		const float val = F * (D * G * dot_term * (ior_term * ior_term));
		*out = RGB{val, val, val};
		return isfinite(val);
	}
	return false;
}

// calcBsdfPdf: returns the solid-angle pdf, or 0 for an empty/invalid pdf (the reference's
// `operator bool` on lta::PDF requires a finite positive value).
static __device__ __noinline__ float bsdf_pdf(const Material& mat, const Frame& f, V3 l, V3 v)
{
	if(!sidedness_agreed(f, l) || !sidedness_agreed(f, v) || mat.type == PG_MAT_ABSORBER)
	{
		return 0.0f;
	}
	const V3 n = f.ns;
	float pdf = 0.0f;
	if(mat.type == PG_MAT_MATTE)
	{
		if(!same_hemisphere(f, l, v))
		{
			return 0.0f;
		}
		pdf = fabsf(dot(l, n)) * kRcpPi;
	}
	else if(mat.type == PG_MAT_CONDUCTOR)
	{
		if(!same_hemisphere(f, l, v))
		{
			return 0.0f;
		}
		V3 h;
		if(!half_vector_same_hemisphere(l, v, n, &h))
		{
			return 0.0f;
		}
		pdf = ggx_vndf(mat.alpha, n, h, v) / (4.0f * fabsf(dot(h, l)));
	}
	else
	{
		if(same_hemisphere(f, l, v))
		{
			V3 h;
			if(!half_vector_same_hemisphere(l, v, n, &h))
			{
				return 0.0f;
			}
			const float F = dielectric_reflectance(mat.ior_outer, mat.ior_inner, dot(h, l));
			const float reflect_prob = reflection_probability(F);
			pdf = ggx_vndf(mat.alpha, n, h, v) / (4.0f * fabsf(dot(h, l))) * reflect_prob;
		}
		else if(opposite_hemisphere(f, l, v))
		{
			const float nol = dot(n, l);
			float eta_i = mat.ior_outer, eta_t = mat.ior_inner;
			if(nol < 0.0f)
			{
				const float tmp = eta_i; eta_i = eta_t; eta_t = tmp;
			}
			V3 h = l * (-eta_i) + v * (-eta_t);
			if(is_zero(h))
			{
				return 0.0f;
			}
			h = normalize(h);
			if(dot(n, h) < 0.0f)
			{
				h = -h;
			}
			const float hov = dot(h, v);
			const float hol = dot(h, l);
			const float ior_term = eta_i * hol + eta_t * hov;
			const float mult = fabsf(eta_i * eta_i * hol) / (ior_term * ior_term);
			const float F = dielectric_reflectance(mat.ior_outer, mat.ior_inner, hol);
			const float refract_prob = 1.0f - reflection_probability(F);
			pdf = ggx_vndf(mat.alpha, n, h, v) * mult * refract_prob;
		}
		else
		{
			pdf = 0.0f;
		}
	}
	return (isfinite(pdf) && pdf > 0.0f) ? pdf : 0.0f;
}

// genBsdfSample with three uniform numbers (u0, u1 for the direction, u2 for the dielectric
// reflect/transmit pick, which the reference draws with `unflowedPick`).
static __device__ __noinline__ BsdfSample bsdf_sample(const Material& mat, const Frame& f, V3 v, float u0, float u1, float u2)
{
	BsdfSample s;
	s.ok = false;
	s.rel_ior = 1.0f;
	s.cos = 0.0f;
	s.weight = RGB{0.0f, 0.0f, 0.0f};
	s.l = v3(0.0f, 0.0f, 0.0f);
	if(!sidedness_agreed(f, v) || mat.type == PG_MAT_ABSORBER)
	{
		return s;
	}
	const V3 n = f.ns;
	RGB w;
	V3 l;
	if(mat.type == PG_MAT_MATTE)
	{
		// Cosine-weighted hemisphere about +y (THemisphere.h:104-120), to world, flipped to V's side.
		const float phi = kTwoPi * u0;
		const float yv = sqrtf(u1);
		const float yr = sqrtf(1.0f - yv * yv);
		float sp, cp;
		sincosf(phi, &sp, &cp);
		l = normalize(local_to_world(f, v3(sp * yr, yv, cp * yr)));
		if(dot(v, n) < 0.0f)
		{
			l = -l;
		}
		w = RGB{mat.cr, mat.cg, mat.cb};
	}
	else if(mat.type == PG_MAT_CONDUCTOR)
	{
		const V3 h = ggx_sample_visible_h(f, mat.alpha, v, u0, u1);
		const V3 mv = -v;
		l = normalize(mv - h * (2.0f * dot(h, mv)));
		const float nov = dot(n, v);
		const float hol = dot(h, l);
		const float dot_terms = fabsf(hol / nov);
		const RGB F = schlick(RGB{mat.cr, mat.cg, mat.cb}, hol);
		const float G = ggx_g(mat.alpha, n, h, l, v);
		const float D = ggx_d(mat.alpha, n, h);
		const float pdf_h = ggx_vndf(mat.alpha, n, h, v);
		w = F * (G * D * dot_terms / pdf_h);
	}
	else
	{
		const V3 h = ggx_sample_visible_h(f, mat.alpha, v, u0, u1);
		const float fr = dielectric_reflectance(mat.ior_outer, mat.ior_inner, dot(h, v));
		const float reflect_prob = reflection_probability(fr);
		float F;
		if(u2 < reflect_prob)
		{
			const V3 mv = -v;
			l = normalize(mv - h * (2.0f * dot(h, mv)));
			if(!same_hemisphere(f, v, l))
			{
				return s;
			}
			F = fr / reflect_prob;
		}
		else
		{
			V3 rl;
			if(!refract_dir(mat.ior_outer, mat.ior_inner, v, h, &rl) || !opposite_hemisphere(f, v, rl))
			{
				return s;
			}
			l = rl;
			F = 1.0f - dielectric_reflectance(mat.ior_outer, mat.ior_inner, dot(h, l));
			float eta_i = mat.ior_outer, eta_t = mat.ior_inner;
			if(dot(n, l) < 0.0f)
			{
				const float tmp = eta_i; eta_i = eta_t; eta_t = tmp;
			}
			const float rel = eta_t / eta_i;
			s.rel_ior = rel;
			F *= rel * rel;
			F /= (1.0f - reflect_prob);
		}
		const float pdf_h = ggx_vndf(mat.alpha, n, h, v);
		const float nov = dot(n, v);
		const float hov = dot(h, v);
		const float dot_terms = fabsf(hov / nov);
		const float G = ggx_g(mat.alpha, n, h, l, v);
		const float D = ggx_d(mat.alpha, n, h);
		const float val = F * (G * D * dot_terms / pdf_h);
		w = RGB{val, val, val};
	}
	const float c = fabsf(dot(n, l));
	// setPdfAppliedBsdfCos measurability (BsdfSampleQuery.h:200-213) and the outer sidedness
	// check on L (SurfaceOptics.cpp:44-49).
	s.ok = is_finite(w) && c > 0.0f && c < 1.1f && sidedness_agreed(f, l);
	s.l = l;
	s.weight = w;
	s.cos = c;
	return s;
}

}// end namespace pg
