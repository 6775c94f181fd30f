// Self-intersection-free ray origins by iterative re-intersection against the source triangle(s),
// the reference's default refine mode (ESurfaceRefineMode::Iterative, one refinement,
// Engine/Include/EngineInitSettings.h:32-35):
//   SurfaceHitRefinery::iterativeOffset        Engine/Source/Core/LTA/SurfaceHitRefinery.cpp:62-153
//   SurfaceHitRefinery::iterativeMutualOffset  Engine/Source/Core/LTA/SurfaceHitRefinery.cpp:155-263
//   escapeIteratively / tryEscapeIteratively   Engine/Source/Core/LTA/SurfaceHitRefinery.h:249-358
// Error factors of a PTriangle hit: mean 5e-8, max 2.5e-5 (PTriangle.cpp:128-129), which
// HitDetail::setDistanceErrorFactors stores as powers of two (Core/HitDetail.h:185-200: exponent
// round(log2(mean)) = -24 and ceil(log2(max)) = -15), so the refinery works with 2^-24 and 2^-15.
// Every re-intersection is the watertight test against one triangle, so the offsets are the
// reference's to the bit. Loops the reference leaves unbounded are capped (64 doublings cover the
// whole float range), which no finite input reaches.
#pragma once

#include "trace.cuh"

namespace pg
{

struct TriVerts
{
	V3 a, b, c;
};

constexpr float kMeanErrorFactor = 5.9604644775390625e-8f;   // 2^-24
constexpr float kMaxErrorFactor = 3.0517578125e-5f;         // 2^-15
constexpr float kFloatMin = 1.17549435e-38f;   // std::numeric_limits<float>::min()
constexpr float kFloatMax = 3.40282347e+38f;
constexpr int   kMaxEscapeIterations = 64;

// One triangle seen along one direction: the direction's axis permutation and shear, and the
// triangle's vertices already permuted. Each refinement loop re-intersects the same triangle from
// a moving origin along a fixed direction, so this is computed once per loop.
struct RefineRay
{
	float sx, sy, sz;
	int   kx, ky, kz;
	float a[3], b[3], c[3];
};

__device__ __forceinline__ RefineRay make_refine_ray(const TriVerts& tri, V3 d)
{
	const RayTraits r = make_ray_traits(0.0f, 0.0f, 0.0f, d.x, d.y, d.z);
	RefineRay q;
	q.sx = r.sx; q.sy = r.sy; q.sz = r.sz;
	q.kx = r.kx; q.ky = r.ky; q.kz = r.kz;
	q.a[0] = pick3(tri.a.x, tri.a.y, tri.a.z, r.kx); q.a[1] = pick3(tri.a.x, tri.a.y, tri.a.z, r.ky); q.a[2] = pick3(tri.a.x, tri.a.y, tri.a.z, r.kz);
	q.b[0] = pick3(tri.b.x, tri.b.y, tri.b.z, r.kx); q.b[1] = pick3(tri.b.x, tri.b.y, tri.b.z, r.ky); q.b[2] = pick3(tri.b.x, tri.b.y, tri.b.z, r.kz);
	q.c[0] = pick3(tri.c.x, tri.c.y, tri.c.z, r.kx); q.c[1] = pick3(tri.c.x, tri.c.y, tri.c.z, r.ky); q.c[2] = pick3(tri.c.x, tri.c.y, tri.c.z, r.kz);
	return q;
}

// Same bits as the full watertight test of a ray from o along the RefineRay's direction. Inlined
// into the out-of-line offset functions below, which keep the shade kernel's own code small.
__device__ __forceinline__ bool reintersect(const RefineRay& q, V3 o, float min_t, float max_t, float* out_t)
{
	float b0, b1, b2;
	return watertight_core(pick3(o.x, o.y, o.z, q.kx), pick3(o.x, o.y, o.z, q.ky), pick3(o.x, o.y, o.z, q.kz),
	                       q.sx, q.sy, q.sz, q.a[0], q.a[1], q.a[2], q.b[0], q.b[1], q.b[2], q.c[0], q.c[1], q.c[2],
	                       min_t, max_t, out_t, &b0, &b1, &b2);
}

struct OffsetResult
{
	V3    offset;
	V3    unit_dir;
	float max_distance;
};

// iterativeOffset (SurfaceHitRefinery.cpp:62-153). Triangles always pass canVerifyOffset
// (planar, triangular face topology), so the empirical fallback never applies. `iters` is the
// number of bisection refinements (EngineInitSettings::numIterativeSurfaceRefinements).
static __device__ __noinline__ OffsetResult iterative_offset(V3 pos, V3 ng, const TriVerts& tri, V3 dir, int iters = 1)
{
	const V3 offset_dir = dot(ng, dir) > 0.0f ? ng : -ng;
	const V3 escape_dir = normalize(dir);
	const float escape_cos = clampf(dot(escape_dir, offset_dir), 0.0f, 1.0f);
	const float initial = length(pos) * kMeanErrorFactor + kFloatMin;
	const RefineRay q = make_refine_ray(tri, escape_dir);

	float max_dist = initial;
	float min_dist = 0.0f;
	for(int it = 0; it < kMaxEscapeIterations; ++it)
	{
		float t;
		if(!reintersect(q, pos + offset_dir * max_dist, 0.0f, kFloatMax, &t))
		{
			break;
		}
		max_dist += t * escape_cos;
		min_dist = max_dist;
		max_dist *= 2.0f;
	}

	// Bisection refinements.
	for(int it = 0, refinements = 0; refinements < iters && it < kMaxEscapeIterations; ++it)
	{
		const float mid = (min_dist + max_dist) * 0.5f;
		if(!(min_dist < mid && mid < max_dist))
		{
			break;
		}
		float t;
		if(!reintersect(q, pos + offset_dir * mid, 0.0f, kFloatMax, &t))
		{
			max_dist = mid;
			++refinements;
		}
		else
		{
			min_dist = clampf(mid + t * escape_cos, mid, max_dist);
		}
	}

	OffsetResult r;
	r.offset = offset_dir * max_dist;
	r.unit_dir = escape_dir;
	r.max_distance = kFloatMax;
	return r;
}

// iterativeMutualOffset (SurfaceHitRefinery.cpp:155-263): escape X towards X2, then shorten the
// segment until it no longer touches X2's triangle.
static __device__ __noinline__ OffsetResult iterative_mutual_offset(
	V3 pos, V3 ng, const TriVerts& tri,
	V3 pos2, const TriVerts& tri2, int iters = 1)
{
	const V3 dir = pos2 - pos;
	const OffsetResult rx = iterative_offset(pos, ng, tri, dir, iters);

	const float initial = length(pos2) * kMaxErrorFactor + kFloatMin;
	const V3 origin = pos + rx.offset;
	const float dist_to_x2 = length(origin - pos2);
	const RefineRay q2 = make_refine_ray(tri2, rx.unit_dir);

	float max_dist = initial;
	float min_dist = 0.0f;
	for(int it = 0; it < kMaxEscapeIterations && dist_to_x2 > max_dist; ++it)
	{
		float t;
		if(!reintersect(q2, origin, 0.0f, dist_to_x2 - max_dist, &t))
		{
			break;
		}
		max_dist = fmaxf(dist_to_x2 - t, max_dist);
		min_dist = max_dist;
		max_dist *= 2.0f;
	}

	for(int it = 0, refinements = 0; dist_to_x2 > max_dist && refinements < iters && it < kMaxEscapeIterations; ++it)
	{
		const float mid = (min_dist + max_dist) * 0.5f;
		if(!(min_dist < mid && mid < max_dist))
		{
			break;
		}
		float t;
		if(!reintersect(q2, origin, 0.0f, dist_to_x2 - mid, &t))
		{
			max_dist = mid;
			++refinements;
		}
		else
		{
			min_dist = clampf(dist_to_x2 - t, mid, max_dist);
		}
	}

	OffsetResult r;
	r.offset = rx.offset;
	r.unit_dir = rx.unit_dir;
	r.max_distance = fmaxf(dist_to_x2 - max_dist, 0.0f);
	return r;
}

// ---------------------------------------------------------------------------------------------
// The reference's other refine modes (ESurfaceRefineMode, selected by RefineMode in its
// Config/EngineConfig.ini): Empirical offsets along the geometry normal by the maximum error bound
// |p| * 2^-15 (SurfaceHitRefinery::empiricalOffsetVec, SurfaceHitRefinery.h:412-428); Manual
// starts the ray at the hit point with minT = delta (selfIntersectDelta, SurfaceHitRefinery.h:220-232,
// 282-305).

enum RefineMode : uint32_t
{
	PG_REFINE_MANUAL = 0,
	PG_REFINE_EMPIRICAL = 1,
	PG_REFINE_ITERATIVE = 2,
};

struct RefineSettings
{
	uint32_t mode = PG_REFINE_ITERATIVE;
	float    delta = 2e-4f;
	int      iters = 1;
};

__device__ __forceinline__ V3 empirical_offset_vec(V3 pos, V3 ng, V3 dir)
{
	const float dist = length(pos) * kMaxErrorFactor;
	return dot(ng, dir) > 0.0f ? ng * dist : ng * -dist;
}

// A ray leaving the surface: origin, unit direction, range [min_t, max_distance].
struct EscapeRay
{
	V3    origin;
	V3    unit_dir;
	float min_t;
	float max_distance;
	bool  ok;
};

// SurfaceHitRefinery::escape (SurfaceHitRefinery.h:200-263) in the iterative mode.
__device__ __forceinline__ EscapeRay escape_iterative(V3 pos, V3 ng, const TriVerts& tri, V3 dir, int iters)
{
	const OffsetResult r = iterative_offset(pos, ng, tri, dir, iters);
	EscapeRay e;
	e.ok = true;
	e.min_t = 0.0f;
	e.origin = pos + r.offset;
	e.unit_dir = r.unit_dir;
	e.max_distance = r.max_distance;
	return e;
}

// SurfaceHitRefinery::tryEscape (SurfaceHitRefinery.h:265-360) in the iterative mode.
__device__ __forceinline__ EscapeRay try_escape_iterative(V3 pos, V3 ng, const TriVerts& tri, V3 pos2,
                                                          const TriVerts& tri2, int iters)
{
	const OffsetResult r = iterative_mutual_offset(pos, ng, tri, pos2, tri2, iters);
	EscapeRay e;
	e.min_t = 0.0f;
	e.origin = pos + r.offset;
	e.unit_dir = r.unit_dir;
	e.max_distance = r.max_distance;
	e.ok = r.max_distance > 0.0f && isfinite(r.max_distance);
	return e;
}

// SurfaceHitRefinery::escape in the empirical and manual modes (no re-intersection).
__device__ __forceinline__ EscapeRay escape_fixed(const RefineSettings& rs, V3 pos, V3 ng, V3 dir)
{
	EscapeRay e;
	e.ok = true;
	e.min_t = 0.0f;
	e.max_distance = kFloatMax;
	if(rs.mode == PG_REFINE_EMPIRICAL)
	{
		e.origin = pos + empirical_offset_vec(pos, ng, dir);
		e.unit_dir = normalize(dir);
	}
	else
	{
		e.origin = pos;
		e.unit_dir = normalize(dir);
		e.min_t = rs.delta;
	}
	return e;
}

// SurfaceHitRefinery::tryEscape in the empirical and manual modes.
__device__ __forceinline__ EscapeRay try_escape_fixed(const RefineSettings& rs, V3 pos, V3 ng, V3 pos2, V3 ng2)
{
	EscapeRay e;
	e.ok = false;
	e.min_t = 0.0f;
	e.max_distance = 0.0f;
	if(rs.mode == PG_REFINE_EMPIRICAL)
	{
		const V3 x_to_x2 = pos2 - pos;
		const V3 origin = pos + empirical_offset_vec(pos, ng, x_to_x2);
		const V3 origin2 = pos2 + empirical_offset_vec(pos2, ng2, -x_to_x2);
		const float distance = length(origin2 - origin);
		const float rcp = 1.0f / distance;
		if(rcp != 0.0f && isfinite(rcp))
		{
			e.origin = origin;
			e.unit_dir = (origin2 - origin) * rcp;
			e.max_distance = distance;
			e.ok = true;
		}
	}
	else
	{
		const V3 x_to_x2 = pos2 - pos;
		const float d2 = length_sq(x_to_x2);
		const float three_delta = rs.delta * 3.0f;
		if(d2 > three_delta * three_delta)
		{
			const float distance = sqrtf(d2);
			const float rcp = 1.0f / distance;
			e.origin = pos;
			e.unit_dir = x_to_x2 * rcp;
			e.min_t = rs.delta;
			e.max_distance = distance - rs.delta;
			e.ok = true;
		}
	}
	return e;
}

}// end namespace pg
