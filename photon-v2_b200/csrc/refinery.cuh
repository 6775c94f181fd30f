// Self-intersection-free ray origins by iterative re-intersection against the source triangle(s),
// the reference's default refine mode (ESurfaceRefineMode::Iterative, one refinement,
// Engine/Include/EngineInitSettings.h:32-35):
//   SurfaceHitRefinery::iterativeOffset        Engine/Source/Core/LTA/SurfaceHitRefinery.cpp:62-153
//   SurfaceHitRefinery::iterativeMutualOffset  Engine/Source/Core/LTA/SurfaceHitRefinery.cpp:155-263
//   escapeIteratively / tryEscapeIteratively   Engine/Source/Core/LTA/SurfaceHitRefinery.h:249-358
// Error factors of a PTriangle hit: mean 5e-8, max 2.5e-5 (PTriangle.cpp:128-129).
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

constexpr float kMeanErrorFactor = 5e-8f;
constexpr float kMaxErrorFactor = 5e-8f * 5e2f;
constexpr float kFloatMin = 1.17549435e-38f;   // std::numeric_limits<float>::min()
constexpr float kFloatMax = 3.40282347e+38f;
constexpr int   kMaxEscapeIterations = 64;

// Out of line (as is iterative_offset): the shade kernel runs up to three offsets per vertex, and
// inlined copies of the watertight test with its FP64 fallback bloated its instruction footprint.
static __device__ __noinline__ bool reintersect(const TriVerts& tri, V3 o, V3 d, float min_t, float max_t, float* out_t)
{
	const RayTraits r = make_ray_traits(o.x, o.y, o.z, d.x, d.y, d.z);
	float b0, b1, b2;
	return watertight_hit(r, tri.a.x, tri.a.y, tri.a.z, tri.b.x, tri.b.y, tri.b.z,
	                      tri.c.x, tri.c.y, tri.c.z, min_t, max_t, out_t, &b0, &b1, &b2);
}

struct OffsetResult
{
	V3    offset;
	V3    unit_dir;
	float max_distance;
};

// iterativeOffset (SurfaceHitRefinery.cpp:62-153). Triangles always pass canVerifyOffset
// (planar, triangular face topology), so the empirical fallback never applies.
static __device__ __noinline__ OffsetResult iterative_offset(V3 pos, V3 ng, const TriVerts& tri, V3 dir)
{
	const V3 offset_dir = dot(ng, dir) > 0.0f ? ng : -ng;
	const V3 escape_dir = normalize(dir);
	const float escape_cos = clampf(dot(escape_dir, offset_dir), 0.0f, 1.0f);
	const float initial = length(pos) * kMeanErrorFactor + kFloatMin;

	float max_dist = initial;
	float min_dist = 0.0f;
	for(int it = 0; it < kMaxEscapeIterations; ++it)
	{
		float t;
		if(!reintersect(tri, pos + offset_dir * max_dist, escape_dir, 0.0f, kFloatMax, &t))
		{
			break;
		}
		max_dist += t * escape_cos;
		min_dist = max_dist;
		max_dist *= 2.0f;
	}

	// One bisection refinement.
	for(int it = 0, refinements = 0; refinements < 1 && it < kMaxEscapeIterations; ++it)
	{
		const float mid = (min_dist + max_dist) * 0.5f;
		if(!(min_dist < mid && mid < max_dist))
		{
			break;
		}
		float t;
		if(!reintersect(tri, pos + offset_dir * mid, escape_dir, 0.0f, kFloatMax, &t))
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
__device__ __forceinline__ OffsetResult iterative_mutual_offset(
	V3 pos, V3 ng, const TriVerts& tri,
	V3 pos2, const TriVerts& tri2)
{
	const V3 dir = pos2 - pos;
	const OffsetResult rx = iterative_offset(pos, ng, tri, dir);

	const float initial = length(pos2) * kMaxErrorFactor + kFloatMin;
	const V3 origin = pos + rx.offset;
	const float dist_to_x2 = length(origin - pos2);

	float max_dist = initial;
	float min_dist = 0.0f;
	for(int it = 0; it < kMaxEscapeIterations && dist_to_x2 > max_dist; ++it)
	{
		float t;
		if(!reintersect(tri2, origin, rx.unit_dir, 0.0f, dist_to_x2 - max_dist, &t))
		{
			break;
		}
		max_dist = fmaxf(dist_to_x2 - t, max_dist);
		min_dist = max_dist;
		max_dist *= 2.0f;
	}

	for(int it = 0, refinements = 0; dist_to_x2 > max_dist && refinements < 1 && it < kMaxEscapeIterations; ++it)
	{
		const float mid = (min_dist + max_dist) * 0.5f;
		if(!(min_dist < mid && mid < max_dist))
		{
			break;
		}
		float t;
		if(!reintersect(tri2, origin, rx.unit_dir, 0.0f, dist_to_x2 - mid, &t))
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

}// end namespace pg
