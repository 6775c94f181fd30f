// Ray traversal of the compressed 8-wide BVH with watertight FP32 triangle tests.
//
// Closest hit replaces the reference's TLAS query
//   TBinaryBvhIntersector::isIntersecting (Engine/Source/Core/Intersection/BVH/
//   TBinaryBvhIntersector.ipp:27-50) -> TLinearDepthFirstBinaryBvh::nearestTraversal
//   (Engine/Source/Math/Algorithm/BVH/TLinearDepthFirstBinaryBvh.ipp:45-138)
//   -> PTriangle::isIntersecting (Engine/Source/Core/Intersection/PTriangle.cpp:37-49)
//   -> TWatertightTriangle::isIntersecting (Engine/Source/Math/Geometry/TWatertightTriangle.ipp:16-149)
// and any hit replaces Scene::isOccluding (Engine/Source/World/Scene.cpp:54-69), which in the
// reference runs the same nearest traversal without an early exit; the boolean is identical.
#pragma once

#include "pg_common.cuh"

namespace pg
{

// Per-ray constants of the watertight test (axis permutation and shear) and of the slab test.
struct RayTraits
{
	float ox, oy, oz;
	float dx, dy, dz;
	int   kx, ky, kz;
	float sx, sy, sz;
	float rdx, rdy, rdz;     // reciprocal direction for the slab test (zero components nudged)
	float obx, oby, obz;     // origin * reciprocal direction
	uint32_t oct;            // bit a set <=> direction component a is negative
	float okx, oky, okz;     // origin permuted like the watertight test's axes
};

__device__ __forceinline__ float pick3(float a, float b, float c, int k)
{
	return k == 0 ? a : (k == 1 ? b : c);
}

__device__ __forceinline__ RayTraits make_ray_traits(float ox, float oy, float oz, float dx, float dy, float dz)
{
	RayTraits r;
	r.ox = ox; r.oy = oy; r.oz = oz;
	r.dx = dx; r.dy = dy; r.dz = dz;

	// Dominant axis becomes z; the others keep the reference's cyclic order
	// (TWatertightTriangle.ipp:31-62).
	const float ax = fabsf(dx), ay = fabsf(dy), az = fabsf(dz);
	if(ax > ay)
	{
		if(ax > az) { r.kx = 1; r.ky = 2; r.kz = 0; }
		else        { r.kx = 0; r.ky = 1; r.kz = 2; }
	}
	else
	{
		if(ay > az) { r.kx = 2; r.ky = 0; r.kz = 1; }
		else        { r.kx = 0; r.ky = 1; r.kz = 2; }
	}
	const float dkx = pick3(dx, dy, dz, r.kx);
	const float dky = pick3(dx, dy, dz, r.ky);
	const float dkz = pick3(dx, dy, dz, r.kz);
	const float rcp_z = __fdiv_rn(1.0f, dkz);
	r.sx = __fmul_rn(-dkx, rcp_z);
	r.sy = __fmul_rn(-dky, rcp_z);
	r.sz = rcp_z;

	const float tiny = 1e-20f;
	r.rdx = 1.0f / (fabsf(dx) > tiny ? dx : copysignf(tiny, dx));
	r.rdy = 1.0f / (fabsf(dy) > tiny ? dy : copysignf(tiny, dy));
	r.rdz = 1.0f / (fabsf(dz) > tiny ? dz : copysignf(tiny, dz));
	r.obx = ox * r.rdx;
	r.oby = oy * r.rdy;
	r.obz = oz * r.rdz;
	r.oct = (dx < 0.0f ? 1u : 0u) | (dy < 0.0f ? 2u : 0u) | (dz < 0.0f ? 4u : 0u);
	r.okx = pick3(ox, oy, oz, r.kx);
	r.oky = pick3(ox, oy, oz, r.ky);
	r.okz = pick3(ox, oy, oz, r.kz);
	return r;
}

// Watertight ray/triangle test, arithmetic identical to TWatertightTriangle::isIntersecting
// (TWatertightTriangle.ipp:16-149) including operand order, the FP64 recomputation of zero edge
// functions (:85-100) and the inclusive [minT, maxT] range in scaled form (:119-133). Every
// FP32 operation is an explicitly rounded intrinsic so that no FMA contraction changes bits.
//
// The core takes the vertices and the origin already permuted (component kx, ky, kz first); the
// permutation commutes with the per-component subtraction, so permuting before or after it gives
// the same bits. Callers that test one triangle from many origins along one direction (the
// refinery) permute the triangle once.
__device__ __forceinline__ bool watertight_core(
	float okx, float oky, float okz, float sx, float sy, float sz,
	float pax, float pay, float paz,
	float pbx, float pby, float pbz,
	float pcx, float pcy, float pcz,
	float min_t, float max_t,
	float* out_t, float* out_b0, float* out_b1, float* out_b2)
{
	float atx = __fsub_rn(pax, okx), aty = __fsub_rn(pay, oky), atz = __fsub_rn(paz, okz);
	float btx = __fsub_rn(pbx, okx), bty = __fsub_rn(pby, oky), btz = __fsub_rn(pbz, okz);
	float ctx = __fsub_rn(pcx, okx), cty = __fsub_rn(pcy, oky), ctz = __fsub_rn(pcz, okz);
	struct { float sx, sy, sz; } r{sx, sy, sz};

	atx = __fadd_rn(atx, __fmul_rn(r.sx, atz));
	aty = __fadd_rn(aty, __fmul_rn(r.sy, atz));
	btx = __fadd_rn(btx, __fmul_rn(r.sx, btz));
	bty = __fadd_rn(bty, __fmul_rn(r.sy, btz));
	ctx = __fadd_rn(ctx, __fmul_rn(r.sx, ctz));
	cty = __fadd_rn(cty, __fmul_rn(r.sy, ctz));

	float ea = __fsub_rn(__fmul_rn(btx, cty), __fmul_rn(bty, ctx));
	float eb = __fsub_rn(__fmul_rn(ctx, aty), __fmul_rn(cty, atx));
	float ec = __fsub_rn(__fmul_rn(atx, bty), __fmul_rn(aty, btx));

	if(ea == 0.0f || eb == 0.0f || ec == 0.0f)
	{
		const double ea64 = __dsub_rn(__dmul_rn((double)btx, (double)cty), __dmul_rn((double)bty, (double)ctx));
		const double eb64 = __dsub_rn(__dmul_rn((double)ctx, (double)aty), __dmul_rn((double)cty, (double)atx));
		const double ec64 = __dsub_rn(__dmul_rn((double)atx, (double)bty), __dmul_rn((double)aty, (double)btx));
		ea = __double2float_rn(ea64);
		eb = __double2float_rn(eb64);
		ec = __double2float_rn(ec64);
	}

	if((ea < 0.0f || eb < 0.0f || ec < 0.0f) && (ea > 0.0f || eb > 0.0f || ec > 0.0f))
	{
		return false;
	}

	const float det = __fadd_rn(__fadd_rn(ea, eb), ec);
	if(det == 0.0f || !isfinite(det))
	{
		return false;
	}

	atz = __fmul_rn(atz, r.sz);
	btz = __fmul_rn(btz, r.sz);
	ctz = __fmul_rn(ctz, r.sz);
	const float t_scaled = __fadd_rn(__fadd_rn(__fmul_rn(ea, atz), __fmul_rn(eb, btz)), __fmul_rn(ec, ctz));
	if(det > 0.0f)
	{
		if(t_scaled < __fmul_rn(min_t, det) || t_scaled > __fmul_rn(max_t, det))
		{
			return false;
		}
	}
	else
	{
		if(t_scaled > __fmul_rn(min_t, det) || t_scaled < __fmul_rn(max_t, det))
		{
			return false;
		}
	}

	const float rcp_det = __fdiv_rn(1.0f, det);
	*out_b0 = __fmul_rn(ea, rcp_det);
	*out_b1 = __fmul_rn(eb, rcp_det);
	*out_b2 = __fmul_rn(ec, rcp_det);
	*out_t  = __fmul_rn(t_scaled, rcp_det);
	return true;
}

__device__ __forceinline__ bool watertight_hit(
	const RayTraits& r,
	float ax, float ay, float az,
	float bx, float by, float bz,
	float cx, float cy, float cz,
	float min_t, float max_t,
	float* out_t, float* out_b0, float* out_b1, float* out_b2)
{
	return watertight_core(r.okx, r.oky, r.okz, r.sx, r.sy, r.sz,
	                       pick3(ax, ay, az, r.kx), pick3(ax, ay, az, r.ky), pick3(ax, ay, az, r.kz),
	                       pick3(bx, by, bz, r.kx), pick3(bx, by, bz, r.ky), pick3(bx, by, bz, r.kz),
	                       pick3(cx, cy, cz, r.kx), pick3(cx, cy, cz, r.ky), pick3(cx, cy, cz, r.kz),
	                       min_t, max_t, out_t, out_b0, out_b1, out_b2);
}

__device__ __forceinline__ bool watertight_hit_tri(
	const RayTraits& r, const LeafTri* __restrict__ tris, uint32_t k,
	float min_t, float max_t, float* t, float* b0, float* b1, float* b2)
{
	const float4* p = reinterpret_cast<const float4*>(tris + k);
	const float4 a = __ldg(p + 0);
	const float4 b = __ldg(p + 1);
	const float4 c = __ldg(p + 2);
	return watertight_hit(r, a.x, a.y, a.z, b.x, b.y, b.z, c.x, c.y, c.z, min_t, max_t, t, b0, b1, b2);
}

__device__ __forceinline__ uint32_t byte_of(uint32_t word, int i)
{
	return (word >> (8 * i)) & 0xFFu;
}

// Intersects the 8 child boxes of a wide node. Returns the hit mask: bits 24..31 are internal
// children at key (slot ^ oct), bits 0..23 are leaf triangles relative to tri_base.
__device__ __forceinline__ uint32_t intersect_children(
	const RayTraits& r, const WideNode* __restrict__ nodes, uint32_t node_index,
	float t_min, float t_max,
	uint32_t* out_child_base, uint32_t* out_tri_base, uint32_t* out_imask)
{
	const uint4* np = reinterpret_cast<const uint4*>(nodes + node_index);
	const uint4 w0 = __ldg(np + 0);
	const uint4 w1 = __ldg(np + 1);
	const uint4 w2 = __ldg(np + 2);
	const uint4 w3 = __ldg(np + 3);
	const uint4 w4 = __ldg(np + 4);

	const float px = __uint_as_float(w0.x);
	const float py = __uint_as_float(w0.y);
	const float pz = __uint_as_float(w0.z);
	const uint32_t ex = byte_of(w0.w, 0), ey = byte_of(w0.w, 1), ez = byte_of(w0.w, 2);
	const uint32_t imask = byte_of(w0.w, 3);
	*out_child_base = w1.x;
	*out_tri_base = w1.y;
	*out_imask = imask;

	const float scx = __uint_as_float(ex << 23) * r.rdx;
	const float scy = __uint_as_float(ey << 23) * r.rdy;
	const float scz = __uint_as_float(ez << 23) * r.rdz;
	const float bx = px * r.rdx - r.obx;
	const float by = py * r.rdy - r.oby;
	const float bz = pz * r.rdz - r.obz;

	// Near/far plane bytes per axis depend on the direction sign.
	const bool nx = r.oct & 1u, ny = r.oct & 2u, nz = r.oct & 4u;
	const uint32_t qlox[2] = {w2.x, w2.y}, qloy[2] = {w2.z, w2.w}, qloz[2] = {w3.x, w3.y};
	const uint32_t qhix[2] = {w3.z, w3.w}, qhiy[2] = {w4.x, w4.y}, qhiz[2] = {w4.z, w4.w};
	const uint32_t meta[2] = {w1.z, w1.w};

	uint32_t hits = 0;
#pragma unroll
	for(int half = 0; half < 2; ++half)
	{
		const uint32_t nearx = nx ? qhix[half] : qlox[half], farx = nx ? qlox[half] : qhix[half];
		const uint32_t neary = ny ? qhiy[half] : qloy[half], fary = ny ? qloy[half] : qhiy[half];
		const uint32_t nearz = nz ? qhiz[half] : qloz[half], farz = nz ? qloz[half] : qhiz[half];
#pragma unroll
		for(int j = 0; j < 4; ++j)
		{
			// Branch-free: every slot is tested (an empty slot, m = 0, contributes no bits), so the
			// lanes of a warp stay converged through the eight tests whatever their nodes hold.
			const uint32_t m = byte_of(meta[half], j);
			const float tnx = fmaf(static_cast<float>(byte_of(nearx, j)), scx, bx);
			const float tny = fmaf(static_cast<float>(byte_of(neary, j)), scy, by);
			const float tnz = fmaf(static_cast<float>(byte_of(nearz, j)), scz, bz);
			const float tfx = fmaf(static_cast<float>(byte_of(farx, j)), scx, bx);
			const float tfy = fmaf(static_cast<float>(byte_of(fary, j)), scy, by);
			const float tfz = fmaf(static_cast<float>(byte_of(farz, j)), scz, bz);
			const float tn = fmaxf(fmaxf(tnx, tny), fmaxf(tnz, t_min));
			const float tf = fminf(fminf(tfx, tfy), fminf(tfz, t_max));
			const int s = half * 4 + j;
			const uint32_t bits = ((imask >> s) & 1u) ? 1u << (24u + (static_cast<uint32_t>(s) ^ r.oct))
			                                          : (m >> 5) << (m & 31u);
			hits |= (tn <= tf && m != 0u) ? bits : 0u;
		}
	}
	return hits;
}

// Closest-hit (ANY_HIT = false) or first-hit (ANY_HIT = true) traversal. COUNT adds the
// visited-node and tested-triangle counters used by the algorithmic-bytes model.
template<bool ANY_HIT, bool COUNT = false>
__device__ __forceinline__ bool traverse(
	const RayTraits& r,
	const WideNode* __restrict__ nodes,
	const LeafTri* __restrict__ tris,
	float t_min, float t_max,
	float* out_t, uint32_t* out_tri, uint32_t* out_error,
	uint32_t* node_count = nullptr, uint32_t* tri_count = nullptr)
{
	uint2 stack[kTraversalStackSize];
	int sp = 0;

	float best_t = t_max;
	uint32_t best_tri = 0xFFFFFFFFu;
	uint32_t best_prim = 0xFFFFFFFFu;

	uint32_t child_base, tri_base, imask;
	uint32_t hits = intersect_children(r, nodes, 0, t_min, best_t, &child_base, &tri_base, &imask);
	if(COUNT) { ++*node_count; }
	uint32_t node_hits = hits >> 24;
	uint32_t tri_hits = hits & 0x00FFFFFFu;

	while(true)
	{
		while(tri_hits)
		{
			const uint32_t bit = __ffs(tri_hits) - 1u;
			tri_hits &= tri_hits - 1u;
			const uint32_t k = tri_base + bit;
			if(COUNT) { ++*tri_count; }
			float t, b0, b1, b2;
			if(watertight_hit_tri(r, tris, k, t_min, best_t, &t, &b0, &b1, &b2))
			{
				if(ANY_HIT)
				{
					*out_t = t;
					*out_tri = k;
					return true;
				}
				const uint32_t prim = __ldg(&tris[k].prim);
				if(t < best_t || prim < best_prim)
				{
					best_t = t;
					best_tri = k;
					best_prim = prim;
				}
			}
		}

		if(node_hits == 0u)
		{
			if(sp == 0)
			{
				break;
			}
			--sp;
			child_base = stack[sp].x;
			imask = stack[sp].y >> 8;
			node_hits = stack[sp].y & 0xFFu;
			continue;
		}

		const uint32_t key = 31u - __clz(node_hits);
		node_hits &= ~(1u << key);
		const uint32_t slot = key ^ r.oct;
		const uint32_t child = child_base + __popc(imask & ((1u << slot) - 1u));
		if(node_hits)
		{
			if(sp < kTraversalStackSize)
			{
				stack[sp++] = make_uint2(child_base, (imask << 8) | node_hits);
			}
			else
			{
				*out_error |= PG_DEV_ERR_STACK;
			}
		}
		hits = intersect_children(r, nodes, child, t_min, best_t, &child_base, &tri_base, &imask);
		if(COUNT) { ++*node_count; }
		node_hits = hits >> 24;
		tri_hits = hits & 0x00FFFFFFu;
	}

	*out_t = best_t;
	*out_tri = best_tri;
	return best_tri != 0xFFFFFFFFu;
}

// ---------------------------------------------------------------------------------------------
// Persistent traversal with dynamic ray fetch.
//
// Rays differ widely in the work they need (nodes visited, triangles tested), and a warp that
// traverses 32 rays to completion runs at the pace of its longest ray while finished lanes idle.
// Here every lane keeps its own traversal state; lanes whose ray has finished are refilled from a
// global ray counter as soon as kRefillMinIdle of them are idle.
//
// Each loop turn a lane does one wide-node step AND one triangle test. A node step that finds
// leaf triangles while the lane still has triangles to test parks them in a second slot; the lane
// then takes no node steps until the first slot drains, so node traversal runs at most one
// triangle group ahead of the triangle tests. Compared with one step of either kind per turn,
// where a warp of mixed lanes pays for both code paths and each lane uses one, most lanes now
// have work in both halves of a turn. Triangles are still tested in the order their groups are
// found, and nodes are visited in the same front-to-back order, so a ray's answer is that of
// traverse() above (same tie rule); node culling only sees a best_t that may lag by the parked
// group, which can cost a few extra node visits.
//
// The traversal stack's first kSharedStack entries per thread live in shared memory, the rest
// (deep trees only) in local memory.
//
// Fetch(uint32_t i, float4* origin_tmin, float4* dir_tmax) loads ray i; Finish(uint32_t i,
// bool hit, uint32_t leaf_tri, float t) consumes its result. n rays are taken from *next_ray,
// which must be zero when the launch starts. Every lane of the warp must call this function, in
// blocks of exactly kTraversalBlock threads.
//
// MULTI: rays of several scenes share the launch; fetch has the form Fetch(i, origin_tmin,
// dir_tmax, const WideNode** nodes, const LeafTri** tris) and names the tree of ray i's scene.
//
// MIXED: rays [0, n_closest) are closest-hit queries and rays [n_closest, n) any-hit queries, so
// one launch serves both queues (each lane switches per ray); counts go to node_count[0] /
// tri_count[0] for closest-hit rays and [1] for any-hit rays. min_idle: the idle lanes that make
// a warp fetch new rays (1..32; fewer refills against more idle lanes).

constexpr uint32_t kFullWarp = 0xFFFFFFFFu;
constexpr int kRefillMinIdle = 8;   // the default of min_idle
constexpr int kTraversalBlock = 128;   // threads per block of every persistent traversal launch
constexpr int kSharedStack = 8;        // stack entries per thread held in shared memory

template<bool ANY_HIT, bool COUNT, bool MIXED = false, bool MULTI = false, class Fetch, class Finish>
__device__ __forceinline__ void traverse_persistent(
	const WideNode* __restrict__ scene_nodes,
	const LeafTri* __restrict__ scene_tris,
	uint32_t n, uint32_t* __restrict__ next_ray,
	Fetch fetch, Finish finish,
	uint32_t* out_error, uint32_t* node_count = nullptr, uint32_t* tri_count = nullptr,
	uint32_t n_closest = 0, int min_idle = kRefillMinIdle)
{
	// [entry][thread]: a lane's entries are 1 KB apart, so lanes at any depths hit distinct banks
	__shared__ uint2 s_stack[kSharedStack][kTraversalBlock];
	uint2 l_stack[kTraversalStackSize - kSharedStack];

	const uint32_t tid = threadIdx.x;
	const uint32_t lane = tid & 31u;
	const uint32_t lanes_below = (1u << lane) - 1u;

	int sp = 0;
	RayTraits r{};
	float t_min = 0.0f;
	float best_t = 0.0f;
	uint32_t best_tri = 0xFFFFFFFFu, best_prim = 0xFFFFFFFFu;
	uint32_t child_base = 0, imask = 0, node_hits = 0;
	uint32_t tri_base = 0, tri_hits = 0;     // the triangle group under test
	uint32_t next_base = 0, next_hits = 0;   // a group found while the first was still under test
	uint32_t ray = 0;
	bool has_ray = false;
	bool any_hit = ANY_HIT;   // this lane's query (varies per ray only when MIXED)
	const WideNode* nodes = scene_nodes;   // this lane's tree (varies per ray only when MULTI)
	const LeafTri* tris = scene_tris;
	bool exhausted = false;   // warp-uniform: the counter has passed n

	while(true)
	{
		// ---- refill idle lanes (warp-uniform branch)
		const uint32_t idle = __ballot_sync(kFullWarp, !has_ray);
		const int num_idle = __popc(idle);
		if(!exhausted && num_idle >= min_idle)
		{
			uint32_t base = 0;
			if(lane == 0)
			{
				base = atomicAdd(next_ray, static_cast<uint32_t>(num_idle));
			}
			base = __shfl_sync(kFullWarp, base, 0);
			exhausted = base >= n || n - base <= static_cast<uint32_t>(num_idle);
			if(!has_ray)
			{
				const uint32_t i = base + __popc(idle & lanes_below);
				if(i < n && i >= base)
				{
					float4 a, b;
					if constexpr(MULTI)
					{
						fetch(i, &a, &b, &nodes, &tris);
					}
					else
					{
						fetch(i, &a, &b);
					}
					r = make_ray_traits(a.x, a.y, a.z, b.x, b.y, b.z);
					t_min = a.w;
					best_t = b.w;
					best_tri = 0xFFFFFFFFu;
					best_prim = 0xFFFFFFFFu;
					// the root as the only internal child of a virtual parent: slot 0, key = oct
					child_base = 0;
					imask = 1u;
					node_hits = 1u << r.oct;
					tri_hits = 0;
					next_hits = 0;
					sp = 0;
					ray = i;
					has_ray = true;
					if(MIXED) { any_hit = i >= n_closest; }
				}
			}
		}
		if(!__any_sync(kFullWarp, has_ray))
		{
			break;   // no lane holds a ray, so the last refill found the counter past n
		}
		if(!has_ray)
		{
			continue;
		}

		// ---- one node step, unless a triangle group is already parked
		if(next_hits == 0u)
		{
			if(node_hits == 0u && sp > 0)
			{
				--sp;
				const uint2 e = sp < kSharedStack ? s_stack[sp][tid] : l_stack[sp - kSharedStack];
				child_base = e.x;
				imask = e.y >> 8;
				node_hits = e.y & 0xFFu;
			}
			if(node_hits)
			{
				const uint32_t key = 31u - __clz(node_hits);
				node_hits &= ~(1u << key);
				const uint32_t slot = key ^ r.oct;
				const uint32_t child = child_base + __popc(imask & ((1u << slot) - 1u));
				if(node_hits)
				{
					if(sp < kTraversalStackSize)
					{
						const uint2 e = make_uint2(child_base, (imask << 8) | node_hits);
						if(sp < kSharedStack)
						{
							s_stack[sp][tid] = e;
						}
						else
						{
							l_stack[sp - kSharedStack] = e;
						}
						++sp;
					}
					else
					{
						*out_error |= PG_DEV_ERR_STACK;
					}
				}
				uint32_t found_base;
				const uint32_t hits = intersect_children(r, nodes, child, t_min, best_t, &child_base, &found_base, &imask);
				if(COUNT) { ++node_count[MIXED && any_hit ? 1 : 0]; }
				node_hits = hits >> 24;
				const uint32_t found = hits & 0x00FFFFFFu;
				if(found)
				{
					if(tri_hits == 0u)
					{
						tri_base = found_base;
						tri_hits = found;
					}
					else
					{
						next_base = found_base;
						next_hits = found;
					}
				}
			}
		}

		// ---- one triangle test
		if(tri_hits)
		{
			const uint32_t bit = __ffs(tri_hits) - 1u;
			tri_hits &= tri_hits - 1u;
			const uint32_t k = tri_base + bit;
			if(COUNT) { ++tri_count[MIXED && any_hit ? 1 : 0]; }
			float t, b0, b1, b2;
			if(watertight_hit_tri(r, tris, k, t_min, best_t, &t, &b0, &b1, &b2))
			{
				if(MIXED ? any_hit : ANY_HIT)
				{
					best_t = t;
					best_tri = k;
					tri_hits = 0;
					next_hits = 0;
					node_hits = 0;
					sp = 0;
				}
				else
				{
					const uint32_t prim = __ldg(&tris[k].prim);
					if(t < best_t || prim < best_prim)
					{
						best_t = t;
						best_tri = k;
						best_prim = prim;
					}
				}
			}
			if(tri_hits == 0u)
			{
				tri_base = next_base;
				tri_hits = next_hits;
				next_hits = 0u;
			}
		}

		if(tri_hits == 0u && node_hits == 0u && sp == 0)
		{
			finish(ray, best_tri != 0xFFFFFFFFu, best_tri, best_t);
			has_ray = false;
		}
	}
}

}// end namespace pg
