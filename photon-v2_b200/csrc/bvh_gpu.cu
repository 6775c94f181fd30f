// GPU builder of the compressed 8-wide BVH (the same node and leaf layout as bvh_build.cpp).
//
// The reference builds its TLAS on the host with a bucketed-SAH binary builder
// (Engine/Source/Math/Algorithm/BVH/TBvhBuilder.ipp:36,516). For multi-million-triangle scenes
// that build dominates turnaround, so this path builds on the device instead:
//   1. per-triangle boxes and centroids, scene centroid bound (block reductions + atomics);
//   2. 63-bit Morton codes of the centroids, sorted with their indices (CUB radix sort);
//   3. the binary tree by parallel locally-ordered clustering (PLOC, Meister & Bittner 2018):
//      every cluster finds, among its neighbours within a radius in Morton order, the one whose
//      merged box has the least surface area; mutual nearest neighbours merge; the survivors
//      are compacted and the pass repeats until one cluster is left;
//   4. collapse to 8-wide nodes level by level, one thread per wide node: open the largest
//      child holding more than 3 triangles until 8 children, assign octant slots and quantise
//      the child boxes conservatively exactly as the host builder does.
// The closest hit a ray finds does not depend on the tree (boxes are conservative, ties are
// resolved by primitive index), only traversal cost does.
#include "pg_geometry.h"
#include "pg_runtime.h"

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_select.cuh>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <stdexcept>
#include <string>

namespace pg
{
namespace
{

constexpr uint32_t kLeafMax = 3;
constexpr uint32_t kLeafRef = 0x80000000u;   // a binary child reference naming a sorted primitive
constexpr uint32_t kNone = 0xFFFFFFFFu;
constexpr int kBlock = 256;

enum BuildError : uint32_t
{
	BUILD_ERR_NODE_OVERFLOW = 1u << 0,
	BUILD_ERR_TRI_OVERFLOW = 1u << 1,
};

// Order-preserving float atomics on int bit patterns (the target starts at +inf / -inf).
__device__ __forceinline__ void atomic_min_f(float* a, float v)
{
	if(v >= 0.0f) { atomicMin(reinterpret_cast<int*>(a), __float_as_int(v)); }
	else          { atomicMax(reinterpret_cast<unsigned*>(a), __float_as_uint(v)); }
}

__device__ __forceinline__ void atomic_max_f(float* a, float v)
{
	if(v >= 0.0f) { atomicMax(reinterpret_cast<int*>(a), __float_as_int(v)); }
	else          { atomicMin(reinterpret_cast<unsigned*>(a), __float_as_uint(v)); }
}

// stats: [0..2] centroid min, [3..5] centroid max, [6] max |coordinate|
__global__ void prim_kernel(const float* __restrict__ tris, uint32_t n, float4* __restrict__ lo,
                            float4* __restrict__ hi, float* __restrict__ stats)
{
	float cmin[3] = {3.0e38f, 3.0e38f, 3.0e38f}, cmax[3] = {-3.0e38f, -3.0e38f, -3.0e38f}, mabs = 0.0f;
	for(uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
	{
		const float* v = tris + 9ull * i;
		float l[3], h[3];
		for(int a = 0; a < 3; ++a)
		{
			l[a] = fminf(fminf(v[a], v[3 + a]), v[6 + a]);
			h[a] = fmaxf(fmaxf(v[a], v[3 + a]), v[6 + a]);
			if(!isfinite(l[a]) || !isfinite(h[a]))
			{
				// non-finite vertices: an empty-but-valid box at the origin; the watertight test
				// rejects the triangle anyway
				l[a] = 0.0f;
				h[a] = 0.0f;
			}
			const float c = 0.5f * (l[a] + h[a]);
			cmin[a] = fminf(cmin[a], c);
			cmax[a] = fmaxf(cmax[a], c);
			mabs = fmaxf(mabs, fmaxf(fabsf(l[a]), fabsf(h[a])));
		}
		lo[i] = make_float4(l[0], l[1], l[2], 0.0f);
		hi[i] = make_float4(h[0], h[1], h[2], 0.0f);
	}
	for(int o = 16; o > 0; o >>= 1)
	{
		for(int a = 0; a < 3; ++a)
		{
			cmin[a] = fminf(cmin[a], __shfl_xor_sync(0xFFFFFFFFu, cmin[a], o));
			cmax[a] = fmaxf(cmax[a], __shfl_xor_sync(0xFFFFFFFFu, cmax[a], o));
		}
		mabs = fmaxf(mabs, __shfl_xor_sync(0xFFFFFFFFu, mabs, o));
	}
	if((threadIdx.x & 31) == 0)
	{
		for(int a = 0; a < 3; ++a)
		{
			atomic_min_f(&stats[a], cmin[a]);
			atomic_max_f(&stats[3 + a], cmax[a]);
		}
		atomic_max_f(&stats[6], mabs);
	}
}

__device__ __forceinline__ uint64_t spread21(uint32_t x)
{
	uint64_t v = x & 0x1FFFFFu;
	v = (v | (v << 32)) & 0x1F00000000FFFFull;
	v = (v | (v << 16)) & 0x1F0000FF0000FFull;
	v = (v | (v << 8)) & 0x100F00F00F00F00Full;
	v = (v | (v << 4)) & 0x10C30C30C30C30C3ull;
	v = (v | (v << 2)) & 0x1249249249249249ull;
	return v;
}

__global__ void morton_kernel(const float4* __restrict__ lo, const float4* __restrict__ hi, uint32_t n,
                              const float* __restrict__ stats, uint64_t* __restrict__ keys, uint32_t* __restrict__ idx)
{
	float scale[3];
	for(int a = 0; a < 3; ++a)
	{
		const float ext = stats[3 + a] - stats[a];
		scale[a] = ext > 0.0f ? 2097151.0f / ext : 0.0f;
	}
	for(uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
	{
		const float4 l = lo[i], h = hi[i];
		const float c[3] = {0.5f * (l.x + h.x), 0.5f * (l.y + h.y), 0.5f * (l.z + h.z)};
		uint32_t q[3];
		for(int a = 0; a < 3; ++a)
		{
			const float t = (c[a] - stats[a]) * scale[a];
			q[a] = static_cast<uint32_t>(fminf(fmaxf(t, 0.0f), 2097151.0f));
		}
		keys[i] = (spread21(q[0]) << 2) | (spread21(q[1]) << 1) | spread21(q[2]);
		idx[i] = i;
	}
}

__device__ __forceinline__ void ref_box(uint32_t ref, const float4* __restrict__ plo, const float4* __restrict__ phi,
                                        const uint32_t* __restrict__ sorted, const float4* nlo, const float4* nhi,
                                        float4* l, float4* h)
{
	if(ref & kLeafRef)
	{
		const uint32_t p = sorted[ref & ~kLeafRef];
		*l = plo[p];
		*h = phi[p];
	}
	else
	{
		*l = __ldcg(nlo + ref);
		*h = __ldcg(nhi + ref);
	}
}

constexpr int kPlocRadius = 16;
constexpr int kPlocBlock = 256;

__device__ __forceinline__ float merged_area(float4 la, float4 ha, float4 lb, float4 hb)
{
	const float dx = fmaxf(ha.x, hb.x) - fminf(la.x, lb.x);
	const float dy = fmaxf(ha.y, hb.y) - fminf(la.y, lb.y);
	const float dz = fmaxf(ha.z, hb.z) - fminf(la.z, lb.z);
	return dx * dy + dy * dz + dz * dx;
}

// Nearest neighbour of every cluster among the kPlocRadius clusters on each side. Pairs are
// ordered by (merged area, index distance, parity of the lower index, lower index), a total
// order, so the globally closest pair is always mutual and every pass merges at least once; the
// parity term pairs equal-area runs (identical boxes) as (0,1), (2,3), ... so that they still
// halve per pass instead of chaining. The block's clusters and the radius around them are staged
// in shared memory.
__global__ void __launch_bounds__(kPlocBlock)
ploc_neighbour_kernel(const uint32_t* __restrict__ clusters, uint32_t m, const uint32_t* __restrict__ sorted,
                      const float4* __restrict__ plo, const float4* __restrict__ phi, const float4* __restrict__ nlo,
                      const float4* __restrict__ nhi, uint32_t* __restrict__ nn)
{
	__shared__ float4 slo[kPlocBlock + 2 * kPlocRadius], shi[kPlocBlock + 2 * kPlocRadius];
	const int base = static_cast<int>(blockIdx.x) * kPlocBlock - kPlocRadius;
	for(int t = threadIdx.x; t < kPlocBlock + 2 * kPlocRadius; t += kPlocBlock)
	{
		const int c = base + t;
		if(c >= 0 && c < static_cast<int>(m))
		{
			ref_box(clusters[c], plo, phi, sorted, nlo, nhi, &slo[t], &shi[t]);
		}
	}
	__syncthreads();
	const int i = static_cast<int>(blockIdx.x) * kPlocBlock + static_cast<int>(threadIdx.x);
	if(i >= static_cast<int>(m))
	{
		return;
	}
	const int ti = i - base;
	float best = 3.0e38f;
	int bj = -1, best_dist = 0, best_par = 0, best_min = 0;
	const int lo = max(0, i - kPlocRadius), hi = min(static_cast<int>(m) - 1, i + kPlocRadius);
	for(int j = lo; j <= hi; ++j)
	{
		if(j == i)
		{
			continue;
		}
		const float area = merged_area(slo[ti], shi[ti], slo[j - base], shi[j - base]);
		const int dist = abs(j - i), mn = min(i, j), par = mn & 1;
		const bool better = bj < 0 || area < best ||
			(area == best && (dist < best_dist || (dist == best_dist && (par < best_par ||
			(par == best_par && mn < best_min)))));
		if(better)
		{
			best = area;
			bj = j;
			best_dist = dist;
			best_par = par;
			best_min = mn;
		}
	}
	nn[i] = bj < 0 ? kNone : static_cast<uint32_t>(bj);
}

// Mutual nearest neighbours merge into a new internal node kept at the lower position; the
// higher position is dropped (flag 0).
__global__ void ploc_merge_kernel(const uint32_t* __restrict__ clusters, uint32_t m, const uint32_t* __restrict__ nn,
                                  const uint32_t* __restrict__ sorted, const float4* __restrict__ plo,
                                  const float4* __restrict__ phi, uint32_t* __restrict__ next_node,
                                  uint32_t* __restrict__ left, uint32_t* __restrict__ right,
                                  uint32_t* __restrict__ count_of, float4* nlo, float4* nhi,
                                  uint32_t* __restrict__ out, uint8_t* __restrict__ keep, uint32_t node_limit,
                                  uint32_t* __restrict__ error)
{
	for(uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x)
	{
		const uint32_t j = nn[i];
		const bool mutual = j != kNone && nn[j] == i;
		if(!mutual)
		{
			out[i] = clusters[i];
			keep[i] = 1;
			continue;
		}
		if(i > j)
		{
			keep[i] = 0;
			continue;
		}
		const uint32_t k = atomicAdd(next_node, 1u);
		if(k >= node_limit)
		{
			atomicOr(error, BUILD_ERR_NODE_OVERFLOW);
			out[i] = clusters[i];
			keep[i] = 1;
			continue;
		}
		const uint32_t a = clusters[i], b = clusters[j];
		float4 la, ha, lb, hb;
		ref_box(a, plo, phi, sorted, nlo, nhi, &la, &ha);
		ref_box(b, plo, phi, sorted, nlo, nhi, &lb, &hb);
		left[k] = a;
		right[k] = b;
		count_of[k] = ((a & kLeafRef) ? 1u : count_of[a]) + ((b & kLeafRef) ? 1u : count_of[b]);
		nlo[k] = make_float4(fminf(la.x, lb.x), fminf(la.y, lb.y), fminf(la.z, lb.z), 0.0f);
		nhi[k] = make_float4(fmaxf(ha.x, hb.x), fmaxf(ha.y, hb.y), fmaxf(ha.z, hb.z), 0.0f);
		out[i] = k;
		keep[i] = 1;
	}
}

__global__ void leaf_refs_kernel(uint32_t n, uint32_t* __restrict__ clusters)
{
	for(uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
	{
		clusters[i] = kLeafRef | i;
	}
}

struct CollapseArgs
{
	const float*    tris;
	const uint32_t* materials;
	const uint32_t* emitters;
	const uint32_t* sorted;
	const float4*   plo;
	const float4*   phi;
	const float4*   nlo;
	const float4*   nhi;
	const uint32_t* left;
	const uint32_t* right;
	const uint32_t* count_of;
	WideNode*       nodes;
	LeafTri*        leaf_tris;
	uint32_t        node_capacity;
	uint32_t        num_tris;
	float           pad;
	uint32_t*       counters;   // [0] nodes used, [1] leaf triangles used, [2] error flags
};

__device__ __forceinline__ void set_byte(WideNode& node, int word, int byte, uint32_t v)
{
	node.w[word] = (node.w[word] & ~(0xFFu << (8 * byte))) | ((v & 0xFFu) << (8 * byte));
}

// One wide node per thread: items are (binary node reference, wide node index) pairs.
__global__ void collapse_kernel(CollapseArgs a, const uint2* __restrict__ items, uint32_t num_items,
                                uint2* __restrict__ next_items, uint32_t* __restrict__ next_count)
{
	const uint32_t it = blockIdx.x * blockDim.x + threadIdx.x;
	if(it >= num_items)
	{
		return;
	}
	const uint2 item = items[it];
	uint32_t child[8];
	float4 clo[8], chi[8];
	int k = 0;
	if(item.x & kLeafRef)
	{
		child[k++] = item.x;   // a lone triangle (one-triangle scenes)
	}
	else
	{
		child[k++] = a.left[item.x];
		child[k++] = a.right[item.x];
	}
	auto count = [&](uint32_t ref) { return (ref & kLeafRef) ? 1u : a.count_of[ref]; };
	for(int c = 0; c < k; ++c)
	{
		ref_box(child[c], a.plo, a.phi, a.sorted, a.nlo, a.nhi, &clo[c], &chi[c]);
	}
	// open the largest child that holds more than a leaf's worth of triangles
	while(k < 8)
	{
		int best = -1;
		float best_area = -1.0f;
		for(int c = 0; c < k; ++c)
		{
			if((child[c] & kLeafRef) || count(child[c]) <= kLeafMax)
			{
				continue;
			}
			const float dx = chi[c].x - clo[c].x, dy = chi[c].y - clo[c].y, dz = chi[c].z - clo[c].z;
			const float area = dx * dy + dy * dz + dz * dx;
			if(area > best_area)
			{
				best_area = area;
				best = c;
			}
		}
		if(best < 0)
		{
			break;
		}
		const uint32_t open = child[best];
		child[best] = a.left[open];
		child[k] = a.right[open];
		ref_box(child[best], a.plo, a.phi, a.sorted, a.nlo, a.nhi, &clo[best], &chi[best]);
		ref_box(child[k], a.plo, a.phi, a.sorted, a.nlo, a.nhi, &clo[k], &chi[k]);
		++k;
	}

	// octant slot assignment, as the host builder: slot bit a set <=> child centroid on the
	// negative side of the node centre along axis a, resolved greedily by best alignment
	float plo3[3] = {3.0e38f, 3.0e38f, 3.0e38f}, phi3[3] = {-3.0e38f, -3.0e38f, -3.0e38f};
	for(int c = 0; c < k; ++c)
	{
		plo3[0] = fminf(plo3[0], clo[c].x); plo3[1] = fminf(plo3[1], clo[c].y); plo3[2] = fminf(plo3[2], clo[c].z);
		phi3[0] = fmaxf(phi3[0], chi[c].x); phi3[1] = fmaxf(phi3[1], chi[c].y); phi3[2] = fmaxf(phi3[2], chi[c].z);
	}
	const float pc[3] = {0.5f * (plo3[0] + phi3[0]), 0.5f * (plo3[1] + phi3[1]), 0.5f * (plo3[2] + phi3[2])};
	int slot_of[8];
	uint32_t slot_used = 0, child_done = 0;
	for(int round = 0; round < k; ++round)
	{
		float best_score = -INFINITY;
		int bc = -1, bs = -1;
		for(int c = 0; c < k; ++c)
		{
			if((child_done >> c) & 1u)
			{
				continue;
			}
			const float d[3] = {0.5f * (clo[c].x + chi[c].x) - pc[0], 0.5f * (clo[c].y + chi[c].y) - pc[1],
			                    0.5f * (clo[c].z + chi[c].z) - pc[2]};
			for(int s = 0; s < 8; ++s)
			{
				if((slot_used >> s) & 1u)
				{
					continue;
				}
				float score = 0.0f;
				for(int ax = 0; ax < 3; ++ax)
				{
					score += ((s >> ax) & 1) ? -d[ax] : d[ax];
				}
				if(score > best_score || bc < 0)
				{
					best_score = score;
					bc = c;
					bs = s;
				}
			}
		}
		child_done |= 1u << bc;
		slot_used |= 1u << bs;
		slot_of[bc] = bs;
	}

	// quantisation frame over the padded child boxes
	float qlo3[3] = {3.0e38f, 3.0e38f, 3.0e38f}, qhi3[3] = {-3.0e38f, -3.0e38f, -3.0e38f};
	float blo[8][3], bhi[8][3];
	for(int c = 0; c < k; ++c)
	{
		const float l[3] = {clo[c].x, clo[c].y, clo[c].z}, h[3] = {chi[c].x, chi[c].y, chi[c].z};
		for(int ax = 0; ax < 3; ++ax)
		{
			blo[c][ax] = l[ax] - a.pad;
			bhi[c][ax] = h[ax] + a.pad;
			qlo3[ax] = fminf(qlo3[ax], blo[c][ax]);
			qhi3[ax] = fmaxf(qhi3[ax], bhi[c][ax]);
		}
	}
	WideNode node;
	for(int w = 0; w < 20; ++w)
	{
		node.w[w] = 0u;
	}
	int e[3];
	float scale[3];
	for(int ax = 0; ax < 3; ++ax)
	{
		const float extent = qhi3[ax] - qlo3[ax];
		// 254 quanta cover the extent, one spare quantum absorbs the rounding of p + q*s
		int ex = extent > 0.0f ? static_cast<int>(ceil(log2(static_cast<double>(extent) / 254.0))) : -126;
		ex = min(max(ex, -126), 127);
		while(ldexp(254.0, ex) < static_cast<double>(extent) && ex < 127)
		{
			++ex;
		}
		e[ax] = ex;
		scale[ax] = ldexpf(1.0f, ex);
		node.w[ax] = __float_as_uint(qlo3[ax]);
	}

	int child_at_slot[8];
	for(int s = 0; s < 8; ++s)
	{
		child_at_slot[s] = -1;
	}
	for(int c = 0; c < k; ++c)
	{
		child_at_slot[slot_of[c]] = c;
	}
	auto is_leaf_group = [&](uint32_t ref) { return (ref & kLeafRef) || count(ref) <= kLeafMax; };
	uint32_t imask = 0, num_internal = 0, total_tris = 0;
	for(int s = 0; s < 8; ++s)
	{
		const int c = child_at_slot[s];
		if(c < 0)
		{
			continue;
		}
		if(is_leaf_group(child[c]))
		{
			total_tris += count(child[c]);
		}
		else
		{
			imask |= 1u << s;
			++num_internal;
		}
	}
	const uint32_t child_base = num_internal ? atomicAdd(&a.counters[0], num_internal) : 0u;
	const uint32_t tri_base = total_tris ? atomicAdd(&a.counters[1], total_tris) : 0u;
	if(child_base + num_internal > a.node_capacity)
	{
		atomicOr(&a.counters[2], BUILD_ERR_NODE_OVERFLOW);
		return;
	}
	if(tri_base + total_tris > a.num_tris)
	{
		atomicOr(&a.counters[2], BUILD_ERR_TRI_OVERFLOW);
		return;
	}
	node.w[3] = static_cast<uint32_t>(e[0] + 127) | (static_cast<uint32_t>(e[1] + 127) << 8) |
	            (static_cast<uint32_t>(e[2] + 127) << 16) | (imask << 24);
	node.w[4] = child_base;
	node.w[5] = tri_base;

	uint32_t internal_rank = 0, tri_offset = 0;
	for(int s = 0; s < 8; ++s)
	{
		const int c = child_at_slot[s];
		if(c < 0)
		{
			continue;
		}
		const uint32_t ref = child[c];
		uint32_t meta;
		if(!is_leaf_group(ref))
		{
			meta = (1u << 5) | (24u + static_cast<uint32_t>(s));
			const uint32_t q = atomicAdd(next_count, 1u);
			next_items[q] = make_uint2(ref, child_base + internal_rank);
			++internal_rank;
		}
		else
		{
			// the subtree's (at most 3) triangles
			uint32_t leaves[kLeafMax], stack[2 * kLeafMax];
			uint32_t cnt = 0;
			int sp = 0;
			stack[sp++] = ref;
			while(sp > 0)
			{
				const uint32_t r = stack[--sp];
				if(r & kLeafRef)
				{
					if(cnt < kLeafMax) { leaves[cnt++] = r & ~kLeafRef; }
				}
				else if(sp + 2 <= static_cast<int>(2 * kLeafMax))
				{
					stack[sp++] = a.right[r];
					stack[sp++] = a.left[r];
				}
			}
			meta = (((1u << cnt) - 1u) << 5) | tri_offset;
			for(uint32_t t = 0; t < cnt; ++t)
			{
				const uint32_t p = a.sorted[leaves[t]];
				const float* v = a.tris + 9ull * p;
				LeafTri lt;
				lt.v0x = v[0]; lt.v0y = v[1]; lt.v0z = v[2]; lt.prim = p;
				lt.v1x = v[3]; lt.v1y = v[4]; lt.v1z = v[5]; lt.material = a.materials ? a.materials[p] : 0u;
				lt.v2x = v[6]; lt.v2y = v[7]; lt.v2z = v[8]; lt.emitter_plus_one = a.emitters ? a.emitters[p] : 0u;
				a.leaf_tris[tri_base + tri_offset + t] = lt;
			}
			tri_offset += cnt;
		}
		set_byte(node, 6 + s / 4, s % 4, meta);

		// conservative quantisation, verified in FP32 exactly as the traversal decodes
		for(int ax = 0; ax < 3; ++ax)
		{
			const float p = qlo3[ax];
			int ql = static_cast<int>(floorf((blo[c][ax] - p) / scale[ax]));
			int qh = static_cast<int>(ceilf((bhi[c][ax] - p) / scale[ax]));
			ql = max(0, min(255, ql));
			qh = max(0, min(255, qh));
			while(ql > 0 && p + static_cast<float>(ql) * scale[ax] > blo[c][ax])
			{
				--ql;
			}
			while(qh < 255 && p + static_cast<float>(qh) * scale[ax] < bhi[c][ax])
			{
				++qh;
			}
			set_byte(node, 8 + 2 * ax + s / 4, s % 4, static_cast<uint32_t>(ql));
			set_byte(node, 14 + 2 * ax + s / 4, s % 4, static_cast<uint32_t>(qh));
		}
	}
	a.nodes[item.y] = node;
}

int blocks_for(uint64_t n)
{
	return static_cast<int>(std::max<uint64_t>(1, std::min<uint64_t>((n + kBlock - 1) / kBlock, 65535u * 8u)));
}

}// end anonymous namespace

std::unique_ptr<Geometry> make_geometry_gpu(const BvhBuildInput& in)
{
	require_device();
	const auto t0 = std::chrono::steady_clock::now();
	if(!in.tris || in.num_tris == 0)
	{
		throw Error(PG_ERR_INVALID_ARGUMENT, "GPU BVH build: no triangles");
	}
	if(in.num_tris > (1u << 30))
	{
		throw Error(PG_ERR_INVALID_ARGUMENT, "GPU BVH build: more than 2^30 triangles");
	}
	const uint32_t n = static_cast<uint32_t>(in.num_tris);
	cudaStream_t s = library_stream();

	DeviceBuffer<float> d_tris(9ull * n);
	DeviceBuffer<uint32_t> d_mat, d_em;
	PG_CUDA_CHECK(cudaMemcpyAsync(d_tris.get(), in.tris, d_tris.bytes(), cudaMemcpyHostToDevice, s));
	if(in.materials)
	{
		d_mat.resize(n);
		PG_CUDA_CHECK(cudaMemcpyAsync(d_mat.get(), in.materials, d_mat.bytes(), cudaMemcpyHostToDevice, s));
	}
	if(in.emitters)
	{
		d_em.resize(n);
		PG_CUDA_CHECK(cudaMemcpyAsync(d_em.get(), in.emitters, d_em.bytes(), cudaMemcpyHostToDevice, s));
	}

	// 1. boxes, centroid bound, coordinate magnitude
	DeviceBuffer<float4> plo(n), phi(n);
	DeviceBuffer<float> stats(8);
	const float init_stats[8] = {3.0e38f, 3.0e38f, 3.0e38f, -3.0e38f, -3.0e38f, -3.0e38f, 0.0f, 0.0f};
	PG_CUDA_CHECK(cudaMemcpyAsync(stats.get(), init_stats, sizeof(init_stats), cudaMemcpyHostToDevice, s));
	prim_kernel<<<std::min(blocks_for(n), sm_count() * 8), kBlock, 0, s>>>(d_tris.get(), n, plo.get(), phi.get(), stats.get());
	PG_CUDA_CHECK(cudaGetLastError());

	// 2. Morton codes, sorted with their triangle indices
	DeviceBuffer<uint64_t> keys(n), keys_sorted(n);
	DeviceBuffer<uint32_t> idx(n), sorted(n);
	morton_kernel<<<std::min(blocks_for(n), sm_count() * 8), kBlock, 0, s>>>(plo.get(), phi.get(), n, stats.get(),
	                                                                      keys.get(), idx.get());
	PG_CUDA_CHECK(cudaGetLastError());
	std::size_t temp_bytes = 0;
	PG_CUDA_CHECK(cub::DeviceRadixSort::SortPairs(nullptr, temp_bytes, keys.get(), keys_sorted.get(), idx.get(),
	                                              sorted.get(), static_cast<int>(n), 0, 63, s));
	DeviceBuffer<unsigned char> temp(std::max<std::size_t>(temp_bytes, 16));
	PG_CUDA_CHECK(cub::DeviceRadixSort::SortPairs(temp.get(), temp_bytes, keys.get(), keys_sorted.get(), idx.get(),
	                                              sorted.get(), static_cast<int>(n), 0, 63, s));

	// 3. the binary tree by locally-ordered clustering
	const uint32_t ni = n > 1 ? n - 1 : 1;
	DeviceBuffer<uint32_t> left(ni), right(ni), count_of(ni);
	DeviceBuffer<float4> nlo(ni), nhi(ni);
	DeviceBuffer<uint32_t> clusters[2] = {DeviceBuffer<uint32_t>(n), DeviceBuffer<uint32_t>(n)};
	DeviceBuffer<uint32_t> nn(n), merged(n), ploc_state(3);   // [0] next internal node, [1] selected, [2] errors
	DeviceBuffer<uint8_t> keep(n);
	PG_CUDA_CHECK(cudaMemsetAsync(ploc_state.get(), 0, ploc_state.bytes(), s));
	leaf_refs_kernel<<<std::min(blocks_for(n), sm_count() * 8), kBlock, 0, s>>>(n, clusters[0].get());
	PG_CUDA_CHECK(cudaGetLastError());
	std::size_t select_bytes = 0;
	PG_CUDA_CHECK(cub::DeviceSelect::Flagged(nullptr, select_bytes, merged.get(), keep.get(), clusters[1].get(),
	                                         ploc_state.get() + 1, static_cast<int>(n), s));
	DeviceBuffer<unsigned char> select_temp(std::max<std::size_t>(select_bytes, 16));
	uint32_t m = n;
	int cur = 0;
	for(int pass = 0; m > 1; ++pass)
	{
		if(pass > 100000)
		{
			throw Error(PG_ERR_SCENE, "GPU BVH build: clustering did not converge");
		}
		ploc_neighbour_kernel<<<(m + kPlocBlock - 1) / kPlocBlock, kPlocBlock, 0, s>>>(
			clusters[cur].get(), m, sorted.get(), plo.get(), phi.get(), nlo.get(), nhi.get(), nn.get());
		PG_CUDA_CHECK(cudaGetLastError());
		ploc_merge_kernel<<<std::min(blocks_for(m), sm_count() * 8), kBlock, 0, s>>>(
			clusters[cur].get(), m, nn.get(), sorted.get(), plo.get(), phi.get(), ploc_state.get(), left.get(),
			right.get(), count_of.get(), nlo.get(), nhi.get(), merged.get(), keep.get(), ni, ploc_state.get() + 2);
		PG_CUDA_CHECK(cudaGetLastError());
		PG_CUDA_CHECK(cub::DeviceSelect::Flagged(select_temp.get(), select_bytes, merged.get(), keep.get(),
		                                         clusters[1 - cur].get(), ploc_state.get() + 1, static_cast<int>(m), s));
		uint32_t state[3];
		PG_CUDA_CHECK(cudaMemcpyAsync(state, ploc_state.get(), sizeof(state), cudaMemcpyDeviceToHost, s));
		PG_CUDA_CHECK(cudaStreamSynchronize(s));
		if(state[2] != 0u || state[1] >= m)
		{
			throw Error(PG_ERR_SCENE, "GPU BVH build: clustering made no progress");
		}
		m = state[1];
		cur = 1 - cur;
	}
	uint32_t root_ref = kLeafRef;
	PG_CUDA_CHECK(cudaMemcpyAsync(&root_ref, clusters[cur].get(), sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
	float h_stats[8];
	PG_CUDA_CHECK(cudaMemcpyAsync(h_stats, stats.get(), sizeof(h_stats), cudaMemcpyDeviceToHost, s));
	PG_CUDA_CHECK(cudaStreamSynchronize(s));
	const float max_abs = std::max(std::max(in.max_origin_abs, 1.0f), h_stats[6]);

	// 5. collapse, level by level
	auto g = std::make_unique<Geometry>();
	g->device = current_device();
	const uint32_t node_capacity = n + 1;
	g->nodes.resize(node_capacity);
	g->tris.resize(n);
	DeviceBuffer<uint32_t> counters(3);
	const uint32_t init_counters[3] = {1u, 0u, 0u};   // the root occupies node 0
	PG_CUDA_CHECK(cudaMemcpyAsync(counters.get(), init_counters, sizeof(init_counters), cudaMemcpyHostToDevice, s));
	DeviceBuffer<uint2> items[2] = {DeviceBuffer<uint2>(node_capacity), DeviceBuffer<uint2>(node_capacity)};
	DeviceBuffer<uint32_t> next_count(1);
	const uint2 root = make_uint2(root_ref, 0u);
	PG_CUDA_CHECK(cudaMemcpyAsync(items[0].get(), &root, sizeof(root), cudaMemcpyHostToDevice, s));

	CollapseArgs args{d_tris.get(), in.materials ? d_mat.get() : nullptr, in.emitters ? d_em.get() : nullptr,
	                  sorted.get(), plo.get(), phi.get(), nlo.get(), nhi.get(), left.get(), right.get(),
	                  count_of.get(), g->nodes.get(), g->tris.get(), node_capacity, n,
	                  4.0e-6f * max_abs, counters.get()};
	uint32_t count = 1;
	int depth = 0;
	while(count > 0)
	{
		++depth;
		if(depth >= kTraversalStackSize)
		{
			throw Error(PG_ERR_SCENE, "GPU BVH build: tree deeper than the traversal stack");
		}
		PG_CUDA_CHECK(cudaMemsetAsync(next_count.get(), 0, sizeof(uint32_t), s));
		collapse_kernel<<<(count + 127) / 128, 128, 0, s>>>(args, items[(depth - 1) & 1].get(), count,
		                                                    items[depth & 1].get(), next_count.get());
		PG_CUDA_CHECK(cudaGetLastError());
		PG_CUDA_CHECK(cudaMemcpyAsync(&count, next_count.get(), sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
		PG_CUDA_CHECK(cudaStreamSynchronize(s));
	}
	uint32_t used[3];
	PG_CUDA_CHECK(cudaMemcpyAsync(used, counters.get(), sizeof(used), cudaMemcpyDeviceToHost, s));
	g->error.resize(1);
	PG_CUDA_CHECK(cudaMemsetAsync(g->error.get(), 0, sizeof(uint32_t), s));
	g->fetch.resize(1);
	PG_CUDA_CHECK(cudaStreamSynchronize(s));
	if(used[2] != 0u || used[1] != n)
	{
		throw Error(PG_ERR_SCENE, "GPU BVH build failed (flags " + std::to_string(used[2]) + ", " +
		                          std::to_string(used[1]) + " of " + std::to_string(n) + " triangles placed)");
	}
	g->stats.num_nodes = used[0];
	g->stats.num_leaf_tris = used[1];
	g->stats.max_depth = depth;
	g->stats.box_padding = 4.0e-6f * max_abs;
	g->stats.build_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
	return g;
}

}// end namespace pg
