// Geometry objects (triangles + compressed 8-wide BVH in HBM) and the ray-query entry points of
// the C ABI (include/photon_gpu.h): closest hit, occlusion, and the counting pass.
#include "pg_geometry.h"
#include "pg_render.h"
#include "trace.cuh"

#include "../../include/photon_gpu.h"

#include <algorithm>
#include <map>
#include <mutex>
#include <string>
#include <vector>

namespace pg
{

Registry<Geometry>& geometry_registry()
{
	static Registry<Geometry> r;
	return r;
}

std::unique_ptr<Geometry> make_geometry(const BvhBuildInput& in)
{
	require_device();
	auto g = std::make_unique<Geometry>();
	g->device = current_device();
	WideBvh bvh = build_wide_bvh(in);
	g->stats = bvh.stats;
	g->nodes.resize(bvh.nodes.size());
	g->tris.resize(bvh.tris.size());
	cudaStream_t s = library_stream();
	PG_CUDA_CHECK(cudaMemcpyAsync(g->nodes.get(), bvh.nodes.data(), g->nodes.bytes(), cudaMemcpyHostToDevice, s));
	PG_CUDA_CHECK(cudaMemcpyAsync(g->tris.get(), bvh.tris.data(), g->tris.bytes(), cudaMemcpyHostToDevice, s));
	g->error.resize(1);
	PG_CUDA_CHECK(cudaMemsetAsync(g->error.get(), 0, sizeof(uint32_t), s));
	g->fetch.resize(1);
	PG_CUDA_CHECK(cudaStreamSynchronize(s));
	return g;
}

namespace
{

constexpr int kTraceBlock = kTraversalBlock;
// Resident blocks per SM the traversal kernels are compiled for: 8 x 128 threads at 64 registers
// fill the register file (a larger register budget leaves room for 7 blocks only).
constexpr int kTraceMinBlocks = 8;

struct HitRecord
{
	uint32_t tri;
	float    t;
};

__global__ void __launch_bounds__(kTraceBlock, kTraceMinBlocks)
trace_closest_kernel(const WideNode* __restrict__ nodes, const LeafTri* __restrict__ tris,
                     const float4* __restrict__ rays, uint32_t n, uint32_t* __restrict__ next_ray,
                     HitRecord* __restrict__ hits, uint32_t* __restrict__ error)
{
	uint32_t err = 0;
	traverse_persistent<false, false>(nodes, tris, n, next_ray,
		[&](uint32_t i, float4* a, float4* b) { *a = __ldg(rays + 2 * i); *b = __ldg(rays + 2 * i + 1); },
		[&](uint32_t i, bool hit, uint32_t tri, float t) { hits[i] = HitRecord{hit ? tri : 0xFFFFFFFFu, hit ? t : 0.0f}; },
		&err);
	if(err)
	{
		atomicOr(error, err);
	}
}

__global__ void __launch_bounds__(kTraceBlock, kTraceMinBlocks)
trace_any_kernel(const WideNode* __restrict__ nodes, const LeafTri* __restrict__ tris,
                 const float4* __restrict__ rays, uint32_t n, uint32_t* __restrict__ next_ray,
                 int32_t* __restrict__ occluded, uint32_t* __restrict__ error)
{
	uint32_t err = 0;
	traverse_persistent<true, false>(nodes, tris, n, next_ray,
		[&](uint32_t i, float4* a, float4* b) { *a = __ldg(rays + 2 * i); *b = __ldg(rays + 2 * i + 1); },
		[&](uint32_t i, bool hit, uint32_t, float) { occluded[i] = hit ? 1 : 0; },
		&err);
	if(err)
	{
		atomicOr(error, err);
	}
}

// Re-runs the winning triangle's test to report the reference-facing results: primitive index in
// input order and the barycentrics (identical arithmetic, so identical bits).
__global__ void resolve_hits_kernel(const LeafTri* __restrict__ tris, const float4* __restrict__ rays,
                                    const HitRecord* __restrict__ hits, uint64_t n,
                                    int32_t* __restrict__ prim, float* __restrict__ t_out,
                                    float* __restrict__ bary)
{
	const uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
	if(i >= n)
	{
		return;
	}
	const HitRecord h = hits[i];
	if(h.tri == 0xFFFFFFFFu)
	{
		prim[i] = -1;
		t_out[i] = 0.0f;
		bary[3 * i + 0] = bary[3 * i + 1] = bary[3 * i + 2] = 0.0f;
		return;
	}
	const float4 a = rays[2 * i];
	const float4 b = rays[2 * i + 1];
	const RayTraits r = make_ray_traits(a.x, a.y, a.z, b.x, b.y, b.z);
	float t, b0, b1, b2;
	// The winning triangle passed with some maxT >= its t, so it passes again with the ray's own
	// range and yields the same bits.
	watertight_hit_tri(r, tris, h.tri, a.w, b.w, &t, &b0, &b1, &b2);
	prim[i] = static_cast<int32_t>(tris[h.tri].prim);
	t_out[i] = h.t;
	bary[3 * i + 0] = b0;
	bary[3 * i + 1] = b1;
	bary[3 * i + 2] = b2;
}

__global__ void count_kernel(const WideNode* __restrict__ nodes, const LeafTri* __restrict__ tris,
                             const float4* __restrict__ rays, uint64_t n, int any_hit,
                             unsigned long long* __restrict__ sums, uint32_t* __restrict__ error)
{
	const uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
	uint32_t nodes_visited = 0, tris_tested = 0, err = 0;
	if(i < n)
	{
		const float4 a = rays[2 * i];
		const float4 b = rays[2 * i + 1];
		const RayTraits r = make_ray_traits(a.x, a.y, a.z, b.x, b.y, b.z);
		float t;
		uint32_t tri;
		if(any_hit)
		{
			traverse<true, true>(r, nodes, tris, a.w, b.w, &t, &tri, &err, &nodes_visited, &tris_tested);
		}
		else
		{
			traverse<false, true>(r, nodes, tris, a.w, b.w, &t, &tri, &err, &nodes_visited, &tris_tested);
		}
	}
	atomicAdd(&sums[0], static_cast<unsigned long long>(nodes_visited));
	atomicAdd(&sums[1], static_cast<unsigned long long>(tris_tested));
	if(err)
	{
		atomicOr(error, err);
	}
}

// Persistent grid: as many blocks as stay resident on the current device at once, computed once
// per (kernel, device).
template<class Kernel>
int persistent_grid(Kernel kernel)
{
	static std::mutex mutex;
	static std::map<std::pair<const void*, int>, int> cache;
	const int dev = current_device();
	const auto key = std::make_pair(reinterpret_cast<const void*>(kernel), dev);
	std::lock_guard<std::mutex> lock(mutex);
	const auto it = cache.find(key);
	if(it != cache.end())
	{
		return it->second;
	}
	int per_sm = 0;
	PG_CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kTraceBlock, 0));
	const int grid = std::max(1, per_sm) * sm_count();
	cache.emplace(key, grid);
	return grid;
}

uint32_t checked_ray_count(uint64_t n)
{
	if(n > 0xFFF00000ull)
	{
		throw Error(PG_ERR_INVALID_ARGUMENT, "too many rays in one call: " + std::to_string(n));
	}
	return static_cast<uint32_t>(n);
}

std::shared_ptr<Geometry> get_geometry(uint64_t id)
{
	auto g = geometry_registry().get(id);
	if(!g)
	{
		throw Error(PG_ERR_NOT_FOUND, "unknown geometry id " + std::to_string(id));
	}
	require_same_device(g->device, ("geometry " + std::to_string(id)).c_str());
	return g;
}

void check_device_error(Geometry& g, cudaStream_t s)
{
	uint32_t flags = 0;
	PG_CUDA_CHECK(cudaMemcpyAsync(&flags, g.error.get(), sizeof(flags), cudaMemcpyDeviceToHost, s));
	PG_CUDA_CHECK(cudaStreamSynchronize(s));
	if(flags & PG_DEV_ERR_STACK)
	{
		PG_CUDA_CHECK(cudaMemsetAsync(g.error.get(), 0, sizeof(uint32_t), s));
		throw Error(PG_ERR_STACK_OVERFLOW, "BVH traversal stack overflow");
	}
}

// An unoccluded NEE contribution (shadow record i): to the owning path's radiance (slot in the
// path buffer the record was made for) or, for paths that ended at that vertex, straight to the
// FP64 film; guided renders also credit the training sample the record belongs to.
__device__ __forceinline__ void add_unoccluded(uint32_t i, const float4* __restrict__ sc,
                                               const float4* __restrict__ st, const float2* __restrict__ sr,
                                               float4* __restrict__ rad_target, const FilmView& film,
                                               float4* __restrict__ train_dirw)
{
	if(train_dirw)
	{
		const float4 tr = __ldg(st + i);
		const uint32_t row = __float_as_uint(tr.x), nee_row = __float_as_uint(tr.z);
		if(row != 0xFFFFFFFFu && tr.y != 0.0f)
		{
			atomicAdd(&train_dirw[row].w, tr.y);
		}
		if(nee_row != 0xFFFFFFFFu && tr.w != 0.0f)
		{
			atomicAdd(&train_dirw[nee_row].w, tr.w);
		}
	}
	const float4 c = __ldg(sc + i);
	const uint32_t target = __float_as_uint(c.w);
	if(target & kTargetFinal)
	{
		if(film.filter == PG_FILTER_BOX)
		{
			film_add_box(film, target & ~kTargetFinal, c.x, c.y, c.z);
		}
		else
		{
			// the path already stored its radiance in its sample slot (it ended in an earlier
			// kernel); each path has at most one such contribution
			float4* s = film.samples + __float_as_uint(__ldg(sr + i).x);
			float4 v = *s;
			v.x += c.x;
			v.y += c.y;
			v.z += c.z;
			*s = v;
		}
	}
	else
	{
		float4 rv = rad_target[target];
		rv.x += c.x;
		rv.y += c.y;
		rv.z += c.z;
		rad_target[target] = rv;
	}
}

// One launch for both traversal queues of an iteration: the closest hits of this iteration's
// rays, then the visibility of the previous iteration's NEE segments, whose owning paths sit in
// this iteration's path buffer (their radiance is read by this iteration's shading, after this
// kernel). A single dynamic-fetch cursor runs over both queues, so the launch has one tail.
// MULTI: the rays belong to the scenes of `batch` (a closest-hit ray's scene in the top bits of its
// path's meta word, a NEE segment's in its record's sid); each ray walks its own scene's tree and
// a final contribution goes to its own scene's film.
template<bool COUNT, bool MULTI>
__global__ void __launch_bounds__(kTraceBlock, kTraceMinBlocks)
trace_kernel(const WideNode* __restrict__ nodes, const LeafTri* __restrict__ tris,
             RenderCounters* __restrict__ counters,
             const float4* __restrict__ ray_o, const float4* __restrict__ ray_d, uint2* __restrict__ hits,
             const float4* __restrict__ so, const float4* __restrict__ sd, const float4* __restrict__ sc,
             const float2* __restrict__ sr, float4* __restrict__ rad_cur, FilmView film, int min_idle,
             const uint32_t* __restrict__ meta, const uint32_t* __restrict__ shadow_sid, BatchView batch,
             const float4* __restrict__ st, float4* __restrict__ train_dirw)
{
	const uint32_t n_closest = counters->n_total;
	const uint32_t n_shadow = counters->n_shadow_prev;
	if(blockIdx.x == 0 && threadIdx.x == 0)
	{
		counters->shadow_rays += n_shadow;
	}
	auto scene_of = [&](uint32_t i) -> uint32_t
	{
		return i < n_closest ? __ldg(meta + i) >> kMetaSceneShift : __ldg(shadow_sid + (i - n_closest));
	};
	auto fetch_ray = [&](uint32_t i, float4* a, float4* b)
	{
		if(i < n_closest)
		{
			*a = __ldg(ray_o + i);
			*b = __ldg(ray_d + i);
		}
		else
		{
			*a = __ldg(so + (i - n_closest));
			*b = __ldg(sd + (i - n_closest));
		}
	};
	auto finish = [&](uint32_t i, bool hit, uint32_t tri, float t)
	{
		if(i < n_closest)
		{
			hits[i] = make_uint2(hit ? tri : 0xFFFFFFFFu, __float_as_uint(t));
		}
		else if(!hit)
		{
			if constexpr(MULTI)
			{
				add_unoccluded(i - n_closest, sc, nullptr, sr, rad_cur, batch.scenes[scene_of(i)].film, nullptr);
			}
			else
			{
				add_unoccluded(i - n_closest, sc, st, sr, rad_cur, film, train_dirw);
			}
		}
	};
	uint32_t err = 0, node_count[2] = {0u, 0u}, tri_count[2] = {0u, 0u};
	if constexpr(MULTI)
	{
		traverse_persistent<false, COUNT, true, true>(nodes, tris, n_closest + n_shadow, &counters->fetch_extend,
			[&](uint32_t i, float4* a, float4* b, const WideNode** ln, const LeafTri** lt)
			{
				fetch_ray(i, a, b);
				const DeviceScene& s = batch.scenes[scene_of(i)].scene;
				*ln = s.nodes;
				*lt = s.tris;
			},
			finish, &err, node_count, tri_count, n_closest, min_idle);
	}
	else
	{
		traverse_persistent<false, COUNT, true>(nodes, tris, n_closest + n_shadow, &counters->fetch_extend,
			fetch_ray, finish, &err, node_count, tri_count, n_closest, min_idle);
	}
	if(COUNT)
	{
		atomicAdd(&counters->nodes_closest, static_cast<unsigned long long>(node_count[0]));
		atomicAdd(&counters->tris_closest, static_cast<unsigned long long>(tri_count[0]));
		atomicAdd(&counters->nodes_any, static_cast<unsigned long long>(node_count[1]));
		atomicAdd(&counters->tris_any, static_cast<unsigned long long>(tri_count[1]));
	}
	if(err)
	{
		atomicOr(&counters->error, err);
	}
}

}// end anonymous namespace

void launch_trace(const DeviceScene& s, RenderCounters* counters, const float4* ray_o, const float4* ray_d,
                  uint2* hits, const ShadowQueue& prev, float4* rad_cur, const FilmView& film, int min_idle,
                  cudaStream_t st, bool count, const uint32_t* meta, const BatchView* batch, float4* train_dirw)
{
	if(batch)
	{
		if(count)
		{
			const int grid = persistent_grid(trace_kernel<true, true>);
			trace_kernel<true, true><<<grid, kTraceBlock, 0, st>>>(s.nodes, s.tris, counters, ray_o, ray_d, hits,
				prev.o, prev.d, prev.c, prev.r, rad_cur, film, min_idle, meta, prev.sid, *batch, nullptr, nullptr);
		}
		else
		{
			const int grid = persistent_grid(trace_kernel<false, true>);
			trace_kernel<false, true><<<grid, kTraceBlock, 0, st>>>(s.nodes, s.tris, counters, ray_o, ray_d, hits,
				prev.o, prev.d, prev.c, prev.r, rad_cur, film, min_idle, meta, prev.sid, *batch, nullptr, nullptr);
		}
	}
	else if(count)
	{
		const int grid = persistent_grid(trace_kernel<true, false>);
		trace_kernel<true, false><<<grid, kTraceBlock, 0, st>>>(s.nodes, s.tris, counters, ray_o, ray_d, hits,
			prev.o, prev.d, prev.c, prev.r, rad_cur, film, min_idle, nullptr, nullptr, BatchView{},
			train_dirw ? prev.t : nullptr, train_dirw);
	}
	else
	{
		const int grid = persistent_grid(trace_kernel<false, false>);
		trace_kernel<false, false><<<grid, kTraceBlock, 0, st>>>(s.nodes, s.tris, counters, ray_o, ray_d, hits,
			prev.o, prev.d, prev.c, prev.r, rad_cur, film, min_idle, nullptr, nullptr, BatchView{},
			train_dirw ? prev.t : nullptr, train_dirw);
	}
	PG_CUDA_CHECK(cudaGetLastError());
}

void launch_trace_closest(const Geometry& g, const float* d_rays, uint64_t n, void* d_hits, cudaStream_t s)
{
	if(n == 0)
	{
		return;
	}
	const int grid = persistent_grid(trace_closest_kernel);
	PG_CUDA_CHECK(cudaMemsetAsync(g.fetch.get(), 0, sizeof(uint32_t), s));
	trace_closest_kernel<<<grid, kTraceBlock, 0, s>>>(
		g.nodes.get(), g.tris.get(), reinterpret_cast<const float4*>(d_rays), checked_ray_count(n),
		g.fetch.get(), reinterpret_cast<HitRecord*>(d_hits), g.error.get());
	PG_CUDA_CHECK(cudaGetLastError());
}

void launch_trace_any(const Geometry& g, const float* d_rays, uint64_t n, int32_t* d_occluded, cudaStream_t s)
{
	if(n == 0)
	{
		return;
	}
	const int grid = persistent_grid(trace_any_kernel);
	PG_CUDA_CHECK(cudaMemsetAsync(g.fetch.get(), 0, sizeof(uint32_t), s));
	trace_any_kernel<<<grid, kTraceBlock, 0, s>>>(
		g.nodes.get(), g.tris.get(), reinterpret_cast<const float4*>(d_rays), checked_ray_count(n),
		g.fetch.get(), d_occluded, g.error.get());
	PG_CUDA_CHECK(cudaGetLastError());
}

}// end namespace pg

using namespace pg;

extern "C" {

const char* pgpu_last_error(void)
{
	return pg::last_error();
}

int pgpu_device_count(void)
{
	int n = 0;
	if(cudaGetDeviceCount(&n) != cudaSuccess)
	{
		cudaGetLastError();
		return 0;
	}
	return n;
}

int pgpu_geometry_create(const float* tris, uint64_t num_tris, float max_origin_abs, uint64_t* out_id)
{
	return pgpu_geometry_create_ex(tris, num_tris, max_origin_abs, PG_BVH_HOST_SAH, out_id);
}

int pgpu_geometry_create_ex(const float* tris, uint64_t num_tris, float max_origin_abs, uint32_t bvh_builder,
                            uint64_t* out_id)
{
	return guarded([&]
	{
		if(!tris || num_tris == 0 || !out_id)
		{
			throw Error(PG_ERR_INVALID_ARGUMENT, "pgpu_geometry_create: empty input");
		}
		if(bvh_builder > PG_BVH_GPU_MORTON)
		{
			throw Error(PG_ERR_INVALID_ARGUMENT, "pgpu_geometry_create_ex: unknown BVH builder");
		}
		BvhBuildInput in{tris, nullptr, nullptr, static_cast<std::size_t>(num_tris), max_origin_abs};
		*out_id = geometry_registry().add(bvh_builder == PG_BVH_GPU_MORTON ? make_geometry_gpu(in) : make_geometry(in));
	});
}

int pgpu_geometry_export(uint64_t id, void* out_nodes, void* out_tris, uint64_t* out_num_nodes, uint64_t* out_num_tris)
{
	return guarded([&]
	{
		auto g = get_geometry(id);
		const uint64_t nn = g->stats.num_nodes, nt = g->stats.num_leaf_tris;
		if(out_num_nodes) { *out_num_nodes = nn; }
		if(out_num_tris) { *out_num_tris = nt; }
		cudaStream_t s = library_stream();
		if(out_nodes)
		{
			PG_CUDA_CHECK(cudaMemcpyAsync(out_nodes, g->nodes.get(), nn * sizeof(WideNode), cudaMemcpyDeviceToHost, s));
		}
		if(out_tris)
		{
			PG_CUDA_CHECK(cudaMemcpyAsync(out_tris, g->tris.get(), nt * sizeof(LeafTri), cudaMemcpyDeviceToHost, s));
		}
		PG_CUDA_CHECK(cudaStreamSynchronize(s));
	});
}

int pgpu_geometry_destroy(uint64_t id)
{
	return guarded([&]
	{
		if(!geometry_registry().remove(id))
		{
			throw Error(PG_ERR_NOT_FOUND, "unknown geometry id " + std::to_string(id));
		}
	});
}

int pgpu_geometry_stats(uint64_t id, uint64_t* out_num_nodes, uint64_t* out_num_tris,
                        int32_t* out_max_depth, double* out_build_seconds)
{
	return guarded([&]
	{
		auto g = get_geometry(id);
		if(out_num_nodes) { *out_num_nodes = g->stats.num_nodes; }
		if(out_num_tris) { *out_num_tris = g->stats.num_leaf_tris; }
		if(out_max_depth) { *out_max_depth = g->stats.max_depth; }
		if(out_build_seconds) { *out_build_seconds = g->stats.build_seconds; }
	});
}

int pgpu_trace_closest(uint64_t id, const float* rays, uint64_t n,
                       int32_t* out_prim, float* out_t, float* out_bary)
{
	return guarded([&]
	{
		if(!rays && n > 0)
		{
			throw Error(PG_ERR_INVALID_ARGUMENT, "pgpu_trace_closest: null rays");
		}
		auto g = get_geometry(id);
		if(n == 0)
		{
			return;
		}
		cudaStream_t s = library_stream();
		DeviceBuffer<float> d_rays(n * 8);
		DeviceBuffer<HitRecord> d_hits(n);
		DeviceBuffer<int32_t> d_prim(n);
		DeviceBuffer<float> d_t(n), d_bary(3 * n);
		PG_CUDA_CHECK(cudaMemcpyAsync(d_rays.get(), rays, d_rays.bytes(), cudaMemcpyHostToDevice, s));
		launch_trace_closest(*g, d_rays.get(), n, d_hits.get(), s);
		resolve_hits_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, s>>>(
			g->tris.get(), reinterpret_cast<const float4*>(d_rays.get()), d_hits.get(), n,
			d_prim.get(), d_t.get(), d_bary.get());
		PG_CUDA_CHECK(cudaGetLastError());
		std::vector<int32_t> prim(n);
		std::vector<float> t(n), bary(3 * n);
		PG_CUDA_CHECK(cudaMemcpyAsync(prim.data(), d_prim.get(), d_prim.bytes(), cudaMemcpyDeviceToHost, s));
		PG_CUDA_CHECK(cudaMemcpyAsync(t.data(), d_t.get(), d_t.bytes(), cudaMemcpyDeviceToHost, s));
		PG_CUDA_CHECK(cudaMemcpyAsync(bary.data(), d_bary.get(), d_bary.bytes(), cudaMemcpyDeviceToHost, s));
		PG_CUDA_CHECK(cudaStreamSynchronize(s));
		check_device_error(*g, s);
		if(out_prim) { std::copy(prim.begin(), prim.end(), out_prim); }
		if(out_t) { std::copy(t.begin(), t.end(), out_t); }
		if(out_bary) { std::copy(bary.begin(), bary.end(), out_bary); }
	});
}

int pgpu_trace_any(uint64_t id, const float* rays, uint64_t n, int32_t* out_occluded)
{
	return guarded([&]
	{
		if((!rays || !out_occluded) && n > 0)
		{
			throw Error(PG_ERR_INVALID_ARGUMENT, "pgpu_trace_any: null pointer");
		}
		auto g = get_geometry(id);
		if(n == 0)
		{
			return;
		}
		cudaStream_t s = library_stream();
		DeviceBuffer<float> d_rays(n * 8);
		DeviceBuffer<int32_t> d_occ(n);
		PG_CUDA_CHECK(cudaMemcpyAsync(d_rays.get(), rays, d_rays.bytes(), cudaMemcpyHostToDevice, s));
		launch_trace_any(*g, d_rays.get(), n, d_occ.get(), s);
		PG_CUDA_CHECK(cudaMemcpyAsync(out_occluded, d_occ.get(), d_occ.bytes(), cudaMemcpyDeviceToHost, s));
		PG_CUDA_CHECK(cudaStreamSynchronize(s));
		check_device_error(*g, s);
	});
}

int pgpu_trace_closest_device(uint64_t id, const float* d_rays, uint64_t n, void* d_hits, float* out_ms)
{
	return guarded([&]
	{
		auto g = get_geometry(id);
		cudaStream_t s = library_stream();
		ScopedEvent e0, e1;
		PG_CUDA_CHECK(cudaEventRecord(e0.get(), s));
		launch_trace_closest(*g, d_rays, n, d_hits, s);
		PG_CUDA_CHECK(cudaEventRecord(e1.get(), s));
		PG_CUDA_CHECK(cudaEventSynchronize(e1.get()));
		float ms = 0.0f;
		PG_CUDA_CHECK(cudaEventElapsedTime(&ms, e0.get(), e1.get()));
		check_device_error(*g, s);
		if(out_ms) { *out_ms = ms; }
	});
}

int pgpu_trace_any_device(uint64_t id, const float* d_rays, uint64_t n, int32_t* d_occluded, float* out_ms)
{
	return guarded([&]
	{
		auto g = get_geometry(id);
		cudaStream_t s = library_stream();
		ScopedEvent e0, e1;
		PG_CUDA_CHECK(cudaEventRecord(e0.get(), s));
		launch_trace_any(*g, d_rays, n, d_occluded, s);
		PG_CUDA_CHECK(cudaEventRecord(e1.get(), s));
		PG_CUDA_CHECK(cudaEventSynchronize(e1.get()));
		float ms = 0.0f;
		PG_CUDA_CHECK(cudaEventElapsedTime(&ms, e0.get(), e1.get()));
		check_device_error(*g, s);
		if(out_ms) { *out_ms = ms; }
	});
}

int pgpu_trace_counts(uint64_t id, const float* rays, uint64_t n, int any_hit,
                      double* out_nodes_per_ray, double* out_tris_per_ray)
{
	return guarded([&]
	{
		auto g = get_geometry(id);
		if(n == 0 || !rays)
		{
			throw Error(PG_ERR_INVALID_ARGUMENT, "pgpu_trace_counts: no rays");
		}
		cudaStream_t s = library_stream();
		DeviceBuffer<float> d_rays(n * 8);
		DeviceBuffer<unsigned long long> d_sums(2);
		PG_CUDA_CHECK(cudaMemcpyAsync(d_rays.get(), rays, d_rays.bytes(), cudaMemcpyHostToDevice, s));
		PG_CUDA_CHECK(cudaMemsetAsync(d_sums.get(), 0, d_sums.bytes(), s));
		count_kernel<<<static_cast<unsigned>((n + 127) / 128), 128, 0, s>>>(
			g->nodes.get(), g->tris.get(), reinterpret_cast<const float4*>(d_rays.get()), n, any_hit,
			d_sums.get(), g->error.get());
		PG_CUDA_CHECK(cudaGetLastError());
		unsigned long long sums[2] = {0, 0};
		PG_CUDA_CHECK(cudaMemcpyAsync(sums, d_sums.get(), sizeof(sums), cudaMemcpyDeviceToHost, s));
		PG_CUDA_CHECK(cudaStreamSynchronize(s));
		check_device_error(*g, s);
		if(out_nodes_per_ray) { *out_nodes_per_ray = static_cast<double>(sums[0]) / n; }
		if(out_tris_per_ray) { *out_tris_per_ray = static_cast<double>(sums[1]) / n; }
	});
}

}// extern "C"

/* ---------------------------------------------------------------------------------------------
 * Closest hit that allocates nothing: pgpu_trace_closest_noalloc.
 *
 * pgpu_trace_closest stages rays and results in device buffers it allocates and frees per call.
 * Some callers cannot afford that at the moment they query a few hits: a host thread working under
 * a fixed device-memory budget that is already spent (a renderer that has sized its path state to
 * fill HBM), or one that must not stall -- cudaFree waits for all work queued on the device, so a
 * per-call free serialises the query behind whatever else the device is running. This variant
 * runs the same two kernels (traversal, then the resolve pass that reports prim / t /
 * barycentrics) on staging space carved from one statically sized device array per device.
 *
 * Scratch layout (kNoAllocMaxRays slots each, offsets multiples of 256 bytes): rays float4[2 n],
 * hit records {u32, f32}[n], prim i32[n], t f32[n], barycentrics f32[3 n]. Nothing in it has to
 * start at zero: every slot a call reads (i < n) is written earlier in the same call -- rays by the
 * host-to-device copy, hit records by the traversal kernel, results by the resolve kernel.
 * ------------------------------------------------------------------------------------------- */

namespace
{

constexpr uint64_t kNoAllocMaxRays = uint64_t(1) << 16;
constexpr size_t kNoAllocRaysOffset = 0;
constexpr size_t kNoAllocHitsOffset = kNoAllocRaysOffset + kNoAllocMaxRays * 32;
constexpr size_t kNoAllocPrimOffset = kNoAllocHitsOffset + kNoAllocMaxRays * sizeof(HitRecord);
constexpr size_t kNoAllocTOffset = kNoAllocPrimOffset + kNoAllocMaxRays * 4;
constexpr size_t kNoAllocBaryOffset = kNoAllocTOffset + kNoAllocMaxRays * 4;
constexpr size_t kNoAllocScratchBytes = kNoAllocBaryOffset + kNoAllocMaxRays * 12;   // 3.75 MiB
static_assert(sizeof(HitRecord) == 8, "scratch layout assumes 8-byte hit records");
static_assert(kNoAllocHitsOffset % 256 == 0 && kNoAllocPrimOffset % 256 == 0 &&
              kNoAllocTOffset % 256 == 0 && kNoAllocBaryOffset % 256 == 0, "scratch offsets");

constexpr int kNoAllocMaxDevices = 64;

}// end anonymous namespace

// One copy per device, part of the module image: it exists once the module is loaded on a device
// and is never freed.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

namespace
{

std::mutex g_noalloc_setup_mutex;
unsigned char* g_noalloc_scratch_ptr[kNoAllocMaxDevices] = {};

// Device address of the current device's scratch, looked up once per device (with that device
// current) on the first call that runs there.
unsigned char* noalloc_scratch_of_current_device()
{
	int dev = -1;
	PG_CUDA_CHECK(cudaGetDevice(&dev));
	if(dev < 0 || dev >= kNoAllocMaxDevices)
	{
		throw Error(PG_ERR_INVALID_ARGUMENT, "pgpu_trace_closest_noalloc: device index out of range");
	}
	std::lock_guard<std::mutex> lock(g_noalloc_setup_mutex);
	if(!g_noalloc_scratch_ptr[dev])
	{
		void* p = nullptr;
		const cudaError_t status = cudaGetSymbolAddress(&p, g_noalloc_scratch);
		if(status != cudaSuccess || !p)
		{
			cudaGetLastError();
			throw Error(PG_ERR_CUDA, std::string("pgpu_trace_closest_noalloc: cudaGetSymbolAddress of the "
			                                     "static scratch failed: ") + cudaGetErrorString(status));
		}
		g_noalloc_scratch_ptr[dev] = static_cast<unsigned char*>(p);
	}
	return g_noalloc_scratch_ptr[dev];
}

}// end anonymous namespace

extern "C" {

int pgpu_trace_closest_noalloc(uint64_t id, const float* rays, uint64_t n,
                               int32_t* out_prim, float* out_t, float* out_bary)
{
	return guarded([&]
	{
		if(n > kNoAllocMaxRays)
		{
			throw Error(PG_ERR_INVALID_ARGUMENT,
				"pgpu_trace_closest_noalloc: " + std::to_string(n) + " rays exceed the static scratch "
				"capacity of " + std::to_string(kNoAllocMaxRays) + " rays per call; split the batch");
		}
		if(!rays && n > 0)
		{
			throw Error(PG_ERR_INVALID_ARGUMENT, "pgpu_trace_closest_noalloc: null rays");
		}
		auto g = get_geometry(id);
		unsigned char* scratch = noalloc_scratch_of_current_device();
		if(n == 0)
		{
			return;
		}
		float* d_rays = reinterpret_cast<float*>(scratch + kNoAllocRaysOffset);
		HitRecord* d_hits = reinterpret_cast<HitRecord*>(scratch + kNoAllocHitsOffset);
		int32_t* d_prim = reinterpret_cast<int32_t*>(scratch + kNoAllocPrimOffset);
		float* d_t = reinterpret_cast<float*>(scratch + kNoAllocTOffset);
		float* d_bary = reinterpret_cast<float*>(scratch + kNoAllocBaryOffset);

		cudaStream_t s = library_stream();
		PG_CUDA_CHECK(cudaMemcpyAsync(d_rays, rays, n * 8 * sizeof(float), cudaMemcpyHostToDevice, s));
		launch_trace_closest(*g, d_rays, n, d_hits, s);
		resolve_hits_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, s>>>(
			g->tris.get(), reinterpret_cast<const float4*>(d_rays), d_hits, n, d_prim, d_t, d_bary);
		PG_CUDA_CHECK(cudaGetLastError());
		// straight into the caller's arrays: no host staging either
		if(out_prim) { PG_CUDA_CHECK(cudaMemcpyAsync(out_prim, d_prim, n * sizeof(int32_t), cudaMemcpyDeviceToHost, s)); }
		if(out_t) { PG_CUDA_CHECK(cudaMemcpyAsync(out_t, d_t, n * sizeof(float), cudaMemcpyDeviceToHost, s)); }
		if(out_bary) { PG_CUDA_CHECK(cudaMemcpyAsync(out_bary, d_bary, 3 * n * sizeof(float), cudaMemcpyDeviceToHost, s)); }
		PG_CUDA_CHECK(cudaStreamSynchronize(s));
		check_device_error(*g, s);
	});
}

}// extern "C"
