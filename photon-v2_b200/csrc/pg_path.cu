// Wavefront BNEEPT / BVPT kernels (camera rays, shading, bookkeeping) and the render driver.
//
// Compiled without FMA contraction (see the Makefile) so that the FP32 shading arithmetic rounds
// like the reference's x86 build. The estimator logic follows
//   BNEEPTEstimator::estimate  Engine/Source/Core/Estimator/BNEEPTEstimator.cpp:38-262
//   BVPTEstimator::estimate    Engine/Source/Core/Estimator/BVPTEstimator.cpp:25-160
// with the per-bounce loop unrolled across kernel launches: one shade invocation is one loop
// iteration of one path.
#include "guide_mlp.h"
#include "pg_render.h"
#include "refinery.cuh"
#include "scene_build.h"

#include "../../include/photon_gpu.h"

#include <cooperative_groups.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>

namespace cg = cooperative_groups;

namespace pg
{
namespace
{

constexpr int kShadeBlock = 128;
// Iterations per training period of a guided render that trains (even: the path buffers alternate).
// Periods of 6 and 8 iterations measured the same equal-time ratio on the slit room within the
// run-to-run spread, with fewer training steps.
constexpr int kTrainPeriod = 4;
static_assert(kTrainPeriod >= 4 && kTrainPeriod % 2 == 0, "training period");
constexpr float kClampMax = 1e9f;

// ---------------------------------------------------------------------------------------------
// Counter-based random numbers: every (path, bounce, dimension) has its own independent uniform,
// so results do not depend on scheduling (the reference draws from per-thread PCG32 streams and
// is not reproducible run to run; parity with it is statistical).

__device__ __forceinline__ uint64_t mix64(uint64_t z)
{
	z += 0x9E3779B97F4A7C15ull;
	z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
	z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
	return z ^ (z >> 31);
}

struct PathRng
{
	uint64_t base;

	__device__ __forceinline__ float u01(uint32_t bounce, uint32_t dim) const
	{
		const uint64_t h = mix64(base + ((static_cast<uint64_t>(bounce) << 4) | dim) * 0xD1B54A32D192ED03ull);
		return static_cast<float>(h >> 40) * (1.0f / 16777216.0f);
	}
};

__device__ __forceinline__ PathRng make_rng(uint64_t seed, uint64_t global_path)
{
	return PathRng{mix64(global_path ^ mix64(seed))};
}

// Dimensions per vertex.
enum : uint32_t
{
	DIM_CAM_X = 0, DIM_CAM_Y = 1,
	DIM_NEE_PICK = 2, DIM_NEE_TRI = 3, DIM_NEE_U = 4, DIM_NEE_V = 5,
	DIM_BSDF_0 = 6, DIM_BSDF_1 = 7, DIM_BSDF_2 = 8,
	DIM_RR = 9,
	DIM_GUIDE_SEL = 10, DIM_GUIDE_0 = 11, DIM_GUIDE_1 = 12, DIM_GUIDE_2 = 13,
	DIM_TRAIN_KEEP = 14,
};

// Relative luminance of linear sRGB (CIE Y), used by Russian roulette
// (RussianRoulette.h:30-55 -> TSpectrumBase::relativeLuminance).
__device__ __forceinline__ float luminance(RGB c)
{
	return static_cast<float>(kLumR) * c.r + static_cast<float>(kLumG) * c.g + static_cast<float>(kLumB) * c.b;
}

__device__ __forceinline__ float4 ld4(const float4* p) { return *p; }

__device__ __forceinline__ V3 xyz(float4 v) { return v3(v.x, v.y, v.z); }

// Face normal as PTriangle stores it: (B-A) x (C-A), normalised, (0,1,0) for degenerate
// triangles (PTriangle.cpp:19-35, TBasicTriangle::safeGetFaceNormal).
__device__ __forceinline__ V3 face_normal(const TriVerts& t)
{
	const V3 n = cross(t.b - t.a, t.c - t.a);
	const float len2 = length_sq(n);
	if(!(len2 > 0.0f) || isinf(len2))
	{
		return v3(0.0f, 1.0f, 0.0f);
	}
	const V3 u = normalize(n);
	return is_finite(u) ? u : v3(0.0f, 1.0f, 0.0f);
}

__device__ __forceinline__ float tri_area(const TriVerts& t)
{
	return length(cross(t.b - t.a, t.c - t.a)) * 0.5f;
}

__device__ __forceinline__ TriVerts load_tri(const LeafTri* tris, uint32_t k, uint32_t* material, uint32_t* emitter)
{
	const float4* p = reinterpret_cast<const float4*>(tris + k);
	const float4 a = p[0], b = p[1], c = p[2];
	if(material) { *material = __float_as_uint(b.w); }
	if(emitter) { *emitter = __float_as_uint(c.w); }
	return TriVerts{v3(a.x, a.y, a.z), v3(b.x, b.y, b.z), v3(c.x, c.y, c.z)};
}

// Area pdf -> solid angle pdf (Engine/Source/Core/LTA/lta.h:17-25).
__device__ __forceinline__ float pdfa_to_pdfw(float pdf_a, V3 da_to_target, V3 da_normal)
{
	const float dist2 = length_sq(da_to_target);
	const float w = pdf_a / dot(normalize(da_to_target), da_normal) * dist2;
	return isfinite(w) ? fabsf(w) : 0.0f;
}

__device__ __forceinline__ RGB emitter_radiance(const EmitterRec& e) { return RGB{e.r, e.g, e.b}; }

// Solid-angle density of a direct light sample at xe on light triangle lt (face normal ne) of
// emitter e, for the receiving point `target`: the power-favouring pick (pmf), the uniform pick
// among the emitter's triangles (1 / count) and the uniform point on the triangle converted to
// solid angle (ESPowerFavoring::calcDirectPdf, ESPowerFavoring.cpp:82-97 ->
// GroupedDiffuseSurfaceEmitter::calcDirectPdf, GroupedDiffuseSurfaceEmitter.cpp:80-84 ->
// SurfaceEmitter::calcDirectPdfWForSrcPrimitive, SurfaceEmitter.cpp:37-61). 0 where the
// triangle's front face does not face the target (one-sided emission, canEmit).
__device__ __forceinline__ float light_triangle_pdf_w(const EmitterRec& e, const TriVerts& lt, V3 ne, V3 xe, V3 target)
{
	const V3 emitter_to_target = target - xe;
	if(!(dot(emitter_to_target, ne) > 0.0f))
	{
		return 0.0f;
	}
	return pdfa_to_pdfw(1.0f / tri_area(lt), emitter_to_target, ne) * e.rcp_count * e.pmf;
}

__device__ __forceinline__ uint32_t alias_pick(const float2* alias, uint32_t n, float u)
{
	const float scaled = u * static_cast<float>(n);
	uint32_t i = min(static_cast<uint32_t>(scaled), n - 1u);
	const float frac = scaled - static_cast<float>(i);
	const float2 a = alias[i];
	return frac < a.x ? i : __float_as_uint(a.y);
}

// Raster position of a path's camera sample: a uniform point in its pixel's cell of the film's
// sample window (film.cuh).
__device__ __forceinline__ float2 raster_position(const FilmView& f, uint32_t pixel, const PathRng& rng)
{
	const uint32_t x = pixel % f.width;
	const uint32_t y = pixel / f.width;
	return make_float2(f.x0 + (static_cast<float>(x) + rng.u01(0, DIM_CAM_X)) * f.sx,
	                   f.y0 + (static_cast<float>(y) + rng.u01(0, DIM_CAM_Y)) * f.sy);
}

// Radiance of a finished path (or a part of it) into the film.
__device__ __forceinline__ void splat(const FilmView& f, uint32_t pixel, uint32_t path, RGB c)
{
	if(f.filter == PG_FILTER_BOX)
	{
		film_add_box(f, pixel, c.r, c.g, c.b);
	}
	else
	{
		f.samples[path] = make_float4(c.r, c.g, c.b, 0.0f);   // splatted by splat_samples_kernel
	}
}

// 4 x 4 filters: every path of the pass into the film, in path order (its raster position from
// the same counter-based draws the camera ray used), radiance and weight W together.
__global__ void __launch_bounds__(kShadeBlock)
splat_samples_kernel(FilmView film, uint64_t seed, uint64_t first_global, uint32_t num_paths)
{
	const uint32_t wh = film.width * film.height;
	for(uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < num_paths; p += gridDim.x * blockDim.x)
	{
		const float4 c = film.samples[p];
		const PathRng rng = make_rng(seed, first_global + p);
		const float2 r = raster_position(film, p % wh, rng);
		film_deposit(film, r.x, r.y, make_float4(c.x, c.y, c.z, 1.0f));
	}
}

// Previews during a render: the continuing paths of the queue the next iteration starts from,
// counted per pixel.
__global__ void count_inflight_kernel(const uint32_t* __restrict__ path, const RenderCounters* __restrict__ c,
                                      uint32_t wh, uint32_t* __restrict__ counts)
{
	const uint32_t n = c->n_next;
	for(uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
	{
		atomicAdd(&counts[path[i] % wh], 1u);
	}
}

// The film's estimate over finished samples (HdrRgbFilm::developRegion, HdrRgbFilm.cpp:167-205,
// on what the finished paths have deposited). The box film's W was raised by this render's spp
// up front, so the samples of the render that have not finished -- not generated yet (path
// indices from `generated` on; pixel = index mod wh) or still in flight -- come off it; the
// 4 x 4 films only hold whole passes, whose W is exact.
__global__ void develop_preview_kernel(const double* __restrict__ sums, const uint32_t* __restrict__ inflight,
                                       uint32_t wh, uint32_t spp, unsigned long long generated, int box,
                                       float* __restrict__ rgb)
{
	const unsigned long long full = generated / wh;
	const uint32_t part = static_cast<uint32_t>(generated % wh);
	for(uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < wh; i += gridDim.x * blockDim.x)
	{
		const double4 s = reinterpret_cast<const double4*>(sums)[i];
		double w = s.w;
		if(box)
		{
			const unsigned long long gen = full + (i < part ? 1ull : 0ull);
			w -= static_cast<double>(spp) - static_cast<double>(gen) + static_cast<double>(inflight[i]);
		}
		const double rcp = w > 0.0 ? 1.0 / w : 0.0;
		rgb[3 * static_cast<size_t>(i) + 0] = static_cast<float>(s.x * rcp);
		rgb[3 * static_cast<size_t>(i) + 1] = static_cast<float>(s.y * rcp);
		rgb[3 * static_cast<size_t>(i) + 2] = static_cast<float>(s.z * rcp);
	}
}

// Box filter: every pixel received spp samples of weight 1.
__global__ void box_weights_kernel(double* sums, uint32_t num_pixels, double spp)
{
	for(uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < num_pixels; i += gridDim.x * blockDim.x)
	{
		sums[static_cast<size_t>(i) * kFilmChannels + 3] += spp;
	}
}

// Surfaces where a guided render samples the learned mixture: non-black matte.
__device__ __forceinline__ bool guidable(const Material& m)
{
	return m.type == PG_MAT_MATTE && (m.cr > 0.0f || m.cg > 0.0f || m.cb > 0.0f);
}

// Whether guide_query_kernel gives the queue entry a network row: a hit on a guidable surface at
// a vertex below the guiding depth, on a path that continues after it.
__device__ __forceinline__ bool guided_vertex(const Material& m, uint32_t meta, uint32_t guide_depth)
{
	return !(meta & kMetaStopAfter) && (meta & kMetaBounceMask) < guide_depth && guidable(m);
}

// Lists every slot of the current queue under its shading class (kShadeClasses): 0 for a miss,
// 1 + the material type of the hit surface, or kGuidedClass for a vertex a guided render guides
// (guide_depth > 0: the vertices below that bounce), in the list of that class for this block's
// residue (kClassLists). Lanes of one class share one atomic. `list_capacity` bounds the slots one
// list can receive: the slots all blocks of one residue visit in the grid-stride loop.
// MULTI: the hit triangle belongs to the scene in the top bits of the slot's meta word.
template<bool MULTI>
__global__ void __launch_bounds__(kShadeBlock)
classify_kernel(DeviceScene s_single, RenderCounters* __restrict__ c, const uint2* __restrict__ hits,
                uint32_t* __restrict__ order, uint32_t list_capacity, const uint32_t* __restrict__ meta, BatchView batch,
                uint32_t guide_depth)
{
	const uint32_t n = c->n_total;
	const uint32_t residue = blockIdx.x % kClassLists;
	for(uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
	{
		const uint32_t tri = hits[i].x;
		uint32_t cls = 0u;
		if(tri != 0xFFFFFFFFu)
		{
			if constexpr(MULTI)
			{
				const DeviceScene& s = batch.scenes[meta[i] >> kMetaSceneShift].scene;
				cls = min(1u + s.materials[__ldg(&s.tris[tri].material)].type, kGuidedClass - 1u);
			}
			else
			{
				const Material& m = s_single.materials[__ldg(&s_single.tris[tri].material)];
				cls = guide_depth > 0u && guided_vertex(m, meta[i], guide_depth) ? kGuidedClass
				                                                                 : min(1u + m.type, kGuidedClass - 1u);
			}
		}
		const uint32_t list = cls * kClassLists + residue;
		const cg::coalesced_group peers = cg::labeled_partition(cg::coalesced_threads(), cls);
		uint32_t base = 0;
		if(peers.thread_rank() == 0)
		{
			base = atomicAdd(&c->n_class[list], peers.size());
		}
		base = peers.shfl(base, 0);
		order[list * list_capacity + base + peers.thread_rank()] = i;
	}
}

// Warp-aggregated slot allocation on a queue counter.
__device__ __forceinline__ uint32_t alloc_slot(uint32_t* counter)
{
	cg::coalesced_group g = cg::coalesced_threads();
	uint32_t base = 0;
	if(g.thread_rank() == 0)
	{
		base = atomicAdd(counter, g.size());
	}
	base = g.shfl(base, 0);
	return base + g.thread_rank();
}

// ---------------------------------------------------------------------------------------------

// Training periods (guided renders that train): at position 0 the count of marked vertices starts
// afresh; at position 1 the count of samples does, and the share of marked vertices that record a
// sample is set so that they fill record_budget rows on average. Every marked vertex is kept with
// the same probability, whatever the material its path reaches next (taking the first rows
// handed out would favour the classes the shading kernel processes first).
__global__ void prepare_kernel(RenderCounters* c, uint32_t capacity, uint32_t period_pos, uint32_t record_budget)
{
	if(threadIdx.x != 0 || blockIdx.x != 0)
	{
		return;
	}
	const uint32_t active = c->n_next;
	const unsigned long long remaining = c->total_paths - c->next_path;
	const unsigned long long room = static_cast<unsigned long long>(capacity - active);
	const uint32_t n_new = static_cast<uint32_t>(remaining < room ? remaining : room);
	c->n_active = active;
	c->n_total = active + n_new;
	c->gen_base = c->next_path;
	c->next_path += n_new;
	c->n_next = 0;
	c->n_shadow_prev = c->n_shadow;
	c->n_shadow = 0;
	c->fetch_extend = 0;
	c->fetch_shadow = 0;
	c->guided_total += c->n_guided;
	c->n_guided = 0;
	if(period_pos == 0u)
	{
		c->n_marked = 0;
	}
	if(period_pos == 1u)
	{
		c->rec_keep = c->n_marked > record_budget ? static_cast<float>(record_budget) / static_cast<float>(c->n_marked)
		                                          : 1.0f;
		c->n_train = 0;
	}
	c->n_refine = 0;
	c->n_refine_mutual = 0;
	for(uint32_t k = 0; k < kOrderLists; ++k)
	{
		c->n_class[k] = 0;
	}
	c->rays_traced += c->n_total;
}

// Camera rays of new paths into the tail of the current queue
// (PinholeCamera::receiveRay, then BNEEPTEstimator.cpp:63-64: reversed, range [0, max]).
// MULTI: new paths are numbered across the scenes of `batch` (scene k owns [path_first,
// path_first + path_count)); each takes its scene's camera, film and sample numbering, and carries
// its scene in the top bits of its meta word.
template<bool MULTI>
__global__ void __launch_bounds__(kShadeBlock)
regen_kernel(const RenderCounters* __restrict__ c, Camera cam_single, FilmView film_single, uint64_t seed,
             uint64_t first_global_single, PathBuffers cur, BatchView batch)
{
	const uint32_t active = c->n_active;
	const uint32_t total = c->n_total;
	const unsigned long long base = c->gen_base;
	for(uint32_t i = active + blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x)
	{
		const unsigned long long pb = base + (i - active);
		uint32_t sid = 0, p;
		Camera cam;
		FilmView film;
		uint64_t first_global;
		if constexpr(MULTI)
		{
			// the last scene whose first path is at or before pb
			uint32_t lo = 0, hi = batch.count - 1u;
			while(lo < hi)
			{
				const uint32_t mid = (lo + hi + 1u) >> 1;
				if(batch.scenes[mid].path_first <= pb) { lo = mid; } else { hi = mid - 1u; }
			}
			sid = lo;
			const BatchScene& bs = batch.scenes[sid];
			p = static_cast<uint32_t>(pb - bs.path_first);
			cam = bs.scene.cam;
			film = bs.film;
			first_global = bs.first_global;
		}
		else
		{
			p = static_cast<uint32_t>(pb);
			cam = cam_single;
			film = film_single;
			first_global = first_global_single;
		}
		const uint32_t wh = cam.width * cam.height;
		const uint32_t pixel = p % wh;
		const PathRng rng = make_rng(seed, first_global + p);
		const float2 raster = raster_position(film, pixel, rng);
		const float rx = raster.x;
		const float ry = raster.y;

		// raster -> sensor (SingleLensObserver::makeRasterToSensor)
		const float sx = -cam.sensor_w / static_cast<float>(cam.width) * rx + cam.sensor_w * 0.5f;
		const float sy = -cam.sensor_h / static_cast<float>(cam.height) * ry + cam.sensor_h * 0.5f;
		const float sz = cam.sensor_offset;
		const V3 recv = normalize(v3(cam.axis_x[0], cam.axis_x[1], cam.axis_x[2]) * sx +
		                          v3(cam.axis_y[0], cam.axis_y[1], cam.axis_y[2]) * sy +
		                          v3(cam.axis_z[0], cam.axis_z[1], cam.axis_z[2]) * sz);
		const V3 d = -recv;

		cur.path[i] = p;
		cur.meta[i] = sid << kMetaSceneShift;
		cur.thr[i] = make_float4(1.0f, 1.0f, 1.0f, 1.0f);
		cur.rad[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
		cur.prev[i] = make_float4(0.0f, 0.0f, 0.0f, 1.0f);
		cur.ray_o[i] = make_float4(cam.pos[0], cam.pos[1], cam.pos[2], 0.0f);
		cur.ray_d[i] = make_float4(d.x, d.y, d.z, kFloatMax);
	}
}

// ---------------------------------------------------------------------------------------------
// Learned guiding at Lambertian vertices.

// Mixture density at unit direction w of a decoded network row (per lobe: weight, mean xyz,
// kappa, weight x normalisation): sum_j c_j exp(kappa_j (mu_j . w - 1)).
__device__ __noinline__ float guide_pdf(const float* __restrict__ mix, V3 w)
{
	const float2* q = reinterpret_cast<const float2*>(mix);
	float p = 0.0f;
	#pragma unroll
	for(int j = 0; j < guide::kLobes; ++j)
	{
		const float2 a = __ldg(q + 3 * j), b = __ldg(q + 3 * j + 1), c = __ldg(q + 3 * j + 2);
		p += c.y * expf(c.x * (a.y * w.x + b.x * w.y + b.y * w.z - 1.0f));
	}
	return p;
}

__device__ __noinline__ V3 guide_sample(const float* __restrict__ mix, float u0, float u1, float u2)
{
	// the lobe as guide::mixture_sample picks it (the first whose running weight sum exceeds u0),
	// then only that lobe's mean and concentration are loaded: no local copy of the mixture
	const float2* q = reinterpret_cast<const float2*>(mix);
	int j = 0;
	float acc = __ldg(q).x;
	while(j < guide::kLobes - 1 && u0 >= acc)
	{
		++j;
		acc += __ldg(q + 3 * j).x;
	}
	const float2 a = __ldg(q + 3 * j), b = __ldg(q + 3 * j + 1), c = __ldg(q + 3 * j + 2);
	return guide::vmf_sample(v3(a.y, b.x, b.y), c.x, u1, u2);
}

// Network inputs for every queue entry that will be shaded at a guidable vertex; entries are
// compacted into rows (map: entry -> row).
__global__ void __launch_bounds__(kShadeBlock)
guide_query_kernel(DeviceScene s, RenderCounters* __restrict__ c, PathBuffers cur, const uint2* __restrict__ hits,
                   GuideArgs g, uint32_t max_bounces)
{
	const uint32_t total = c->n_total;
	for(uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x)
	{
		const uint2 hit = hits[i];
		const uint32_t meta = cur.meta[i];
		uint32_t row = 0xFFFFFFFFu;
		if(hit.x != 0xFFFFFFFFu)
		{
			const LeafTri& lt = s.tris[hit.x];
			if(guided_vertex(s.materials[lt.material], meta, max_bounces))
			{
				const float4 o = cur.ray_o[i];
				const float4 d4 = cur.ray_d[i];
				const V3 d = v3(d4.x, d4.y, d4.z);
				const float t = __uint_as_float(hit.y);
				const V3 pos = v3(o.x, o.y, o.z) + d * t;
				const V3 a = v3(lt.v0x, lt.v0y, lt.v0z), b = v3(lt.v1x, lt.v1y, lt.v1z), cc = v3(lt.v2x, lt.v2y, lt.v2z);
				V3 n = normalize(cross(b - a, cc - a));
				if(dot(n, d) > 0.0f)
				{
					n = -n;   // the side the path arrives on
				}
				const guide::Features f = guide::make_features(pos, v3(g.lo[0], g.lo[1], g.lo[2]),
				                                               v3(g.rcp[0], g.rcp[1], g.rcp[2]), n, -d);
				row = alloc_slot(&c->n_guided);
				float4* dst = reinterpret_cast<float4*>(g.feat + static_cast<size_t>(row) * 8);
				dst[0] = make_float4(f.v[0], f.v[1], f.v[2], f.v[3]);
				dst[1] = make_float4(f.v[4], f.v[5], f.v[6], 0.0f);
			}
		}
		g.map[i] = row;
	}
}

// Running mean of the per-step training loss over a render (steps that had samples).
__global__ void guide_loss_kernel(float* scalars, const uint32_t* n_train)
{
	if(*n_train > 0u)
	{
		scalars[2] += scalars[0];
		scalars[3] += 1.0f;
	}
}

struct ShadeArgs
{
	DeviceScene   scene;
	PathBuffers   cur;
	PathBuffers   next;
	const uint2*  hits;
	ShadowQueue   shadow;
	RenderCounters* counters;
	FilmView      film;
	uint64_t      seed;
	uint64_t      first_global;
	uint32_t      max_bounces;
	uint32_t      estimator;
	uint32_t      width_height;
	GuideArgs     guide;
	RefineSettings refine;
	RefineQueue   refine_queue;   // iterative refine mode: requests for refine_kernel
	const uint32_t* order;        // slots listed per shading class (classify_kernel), or null: slot order
	uint32_t      order_capacity; // slots per list of `order`
	BatchView     batch;          // multi-scene renders: scene, film and numbering of every path
};

__device__ __forceinline__ float4 cur_gf0(const ShadeArgs& a, uint32_t i) { return a.cur.gf0[i]; }
__device__ __forceinline__ float4 cur_gf1(const ShadeArgs& a, uint32_t i) { return a.cur.gf1[i]; }

// GUIDED instantiates the learned-guiding paths; the plain estimator compiles without them.
// MULTI: each path shades in the scene of its meta word's top bits (a.batch), into that scene's
// film, and passes the scene on to its continuation and its NEE record.
template<bool GUIDED, bool MULTI>
__global__ void __launch_bounds__(kShadeBlock)
shade_kernel(ShadeArgs a)
{
	const uint32_t total = a.counters->n_total;
	// work item w -> queue slot: list by list (class-major) through the lists classify_kernel made
	__shared__ uint32_t list_end[kOrderLists];
	if(a.order && threadIdx.x == 0)
	{
		uint32_t end = 0;
		for(uint32_t l = 0; l < kOrderLists; ++l)
		{
			end += a.counters->n_class[l];
			list_end[l] = end;
		}
	}
	__syncthreads();
	for(uint32_t w = blockIdx.x * blockDim.x + threadIdx.x; w < total; w += gridDim.x * blockDim.x)
	{
		uint32_t i = w;
		if(a.order)
		{
			// first list whose end exceeds w
			uint32_t lo = 0, hi = kOrderLists - 1u;
			while(lo < hi)
			{
				const uint32_t mid = (lo + hi) >> 1;
				if(w < list_end[mid]) { hi = mid; } else { lo = mid + 1u; }
			}
			i = a.order[lo * a.order_capacity + (w - (lo ? list_end[lo - 1u] : 0u))];
		}
		const uint32_t p = a.cur.path[i];
		const uint32_t meta = a.cur.meta[i];
		const uint32_t bounce = meta & kMetaBounceMask;
		const uint32_t sid = MULTI ? meta >> kMetaSceneShift : 0u;
		const DeviceScene& s = MULTI ? a.batch.scenes[sid].scene : a.scene;
		const FilmView& film = MULTI ? a.batch.scenes[sid].film : a.film;
		const uint32_t width_height = MULTI ? a.batch.scenes[sid].width_height : a.width_height;
		const uint64_t first_global = MULTI ? a.batch.scenes[sid].first_global : a.first_global;
		const float4 thr4 = ld4(a.cur.thr + i);
		const float4 rad4 = ld4(a.cur.rad + i);
		const float4 prev4 = ld4(a.cur.prev + i);
		const float4 ro = ld4(a.cur.ray_o + i);
		const float4 rd = ld4(a.cur.ray_d + i);
		const uint2 hit = a.hits[i];
		const uint32_t pixel = p % width_height;
		const PathRng rng = make_rng(a.seed, first_global + p);

		const RGB thr_emit = RGB{thr4.x, thr4.y, thr4.z};
		const float cont = thr4.w;
		RGB radiance = RGB{rad4.x, rad4.y, rad4.z};
		const float prev_bsdf_pdf = rad4.w;
		const V3 prev_pos = xyz(prev4);
		float rr_scale = prev4.w;
		const V3 d = xyz(rd);
		// BVPT and BVPTDL add the emission their BSDF-sampled rays find; BVPTDL clamps the emitted
		// radiance and not the path weight (BVPTDLEstimator.cpp:58-61, 88-91).
		const bool bvpt = a.estimator != PG_EST_BNEEPT;
		const bool dl = a.estimator == PG_EST_BVPTDL;

		// ---- training sample for the guided vertex this ray left from: its incident radiance
		//      is estimated by the emission found here plus the unoccluded NEE at this vertex
		//      (added by the shadow kernel)
		uint32_t train_row = 0xFFFFFFFFu;
		float train_wfac = 0.0f;
		// (a miss without an environment brings no light: its sample would weigh 0)
		if(GUIDED && (meta & kMetaGuideRec) && a.guide.train_cap && (hit.x != 0xFFFFFFFFu || s.env_emitter >= 0) &&
		   rng.u01(bounce, DIM_TRAIN_KEEP) < a.counters->rec_keep)
		{
			const uint32_t k = alloc_slot(&a.counters->n_train);
			if(k < a.guide.train_cap)
			{
				const float4 g0 = cur_gf0(a, i);
				const float4 g1 = cur_gf1(a, i);
				float4* dst = reinterpret_cast<float4*>(a.guide.train_feat + static_cast<size_t>(k) * 8);
				dst[0] = g0;
				dst[1] = g1;
				train_row = k;
				train_wfac = g1.w;
				a.guide.train_dirw[k] = make_float4(d.x, d.y, d.z, 0.0f);
			}
		}
		// The training record this path's contributions are credited to: the one made here, or one
		// made at an earlier vertex and still open. An open record collects what the path gathers
		// after its next vertex (emission found later, NEE further on) divided by the path
		// throughput at that vertex, i.e. the radiance that arrived along the sampled direction
		// after more bounces, such as light reaching a matte surface through glass.
		uint32_t rec_row = GUIDED ? train_row : 0xFFFFFFFFu;
		float rec_scale = 0.0f;   // the record's |cos| / pdf over the throughput at its next vertex
		const bool rec_new = GUIDED && train_row != 0xFFFFFFFFu;
		if(GUIDED && !rec_new && (meta & kMetaGuideOpen) && a.guide.open)
		{
			const float4 g0 = cur_gf0(a, i);
			rec_row = __float_as_uint(g0.x);
			rec_scale = g0.y;
		}
		const float lum_before = GUIDED ? luminance(radiance) : 0.0f;
		// emission this vertex added to the path, credited to an open record
		auto credit_open = [&]
		{
			if(GUIDED && rec_row != 0xFFFFFFFFu && !rec_new)
			{
				const float added = luminance(radiance) - lum_before;
				if(added > 0.0f && isfinite(added))
				{
					a.guide.train_dirw[rec_row].w += added * rec_scale;
				}
			}
		};

		// ---- miss: environment (the dome primitive is hit after every triangle missed)
		if(hit.x == 0xFFFFFFFFu)
		{
			const RGB le = s.env_emitter < 0 ? RGB{0.0f, 0.0f, 0.0f} : env_lookup(s.env_map, env_uv(s.env_map, d));
			if(train_row != 0xFFFFFFFFu && s.env_emitter >= 0)
			{
				a.guide.train_dirw[train_row].w = luminance(le) * train_wfac;
			}
			if(s.env_emitter >= 0)
			{
				if(bvpt)
				{
					radiance = radiance + (dl ? safe_clamp(le, 0.0f, kClampMax) * (thr_emit * cont)
					                          : le * safe_clamp(thr_emit * cont, 0.0f, kClampMax));
				}
				else if(bounce == 0)
				{
					radiance = radiance + le;
				}
				else if(meta & kMetaPrevNee)
				{
					if(prev_bsdf_pdf > 0.0f)
					{
						const EmitterRec e = s.emitters[s.env_emitter];
						const float light_pdf = e.pmf * env_pdf_hit(s.env_map, prev_pos, d);
						const float mis = prev_bsdf_pdf * prev_bsdf_pdf /
						                  (prev_bsdf_pdf * prev_bsdf_pdf + light_pdf * light_pdf);
						radiance = radiance + le * safe_clamp(thr_emit * mis, 0.0f, kClampMax);
					}
				}
				else
				{
					radiance = radiance + le * safe_clamp(thr_emit, 0.0f, kClampMax);
				}
			}
			credit_open();
			splat(film, pixel, p, radiance);
			continue;
		}

		// ---- surface hit: recover barycentrics, position and normals
		uint32_t mat_index, emitter_plus_one;
		const TriVerts tri = load_tri(s.tris, hit.x, &mat_index, &emitter_plus_one);
		const RayTraits rt = make_ray_traits(ro.x, ro.y, ro.z, d.x, d.y, d.z);
		float t_hit, b0, b1, b2;
		watertight_hit(rt, tri.a.x, tri.a.y, tri.a.z, tri.b.x, tri.b.y, tri.b.z, tri.c.x, tri.c.y, tri.c.z,
		               ro.w, rd.w, &t_hit, &b0, &b1, &b2);
		const V3 pos = tri.a * b0 + tri.b * b1 + tri.c * b2;
		const V3 ng = face_normal(tri);
		const Frame frame = make_frame(ng, ng);

		// traceNextSurface rejects hits whose sidedness disagrees (SurfaceTracer.h:126-141).
		if(!(dot(ng, d) * dot(frame.ns, d) > 0.0f))
		{
			splat(film, pixel, p, radiance);
			continue;
		}

		// ---- emission arriving at this vertex
		if(emitter_plus_one != 0u)
		{
			const EmitterRec e = s.emitters[emitter_plus_one - 1u];
			// one-sided emission: canEmit(-d, Ns) (SurfaceEmitter.cpp:20-25)
			const RGB le = dot(-d, frame.ns) > 0.0f ? emitter_radiance(e) : RGB{0.0f, 0.0f, 0.0f};
			if(train_row != 0xFFFFFFFFu)
			{
				a.guide.train_dirw[train_row].w = luminance(le) * train_wfac;
			}
			if(bvpt)
			{
				radiance = radiance + (dl ? safe_clamp(le, 0.0f, kClampMax) * (thr_emit * cont)
				                          : le * safe_clamp(thr_emit * cont, 0.0f, kClampMax));
			}
			else if(bounce == 0)
			{
				radiance = radiance + le;   // zero-bounce emission (BNEEPTEstimator.cpp:74-82)
			}
			else if((meta & kMetaPrevNee) && !is_zero(le))
			{
				// MIS of the BSDF-sampled hit against NEE (BNEEPTEstimator.cpp:178-213)
				if(prev_bsdf_pdf > 0.0f)
				{
					float light_pdf = 0.0f;
					const V3 to_target = prev_pos - pos;
					if(dot(to_target, frame.ns) > 0.0f)
					{
						light_pdf = pdfa_to_pdfw(1.0f / tri_area(tri), to_target, frame.ns) * e.rcp_count * e.pmf;
					}
					const float mis = prev_bsdf_pdf * prev_bsdf_pdf /
					                  (prev_bsdf_pdf * prev_bsdf_pdf + light_pdf * light_pdf);
					radiance = radiance + le * safe_clamp(thr_emit * mis, 0.0f, kClampMax);
				}
			}
			else
			{
				radiance = radiance + le * safe_clamp(thr_emit, 0.0f, kClampMax);
			}
			credit_open();
		}

		// ---- does the path continue past this vertex?
		if((meta & kMetaStopAfter) || bounce >= a.max_bounces)
		{
			splat(film, pixel, p, radiance);
			continue;
		}
		const RGB throughput = thr_emit * cont;
		if(rec_new)
		{
			rec_scale = train_wfac / fmaxf(luminance(throughput), 1e-20f);
		}
		const Material mat = s.materials[mat_index];
		const V3 v = -d;

		// ---- next-event estimation (TDirectLightEstimator::neeSampleEmission,
		//      TDirectLightEstimator.ipp:71-102; BNEEPTEstimator.cpp:103-149)
		bool has_shadow = false;
		V3 sh_o{}, sh_d{};
		float sh_tmin = 0.0f, sh_tmax = 0.0f;   // the record's .w words: range, or refinery inputs
		uint32_t sh_refine = 0u;   // 1: escape towards a direction, 2: towards a light-triangle point
		// In the iterative refine mode the re-intersection loops run in refine_kernel, whose warps
		// all execute the same loop; this kernel leaves the hit point, its triangle and the target.
		const bool defer_refine = a.refine.mode == PG_REFINE_ITERATIVE;
		RGB sh_c{};
		uint32_t nee_row = 0xFFFFFFFFu;   // this vertex's NEE direction as a training sample of its own
		float nee_w = 0.0f;
		const uint32_t grow = GUIDED ? a.guide.map[i] : 0xFFFFFFFFu;
		const bool guided = GUIDED && grow != 0xFFFFFFFFu;
		const float* graw = guided ? a.guide.raw + static_cast<size_t>(grow) * guide::kMixFloats : nullptr;
		const float alpha = a.guide.alpha;
		// Every material here is non-delta, so NEE applies at every vertex of BNEEPT
		// (TDirectLightEstimator::isNeeSamplable); a black Lambertian surface can gain nothing
		// from it, so its shadow ray is skipped (its contribution would be exactly zero).
		const bool black_matte = (mat.type == PG_MAT_MATTE && mat.cr == 0.0f && mat.cg == 0.0f && mat.cb == 0.0f) ||
		                         mat.type == PG_MAT_ABSORBER;
		const bool nee_samplable = !bvpt;
		const bool use_nee = nee_samplable && s.num_emitters > 0 && !black_matte;
		if(use_nee)
		{
			const uint32_t ei = alias_pick(s.alias, s.num_emitters, rng.u01(bounce, DIM_NEE_PICK));
			const EmitterRec e = s.emitters[ei];
			bool ok = false;
			V3 to_light{};
			float pdf_w = 0.0f;
			RGB le{};
			if(e.type == PG_EMITTER_ENV)
			{
				// a texel by the image's luminance x sin(theta) distribution, a point inside it
				float env_pdf = 0.0f;
				V3 shadow_dir{};
				const bool env_ok = env_sample(s.env_map, pos, rng.u01(bounce, DIM_NEE_TRI), rng.u01(bounce, DIM_NEE_U),
				                               rng.u01(bounce, DIM_NEE_V), &to_light, &env_pdf, &le, &shadow_dir);
				pdf_w = e.pmf * env_pdf;
				if(env_ok && sidedness_agreed(frame, to_light))
				{
					if(defer_refine)
					{
						sh_o = pos;
						sh_d = shadow_dir;
						sh_tmin = __uint_as_float(hit.x);
						sh_tmax = kFloatMax;
						sh_refine = 1u;
					}
					else
					{
						const EscapeRay er = escape_fixed(a.refine, pos, ng, shadow_dir);
						sh_o = er.origin;
						sh_d = er.unit_dir;
						sh_tmin = er.min_t;
						sh_tmax = er.max_distance;
					}
					ok = true;
				}
			}
			else if(e.count > 0u)
			{
				const uint32_t j = e.first + min(static_cast<uint32_t>(rng.u01(bounce, DIM_NEE_TRI) * e.count), e.count - 1u);
				const uint32_t light_tri = s.emitter_tris ? s.emitter_tris[j] : 0u;
				const TriVerts lt = load_tri(s.tris, light_tri, nullptr, nullptr);
				// Osada uniform triangle sampling (TBasicTriangle::sampleToBarycentricOsada)
				const float su = sqrtf(rng.u01(bounce, DIM_NEE_U));
				const float sv = rng.u01(bounce, DIM_NEE_V);
				const float lb0 = 1.0f - su, lb1 = su * (1.0f - sv), lb2 = sv * su;
				const V3 xe = lt.a * lb0 + lt.b * lb1 + lt.c * lb2;
				const V3 ne = face_normal(lt);
				pdf_w = light_triangle_pdf_w(e, lt, ne, xe, pos);
				if(pdf_w > 0.0f)
				{
					le = emitter_radiance(e);
					const V3 target_to_emit = xe - pos;
					if(pdf_w > 0.0f && isfinite(pdf_w) && sidedness_agreed(frame, target_to_emit))
					{
						if(defer_refine)
						{
							// a failed mutual escape zeroes the contribution in refine_kernel
							sh_o = pos;
							sh_d = xe;
							sh_tmin = __uint_as_float(hit.x);
							sh_tmax = __uint_as_float(light_tri);
							sh_refine = 2u;
							to_light = target_to_emit;
							ok = true;
						}
						else
						{
							const EscapeRay er = try_escape_fixed(a.refine, pos, ng, xe, ne);
							if(er.ok)
							{
								sh_o = er.origin;
								sh_d = er.unit_dir;
								sh_tmin = er.min_t;
								sh_tmax = er.max_distance;
								to_light = target_to_emit;
								ok = true;
							}
						}
					}
				}
			}
			if(ok && pdf_w > 0.0f)
			{
				const V3 l = normalize(to_light);
				RGB f;
				if(bsdf_eval(mat, frame, l, v, &f))
				{
					float pdf_bsdf = bsdf_pdf(mat, frame, l, v);
					if(guided)
					{
						// the direction-sampling technique at a guided vertex is the one-sample mixture
						pdf_bsdf = alpha * guide_pdf(graw, l) + (1.0f - alpha) * pdf_bsdf;
					}
					if(GUIDED && guided && a.guide.train_cap)
					{
						// The light sample is a direction with known incident radiance and density:
						// an importance-weighted sample of the incident-light distribution the network
						// learns (weight lum(Le) |cos| / pdf, credited only if the segment turns out
						// unoccluded). Light seen through a narrow opening is found far more often this
						// way than by directions the BSDF or the network sampled.
						const float wn = luminance(le) * fabsf(dot(frame.ns, l)) / pdf_w;
						if(wn > 0.0f && isfinite(wn))
						{
							const uint32_t k2 = alloc_slot(&a.counters->n_train);
							if(k2 < a.guide.train_cap)
							{
								const float4* fr = reinterpret_cast<const float4*>(a.guide.feat + static_cast<size_t>(grow) * 8);
								float4* dst = reinterpret_cast<float4*>(a.guide.train_feat + static_cast<size_t>(k2) * 8);
								const float4 f1 = fr[1];
								dst[0] = fr[0];
								dst[1] = make_float4(f1.x, f1.y, f1.z, 0.0f);
								a.guide.train_dirw[k2] = make_float4(l.x, l.y, l.z, 0.0f);
								nee_row = k2;
								nee_w = wn;
							}
						}
					}
					const float mis = pdf_w * pdf_w / (pdf_w * pdf_w + pdf_bsdf * pdf_bsdf);
					RGB w = f * fabsf(dot(frame.ns, l));
					w = w * throughput;
					w = w * (mis / pdf_w);
					w = safe_clamp(w, 0.0f, kClampMax);
					sh_c = le * w;
					has_shadow = !is_zero(sh_c);
				}
			}
		}

		// ---- BSDF sampling and extension (BNEEPTEstimator.cpp:155-247, BVPTEstimator.cpp:80-110)
		BsdfSample bs;
		float guided_pdf = 0.0f;
		if(guided)
		{
			// one-sample MIS of the learned mixture (probability alpha) and the BSDF
			V3 l;
			bool have;
			if(rng.u01(bounce, DIM_GUIDE_SEL) < alpha)
			{
				l = guide_sample(graw, rng.u01(bounce, DIM_GUIDE_0), rng.u01(bounce, DIM_GUIDE_1),
				                 rng.u01(bounce, DIM_GUIDE_2));
				have = true;
			}
			else
			{
				const BsdfSample b0 = bsdf_sample(mat, frame, v, rng.u01(bounce, DIM_BSDF_0),
				                                  rng.u01(bounce, DIM_BSDF_1), rng.u01(bounce, DIM_BSDF_2));
				l = b0.l;
				have = b0.ok;
			}
			bs.ok = false;
			RGB f;
			if(have && bsdf_eval(mat, frame, l, v, &f))
			{
				const float pdf = alpha * guide_pdf(graw, l) + (1.0f - alpha) * bsdf_pdf(mat, frame, l, v);
				const float c = fabsf(dot(frame.ns, l));
				if(pdf > 0.0f && isfinite(pdf))
				{
					bs.l = l;
					bs.weight = f * (c / pdf);
					bs.rel_ior = 1.0f;
					bs.cos = c;
					bs.ok = is_finite(bs.weight) && c > 0.0f;
					guided_pdf = pdf;
				}
			}
		}
		else
		{
			bs = bsdf_sample(mat, frame, v, rng.u01(bounce, DIM_BSDF_0),
			                 rng.u01(bounce, DIM_BSDF_1), rng.u01(bounce, DIM_BSDF_2));
		}
		bool continues = bs.ok;
		RGB next_thr_emit{};
		float next_cont = 1.0f;
		float next_pdf = 0.0f;
		uint32_t next_meta = 0u;
		if(continues)
		{
			next_thr_emit = throughput * bs.weight;
			rr_scale /= bs.rel_ior * bs.rel_ior;
			if(!bvpt)
			{
				next_pdf = guided ? guided_pdf : bsdf_pdf(mat, frame, bs.l, v);
			}
			bool stop_after = false;
			if(bounce >= 3)
			{
				const float survival = safe_clamp(luminance(next_thr_emit * rr_scale), 0.0f, 0.95f);
				if(rng.u01(bounce, DIM_RR) < survival)
				{
					next_cont = 1.0f / survival;
				}
				else
				{
					stop_after = true;
				}
			}
			if(is_zero(next_thr_emit) || (bvpt && stop_after))
			{
				// zero throughput: nothing more can be gathered (the emission at the next hit
				// is weighted by it); BVPT gathers emission only with the post-roulette
				// throughput, so a killed BVPT path ends here
				continues = false;
			}
			const bool new_rec = guided && a.guide.mark;
			if(GUIDED && new_rec)
			{
				alloc_slot(&a.counters->n_marked);   // counted: sets the next iteration's keep share
			}
			const bool keep_rec = GUIDED && !new_rec && rec_row != 0xFFFFFFFFu && a.guide.keep;
			next_meta = (bounce + 1u) | (nee_samplable ? kMetaPrevNee : 0u) | (stop_after ? kMetaStopAfter : 0u) |
			            (new_rec ? kMetaGuideRec : 0u) | (keep_rec ? kMetaGuideOpen : 0u) | (sid << kMetaSceneShift);
		}

		uint32_t slot = 0;
		if(continues)
		{
			slot = alloc_slot(&a.counters->n_next);
			a.next.path[slot] = p;
			a.next.meta[slot] = next_meta;
			a.next.thr[slot] = make_float4(next_thr_emit.r, next_thr_emit.g, next_thr_emit.b, next_cont);
			a.next.rad[slot] = make_float4(radiance.r, radiance.g, radiance.b, next_pdf);
			a.next.prev[slot] = make_float4(pos.x, pos.y, pos.z, rr_scale);
			if(defer_refine)
			{
				a.next.ray_o[slot] = make_float4(pos.x, pos.y, pos.z, __uint_as_float(hit.x));
				a.next.ray_d[slot] = make_float4(bs.l.x, bs.l.y, bs.l.z, kFloatMax);
				a.refine_queue.single[alloc_slot(&a.counters->n_refine)] = slot;
			}
			else
			{
				const EscapeRay off = escape_fixed(a.refine, pos, ng, bs.l);
				const V3 o = off.origin;
				a.next.ray_o[slot] = make_float4(o.x, o.y, o.z, off.min_t);
				a.next.ray_d[slot] = make_float4(off.unit_dir.x, off.unit_dir.y, off.unit_dir.z, kFloatMax);
			}
			if(GUIDED && (next_meta & kMetaGuideRec))
			{
				const float4* fr = reinterpret_cast<const float4*>(a.guide.feat + static_cast<size_t>(grow) * 8);
				const float4 f1 = fr[1];
				a.next.gf0[slot] = fr[0];
				a.next.gf1[slot] = make_float4(f1.x, f1.y, f1.z, bs.cos / guided_pdf);
			}
			else if(GUIDED && (next_meta & kMetaGuideOpen))
			{
				a.next.gf0[slot] = make_float4(__uint_as_float(rec_row), rec_scale, 0.0f, 0.0f);
			}
		}
		else
		{
			splat(film, pixel, p, radiance);
		}

		if(has_shadow)
		{
			const uint32_t k = alloc_slot(&a.counters->n_shadow);
			const uint32_t target = continues ? slot : (kTargetFinal | pixel);
			a.shadow.o[k] = make_float4(sh_o.x, sh_o.y, sh_o.z, sh_tmin);
			a.shadow.d[k] = make_float4(sh_d.x, sh_d.y, sh_d.z, sh_tmax);
			a.shadow.c[k] = make_float4(sh_c.r, sh_c.g, sh_c.b, __uint_as_float(target));
			if constexpr(MULTI)
			{
				a.shadow.sid[k] = sid;
			}
			if(GUIDED && a.shadow.t)
			{
				// credited when the next iteration's trace finds the segment unoccluded, if that
				// trace comes before the training step
				const bool credit = rec_row != 0xFFFFFFFFu && a.guide.nee_credit;
				a.shadow.t[k] = make_float4(__uint_as_float(credit ? rec_row : 0xFFFFFFFFu),
				                            credit ? luminance(sh_c) * rec_scale : 0.0f,
				                            __uint_as_float(nee_row), nee_w);
			}
			if(!continues && film.filter != PG_FILTER_BOX)
			{
				a.shadow.r[k] = make_float2(__uint_as_float(p), 0.0f);   // the path, for its sample slot
			}
			if(sh_refine == 1u)
			{
				a.refine_queue.single[alloc_slot(&a.counters->n_refine)] = k | 0x80000000u;
			}
			else if(sh_refine == 2u)
			{
				a.refine_queue.mutual[alloc_slot(&a.counters->n_refine_mutual)] = k;
			}
		}
	}
}

// The surface refinery of one iteration (iterative refine mode): every queued ray slot holds the
// hit point and its leaf triangle (and, towards a light, the light point and its triangle); the
// slot is rewritten with the refined origin, unit direction and range (SurfaceHitRefinery::escape
// / tryEscape, SurfaceHitRefinery.h:200-360). One-sided escapes come first in the grid-stride
// order and mutual ones after them, so nearly every warp runs one loop.
template<bool MULTI>
__global__ void __launch_bounds__(kShadeBlock)
refine_kernel(DeviceScene s_single, const RenderCounters* __restrict__ c, PathBuffers next, ShadowQueue shadow,
              RefineQueue q, int iters, BatchView batch)
{
	const uint32_t n_single = c->n_refine;
	const uint32_t n = n_single + c->n_refine_mutual;
	for(uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
	{
		if(i < n_single)
		{
			const uint32_t r = q.single[i];
			const uint32_t k = r & 0x7FFFFFFFu;
			float4* o = (r & 0x80000000u) ? shadow.o + k : next.ray_o + k;
			float4* d = (r & 0x80000000u) ? shadow.d + k : next.ray_d + k;
			const float4 o4 = *o, d4 = *d;
			// the scene of the ray: its path's (continuation) or its record's (NEE segment)
			const LeafTri* tris = MULTI ? batch.scenes[(r & 0x80000000u) ? shadow.sid[k]
			                                                        : next.meta[k] >> kMetaSceneShift].scene.tris
			                            : s_single.tris;
			const TriVerts tri = load_tri(tris, __float_as_uint(o4.w), nullptr, nullptr);
			const EscapeRay e = escape_iterative(xyz(o4), face_normal(tri), tri, xyz(d4), iters);
			*o = make_float4(e.origin.x, e.origin.y, e.origin.z, e.min_t);
			*d = make_float4(e.unit_dir.x, e.unit_dir.y, e.unit_dir.z, e.max_distance);
		}
		else
		{
			const uint32_t k = q.mutual[i - n_single];
			const float4 o4 = shadow.o[k], d4 = shadow.d[k];
			const LeafTri* tris = MULTI ? batch.scenes[shadow.sid[k]].scene.tris : s_single.tris;
			const TriVerts tri = load_tri(tris, __float_as_uint(o4.w), nullptr, nullptr);
			const TriVerts tri2 = load_tri(tris, __float_as_uint(d4.w), nullptr, nullptr);
			const EscapeRay e = try_escape_iterative(xyz(o4), face_normal(tri), tri, xyz(d4), tri2, iters);
			if(e.ok)
			{
				shadow.o[k] = make_float4(e.origin.x, e.origin.y, e.origin.z, e.min_t);
				shadow.d[k] = make_float4(e.unit_dir.x, e.unit_dir.y, e.unit_dir.z, e.max_distance);
			}
			else
			{
				// no self-intersection-free segment: the light sample contributes nothing
				// (the shading kernel counted it only if the escape succeeds)
				const float4 c4 = shadow.c[k];
				shadow.c[k] = make_float4(0.0f, 0.0f, 0.0f, c4.w);
				if(shadow.t)
				{
					shadow.t[k].y = 0.0f;
					shadow.t[k].w = 0.0f;
				}
				shadow.o[k] = make_float4(o4.x, o4.y, o4.z, 0.0f);
				shadow.d[k] = make_float4(0.0f, 0.0f, 1.0f, 0.0f);
			}
		}
	}
}

}// end anonymous namespace

// ---------------------------------------------------------------------------------------------
// RenderScene

namespace
{

// Alias table (Vose) over non-negative weights; out_pmf[i] = weights[i] / sum. Weights that sum to
// zero give the uniform pmf, as the reference's piecewise-constant distribution falls back to a
// linear CDF then (Math/Random/TPwcDistribution1D.ipp:53-74); a non-finite sum is treated the same
// way, so that the table stays valid. Every column of a uniform table keeps itself.
void build_alias(const std::vector<double>& weights, std::vector<float2>& out_alias, std::vector<double>& out_pmf)
{
	const std::size_t n = weights.size();
	out_alias.resize(n);
	for(std::size_t i = 0; i < n; ++i)
	{
		const uint32_t self = static_cast<uint32_t>(i);
		float fself;
		std::memcpy(&fself, &self, 4);
		out_alias[i] = make_float2(1.0f, fself);
	}
	out_pmf.assign(n, 0.0);
	double sum = 0.0;
	for(double w : weights)
	{
		sum += w;
	}
	if(n == 0)
	{
		return;
	}
	if(!(sum > 0.0) || !std::isfinite(sum))
	{
		out_pmf.assign(n, 1.0 / static_cast<double>(n));
		return;
	}
	std::vector<double> scaled(n);
	std::vector<std::size_t> small, large;
	for(std::size_t i = 0; i < n; ++i)
	{
		out_pmf[i] = weights[i] / sum;
		scaled[i] = out_pmf[i] * static_cast<double>(n);
		(scaled[i] < 1.0 ? small : large).push_back(i);
	}
	std::vector<double> prob(n, 1.0);
	std::vector<uint32_t> alias(n);
	for(std::size_t i = 0; i < n; ++i)
	{
		alias[i] = static_cast<uint32_t>(i);
	}
	while(!small.empty() && !large.empty())
	{
		const std::size_t s = small.back(); small.pop_back();
		const std::size_t l = large.back(); large.pop_back();
		prob[s] = scaled[s];
		alias[s] = static_cast<uint32_t>(l);
		scaled[l] = (scaled[l] + scaled[s]) - 1.0;
		(scaled[l] < 1.0 ? small : large).push_back(l);
	}
	for(std::size_t i = 0; i < n; ++i)
	{
		uint32_t bits;
		std::memcpy(&bits, &alias[i], 4);
		float fbits;
		std::memcpy(&fbits, &bits, 4);
		out_alias[i] = make_float2(static_cast<float>(prob[i]), fbits);
	}
}

}// end anonymous namespace

RenderScene::RenderScene(const SceneDesc& desc, float max_origin_abs)
{
	require_device();
	PG_CUDA_CHECK(cudaStreamCreateWithFlags(&m_stream, cudaStreamNonBlocking));
	const std::size_t n = desc.tris.size() / 9;
	if(n == 0)
	{
		throw Error(PG_ERR_SCENE, "scene has no triangles");
	}
	BvhBuildInput in{desc.tris.data(), desc.tri_material.data(), desc.tri_emitter.data(), n, max_origin_abs};
	m_geometry = desc.bvh_builder == PG_BVH_GPU_MORTON ? make_geometry_gpu(in) : make_geometry(in);
	m_max_origin_abs = max_origin_abs;
	m_bvh_builder = desc.bvh_builder;
	for(const Material& m : desc.materials)
	{
		m_material_types.push_back(m.type);
	}

	// scene bound, normalising the guiding network's position inputs
	{
		float lo[3] = {desc.tris[0], desc.tris[1], desc.tris[2]}, hi[3] = {lo[0], lo[1], lo[2]};
		for(std::size_t k = 0; k < desc.tris.size(); ++k)
		{
			lo[k % 3] = std::min(lo[k % 3], desc.tris[k]);
			hi[k % 3] = std::max(hi[k % 3], desc.tris[k]);
		}
		for(int a = 0; a < 3; ++a)
		{
			m_bound_lo[a] = lo[a];
			m_bound_rcp[a] = hi[a] > lo[a] ? 1.0f / (hi[a] - lo[a]) : 1.0f;
		}
	}

	// Map original triangle index -> leaf slot to build the per-emitter triangle lists.
	std::vector<LeafTri> leaf(m_geometry->tris.size());
	cudaStream_t st = library_stream();
	PG_CUDA_CHECK(cudaMemcpyAsync(leaf.data(), m_geometry->tris.get(), m_geometry->tris.bytes(), cudaMemcpyDeviceToHost, st));
	PG_CUDA_CHECK(cudaStreamSynchronize(st));

	std::vector<EmitterRec> emitters = desc.emitters;
	std::vector<std::vector<uint32_t>> per_emitter(emitters.size());
	std::vector<double> area(emitters.size(), 0.0);
	for(uint32_t k = 0; k < leaf.size(); ++k)
	{
		const uint32_t e = leaf[k].emitter_plus_one;
		if(e == 0u)
		{
			continue;
		}
		if(e > emitters.size())
		{
			throw Error(PG_ERR_SCENE, "triangle refers to a missing emitter");
		}
		per_emitter[e - 1].push_back(k);
		const float* v = &desc.tris[9 * static_cast<std::size_t>(leaf[k].prim)];
		const double ax = v[3] - v[0], ay = v[4] - v[1], az = v[5] - v[2];
		const double bx = v[6] - v[0], by = v[7] - v[1], bz = v[8] - v[2];
		const double cx = ay * bz - az * by, cy = az * bx - ax * bz, cz = ax * by - ay * bx;
		area[e - 1] += 0.5 * std::sqrt(cx * cx + cy * cy + cz * cz);
	}
	// The reference keeps emitter triangles in cooked order; sort each list by original index.
	std::vector<uint32_t> emitter_tris;
	std::vector<double> weights(emitters.size(), 0.0);
	int32_t env_index = -1;

	// the dome image (a constant environment is a 1 x 1 image): texel sampling weights
	// max(luminance, 1e-6) * sin(theta) at texel centres (LatLongEnvEmitter.cpp:52-79), their alias
	// table, and each texel's uv-space density
	const bool env_image = !desc.env_image.empty() && desc.env_width > 0 && desc.env_height > 0;
	double env_weight_sum = 0.0;
	std::vector<float4> env_texels;
	std::vector<float2> env_alias;
	if(desc.has_env)
	{
		std::vector<float> constant_image;
		if(!env_image)
		{
			constant_image.assign(desc.env_rgb, desc.env_rgb + 3);
		}
		const std::vector<float>& image = env_image ? desc.env_image : constant_image;
		const uint32_t w = env_image ? desc.env_width : 1u, h = env_image ? desc.env_height : 1u;
		if(image.size() != static_cast<std::size_t>(w) * h * 3)
		{
			throw Error(PG_ERR_SCENE, "environment image size does not match its dimensions");
		}
		std::vector<double> texel_weights(static_cast<std::size_t>(w) * h);
		for(uint32_t j = 0; j < h; ++j)
		{
			const double v = (j + 0.5) / h;
			const double sin_theta = std::sin((1.0 - v) * 3.14159265358979323846);
			for(uint32_t i = 0; i < w; ++i)
			{
				const float* c = &image[3 * (static_cast<std::size_t>(j) * w + i)];
				const double lum = kLumR * c[0] + kLumG * c[1] + kLumB * c[2];
				texel_weights[static_cast<std::size_t>(j) * w + i] = std::max(lum, 1e-6) * sin_theta;
				env_weight_sum += texel_weights[static_cast<std::size_t>(j) * w + i];
			}
		}
		std::vector<double> texel_pmf;
		build_alias(texel_weights, env_alias, texel_pmf);
		env_texels.resize(texel_weights.size());
		for(std::size_t k = 0; k < texel_weights.size(); ++k)
		{
			const float* c = &image[3 * k];
			env_texels[k] = make_float4(c[0], c[1], c[2], static_cast<float>(texel_pmf[k] * texel_weights.size()));
		}
		m_dev.env_map.width = w;
		m_dev.env_map.height = h;
	}
	for(std::size_t e = 0; e < emitters.size(); ++e)
	{
		auto& list = per_emitter[e];
		std::sort(list.begin(), list.end(), [&](uint32_t x, uint32_t y) { return leaf[x].prim < leaf[y].prim; });
		emitters[e].first = static_cast<uint32_t>(emitter_tris.size());
		emitters[e].count = static_cast<uint32_t>(list.size());
		emitters[e].rcp_count = list.empty() ? 0.0f : 1.0f / static_cast<float>(list.size());
		emitter_tris.insert(emitter_tris.end(), list.begin(), list.end());
		if(emitters[e].type == PG_EMITTER_ENV)
		{
			// luminance x sin(theta) summed over the image's texels, times the dome area
			// (LatLongEnvEmitter.cpp:36-80); a constant environment is a 1 x 1 image
			env_index = static_cast<int32_t>(e);
			weights[e] = env_weight_sum * desc.env_area;
		}
		else
		{
			// radiant flux approximation: energy(radiance) * area * pi, summed over the group
			// (DiffuseSurfaceEmitter.cpp:55-86, GroupedDiffuseSurfaceEmitter.cpp:110-120)
			weights[e] = list.empty() ? 0.0
				: color_energy(emitters[e].r, emitters[e].g, emitters[e].b) * area[e] * 3.14159265358979323846;
		}
	}
	std::vector<float2> alias;
	std::vector<double> pmf;
	build_alias(weights, alias, pmf);
	for(std::size_t e = 0; e < emitters.size(); ++e)
	{
		emitters[e].pmf = static_cast<float>(pmf[e]);
	}

	m_materials.resize(std::max<std::size_t>(1, desc.materials.size()));
	if(!desc.materials.empty())
	{
		PG_CUDA_CHECK(cudaMemcpyAsync(m_materials.get(), desc.materials.data(), desc.materials.size() * sizeof(Material), cudaMemcpyHostToDevice, st));
	}
	m_emitters.resize(std::max<std::size_t>(1, emitters.size()));
	if(!emitters.empty())
	{
		PG_CUDA_CHECK(cudaMemcpyAsync(m_emitters.get(), emitters.data(), emitters.size() * sizeof(EmitterRec), cudaMemcpyHostToDevice, st));
	}
	m_emitter_tris.resize(std::max<std::size_t>(1, emitter_tris.size()));
	if(!emitter_tris.empty())
	{
		PG_CUDA_CHECK(cudaMemcpyAsync(m_emitter_tris.get(), emitter_tris.data(), emitter_tris.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
	}
	m_alias.resize(std::max<std::size_t>(1, alias.size()));
	if(!alias.empty())
	{
		PG_CUDA_CHECK(cudaMemcpyAsync(m_alias.get(), alias.data(), alias.size() * sizeof(float2), cudaMemcpyHostToDevice, st));
	}
	if(desc.has_env)
	{
		m_env_texels.resize(env_texels.size());
		m_env_alias.resize(env_alias.size());
		PG_CUDA_CHECK(cudaMemcpyAsync(m_env_texels.get(), env_texels.data(), env_texels.size() * sizeof(float4),
		                              cudaMemcpyHostToDevice, st));
		PG_CUDA_CHECK(cudaMemcpyAsync(m_env_alias.get(), env_alias.data(), env_alias.size() * sizeof(float2),
		                              cudaMemcpyHostToDevice, st));
		m_dev.env_map.texels = m_env_texels.get();
		m_dev.env_map.alias = m_env_alias.get();
		for(int k = 0; k < 9; ++k) { m_dev.env_map.rot[k] = desc.env_rot[k]; }
		for(int k = 0; k < 3; ++k) { m_dev.env_map.center[k] = desc.env_center[k]; }
		m_dev.env_map.radius = static_cast<float>(std::sqrt(desc.env_area / (4.0 * 3.14159265358979323846)));
	}
	m_counters.resize(1);
	PG_CUDA_CHECK(cudaStreamSynchronize(st));

	m_dev.nodes = m_geometry->nodes.get();
	m_dev.tris = m_geometry->tris.get();
	m_dev.materials = m_materials.get();
	m_dev.emitters = m_emitters.get();
	m_dev.emitter_tris = m_emitter_tris.get();
	m_dev.alias = m_alias.get();
	m_dev.num_emitters = static_cast<uint32_t>(emitters.size());
	m_dev.env_emitter = env_index;
	m_dev.cam = desc.camera;
}

RenderScene::~RenderScene()
{
	if(m_exec)
	{
		cudaGraphExecDestroy(m_exec);
	}
	if(m_stream)
	{
		cudaStreamSynchronize(m_stream);
		cudaStreamDestroy(m_stream);
	}
	if(m_host_counters)
	{
		cudaFreeHost(m_host_counters);
	}
}

void RenderScene::ensure_capacity(uint32_t capacity, uint32_t grid)
{
	if(capacity <= m_capacity && grid == m_order_grid)
	{
		return;
	}
	capacity = std::max(capacity, m_capacity);
	for(int b = 0; b < 2; ++b)
	{
		m_path[b].resize(capacity);
		m_meta[b].resize(capacity);
		m_thr[b].resize(capacity);
		m_rad[b].resize(capacity);
		m_prev[b].resize(capacity);
		m_ro[b].resize(capacity);
		m_rd[b].resize(capacity);
	}
	m_hits.resize(capacity);
	for(int b = 0; b < 2; ++b)
	{
		m_so[b].resize(capacity);
		m_sd[b].resize(capacity);
		m_sc[b].resize(capacity);
		m_sr[b].resize(capacity);
	}
	m_req_single.resize(2 * static_cast<size_t>(capacity));   // continuation + environment NEE per path
	m_req_mutual.resize(capacity);
	{
		// the slots the blocks of one residue visit in classify_kernel's grid-stride loop
		const uint32_t rounds = (capacity + grid * kShadeBlock - 1u) / (grid * kShadeBlock);
		m_order_list = (grid + kClassLists - 1u) / kClassLists * rounds * kShadeBlock;
		m_order.resize(static_cast<size_t>(kOrderLists) * m_order_list);
	}
	m_capacity = capacity;
	m_order_grid = grid;
}

void RenderScene::ensure_guiding(uint32_t capacity)
{
	cudaStream_t st = m_stream;
	if(capacity > m_guide_capacity)
	{
		for(int b = 0; b < 2; ++b)
		{
			m_gf0[b].resize(capacity);
			m_gf1[b].resize(capacity);
		}
		m_st[0].resize(capacity);
		m_st[1].resize(capacity);
		m_gmap.resize(capacity);
		m_gfeat.resize(static_cast<std::size_t>(capacity) * 8);
		m_graw.resize(static_cast<std::size_t>(capacity) * guide::kMixFloats);
		m_guide_capacity = capacity;
	}
	const uint32_t batch = std::max<uint32_t>(m_guide_params.batch, guide::kTile);
	if(m_tdirw.size() < batch)
	{
		m_tfeat.resize(static_cast<std::size_t>(batch) * 8);
		m_traw.resize(static_cast<std::size_t>(batch) * guide::kOut);
		m_tdirw.resize(batch);
		m_tacts.resize(static_cast<std::size_t>(batch) * guide::kHiddenLayers * guide::kHidden);
	}
	if(!m_guide_ready)
	{
		// He-initialised weights (fixed seed), zero biases, output layer scaled down so that the
		// first mixtures are broad
		std::vector<float> p(guide::kNumParams, 0.0f);
		uint64_t state = 0x853C49E6748FEA9Bull;
		auto gauss = [&]()
		{
			auto u = [&]()
			{
				state = state * 6364136223846793005ull + 1442695040888963407ull;
				return (static_cast<double>(state >> 11) + 0.5) * (1.0 / 9007199254740992.0);
			};
			const double a = u(), b = u();
			return std::sqrt(-2.0 * std::log(a)) * std::cos(6.283185307179586 * b);
		};
		auto fill = [&](int off, int fan_in, int count, double scale)
		{
			for(int k = 0; k < count; ++k)
			{
				p[off + k] = static_cast<float>(gauss() * std::sqrt(2.0 / fan_in) * scale);
			}
		};
		fill(guide::kOffW0, guide::kIn, guide::kIn * guide::kHidden, 1.0);
		fill(guide::kOffW1, guide::kHidden, guide::kHidden * guide::kHidden, 1.0);
		fill(guide::kOffW2, guide::kHidden, guide::kHidden * guide::kHidden, 1.0);
		fill(guide::kOffW3, guide::kHidden, guide::kHidden * guide::kHidden, 1.0);
		fill(guide::kOffW4, guide::kHidden, guide::kHidden * guide::kOut, 0.1);
		m_gparams.resize(guide::kNumParams);
		m_gm.resize(guide::kNumParams);
		m_gv.resize(guide::kNumParams);
		m_ggrads.resize(guide::kNumParams);
		m_gscalars.resize(4);   // step loss, weight total, loss sum over the render, steps with samples
		m_gimage.resize(guide::image_bytes());
		m_gstep.resize(1);
		m_gerr.resize(1);
		PG_CUDA_CHECK(cudaMemcpyAsync(m_gparams.get(), p.data(), m_gparams.bytes(), cudaMemcpyHostToDevice, st));
		PG_CUDA_CHECK(cudaMemsetAsync(m_gm.get(), 0, m_gm.bytes(), st));
		PG_CUDA_CHECK(cudaMemsetAsync(m_gv.get(), 0, m_gv.bytes(), st));
		PG_CUDA_CHECK(cudaMemsetAsync(m_ggrads.get(), 0, m_ggrads.bytes(), st));
		PG_CUDA_CHECK(cudaMemsetAsync(m_gscalars.get(), 0, m_gscalars.bytes(), st));
		PG_CUDA_CHECK(cudaMemsetAsync(m_gstep.get(), 0, m_gstep.bytes(), st));
		PG_CUDA_CHECK(cudaMemsetAsync(m_gerr.get(), 0, m_gerr.bytes(), st));
		guide::pack_image(m_gparams.get(), m_gimage.get(), st);
		PG_CUDA_CHECK(cudaStreamSynchronize(st));
		m_guide_ready = true;
	}
}

void RenderScene::reset_guiding()
{
	m_guide_ready = false;
}

void RenderScene::guide_params(float* out) const
{
	if(!m_guide_ready)
	{
		throw Error(PG_ERR_INVALID_ARGUMENT, "guiding network not created yet");
	}
	PG_CUDA_CHECK(cudaMemcpyAsync(out, m_gparams.get(), m_gparams.bytes(), cudaMemcpyDeviceToHost, library_stream()));
	PG_CUDA_CHECK(cudaStreamSynchronize(library_stream()));
}

namespace
{

// Density of direct light samples (light_triangle_pdf_w, the shading kernel's NEE code) for
// queries (target xyz, light point xyz) on leaf triangles; 0 for triangles of no emitter.
__global__ void light_pdf_kernel(DeviceScene s, const float* __restrict__ queries, const uint32_t* __restrict__ leaf,
                                 uint64_t n, float* __restrict__ out)
{
	const uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
	if(i >= n)
	{
		return;
	}
	uint32_t emitter_plus_one = 0;
	const TriVerts lt = load_tri(s.tris, leaf[i], nullptr, &emitter_plus_one);
	if(emitter_plus_one == 0u || emitter_plus_one > s.num_emitters)
	{
		out[i] = 0.0f;
		return;
	}
	const EmitterRec e = s.emitters[emitter_plus_one - 1u];
	const float* q = queries + 6 * i;
	out[i] = light_triangle_pdf_w(e, lt, face_normal(lt), v3(q[3], q[4], q[5]), v3(q[0], q[1], q[2]));
}

}// end anonymous namespace

void RenderScene::light_pmf(float* out_pmf, double* out_alias_pmf, uint32_t* out_count) const
{
	require_same_device(m_geometry->device, "render scene");
	const uint32_t n = m_dev.num_emitters;
	if(out_count)
	{
		*out_count = n;
	}
	if(n == 0)
	{
		return;
	}
	std::vector<EmitterRec> emitters(n);
	std::vector<float2> alias(n);
	cudaStream_t st = library_stream();
	PG_CUDA_CHECK(cudaMemcpyAsync(emitters.data(), m_emitters.get(), n * sizeof(EmitterRec), cudaMemcpyDeviceToHost, st));
	PG_CUDA_CHECK(cudaMemcpyAsync(alias.data(), m_alias.get(), n * sizeof(float2), cudaMemcpyDeviceToHost, st));
	PG_CUDA_CHECK(cudaStreamSynchronize(st));
	if(out_pmf)
	{
		for(uint32_t k = 0; k < n; ++k)
		{
			out_pmf[k] = emitters[k].pmf;
		}
	}
	if(out_alias_pmf)
	{
		// alias_pick keeps column k with probability x and otherwise takes its alias: column k
		// gives 1/n x to itself and 1/n (1 - x) to its alias
		std::vector<double> p(n, 0.0);
		for(uint32_t k = 0; k < n; ++k)
		{
			uint32_t to = 0;
			std::memcpy(&to, &alias[k].y, sizeof(to));
			const double keep = std::min(1.0, std::max(0.0, static_cast<double>(alias[k].x)));
			p[k] += keep / n;
			if(to < n)
			{
				p[to] += (1.0 - keep) / n;
			}
		}
		std::copy(p.begin(), p.end(), out_alias_pmf);
	}
}

void RenderScene::light_pdf(const float* queries, const uint32_t* prims, uint64_t n, float* out_pdf_w) const
{
	require_same_device(m_geometry->device, "render scene");
	if(n == 0)
	{
		return;
	}
	// input triangle index -> leaf slot
	const std::size_t num_tris = m_geometry->tris.size();
	std::vector<LeafTri> leaf_tris(num_tris);
	cudaStream_t st = library_stream();
	PG_CUDA_CHECK(cudaMemcpyAsync(leaf_tris.data(), m_geometry->tris.get(), m_geometry->tris.bytes(), cudaMemcpyDeviceToHost, st));
	PG_CUDA_CHECK(cudaStreamSynchronize(st));
	std::vector<uint32_t> slot_of(num_tris, 0xFFFFFFFFu);
	for(std::size_t k = 0; k < num_tris; ++k)
	{
		if(leaf_tris[k].prim < num_tris)
		{
			slot_of[leaf_tris[k].prim] = static_cast<uint32_t>(k);
		}
	}
	std::vector<uint32_t> leaf(n);
	for(uint64_t i = 0; i < n; ++i)
	{
		if(prims[i] >= num_tris || slot_of[prims[i]] == 0xFFFFFFFFu)
		{
			throw Error(PG_ERR_INVALID_ARGUMENT, "light pdf query " + std::to_string(i) + ": triangle " +
			            std::to_string(prims[i]) + " is not in the scene (degenerate triangles are dropped)");
		}
		leaf[i] = slot_of[prims[i]];
	}
	DeviceBuffer<float> d_q(6 * n), d_out(n);
	DeviceBuffer<uint32_t> d_leaf(n);
	PG_CUDA_CHECK(cudaMemcpyAsync(d_q.get(), queries, d_q.bytes(), cudaMemcpyHostToDevice, st));
	PG_CUDA_CHECK(cudaMemcpyAsync(d_leaf.get(), leaf.data(), d_leaf.bytes(), cudaMemcpyHostToDevice, st));
	light_pdf_kernel<<<static_cast<unsigned>((n + 127) / 128), 128, 0, st>>>(m_dev, d_q.get(), d_leaf.get(), n, d_out.get());
	PG_CUDA_CHECK(cudaGetLastError());
	PG_CUDA_CHECK(cudaMemcpyAsync(out_pdf_w, d_out.get(), d_out.bytes(), cudaMemcpyDeviceToHost, st));
	PG_CUDA_CHECK(cudaStreamSynchronize(st));
}

void RenderScene::rebuild_bvh(uint32_t max_leaf_tris)
{
	require_same_device(m_geometry->device, "render scene");
	cudaStream_t st = library_stream();
	const std::size_t n = m_geometry->tris.size();
	// the resident triangles back in input order
	std::vector<LeafTri> leaf(n);
	PG_CUDA_CHECK(cudaMemcpyAsync(leaf.data(), m_geometry->tris.get(), m_geometry->tris.bytes(), cudaMemcpyDeviceToHost, st));
	PG_CUDA_CHECK(cudaStreamSynchronize(st));
	std::vector<float> tris(9 * n);
	std::vector<uint32_t> materials(n), emitters(n);
	for(const LeafTri& t : leaf)
	{
		if(t.prim >= n)
		{
			throw Error(PG_ERR_SCENE, "rebuild_bvh: leaf triangle with an out-of-range input index");
		}
		float* v = &tris[9 * static_cast<std::size_t>(t.prim)];
		v[0] = t.v0x; v[1] = t.v0y; v[2] = t.v0z;
		v[3] = t.v1x; v[4] = t.v1y; v[5] = t.v1z;
		v[6] = t.v2x; v[7] = t.v2y; v[8] = t.v2z;
		materials[t.prim] = t.material;
		emitters[t.prim] = t.emitter_plus_one;
	}
	BvhBuildInput in{tris.data(), materials.data(), emitters.data(), n, m_max_origin_abs};
	in.max_leaf_tris = max_leaf_tris;
	std::unique_ptr<Geometry> g = m_bvh_builder == PG_BVH_GPU_MORTON ? make_geometry_gpu(in) : make_geometry(in);

	// the emitters' triangle lists in the new leaf order, each sorted by input index as the
	// constructor sorts them (their offsets and counts do not change)
	PG_CUDA_CHECK(cudaMemcpyAsync(leaf.data(), g->tris.get(), g->tris.bytes(), cudaMemcpyDeviceToHost, st));
	PG_CUDA_CHECK(cudaStreamSynchronize(st));
	std::vector<std::vector<uint32_t>> per_emitter(m_dev.num_emitters);
	for(uint32_t k = 0; k < leaf.size(); ++k)
	{
		const uint32_t e = leaf[k].emitter_plus_one;
		if(e != 0u && e <= per_emitter.size())
		{
			per_emitter[e - 1].push_back(k);
		}
	}
	std::vector<uint32_t> emitter_tris;
	for(auto& list : per_emitter)
	{
		std::sort(list.begin(), list.end(), [&](uint32_t x, uint32_t y) { return leaf[x].prim < leaf[y].prim; });
		emitter_tris.insert(emitter_tris.end(), list.begin(), list.end());
	}
	if(!emitter_tris.empty())
	{
		PG_CUDA_CHECK(cudaMemcpyAsync(m_emitter_tris.get(), emitter_tris.data(), emitter_tris.size() * sizeof(uint32_t),
		                              cudaMemcpyHostToDevice, st));
		PG_CUDA_CHECK(cudaStreamSynchronize(st));
	}
	m_geometry = std::move(g);
	m_dev.nodes = m_geometry->nodes.get();
	m_dev.tris = m_geometry->tris.get();
	m_launch.leaf_tris = max_leaf_tris;
}

void RenderScene::set_launch(const LaunchConfig& c)
{
	if(c.capacity < 1024u || c.capacity > (1u << 24) || c.refill < 1u || c.refill > 32u || c.blocks_per_sm < 1u ||
	   c.blocks_per_sm > 64u || c.leaf_tris < 1u || c.leaf_tris > 3u)
	{
		throw Error(PG_ERR_INVALID_ARGUMENT, "launch config out of range (capacity 1024..2^24, refill 1..32, "
		                                     "blocks per SM 1..64, leaf triangles 1..3)");
	}
	if(c.leaf_tris != m_launch.leaf_tris)
	{
		rebuild_bvh(c.leaf_tris);
	}
	m_launch = c;
}

std::string RenderScene::fingerprint(const RenderParams& base) const
{
	uint32_t kinds[8] = {};
	for(uint32_t t : m_material_types)
	{
		++kinds[std::min<uint32_t>(t, 7u)];
	}
	std::string key = "tris=" + std::to_string(m_geometry->tris.size()) + ";res=" + std::to_string(base.width) + "x" +
	                  std::to_string(base.height) + ";emitters=" + std::to_string(m_dev.num_emitters) +
	                  ";env=" + std::to_string(m_dev.env_emitter >= 0 ? 1 : 0) + ";materials=";
	for(int k = 0; k < 4; ++k)
	{
		key += std::to_string(kinds[k]) + (k < 3 ? "," : "");
	}
	key += ";estimator=" + std::to_string(base.estimator) + ";bounces=" + std::to_string(base.max_bounces) +
	       ";filter=" + std::to_string(base.filter) + ";builder=" + std::to_string(m_bvh_builder);
	return key;
}

namespace
{

bool read_tuning(const char* path, const std::string& key, LaunchConfig* out)
{
	std::FILE* f = path ? std::fopen(path, "r") : nullptr;
	if(!f)
	{
		return false;
	}
	char line[1024];
	bool found = false;
	while(std::fgets(line, sizeof(line), f))
	{
		char k[900];
		LaunchConfig c;
		if(std::sscanf(line, "%899s %u %u %u %u", k, &c.capacity, &c.refill, &c.blocks_per_sm, &c.leaf_tris) == 5 &&
		   key == k)
		{
			*out = c;   // the last entry of a key wins
			found = true;
		}
	}
	std::fclose(f);
	return found;
}

void append_tuning(const char* path, const std::string& key, const LaunchConfig& c)
{
	std::FILE* f = path ? std::fopen(path, "a") : nullptr;
	if(!f)
	{
		throw Error(PG_ERR_INVALID_ARGUMENT, std::string("autotune: cannot write the cache file ") + path);
	}
	std::fprintf(f, "%s %u %u %u %u\n", key.c_str(), c.capacity, c.refill, c.blocks_per_sm, c.leaf_tris);
	std::fclose(f);
}

}// end anonymous namespace

AutotuneResult RenderScene::autotune(const RenderParams& base, bool rebuild, const char* cache_path, bool ignore_cache)
{
	require_same_device(m_geometry->device, "render scene");
	AutotuneResult result;
	const std::string key = fingerprint(base);
	if(cache_path && !ignore_cache)
	{
		LaunchConfig cached;
		if(read_tuning(cache_path, key, &cached))
		{
			set_launch(cached);
			result.config = m_launch;
			result.from_cache = true;
			return result;
		}
	}

	// calibration: the scene's own render at a few million paths (whole samples per pixel),
	// without guiding (its training would run during the calibration renders)
	const GuideParams guide_before = m_guide_params;
	m_guide_params.enabled = false;
	struct RestoreGuide
	{
		GuideParams& dst;
		GuideParams src;
		~RestoreGuide() { dst = src; }
	} restore_guide{m_guide_params, guide_before};
	const unsigned long long wh = static_cast<unsigned long long>(base.width) * base.height;
	RenderParams p = base;
	p.mode = PG_RENDER_GRAPH;
	p.progress = nullptr;
	p.capacity = 0;
	p.first_sample = 0;
	p.spp = static_cast<uint32_t>(std::max<unsigned long long>(1ull, std::min<unsigned long long>(
		base.spp, (16ull << 20) / std::max<unsigned long long>(1ull, wh))));
	DeviceBuffer<double> film(static_cast<std::size_t>(wh) * kFilmChannels);
	PG_CUDA_CHECK(cudaMemsetAsync(film.get(), 0, film.bytes(), m_stream));
	auto measure = [&](const LaunchConfig& c)
	{
		set_launch(c);
		float best = 0.0f;
		for(int rep = 0; rep < 3; ++rep)
		{
			const float ms = render(p, film.get());   // the first run also warms the graph up
			if(rep > 0 && (best == 0.0f || ms < best))
			{
				best = ms;
			}
			++result.trials;
		}
		return best;
	};

	descend(result, measure, rebuild && m_bvh_builder == PG_BVH_HOST_SAH);
	if(cache_path)
	{
		append_tuning(cache_path, key, result.config);
	}
	return result;
}

void RenderScene::descend(AutotuneResult& result, const std::function<float(const LaunchConfig&)>& measure,
                          bool leaf_size)
{
	LaunchConfig best = m_launch;
	float best_ms = measure(best);
	result.ms_default = best_ms;
	auto try_values = [&](uint32_t LaunchConfig::*field, std::initializer_list<uint32_t> values)
	{
		const uint32_t current = best.*field;
		for(uint32_t v : values)
		{
			if(v == current)
			{
				continue;
			}
			LaunchConfig c = best;
			c.*field = v;
			const float ms = measure(c);
			if(ms < best_ms * 0.99f)
			{
				best = c;
				best_ms = ms;
			}
		}
	};
	try_values(&LaunchConfig::capacity, {1u << 19, 1u << 20, 1u << 21, 1u << 22});
	try_values(&LaunchConfig::refill, {4u, 8u, 12u, 16u});
	try_values(&LaunchConfig::blocks_per_sm, {4u, 8u, 16u});
	if(leaf_size)
	{
		try_values(&LaunchConfig::leaf_tris, {1u, 2u, 3u});
	}
	set_launch(best);
	result.config = best;
	result.ms_tuned = best_ms;
}

AutotuneResult RenderScene::autotune_batch(const std::vector<const RenderScene*>& scenes, const std::vector<uint32_t>& spp,
                                           const RenderParams& params)
{
	// calibration: the batch at a sixteenth of its samples (at least one per scene), into scratch films
	std::vector<DeviceBuffer<double>> films;
	std::vector<double*> film_ptrs;
	std::vector<uint32_t> counts;
	std::vector<uint64_t> first(scenes.size(), 0);
	for(std::size_t k = 0; k < scenes.size(); ++k)
	{
		if(!scenes[k])
		{
			throw Error(PG_ERR_INVALID_ARGUMENT, "autotune_batch: missing scene");
		}
		films.emplace_back(static_cast<std::size_t>(scenes[k]->width()) * scenes[k]->height() * kFilmChannels);
		PG_CUDA_CHECK(cudaMemsetAsync(films.back().get(), 0, films.back().bytes(), m_stream));
		film_ptrs.push_back(films.back().get());
		counts.push_back(std::max<uint32_t>(1u, spp.at(k) / 16u));
	}
	AutotuneResult result;
	auto measure = [&](const LaunchConfig& c)
	{
		set_launch(c);
		float best = 0.0f;
		for(int rep = 0; rep < 3; ++rep)
		{
			const float ms = render_batch(scenes, film_ptrs, counts, first, params);
			if(rep > 0 && (best == 0.0f || ms < best))
			{
				best = ms;
			}
			++result.trials;
		}
		return best;
	};
	descend(result, measure, false);
	return result;
}

float RenderScene::render_batch(const std::vector<const RenderScene*>& scenes, const std::vector<double*>& films,
                                const std::vector<uint32_t>& spp, const std::vector<uint64_t>& first_sample,
                                const RenderParams& params)
{
	require_same_device(m_geometry->device, "render scene");
	const std::size_t n = scenes.size();
	if(n == 0 || films.size() != n || spp.size() != n || first_sample.size() != n)
	{
		throw Error(PG_ERR_INVALID_ARGUMENT, "render_batch: scenes, films, spp and first samples differ in number");
	}
	for(std::size_t k = 0; k < n; ++k)
	{
		if(!scenes[k] || !films[k] || spp[k] == 0)
		{
			throw Error(PG_ERR_INVALID_ARGUMENT, "render_batch: missing scene or film, or zero samples");
		}
		require_same_device(scenes[k]->m_geometry->device, "render_batch scene");
	}
	constexpr unsigned long long kMaxPaths = 1ull << 31;
	float ms = 0.0f;
	unsigned long long rays = 0, shadow = 0, iterations = 0, launches = 0;
	std::vector<BatchScene> chunk;
	unsigned long long acc = 0;
	auto flush = [&]
	{
		if(chunk.empty())
		{
			return;
		}
		RenderParams p = params;
		p.width = 1;
		p.height = 1;
		p.spp = 1;
		p.filter = PG_FILTER_BOX;
		p.first_sample = 0;
		p.progress = nullptr;
		ms += render_pass(p, nullptr, &chunk);
		rays += m_last_rays;
		shadow += m_last_shadow;
		iterations += m_last_iterations;
		launches += m_last_launches + chunk.size() - 1u;   // one box-weight launch per scene part
		chunk.clear();
		acc = 0;
	};
	for(std::size_t k = 0; k < n; ++k)
	{
		const RenderScene& sc = *scenes[k];
		const unsigned long long wh = static_cast<unsigned long long>(sc.m_dev.cam.width) * sc.m_dev.cam.height;
		if(wh == 0 || wh > kMaxPaths)
		{
			throw Error(PG_ERR_INVALID_ARGUMENT, "render_batch: a scene's resolution is empty or too large");
		}
		uint64_t sample = first_sample[k];
		uint32_t remaining = spp[k];
		while(remaining > 0)
		{
			const unsigned long long room = (kMaxPaths - acc) / wh;
			if(room == 0)
			{
				flush();
				continue;
			}
			const uint32_t take = static_cast<uint32_t>(std::min<unsigned long long>(remaining, room));
			BatchScene b;
			b.scene = sc.m_dev;
			b.film = make_film_view(films[k], sc.m_dev.cam.width, sc.m_dev.cam.height, PG_FILTER_BOX);
			b.path_first = acc;
			b.path_count = wh * take;
			b.first_global = sample * wh;
			b.width_height = static_cast<uint32_t>(wh);
			b.spp = take;
			chunk.push_back(b);
			acc += wh * take;
			sample += take;
			remaining -= take;
			if(chunk.size() == kMaxBatchScenes)
			{
				flush();
			}
		}
	}
	flush();
	m_last_rays = rays;
	m_last_shadow = shadow;
	m_last_iterations = iterations;
	m_last_launches = launches;
	return ms;
}

// Paths whose radiance a pass of a 4 x 4-filter render keeps (16 B each): larger renders are
// split into passes of whole samples per pixel.
constexpr unsigned long long kMaxFilteredPassPaths = 1ull << 27;
constexpr unsigned long long kMaxBoxPassPaths = 1ull << 31;

float RenderScene::render(const RenderParams& params, double* film_sums)
{
	require_same_device(m_geometry->device, "render scene");
	const unsigned long long wh = static_cast<unsigned long long>(params.width) * params.height;
	// passes of whole samples per pixel: 4 x 4 films keep every path's radiance for the pass; a
	// box film's pass only has to stay within the path numbering of one pass (2^31 paths)
	const unsigned long long max_pass = params.filter == PG_FILTER_BOX ? kMaxBoxPassPaths : kMaxFilteredPassPaths;
	if(wh == 0 || wh * params.spp <= max_pass)
	{
		return render_pass(params, film_sums);
	}
	const uint32_t pass_spp = static_cast<uint32_t>(std::max<unsigned long long>(1ull, max_pass / wh));
	float ms = 0.0f;
	unsigned long long rays = 0, shadow = 0, iterations = 0, launches = 0, counts[4] = {0, 0, 0, 0};
	double kernel_ms[7] = {0, 0, 0, 0, 0, 0, 0};
	for(uint32_t done = 0; done < params.spp; )
	{
		RenderParams p = params;
		p.spp = std::min(pass_spp, params.spp - done);
		p.first_sample = params.first_sample + done;
		ms += render_pass(p, film_sums);
		rays += m_last_rays;
		shadow += m_last_shadow;
		iterations += m_last_iterations;
		launches += m_last_launches;
		for(int k = 0; k < 4; ++k) { counts[k] += m_last_counts[k]; }
		for(int k = 0; k < 7; ++k) { kernel_ms[k] += m_kernel_ms[k]; }
		done += p.spp;
	}
	m_last_rays = rays;
	m_last_shadow = shadow;
	m_last_iterations = iterations;
	m_last_launches = launches;
	for(int k = 0; k < 4; ++k) { m_last_counts[k] = counts[k]; }
	for(int k = 0; k < 7; ++k) { m_kernel_ms[k] = kernel_ms[k]; }
	return ms;
}

float RenderScene::render_pass(const RenderParams& params, double* film_sums, const std::vector<BatchScene>* batch)
{
	const bool multi = batch != nullptr;
	if(params.width == 0 || params.height == 0 || params.spp == 0)
	{
		throw Error(PG_ERR_INVALID_ARGUMENT, "render: empty image or zero samples");
	}
	if(!multi && (params.width != m_dev.cam.width || params.height != m_dev.cam.height))
	{
		throw Error(PG_ERR_INVALID_ARGUMENT, "render: resolution differs from the camera's");
	}
	const unsigned long long wh = static_cast<unsigned long long>(params.width) * params.height;
	unsigned long long total = wh * params.spp;
	if(multi)
	{
		if(batch->empty() || batch->size() > kMaxBatchScenes || params.progress || params.filter != PG_FILTER_BOX ||
		   (m_guide_params.enabled && params.estimator == PG_EST_BNEEPT))
		{
			throw Error(PG_ERR_INVALID_ARGUMENT, "render: a multi-scene render takes 1..65536 box-filtered scenes, "
			                                     "without guiding or previews");
		}
		total = batch->back().path_first + batch->back().path_count;
	}
	if(total > 0xFFFFFFFFull)
	{
		throw Error(PG_ERR_INVALID_ARGUMENT, "render: more than 2^32 paths in one call; split the samples");
	}
	const LaunchConfig& lc = m_launch;
	const uint32_t capacity = static_cast<uint32_t>(std::min<unsigned long long>(params.capacity ? params.capacity
	                                                                                             : lc.capacity, total));
	const int sms = sm_count();
	const int grid = sms * static_cast<int>(lc.blocks_per_sm);   // grid-stride kernels: 128-thread blocks
	ensure_capacity(std::max<uint32_t>(capacity, 1024u), static_cast<uint32_t>(grid));
	const int refill = static_cast<int>(lc.refill);

	cudaStream_t st = m_stream;
	RenderCounters init{};
	init.total_paths = total;
	PG_CUDA_CHECK(cudaMemcpyAsync(m_counters.get(), &init, sizeof(init), cudaMemcpyHostToDevice, st));
	PathBuffers buf[2];
	for(int b = 0; b < 2; ++b)
	{
		buf[b] = PathBuffers{m_path[b].get(), m_meta[b].get(), m_thr[b].get(), m_rad[b].get(),
		                     m_prev[b].get(), m_ro[b].get(), m_rd[b].get()};
	}
	ShadowQueue sqs[2];
	for(int b = 0; b < 2; ++b)
	{
		sqs[b] = ShadowQueue{m_so[b].get(), m_sd[b].get(), m_sc[b].get()};
		sqs[b].r = m_sr[b].get();
	}
	BatchView bview;
	if(multi)
	{
		for(int b = 0; b < 2; ++b)
		{
			if(m_ssid[b].size() < m_capacity)
			{
				m_ssid[b].resize(m_capacity);
			}
			sqs[b].sid = m_ssid[b].get();
		}
		if(m_batch_table.size() < batch->size())
		{
			m_batch_table.resize(batch->size());
		}
		PG_CUDA_CHECK(cudaMemcpyAsync(m_batch_table.get(), batch->data(), batch->size() * sizeof(BatchScene),
		                              cudaMemcpyHostToDevice, st));
		bview = BatchView{m_batch_table.get(), static_cast<uint32_t>(batch->size())};
	}
	FilmView film = make_film_view(film_sums, params.width, params.height, params.filter);
	if(params.filter != PG_FILTER_BOX)
	{
		if(m_samples.size() < total)
		{
			m_samples.resize(total);
		}
		film.samples = m_samples.get();
	}
	const uint64_t first_global = params.first_sample * wh;
	const bool counting = params.mode == PG_RENDER_COUNT;
	// BVPTDL follows one BSDF-sampled bounce whatever the configured depth (BVPTDLEstimator.cpp:62-95)
	const uint32_t max_bounces = params.estimator == PG_EST_BVPTDL ? 1u : params.max_bounces;

	// learned guiding (BNEEPT only)
	const bool guided = m_guide_params.enabled && params.estimator == PG_EST_BNEEPT;
	// the vertices a guided render guides: those below this bounce (0: none)
	const uint32_t guide_depth = !guided ? 0u
	                             : (m_guide_params.depth == 0u || m_guide_params.depth > max_bounces ? max_bounces
	                                                                                                : m_guide_params.depth);
	const bool training = guided && m_guide_params.train;
	GuideArgs gargs;
	uint32_t train_cap = 0;
	if(guided)
	{
		ensure_guiding(m_capacity);
		train_cap = training ? std::max<uint32_t>(m_guide_params.batch, guide::kTile) : 0u;
		for(int b = 0; b < 2; ++b)
		{
			buf[b].gf0 = m_gf0[b].get();
			buf[b].gf1 = m_gf1[b].get();
		}
		if(training)
		{
			// NEE records name the training samples their unoccluded contribution is credited to
			sqs[0].t = m_st[0].get();
			sqs[1].t = m_st[1].get();
		}
		gargs.map = m_gmap.get();
		gargs.feat = m_gfeat.get();
		gargs.raw = m_graw.get();
		gargs.train_feat = m_tfeat.get();
		gargs.train_dirw = m_tdirw.get();
		gargs.train_cap = train_cap;
		gargs.alpha = m_guide_params.alpha;
		for(int a = 0; a < 3; ++a)
		{
			gargs.lo[a] = m_bound_lo[a];
			gargs.rcp[a] = m_bound_rcp[a];
		}
		PG_CUDA_CHECK(cudaMemsetAsync(m_gerr.get(), 0, sizeof(uint32_t), st));
		PG_CUDA_CHECK(cudaMemsetAsync(m_gscalars.get(), 0, 4 * sizeof(float), st));
	}
	RenderCounters* const d_counters = m_counters.get();
	// The NEE segments made by an iteration's shading are traced by the next iteration's
	// trace_kernel together with its closest-hit rays (one launch, one tail). Training runs in
	// periods of P = kTrainPeriod iterations (position q = iteration mod P):
	//   q = 0        guided vertices are marked;
	//   q = 1        the next vertex makes their training samples (the emission found there, and
	//                its NEE) and opens them;
	//   1 <= q < P-1 open samples collect the emission and NEE their paths gather; guided vertices
	//                also record their NEE directions as samples;
	//   q = P-1      open samples collect the emission found; the iteration ends with one Adam step.
	// The trace of q = 2 ... P-1 resolves the NEE of q = 1 ... P-2, so every credit lands before
	// the step. Without training the period is two iterations (the two path buffers).
	const int period = training ? kTrainPeriod : 2;
	GuideArgs gargs_of[kTrainPeriod];
	for(int q = 0; q < kTrainPeriod; ++q)
	{
		gargs_of[q] = gargs;
		if(training)
		{
			const bool mid = q >= 1 && q <= kTrainPeriod - 2;
			gargs_of[q].mark = q == 0 ? 1u : 0u;
			gargs_of[q].train_cap = mid ? train_cap : 0u;
			gargs_of[q].open = q >= 1 ? 1u : 0u;
			gargs_of[q].keep = mid ? 1u : 0u;
			gargs_of[q].nee_credit = mid ? 1u : 0u;
		}
	}

	// The launches of one iteration at position q of the period (path buffer q & 1); `ev`
	// (optional) brackets each with events.
	auto iteration = [&](int q, cudaEvent_t* ev)
	{
		const int b = q & 1;
		const PathBuffers& cur = buf[b];
		const PathBuffers& nxt = buf[1 - b];
		if(ev) { PG_CUDA_CHECK(cudaEventRecord(ev[0], st)); }
		// the training samples of a period start at q = 1
		prepare_kernel<<<1, 32, 0, st>>>(m_counters.get(), capacity, training ? static_cast<uint32_t>(q) : 2u,
		                                 train_cap / 4u * 3u);
		if(ev) { PG_CUDA_CHECK(cudaEventRecord(ev[1], st)); }
		if(multi)
		{
			regen_kernel<true><<<grid, kShadeBlock, 0, st>>>(m_counters.get(), m_dev.cam, film, params.seed, first_global,
			                                                 cur, bview);
		}
		else
		{
			regen_kernel<false><<<grid, kShadeBlock, 0, st>>>(m_counters.get(), m_dev.cam, film, params.seed, first_global,
			                                                  cur, bview);
		}
		if(ev) { PG_CUDA_CHECK(cudaEventRecord(ev[2], st)); }
		const ShadowQueue& sq = sqs[b];   // this iteration's NEE segments
		// closest hits of this iteration and the previous iteration's NEE segments (whose
		// unoccluded contributions, in a training render, are also credited to training samples)
		launch_trace(m_dev, d_counters, cur.ray_o, cur.ray_d, m_hits.get(), sqs[1 - b], cur.rad, film, refill, st,
		             counting, cur.meta, multi ? &bview : nullptr, sqs[1 - b].t ? m_tdirw.get() : nullptr);
		if(multi)
		{
			classify_kernel<true><<<grid, kShadeBlock, 0, st>>>(m_dev, d_counters, m_hits.get(), m_order.get(),
			                                                    m_order_list, cur.meta, bview, 0u);
		}
		else
		{
			classify_kernel<false><<<grid, kShadeBlock, 0, st>>>(m_dev, d_counters, m_hits.get(), m_order.get(),
			                                                     m_order_list, cur.meta, bview, guide_depth);
		}
		PG_CUDA_CHECK(cudaGetLastError());
		if(ev) { PG_CUDA_CHECK(cudaEventRecord(ev[3], st)); }
		const GuideArgs& gargs_b = gargs_of[q];
		if(guided)
		{
			// network inputs of this iteration's guidable vertices, then the tensor-core forward pass
			guide_query_kernel<<<grid, kShadeBlock, 0, st>>>(m_dev, d_counters, cur, m_hits.get(), gargs_b, guide_depth);
			PG_CUDA_CHECK(cudaGetLastError());
			guide::launch_forward(m_gimage.get(), m_gfeat.get(), capacity, nullptr, nullptr, m_gerr.get(), st,
			                      &d_counters->n_guided, m_graw.get());
		}
		if(ev) { PG_CUDA_CHECK(cudaEventRecord(ev[4], st)); }
		ShadeArgs sa{m_dev, cur, nxt, m_hits.get(), sq, m_counters.get(), film, params.seed, first_global,
		             max_bounces, params.estimator, static_cast<uint32_t>(wh)};
		sa.guide = gargs_b;
		sa.refine.mode = params.refine_mode;
		sa.refine.delta = params.refine_delta;
		sa.refine.iters = static_cast<int>(params.refine_iters);
		sa.refine_queue = RefineQueue{m_req_single.get(), m_req_mutual.get()};
		sa.order = m_order.get();
		sa.order_capacity = m_order_list;
		sa.batch = bview;
		if(multi)
		{
			shade_kernel<false, true><<<grid, kShadeBlock, 0, st>>>(sa);
		}
		else if(guided)
		{
			shade_kernel<true, false><<<grid, kShadeBlock, 0, st>>>(sa);
		}
		else
		{
			shade_kernel<false, false><<<grid, kShadeBlock, 0, st>>>(sa);
		}
		PG_CUDA_CHECK(cudaGetLastError());
		if(params.refine_mode == PG_REFINE_ITERATIVE)
		{
			if(multi)
			{
				refine_kernel<true><<<grid, kShadeBlock, 0, st>>>(m_dev, d_counters, nxt, sq, sa.refine_queue,
				                                                  static_cast<int>(params.refine_iters), bview);
			}
			else
			{
				refine_kernel<false><<<grid, kShadeBlock, 0, st>>>(m_dev, d_counters, nxt, sq, sa.refine_queue,
				                                                   static_cast<int>(params.refine_iters), bview);
			}
			PG_CUDA_CHECK(cudaGetLastError());
		}
		if(ev) { PG_CUDA_CHECK(cudaEventRecord(ev[5], st)); }
		if(ev) { PG_CUDA_CHECK(cudaEventRecord(ev[6], st)); }
		if(training && q == kTrainPeriod - 1)
		{
			// one Adam step on the period's samples, complete now; the new weights serve the
			// next period
			PG_CUDA_CHECK(cudaMemsetAsync(m_gscalars.get(), 0, sizeof(float), st));
			guide::launch_gradients(m_gparams.get(), m_gimage.get(), m_tfeat.get(), m_tdirw.get(), train_cap,
			                        m_traw.get(), reinterpret_cast<__nv_bfloat16*>(m_tacts.get()), m_ggrads.get(),
			                        m_gscalars.get(), m_gscalars.get() + 1, m_gerr.get(), st, &d_counters->n_train,
			                        m_guide_params.clamp);
			guide::launch_adam(m_gparams.get(), m_ggrads.get(), m_gm.get(), m_gv.get(), m_gstep.get(),
			                   m_guide_params.lr, st);
			guide::pack_image(m_gparams.get(), m_gimage.get(), st);
			guide_loss_kernel<<<1, 1, 0, st>>>(m_gscalars.get(), &d_counters->n_train);
			PG_CUDA_CHECK(cudaGetLastError());
		}
		if(ev) { PG_CUDA_CHECK(cudaEventRecord(ev[7], st)); }
	};

	// the box filter's W: spp per pixel, added once (film.cuh)
	auto add_box_weights = [&]
	{
		if(multi)
		{
			for(const BatchScene& b : *batch)
			{
				box_weights_kernel<<<sms * 4, 256, 0, st>>>(b.film.sums, b.width_height, static_cast<double>(b.spp));
				PG_CUDA_CHECK(cudaGetLastError());
			}
		}
		else if(params.filter == PG_FILTER_BOX)
		{
			box_weights_kernel<<<sms * 4, 256, 0, st>>>(film_sums, static_cast<uint32_t>(wh), static_cast<double>(params.spp));
			PG_CUDA_CHECK(cudaGetLastError());
		}
	};
	// the 4 x 4 filters: every path's radiance, kept per path during the pass, into the film
	auto splat_samples = [&]
	{
		if(params.filter != PG_FILTER_BOX)
		{
			splat_samples_kernel<<<grid, kShadeBlock, 0, st>>>(film, params.seed, first_global, static_cast<uint32_t>(total));
			PG_CUDA_CHECK(cudaGetLastError());
		}
	};

	if(!m_host_counters)
	{
		PG_CUDA_CHECK(cudaMallocHost(&m_host_counters, sizeof(RenderCounters)));
	}
	RenderCounters* const host_counters = m_host_counters;

	// a preview of the film at a batch boundary (the stream is idle there); see RenderProgress
	if(params.progress && m_inflight.size() < wh)
	{
		m_inflight.resize(wh);
	}
	auto publish_preview = [&](const RenderCounters& hc)
	{
		RenderProgress& pr = *params.progress;
		{
			std::lock_guard<std::mutex> lock(*pr.mutex);
			const uint32_t pixels = static_cast<uint32_t>(wh);
			const bool box = params.filter == PG_FILTER_BOX;
			if(box)
			{
				PG_CUDA_CHECK(cudaMemsetAsync(m_inflight.get(), 0, wh * sizeof(uint32_t), st));
				count_inflight_kernel<<<grid, kShadeBlock, 0, st>>>(buf[0].path, m_counters.get(), pixels, m_inflight.get());
				PG_CUDA_CHECK(cudaGetLastError());
			}
			develop_preview_kernel<<<grid, kShadeBlock, 0, st>>>(film_sums, m_inflight.get(), pixels, params.spp,
			                                                    hc.next_path, box ? 1 : 0, pr.preview_rgb);
			PG_CUDA_CHECK(cudaGetLastError());
			PG_CUDA_CHECK(cudaStreamSynchronize(st));
		}
		if(pr.published)
		{
			pr.published(hc.next_path - hc.n_next, total);
		}
	};
	cudaEvent_t e0, e1;
	PG_CUDA_CHECK(cudaEventCreate(&e0));
	PG_CUDA_CHECK(cudaEventCreate(&e1));
	unsigned long long iterations = 0;
	const unsigned long long max_iterations = 1ull << 25;
	bool done = false;
	for(double& k : m_kernel_ms) { k = 0.0; }

	if(params.mode == PG_RENDER_GRAPH)
	{
		// One graph = one period: two iterations (ping -> pong -> ping), four when training. The
		// launch sequence only depends on whether guiding and training run, so the executable
		// graph of the previous render is updated with this render's kernel arguments and
		// instantiated again only when its topology changed.
		cudaGraph_t graph;
		PG_CUDA_CHECK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
		for(int q = 0; q < period; ++q)
		{
			iteration(q, nullptr);
		}
		PG_CUDA_CHECK(cudaStreamEndCapture(st, &graph));
		const int key = (guided ? 1 : 0) | (training ? 2 : 0) | (multi ? 4 : 0);
		bool updated = false;
		if(m_exec && m_exec_key == key)
		{
			cudaGraphExecUpdateResultInfo info;
			updated = cudaGraphExecUpdate(m_exec, graph, &info) == cudaSuccess;
			if(!updated)
			{
				(void)cudaGetLastError();   // a failed update is not sticky; instantiate anew
			}
		}
		if(!updated)
		{
			if(m_exec)
			{
				PG_CUDA_CHECK(cudaGraphExecDestroy(m_exec));
				m_exec = nullptr;
			}
			PG_CUDA_CHECK(cudaGraphInstantiate(&m_exec, graph, 0));
			m_exec_key = key;
		}
		PG_CUDA_CHECK(cudaGraphDestroy(graph));
		cudaGraphExec_t exec = m_exec;
		PG_CUDA_CHECK(cudaEventRecord(e0, st));
		add_box_weights();
		int batch = 4;
		while(!done && iterations < max_iterations)
		{
			for(int k = 0; k < batch; ++k)
			{
				PG_CUDA_CHECK(cudaGraphLaunch(exec, st));
			}
			iterations += static_cast<unsigned long long>(period) * batch;
			PG_CUDA_CHECK(cudaMemcpyAsync(host_counters, m_counters.get(), sizeof(RenderCounters), cudaMemcpyDeviceToHost, st));
			PG_CUDA_CHECK(cudaStreamSynchronize(st));
			done = host_counters->next_path >= host_counters->total_paths && host_counters->n_next == 0 &&
			       host_counters->n_shadow == 0;
			if(host_counters->error)
			{
				break;
			}
			if(params.progress && !done)
			{
				publish_preview(*host_counters);
			}
			batch = std::min(batch * 2, 64);
		}
		splat_samples();
		PG_CUDA_CHECK(cudaEventRecord(e1, st));
		PG_CUDA_CHECK(cudaEventSynchronize(e1));
	}
	else
	{
		// Plain launches, one iteration at a time; in timing mode every kernel is bracketed by
		// events on the launching stream and the durations are summed per kernel.
		cudaEvent_t ev[8];
		const bool timing = params.mode == PG_RENDER_TIMING;
		for(cudaEvent_t& e : ev) { PG_CUDA_CHECK(cudaEventCreate(&e)); }
		PG_CUDA_CHECK(cudaEventRecord(e0, st));
		add_box_weights();
		while(!done && iterations < max_iterations)
		{
			iteration(static_cast<int>(iterations % static_cast<unsigned long long>(period)), timing ? ev : nullptr);
			++iterations;
			PG_CUDA_CHECK(cudaMemcpyAsync(host_counters, m_counters.get(), sizeof(RenderCounters), cudaMemcpyDeviceToHost, st));
			PG_CUDA_CHECK(cudaStreamSynchronize(st));
			if(timing)
			{
				// event pairs: prepare, regen, extend, guide inference, shade, shadow, guide training
				static const int slot[7] = {0, 1, 2, 5, 3, 4, 6};
				for(int k = 0; k < 7; ++k)
				{
					float ms = 0.0f;
					PG_CUDA_CHECK(cudaEventElapsedTime(&ms, ev[k], ev[k + 1]));
					m_kernel_ms[slot[k]] += ms;
				}
			}
			done = host_counters->next_path >= host_counters->total_paths && host_counters->n_next == 0 &&
			       host_counters->n_shadow == 0;
			if(host_counters->error)
			{
				break;
			}
		}
		splat_samples();
		PG_CUDA_CHECK(cudaEventRecord(e1, st));
		PG_CUDA_CHECK(cudaEventSynchronize(e1));
		for(cudaEvent_t& e : ev) { cudaEventDestroy(e); }
	}

	float ms = 0.0f;
	PG_CUDA_CHECK(cudaEventElapsedTime(&ms, e0, e1));
	cudaEventDestroy(e0);
	cudaEventDestroy(e1);
	const RenderCounters final_counters = *host_counters;

	m_last_rays = final_counters.rays_traced;
	m_last_shadow = final_counters.shadow_rays;
	m_last_iterations = iterations;
	{
		// prepare, regen, trace + classify (or extend + shadow), shade (+ refine in the iterative
		// mode); guide query + forward; training: weight sums (and clamp), forward, backward, Adam,
		// step, repack, loss
		const unsigned long long per_iteration = 5ull +
		                                         (params.refine_mode == PG_REFINE_ITERATIVE ? 1ull : 0ull) +
		                                         (guided ? 2ull : 0ull);
		const unsigned long long per_step = training ? (m_guide_params.clamp > 0.0f ? 8ull : 6ull) : 0ull;
		// + one training step per training period, + the film's box-weight or splat launch
		m_last_launches = iterations * per_iteration + iterations / kTrainPeriod * per_step + 1ull;
	}
	m_last_counts[0] = final_counters.nodes_closest;
	m_last_counts[1] = final_counters.tris_closest;
	m_last_counts[2] = final_counters.nodes_any;
	m_last_counts[3] = final_counters.tris_any;
	m_last_guided = final_counters.guided_total + final_counters.n_guided;
	if(guided)
	{
		uint32_t gerr = 0;
		float sc[4] = {0.0f, 0.0f, 0.0f, 0.0f};
		PG_CUDA_CHECK(cudaMemcpyAsync(sc, m_gscalars.get(), sizeof(sc), cudaMemcpyDeviceToHost, st));
		PG_CUDA_CHECK(cudaMemcpyAsync(&gerr, m_gerr.get(), sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
		PG_CUDA_CHECK(cudaStreamSynchronize(st));
		m_last_guide_loss = sc[3] > 0.0f ? sc[2] / sc[3] : 0.0f;
		if(gerr)
		{
			throw Error(PG_ERR_CUDA, "render: guiding network kernel timed out waiting on its tensor cores");
		}
	}
	if(final_counters.error & PG_DEV_ERR_STACK)
	{
		throw Error(PG_ERR_STACK_OVERFLOW, "render: BVH traversal stack overflow");
	}
	if(!done)
	{
		throw Error(PG_ERR_ITERATION_LIMIT, "render: iteration limit reached before all paths finished");
	}
	return ms;
}

}// end namespace pg
