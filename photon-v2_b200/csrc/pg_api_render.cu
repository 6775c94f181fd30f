// Render-scene entry points of the low-level C ABI (include/photon_gpu.h): a flat scene
// description in, FP64 film sums and developed frames out.
#include "pg_render_object.h"
#include "scene_build.h"

#include "../../include/photon_gpu.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <exception>
#include <thread>
#include <vector>

namespace pg
{

Registry<RenderObject>& render_registry()
{
	static Registry<RenderObject> r;
	return r;
}

namespace
{

std::shared_ptr<RenderObject> get_render(uint64_t id)
{
	auto r = render_registry().get(id);
	if(!r)
	{
		throw Error(PG_ERR_NOT_FOUND, "unknown scene id " + std::to_string(id));
	}
	return r;
}

}// end anonymous namespace

// Builds a RenderObject from flat arrays (shared with the Photon C API engine).
std::unique_ptr<RenderObject> make_render_object(SceneDesc&& desc)
{
	float max_abs = 1.0f;
	for(float v : desc.tris)
	{
		if(std::isfinite(v))
		{
			max_abs = std::max(max_abs, std::fabs(v));
		}
	}
	for(float v : desc.camera.pos)
	{
		max_abs = std::max(max_abs, std::fabs(v));
	}
	if(desc.has_env && desc.env_area <= 0.0)
	{
		const float origin[3] = {0.0f, 0.0f, 0.0f};
		desc.env_area = dome_area(desc.tris, origin);
	}
	auto obj = std::make_unique<RenderObject>();
	obj->scene = std::make_unique<RenderScene>(desc, max_abs);
	obj->width = desc.camera.width;
	obj->height = desc.camera.height;
	obj->film.resize(static_cast<std::size_t>(obj->width) * obj->height * kFilmChannels);
	PG_CUDA_CHECK(cudaMemsetAsync(obj->film.get(), 0, obj->film.bytes(), library_stream()));
	PG_CUDA_CHECK(cudaStreamSynchronize(library_stream()));
	return obj;
}

namespace
{

// RGB / W per pixel in FP64, rounded once to FP32; 0 where W is 0
// (HdrRgbFilm::developRegion, Engine/Source/Core/Filmic/HdrRgbFilm.cpp:167-205).
__global__ void develop_kernel(const double* __restrict__ sums, float* __restrict__ rgb, uint32_t num_pixels)
{
	for(uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < num_pixels; i += gridDim.x * blockDim.x)
	{
		const double4 s = reinterpret_cast<const double4*>(sums)[i];
		const double rcp = s.w == 0.0 ? 0.0 : 1.0 / s.w;
		rgb[3 * static_cast<size_t>(i) + 0] = static_cast<float>(s.x * rcp);
		rgb[3 * static_cast<size_t>(i) + 1] = static_cast<float>(s.y * rcp);
		rgb[3 * static_cast<size_t>(i) + 2] = static_cast<float>(s.z * rcp);
	}
}

}// end anonymous namespace

void develop_frame(const RenderObject& r, float* out_rgb, uint32_t x, uint32_t y, uint32_t w, uint32_t h)
{
	const uint32_t pixels = r.width * r.height;
	if(x >= r.width || y >= r.height || w == 0 || h == 0)
	{
		return;
	}
	w = std::min(w, r.width - x);
	h = std::min(h, r.height - y);
	std::lock_guard<std::mutex> lock(r.frame_mutex);
	cudaStream_t st = library_stream();
	const float* src = r.preview.get();
	if(!r.preview_valid)
	{
		r.frame.resize(static_cast<std::size_t>(pixels) * 3);
		develop_kernel<<<sm_count() * 4, 256, 0, st>>>(r.film.get(), r.frame.get(), pixels);
		PG_CUDA_CHECK(cudaGetLastError());
		src = r.frame.get();
	}
	const std::size_t pitch = static_cast<std::size_t>(r.width) * 3 * sizeof(float);
	const std::size_t offset = (static_cast<std::size_t>(y) * r.width + x) * 3;
	PG_CUDA_CHECK(cudaMemcpy2DAsync(out_rgb + offset, pitch, src + offset, pitch,
	                                static_cast<std::size_t>(w) * 3 * sizeof(float), h, cudaMemcpyDeviceToHost, st));
	PG_CUDA_CHECK(cudaStreamSynchronize(st));
}

void begin_preview(RenderObject& r)
{
	const uint32_t pixels = r.width * r.height;
	std::lock_guard<std::mutex> lock(r.frame_mutex);
	r.preview.resize(static_cast<std::size_t>(pixels) * 3);
	cudaStream_t st = library_stream();
	develop_kernel<<<sm_count() * 4, 256, 0, st>>>(r.film.get(), r.preview.get(), pixels);
	PG_CUDA_CHECK(cudaGetLastError());
	PG_CUDA_CHECK(cudaStreamSynchronize(st));
	r.preview_valid = true;
}

void end_preview(RenderObject& r)
{
	std::lock_guard<std::mutex> lock(r.frame_mutex);
	r.preview_valid = false;
}

void download_film(const RenderObject& r, double* out_sum)
{
	const std::size_t n = static_cast<std::size_t>(r.width) * r.height * kFilmChannels;
	PG_CUDA_CHECK(cudaMemcpyAsync(out_sum, r.film.get(), n * sizeof(double), cudaMemcpyDeviceToHost, library_stream()));
	PG_CUDA_CHECK(cudaStreamSynchronize(library_stream()));
}

}// end namespace pg

using namespace pg;

extern "C" {

int pgpu_scene_create(const float* tris, const uint32_t* tri_material, const uint32_t* tri_emitter,
                      uint64_t num_tris, const float* materials, uint32_t num_materials,
                      const float* emitters, uint32_t num_emitters, const float* camera, uint64_t* out_id)
{
	return pgpu_scene_create_ex(tris, tri_material, tri_emitter, num_tris, materials, num_materials, emitters,
	                            num_emitters, camera, PG_BVH_HOST_SAH, out_id);
}

int pgpu_scene_create_ex(const float* tris, const uint32_t* tri_material, const uint32_t* tri_emitter,
                         uint64_t num_tris, const float* materials, uint32_t num_materials,
                         const float* emitters, uint32_t num_emitters, const float* camera, uint32_t bvh_builder,
                         uint64_t* out_id)
{
	return guarded([&]
	{
		if(bvh_builder > PG_BVH_GPU_MORTON)
		{
			throw Error(PG_ERR_INVALID_ARGUMENT, "pgpu_scene_create_ex: unknown BVH builder");
		}
		if(!tris || num_tris == 0 || !tri_material || !materials || num_materials == 0 || !camera || !out_id ||
		   (num_emitters > 0 && !emitters))
		{
			throw Error(PG_ERR_INVALID_ARGUMENT, "pgpu_scene_create: missing input");
		}
		uint32_t w = 0, h = 0;
		checked_resolution(camera[10], camera[11], "pgpu_scene_create", &w, &h);
		SceneDesc d;
		d.tris.assign(tris, tris + 9 * num_tris);
		d.tri_material.assign(tri_material, tri_material + num_tris);
		d.tri_emitter.assign(num_tris, 0u);
		if(tri_emitter)
		{
			d.tri_emitter.assign(tri_emitter, tri_emitter + num_tris);
		}
		for(uint64_t i = 0; i < num_tris; ++i)
		{
			if(d.tri_material[i] >= num_materials)
			{
				throw Error(PG_ERR_INVALID_ARGUMENT, "pgpu_scene_create: material index out of range");
			}
			if(d.tri_emitter[i] > num_emitters)
			{
				throw Error(PG_ERR_INVALID_ARGUMENT, "pgpu_scene_create: emitter index out of range");
			}
		}
		for(uint32_t m = 0; m < num_materials; ++m)
		{
			const float* p = materials + 8 * m;
			const float type = p[0];
			if(type == 0.0f)      { d.materials.push_back(make_matte(p[1], p[2], p[3])); }
			else if(type == 1.0f) { d.materials.push_back(make_conductor(p[4], p[1], p[2], p[3])); }
			else if(type == 2.0f) { d.materials.push_back(make_dielectric(p[4], p[5], p[6])); }
			else
			{
				throw Error(PG_ERR_INVALID_ARGUMENT, "pgpu_scene_create: unknown material type");
			}
		}
		for(uint32_t e = 0; e < num_emitters; ++e)
		{
			const float* p = emitters + 4 * e;
			if(p[3] != static_cast<float>(PG_EMITTER_TRIANGLES) && p[3] != static_cast<float>(PG_EMITTER_ENV))
			{
				throw Error(PG_ERR_INVALID_ARGUMENT, "pgpu_scene_create: unknown emitter type");
			}
			EmitterRec rec{};
			rec.r = p[0]; rec.g = p[1]; rec.b = p[2];
			rec.type = static_cast<uint32_t>(p[3]);
			if(rec.type == PG_EMITTER_ENV)
			{
				if(d.has_env)
				{
					throw Error(PG_ERR_INVALID_ARGUMENT, "pgpu_scene_create: more than one environment");
				}
				d.has_env = true;
				d.env_rgb[0] = p[0]; d.env_rgb[1] = p[1]; d.env_rgb[2] = p[2];
			}
			d.emitters.push_back(rec);
		}
		d.camera = make_camera(camera, camera + 3, camera + 6, camera[9], w, h);
		d.bvh_builder = bvh_builder;
		*out_id = render_registry().add(make_render_object(std::move(d)));
	});
}

int pgpu_scene_destroy(uint64_t id)
{
	return guarded([&]
	{
		if(!render_registry().remove(id))
		{
			throw Error(PG_ERR_NOT_FOUND, "unknown scene id " + std::to_string(id));
		}
	});
}

int pgpu_scene_render(uint64_t id, uint32_t spp, uint32_t max_bounces, uint32_t estimator, uint64_t seed,
                      uint64_t first_sample, float* out_ms, uint64_t* out_rays, uint64_t* out_shadow_rays)
{
	return guarded([&]
	{
		auto r = get_render(id);
		if(estimator > PG_EST_BVPTDL)
		{
			throw Error(PG_ERR_INVALID_ARGUMENT, "pgpu_scene_render: unknown estimator");
		}
		RenderParams p;
		p.width = r->width;
		p.height = r->height;
		p.spp = spp;
		p.max_bounces = max_bounces;
		p.estimator = estimator;
		p.filter = r->filter;
		p.seed = seed;
		p.first_sample = first_sample;
		const float ms = r->scene->render(p, r->film.get());
		r->samples += spp;
		r->last_ms = ms;
		if(out_ms) { *out_ms = ms; }
		if(out_rays) { *out_rays = r->scene->last_rays(); }
		if(out_shadow_rays) { *out_shadow_rays = r->scene->last_shadow_rays(); }
	});
}

int pgpu_scene_profile(uint64_t id, uint32_t spp, uint32_t max_bounces, uint32_t estimator, uint64_t seed,
                       double* out_kernel_ms)
{
	return guarded([&]
	{
		auto r = get_render(id);
		if(estimator > PG_EST_BVPTDL)
		{
			throw Error(PG_ERR_INVALID_ARGUMENT, "pgpu_scene_profile: unknown estimator");
		}
		RenderParams p;
		p.width = r->width;
		p.height = r->height;
		p.spp = spp;
		p.max_bounces = max_bounces;
		p.estimator = estimator;
		p.filter = r->filter;
		p.seed = seed;
		p.mode = PG_RENDER_TIMING;
		DeviceBuffer<double> scratch(static_cast<std::size_t>(r->width) * r->height * kFilmChannels);
		PG_CUDA_CHECK(cudaMemsetAsync(scratch.get(), 0, scratch.bytes(), library_stream()));
		r->scene->render(p, scratch.get());
		if(out_kernel_ms)
		{
			for(int k = 0; k < 7; ++k)
			{
				out_kernel_ms[k] = r->scene->last_kernel_ms()[k];
			}
		}
	});
}

int pgpu_scenes_render_wavefront(const uint64_t* ids, uint32_t n, const uint32_t* spp, uint32_t max_bounces,
                                 uint32_t estimator, uint64_t seed, float* out_ms)
{
	return guarded([&]
	{
		if(n == 0)
		{
			if(out_ms) { *out_ms = 0.0f; }
			return;
		}
		if(!ids || !spp)
		{
			throw Error(PG_ERR_INVALID_ARGUMENT, "pgpu_scenes_render_wavefront: null ids or spp");
		}
		if(estimator > PG_EST_BVPTDL)
		{
			throw Error(PG_ERR_INVALID_ARGUMENT, "pgpu_scenes_render_wavefront: unknown estimator");
		}
		std::vector<std::shared_ptr<RenderObject>> objects;
		std::vector<const RenderScene*> scenes;
		std::vector<double*> films;
		std::vector<uint32_t> counts;
		std::vector<uint64_t> first;
		for(uint32_t i = 0; i < n; ++i)
		{
			for(uint32_t k = 0; k < i; ++k)
			{
				if(ids[k] == ids[i])
				{
					throw Error(PG_ERR_INVALID_ARGUMENT, "pgpu_scenes_render_wavefront: a scene appears twice");
				}
			}
			objects.push_back(get_render(ids[i]));
			RenderObject& r = *objects.back();
			if(r.filter != PG_FILTER_BOX)
			{
				throw Error(PG_ERR_INVALID_ARGUMENT, "pgpu_scenes_render_wavefront: every film must use the box filter");
			}
			if(spp[i] == 0)
			{
				throw Error(PG_ERR_INVALID_ARGUMENT, "pgpu_scenes_render_wavefront: zero samples");
			}
			scenes.push_back(r.scene.get());
			films.push_back(r.film.get());
			counts.push_back(spp[i]);
			first.push_back(r.samples);
		}
		RenderParams p;
		p.max_bounces = max_bounces;
		p.estimator = estimator;
		p.seed = seed;
		// the first scene's pool, stream and graphs run the wavefront of all of them
		const float ms = objects[0]->scene->render_batch(scenes, films, counts, first, p);
		for(uint32_t i = 0; i < n; ++i)
		{
			objects[i]->samples += spp[i];
		}
		if(out_ms) { *out_ms = ms; }
	});
}

int pgpu_scenes_autotune_wavefront(const uint64_t* ids, uint32_t n, const uint32_t* spp, uint32_t max_bounces,
                                   uint32_t estimator, uint32_t* out_config, float* out_ms)
{
	return guarded([&]
	{
		if(n == 0 || !ids || !spp)
		{
			throw Error(PG_ERR_INVALID_ARGUMENT, "pgpu_scenes_autotune_wavefront: no scenes");
		}
		if(estimator > PG_EST_BVPTDL)
		{
			throw Error(PG_ERR_INVALID_ARGUMENT, "pgpu_scenes_autotune_wavefront: unknown estimator");
		}
		std::vector<std::shared_ptr<RenderObject>> objects;
		std::vector<const RenderScene*> scenes;
		std::vector<uint32_t> counts(spp, spp + n);
		for(uint32_t i = 0; i < n; ++i)
		{
			objects.push_back(get_render(ids[i]));
			scenes.push_back(objects.back()->scene.get());
		}
		RenderParams p;
		p.max_bounces = max_bounces;
		p.estimator = estimator;
		p.seed = 0x2545F4914F6CDD1Dull;
		const AutotuneResult a = objects[0]->scene->autotune_batch(scenes, counts, p);
		if(out_config)
		{
			out_config[0] = a.config.capacity;
			out_config[1] = a.config.refill;
			out_config[2] = a.config.blocks_per_sm;
			out_config[3] = a.config.leaf_tris;
		}
		if(out_ms)
		{
			out_ms[0] = a.ms_default;
			out_ms[1] = a.ms_tuned;
			out_ms[2] = static_cast<float>(a.trials);
			out_ms[3] = 0.0f;
		}
	});
}

int pgpu_scenes_render(const uint64_t* ids, uint32_t n, const uint32_t* spp, uint32_t max_bounces,
                       uint32_t estimator, uint64_t seed, uint32_t concurrency, float* out_ms)
{
	return guarded([&]
	{
		if(n == 0)
		{
			if(out_ms) { *out_ms = 0.0f; }
			return;
		}
		if(!ids || !spp)
		{
			throw Error(PG_ERR_INVALID_ARGUMENT, "pgpu_scenes_render: null ids or spp");
		}
		if(estimator > PG_EST_BVPTDL)
		{
			throw Error(PG_ERR_INVALID_ARGUMENT, "pgpu_scenes_render: unknown estimator");
		}
		std::vector<std::shared_ptr<RenderObject>> objects;
		for(uint32_t i = 0; i < n; ++i)
		{
			for(uint32_t k = 0; k < i; ++k)
			{
				if(ids[k] == ids[i])
				{
					throw Error(PG_ERR_INVALID_ARGUMENT, "pgpu_scenes_render: a scene appears twice");
				}
			}
			objects.push_back(get_render(ids[i]));
		}
		int device = 0;
		PG_CUDA_CHECK(cudaGetDevice(&device));
		const uint32_t workers = std::max(1u, std::min(concurrency, n));
		ScopedEvent e0, e1;
		PG_CUDA_CHECK(cudaEventRecord(e0.get(), library_stream()));
		// scenes are handed out in order to `workers` host threads, each rendering on its scene's
		// own stream, so the scenes' kernels overlap on the device
		std::atomic<uint32_t> next{0};
		std::vector<std::exception_ptr> errors(workers);
		auto work = [&](uint32_t w)
		{
			try
			{
				PG_CUDA_CHECK(cudaSetDevice(device));
				for(uint32_t i = next++; i < n; i = next++)
				{
					RenderObject& r = *objects[i];
					RenderParams p;
					p.width = r.width;
					p.height = r.height;
					p.spp = spp[i];
					p.max_bounces = max_bounces;
					p.estimator = estimator;
					p.filter = r.filter;
					p.seed = seed;
					p.first_sample = r.samples;
					r.last_ms = r.scene->render(p, r.film.get());
					r.samples += spp[i];
				}
			}
			catch(...)
			{
				errors[w] = std::current_exception();
				next = n;   // hand out no further scenes
			}
		};
		std::vector<std::thread> pool;
		for(uint32_t w = 1; w < workers; ++w)
		{
			pool.emplace_back(work, w);
		}
		work(0);
		for(auto& t : pool)
		{
			t.join();
		}
		PG_CUDA_CHECK(cudaEventRecord(e1.get(), library_stream()));
		PG_CUDA_CHECK(cudaEventSynchronize(e1.get()));
		float ms = 0.0f;
		PG_CUDA_CHECK(cudaEventElapsedTime(&ms, e0.get(), e1.get()));
		for(const auto& e : errors)
		{
			if(e)
			{
				std::rethrow_exception(e);
			}
		}
		if(out_ms) { *out_ms = ms; }
	});
}

int pgpu_scene_light_pmf(uint64_t id, float* out_pmf, double* out_alias_pmf, uint32_t* out_num_emitters)
{
	return guarded([&]
	{
		auto r = get_render(id);
		r->scene->light_pmf(out_pmf, out_alias_pmf, out_num_emitters);
	});
}

int pgpu_scene_light_pdf(uint64_t id, const float* queries, const uint32_t* prims, uint64_t n, float* out_pdf_w)
{
	return guarded([&]
	{
		if(n > 0 && (!queries || !prims || !out_pdf_w))
		{
			throw Error(PG_ERR_INVALID_ARGUMENT, "pgpu_scene_light_pdf: null pointer");
		}
		if(n > (uint64_t(1) << 31))
		{
			throw Error(PG_ERR_INVALID_ARGUMENT, "pgpu_scene_light_pdf: too many queries in one call");
		}
		auto r = get_render(id);
		r->scene->light_pdf(queries, prims, n, out_pdf_w);
	});
}

int pgpu_scene_autotune(uint64_t id, uint32_t spp, uint32_t max_bounces, uint32_t estimator, uint32_t flags,
                        const char* cache_path, uint32_t* out_config, float* out_ms)
{
	return guarded([&]
	{
		auto r = get_render(id);
		if(estimator > PG_EST_BVPTDL || spp == 0)
		{
			throw Error(PG_ERR_INVALID_ARGUMENT, "pgpu_scene_autotune: unknown estimator or zero samples");
		}
		RenderParams p;
		p.width = r->width;
		p.height = r->height;
		p.spp = spp;
		p.max_bounces = max_bounces;
		p.estimator = estimator;
		p.filter = r->filter;
		const AutotuneResult a = r->scene->autotune(p, (flags & PG_AUTOTUNE_REBUILD) != 0u, cache_path,
		                                            (flags & PG_AUTOTUNE_IGNORE_CACHE) != 0u);
		if(out_config)
		{
			out_config[0] = a.config.capacity;
			out_config[1] = a.config.refill;
			out_config[2] = a.config.blocks_per_sm;
			out_config[3] = a.config.leaf_tris;
		}
		if(out_ms)
		{
			out_ms[0] = a.ms_default;
			out_ms[1] = a.ms_tuned;
			out_ms[2] = static_cast<float>(a.trials);
			out_ms[3] = a.from_cache ? 1.0f : 0.0f;
		}
	});
}

int pgpu_scene_set_launch(uint64_t id, const uint32_t* config)
{
	return guarded([&]
	{
		if(!config)
		{
			throw Error(PG_ERR_INVALID_ARGUMENT, "pgpu_scene_set_launch: null config");
		}
		auto r = get_render(id);
		r->scene->set_launch(LaunchConfig{config[0], config[1], config[2], config[3]});
	});
}

int pgpu_scene_get_launch(uint64_t id, uint32_t* out_config)
{
	return guarded([&]
	{
		if(!out_config)
		{
			throw Error(PG_ERR_INVALID_ARGUMENT, "pgpu_scene_get_launch: null config");
		}
		const LaunchConfig& c = get_render(id)->scene->launch();
		out_config[0] = c.capacity;
		out_config[1] = c.refill;
		out_config[2] = c.blocks_per_sm;
		out_config[3] = c.leaf_tris;
	});
}

int pgpu_scene_launches(uint64_t id, uint64_t* out_launches)
{
	return guarded([&]
	{
		auto r = get_render(id);
		if(out_launches) { *out_launches = r->scene->last_launches(); }
	});
}

int pgpu_scene_count(uint64_t id, uint32_t spp, uint32_t max_bounces, uint32_t estimator, uint64_t seed,
                     uint64_t* out_counts)
{
	return guarded([&]
	{
		auto r = get_render(id);
		if(estimator > PG_EST_BVPTDL || !out_counts)
		{
			throw Error(PG_ERR_INVALID_ARGUMENT, "pgpu_scene_count: unknown estimator or null output");
		}
		RenderParams p;
		p.width = r->width;
		p.height = r->height;
		p.spp = spp;
		p.max_bounces = max_bounces;
		p.estimator = estimator;
		p.filter = r->filter;
		p.seed = seed;
		p.mode = PG_RENDER_COUNT;
		DeviceBuffer<double> scratch(static_cast<std::size_t>(r->width) * r->height * kFilmChannels);
		PG_CUDA_CHECK(cudaMemsetAsync(scratch.get(), 0, scratch.bytes(), library_stream()));
		r->scene->render(p, scratch.get());
		out_counts[0] = r->scene->last_rays();
		out_counts[1] = r->scene->last_shadow_rays();
		for(int k = 0; k < 4; ++k) { out_counts[2 + k] = r->scene->last_counts()[k]; }
		out_counts[6] = r->scene->last_iterations();
	});
}

int pgpu_scene_film(uint64_t id, float* out_rgb, double* out_sum, uint64_t* out_spp)
{
	return guarded([&]
	{
		auto r = get_render(id);
		if(out_sum)
		{
			download_film(*r, out_sum);
		}
		if(out_rgb)
		{
			develop_frame(*r, out_rgb, 0, 0, r->width, r->height);
		}
		if(out_spp) { *out_spp = r->samples; }
	});
}

int pgpu_scene_set_dome_pdf(uint64_t id, uint32_t mode)
{
	return guarded([&]
	{
		auto r = get_render(id);
		if(mode > 1u)
		{
			throw Error(PG_ERR_INVALID_ARGUMENT, "pgpu_scene_set_dome_pdf: mode must be 0 or 1");
		}
		r->scene->set_dome_exact(mode == 1u);
	});
}

int pgpu_scene_set_filter(uint64_t id, uint32_t filter)
{
	return guarded([&]
	{
		auto r = get_render(id);
		if(filter > PG_FILTER_BLACKMAN_HARRIS)
		{
			throw Error(PG_ERR_INVALID_ARGUMENT, "pgpu_scene_set_filter: unknown sample filter");
		}
		r->filter = filter;
		PG_CUDA_CHECK(cudaMemsetAsync(r->film.get(), 0, r->film.bytes(), library_stream()));
		PG_CUDA_CHECK(cudaStreamSynchronize(library_stream()));
		r->samples = 0;
	});
}

int pgpu_scene_clear(uint64_t id)
{
	return guarded([&]
	{
		auto r = get_render(id);
		PG_CUDA_CHECK(cudaMemsetAsync(r->film.get(), 0, r->film.bytes(), library_stream()));
		PG_CUDA_CHECK(cudaStreamSynchronize(library_stream()));
		r->samples = 0;
	});
}

int pgpu_scene_set_guiding(uint64_t id, int enabled, int train, float alpha, float lr, uint32_t batch)
{
	return guarded([&]
	{
		auto r = get_render(id);
		if(!(alpha > 0.0f && alpha < 1.0f) || !(lr > 0.0f) || batch == 0 || batch > (1u << 22))
		{
			throw Error(PG_ERR_INVALID_ARGUMENT, "pgpu_scene_set_guiding: alpha must lie in (0, 1), lr > 0, "
			                                     "0 < batch <= 2^22");
		}
		GuideParams g = r->scene->guiding();
		g.enabled = enabled != 0;
		g.train = train != 0;
		g.alpha = alpha;
		g.lr = lr;
		g.batch = batch;
		r->scene->set_guiding(g);
	});
}

int pgpu_scene_set_guiding_depth(uint64_t id, uint32_t depth)
{
	return guarded([&]
	{
		auto r = get_render(id);
		GuideParams g = r->scene->guiding();
		g.depth = depth;
		r->scene->set_guiding(g);
	});
}

int pgpu_scene_guide_reset(uint64_t id)
{
	return guarded([&]
	{
		get_render(id)->scene->reset_guiding();
	});
}

int pgpu_scene_guide_info(uint64_t id, float* out_loss, uint64_t* out_guided_vertices, double* out_kernel_ms,
                          float* out_params)
{
	return guarded([&]
	{
		auto r = get_render(id);
		const RenderScene& rs = *r->scene;
		if(out_loss) { *out_loss = rs.last_guide_loss(); }
		if(out_guided_vertices) { *out_guided_vertices = rs.last_guided_vertices(); }
		if(out_kernel_ms)
		{
			for(int k = 0; k < 7; ++k)
			{
				out_kernel_ms[k] = rs.last_kernel_ms()[k];
			}
		}
		if(out_params) { rs.guide_params(out_params); }
	});
}

}// extern "C"
