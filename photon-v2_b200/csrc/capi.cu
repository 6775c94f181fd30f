// The Photon C API (include/ph_c_core.h) over the GPU engine. Each function follows the
// behaviour of its reference implementation in Engine/CEngine/Source/Api/ph_c_core.cpp: ids index
// process-wide tables, unknown ids are ignored, failures are logged.
#include "engine.h"
#include "pg_render.h"
#include "pg_runtime.h"

#include "../../include/ph_c_core.h"
#include "../../include/photon_gpu.h"

#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

using namespace pg;

namespace
{

struct Buffer
{
	std::vector<unsigned char> bytes;
};

struct EngineSlot
{
	Engine engine;
	std::string error_copy;
};

Registry<EngineSlot>& engines() { static Registry<EngineSlot> r; return r; }
Registry<HdrFrame>& frames() { static Registry<HdrFrame> r; return r; }
Registry<Buffer>& buffers() { static Registry<Buffer> r; return r; }

void log_error(const char* where, const std::exception& e)
{
	std::fprintf(stderr, "[photon-gpu] %s: %s\n", where, e.what());
}

}// end anonymous namespace

extern "C" {

void phConfigRendererResourceDirectory(const PhChar* /*directory*/)
{
	// The GPU renderer reads no resource files of its own.
}

PhBool phInit(void)
{
	try
	{
		require_device();
		library_stream();
		// the reference's engine settings file, when present (it is not created here)
		load_engine_settings("./Config/EngineConfig.ini", engine_settings());
		return PH_TRUE;
	}
	catch(const std::exception& e)
	{
		log_error("phInit", e);
		return PH_FALSE;
	}
}

PhBool phExit(void)
{
	return PH_TRUE;
}

void phCreateEngine(PhUInt64* const out_engineId, const PhUInt32 numRenderThreads)
{
	if(!out_engineId)
	{
		return;
	}
	auto slot = std::make_unique<EngineSlot>();
	slot->engine.set_num_threads(numRenderThreads);
	*out_engineId = engines().add(std::move(slot));
}

void phSetNumRenderThreads(PhUInt64 engineId, const PhUInt32 numRenderThreads)
{
	if(auto e = engines().get(engineId))
	{
		e->engine.set_num_threads(numRenderThreads);
	}
}

void phEnterCommand(PhUInt64 engineId, const PhChar* commandFragment)
{
	if(!commandFragment)
	{
		return;
	}
	if(auto e = engines().get(engineId))
	{
		e->engine.enter_command(commandFragment);
	}
}

PhBool phLoadCommands(PhUInt64 engineId, const PhChar* filePath)
{
	if(!filePath)
	{
		return PH_FALSE;
	}
	if(auto e = engines().get(engineId))
	{
		return e->engine.load_commands(filePath) ? PH_TRUE : PH_FALSE;
	}
	return PH_FALSE;
}

void phRender(PhUInt64 engineId)
{
	if(auto e = engines().get(engineId))
	{
		e->engine.render();
	}
}

void phUpdate(PhUInt64 engineId)
{
	if(auto e = engines().get(engineId))
	{
		e->engine.update();
	}
}

void phGetRenderDimension(PhUInt64 engineId, PhUInt32* out_widthPx, PhUInt32* out_heightPx)
{
	if(auto e = engines().get(engineId))
	{
		e->engine.get_render_dimension(out_widthPx, out_heightPx);
	}
}

void phGetObservableRenderData(PhUInt64 engineId, struct PHObservableRenderData* out_data)
{
	if(!out_data || !engines().get(engineId))
	{
		return;
	}
	std::memset(out_data, 0, sizeof(*out_data));
	std::snprintf(out_data->layers[0], PH_MAX_NAME_LENGTH + 1, "%s", "Main");
	std::snprintf(out_data->reals[0], PH_MAX_NAME_LENGTH + 1, "%s", "samples/s");
}

void phDeleteEngine(PhUInt64 engineId)
{
	engines().remove(engineId);
}

void phSetWorkingDirectory(PhUInt64 engineId, const PhChar* workingDirectory)
{
	if(!workingDirectory)
	{
		return;
	}
	if(auto e = engines().get(engineId))
	{
		e->engine.set_working_directory(workingDirectory);
	}
}

void phAquireFrame(PhUInt64 engineId, PhUInt64 channelIndex, PhUInt64 frameId)
{
	// The reference applies its tone mapper here (Engine::retrieveFrame(..., true),
	// Engine/Source/Core/Engine.cpp:167-190); the GPU build returns the linear frame.
	phAquireFrameRaw(engineId, channelIndex, frameId);
}

void phAquireFrameRaw(PhUInt64 engineId, PhUInt64 /*channelIndex*/, PhUInt64 frameId)
{
	auto e = engines().get(engineId);
	auto f = frames().get(frameId);
	if(e && f)
	{
		try
		{
			e->engine.retrieve_frame(*f);
		}
		catch(const std::exception& ex)
		{
			log_error("phAquireFrameRaw", ex);
		}
	}
}

void phCreateFrame(PhUInt64* out_frameId, PhUInt32 widthPx, PhUInt32 heightPx)
{
	if(!out_frameId)
	{
		return;
	}
	*out_frameId = 0;
	try
	{
		auto f = std::make_unique<HdrFrame>();
		f->width = widthPx;
		f->height = heightPx;
		f->rgb.assign(static_cast<std::size_t>(widthPx) * heightPx * 3, 0.0f);
		*out_frameId = frames().add(std::move(f));
	}
	catch(const std::exception& ex)
	{
		log_error("phCreateFrame", ex);   // no frame: the id stays 0
	}
}

void phGetFrameDimension(PhUInt64 frameId, PhUInt32* out_widthPx, PhUInt32* out_heightPx)
{
	if(auto f = frames().get(frameId))
	{
		if(out_widthPx) { *out_widthPx = f->width; }
		if(out_heightPx) { *out_heightPx = f->height; }
	}
}

void phGetFrameRgbData(PhUInt64 frameId, const PhFloat32** out_data)
{
	if(!out_data)
	{
		return;
	}
	if(auto f = frames().get(frameId))
	{
		*out_data = f->rgb.data();
	}
}

void phDeleteFrame(PhUInt64 frameId)
{
	frames().remove(frameId);
}

PhBool phLoadFrame(PhUInt64 frameId, const PhChar* filePath)
{
	auto f = frames().get(frameId);
	if(!f || !filePath)
	{
		return PH_FALSE;
	}
	try
	{
		return read_pfm(filePath, *f) ? PH_TRUE : PH_FALSE;
	}
	catch(const std::exception& ex)
	{
		log_error("phLoadFrame", ex);
		return PH_FALSE;
	}
}

PhBool phSaveFrame(PhUInt64 frameId, const PhChar* filePath, const PhFrameSaveInfo* /*saveInfo*/)
{
	auto f = frames().get(frameId);
	if(!f || !filePath)
	{
		return PH_FALSE;
	}
	const std::string path(filePath);
	if(path.size() < 4 || (path.substr(path.size() - 4) != ".pfm" && path.substr(path.size() - 4) != ".PFM"))
	{
		std::fprintf(stderr, "[photon-gpu] phSaveFrame: only .pfm output is supported (%s)\n", filePath);
		return PH_FALSE;
	}
	return write_pfm(path, *f) ? PH_TRUE : PH_FALSE;
}

PhBool phSaveFrameToBuffer(PhUInt64 frameId, PhUInt64 bufferId, PhBufferFormat format, const PhFrameSaveInfo* /*saveInfo*/)
{
	auto f = frames().get(frameId);
	auto b = buffers().get(bufferId);
	if(!f || !b || format != PH_BUFFER_FORMAT_FLOAT32_ARRAY)
	{
		return PH_FALSE;
	}
	b->bytes.resize(f->rgb.size() * sizeof(float));
	std::memcpy(b->bytes.data(), f->rgb.data(), b->bytes.size());
	return PH_TRUE;
}

void phFrameOpAbsDifference(PhUInt64 frameAId, PhUInt64 frameBId, PhUInt64 resultFrameId)
{
	auto a = frames().get(frameAId), b = frames().get(frameBId), r = frames().get(resultFrameId);
	if(!a || !b || !r || a->rgb.size() != b->rgb.size())
	{
		return;
	}
	r->width = a->width;
	r->height = a->height;
	r->rgb.resize(a->rgb.size());
	for(std::size_t i = 0; i < a->rgb.size(); ++i)
	{
		r->rgb[i] = std::fabs(a->rgb[i] - b->rgb[i]);
	}
}

PhFloat32 phFrameOpMSE(PhUInt64 expectedFrameId, PhUInt64 estimatedFramIde)
{
	auto a = frames().get(expectedFrameId), b = frames().get(estimatedFramIde);
	if(!a || !b || a->rgb.size() != b->rgb.size() || a->rgb.empty())
	{
		return 0.0f;
	}
	double sum = 0.0;
	for(std::size_t i = 0; i < a->rgb.size(); ++i)
	{
		const double d = static_cast<double>(a->rgb[i]) - b->rgb[i];
		sum += d * d;
	}
	return static_cast<PhFloat32>(sum / static_cast<double>(a->rgb.size()));
}

void phCreateBuffer(PhUInt64* out_bufferId)
{
	if(out_bufferId)
	{
		*out_bufferId = buffers().add(std::make_unique<Buffer>());
	}
}

void phGetBufferBytes(PhUInt64 bufferId, const PhUChar** out_bytesPtr, PhSize* out_numBytes)
{
	if(auto b = buffers().get(bufferId))
	{
		if(out_bytesPtr) { *out_bytesPtr = b->bytes.data(); }
		if(out_numBytes) { *out_numBytes = b->bytes.size(); }
	}
}

void phDeleteBuffer(PhUInt64 bufferId)
{
	buffers().remove(bufferId);
}

void phAsyncGetRenderProgress(PhUInt64 engineId, PhRenderProgress* out_progress)
{
	if(!out_progress)
	{
		return;
	}
	if(auto e = engines().get(engineId))
	{
		uint64_t total = 0, done = 0, ms = 0;
		e->engine.get_progress(&total, &done, &ms);
		out_progress->totalWork = total;
		out_progress->workDone = done;
		out_progress->elapsedMs = ms;
	}
}

void phAsyncGetRenderStatistics(PhUInt64 engineId, PhFloat32* out_percentageProgress, PhFloat32* out_samplesPerSecond)
{
	if(auto e = engines().get(engineId))
	{
		e->engine.get_statistics(out_percentageProgress, out_samplesPerSecond);
	}
}

void phAsyncGetRenderState(PhUInt64 engineId, struct PHRenderState* out_state)
{
	if(!out_state)
	{
		return;
	}
	std::memset(out_state, 0, sizeof(*out_state));
	if(auto e = engines().get(engineId))
	{
		float pct = 0.0f, sps = 0.0f;
		e->engine.get_statistics(&pct, &sps);
		out_state->reals[0] = sps;
	}
}

namespace
{

PhFrameRegionInfo to_region_info(const Engine::RegionUpdate& r)
{
	return PhFrameRegionInfo{r.x, r.y, r.w, r.h,
	                         r.finished ? PH_FRAME_REGION_STATUS_FINISHED : PH_FRAME_REGION_STATUS_UPDATING};
}

}// end anonymous namespace

PhBool phAsyncPollUpdatedFrameRegion(PhUInt64 engineId, PhFrameRegionInfo* out_regionInfo)
{
	auto e = engines().get(engineId);
	if(!e || !out_regionInfo)
	{
		return PH_FALSE;
	}
	Engine::RegionUpdate r{};
	if(e->engine.poll_regions(&r, 1) == 0)
	{
		return PH_FALSE;
	}
	*out_regionInfo = to_region_info(r);
	return PH_TRUE;
}

PhSize phAsyncPollUpdatedFrameRegions(PhUInt64 engineId, PhUInt64 /*bufferId*/, PhFrameRegionInfo* out_regionInfos,
                                      PhSize maxRegionInfos)
{
	auto e = engines().get(engineId);
	if(!e || maxRegionInfos == 0 || !out_regionInfos)
	{
		return 0;
	}
	std::vector<Engine::RegionUpdate> regions(std::min<PhSize>(maxRegionInfos, Engine::kMaxQueuedRegions + 1));
	const std::size_t n = e->engine.poll_regions(regions.data(), regions.size());
	for(std::size_t i = 0; i < n; ++i)
	{
		out_regionInfos[i] = to_region_info(regions[i]);
	}
	return n;
}

PhSize phAsyncPollMergedUpdatedFrameRegions(PhUInt64 engineId, PhUInt64 /*bufferId*/, PhSize /*mergeSize*/,
                                            PhFrameRegionInfo* out_regionInfos, PhSize maxRegionInfos)
{
	auto e = engines().get(engineId);
	if(!e || maxRegionInfos == 0 || !out_regionInfos)
	{
		return 0;
	}
	Engine::RegionUpdate r{};
	if(e->engine.poll_merged_regions(&r, 1) == 0)
	{
		return 0;
	}
	out_regionInfos[0] = to_region_info(r);
	return 1;
}

void phAsyncPeekFrame(PhUInt64 engineId, PhUInt64 layerIndex, PhUInt32 xPx, PhUInt32 yPx,
                      PhUInt32 widthPx, PhUInt32 heightPx, PhUInt64 frameId)
{
	phAsyncPeekFrameRaw(engineId, layerIndex, xPx, yPx, widthPx, heightPx, frameId);
}

void phAsyncPeekFrameRaw(PhUInt64 engineId, PhUInt64 /*layerIndex*/, PhUInt32 xPx, PhUInt32 yPx,
                         PhUInt32 widthPx, PhUInt32 heightPx, PhUInt64 frameId)
{
	auto e = engines().get(engineId);
	auto f = frames().get(frameId);
	if(e && f)
	{
		try
		{
			e->engine.peek_frame(xPx, yPx, widthPx, heightPx, *f);
		}
		catch(const std::exception& ex)
		{
			log_error("phAsyncPeekFrameRaw", ex);
		}
	}
}

PhBool phGpuGetErrors(PhUInt64 engineId, const PhChar** out_message)
{
	auto e = engines().get(engineId);
	if(!e)
	{
		return PH_FALSE;
	}
	e->error_copy = e->engine.last_error();
	if(out_message) { *out_message = e->error_copy.c_str(); }
	return e->error_copy.empty() ? PH_FALSE : PH_TRUE;
}

void phGpuSetMaxRayBounces(PhUInt64 engineId, PhUInt32 maxRayBounces)
{
	if(auto e = engines().get(engineId))
	{
		e->engine.set_max_ray_bounces(maxRayBounces);
	}
}

void phGpuSetSeed(PhUInt64 engineId, PhUInt64 seed)
{
	if(auto e = engines().get(engineId))
	{
		e->engine.set_seed(seed);
	}
}

void phGpuSetSurfaceRefine(PhUInt64 engineId, PhUInt32 mode, PhFloat32 selfIntersectDelta, PhUInt32 numIterations)
{
	if(auto e = engines().get(engineId))
	{
		if(mode <= 2u && selfIntersectDelta >= 0.0f && numIterations >= 1u)
		{
			e->engine.set_refine(mode, selfIntersectDelta, numIterations);
		}
	}
}

void phGpuSetBvhBuilder(PhUInt64 engineId, PhUInt32 builder)
{
	if(auto e = engines().get(engineId))
	{
		if(builder <= 1u)
		{
			e->engine.set_bvh_builder(builder);
		}
	}
}

void phGpuSetDomePdf(PhUInt64 engineId, PhUInt32 mode)
{
	if(auto e = engines().get(engineId))
	{
		if(mode <= 1u)
		{
			e->engine.set_dome_pdf(mode);
		}
	}
}

void phGpuSetGuiding(PhUInt64 engineId, PhBool enabled)
{
	if(auto e = engines().get(engineId))
	{
		e->engine.set_guiding(enabled == PH_TRUE);
	}
}

void phGpuClearFilm(PhUInt64 engineId)
{
	if(auto e = engines().get(engineId))
	{
		try
		{
			e->engine.clear_film();
		}
		catch(const std::exception& ex)
		{
			log_error("phGpuClearFilm", ex);
		}
	}
}

void phGpuGetRenderInfo(PhUInt64 engineId, PhFloat64* out_deviceMs, PhUInt64* out_paths, PhUInt64* out_rays,
                        PhUInt64* out_shadowRays, PhFloat64* out_updateSeconds)
{
	if(auto e = engines().get(engineId))
	{
		const RenderInfo& i = e->engine.info();
		if(out_deviceMs) { *out_deviceMs = i.device_ms; }
		if(out_paths) { *out_paths = i.paths; }
		if(out_rays) { *out_rays = i.rays; }
		if(out_shadowRays) { *out_shadowRays = i.shadow_rays; }
		if(out_updateSeconds) { *out_updateSeconds = i.update_seconds; }
	}
}

PhUInt64 phGpuGetLaunchCount(PhUInt64 engineId)
{
	auto e = engines().get(engineId);
	return e ? e->engine.launch_count() : 0;
}

void phGpuProfileRender(PhUInt64 engineId, PhUInt32 mode, PhUInt32 samplesPerPixel, PhFloat64* out_stats)
{
	auto e = engines().get(engineId);
	if(!e || !out_stats)
	{
		return;
	}
	try
	{
		e->engine.profile(mode, samplesPerPixel, out_stats);
	}
	catch(const std::exception& ex)
	{
		log_error("phGpuProfileRender", ex);
	}
}

PhBool phGpuAutotune(PhUInt64 engineId, const PhChar* cachePath, PhUInt32 flags, PhUInt32* outConfig,
                     PhFloat32* outMs)
{
	auto e = engines().get(engineId);
	if(!e)
	{
		return PH_FALSE;
	}
	try
	{
		const AutotuneResult a = e->engine.autotune(cachePath, flags);
		if(outConfig)
		{
			outConfig[0] = a.config.capacity;
			outConfig[1] = a.config.refill;
			outConfig[2] = a.config.blocks_per_sm;
			outConfig[3] = a.config.leaf_tris;
		}
		if(outMs)
		{
			outMs[0] = a.ms_default;
			outMs[1] = a.ms_tuned;
			outMs[2] = static_cast<float>(a.trials);
			outMs[3] = a.from_cache ? 1.0f : 0.0f;
		}
		return PH_TRUE;
	}
	catch(const std::exception& ex)
	{
		e->engine.report_error(std::string("autotune failed: ") + ex.what());
		return PH_FALSE;
	}
}

int pgpu_sdl_cook(const char* sdl_text, const char* working_dir, uint64_t* out_num_tris,
                  uint32_t* out_num_materials, uint32_t* out_num_emitters, uint32_t* out_dims,
                  float* out_tris, uint32_t* out_tri_material, uint32_t* out_tri_emitter,
                  float* out_emitters, float* out_camera)
{
	return guarded([&]
	{
		if(!sdl_text)
		{
			throw Error(PG_ERR_INVALID_ARGUMENT, "pgpu_sdl_cook: null text");
		}
		Engine e;
		if(working_dir)
		{
			e.set_working_directory(working_dir);
		}
		e.enter_command(sdl_text);
		e.enter_command(";");
		const std::string parse_errors = e.last_error();
		if(!parse_errors.empty())
		{
			throw Error(PG_ERR_SCENE, parse_errors);
		}
		SceneDesc d;
		e.cook(d);
		const uint64_t n = d.tris.size() / 9;
		if(out_num_tris) { *out_num_tris = n; }
		if(out_num_materials) { *out_num_materials = static_cast<uint32_t>(d.materials.size()); }
		if(out_num_emitters) { *out_num_emitters = static_cast<uint32_t>(d.emitters.size()); }
		if(out_dims)
		{
			e.get_render_dimension(&out_dims[0], &out_dims[1]);
			out_dims[2] = e.spp();
			out_dims[3] = e.estimator();
			out_dims[4] = e.sample_filter();
		}
		if(out_tris) { std::memcpy(out_tris, d.tris.data(), d.tris.size() * sizeof(float)); }
		if(out_tri_material) { std::memcpy(out_tri_material, d.tri_material.data(), n * sizeof(uint32_t)); }
		if(out_tri_emitter) { std::memcpy(out_tri_emitter, d.tri_emitter.data(), n * sizeof(uint32_t)); }
		if(out_emitters)
		{
			for(std::size_t k = 0; k < d.emitters.size(); ++k)
			{
				out_emitters[4 * k + 0] = d.emitters[k].r;
				out_emitters[4 * k + 1] = d.emitters[k].g;
				out_emitters[4 * k + 2] = d.emitters[k].b;
				out_emitters[4 * k + 3] = static_cast<float>(d.emitters[k].type);
			}
		}
		if(out_camera)
		{
			const Camera& c = d.camera;
			const float v[16] = {c.pos[0], c.pos[1], c.pos[2], c.axis_x[0], c.axis_x[1], c.axis_x[2],
			                     c.axis_y[0], c.axis_y[1], c.axis_y[2], c.axis_z[0], c.axis_z[1], c.axis_z[2],
			                     c.sensor_w, c.sensor_h, c.sensor_offset, static_cast<float>(d.env_area)};
			std::memcpy(out_camera, v, sizeof(v));
		}
	});
}

}// extern "C"
