// The engine behind the Photon C API (ph_c_core.h): SDL commands in, a GPU render out.
//
// Mirrors the reference Engine facade (Engine/Source/Core/Engine.cpp:43-190): commands are
// entered as text (phEnterCommand / phLoadCommands), phUpdate cooks the described scene into the
// GPU renderer's records (triangles in world space, materials, emitters, camera) and builds the
// BVH, phRender runs the estimator the visualizer names, and frames are developed from the FP64
// film on retrieval.
#pragma once

#include "film.cuh"
#include "pg_render.h"
#include "sdl.h"

#include <atomic>
#include <cstdint>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

namespace pg
{

struct RenderObject;
struct SceneDesc;

struct HdrFrame
{
	uint32_t width = 0, height = 0;
	std::vector<float> rgb;   // row-major, row 0 = bottom (the reference's frame layout)
};

struct RenderInfo
{
	double   device_ms = 0.0;      // device time of the last phRender (CUDA events)
	uint64_t paths = 0;
	uint64_t rays = 0;             // closest-hit rays
	uint64_t shadow_rays = 0;
	double   update_seconds = 0.0; // cooking + BVH build + upload of the last phUpdate
	uint64_t num_triangles = 0;
};

// The reference engine's global settings read at phInit from ./Config/EngineConfig.ini
// (EngineInitSettings::loadStandardConfig / load, Engine/Source/EngineInitSettings.cpp:13-72):
// the surface refiner's mode, self-intersection delta and number of bisection refinements.
// Engines created afterwards start from these values.
struct EngineSettings
{
	uint32_t refine_mode = 2;     // 0 manual, 1 empirical, 2 iterative (the reference default)
	float    refine_delta = 2e-4f;
	uint32_t refine_iters = 1;
};

EngineSettings& engine_settings();
// Parses an EngineConfig.ini (keys RefineMode, SelfIntersectDelta, NumIterativeSurfaceRefinements);
// returns false when the file cannot be read. Other keys are ignored.
bool load_engine_settings(const std::string& path, EngineSettings& out);

class Engine
{
public:
	Engine();
	~Engine();

	void enter_command(std::string_view fragment);
	bool load_commands(const std::string& path);
	void set_working_directory(const std::string& dir) { m_working_dir = dir; }
	void set_num_threads(uint32_t n) { m_num_threads = n; }

	// Cooks the scene and uploads it (phUpdate).
	void update();
	// Cooks the entered commands into renderer records without touching the GPU; throws on
	// unsupported or malformed input. Also fixes the render dimension, spp and estimator.
	void cook(SceneDesc& out);
	uint32_t spp() const { return m_spp; }
	uint32_t estimator() const { return m_estimator; }
	uint32_t sample_filter() const { return m_filter; }
	// Renders all samples of the current scene (phRender).
	void render();

	void get_render_dimension(uint32_t* w, uint32_t* h) const;
	// Develops the film into `frame` (resized when its dimensions differ).
	void retrieve_frame(HdrFrame& frame) const;
	// Developed sub-region into the frame's own coordinates (phAsyncPeekFrame).
	void peek_frame(uint32_t x, uint32_t y, uint32_t w, uint32_t h, HdrFrame& frame) const;

	// Progress for the async queries.
	void get_progress(uint64_t* total, uint64_t* done, uint64_t* elapsed_ms) const;
	void get_statistics(float* percentage, float* samples_per_second) const;

	// A frame region whose developed pixels changed (phAsyncPollUpdatedFrameRegion(s)): while a
	// render runs, the whole frame is reported UPDATING at every progress point (the film's
	// estimate over the samples finished so far, which phAsyncPeekFrame returns); when the render
	// completes, FINISHED. Every sample of a pass covers the whole frame, so regions are the whole
	// frame. The queue keeps at most kMaxQueuedRegions: further UPDATING regions are dropped,
	// FINISHED ones always kept (EqualSamplingRenderer::asyncAddUpdatedRegion,
	// Engine/Source/Core/Renderer/Sampling/EqualSamplingRenderer.cpp:240-254).
	struct RegionUpdate
	{
		uint32_t x, y, w, h;
		bool finished;
	};
	static constexpr std::size_t kMaxQueuedRegions = 1024;
	// Oldest first; returns the number written.
	std::size_t poll_regions(RegionUpdate* out, std::size_t max);
	// Everything queued, merged: at most one region (the frame), FINISHED if the last queued was.
	std::size_t poll_merged_regions(RegionUpdate* out, std::size_t max);

	// Extensions (ph_c_core.h, "GPU build extensions").
	void set_max_ray_bounces(uint32_t n) { m_max_bounces = n; }
	void set_seed(uint64_t seed) { m_seed = seed; }
	void set_sample_offset(uint64_t first_sample) { m_first_sample = first_sample; }
	// Learned path guiding of the BNEEPT estimator (network trained online during rendering).
	void set_guiding(bool enabled) { m_guiding = enabled; }
	void set_refine(uint32_t mode, float delta, uint32_t iters) { m_refine = EngineSettings{mode, delta, iters}; }
	// BVH builder used by the next update: 0 host binned SAH, 1 GPU Morton.
	void set_bvh_builder(uint32_t builder) { m_bvh_builder = builder; }
	// Environment (dome) densities: 0 as the reference computes them (default), 1 exact.
	void set_dome_pdf(uint32_t mode);
	// Path of an SDL resource identifier (":relative" to the working directory, "ext:/absolute").
	std::string resolve_resource(const std::string& identifier) const;
	const RenderInfo& info() const { return m_info; }
	uint64_t launch_count() const { return m_launches; }
	// Renders into a scratch film with the given render mode and returns the statistics of
	// phGpuProfileRender.
	void profile(uint32_t mode, uint32_t spp, double out_stats[14]);
	// Launch-shape autotuning of the updated scene (RenderScene::autotune) at the session's spp,
	// estimator and bounce cap.
	AutotuneResult autotune(const char* cache_path, uint32_t flags);
	std::string last_error() const;
	// Adds a message to the errors phGpuGetErrors reports.
	void report_error(const std::string& msg) { record_error(msg); }
	void clear_film();

private:
	void handle(SdlCommand&& cmd);
	void record_error(const std::string& msg);
	void push_region(bool finished);

	struct Resource
	{
		std::string category, type, name;
		std::vector<SdlClause> clauses;
		// actor transform, T * R * S (TDecomposedTransform, Math/Transform/TDecomposedTransform.h)
		double pos[3] = {0, 0, 0};
		double rot[4] = {1, 0, 0, 0};   // quaternion (w, x, y, z)
		double scale[3] = {1, 1, 1};
	};

	SdlParser m_parser;
	std::map<std::string, Resource> m_resources;   // key: name
	std::vector<std::string> m_actor_order;
	std::string m_working_dir = ".";
	uint32_t m_num_threads = 1;
	uint32_t m_max_bounces = 10000;
	uint64_t m_seed = 42;
	uint64_t m_first_sample = 0;
	bool m_guiding = false;
	EngineSettings m_refine = engine_settings();
	uint32_t m_bvh_builder = 0;
	uint32_t m_dome_pdf = 0;

	std::shared_ptr<RenderObject> m_render;
	uint32_t m_width = 0, m_height = 0;
	uint32_t m_spp = 0;
	uint32_t m_estimator = 0;
	uint32_t m_filter = PG_FILTER_BLACKMAN_HARRIS;   // the path-tracing visualizer's default

	RenderInfo m_info;
	uint64_t m_launches = 0;
	std::atomic<uint64_t> m_work_total{0}, m_work_done{0}, m_elapsed_ms{0};
	std::atomic<float> m_samples_per_second{0.0f};
	mutable std::mutex m_error_mutex;
	std::string m_errors;
	std::mutex m_region_mutex;
	std::deque<RegionUpdate> m_regions;
};

bool write_pfm(const std::string& path, const HdrFrame& frame);
bool read_pfm(const std::string& path, HdrFrame& frame);

}// end namespace pg
