// Wavefront path tracer: scene records, per-path state in HBM, and the render driver.
//
// One render = W x H x spp independent paths of the BNEEPT (or BVPT) estimator. Paths live in a
// fixed-capacity pool of slots; every iteration
//   prepare  -> compacts bookkeeping and decides how many new camera paths join,
//   regen    -> writes the new camera rays into the free tail of the ray queue,
//   extend   -> closest hit for every queued ray (pg_trace.cu),
//   shade    -> emission / NEE / BSDF sampling / Russian roulette per hit, writing continuing
//               paths compacted (warp-aggregated) into the other buffer and shadow rays into the
//               shadow queue,
//   shadow   -> any hit for the shadow queue; unoccluded contributions are added to the path
//               (or straight to the film for paths that ended at that vertex),
// and the buffers swap. Two iterations (ping and pong) are captured in one CUDA graph.
#pragma once

#include "bsdf.cuh"
#include "env.cuh"
#include "film.cuh"
#include "pg_common.cuh"
#include "pg_geometry.h"

#include <cstdint>
#include <functional>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

namespace pg
{

enum EmitterType : uint32_t
{
	PG_EMITTER_TRIANGLES = 0,   // a group of triangles with one constant radiance
	PG_EMITTER_ENV = 1,         // constant environment radiance (the dome)
};

// 32-byte emitter record.
struct alignas(16) EmitterRec
{
	float    r, g, b;        // emitted radiance
	uint32_t type;
	uint32_t first;          // first entry in the emitter-triangle list
	uint32_t count;          // number of triangles
	float    pmf;            // pick probability (power-proportional)
	float    rcp_count;
};

// Pinhole camera: raster -> sensor -> world, as SingleLensObserver builds it
// (Engine/Source/EngineEnv/Observer/SingleLensObserver.cpp:30-80,
//  Engine/Source/EngineEnv/Observer/OrientedRasterObserver.cpp:48-100) and as
// PinholeCamera::receiveRay uses it (Engine/Source/Core/Receiver/PinholeCamera.cpp:26-62).
struct Camera
{
	float pos[3];
	float axis_x[3], axis_y[3], axis_z[3];   // camera-to-world rotation columns
	float sensor_w, sensor_h, sensor_offset; // metres
	uint32_t width, height;
};

enum Estimator : uint32_t
{
	PG_EST_BNEEPT = 0,
	PG_EST_BVPT = 1,
	PG_EST_BVPTDL = 2,   // zero- and one-bounce emission only (BVPTDLEstimator.cpp:21-96)
};

enum RenderMode : uint32_t
{
	PG_RENDER_GRAPH = 0,    // iterations captured in a CUDA graph (the production path)
	PG_RENDER_TIMING = 1,   // plain launches with per-kernel CUDA events (profiling)
	PG_RENDER_COUNT = 2,    // plain launches, traversal kernels count nodes and triangles
};

// Progress of a render while it runs (graph mode). At every batch boundary -- the scene's stream
// idle, every kernel of the batch complete, so the film holds exactly what finished paths put
// there -- the film's estimate over the samples finished so far is developed into preview_rgb
// (device memory, [h][w][3] float32, RGB / W with the box film's W counting finished samples
// only) while `mutex` is held, and then `published` is called with the paths finished so far and
// the total of the render call. The callback runs on the rendering thread.
struct RenderProgress
{
	std::mutex* mutex = nullptr;
	float* preview_rgb = nullptr;
	std::function<void(unsigned long long finished, unsigned long long total)> published;
};

// Launch shapes of a scene's renders. The defaults were picked by hand on the 1M-triangle GGX
// scene; RenderScene::autotune picks them per scene from short calibration renders.
struct LaunchConfig
{
	uint32_t capacity = 1u << 21;   // path slots in flight (the wavefront's queue depth)
	uint32_t refill = 8;            // idle lanes that make a traversal warp fetch new rays
	uint32_t blocks_per_sm = 8;     // 128-thread blocks per SM of the grid-stride kernels
	uint32_t leaf_tris = 3;         // triangles per BVH leaf at most (host SAH tree; 1..3)
};

// What RenderScene::autotune found: the chosen shapes and the calibration render's device
// milliseconds with the defaults and with the choice.
struct AutotuneResult
{
	LaunchConfig config;
	float ms_default = 0.0f;
	float ms_tuned = 0.0f;
	uint32_t trials = 0;
	bool from_cache = false;
};

struct RenderParams
{
	uint32_t width = 0, height = 0;
	uint32_t spp = 1;
	uint32_t max_bounces = 10000;       // MAX_RAY_BOUNCES of the reference estimators
	uint32_t estimator = PG_EST_BNEEPT;
	uint32_t filter = PG_FILTER_BOX;    // SampleFilterType of the film being rendered into
	uint64_t seed = 42;
	uint64_t first_sample = 0;          // sample index offset (resume / replicas)
	uint32_t capacity = 0;              // path slots in flight (0: the scene's LaunchConfig)
	uint32_t mode = PG_RENDER_GRAPH;
	// SurfaceHitRefinery settings (the reference's EngineInitSettings: RefineMode,
	// SelfIntersectDelta, NumIterativeSurfaceRefinements): 0 manual, 1 empirical, 2 iterative.
	uint32_t refine_mode = 2;
	float    refine_delta = 2e-4f;
	uint32_t refine_iters = 1;
	RenderProgress* progress = nullptr;  // previews and progress during the render (graph mode only)
};

// Learned path guiding (BNEEPT only). At Lambertian vertices the direction is drawn from the
// network's vMF mixture with probability alpha, else from the BSDF, and weighted by the one-sample
// MIS density alpha q + (1 - alpha) p_bsdf, which keeps the estimator unbiased. With training on,
// every iteration records up to `batch` (vertex, direction, incident radiance) samples and takes
// one Adam step on them, so the network keeps learning across renders of the scene.
struct GuideParams
{
	bool     enabled = false;
	bool     train = true;
	float    alpha = 0.5f;
	float    lr = 1e-2f;
	uint32_t batch = 16384;
	float    clamp = 10.0f;     // training weights capped at clamp x the batch mean (0 = off)
	uint32_t depth = 1;         // vertices guided: the first `depth` of each path (0 = every vertex)
};

// Host-side scene description handed to the renderer.
struct SceneDesc
{
	std::vector<float>    tris;           // [n][3][3]
	std::vector<uint32_t> tri_material;   // [n]
	std::vector<uint32_t> tri_emitter;    // [n] emitter index + 1 (0 = none)
	std::vector<Material> materials;
	std::vector<EmitterRec> emitters;     // pmf / first / count filled by the scene builder
	float env_rgb[3] = {0.0f, 0.0f, 0.0f};
	bool  has_env = false;
	// An image dome larger than 1 x 1: linear sRGB radiance [env_height][env_width][3], row 0 at the
	// bottom (looking down), and the dome's local-to-world rotation (row-major). Empty: the
	// environment is the constant env_rgb.
	std::vector<float> env_image;
	uint32_t env_width = 0, env_height = 0;
	float env_rot[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
	float env_center[3] = {0.0f, 0.0f, 0.0f};   // dome centre (its actor position)
	// Surface area of the dome sphere (4 pi r^2, r = 1.01 x the farthest scene-bound corner from
	// the dome centre, ADome.cpp:45-60); the environment's flux approximation is its luminance
	// times this area (LatLongEnvEmitter.cpp:36-68), which sets its share of NEE samples.
	double env_area = 0.0;
	Camera camera{};
	uint32_t bvh_builder = 0;   // BvhBuilder: 0 host binned SAH, 1 GPU Morton
};

// Device view of a scene (all pointers are device memory).
struct DeviceScene
{
	const WideNode*   nodes;
	const LeafTri*    tris;
	const Material*   materials;
	const EmitterRec* emitters;
	const uint32_t*   emitter_tris;     // leaf triangle indices, grouped per emitter
	const float2*     alias;            // per emitter: (accept probability, alias index bits)
	uint32_t          num_emitters;
	int32_t           env_emitter;      // index of the environment emitter or -1
	EnvMap            env_map;          // the dome (a constant environment is a 1 x 1 image)
	Camera            cam;
};

// Shading classes of a closest-hit result: 0 = miss, then 1 + the hit surface's material type
// (matte, conductor, dielectric, absorber), and last the matte vertices that a guided render
// guides (kGuidedClass), whose shading also evaluates and samples the learned mixture: kept apart,
// they fill whole warps instead of making every matte warp wait on its guided lanes.
// classify_kernel lists the queue slots of each class so that the shading kernel's warps mostly
// run one code path. Each class has kClassLists lists, one per residue of the block index, so that
// the list counters' atomics spread over kOrderLists addresses instead of queuing on six.
constexpr uint32_t kShadeClasses = 6;
constexpr uint32_t kGuidedClass = kShadeClasses - 1u;
constexpr uint32_t kClassLists = 16;
constexpr uint32_t kOrderLists = kShadeClasses * kClassLists;

// Counters shared by the kernels of one render (device memory).
struct alignas(16) RenderCounters
{
	uint32_t n_active;      // continuing paths at the head of the current queue
	uint32_t n_total;       // n_active + newly generated paths this iteration
	uint32_t n_next;        // compaction counter of the next queue
	uint32_t n_shadow;      // shadow queue length (records made this iteration)
	unsigned long long next_path;   // next path index to generate
	unsigned long long total_paths;
	unsigned long long gen_base;    // first path index generated this iteration
	unsigned long long rays_traced; // closest-hit rays (extension + camera)
	unsigned long long shadow_rays;
	unsigned long long nodes_closest, tris_closest;   // counting mode only
	unsigned long long nodes_any, tris_any;
	unsigned long long guided_total;   // guided vertices over the whole render
	uint32_t error;
	uint32_t pad;
	uint32_t fetch_extend;   // dynamic-fetch cursors of the persistent traversal kernels,
	uint32_t fetch_shadow;   // zeroed by prepare_kernel at the start of every iteration
	uint32_t n_guided;       // guided vertices this iteration (network rows)
	uint32_t n_train;        // training samples recorded this iteration (may exceed the batch)
	uint32_t n_shadow_prev;  // records made by the previous iteration, traced by this one's trace_kernel
	uint32_t n_class[kOrderLists];   // closest-hit results per shading-class list (classify_kernel)
	uint32_t n_refine;       // surface-refinery requests this iteration: one-sided escapes
	uint32_t n_refine_mutual;// and escapes towards a light-triangle point
	uint32_t n_marked;       // guided vertices marked for training samples in this training period
	float    rec_keep;       // probability that a marked vertex's sample is recorded (fits the batch)
};

// Surface-refinery requests of one iteration (iterative refine mode). The shading kernel leaves
// the hit point and triangle in the ray slot it fills and queues the slot; the refinery kernel
// replaces them with the refined origin and range. `single` entries are (slot | kind << 31):
// kind 0 = a continuation ray in the next path buffer, 1 = a shadow ray towards a direction
// (environment light); `mutual` entries are shadow rays towards a point on a light triangle.
struct RefineQueue
{
	uint32_t* single;
	uint32_t* mutual;
};

// Per-path state, one buffer of the ping-pong pair (structure of arrays).
struct PathBuffers
{
	uint32_t* path;     // global path index
	uint32_t* meta;     // bounce (bits 0-7) | flags
	float4*   thr;      // throughput used for emission at this vertex (rgb), continuation factor (w)
	float4*   rad;      // accumulated radiance (rgb), BSDF pdf of the ray that led here (w)
	float4*   prev;     // previous vertex position (xyz), Russian-roulette scale (w)
	float4*   ray_o;    // origin, tmin
	float4*   ray_d;    // direction, tmax
	float4*   gf0;      // guiding record of the previous vertex: features 0-3
	float4*   gf1;      // features 4-6, |cos| / pdf of the sampled direction (guided renders only)
};

struct ShadowQueue
{
	float4* o;          // origin, tmin
	float4* d;          // direction, tmax
	float4* c;          // contribution rgb, target (slot in next buffer, or 0x80000000|pixel)
	float4* t;          // guided renders: two training samples (index bits, or ~0; weight added if unoccluded):
	                    // the previous vertex's sample, and this vertex's own NEE-direction sample
	float2* r;          // filtered films: raster position of the sample a final contribution belongs to
	uint32_t* sid;      // multi-scene renders: the scene of each record
};

// One scene of a multi-scene render: its device records, film, and where its paths sit in the
// render's path numbering (scene k owns batch paths [path_first, path_first + path_count); a
// path's sample draws use its index within the scene, offset by first_global, so every scene
// gets the paths its own render would).
struct BatchScene
{
	DeviceScene scene;
	FilmView    film;
	unsigned long long path_first;
	unsigned long long path_count;
	unsigned long long first_global;
	uint32_t    width_height;
	uint32_t    spp;
};

// The scene table of a multi-scene render (device memory).
struct BatchView
{
	const BatchScene* scenes = nullptr;
	uint32_t count = 0;
};

// Device view of the guiding buffers for one render iteration.
struct GuideArgs
{
	uint32_t*       map = nullptr;        // queue entry -> network row, 0xFFFFFFFF = not guided
	float*          feat = nullptr;       // [capacity][8] network input rows
	const float*    raw = nullptr;        // [capacity][48] decoded mixtures (guide::kMixFloats per row)
	float*          train_feat = nullptr; // [batch][8]: features 0-6, |cos| / pdf
	float4*         train_dirw = nullptr; // [batch]: direction, weight
	uint32_t        train_cap = 0;        // 0: no training samples recorded
	uint32_t        mark = 0;             // 1: guided vertices await their training sample at the next vertex
	uint32_t        open = 0;             // 1: open training records collect this iteration's emission
	uint32_t        keep = 0;             // 1: open records stay open into the next iteration
	uint32_t        nee_credit = 0;       // 1: this iteration's NEE records credit training samples
	float           alpha = 0.0f;         // 0: guiding off
	float           lo[3] = {0, 0, 0};    // scene bound, for the position features
	float           rcp[3] = {1, 1, 1};
};

// A multi-scene render (RenderScene::render_batch) keeps each path's scene in the top bits of its
// meta word; a single-scene render leaves them 0.
constexpr uint32_t kMetaSceneShift = 16u;
constexpr uint32_t kMaxBatchScenes = 1u << 16;
constexpr uint32_t kMetaBounceMask = 0xFFu;
constexpr uint32_t kMetaPrevNee = 1u << 8;      // the previous vertex used NEE (MIS applies)
constexpr uint32_t kMetaStopAfter = 1u << 9;    // Russian roulette ended the path after this hit
constexpr uint32_t kMetaGuideRec = 1u << 10;    // gf0/gf1 hold a guided vertex awaiting its training sample
constexpr uint32_t kMetaGuideOpen = 1u << 11;   // gf0 holds an open training record (row, weight scale)
constexpr uint32_t kTargetFinal = 0x80000000u;

// Launcher implemented in pg_trace.cu (FMA-enabled traversal kernels); min_idle is the
// traversal's refill threshold (LaunchConfig::refill). Closest hits of this iteration's queue and visibility of the previous iteration's shadow
// queue `prev` in one persistent launch; unoccluded contributions go to rad_cur / the film.
// With a batch (multi-scene render), `meta` is the current path buffer's meta words and prev.sid
// the records' scenes. With train_dirw (guided training renders), an unoccluded record whose
// prev.t names a training sample adds its weight to that sample.
void launch_trace(const DeviceScene& s, RenderCounters* counters, const float4* ray_o, const float4* ray_d,
                  uint2* hits, const ShadowQueue& prev, float4* rad_cur, const FilmView& film, int min_idle,
                  cudaStream_t st, bool count, const uint32_t* meta = nullptr, const BatchView* batch = nullptr,
                  float4* train_dirw = nullptr);

// A scene resident on the GPU together with its render buffers.
class RenderScene
{
public:
	explicit RenderScene(const SceneDesc& desc, float max_origin_abs);
	~RenderScene();

	// Renders `params` and accumulates into the FP64 film (R, G, B, W sums per pixel, film.cuh).
	// Returns the device time of the render in milliseconds (CUDA events on the library stream).
	float render(const RenderParams& params, double* film_device);

	const DeviceScene& device() const { return m_dev; }
	const Geometry& geometry() const { return *m_geometry; }
	unsigned long long last_rays() const { return m_last_rays; }
	unsigned long long last_shadow_rays() const { return m_last_shadow; }
	unsigned long long last_iterations() const { return m_last_iterations; }
	// Kernels launched by the last render (every iteration's launches, empty trailing iterations
	// of the last graph batch included, and the per-render film launch).
	unsigned long long last_launches() const { return m_last_launches; }
	// Per-kernel device milliseconds of the last timing-mode render: prepare, regen, extend,
	// shade, shadow, guiding inference (query + network), guiding training.
	const double* last_kernel_ms() const { return m_kernel_ms; }
	// Nodes / triangles visited by closest-hit and any-hit queries in the last counting render.
	const unsigned long long* last_counts() const { return m_last_counts; }

	// Launch shapes of subsequent renders (leaf_tris differing from the tree's rebuilds it).
	void set_launch(const LaunchConfig& c);
	const LaunchConfig& launch() const { return m_launch; }
	// Picks the launch shapes by coordinate descent over calibration renders of `base` (a few
	// million paths at its estimator and bounce cap, into a scratch film): path-pool depth,
	// traversal refill threshold, grid of the grid-stride kernels and, with rebuild, the BVH leaf
	// size. A candidate replaces the current choice only when it is more than 1 % faster. With a
	// cache file, a scene of the same fingerprint takes the stored choice without calibrating,
	// and a new choice is appended to it.
	AutotuneResult autotune(const RenderParams& base, bool rebuild, const char* cache_path, bool ignore_cache);
	// The launch shapes of render_batch on this scene's pool for the given batch (calibrated at a
	// sixteenth of its samples; leaf sizes stay as they are).
	AutotuneResult autotune_batch(const std::vector<const RenderScene*>& scenes, const std::vector<uint32_t>& spp,
	                              const RenderParams& params);
	// Identifies scenes that tune alike: triangles, resolution, emitters, material kinds.
	std::string fingerprint(const RenderParams& base) const;

	// Learned guiding for subsequent renders; the network is created (He-initialised, fixed seed)
	// on first use and keeps its training state until reset_guiding().
	void set_guiding(const GuideParams& g) { m_guide_params = g; }
	// Dome densities: false (default) the reference's finite-dome densities, true exact ones (env.cuh).
	void set_dome_exact(bool exact) { m_dev.env_map.exact = exact ? 1u : 0u; }
	const GuideParams& guiding() const { return m_guide_params; }
	void reset_guiding();
	// Mean training loss over the training steps of the last guided render, and its number of
	// guided vertices.
	float last_guide_loss() const { return m_last_guide_loss; }
	unsigned long long last_guided_vertices() const { return m_last_guided; }
	// The FP32 network parameters (kNumParams) to the host.
	void guide_params(float* out) const;

	// Light selection as the kernels see it: each emitter's pick probability (EmitterRec::pmf,
	// which the NEE and MIS weights use) and the probability the device alias table realises.
	void light_pmf(float* out_pmf, double* out_alias_pmf, uint32_t* out_count) const;
	// Direct-light densities of the shading kernel's NEE code: queries [n][6] = receiving point,
	// point on the light triangle; prims [n] = that triangle's input index.
	void light_pdf(const float* queries, const uint32_t* prims, uint64_t n, float* out_pdf_w) const;

	// Renders several scenes in one wavefront: one path pool, one launch of every kernel per
	// iteration for all of them, the iterations captured as graphs. This scene's pool, stream and
	// graphs run it; every scene listed (this one included or not) must live on this device and
	// outlive the call. Scene k renders spp[k] more samples into films[k] (box filter, FP64 sums
	// [h][w][4]) starting at sample first_sample[k]; `params` gives the estimator, bounce cap,
	// seed and refine settings. The scenes are split into renders of at most 2^31 paths each.
	// Returns the device milliseconds of all of them.
	float render_batch(const std::vector<const RenderScene*>& scenes, const std::vector<double*>& films,
	                   const std::vector<uint32_t>& spp, const std::vector<uint64_t>& first_sample,
	                   const RenderParams& params);
	uint32_t width() const { return m_dev.cam.width; }
	uint32_t height() const { return m_dev.cam.height; }

private:
	float render_pass(const RenderParams& params, double* film_device, const std::vector<BatchScene>* batch = nullptr);
	void ensure_capacity(uint32_t capacity, uint32_t grid);
	// Coordinate descent over the launch shapes (pool depth, refill threshold, blocks per SM, and
	// optionally leaf size), `measure` giving a candidate's calibration milliseconds; the winner is
	// set on this scene.
	void descend(AutotuneResult& result, const std::function<float(const LaunchConfig&)>& measure, bool leaf_size);
	// Rebuilds the BVH from the resident triangles with at most max_leaf_tris per leaf.
	void rebuild_bvh(uint32_t max_leaf_tris);
	void ensure_guiding(uint32_t capacity);

	std::unique_ptr<Geometry> m_geometry;
	DeviceBuffer<Material>    m_materials;
	DeviceBuffer<EmitterRec>  m_emitters;
	DeviceBuffer<uint32_t>    m_emitter_tris;
	DeviceBuffer<float2>      m_alias;
	DeviceBuffer<float4>      m_env_texels;
	DeviceBuffer<float2>      m_env_alias;
	DeviceScene               m_dev{};

	uint32_t m_capacity = 0;
	uint32_t m_order_grid = 0;
	LaunchConfig m_launch;
	float m_max_origin_abs = 0.0f;
	uint32_t m_bvh_builder = 0;
	std::vector<uint32_t> m_material_types;   // per material (fingerprint)
	DeviceBuffer<uint32_t> m_path[2], m_meta[2];
	DeviceBuffer<float4>   m_thr[2], m_rad[2], m_prev[2], m_ro[2], m_rd[2];
	DeviceBuffer<uint2>    m_hits;
	DeviceBuffer<float4>   m_so[2], m_sd[2], m_sc[2];   // shadow queues, one per iteration parity
	DeviceBuffer<float2>   m_sr[2];
	DeviceBuffer<uint32_t> m_req_single, m_req_mutual;
	DeviceBuffer<uint32_t> m_order;   // shading order: kOrderLists lists of m_order_list slots
	DeviceBuffer<float4>   m_samples; // 4 x 4 filters: radiance of every path of a pass
	DeviceBuffer<uint32_t> m_inflight;   // previews: paths in flight per pixel
	DeviceBuffer<uint32_t> m_ssid[2];    // multi-scene renders: scene of each NEE record
	DeviceBuffer<BatchScene> m_batch_table;
	uint32_t m_order_list = 0;
	DeviceBuffer<RenderCounters> m_counters;

	// learned guiding
	GuideParams m_guide_params;
	uint32_t m_guide_capacity = 0;
	bool m_guide_ready = false;
	float m_bound_lo[3] = {0, 0, 0}, m_bound_rcp[3] = {1, 1, 1};
	DeviceBuffer<float4>   m_gf0[2], m_gf1[2];
	DeviceBuffer<float4>   m_st[2];
	DeviceBuffer<uint32_t> m_gmap;
	DeviceBuffer<float>    m_gfeat, m_graw;
	DeviceBuffer<float>    m_tfeat, m_traw;
	DeviceBuffer<float4>   m_tdirw;
	DeviceBuffer<uint16_t> m_tacts;
	DeviceBuffer<float>    m_gparams, m_gm, m_gv, m_ggrads, m_gscalars;
	DeviceBuffer<unsigned char> m_gimage;
	DeviceBuffer<uint32_t> m_gstep, m_gerr;
	float m_last_guide_loss = 0.0f;
	unsigned long long m_last_guided = 0;

	// the scene's own stream: renders of different scenes, from different host threads, overlap
	cudaStream_t m_stream = nullptr;
	// pinned readback of the counters, and the instantiated two-iteration graph of the last
	// render (kept across renders and updated in place when only kernel arguments change)
	RenderCounters* m_host_counters = nullptr;
	cudaGraphExec_t m_exec = nullptr;
	int m_exec_key = -1;

	unsigned long long m_last_rays = 0, m_last_shadow = 0, m_last_iterations = 0, m_last_launches = 0;
	unsigned long long m_last_counts[4] = {0, 0, 0, 0};
	double m_kernel_ms[7] = {0, 0, 0, 0, 0, 0, 0};
};

}// end namespace pg
