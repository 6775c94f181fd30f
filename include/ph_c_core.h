/* Photon C API, implemented by libphoton_gpu.so on the B200 path-tracing core.
 *
 * Every function keeps the signature, argument meaning and error behaviour of the reference
 * header Engine/CEngine/Include/ph_c_core.h:97-244 (implementation Engine/CEngine/Source/Api/
 * ph_c_core.cpp): resources are 64-bit ids, an unknown id is a silent no-op, parse and cook
 * errors are logged rather than returned. phRender renders the path-tracing visualizer's BNEEPT or
 * BVPT estimator on the GPU instead of the CPU EqualSamplingRenderer. The GPU build adds the
 * functions at the end of this file (error query, bounce cap, seed, sample offset, render
 * statistics); they have no counterpart in the reference.
 *
 * Threading: as in the reference, phInit/phExit on one thread; phAsync* may be called from
 * another thread while phRender runs.
 */
#ifndef PH_C_CORE_H
#define PH_C_CORE_H

#include "ph_c_core_types.h"

#if defined(__GNUC__)
#define PH_API __attribute__((visibility("default")))
#else
#define PH_API
#endif

enum PH_EATTRIBUTE { LIGHT_ENERGY, NORMAL, DEPTH };

#define PH_NUM_RENDER_LAYERS         4
#define PH_NUM_RENDER_STATE_INTEGERS 4
#define PH_NUM_RENDER_STATE_REALS    4
#define PH_MAX_NAME_LENGTH           128

struct PHRenderState
{
	PhInt64   integers[PH_NUM_RENDER_STATE_INTEGERS];
	PhFloat32 reals[PH_NUM_RENDER_STATE_REALS];
};

struct PHObservableRenderData
{
	PhChar layers[PH_NUM_RENDER_LAYERS][PH_MAX_NAME_LENGTH + 1];
	PhChar integers[PH_NUM_RENDER_STATE_INTEGERS][PH_MAX_NAME_LENGTH + 1];
	PhChar reals[PH_NUM_RENDER_STATE_REALS][PH_MAX_NAME_LENGTH + 1];
};

enum PH_ERenderStateType { INTEGER, REAL };

#ifdef __cplusplus
extern "C" {
#endif

/* starting and exiting (ph_c_core.h:107-108) */
extern PH_API void phConfigRendererResourceDirectory(const PhChar* directory);
extern PH_API PhBool phInit(void);
extern PH_API PhBool phExit(void);

/* engines (ph_c_core.h:118-140) */
extern PH_API void phCreateEngine(PhUInt64* out_engineId, const PhUInt32 numRenderThreads);
extern PH_API void phSetNumRenderThreads(PhUInt64 engineId, const PhUInt32 numRenderThreads);
extern PH_API void phEnterCommand(PhUInt64 engineId, const PhChar* commandFragment);
extern PH_API PhBool phLoadCommands(PhUInt64 engineId, const PhChar* filePath);
extern PH_API void phRender(PhUInt64 engineId);
extern PH_API void phUpdate(PhUInt64 engineId);
extern PH_API void phGetRenderDimension(PhUInt64 engineId, PhUInt32* out_widthPx, PhUInt32* out_heightPx);
extern PH_API void phGetObservableRenderData(PhUInt64 engineId, struct PHObservableRenderData* out_data);
extern PH_API void phDeleteEngine(PhUInt64 engineId);
extern PH_API void phSetWorkingDirectory(PhUInt64 engineId, const PhChar* workingDirectory);
extern PH_API void phAquireFrame(PhUInt64 engineId, PhUInt64 channelIndex, PhUInt64 frameId);
extern PH_API void phAquireFrameRaw(PhUInt64 engineId, PhUInt64 channelIndex, PhUInt64 frameId);

/* frames (ph_c_core.h:146-171) */
extern PH_API void phCreateFrame(PhUInt64* out_frameId, PhUInt32 widthPx, PhUInt32 heightPx);
extern PH_API void phGetFrameDimension(PhUInt64 frameId, PhUInt32* out_widthPx, PhUInt32* out_heightPx);
extern PH_API void phGetFrameRgbData(PhUInt64 frameId, const PhFloat32** out_data);
extern PH_API void phDeleteFrame(PhUInt64 frameId);
extern PH_API PhBool phLoadFrame(PhUInt64 frameId, const PhChar* filePath);
extern PH_API PhBool phSaveFrame(PhUInt64 frameId, const PhChar* filePath, const PhFrameSaveInfo* saveInfo);
extern PH_API PhBool phSaveFrameToBuffer(PhUInt64 frameId, PhUInt64 bufferId, PhBufferFormat format,
                                         const PhFrameSaveInfo* saveInfo);
extern PH_API void phFrameOpAbsDifference(PhUInt64 frameAId, PhUInt64 frameBId, PhUInt64 resultFrameId);
extern PH_API PhFloat32 phFrameOpMSE(PhUInt64 expectedFrameId, PhUInt64 estimatedFramIde);

/* buffers (ph_c_core.h:177-179) */
extern PH_API void phCreateBuffer(PhUInt64* out_bufferId);
extern PH_API void phGetBufferBytes(PhUInt64 bufferId, const PhUChar** out_bytesPtr, PhSize* out_numBytes);
extern PH_API void phDeleteBuffer(PhUInt64 bufferId);

/* asynchronous queries (ph_c_core.h:185-244) */
extern PH_API void phAsyncGetRenderProgress(PhUInt64 engineId, PhRenderProgress* out_progress);
extern PH_API void phAsyncGetRenderStatistics(PhUInt64 engineId, PhFloat32* out_percentageProgress,
                                              PhFloat32* out_samplesPerSecond);
extern PH_API void phAsyncGetRenderState(PhUInt64 engineId, struct PHRenderState* out_state);
extern PH_API PhBool phAsyncPollUpdatedFrameRegion(PhUInt64 engineId, PhFrameRegionInfo* out_regionInfo);
extern PH_API PhSize phAsyncPollUpdatedFrameRegions(PhUInt64 engineId, PhUInt64 bufferId,
                                                    PhFrameRegionInfo* out_regionInfos, PhSize maxRegionInfos);
extern PH_API PhSize phAsyncPollMergedUpdatedFrameRegions(PhUInt64 engineId, PhUInt64 bufferId, PhSize mergeSize,
                                                          PhFrameRegionInfo* out_regionInfos, PhSize maxRegionInfos);
extern PH_API void phAsyncPeekFrame(PhUInt64 engineId, PhUInt64 layerIndex, PhUInt32 xPx, PhUInt32 yPx,
                                    PhUInt32 widthPx, PhUInt32 heightPx, PhUInt64 frameId);
extern PH_API void phAsyncPeekFrameRaw(PhUInt64 engineId, PhUInt64 layerIndex, PhUInt32 xPx, PhUInt32 yPx,
                                       PhUInt32 widthPx, PhUInt32 heightPx, PhUInt64 frameId);

/* ---- GPU build extensions (no counterpart in the reference) ---------------------------------- */

/* Errors recorded by the engine since the last clear (parse, cook and render failures), joined by
 * newlines; *out_message stays valid until the next call on this engine. Returns PH_TRUE if any. */
extern PH_API PhBool phGpuGetErrors(PhUInt64 engineId, const PhChar** out_message);
/* Bounce cap of the estimators (the reference's compile-time MAX_RAY_BOUNCES, default 10000). */
extern PH_API void phGpuSetMaxRayBounces(PhUInt64 engineId, PhUInt32 maxRayBounces);
/* Seed of the counter-based random numbers (default 42). */
extern PH_API void phGpuSetSeed(PhUInt64 engineId, PhUInt64 seed);
/* Learned path guiding for the BNEEPT estimator: a small MLP proposes incident directions at
 * Lambertian vertices (mixed with BSDF sampling by one-sample MIS, so results stay unbiased) and
 * is trained online on the render's own radiance samples. Off by default. */
extern PH_API void phGpuSetGuiding(PhUInt64 engineId, PhBool enabled);
/* BVH builder of the next phUpdate: 0 host binned SAH (default), 1 on the GPU from Morton-ordered
 * triangles (seconds faster on multi-million-triangle scenes, somewhat costlier to traverse). */
extern PH_API void phGpuSetBvhBuilder(PhUInt64 engineId, PhUInt32 builder);
/* Densities of dome (image-dome) light samples: 0 (the default) as the reference computes them on
 * its finite dome sphere (Core/Intersection/PLatLongEnvSphere.cpp:125-186, lta::pdfA_to_pdfW),
 * which matches its images but is biased away from the dome centre; 1 the exact density of the
 * sampled direction (unbiased). Invalid values are ignored. */
extern PH_API void phGpuSetDomePdf(PhUInt64 engineId, PhUInt32 mode);
/* Surface refinement of rays leaving surfaces, as the reference's EngineConfig.ini sets it
 * (RefineMode / SelfIntersectDelta / NumIterativeSurfaceRefinements, which phInit also reads from
 * ./Config/EngineConfig.ini when the file exists): mode 0 manual, 1 empirical, 2 iterative
 * (the default). Invalid values are ignored. */
extern PH_API void phGpuSetSurfaceRefine(PhUInt64 engineId, PhUInt32 mode, PhFloat32 selfIntersectDelta,
                                         PhUInt32 numIterations);
/* Clears the film; the next phRender starts a fresh image. */
extern PH_API void phGpuClearFilm(PhUInt64 engineId);
/* Device milliseconds, paths, closest-hit rays and shadow rays of the last phRender, and the
 * seconds of the last phUpdate (cooking, BVH build, upload). Any output may be NULL. */
extern PH_API void phGpuGetRenderInfo(PhUInt64 engineId, PhFloat64* out_deviceMs, PhUInt64* out_paths,
                                      PhUInt64* out_rays, PhUInt64* out_shadowRays, PhFloat64* out_updateSeconds);

/* Kernel launches of the last phRender (five per wavefront iteration). */
extern PH_API PhUInt64 phGpuGetLaunchCount(PhUInt64 engineId);
/* Profiling render of `samplesPerPixel` samples into a scratch film (the engine's own image is
 * untouched). mode 1: plain launches with CUDA events around every kernel; mode 2: traversal
 * kernels count visited BVH nodes and tested triangles. out_stats (PhFloat64 [14]):
 *   [0..4] device ms of prepare, regen, extend (closest hit), shade, shadow (any hit) -- mode 1
 *   [5] total device ms, [6] paths, [7] closest-hit rays, [8] shadow rays, [9] iterations,
 *   [10] nodes visited by closest-hit rays, [11] triangles tested by them,
 *   [12] nodes visited by shadow rays, [13] triangles tested by them -- mode 2 */
extern PH_API void phGpuProfileRender(PhUInt64 engineId, PhUInt32 mode, PhUInt32 samplesPerPixel,
                                      PhFloat64* out_stats);

/* Picks the launch shapes of the updated scene for the session's samples per pixel, estimator and
 * bounce cap (pgpu_scene_autotune in photon_gpu.h: path-pool depth, traversal refill threshold,
 * blocks per SM, and with flags bit 0 the BVH leaf size; bit 1 ignores the cache). cachePath (may
 * be NULL) keeps choices across sessions. outConfig [4] and outMs [4] as in pgpu_scene_autotune
 * (either may be NULL). PH_FALSE when no scene is updated or the calibration fails (the error
 * text goes to phGpuGetErrors). */
extern PH_API PhBool phGpuAutotune(PhUInt64 engineId, const PhChar* cachePath, PhUInt32 flags,
                                   PhUInt32* outConfig, PhFloat32* outMs);

#ifdef __cplusplus
}
#endif

#endif /* PH_C_CORE_H */
