/* Low-level C ABI of the B200 path-tracing core (libphoton_gpu.so).
 *
 * Plain pointers and sizes only. Every function returns 0 on success or a nonzero status code
 * (see pg::Status in photon-v2_b200/csrc/pg_common.cuh); pgpu_last_error() returns the message of
 * the most recent failure on the calling thread. These entry points sit below the Photon C API
 * (ph_c_core.h, also exported by this library) and expose the hot-path stages one by one so that
 * each can be checked against the reference and measured on its own.
 *
 * Devices: an object (geometry, render scene) lives on the device that was current when it was
 * created, and every later call on it must be made with that device current; otherwise the call
 * fails with PG_ERR_INVALID_ARGUMENT before any work. Library work runs on one stream per device.
 * One process may drive several devices this way; the usual layout is one process per GPU.
 */
#ifndef PHOTON_GPU_H
#define PHOTON_GPU_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define PGPU_API __attribute__((visibility("default")))
#else
#define PGPU_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* Message of the last failed call on this thread ("" if none). */
PGPU_API const char* pgpu_last_error(void);

/* Number of CUDA devices visible (0 without a GPU). Never fails. */
PGPU_API int pgpu_device_count(void);

/* ---------------------------------------------------------------------------------------------
 * Geometry: a triangle soup with its compressed 8-wide BVH resident on the current device.
 *
 * Replaces the reference TLAS build over cooked PTriangles:
 *   TBinaryBvhIntersector<Index>::update/rebuildWithIntersectables
 *   (Engine/Source/Core/Intersection/BVH/TBinaryBvhIntersector.ipp:20-97), built by
 *   TBvhBuilder<2> (Engine/Source/Math/Algorithm/BVH/TBvhBuilder.ipp:36).
 * tris: float32 [num_tris][3][3] host array. max_origin_abs: largest |coordinate| of any ray
 * origin that will be traced (sizes the conservative box padding; 0 = scene bound only).
 */
PGPU_API int pgpu_geometry_create(const float* tris, uint64_t num_tris, float max_origin_abs, uint64_t* out_id);
/* As pgpu_geometry_create with a choice of builder: 0 = host binned SAH (the default above),
 * 1 = on the GPU from Morton-ordered triangles (a radix tree collapsed to the same 8-wide layout;
 * much faster to build on millions of triangles, somewhat costlier to traverse). Hits are the
 * same either way: they depend only on the triangles. */
PGPU_API int pgpu_geometry_create_ex(const float* tris, uint64_t num_tris, float max_origin_abs,
                       uint32_t bvh_builder, uint64_t* out_id);
/* Copies the built tree to the host: out_nodes [num_nodes] x 80-byte wide nodes, out_tris
 * [num_tris] x 48-byte leaf triangles (either may be NULL to query the counts only). */
PGPU_API int pgpu_geometry_export(uint64_t id, void* out_nodes, void* out_tris, uint64_t* out_num_nodes,
                       uint64_t* out_num_tris);
PGPU_API int pgpu_geometry_destroy(uint64_t id);
/* num_nodes, num_tris, wide-tree depth, host build seconds. Any output may be NULL. */
PGPU_API int pgpu_geometry_stats(uint64_t id, uint64_t* out_num_nodes, uint64_t* out_num_tris,
                        int32_t* out_max_depth, double* out_build_seconds);

/* Closest hit for host rays [n][8] = origin(3), minT, direction(3), maxT (two float4 per ray).
 * Replaces TBinaryBvhIntersector::isIntersecting (TBinaryBvhIntersector.ipp:27-50) and
 * TWatertightTriangle::isIntersecting (Engine/Source/Math/Geometry/TWatertightTriangle.ipp:16-149).
 * Outputs (host): prim index in input order or -1, hit t, barycentrics [n][3] (any may be NULL). */
PGPU_API int pgpu_trace_closest(uint64_t id, const float* rays, uint64_t n,
                       int32_t* out_prim, float* out_t, float* out_bary);

/* Occlusion for host rays [n][8]; out_occluded[i] = 1 if any triangle is hit in [minT, maxT].
 * Replaces Scene::isOccluding / Intersectable::isOccluding (Engine/Source/World/Scene.cpp:54-69,
 * Engine/Source/Core/Intersection/Intersectable.cpp:8). */
PGPU_API int pgpu_trace_any(uint64_t id, const float* rays, uint64_t n, int32_t* out_occluded);

/* Device-resident variants for throughput measurement: d_rays is a device pointer to [n][8]
 * float32, d_hits a device pointer to [n] x (uint32 leaf triangle or 0xFFFFFFFF, float32 t).
 * The launch runs on the library's stream; *out_ms (optional) receives the kernel time
 * measured with CUDA events on that stream. */
PGPU_API int pgpu_trace_closest_device(uint64_t id, const float* d_rays, uint64_t n, void* d_hits, float* out_ms);
PGPU_API int pgpu_trace_any_device(uint64_t id, const float* d_rays, uint64_t n, int32_t* d_occluded, float* out_ms);

/* Closest hit like pgpu_trace_closest (same kernels, same results), but the call allocates
 * nothing -- no device or host buffers -- for callers that cannot allocate at query time (a
 * device-memory budget already spent, or a thread that must not wait on cudaFree, which stalls
 * behind all work queued on the device). No counterpart in the reference: its CPU intersector
 * needs no staging memory.
 * Staging lives in one static device array per device, 3.75 MiB, holding at most 65536 rays per
 * call; larger n is rejected with PG_ERR_INVALID_ARGUMENT before any work. The array needs no
 * zero-initialisation (every slot a call reads is written earlier in that call).
 * Setup: the first call on a device (with that device current) looks up the array's device
 * address once; a call with n = 0 does only that. Like every call on a geometry, it must be made
 * with the geometry's device current (PG_ERR_INVALID_ARGUMENT otherwise), so that the array, the
 * stream and the geometry all belong to one device. Make that first call before beginning any
 * stream capture on the device.
 * Calls that overlap in time on the same device (several host threads) race on the one array:
 * the caller serialises them. */
PGPU_API int pgpu_trace_closest_noalloc(uint64_t id, const float* rays, uint64_t n,
                       int32_t* out_prim, float* out_t, float* out_bary);

/* Mean BVH nodes visited and triangles tested per ray over the given host rays (a counting
 * pass of the same traversal), for the algorithmic-bytes model of the roofline. */
PGPU_API int pgpu_trace_counts(uint64_t id, const float* rays, uint64_t n, int any_hit,
                      double* out_nodes_per_ray, double* out_tris_per_ray);

/* ---------------------------------------------------------------------------------------------
 * Learned path guiding (no reference counterpart: the reference has no guiding). The network maps
 * a surface query -- 7 scalars in [0, 1]: position (3), normal (2), outgoing direction (2) -- to
 * 40 raw outputs, 8 von Mises-Fisher lobes x (weight logit, mean xyz, log concentration).
 * params: the 29,480 FP32 parameters in the packed order W0[224][64], b0, W1[64][64], b1, W2, b2,
 * W3, b3, W4[64][40], b4 (W[in][out]). The forward pass runs on the tensor cores (tcgen05, BF16
 * operands, FP32 accumulation). features: host [n][7]; out_raw: host [n][40]. */
PGPU_API int pgpu_guide_forward(const float* params, const float* features, uint64_t n, float* out_raw);
/* The same forward pass, returning the decoded mixtures the renderer samples: host [n][48], per
 * lobe (weight, mean x, y, z, concentration kappa, weight x kappa / (2 pi (1 - exp(-2 kappa)))),
 * weights the softmax of the logits, means normalised, kappa = exp(raw) clamped to [1e-2, 5e3]. */
PGPU_API int pgpu_guide_mixture(const float* params, const float* features, uint64_t n, float* out_mix);

/* Training loss -sum_i w_i log q(d_i | x_i) / sum_i w_i of a batch (features [n][7], unit
 * directions [n][3], weights [n]) and its gradient with respect to all parameters
 * (out_grads[29480]). Forward and backward passes on the tensor cores (BF16 operands, FP32
 * accumulation; weight gradients accumulated in tensor memory). */
PGPU_API int pgpu_guide_gradients(const float* params, const float* features, const float* dirs,
                       const float* weights, uint64_t n, float* out_loss, float* out_grads);
/* As pgpu_guide_gradients; flags PG_GUIDE_BACKWARD_CUDA_CORES runs the backward pass in FP32 on
 * the CUDA cores instead (a cross-check of the tensor-core pass). */
#define PG_GUIDE_BACKWARD_CUDA_CORES 1u
PGPU_API int pgpu_guide_gradients_ex(const float* params, const float* features, const float* dirs,
                                     const float* weights, uint64_t n, uint32_t flags, float* out_loss,
                                     float* out_grads);

/* `steps` Adam steps (learning rate lr) over consecutive batches of `batch` samples of the data
 * set (cycled); params is updated in place, out_losses[steps] (optional) receives each step's loss. */
PGPU_API int pgpu_guide_train(float* params, const float* features, const float* dirs, const float* weights,
                       uint64_t n, uint32_t steps, uint32_t batch, float lr, float* out_losses);

/* ---------------------------------------------------------------------------------------------
 * BSDF kernels, evaluated one case per thread on the GPU with the same device functions the path
 * tracer uses. cases: float32 [n][19] (type, p0..p5, N(3), V(3), L(3), u(3)) with
 *   type 0 Lambertian (p0..p2 albedo)                   LambertianReflector.cpp:39-99
 *   type 1 GGX conductor (p0 roughness, p1..p3 F0)      OpaqueMicrofacet.cpp:59-155
 *   type 2 GGX dielectric (p0 roughness, p1 ior outer, p2 ior inner) TranslucentMicrofacet.cpp:62-364
 * and normals: float32 [n][6] = geometry normal, shading normal.
 * out: float32 [n][16] = eval_ok, bsdf(3), pdf_ok, pdfW, sample_ok, L(3),
 *      pdfAppliedBsdfCos(3), relativeIor, cos, 0. Strict sidedness, radiance transport. */
PGPU_API int pgpu_bsdf_eval(const float* cases, const float* normals, uint64_t n, float* out);

/* Film splat of given samples through the device filter and deposit functions the renderer uses,
 * for checking the film against the reference's HdrRgbFilm::addRgbSample
 * (Engine/Source/Core/Filmic/HdrRgbFilm.cpp:82-123) and its sample filters
 * (Engine/Source/Core/Filmic/SampleFilter.cpp:12-59). filter: 1 gaussian, 2 Mitchell-Netravali,
 * 3 Blackman-Harris (the 4 x 4 filters; the box filter's samples go to their own pixel without a
 * weight and are not splatted). samples: float32 [n][5] = raster x, raster y (pixel (i, j) covers
 * [i, i + 1) x [j, j + 1)), r, g, b; n at most 2^26. out_sums: float64 [height][width][4] =
 * filter-weighted R, G, B sums and the weight sum W of every pixel (developed value = RGB / W),
 * starting from zero. The film has 1 to 2^24 pixels. */
PGPU_API int pgpu_film_splat(uint32_t filter, uint32_t width, uint32_t height, const float* samples, uint64_t n,
                       double* out_sums);

/* ---------------------------------------------------------------------------------------------
 * Render scenes: the full BNEEPT / BVPT / BVPTDL estimators on the GPU.
 *
 * Replaces EqualSamplingRenderer::doRender (Engine/Source/Core/Renderer/Sampling/
 * EqualSamplingRenderer.cpp:119-203) driving BNEEPTEstimator::estimate
 * (Engine/Source/Core/Estimator/BNEEPTEstimator.cpp:38-262), BVPTEstimator::estimate
 * (Engine/Source/Core/Estimator/BVPTEstimator.cpp:25-160) or BVPTDLEstimator::estimate
 * (Engine/Source/Core/Estimator/BVPTDLEstimator.cpp:21-96) into an HdrRgbFilm (box filter unless
 * pgpu_scene_set_filter picks another).
 *
 * tris: float32 [n][3][3]; tri_material: uint32 [n]; tri_emitter: uint32 [n] = emitter index + 1
 *   (0 = not emissive; may be NULL).
 * materials: float32 [m][8] = type (0 matte, 1 GGX conductor, 2 GGX dielectric), c0, c1, c2,
 *   roughness, ior_outer, ior_inner, 0 -- c = albedo (matte) or F0 (conductor).
 * emitters: float32 [e][4] = radiance r, g, b, type (0 triangle group, 1 constant environment).
 * camera: float32 [12] = position(3), direction(3), up(3), horizontal fov (degrees), width, height;
 *   width and height whole numbers of at least 1, at most 2^31 pixels in all.
 * Every check (null arrays, index and type ranges, resolution) runs before any device work and
 * fails with PG_ERR_INVALID_ARGUMENT.
 */
PGPU_API int pgpu_scene_create(const float* tris, const uint32_t* tri_material, const uint32_t* tri_emitter,
                               uint64_t num_tris, const float* materials, uint32_t num_materials,
                               const float* emitters, uint32_t num_emitters, const float* camera,
                               uint64_t* out_id);
/* As pgpu_scene_create with a choice of BVH builder (see pgpu_geometry_create_ex). */
PGPU_API int pgpu_scene_create_ex(const float* tris, const uint32_t* tri_material, const uint32_t* tri_emitter,
                       uint64_t num_tris, const float* materials, uint32_t num_materials,
                       const float* emitters, uint32_t num_emitters, const float* camera,
                       uint32_t bvh_builder, uint64_t* out_id);
PGPU_API int pgpu_scene_destroy(uint64_t id);

/* Renders spp samples per pixel (estimator 0 = BNEEPT, 1 = BVPT, 2 = BVPTDL, which follows one
 * bounce whatever max_bounces says; max_bounces = the reference's MAX_RAY_BOUNCES) and adds them to the scene's FP64 film. Samples are numbered from first_sample
 * so that separate calls draw independent random numbers. Optional outputs: device time of the
 * render (CUDA events), closest-hit rays and shadow rays traced. */
PGPU_API int pgpu_scene_render(uint64_t id, uint32_t spp, uint32_t max_bounces, uint32_t estimator,
                               uint64_t seed, uint64_t first_sample, float* out_ms,
                               uint64_t* out_rays, uint64_t* out_shadow_rays);

/* Developed frame (host float32 [h][w][3], row 0 = bottom, the reference's frame layout: RGB / W
 * per pixel), the raw FP64 sums (host double [h][w][4] = filter-weighted R, G, B and the weight W,
 * the reference's RadianceSensor, Engine/Source/Core/Receiver/RadianceSensor.h:13-16) and the
 * samples per pixel accumulated; any may be NULL. */
PGPU_API int pgpu_scene_film(uint64_t id, float* out_rgb, double* out_sum, uint64_t* out_spp);
/* Sample filter of the scene's film (HdrRgbFilm::addRgbSample with SampleFilter::make*,
 * Engine/Source/Core/Filmic/HdrRgbFilm.cpp:82-123, SampleFilter.cpp:12-61): 0 box (the default
 * here), 1 gaussian, 2 mitchell-netravali, 3 blackman-harris. Clears the film. */
PGPU_API int pgpu_scene_set_filter(uint64_t id, uint32_t filter);
/* Densities of environment light samples: 0 the reference's (default), 1 exact; see
 * phGpuSetDomePdf in ph_c_core.h. */
PGPU_API int pgpu_scene_set_dome_pdf(uint64_t id, uint32_t mode);
/* A render into a scratch film with every kernel bracketed by CUDA events: per-kernel device
 * milliseconds (prepare, regen, extend, shade, shadow, guide inference, guide training). */
PGPU_API int pgpu_scene_profile(uint64_t id, uint32_t spp, uint32_t max_bounces, uint32_t estimator,
                       uint64_t seed, double* out_kernel_ms);
PGPU_API int pgpu_scene_clear(uint64_t id);
/* Renders several scenes as ONE wavefront: one pool of paths in flight, one launch of every kernel
 * per iteration for all the scenes (each queue entry carries its scene), the iterations captured
 * as CUDA graphs. Scene i renders spp[i] more samples into its film, exactly the paths its own
 * pgpu_scene_render with the same seed would trace. Replaces the reference's scene-by-scene
 * EqualSamplingRenderer::doRender (Engine/Source/Core/Renderer/Sampling/
 * EqualSamplingRenderer.cpp:119-203), one renderer per engine. Every film must use the box filter
 * and every scene live on the current device; guiding is not applied. The scenes are rendered in
 * renders of at most 2^31 paths each. *out_ms: device milliseconds of the whole batch. */
PGPU_API int pgpu_scenes_render_wavefront(const uint64_t* ids, uint32_t n, const uint32_t* spp, uint32_t max_bounces,
                                          uint32_t estimator, uint64_t seed, float* out_ms);
/* The launch shapes of pgpu_scenes_render_wavefront for these scenes: the autotuner's coordinate
 * descent (pool depth, refill threshold, blocks per SM) over calibration wavefronts of the batch at
 * a sixteenth of its samples, into scratch films. The choice is set on the first scene, whose pool
 * runs the wavefront. out_config [4] and out_ms [4] as in pgpu_scene_autotune. */
PGPU_API int pgpu_scenes_autotune_wavefront(const uint64_t* ids, uint32_t n, const uint32_t* spp, uint32_t max_bounces,
                                            uint32_t estimator, uint32_t* out_config, float* out_ms);
/* Renders several scenes at once: scene ids[i] gets spp[i] more samples (numbered after its
 * earlier ones) with the same bounce cap, estimator and seed. Up to `concurrency` host threads
 * render one scene each at a time on the scene's own stream, so small scenes fill the GPU
 * together. out_ms: time from the batch's start to its last scene's end (CUDA events on the
 * library stream around the whole batch). Each id may appear once. */
PGPU_API int pgpu_scenes_render(const uint64_t* ids, uint32_t n, const uint32_t* spp, uint32_t max_bounces,
                                uint32_t estimator, uint64_t seed, uint32_t concurrency, float* out_ms);
/* Light selection of a scene as its kernels use it. Replaces ESPowerFavoring::update / pickEmitter
 * (Engine/Source/Core/Emitter/Sampler/ESPowerFavoring.cpp:21-59): each emitter's pick
 * probability, proportional to its approximate flux -- colour energy x area x pi summed over its
 * triangles for an area light (DiffuseSurfaceEmitter.cpp:55-86, GroupedDiffuseSurfaceEmitter.cpp:
 * 110-120), luminance x sin(theta) x dome area for the environment. out_pmf [num_emitters] float:
 * the probability the NEE and MIS weights use; out_alias_pmf [num_emitters] double: the
 * probability the device alias table realises. Emitters are numbered as at pgpu_scene_create
 * (the environment last). Any output may be NULL. */
PGPU_API int pgpu_scene_light_pmf(uint64_t id, float* out_pmf, double* out_alias_pmf, uint32_t* out_num_emitters);
/* Solid-angle density of direct light samples, computed by the shading kernel's NEE code.
 * Replaces ESPowerFavoring::calcDirectPdf (ESPowerFavoring.cpp:82-97) over area emitters
 * (GroupedDiffuseSurfaceEmitter.cpp:80-84, SurfaceEmitter.cpp:37-61): pick probability x
 * 1 / (triangles of the emitter) x area density converted to solid angle; 0 where the light
 * triangle's front face does not face the receiving point or the triangle emits nothing.
 * queries [n][6] float = receiving point (3), point on the light triangle (3); prims [n] = the
 * light triangle's index in the scene's input order; out_pdf_w [n]. */
PGPU_API int pgpu_scene_light_pdf(uint64_t id, const float* queries, const uint32_t* prims, uint64_t n,
                                  float* out_pdf_w);
/* Launch-shape autotuner. No counterpart in the reference, whose EqualSamplingRenderer fixes its
 * scheduler and tile choice up front (Engine/Source/Core/Renderer/Sampling/
 * EqualSamplingRenderer.cpp:45-60,94-108); here the knobs are launch shapes. Picks, by coordinate
 * descent over calibration renders of the scene (spp samples at most, ~16M paths, into a scratch
 * film; estimator and bounce cap as given), the path-pool depth (queue depth), the traversal
 * refill threshold, the grid of the grid-stride kernels (blocks per SM) and, with
 * PG_AUTOTUNE_REBUILD, the BVH leaf size (the tree is rebuilt for each candidate). A candidate
 * wins only when more than 1 % faster. The choice stays with the scene for later renders.
 * cache_path (may be NULL): a text file of "fingerprint capacity refill blocks leaf" lines; a scene
 * whose fingerprint (triangles, resolution, emitters, material kinds, estimator, bounces, filter,
 * builder) is listed takes that line without calibrating (unless PG_AUTOTUNE_IGNORE_CACHE), and a
 * new choice is appended. out_config [4] (may be NULL): capacity, refill, blocks per SM, leaf
 * triangles. out_ms [4] (may be NULL): calibration device ms with the defaults, with the choice,
 * renders run, 1 if taken from the cache. */
#define PG_AUTOTUNE_REBUILD 1u
#define PG_AUTOTUNE_IGNORE_CACHE 2u
PGPU_API int pgpu_scene_autotune(uint64_t id, uint32_t spp, uint32_t max_bounces, uint32_t estimator, uint32_t flags,
                                 const char* cache_path, uint32_t* out_config, float* out_ms);
/* Sets / reads the launch shapes [4] = capacity (1024..2^24 path slots), refill (1..32 idle
 * lanes), blocks per SM (1..64), leaf triangles (1..3; a different value rebuilds the BVH). */
PGPU_API int pgpu_scene_set_launch(uint64_t id, const uint32_t* config);
PGPU_API int pgpu_scene_get_launch(uint64_t id, uint32_t* out_config);
/* Kernels the scene's last render launched (all iterations, including the empty ones that end the
 * last CUDA-graph batch). */
PGPU_API int pgpu_scene_launches(uint64_t id, uint64_t* out_launches);
/* A render into a scratch film whose traversal kernels count their work: out_counts uint64 [7] =
 * closest-hit rays, shadow rays, BVH nodes and triangles visited by closest-hit queries, the same
 * for shadow queries, render iterations. */
PGPU_API int pgpu_scene_count(uint64_t id, uint32_t spp, uint32_t max_bounces, uint32_t estimator,
                              uint64_t seed, uint64_t* out_counts);

/* Learned path guiding for the scene's subsequent BNEEPT renders (no reference counterpart). At
 * guided Lambertian vertices the next direction comes from the network's vMF mixture with
 * probability alpha, else from the BSDF, weighted by the one-sample MIS density, so renders stay
 * unbiased; NEE's MIS uses the same density. With train != 0 every period of four render
 * iterations records up to `batch` (vertex, direction, incident radiance) samples and takes one
 * Adam step (learning rate lr). The network persists across renders until pgpu_scene_guide_reset. */
PGPU_API int pgpu_scene_set_guiding(uint64_t id, int enabled, int train, float alpha, float lr, uint32_t batch);
/* Which vertices are guided: the first `depth` of every path (default 1, the surfaces the camera
 * sees; 0 = every vertex). Kept across pgpu_scene_set_guiding calls. */
PGPU_API int pgpu_scene_set_guiding_depth(uint64_t id, uint32_t depth);
PGPU_API int pgpu_scene_guide_reset(uint64_t id);
/* Last render's mean training loss, guided vertices, per-kernel milliseconds of a profiled render
 * (prepare, regen, extend, shade, shadow, guide inference, guide training; 7 doubles) and the FP32
 * network parameters (29,480 floats). Any output may be NULL. */
PGPU_API int pgpu_scene_guide_info(uint64_t id, float* out_loss, uint64_t* out_guided_vertices,
                        double* out_kernel_ms, float* out_params);

/* ---------------------------------------------------------------------------------------------
 * Scene cooking without a GPU: parses SDL text (the grammar of the reference's SdlCommandParser,
 * Engine/Source/SDL/SdlCommandParser.cpp:84-560) and cooks it the way phUpdate does (actors to
 * world-space triangles, materials, emitters, camera). Call once with NULL arrays to get the
 * counts, then again with arrays of those sizes. out_dims: uint32 [5] = width, height, spp,
 * estimator, sample filter (pgpu_scene_set_filter's numbering). out_emitters: float32 [e][4] = radiance rgb, type. out_camera: float32 [16] =
 * position, camera x/y/z axes, sensor width, height, offset (metres), dome area. */
PGPU_API int pgpu_sdl_cook(const char* sdl_text, const char* working_dir, uint64_t* out_num_tris,
                           uint32_t* out_num_materials, uint32_t* out_num_emitters, uint32_t* out_dims,
                           float* out_tris, uint32_t* out_tri_material, uint32_t* out_tri_emitter,
                           float* out_emitters, float* out_camera);

#ifdef __cplusplus
}
#endif

#endif /* PHOTON_GPU_H */
