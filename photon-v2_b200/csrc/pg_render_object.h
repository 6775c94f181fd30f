// A render scene plus its FP64 film, shared by the flat C ABI and the Photon C API engine.
#pragma once

#include "pg_render.h"

#include <mutex>

namespace pg
{

struct RenderObject
{
	std::unique_ptr<RenderScene> scene;
	DeviceBuffer<double> film;      // [h][w][4] sums of filter-weighted radiance and weight (film.cuh)
	uint32_t filter = PG_FILTER_BOX;
	mutable DeviceBuffer<float> frame;   // [h][w][3] developed frame (develop_frame)
	mutable std::mutex frame_mutex;      // one develop at a time: a peek from a polling thread may
	                                     // overlap a frame readback of the rendering thread; also
	                                     // guards the preview below
	// While a render runs: the film's estimate over the samples finished so far ([h][w][3]),
	// refreshed at the render's progress points; frames are read from it while preview_valid.
	DeviceBuffer<float> preview;
	bool preview_valid = false;
	uint32_t width = 0, height = 0;
	uint64_t samples = 0;           // samples per pixel accumulated in the film
	float last_ms = 0.0f;
};

// Builds the BVH, uploads the scene and allocates a cleared film.
std::unique_ptr<RenderObject> make_render_object(SceneDesc&& desc);

// Copies the film sums to the host (double [h][w][4]).
void download_film(const RenderObject& r, double* out_sum);

// Develops the film on the GPU and copies the rectangle [x, x + w) x [y, y + h) of the developed
// frame into `out_rgb`, a host frame of the film's full size (float [height][width][3]); pixels
// outside the rectangle are left untouched. While a render runs (the preview is valid) the
// rectangle comes from the preview instead. Safe to call from several threads at once (the
// shared developed-frame buffer is held under the object's frame_mutex).
void develop_frame(const RenderObject& r, float* out_rgb, uint32_t x, uint32_t y, uint32_t w, uint32_t h);

// Starts serving frames from the preview: develops the film as it stands (nothing of the coming
// render in it yet) into the preview and marks it valid. Call before a render starts.
void begin_preview(RenderObject& r);
// Back to developing the film itself (the render has finished).
void end_preview(RenderObject& r);


}// end namespace pg
