// A render scene plus its FP64 film, shared by the flat C ABI and the Photon C API engine.
#pragma once

#include "pg_render.h"

namespace pg
{

struct RenderObject
{
	std::unique_ptr<RenderScene> scene;
	DeviceBuffer<double> film;      // [h][w][3] sums of sample radiance
	uint32_t width = 0, height = 0;
	uint64_t samples = 0;           // samples per pixel accumulated in the film
	float last_ms = 0.0f;
};

// Builds the BVH, uploads the scene and allocates a cleared film.
std::unique_ptr<RenderObject> make_render_object(SceneDesc&& desc);

// Copies the film sums to the host (double [h][w][3]).
void download_film(const RenderObject& r, double* out_sum);

}// end namespace pg
