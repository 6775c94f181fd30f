// A triangle scene resident on the GPU: compressed 8-wide BVH nodes and leaf-ordered triangles.
#pragma once

#include "bvh_build.h"
#include "pg_runtime.h"

namespace pg
{

struct Geometry
{
	DeviceBuffer<WideNode> nodes;
	DeviceBuffer<LeafTri>  tris;
	DeviceBuffer<uint32_t> error;     // device error flags (PG_DEV_ERR_*)
	DeviceBuffer<uint32_t> fetch;     // dynamic-fetch cursor of the trace kernels, zeroed per launch
	BvhBuildStats          stats;
	int                    device = -1;   // the device current at creation; it holds every buffer above
};

Registry<Geometry>& geometry_registry();

// Builds the BVH on the host (binned SAH) and uploads nodes and triangles on the library stream.
std::unique_ptr<Geometry> make_geometry(const BvhBuildInput& in);
// Builds the same wide BVH layout on the device from Morton-ordered triangles (bvh_gpu.cu).
std::unique_ptr<Geometry> make_geometry_gpu(const BvhBuildInput& in);

enum BvhBuilder : uint32_t
{
	PG_BVH_HOST_SAH = 0,
	PG_BVH_GPU_MORTON = 1,
};

// Launch helpers on a given stream (no synchronisation). d_rays: [n][8] float32;
// d_hits: [n] x (uint32 leaf triangle or 0xFFFFFFFF, float32 t).
void launch_trace_closest(const Geometry& g, const float* d_rays, uint64_t n, void* d_hits, cudaStream_t s);
void launch_trace_any(const Geometry& g, const float* d_rays, uint64_t n, int32_t* d_occluded, cudaStream_t s);

}// end namespace pg
