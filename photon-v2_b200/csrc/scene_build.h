// Host helpers that turn reference-level scene parameters into the renderer's records.
#pragma once

#include "pg_render.h"

namespace pg
{

// Pinhole camera of a single-lens observer given position, viewing direction, up axis and the
// horizontal field of view (OrientedRasterObserver::makeRotFromVectors,
// Engine/Source/EngineEnv/Observer/OrientedRasterObserver.cpp:48-100; SingleLensObserver::
// makeRasterToSensor / getSensorSize / getSensorOffset, SingleLensObserver.cpp:30-80, with the
// default 36 mm sensor width).
Camera make_camera(const float pos[3], const float dir[3], const float up[3], float fov_degrees,
                   uint32_t width, uint32_t height, float sensor_width_mm = 36.0f);

// Material record from the SDL-level parameters. Roughness maps to alpha = roughness^2
// (RoughnessToAlphaMapping::Squared, the MicrosurfaceInfo default) with the floor of
// IsoTrowbridgeReitzConstant (alpha >= 0.001).
Material make_matte(float r, float g, float b);
Material make_conductor(float roughness, float f0r, float f0g, float f0b);
Material make_dielectric(float roughness, float ior_outer, float ior_inner);

// Surface area of the dome sphere around the scene (ADome::cook, Engine/Source/Actor/ADome.cpp:
// 45-60: radius = 1.01 x the farthest bound corner from the dome centre, at least 1).
double dome_area(const std::vector<float>& tris, const float center[3]);

}// end namespace pg
