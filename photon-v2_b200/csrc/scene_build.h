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

// Film resolution from caller-supplied numbers (the session's frame-size, a vector of two uint32,
// SingleFrameRenderSession.h:43): each a whole number of at least 1, and at most 2^31 pixels in
// all, so that every per-pixel kernel's 32-bit grid-stride index stays below 2^32. Throws Error
// (PG_ERR_INVALID_ARGUMENT) naming `who` otherwise.
void checked_resolution(double width, double height, const char* who, uint32_t* out_width, uint32_t* out_height);

// Material record from the SDL-level parameters. Roughness maps to alpha = roughness^2
// (RoughnessToAlphaMapping::Squared, the MicrosurfaceInfo default) with the floor of
// IsoTrowbridgeReitzConstant (alpha >= 0.001).
Material make_matte(float r, float g, float b);
Material make_conductor(float roughness, float f0r, float f0g, float f0b);
Material make_dielectric(float roughness, float ior_outer, float ior_inner);

// Energy of a linear-sRGB colour as the reference estimates it (estimate_color_energy,
// Engine/Source/Math/Color/color_spaces.ipp:744-764: Smits' RGB -> spectrum upsampling, then the
// sum of the spectral samples). Drives area-light radiance from watts and the power-proportional
// light pick.
double color_energy(double r, double g, double b);

// Relative luminance (CIE Y) of linear sRGB with the coefficients of the reference's colour
// transform (TSpectrumBase::relativeLuminance).
constexpr double kLumR = 0.212639004, kLumG = 0.715168655, kLumB = 0.0721923187;

// Surface area of the dome sphere around the scene (ADome::cook, Engine/Source/Actor/ADome.cpp:
// 45-60: radius = 1.01 x the farthest bound corner from the dome centre, at least 1).
double dome_area(const std::vector<float>& tris, const float center[3]);

}// end namespace pg
