// Oracle build shim (test infrastructure only, never linked into the product).
//
// The reference engine includes <stb_image.h> for LDR/HDR picture loading
// (Engine/Source/DataIO/io_utils.cpp:39-203). The third-party header is not vendored with the
// reference. The oracle renders only scenes whose images are PFM files, which the engine loads
// with its own reader (io_utils.cpp:370), so every stb entry point here reports failure.
#pragma once

#include <cstddef>

typedef unsigned char stbi_uc;

inline void stbi_set_flip_vertically_on_load(int) {}
inline const char* stbi_failure_reason() { return "stb_image is not available in the oracle build"; }
inline stbi_uc* stbi_load(const char*, int*, int*, int*, int) { return nullptr; }
inline float* stbi_loadf(const char*, int*, int*, int*, int) { return nullptr; }
inline int stbi_info(const char*, int*, int*, int*) { return 0; }
inline void stbi_image_free(void*) {}
