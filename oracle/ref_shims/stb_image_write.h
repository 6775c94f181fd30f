// Oracle build shim (test infrastructure only, never linked into the product).
//
// LDR/HDR writers used by Engine/Source/DataIO/io_utils.cpp:580-690. The oracle writes PFM only
// (the engine's own writer), so every stb writer here reports failure.
#pragma once

inline void stbi_flip_vertically_on_write(int) {}
inline int stbi_write_png(const char*, int, int, int, const void*, int) { return 0; }
inline int stbi_write_jpg(const char*, int, int, int, const void*, int) { return 0; }
inline int stbi_write_bmp(const char*, int, int, int, const void*) { return 0; }
inline int stbi_write_tga(const char*, int, int, int, const void*) { return 0; }
inline int stbi_write_hdr(const char*, int, int, int, const float*) { return 0; }
