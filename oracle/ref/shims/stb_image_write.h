// Stand-in for the stb_image_write declarations that the reference's image
// types (visualizer/Image.cpp, raytracer/HdrImage.cpp) compile against. Test
// infrastructure for the oracle build only: the oracle never writes image
// files, so every writer reports failure.
#pragma once

#include <cstdlib>
#include <cstring>

typedef void stbi_write_func(void* context, void* data, int size);

inline int stbi_write_png(const char*, int, int, int, const void*, int) { return 0; }
inline int stbi_write_png_to_func(stbi_write_func*, void*, int, int, int, const void*, int) { return 0; }
inline int stbi_write_hdr(const char*, int, int, int, const float*) { return 0; }
inline int stbi_write_hdr_to_func(stbi_write_func*, void*, int, int, int, const float*) { return 0; }
