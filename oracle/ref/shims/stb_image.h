// Stand-in for the stb_image declarations that the reference's HDR image
// type (visualizer/raytracer/HdrImage.cpp) compiles against. Test
// infrastructure for the oracle build only: the oracle never reads image
// files, so every loader reports failure.
#pragma once

#include <cstdlib>
#include <cstring>

inline float* stbi_loadf(const char*, int*, int*, int*, int) { return nullptr; }
inline float* stbi_loadf_from_memory(const unsigned char*, int, int*, int*, int*, int) { return nullptr; }
