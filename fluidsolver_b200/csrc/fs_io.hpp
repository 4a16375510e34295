// Particle files: ParticleSerializer's version-1 layout (ParticleSerializer.cpp:41-141)
// inside an LZ4 frame (fs_lz4.hpp), little-endian throughout (EndianSafeBinaryStream.hpp:29-30):
//
//   u32 version = 1 | u32 component count | u32 component ids | u64 particle count
//   per particle, in this order, the components present:
//     1 MovementData      position, velocity, acceleration   (vec2 each)
//     2 MovementData3D    position, velocity, acceleration   (vec3 each)
//     3 ParticleInfo      type (u8), tag (u32)
//     4 ParticleData      density, mass, pressure             (f32 each)
//     5 ExternalForces    non_pressure_acceleration           (vec2)
//     6 ExternalForces3D  non_pressure_acceleration           (vec3)
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace fsio {

enum Component : uint32_t {
    kMovement2D = 1,
    kMovement3D = 2,
    kInfo = 3,
    kData = 4,
    kExternal2D = 5,
    kExternal3D = 6,
};

// a particle file's contents, structure of arrays (dim values per vector)
struct ParticleFile {
    int dim = 3;
    uint32_t components = 0;   // bit (1 << id) per component present
    uint64_t n = 0;
    std::vector<float> position, velocity, acceleration, external, mass, density, pressure;
    std::vector<uint8_t> type;
    std::vector<uint32_t> tag;
    bool has(uint32_t id) const { return (components >> id) & 1u; }
};

// Both return an empty string on success, else the reason.
std::string read_particle_file(const std::string& path, ParticleFile& out);
std::string write_particle_file(const std::string& path, const ParticleFile& in);

// the v1 payload without the LZ4 frame (the tests check both layers)
std::string parse_particles(const uint8_t* data, size_t len, ParticleFile& out);
std::vector<uint8_t> serialize_particles(const ParticleFile& in);

}  // namespace fsio
