// Particle files (fs_io.hpp): ParticleSerializer's version-1 layout in an LZ4 frame.
#include "fs_io.hpp"

#include <cstdio>
#include <cstring>
#include <memory>

#include "fs_lz4.hpp"

namespace fsio {

namespace {

struct Reader {
    const uint8_t* p;
    size_t left;
    bool ok = true;
    template <typename T> T get() {
        T v{};
        if (left < sizeof(T)) {
            ok = false;
            return v;
        }
        std::memcpy(&v, p, sizeof(T));   // little-endian host (x86-64 and aarch64 hosts of the B200)
        p += sizeof(T);
        left -= sizeof(T);
        return v;
    }
    void vec(float* dst, int dim) {
        for (int a = 0; a < dim; a++) dst[a] = get<float>();
    }
};

template <typename T> void put(std::vector<uint8_t>& out, T v) {
    const uint8_t* b = reinterpret_cast<const uint8_t*>(&v);
    out.insert(out.end(), b, b + sizeof(T));
}

}  // namespace

std::string parse_particles(const uint8_t* data, size_t len, ParticleFile& out) {
    Reader r{data, len};
    const uint32_t version = r.get<uint32_t>();
    if (!r.ok) return "truncated particle data";
    if (version != 1) return "Unsupported particle data format version";   // ParticleSerializer.cpp:96-98
    const uint32_t count = r.get<uint32_t>();
    out.components = 0;
    for (uint32_t i = 0; i < count && r.ok; i++) {
        const uint32_t id = r.get<uint32_t>();
        if (id < kMovement2D || id > kExternal3D) return "unknown particle component id " + std::to_string(id);
        out.components |= 1u << id;
    }
    out.n = r.get<uint64_t>();
    if (!r.ok) return "truncated particle data";
    if (out.has(kMovement2D) && out.has(kMovement3D)) return "both 2D and 3D movement data";
    out.dim = out.has(kMovement2D) || out.has(kExternal2D) ? 2 : 3;
    const int d = out.dim;
    // every record has a fixed size: check the payload before allocating
    const size_t rec = (out.has(kMovement2D) ? 24 : 0) + (out.has(kMovement3D) ? 36 : 0) + (out.has(kInfo) ? 5 : 0) +
                       (out.has(kData) ? 12 : 0) + (out.has(kExternal2D) ? 8 : 0) + (out.has(kExternal3D) ? 12 : 0);
    if (rec != 0 && out.n > r.left / rec) return "particle data shorter than its particle count";
    const size_t n = (size_t)out.n;
    const bool mv = out.has(kMovement2D) || out.has(kMovement3D), ex = out.has(kExternal2D) || out.has(kExternal3D);
    out.position.assign(mv ? n * d : 0, 0.f);
    out.velocity.assign(mv ? n * d : 0, 0.f);
    out.acceleration.assign(mv ? n * d : 0, 0.f);
    out.external.assign(ex ? n * d : 0, 0.f);
    out.type.assign(out.has(kInfo) ? n : 0, 0);
    out.tag.assign(out.has(kInfo) ? n : 0, 0);
    out.mass.assign(out.has(kData) ? n : 0, 0.f);
    out.density.assign(out.has(kData) ? n : 0, 0.f);
    out.pressure.assign(out.has(kData) ? n : 0, 0.f);
    for (size_t i = 0; i < n; i++) {   // the order of ParticleSerializer.cpp:112-140 (and :57-81)
        if (mv) {
            r.vec(&out.position[i * d], d);
            r.vec(&out.velocity[i * d], d);
            r.vec(&out.acceleration[i * d], d);
        }
        if (out.has(kInfo)) {
            out.type[i] = r.get<uint8_t>();
            out.tag[i] = r.get<uint32_t>();
        }
        if (out.has(kData)) {
            out.density[i] = r.get<float>();
            out.mass[i] = r.get<float>();
            out.pressure[i] = r.get<float>();
        }
        if (ex) r.vec(&out.external[i * d], d);
    }
    if (!r.ok) return "truncated particle data";
    if (r.left != 0) return "trailing bytes after the particle data";
    return std::string();
}

std::vector<uint8_t> serialize_particles(const ParticleFile& in) {
    std::vector<uint8_t> out;
    const int d = in.dim;
    const bool mv = !in.position.empty(), info = !in.type.empty() || !in.tag.empty();
    const bool data = !in.mass.empty() || !in.density.empty() || !in.pressure.empty(), ex = !in.external.empty();
    std::vector<uint32_t> ids;   // ParticleSerializer.cpp:165-184: ascending ids
    if (mv) ids.push_back(d == 2 ? kMovement2D : kMovement3D);
    if (info) ids.push_back(kInfo);
    if (data) ids.push_back(kData);
    if (ex) ids.push_back(d == 2 ? kExternal2D : kExternal3D);
    const size_t n = (size_t)in.n;
    out.reserve(16 + 4 * ids.size() + n * (9 * 4 + 5 + 12 + 12));
    put<uint32_t>(out, 1);
    put<uint32_t>(out, (uint32_t)ids.size());
    for (uint32_t id : ids) put<uint32_t>(out, id);
    put<uint64_t>(out, (uint64_t)n);
    auto at = [](const std::vector<float>& v, size_t i) { return v.empty() ? 0.0f : v[i]; };
    for (size_t i = 0; i < n; i++) {
        if (mv)
            for (const std::vector<float>* f : {&in.position, &in.velocity, &in.acceleration})
                for (int a = 0; a < d; a++) put<float>(out, at(*f, i * d + a));
        if (info) {
            put<uint8_t>(out, in.type.empty() ? (uint8_t)0 : in.type[i]);
            put<uint32_t>(out, in.tag.empty() ? (uint32_t)i : in.tag[i]);
        }
        if (data) {
            put<float>(out, at(in.density, i));
            put<float>(out, at(in.mass, i));
            put<float>(out, at(in.pressure, i));
        }
        if (ex)
            for (int a = 0; a < d; a++) put<float>(out, in.external[i * d + a]);
    }
    return out;
}

std::string read_particle_file(const std::string& path, ParticleFile& out) {
    std::unique_ptr<FILE, int (*)(FILE*)> f(std::fopen(path.c_str(), "rb"), &std::fclose);
    if (!f) return "cannot open " + path;
    std::vector<uint8_t> raw;
    uint8_t buf[1 << 16];
    size_t got;
    while ((got = std::fread(buf, 1, sizeof(buf), f.get())) > 0) raw.insert(raw.end(), buf, buf + got);
    std::vector<uint8_t> payload;
    std::string e = lz4_frame_decode(raw.data(), raw.size(), payload);
    if (!e.empty()) return path + ": " + e;
    e = parse_particles(payload.data(), payload.size(), out);
    return e.empty() ? e : path + ": " + e;
}

std::string write_particle_file(const std::string& path, const ParticleFile& in) {
    const std::vector<uint8_t> payload = serialize_particles(in);
    const std::vector<uint8_t> frame = lz4_frame_encode(payload.data(), payload.size());
    std::unique_ptr<FILE, int (*)(FILE*)> f(std::fopen(path.c_str(), "wb"), &std::fclose);
    if (!f) return "cannot create " + path;
    if (std::fwrite(frame.data(), 1, frame.size(), f.get()) != frame.size()) return "write failed: " + path;
    return std::string();
}

}  // namespace fsio
