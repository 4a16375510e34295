// Drop-in test of the C++ adapter (fluidsolver_b200/host/CudaFluidSolvers.hpp):
// libFluid's own IISPHFluidSolver3D<CubicSplineKernel3D, HashedNeighborhoodSearch3D>
// and LibFluid::Cuda::IISPHFluidSolver3D<FS_SEARCH_HASHED_3D> are driven side by
// side the way Simulator::execute_simulation_step does (Simulator.cpp:7-57),
// on the same particle collection contents. With FP32 and the reference order
// the collections must stay bit-identical; the neighborhood interfaces must
// give the same sets. Then the default (compensated) mode runs the same scene
// within tolerance. Exit status 0 on success.
//
// Built by tests/cpp/Makefile against the reference's headers (the reference
// checkout) and oracle/_ref/libfsref_serial.so; run by tests/test_gpu_dropin.py.
#include "CudaFluidSolvers.hpp"
#include "fluidSolver/kernel/CubicSplineKernel3D.hpp"
#include "fluidSolver/neighborhoodSearch/HashedNeighborhoodSearch3D.hpp"
#include "fluidSolver/solver/IISPHFluidSolver3D.hpp"
#include "time/DynamicCflTimestepGenerator.hpp"
#include "entities/BoundaryPreprocessor.hpp"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <set>

using namespace LibFluid;

static std::shared_ptr<ParticleCollection> make_scene(uint32_t seed) {
    auto c = std::make_shared<ParticleCollection>();
    c->add_type<MovementData3D>();
    c->add_type<ParticleData>();
    c->add_type<ParticleInfo>();
    c->add_type<ExternalForces3D>();
    uint32_t s = seed;
    auto rnd = [&]() {  // xorshift32 in [-1, 1)
        s ^= s << 13;
        s ^= s >> 17;
        s ^= s << 5;
        return (float)((double)s / 4294967296.0 * 2.0 - 1.0);
    };
    auto add = [&](float x, float y, float z, uint8_t type) {
        size_t i = c->add();
        auto& m = c->get<MovementData3D>(i);
        m.position = glm::vec3(x, y, z);
        m.velocity = glm::vec3(0.0f);
        m.acceleration = glm::vec3(0.0f);
        c->get<ExternalForces3D>(i).non_pressure_acceleration = glm::vec3(0.0f);
        auto& pd = c->get<ParticleData>(i);
        pd.mass = 1.0f;
        pd.density = 1.0f;
        pd.pressure = 0.0f;
        c->get<ParticleInfo>(i).type = type;
        c->get<ParticleInfo>(i).tag = (uint32_t)i;
    };
    for (int i = 0; i < 8; i++)
        for (int j = 0; j < 10; j++)
            for (int k = 0; k < 7; k++) add(i + 0.01f * rnd(), j + 0.01f * rnd(), k + 0.01f * rnd(), ParticleTypeNormal);
    const int nx = 16, ny = 14, nz = 12;
    for (int i = -1; i <= nx; i++)
        for (int k = -1; k <= nz; k++) add((float)i, -1.0f, (float)k, ParticleTypeBoundary);
    for (int j = 0; j < ny; j++) {
        for (int k = 0; k < nz; k++) {
            add(-1.0f, (float)j, (float)k, ParticleTypeBoundary);
            add((float)nx, (float)j, (float)k, ParticleTypeBoundary);
        }
        for (int i = -1; i <= nx; i++) {
            add((float)i, (float)j, -1.0f, ParticleTypeBoundary);
            add((float)i, (float)j, (float)nz, ParticleTypeBoundary);
        }
    }
    return c;
}

template <typename S>
static void setup(S& solver, std::shared_ptr<ParticleCollection> c, std::shared_ptr<TimestepGenerator> g) {
    solver.parameters.rest_density = 1.0f;
    solver.parameters.gravity = 9.81f;
    solver.parameters.particle_size = 1.0f;
    solver.parameters.notify_that_data_changed();
    solver.settings.viscosity = 0.01f;
    solver.settings.single_layer_boundary = true;
    solver.data.collection = c;
    solver.data.timestep_generator = g;
    solver.data.notify_that_data_changed();
}

static bool same_bits(float a, float b) { return std::memcmp(&a, &b, sizeof(float)) == 0; }

static int compare(ParticleCollection& a, ParticleCollection& b, bool exact, int step) {
    int bad = 0;
    for (size_t i = 0; i < a.size(); i++) {
        auto& ma = a.get<MovementData3D>(i);
        auto& mb = b.get<MovementData3D>(i);
        for (int k = 0; k < 3; k++) {
            float pa = ma.position[k], pb = mb.position[k], va = ma.velocity[k], vb = mb.velocity[k];
            if (exact ? (!same_bits(pa, pb) || !same_bits(va, vb)) : (std::fabs(pa - pb) > 1e-4f * (1.0f + std::fabs(pb))))
                bad++;
        }
        float da = a.get<ParticleData>(i).density, db = b.get<ParticleData>(i).density;
        float qa = a.get<ParticleData>(i).pressure, qb = b.get<ParticleData>(i).pressure;
        if (exact ? (!same_bits(da, db) || !same_bits(qa, qb)) : (std::fabs(da - db) > 1e-5f * std::fabs(db))) bad++;
    }
    if (bad) std::printf("step %d: %d mismatching values (%s)\n", step, bad, exact ? "bit-exact" : "tolerance");
    return bad;
}

int main() {
    const int steps = 12;
    // ---- bit-exact: FP32 with the reference order ------------------------
    {
        auto gen = std::make_shared<ConstantTimestepGenerator>();
        gen->settings.timestep = 0.005f;
        gen->parameters.particle_size = 1.0f;
        auto c_ref = make_scene(7), c_gpu = make_scene(7);
        IISPHFluidSolver3D<CubicSplineKernel3D, HashedNeighborhoodSearch3D> ref;
        Cuda::IISPHFluidSolver3D<FS_SEARCH_HASHED_3D> gpu;
        gpu.precision = FS_PRECISION_FP32;
        gpu.flags = FS_FLAG_REFERENCE_ORDER;
        setup(ref, c_ref, gen);
        setup(gpu, c_gpu, gen);
        for (int st = 0; st < steps; st++) {
            Timepoint t1, t2;
            gen->generate_next_timestep();
            t1.desired_time_step = t1.actual_time_step = gen->get_generated_timestep();
            t2 = t1;
            ref.execute_neighborhood_search();
            gpu.execute_neighborhood_search();
            if (st == 0) {
                // neighborhood interfaces (entities and sensors use these)
                auto ir = ref.create_neighborhood_interface();
                auto ig = gpu.create_neighborhood_interface();
                for (size_t i = 0; i < c_ref->size(); i += 37) {
                    std::set<size_t> a, b;
                    for (size_t j : ir->get_neighbors(i)) a.insert(j);
                    for (size_t j : ig->get_neighbors(i)) b.insert(j);
                    if (a != b) {
                        std::printf("neighbor set of %zu differs\n", i);
                        return 1;
                    }
                }
                glm::vec3 q(3.3f, 2.2f, 1.1f);
                std::set<size_t> a, b;
                for (size_t j : ir->get_neighbors(q)) a.insert(j);
                for (size_t j : ig->get_neighbors(q)) b.insert(j);
                if (a != b) {
                    std::printf("position query differs\n");
                    return 1;
                }
            }
            ref.execute_simulation_step(t1);
            gpu.execute_simulation_step(t2);
            if (!same_bits(t1.actual_time_step, t2.actual_time_step) ||
                ref.stat_last_iteration_count != gpu.stat_last_iteration_count) {
                std::printf("step %d: dt %g vs %g, iterations %zu vs %zu\n", st, t1.actual_time_step,
                            t2.actual_time_step, ref.stat_last_iteration_count, gpu.stat_last_iteration_count);
                return 1;
            }
            if (compare(*c_ref, *c_gpu, true, st)) return 1;
        }
        std::printf("bit-exact: %d steps of %zu particles identical\n", steps, c_ref->size());
    }
    // ---- bit-exact with DynamicCflTimestepGenerator -------------------------
    // The reference's generator runs on the host over the reference's
    // collection (DynamicCflTimestepGenerator.cpp:45-59); the drop-in's device
    // chooses the time step inside its step and reports it in the timepoint.
    // Fluid particles start with velocities and accelerations, so that the
    // generator's CFL bounds, not its min/max clamp, decide the first steps.
    {
        auto make = [](std::shared_ptr<ParticleCollection> c) {
            auto g = std::make_shared<DynamicCflTimestepGenerator>();
            g->settings.max_timestep = 0.2f;
            g->settings.min_timestep = 0.0001f;
            g->parameters.particle_size = 1.0f;
            g->parameters.particle_collection = c;
            return g;
        };
        auto c_ref = make_scene(5), c_gpu = make_scene(5);
        for (auto c : {c_ref, c_gpu}) {
            uint32_t s = 99;
            auto rnd = [&]() {
                s ^= s << 13;
                s ^= s >> 17;
                s ^= s << 5;
                return (float)((double)s / 4294967296.0 * 2.0 - 1.0);
            };
            for (size_t i = 0; i < c->size(); i++) {
                if (c->get<ParticleInfo>(i).type != ParticleTypeNormal) continue;
                auto& m = c->get<MovementData3D>(i);
                m.velocity = glm::vec3(2.0f * rnd(), 2.0f * rnd(), 2.0f * rnd());
                m.acceleration = glm::vec3(0.5f * rnd(), -9.81f + 0.5f * rnd(), 0.5f * rnd());
            }
        }
        auto gen_ref = make(c_ref), gen_gpu = make(c_gpu);
        IISPHFluidSolver3D<CubicSplineKernel3D, HashedNeighborhoodSearch3D> ref;
        Cuda::IISPHFluidSolver3D<FS_SEARCH_HASHED_3D> gpu;
        gpu.precision = FS_PRECISION_FP32;
        gpu.flags = FS_FLAG_REFERENCE_ORDER;
        setup(ref, c_ref, gen_ref);
        setup(gpu, c_gpu, gen_gpu);
        float first = 0.0f;
        for (int st = 0; st < steps; st++) {
            Timepoint t1, t2;
            gen_ref->generate_next_timestep();
            t1.desired_time_step = t1.actual_time_step = gen_ref->get_generated_timestep();
            t2.desired_time_step = t2.actual_time_step = 1.0f;   // not used: the device generates it
            ref.execute_neighborhood_search();
            gpu.execute_neighborhood_search();
            ref.execute_simulation_step(t1);
            gpu.execute_simulation_step(t2);
            if (!same_bits(t1.desired_time_step, t2.desired_time_step) ||
                !same_bits(t1.actual_time_step, t2.actual_time_step) ||
                ref.stat_last_iteration_count != gpu.stat_last_iteration_count) {
                std::printf("dynamic step %d: desired %.9g vs %.9g, actual %.9g vs %.9g, iterations %zu vs %zu\n", st,
                            t1.desired_time_step, t2.desired_time_step, t1.actual_time_step, t2.actual_time_step,
                            ref.stat_last_iteration_count, gpu.stat_last_iteration_count);
                return 1;
            }
            if (st == 0) first = t1.desired_time_step;
            if (compare(*c_ref, *c_gpu, true, st)) return 1;
        }
        if (!(first > 0.0001f && first < 0.2f)) {
            std::printf("dynamic: first time step %g was clamped, the CFL bounds were not exercised\n", first);
            return 1;
        }
        std::printf("dynamic CFL generator: %d steps bit-exact (first dt %g)\n", steps, first);
    }
    // ---- bit-exact with the boundary preprocessor ----------------------------
    // libFluid's BoundaryPreprocessor on the host collection through the
    // reference solver's interface, and Cuda::BoundaryPreprocessor on the
    // device state, each run between the search and the step as the Simulator
    // does for entities executed before the solver (Simulator.cpp:28-36).
    {
        auto gen = std::make_shared<ConstantTimestepGenerator>();
        gen->settings.timestep = 0.005f;
        gen->parameters.particle_size = 1.0f;
        auto c_ref = make_scene(11), c_gpu = make_scene(11);
        IISPHFluidSolver3D<CubicSplineKernel3D, HashedNeighborhoodSearch3D> ref;
        Cuda::IISPHFluidSolver3D<FS_SEARCH_HASHED_3D> gpu;
        gpu.precision = FS_PRECISION_FP32;
        gpu.flags = FS_FLAG_REFERENCE_ORDER;
        setup(ref, c_ref, gen);
        setup(gpu, c_gpu, gen);
        BoundaryPreprocessor bp_ref;
        bp_ref.simulation_data.collection = c_ref;
        bp_ref.simulation_data.particle_size = 1.0f;
        bp_ref.simulation_data.rest_density = 1.0f;
        Cuda::BoundaryPreprocessor<Cuda::IISPHFluidSolver3D<FS_SEARCH_HASHED_3D>> bp_gpu(gpu);
        for (int st = 0; st < 6; st++) {
            Timepoint t1, t2;
            gen->generate_next_timestep();
            t1.desired_time_step = t1.actual_time_step = gen->get_generated_timestep();
            t2 = t1;
            ref.execute_neighborhood_search();
            gpu.execute_neighborhood_search();
            bp_ref.simulation_data.neighborhood_interface = ref.create_neighborhood_interface();
            bp_ref.simulation_data.notify_that_data_changed();
            bp_ref.execute_simulation_step(t1, true);
            bp_gpu.execute_simulation_step(t2, true);
            ref.execute_simulation_step(t1);
            gpu.execute_simulation_step(t2);
            int bad = 0;
            for (size_t i = 0; i < c_ref->size(); i++)
                if (!same_bits(c_ref->get<ParticleData>(i).mass, c_gpu->get<ParticleData>(i).mass)) bad++;
            if (bad) {
                std::printf("boundary preprocessor step %d: %d masses differ\n", st, bad);
                return 1;
            }
            if (compare(*c_ref, *c_gpu, true, st)) return 1;
        }
        std::printf("boundary preprocessor: 6 steps bit-exact\n");
    }
    // ---- default mode within tolerance -------------------------------------
    {
        auto gen = std::make_shared<ConstantTimestepGenerator>();
        gen->settings.timestep = 0.005f;
        gen->parameters.particle_size = 1.0f;
        auto c_ref = make_scene(9), c_gpu = make_scene(9);
        IISPHFluidSolver3D<CubicSplineKernel3D, HashedNeighborhoodSearch3D> ref;
        Cuda::IISPHFluidSolver3D<FS_SEARCH_HASHED_3D> gpu;
        setup(ref, c_ref, gen);
        setup(gpu, c_gpu, gen);
        for (int st = 0; st < 3; st++) {
            Timepoint t1, t2;
            gen->generate_next_timestep();
            t1.desired_time_step = t1.actual_time_step = gen->get_generated_timestep();
            t2 = t1;
            ref.execute_neighborhood_search();
            ref.execute_simulation_step(t1);
            gpu.execute_neighborhood_search();
            gpu.execute_simulation_step(t2);
            if (compare(*c_ref, *c_gpu, false, st)) return 1;
        }
        std::printf("compensated mode: within tolerance\n");
    }
    CompatibilityReport report;
    Cuda::IISPHFluidSolver3D<FS_SEARCH_HASHED_3D> probe;
    probe.create_compatibility_report(report);
    if (!report.has_issues()) std::printf("compatibility report: collection null reported? no\n");
    std::printf("PASS\n");
    return 0;
}
