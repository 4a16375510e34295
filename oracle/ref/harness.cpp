// Oracle harness around the reference's own hot-path sources (libFluid),
// compiled unmodified against the shims in oracle/ref/shims. TEST
// INFRASTRUCTURE ONLY: the parity tests, the golden-fixture generator and the
// CPU-baseline leg of bench.py load the resulting library to obtain the
// reference's results and timings; the product never links it.
//
// Everything is exposed as extern "C" over plain arrays in *tag space*: the
// i-th input particle gets ParticleInfo.tag = i, and every output is mapped
// back through the tag, because the reference searches permute the particle
// collection in place (CompressedNeighbors.cpp:192-201 every call,
// HashedNeighborhoodSearch3D.cpp:187-217 every 101st call).
//
// The driving sequence mirrors Simulator::execute_simulation_step
// (Simulator.cpp:7-57): generate_next_timestep -> desired/actual = generated ->
// execute_neighborhood_search -> execute_simulation_step(timepoint).

#include "fluidSolver/ParticleCollection.hpp"
#include "fluidSolver/kernel/CubicSplineKernel.hpp"
#include "fluidSolver/kernel/CubicSplineKernel3D.hpp"
#include "fluidSolver/neighborhoodSearch/CompressedNeighbors.hpp"
#include "fluidSolver/neighborhoodSearch/HashedNeighborhoodSearch.hpp"
#include "fluidSolver/neighborhoodSearch/HashedNeighborhoodSearch3D.hpp"
#include "fluidSolver/neighborhoodSearch/QuadraticNeighborhoodSearch3D.hpp"
#include "fluidSolver/neighborhoodSearch/QuadraticNeighborhoodSearchDynamicAllocated.hpp"
#include "fluidSolver/solver/IISPHFluidSolver.hpp"
#include "fluidSolver/solver/IISPHFluidSolver3D.hpp"
#include "fluidSolver/solver/SESPHFluidSolver.hpp"
#include "fluidSolver/solver/SESPHFluidSolver3D.hpp"
#include "time/ConstantTimestepGenerator.hpp"
#include "time/DynamicCflTimestepGenerator.hpp"
#include "entities/BoundaryPreprocessor.hpp"
#include "visualizer/raytracer/ParticleIntersectionAccelerator.hpp"
#include "visualizer/raytracer/ToneMapper.hpp"
#include "sensors/ParticleStatistics.hpp"

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <exception>
#include <memory>
#include <string>
#include <vector>

using namespace LibFluid;

namespace {
    std::string g_last_error;

    enum NsKind {
        NS_QUADRATIC_2D = 0,   // QuadraticNeighborhoodSearchDynamicAllocated
        NS_HASHED_2D = 1,      // HashedNeighborhoodSearch
        NS_QUADRATIC_3D = 2,   // QuadraticNeighborhoodSearch3D
        NS_HASHED_3D = 3,      // HashedNeighborhoodSearch3D
        NS_COMPRESSED_3D = 4,  // CompressedNeighborhoodSearch
    };

    enum SolverKind {
        SOLVER_SESPH_2D = 0,
        SOLVER_SESPH_3D = 1,
        SOLVER_IISPH_2D = 2,
        SOLVER_IISPH_3D = 3,
    };

    bool is_3d_ns(int kind) { return kind >= NS_QUADRATIC_3D; }

    // ------------------------------------------------------------------
    // neighborhood search wrapper
    // ------------------------------------------------------------------
    struct NsBase {
        std::shared_ptr<ParticleCollection> collection;
        int dim = 3;
        virtual ~NsBase() = default;
        virtual void find() = 0;
        // neighbors of the particle currently stored at collection index i
        virtual void neighbors_of(size_t i, std::vector<size_t>& out) = 0;
        virtual void neighbors_of_position(const float* p, std::vector<size_t>& out) = 0;
        virtual std::shared_ptr<NeighborhoodInterface> interface() = 0;
    };

    template <typename NS>
    struct NsImpl : NsBase {
        NS search;
        void find() override { search.find_neighbors(); }
        std::shared_ptr<NeighborhoodInterface> interface() override { return search.create_interface(); }
        void neighbors_of(size_t i, std::vector<size_t>& out) override {
            out.clear();
            auto nb = search.get_neighbors(i);
            for (auto it = nb.begin(); it != nb.end(); ++it)
                out.push_back(*it);
        }
        void neighbors_of_position(const float* p, std::vector<size_t>& out) override {
            out.clear();
            if constexpr (std::is_same_v<NS, HashedNeighborhoodSearch3D> || std::is_same_v<NS, CompressedNeighborhoodSearch> ||
                          std::is_same_v<NS, QuadraticNeighborhoodSearch3D>) {
                auto nb = search.get_neighbors(glm::vec3(p[0], p[1], p[2]));
                for (auto it = nb.begin(); it != nb.end(); ++it)
                    out.push_back(*it);
            } else {
                auto nb = search.get_neighbors(glm::vec2(p[0], p[1]));
                for (auto it = nb.begin(); it != nb.end(); ++it)
                    out.push_back(*it);
            }
        }
    };

    void fill_collection(ParticleCollection& c, int dim, int64_t n, const float* pos, const uint8_t* type) {
        if (dim == 2) {
            c.add_type<MovementData>();
            c.add_type<ExternalForces>();
        } else {
            c.add_type<MovementData3D>();
            c.add_type<ExternalForces3D>();
        }
        c.add_type<ParticleInfo>();
        c.add_type<ParticleData>();
        c.resize((size_t)n);
        for (int64_t i = 0; i < n; i++) {
            if (dim == 2) {
                auto& m = c.get<MovementData>(i);
                m.position = glm::vec2(pos[2 * i], pos[2 * i + 1]);
                m.velocity = glm::vec2(0.0f);
                m.acceleration = glm::vec2(0.0f);
                c.get<ExternalForces>(i).non_pressure_acceleration = glm::vec2(0.0f);
            } else {
                auto& m = c.get<MovementData3D>(i);
                m.position = glm::vec3(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]);
                m.velocity = glm::vec3(0.0f);
                m.acceleration = glm::vec3(0.0f);
                c.get<ExternalForces3D>(i).non_pressure_acceleration = glm::vec3(0.0f);
            }
            auto& info = c.get<ParticleInfo>(i);
            info.tag = (uint32_t)i;
            info.type = type ? type[i] : (uint8_t)ParticleTypeNormal;
            auto& pd = c.get<ParticleData>(i);
            pd.mass = 1.0f;
            pd.density = 1.0f;
            pd.pressure = 0.0f;
        }
    }

    // collection index of every tag
    std::vector<size_t> index_of_tag(ParticleCollection& c) {
        std::vector<size_t> idx(c.size());
        for (size_t i = 0; i < c.size(); i++)
            idx[c.get<ParticleInfo>(i).tag] = i;
        return idx;
    }

    // ------------------------------------------------------------------
    // solver wrapper
    // ------------------------------------------------------------------
    struct SolverBase {
        std::shared_ptr<ParticleCollection> collection;
        std::shared_ptr<ConstantTimestepGenerator> generator;
        Timepoint timepoint;
        int dim = 3;
        virtual ~SolverBase() = default;
        virtual IFluidSolverBase& base() = 0;
        virtual size_t last_iterations() { return 0; }
        virtual float last_avg_error() { return 0.0f; }
        virtual void iisph_extras(size_t i, float* out /*v*3, anp*3, s, aii, err*/) { (void)i; std::memset(out, 0, 9 * sizeof(float)); }
        virtual void neighbors_of(size_t i, std::vector<size_t>& out) = 0;
    };

    template <typename Solver>
    struct SolverImpl : SolverBase {
        std::shared_ptr<Solver> solver = std::make_shared<Solver>();
        IFluidSolverBase& base() override { return *solver; }
        void neighbors_of(size_t i, std::vector<size_t>& out) override {
            out.clear();
            auto nb = solver->neighborhood_search.get_neighbors(i);
            for (auto it = nb.begin(); it != nb.end(); ++it)
                out.push_back(*it);
        }
    };

    template <typename Solver>
    struct IisphImpl3D : SolverImpl<Solver> {
        size_t last_iterations() override { return this->solver->stat_last_iteration_count; }
        float last_avg_error() override { return this->solver->stat_last_average_predicted_density_error; }
        void iisph_extras(size_t i, float* out) override {
            auto& d = this->collection->template get<IISPHParticleData3D>(i);
            out[0] = d.predicted_velocity.x;
            out[1] = d.predicted_velocity.y;
            out[2] = d.predicted_velocity.z;
            out[3] = d.original_non_pressure_acceleration.x;
            out[4] = d.original_non_pressure_acceleration.y;
            out[5] = d.original_non_pressure_acceleration.z;
            out[6] = d.source_term;
            out[7] = d.diagonal_element;
            out[8] = d.predicted_density_error;
        }
    };

    template <typename Solver>
    struct IisphImpl2D : SolverImpl<Solver> {
        void iisph_extras(size_t i, float* out) override {
            auto& d = this->collection->template get<IISPHParticleData>(i);
            std::memset(out, 0, 9 * sizeof(float));
            out[0] = d.predicted_velocity.x;
            out[1] = d.predicted_velocity.y;
            out[6] = d.source_term;
            out[7] = d.diagonal_element;
        }
    };

    template <typename NS>
    SolverBase* make_solver_for_ns(int solver_kind, const float* settings) {
        // settings layout per solver kind (see ref_solver_create)
        if constexpr (std::is_same_v<NS, QuadraticNeighborhoodSearchDynamicAllocated> ||
                      std::is_same_v<NS, HashedNeighborhoodSearch>) {
            if (solver_kind == SOLVER_SESPH_2D) {
                auto* s = new SolverImpl<SESPHFluidSolver<CubicSplineKernel, NS, StdParallelForEach>>();
                s->solver->settings.StiffnessK = settings[0];
                s->solver->settings.Viscosity = settings[1];
                s->dim = 2;
                return s;
            }
            if (solver_kind == SOLVER_IISPH_2D) {
                auto* s = new IisphImpl2D<IISPHFluidSolver<CubicSplineKernel, NS, StdParallelForEach>>();
                s->solver->settings.MaxDensityErrorAllowed = settings[0];
                s->solver->settings.MinNumberOfIterations = (size_t)settings[1];
                s->solver->settings.MaxNumberOfIterations = (size_t)settings[2];
                s->solver->settings.Omega = settings[3];
                s->solver->settings.Gamma = settings[4];
                s->solver->settings.Viscosity = settings[5];
                s->dim = 2;
                return s;
            }
        } else {
            if (solver_kind == SOLVER_SESPH_3D) {
                auto* s = new SolverImpl<SESPHFluidSolver3D<CubicSplineKernel3D, NS, StdParallelForEach>>();
                s->solver->settings.StiffnessK = settings[0];
                s->solver->settings.Viscosity = settings[1];
                s->solver->settings.single_layer_boundary = settings[2] != 0.0f;
                s->solver->settings.single_layer_boundary_gamma_1 = settings[3];
                s->solver->settings.single_layer_boundary_gamma_2 = settings[4];
                s->dim = 3;
                return s;
            }
            if (solver_kind == SOLVER_IISPH_3D) {
                auto* s = new IisphImpl3D<IISPHFluidSolver3D<CubicSplineKernel3D, NS, StdParallelForEach>>();
                s->solver->settings.max_density_error_allowed = settings[0];
                s->solver->settings.min_number_of_iterations = (size_t)settings[1];
                s->solver->settings.max_number_of_iterations = (size_t)settings[2];
                s->solver->settings.omega = settings[3];
                s->solver->settings.gamma = settings[4];
                s->solver->settings.viscosity = settings[5];
                s->solver->settings.single_layer_boundary = settings[6] != 0.0f;
                s->solver->settings.single_layer_boundary_gamma_1 = settings[7];
                s->dim = 3;
                return s;
            }
        }
        return nullptr;
    }
} // namespace

extern "C" {

const char* ref_last_error() { return g_last_error.c_str(); }

// Kernel values for n vectors x (dim floats each) at the given support:
// W[i] = GetKernelValue(x_i), dW[i*dim..] = GetKernelDerivativeValue(x_i)
// (CubicSplineKernel.cpp:9-63, CubicSplineKernel3D.cpp:7-48).
void ref_kernel_eval(int dim, float support, int64_t n, const float* x, float* W, float* dW) {
    if (dim == 2) {
        CubicSplineKernel k;
        k.kernel_support = support;
        k.initialize();
        for (int64_t i = 0; i < n; i++) {
            glm::vec2 v(x[2 * i], x[2 * i + 1]);
            W[i] = k.GetKernelValue(v);
            glm::vec2 d = k.GetKernelDerivativeValue(v);
            dW[2 * i] = d.x;
            dW[2 * i + 1] = d.y;
        }
    } else {
        CubicSplineKernel3D k;
        k.kernel_support = support;
        k.initialize();
        for (int64_t i = 0; i < n; i++) {
            glm::vec3 v(x[3 * i], x[3 * i + 1], x[3 * i + 2]);
            W[i] = k.GetKernelValue(v);
            glm::vec3 d = k.GetKernelDerivativeValue(v);
            dW[3 * i] = d.x;
            dW[3 * i + 1] = d.y;
            dW[3 * i + 2] = d.z;
        }
    }
}

// ConstantTimestepGenerator::get_non_cfl_validating_timestep
// (ConstantTimestepGenerator.cpp:17-41) for n (max_acc, max_vel) pairs.
void ref_cfl_timestep(float timestep, float lambda_v, float lambda_a, float particle_size, int64_t n,
                      const float* max_acc, const float* max_vel, float* out) {
    ConstantTimestepGenerator g;
    g.settings.timestep = timestep;
    g.settings.lambda_v = lambda_v;
    g.settings.lambda_a = lambda_a;
    g.parameters.particle_size = particle_size;
    for (int64_t i = 0; i < n; i++)
        out[i] = g.get_non_cfl_validating_timestep(max_acc[i], max_vel[i]);
}

// DynamicCflTimestepGenerator::generate_next_timestep
// (DynamicCflTimestepGenerator.cpp:45-59) over one collection of n particles
// (dim 2 or 3: MovementData or MovementData3D): its generated time step.
float ref_dynamic_timestep(int dim, int64_t n, const float* vel, const float* acc, const uint8_t* type,
                           float particle_size, float min_ts, float max_ts, float lambda_v, float lambda_a) {
    auto c = std::make_shared<ParticleCollection>();
    if (dim == 3) c->add_type<MovementData3D>();
    else c->add_type<MovementData>();
    c->add_type<ParticleInfo>();
    for (int64_t i = 0; i < n; i++) {
        const size_t k = c->add();
        if (dim == 3) {
            auto& m = c->get<MovementData3D>(k);
            m.velocity = glm::vec3(vel[3 * i], vel[3 * i + 1], vel[3 * i + 2]);
            m.acceleration = glm::vec3(acc[3 * i], acc[3 * i + 1], acc[3 * i + 2]);
        } else {
            auto& m = c->get<MovementData>(k);
            m.velocity = glm::vec2(vel[2 * i], vel[2 * i + 1]);
            m.acceleration = glm::vec2(acc[2 * i], acc[2 * i + 1]);
        }
        c->get<ParticleInfo>(k).type = type[i];
        c->get<ParticleInfo>(k).tag = (uint32_t)i;
    }
    DynamicCflTimestepGenerator g;
    g.settings.min_timestep = min_ts;
    g.settings.max_timestep = max_ts;
    g.settings.lambda_v = lambda_v;
    g.settings.lambda_a = lambda_a;
    g.parameters.particle_size = particle_size;
    g.parameters.particle_collection = c;
    g.generate_next_timestep();
    return g.get_generated_timestep();
}

// ---------------------------------------------------------------------------
// neighborhood search
// ---------------------------------------------------------------------------
void* ref_ns_create(int kind, int64_t n, const float* pos, const uint8_t* type, float radius) {
    NsBase* ns = nullptr;
    switch (kind) {
        case NS_QUADRATIC_2D: ns = new NsImpl<QuadraticNeighborhoodSearchDynamicAllocated>(); break;
        case NS_HASHED_2D: ns = new NsImpl<HashedNeighborhoodSearch>(); break;
        case NS_QUADRATIC_3D: ns = new NsImpl<QuadraticNeighborhoodSearch3D>(); break;
        case NS_HASHED_3D: ns = new NsImpl<HashedNeighborhoodSearch3D>(); break;
        case NS_COMPRESSED_3D: ns = new NsImpl<CompressedNeighborhoodSearch>(); break;
        default: g_last_error = "unknown search kind"; return nullptr;
    }
    ns->dim = is_3d_ns(kind) ? 3 : 2;
    ns->collection = std::make_shared<ParticleCollection>();
    fill_collection(*ns->collection, ns->dim, n, pos, type);
    switch (kind) {
#define FS_SETUP(T)                                              \
    {                                                            \
        auto* impl = static_cast<NsImpl<T>*>(ns);                \
        impl->search.collection = ns->collection;                \
        impl->search.search_radius = radius;                     \
        impl->search.initialize();                               \
    }                                                            \
    break;
        case NS_QUADRATIC_2D: FS_SETUP(QuadraticNeighborhoodSearchDynamicAllocated)
        case NS_HASHED_2D: FS_SETUP(HashedNeighborhoodSearch)
        case NS_QUADRATIC_3D: FS_SETUP(QuadraticNeighborhoodSearch3D)
        case NS_HASHED_3D: FS_SETUP(HashedNeighborhoodSearch3D)
        case NS_COMPRESSED_3D: FS_SETUP(CompressedNeighborhoodSearch)
#undef FS_SETUP
    }
    return ns;
}

void ref_ns_destroy(void* h) { delete static_cast<NsBase*>(h); }

// Overwrite the positions, addressed by tag (input index).
void ref_ns_set_positions(void* h, const float* pos) {
    auto* ns = static_cast<NsBase*>(h);
    auto& c = *ns->collection;
    for (size_t i = 0; i < c.size(); i++) {
        uint32_t t = c.get<ParticleInfo>(i).tag;
        if (ns->dim == 2)
            c.get<MovementData>(i).position = glm::vec2(pos[2 * t], pos[2 * t + 1]);
        else
            c.get<MovementData3D>(i).position = glm::vec3(pos[3 * t], pos[3 * t + 1], pos[3 * t + 2]);
    }
}

// Runs find_neighbors(); returns 0, or -1 when the reference threw (message in ref_last_error).
int ref_ns_find(void* h) {
    try {
        static_cast<NsBase*>(h)->find();
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return -1;
    }
    return 0;
}

// BoundaryPreprocessor::execute_simulation_step (BoundaryPreprocessor.cpp:7-48)
// on search h's collection (3D) through the search's own neighborhood
// interface, after ref_ns_find. mass: the masses to start from, by tag; out:
// the masses afterwards, by tag. Returns 0, or -1 when the reference threw.
int ref_boundary_preprocess(void* h, const float* mass, float particle_size, float rest_density, float* out) {
    auto* ns = static_cast<NsBase*>(h);
    auto& c = *ns->collection;
    for (size_t i = 0; i < c.size(); i++) c.get<ParticleData>(i).mass = mass[c.get<ParticleInfo>(i).tag];
    try {
        BoundaryPreprocessor bp;
        bp.simulation_data.collection = ns->collection;
        bp.simulation_data.particle_size = particle_size;
        bp.simulation_data.rest_density = rest_density;
        bp.simulation_data.neighborhood_interface = ns->interface();
        bp.simulation_data.notify_that_data_changed();
        Timepoint t;
        bp.execute_simulation_step(t, true);
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return -1;
    }
    for (size_t i = 0; i < c.size(); i++) out[c.get<ParticleInfo>(i).tag] = c.get<ParticleData>(i).mass;
    return 0;
}

// ParticleIntersectionAccelerator::is_intersecting_with_particles
// (ParticleIntersectionAccelerator.cpp:20-74) after prepare() (:8-18), without
// a sampler (no random offset along the ray): for each ray the hit type (-1:
// none; 0/1: the fluid surface from outside/inside; 2: a boundary surface),
// the point and normal of the intersection and length_until_hit.
int ref_trace_rays(int64_t n, const float* pos, const float* mass, const uint8_t* type, float particle_size,
                   float rest_density, int64_t nrays, const float* origins, const float* directions, int32_t* hit,
                   float* point, float* normal, float* length) {
    try {
        auto c = std::make_shared<ParticleCollection>();
        fill_collection(*c, 3, n, pos, type);
        for (size_t i = 0; i < c->size(); i++) c->get<ParticleData>(i).mass = mass[c->get<ParticleInfo>(i).tag];
        Raytracer::ParticleIntersectionAccelerator acc;
        acc.particle_collection = c;
        acc.particle_size = particle_size;
        acc.rest_density = rest_density;
        acc.sampler = nullptr;
        acc.prepare();
        for (int64_t r = 0; r < nrays; r++) {
            Raytracer::Ray ray;
            ray.starting_point = glm::vec3(origins[3 * r], origins[3 * r + 1], origins[3 * r + 2]);
            ray.normalized_direction = glm::vec3(directions[3 * r], directions[3 * r + 1], directions[3 * r + 2]);
            Raytracer::IntersectionResult res{};
            const bool h = acc.is_intersecting_with_particles(ray, res);
            hit[r] = h ? (int32_t)res.intersection_result_type : -1;
            for (int a = 0; a < 3; a++) {
                point[3 * r + a] = h ? res.point_of_intersection[a] : 0.0f;
                normal[3 * r + a] = h ? res.normal_at_intersection[a] : 0.0f;
            }
            length[r] = h ? ray.length_until_hit : -1.0f;
        }
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return -1;
    }
    return 0;
}

// Neighbor lists in tag space, in the reference's own list order: for tag t,
// idx[offsets[t] .. offsets[t+1]) are the tags of its neighbors. With
// idx == nullptr only offsets are filled. Returns the total count.
// ToneMapper::map_render_target_to_image (ToneMapper.cpp:71-102) on a w x h
// render target of radiance (3 floats per pixel, row-major from the top-left
// pixel); rgba receives the image's 4 bytes per pixel. filmic selects the
// ACES curve instead of the exponential one.
int ref_tone_map(int64_t w, int64_t h, const float* radiance, float exposure, float gamma, int gamma_enabled,
                 int filmic, uint8_t* rgba) {
    try {
        Raytracer::RenderTarget target;
        target.set_size((size_t)w, (size_t)h);
        for (int64_t y = 0; y < h; y++)
            for (int64_t x = 0; x < w; x++) {
                const float* v = radiance + 3 * (y * w + x);
                target.set((size_t)x, (size_t)y, glm::vec3(v[0], v[1], v[2]));
            }
        Image image((size_t)w, (size_t)h);
        Raytracer::ToneMapper tm;
        tm.settings.exposure = exposure;
        tm.settings.gamma = gamma;
        tm.settings.gamma_correction_enabled = gamma_enabled != 0;
        tm.settings.tone_mapper_function = filmic ? Raytracer::ToneMapper::ToneMapperSettings::ToneMapperFunction::Filmic
                                                  : Raytracer::ToneMapper::ToneMapperSettings::ToneMapperFunction::Exponential;
        tm.map_render_target_to_image(target, image);
        for (int64_t y = 0; y < h; y++)
            for (int64_t x = 0; x < w; x++) {
                const Image::Color c = image.get((size_t)x, (size_t)y);
                uint8_t* o = rgba + 4 * (y * w + x);
                o[0] = c.r;
                o[1] = c.g;
                o[2] = c.b;
                o[3] = c.a;
            }
        return 0;
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return -1;
    }
}

// The global sensors of ParticleStatistics.cpp through their own
// calculate_for_timepoint: out = {density max, min, avg, pressure max, min,
// avg, velocity max, min, avg, kinetic energy, potential energy}, counts =
// {normal, boundary, inactive}. The velocity and energy sensors read the 2D
// MovementData (ParticleStatistics.cpp:101-167); for dim 3 they are not run
// and their entries are NaN.
int ref_global_stats(int dim, int64_t n, const float* pos, const float* vel, const float* mass, const float* density,
                     const float* pressure, const uint8_t* type, float gravity, float zero_height, float* out,
                     int64_t* counts) {
    try {
        auto c = std::make_shared<ParticleCollection>();
        fill_collection(*c, dim, n, pos, type);
        for (int64_t i = 0; i < n; i++) {
            if (dim == 2) c->get<MovementData>(i).velocity = glm::vec2(vel[2 * i], vel[2 * i + 1]);
            else c->get<MovementData3D>(i).velocity = glm::vec3(vel[3 * i], vel[3 * i + 1], vel[3 * i + 2]);
            auto& pd = c->get<ParticleData>(i);
            pd.mass = mass[i];
            pd.density = density[i];
            pd.pressure = pressure[i];
        }
        Timepoint tp;
        Sensors::GlobalDensitySensor ds;
        ds.simulator_data.collection = c;
        const auto d = ds.calculate_for_timepoint(tp);
        Sensors::GlobalPressureSensor ps;
        ps.simulator_data.collection = c;
        const auto p = ps.calculate_for_timepoint(tp);
        Sensors::GlobalParticleCountSensor cs;
        cs.simulator_data.collection = c;
        const auto k = cs.calculate_for_timepoint(tp);
        const float nan = std::numeric_limits<float>::quiet_NaN();
        float v[3] = {nan, nan, nan}, e[2] = {nan, nan};
        if (dim == 2) {
            Sensors::GlobalVelocitySensor vs;
            vs.simulator_data.collection = c;
            const auto vd = vs.calculate_for_timepoint(tp);
            v[0] = vd.maximum;
            v[1] = vd.minimum;
            v[2] = vd.average;
            Sensors::GlobalEnergySensor es;
            es.simulator_data.collection = c;
            es.simulator_parameters.gravity = gravity;
            es.settings.relative_zero_height = zero_height;
            const auto ed = es.calculate_for_timepoint(tp);
            e[0] = ed.kinetic;
            e[1] = ed.potential;
        }
        const float vals[11] = {d.maximum, d.minimum, d.average, p.maximum, p.minimum, p.average,
                                v[0], v[1], v[2], e[0], e[1]};
        std::memcpy(out, vals, sizeof(vals));
        counts[0] = (int64_t)k.normal_particles;
        counts[1] = (int64_t)k.boundary_particles;
        counts[2] = (int64_t)k.inactive_particles;
        return 0;
    } catch (const std::exception& ex) {
        g_last_error = ex.what();
        return -1;
    }
}

int64_t ref_ns_lists(void* h, int64_t* offsets, int64_t* idx) {
    auto* ns = static_cast<NsBase*>(h);
    auto& c = *ns->collection;
    auto where = index_of_tag(c);
    std::vector<size_t> tmp;
    int64_t total = 0;
    for (size_t t = 0; t < c.size(); t++) {
        offsets[t] = total;
        try {
            ns->neighbors_of(where[t], tmp);
        } catch (const std::exception& e) {
            g_last_error = e.what();
            return -1;
        }
        if (idx)
            for (size_t k = 0; k < tmp.size(); k++)
                idx[total + (int64_t)k] = c.get<ParticleInfo>(tmp[k]).tag;
        total += (int64_t)tmp.size();
    }
    offsets[c.size()] = total;
    return total;
}

// Position-based query (get_neighbors(vec)); writes up to cap neighbor tags, returns the count.
int64_t ref_ns_query_position(void* h, const float* p, int64_t* out, int64_t cap) {
    auto* ns = static_cast<NsBase*>(h);
    std::vector<size_t> tmp;
    try {
        ns->neighbors_of_position(p, tmp);
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return -1;
    }
    auto& c = *ns->collection;
    for (size_t k = 0; k < tmp.size() && (int64_t)k < cap; k++)
        out[k] = c.get<ParticleInfo>(tmp[k]).tag;
    return (int64_t)tmp.size();
}

// ---------------------------------------------------------------------------
// solvers
// ---------------------------------------------------------------------------
// settings layout:
//   SESPH_2D: StiffnessK, Viscosity
//   SESPH_3D: StiffnessK, Viscosity, single_layer_boundary, gamma_1, gamma_2
//   IISPH_2D: MaxDensityErrorAllowed, MinIter, MaxIter, Omega, Gamma, Viscosity
//   IISPH_3D: max_density_error, min_iter, max_iter, omega, gamma, viscosity, single_layer_boundary, gamma_1
// params: rest_density, gravity, particle_size
// generator: timestep, lambda_v, lambda_a
// Arrays are in input (tag) order; vectors have dim floats per particle.
void* ref_solver_create(int solver_kind, int ns_kind, int64_t n, const float* pos, const float* vel, const float* acc,
                        const float* mass, const float* density, const float* pressure, const uint8_t* type,
                        const float* ext, const float* params, const float* settings, const float* generator) {
    SolverBase* s = nullptr;
    switch (ns_kind) {
        case NS_QUADRATIC_2D: s = make_solver_for_ns<QuadraticNeighborhoodSearchDynamicAllocated>(solver_kind, settings); break;
        case NS_HASHED_2D: s = make_solver_for_ns<HashedNeighborhoodSearch>(solver_kind, settings); break;
        case NS_QUADRATIC_3D: s = make_solver_for_ns<QuadraticNeighborhoodSearch3D>(solver_kind, settings); break;
        case NS_HASHED_3D: s = make_solver_for_ns<HashedNeighborhoodSearch3D>(solver_kind, settings); break;
        case NS_COMPRESSED_3D: s = make_solver_for_ns<CompressedNeighborhoodSearch>(solver_kind, settings); break;
        default: break;
    }
    if (!s) {
        g_last_error = "unsupported solver / neighborhood search combination";
        return nullptr;
    }
    const int dim = s->dim;
    s->collection = std::make_shared<ParticleCollection>();
    fill_collection(*s->collection, dim, n, pos, type);
    auto& c = *s->collection;
    for (int64_t i = 0; i < n; i++) {
        if (dim == 2) {
            auto& m = c.get<MovementData>(i);
            m.velocity = glm::vec2(vel[2 * i], vel[2 * i + 1]);
            m.acceleration = glm::vec2(acc[2 * i], acc[2 * i + 1]);
            c.get<ExternalForces>(i).non_pressure_acceleration = ext ? glm::vec2(ext[2 * i], ext[2 * i + 1]) : glm::vec2(0.0f);
        } else {
            auto& m = c.get<MovementData3D>(i);
            m.velocity = glm::vec3(vel[3 * i], vel[3 * i + 1], vel[3 * i + 2]);
            m.acceleration = glm::vec3(acc[3 * i], acc[3 * i + 1], acc[3 * i + 2]);
            c.get<ExternalForces3D>(i).non_pressure_acceleration =
                ext ? glm::vec3(ext[3 * i], ext[3 * i + 1], ext[3 * i + 2]) : glm::vec3(0.0f);
        }
        auto& pd = c.get<ParticleData>(i);
        pd.mass = mass[i];
        pd.density = density[i];
        pd.pressure = pressure[i];
    }
    s->generator = std::make_shared<ConstantTimestepGenerator>();
    s->generator->settings.timestep = generator[0];
    s->generator->settings.lambda_v = generator[1];
    s->generator->settings.lambda_a = generator[2];
    s->generator->parameters.particle_size = params[2];
    s->generator->parameters.particle_collection = s->collection;

    auto& b = s->base();
    b.parameters.rest_density = params[0];
    b.parameters.gravity = params[1];
    b.parameters.particle_size = params[2];
    b.parameters.notify_that_data_changed();
    b.data.collection = s->collection;
    b.data.timestep_generator = s->generator;
    b.data.notify_that_data_changed();
    return s;
}

void ref_solver_destroy(void* h) { delete static_cast<SolverBase*>(h); }

// One Simulator-style step. stats = {desired_dt, actual_dt, iterations, avg_density_error}.
int ref_solver_step(void* h, float* stats) {
    auto* s = static_cast<SolverBase*>(h);
    try {
        s->generator->generate_next_timestep();
        float dt = s->generator->get_generated_timestep();
        s->timepoint.desired_time_step = dt;
        s->timepoint.actual_time_step = dt;
        s->base().execute_neighborhood_search();
        s->base().execute_simulation_step(s->timepoint);
        s->timepoint.simulation_time += s->timepoint.actual_time_step;
        s->timepoint.timestep_number++;
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return -1;
    }
    if (stats) {
        stats[0] = s->timepoint.desired_time_step;
        stats[1] = s->timepoint.actual_time_step;
        stats[2] = (float)s->last_iterations();
        stats[3] = s->last_avg_error();
    }
    return 0;
}

// Runs `steps` steps back to back (used for CPU timing); stats of the last one.
int ref_solver_run(void* h, int64_t steps, float* stats) {
    for (int64_t k = 0; k < steps; k++)
        if (ref_solver_step(h, stats) != 0)
            return -1;
    return 0;
}

// Current state in tag order. Any pointer may be null. iisph: 9 floats per
// particle {v* (3, 2D: 2 + pad), a_np (3), source term, diagonal, density error}.
void ref_solver_state(void* h, float* pos, float* vel, float* acc, float* mass, float* density, float* pressure,
                      uint8_t* type, float* ext, float* iisph) {
    auto* s = static_cast<SolverBase*>(h);
    auto& c = *s->collection;
    const int dim = s->dim;
    for (size_t i = 0; i < c.size(); i++) {
        size_t t = c.get<ParticleInfo>(i).tag;
        if (dim == 2) {
            auto& m = c.get<MovementData>(i);
            if (pos) { pos[2 * t] = m.position.x; pos[2 * t + 1] = m.position.y; }
            if (vel) { vel[2 * t] = m.velocity.x; vel[2 * t + 1] = m.velocity.y; }
            if (acc) { acc[2 * t] = m.acceleration.x; acc[2 * t + 1] = m.acceleration.y; }
            if (ext) {
                auto& e = c.get<ExternalForces>(i).non_pressure_acceleration;
                ext[2 * t] = e.x; ext[2 * t + 1] = e.y;
            }
        } else {
            auto& m = c.get<MovementData3D>(i);
            if (pos) { pos[3 * t] = m.position.x; pos[3 * t + 1] = m.position.y; pos[3 * t + 2] = m.position.z; }
            if (vel) { vel[3 * t] = m.velocity.x; vel[3 * t + 1] = m.velocity.y; vel[3 * t + 2] = m.velocity.z; }
            if (acc) { acc[3 * t] = m.acceleration.x; acc[3 * t + 1] = m.acceleration.y; acc[3 * t + 2] = m.acceleration.z; }
            if (ext) {
                auto& e = c.get<ExternalForces3D>(i).non_pressure_acceleration;
                ext[3 * t] = e.x; ext[3 * t + 1] = e.y; ext[3 * t + 2] = e.z;
            }
        }
        auto& pd = c.get<ParticleData>(i);
        if (mass) mass[t] = pd.mass;
        if (density) density[t] = pd.density;
        if (pressure) pressure[t] = pd.pressure;
        if (type) type[t] = c.get<ParticleInfo>(i).type;
        if (iisph) s->iisph_extras(i, iisph + 9 * t);
    }
}

// The solver's current neighbor lists in tag space (after the last step's search).
int64_t ref_solver_lists(void* h, int64_t* offsets, int64_t* idx) {
    auto* s = static_cast<SolverBase*>(h);
    auto& c = *s->collection;
    auto where = index_of_tag(c);
    std::vector<size_t> tmp;
    int64_t total = 0;
    for (size_t t = 0; t < c.size(); t++) {
        offsets[t] = total;
        s->neighbors_of(where[t], tmp);
        if (idx)
            for (size_t k = 0; k < tmp.size(); k++)
                idx[total + (int64_t)k] = c.get<ParticleInfo>(tmp[k]).tag;
        total += (int64_t)tmp.size();
    }
    offsets[c.size()] = total;
    return total;
}

} // extern "C"
