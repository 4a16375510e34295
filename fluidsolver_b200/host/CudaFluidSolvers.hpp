// C++ drop-in solvers for libFluid: IFluidSolverBase implementations
// (src/libFluid/fluidSolver/IFluidSolver.hpp:16-34) that run the neighborhood
// search and the SESPH / IISPH timestep on a B200 through the C-ABI in
// include/fluidsolver_b200.h. They mirror the reference solvers' public
// surface -- `parameters`, `data`, `settings`, the IISPH statistics and the
// neighborhood interface -- so that SolverSerializer, the Simulator, entities
// and sensors use them unchanged. To be selectable from scenario files they
// are registered where the reference maps its type strings to solver types
// (SolverSerializer.cpp:137-219 and the dynamic_pointer_cast chains of
// :15-95, FluidSolverTypes.cpp, IisphSensor.cpp:61-78).
//
//   LibFluid::Cuda::IISPHFluidSolver3D   replaces IISPHFluidSolver3D<...>  (IISPHFluidSolver3D.hpp:22-610)
//   LibFluid::Cuda::SESPHFluidSolver3D   replaces SESPHFluidSolver3D<...>  (SESPHFluidSolver3D.hpp:12-339)
//   LibFluid::Cuda::IISPHFluidSolver     replaces IISPHFluidSolver<...>    (IISPHFluidSolver.hpp:21-548)
//   LibFluid::Cuda::SESPHFluidSolver     replaces SESPHFluidSolver<...>    (SESPHFluidSolver.hpp:12-299)
//
// The template argument selects the neighbor-set contract of the reference
// search the solver was instantiated with (FS_SEARCH_*).
//
// Host collection. With `sync_host_collection` (the default) the collection
// stays authoritative as in the reference: it is uploaded before every search
// and the step's results are written back after every step, so entities and
// sensors see and may change every field. Without it the state stays on the
// device between steps and download_collection() writes it back on demand.
#pragma once

#include "fluidSolver/IFluidSolver.hpp"
#include "fluidSolver/Particle.hpp"
#include "fluidSolver/solver/settings/IISPHSettings.hpp"
#include "fluidSolver/solver/settings/IISPHSettings3D.hpp"
#include "fluidSolver/solver/settings/SESPHSettings.hpp"
#include "fluidSolver/solver/settings/SESPHSettings3D.hpp"
#include "time/ConstantTimestepGenerator.hpp"
#include "time/DynamicCflTimestepGenerator.hpp"
#include "entities/SimulationEntity.hpp"

#include "fluidsolver_b200.h"

#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace LibFluid {
    namespace Cuda {

        class Error : public std::runtime_error {
          public:
            fs_status status;
            Error(fs_status s, const std::string& what) : std::runtime_error(what), status(s) {}
        };

        inline void check(fs_status s, const char* call) {
            if (s != FS_OK) throw Error(s, std::string(call) + ": " + fs_last_error());
        }

        // Dense host copies of the collection's components (the collection
        // stores one struct vector per component, ParticleCollection.hpp:11-177).
        template <int DIM>
        struct HostArrays {
            std::vector<float> position, velocity, acceleration, external, mass, density, pressure;
            std::vector<uint8_t> type;
            std::vector<uint32_t> tag;

            void resize(size_t n) {
                position.resize(n * DIM);
                velocity.resize(n * DIM);
                acceleration.resize(n * DIM);
                external.resize(n * DIM);
                mass.resize(n);
                density.resize(n);
                pressure.resize(n);
                type.resize(n);
                tag.resize(n);
            }

            fs_particles view(size_t n) {
                fs_particles p{};
                p.n = (int64_t)n;
                p.position = position.data();
                p.velocity = velocity.data();
                p.acceleration = acceleration.data();
                p.external = external.data();
                p.mass = mass.data();
                p.density = density.data();
                p.pressure = pressure.data();
                p.type = type.data();
                p.tag = tag.data();
                return p;
            }
        };

        template <int DIM>
        struct Components;
        template <>
        struct Components<2> {
            using Movement = MovementData;
            using External = ExternalForces;
        };
        template <>
        struct Components<3> {
            using Movement = MovementData3D;
            using External = ExternalForces3D;
        };

        template <int DIM, int SOLVER, int SEARCH>
        class FluidSolverBase : public IFluidSolverBase {
          public:
            using M = typename Components<DIM>::Movement;
            using E = typename Components<DIM>::External;

            int32_t precision = FS_PRECISION_FP32_KAHAN;
            uint32_t flags = 0;
            int32_t device = 0;
            bool sync_host_collection = true;
            fs_step_stats last_stats{};

            FluidSolverBase() = default;
            FluidSolverBase(const FluidSolverBase&) = delete;
            FluidSolverBase& operator=(const FluidSolverBase&) = delete;
            ~FluidSolverBase() override {
                if (ctx) fs_destroy(ctx);
            }

            void initialize() override {
                if (!data.collection) throw Error(FS_ERR_INVALID, "Particle collection is null.");
                const size_t n = data.collection->size();
                fs_params p = make_params(n);
                if (!ctx || (size_t)capacity < n || p.precision != made.precision || p.flags != made.flags) {
                    if (ctx) fs_destroy(ctx);
                    ctx = nullptr;
                    p.max_particles = (int64_t)(n + n / 4 + 64);
                    check(fs_create(&p, &ctx), "fs_create");
                    capacity = p.max_particles;
                    made = p;
                    host_dirty = true;
                } else {
                    p.max_particles = capacity;
                    check(fs_set_params(ctx, &p), "fs_set_params");
                    made = p;
                }
                if (data.has_data_changed()) {
                    data.acknowledge_data_change();
                    host_dirty = true;
                }
                parameters.acknowledge_data_change();
                settings_acknowledge();
            }

            void execute_neighborhood_search() override {
                initialize();
                if (host_dirty || sync_host_collection) upload_collection();
                check(fs_find_neighbors(ctx), "fs_find_neighbors");
                neighbors_valid = false;
            }

            void execute_simulation_step(Timepoint& timestep) override {
                initialize();
                check(fs_solve_step(ctx, timestep.desired_time_step, &last_stats), "fs_solve_step");
                timestep.desired_time_step = last_stats.desired_dt;   // the generator's (device's with the dynamic one)
                timestep.actual_time_step = last_stats.actual_dt;
                if (sync_host_collection) download_collection();
            }

            std::shared_ptr<NeighborhoodInterface> create_neighborhood_interface() override {
                auto res = std::make_shared<NeighborhoodInterface>();
                res->link.get_by_index = [this](size_t index) { return wrap(lists_of(index)); };
                res->link.get_by_position = [this](const glm::vec2& p) {
                    float q[3] = {p.x, p.y, 0.0f};
                    return wrap(query(q));
                };
                res->link.get_by_position_3d = [this](const glm::vec3& p) {
                    float q[3] = {p.x, p.y, p.z};
                    return wrap(query(q));
                };
                res->link.get_search_radius = [this] { return parameters.particle_size * 2.0f; };
                return res;
            }

            void create_compatibility_report(CompatibilityReport& report) override {
                report.begin_scope("Cuda::FluidSolver");
                if (data.collection == nullptr) {
                    report.add_issue("Particle collection is null.");
                } else {
                    if (!data.collection->template is_type_present<M>())
                        report.add_issue("Particles are missing the movement data attribute.");
                    if (!data.collection->template is_type_present<ParticleData>())
                        report.add_issue("Particles are missing the ParticleData attribute.");
                    if (!data.collection->template is_type_present<ParticleInfo>())
                        report.add_issue("Particles are missing the ParticleInfo attribute.");
                }
                if (data.timestep_generator == nullptr) report.add_issue("Timestep generator is null");
                fs_params p = make_params(data.collection ? data.collection->size() : 1);
                fs_ctx* probe = nullptr;
                p.max_particles = 1;
                const fs_status s = fs_create(&p, &probe);
                if (s == FS_ERR_INVALID) report.add_issue(fs_last_error());
                if (s == FS_ERR_NO_DEVICE) report.add_issue("No B200-class (sm_100) device available.");
                if (probe) fs_destroy(probe);
                report.end_scope();
            }

            // copies the device state into the collection (host order)
            void download_collection() {
                auto& c = *data.collection;
                const size_t n = c.size();
                host.resize(n);
                fs_particles v = host.view(n);
                v.type = nullptr;
                v.tag = nullptr;
                check(fs_download(ctx, &v), "fs_download");
                for (size_t i = 0; i < n; i++) {
                    auto& m = c.template get<M>(i);
                    for (int a = 0; a < DIM; a++) {
                        m.position[a] = host.position[i * DIM + a];
                        m.velocity[a] = host.velocity[i * DIM + a];
                        m.acceleration[a] = host.acceleration[i * DIM + a];
                    }
                    if (c.template is_type_present<E>()) {
                        auto& e = c.template get<E>(i).non_pressure_acceleration;
                        for (int a = 0; a < DIM; a++) e[a] = host.external[i * DIM + a];
                    }
                    auto& pd = c.template get<ParticleData>(i);
                    pd.mass = host.mass[i];   // the boundary preprocessor changes it on the device
                    pd.density = host.density[i];
                    pd.pressure = host.pressure[i];
                }
            }

            fs_ctx* context() const { return ctx; }

            // BoundaryPreprocessor's arithmetic (BoundaryPreprocessor.cpp:7-48) on the device state,
            // between the search and the step; the masses reach the collection with the next download
            void boundary_preprocess() {
                initialize();
                check(fs_boundary_preprocess(ctx), "fs_boundary_preprocess");
            }

            // the global sensors of ParticleStatistics.cpp:17-201 over the device state
            fs_global_stats global_statistics(float zero_height = 0.0f) {
                initialize();
                fs_global_stats st{};
                check(fs_global_statistics(ctx, zero_height, &st), "fs_global_statistics");
                return st;
            }

          protected:
            virtual void fill_settings(fs_params& p) = 0;
            virtual void settings_acknowledge() = 0;

            fs_params make_params(size_t n) {
                fs_params p;
                fs_params_default(&p, DIM, SOLVER, SEARCH);
                p.precision = precision;
                p.flags = flags;
                p.device = device;
                p.rest_density = parameters.rest_density;
                p.gravity = parameters.gravity;
                p.particle_size = parameters.particle_size;
                p.max_particles = (int64_t)(n ? n : 1);
                if (auto g = std::dynamic_pointer_cast<ConstantTimestepGenerator>(data.timestep_generator)) {
                    p.timestep = g->settings.timestep;
                    p.lambda_v = g->settings.lambda_v;
                    p.lambda_a = g->settings.lambda_a;
                } else if (auto d = std::dynamic_pointer_cast<DynamicCflTimestepGenerator>(data.timestep_generator)) {
                    // the device generates the time step inside the step (the value the
                    // Simulator passes in is then ignored)
                    p.timestep_generator = FS_TIMESTEP_DYNAMIC_CFL;
                    p.min_timestep = d->settings.min_timestep;
                    p.max_timestep = d->settings.max_timestep;
                    p.timestep = d->settings.max_timestep;
                    p.lambda_v = d->settings.lambda_v;
                    p.lambda_a = d->settings.lambda_a;
                }
                fill_settings(p);
                return p;
            }

            void upload_collection() {
                auto& c = *data.collection;
                const size_t n = c.size();
                host.resize(n);
                const bool has_ext = c.template is_type_present<E>();
                for (size_t i = 0; i < n; i++) {
                    const auto& m = c.template get<M>(i);
                    for (int a = 0; a < DIM; a++) {
                        host.position[i * DIM + a] = m.position[a];
                        host.velocity[i * DIM + a] = m.velocity[a];
                        host.acceleration[i * DIM + a] = m.acceleration[a];
                        host.external[i * DIM + a] = has_ext ? c.template get<E>(i).non_pressure_acceleration[a] : 0.0f;
                    }
                    const auto& pd = c.template get<ParticleData>(i);
                    host.mass[i] = pd.mass;
                    host.density[i] = pd.density;
                    host.pressure[i] = pd.pressure;
                    const auto& info = c.template get<ParticleInfo>(i);
                    host.type[i] = info.type;
                    host.tag[i] = info.tag;
                }
                fs_particles v = host.view(n);
                check(fs_upload(ctx, &v), "fs_upload");
                host_dirty = false;
            }

            // neighbor lists of the last search, host index space
            const std::vector<size_t>* lists_of(size_t index) {
                if (!neighbors_valid) {
                    const size_t n = data.collection->size();
                    std::vector<int64_t> off(n + 1);
                    int64_t total = 0;
                    fs_status s = fs_get_neighbors_csr(ctx, off.data(), nullptr, &total);
                    if (s != FS_OK && s != FS_ERR_CAPACITY) check(s, "fs_get_neighbors_csr");
                    std::vector<int64_t> idx((size_t)total);
                    s = fs_get_neighbors_csr(ctx, off.data(), idx.data(), &total);
                    if (s != FS_OK && s != FS_ERR_CAPACITY) check(s, "fs_get_neighbors_csr");
                    lists.assign(n, {});
                    for (size_t i = 0; i < n; i++) lists[i].assign(idx.begin() + off[i], idx.begin() + off[i + 1]);
                    neighbors_valid = true;
                }
                return &lists.at(index);
            }

            std::shared_ptr<std::vector<size_t>> query(const float* q) {
                std::vector<int64_t> out(4096);
                int64_t count = 0;
                check(fs_query_position(ctx, q, out.data(), (int64_t)out.size(), &count), "fs_query_position");
                if (count > (int64_t)out.size()) {
                    out.resize((size_t)count);
                    check(fs_query_position(ctx, q, out.data(), count, &count), "fs_query_position");
                }
                return std::make_shared<std::vector<size_t>>(out.begin(), out.begin() + count);
            }

            // NeighborhoodInterface iterators over a list of indices
            struct It {
                std::shared_ptr<const std::vector<size_t>> keep;
                const std::vector<size_t>* v;
                size_t pos;
            };
            static NeighborhoodInterface::Neighbors wrap_shared(std::shared_ptr<const std::vector<size_t>> keep,
                                                               const std::vector<size_t>* v) {
                NeighborhoodInterface::Neighbors nb;
                nb.iterator_link.begin = [keep, v]() -> void* { return new It{keep, v, 0}; };
                nb.iterator_link.end = [keep, v]() -> void* { return new It{keep, v, v->size()}; };
                nb.iterator_link.iterator_copy = [](void* it) -> void* { return new It(*(It*)it); };
                nb.iterator_link.iterator_delete = [](void* it) { delete (It*)it; };
                nb.iterator_link.iterator_increment = [](void* it) { ((It*)it)->pos++; };
                nb.iterator_link.iterator_equals = [](void* a, void* b) {
                    return ((It*)a)->v == ((It*)b)->v && ((It*)a)->pos == ((It*)b)->pos;
                };
                nb.iterator_link.iterator_dereference = [](void* it) -> size_t* {
                    It* i = (It*)it;
                    return const_cast<size_t*>(&(*i->v)[i->pos]);
                };
                return nb;
            }
            NeighborhoodInterface::Neighbors wrap(const std::vector<size_t>* v) { return wrap_shared(nullptr, v); }
            NeighborhoodInterface::Neighbors wrap(std::shared_ptr<std::vector<size_t>> v) {
                return wrap_shared(v, v.get());
            }

            fs_ctx* ctx = nullptr;
            int64_t capacity = 0;
            fs_params made{};
            bool host_dirty = true;
            bool neighbors_valid = false;
            HostArrays<DIM> host;
            std::vector<std::vector<size_t>> lists;
        };

        // IISPHFluidSolver3D (IISPHFluidSolver3D.hpp:22-610)
        template <int SEARCH = FS_SEARCH_HASHED_3D>
        class IISPHFluidSolver3D : public FluidSolverBase<3, FS_SOLVER_IISPH_3D, SEARCH> {
          public:
            IISPHSettings3D settings;
            size_t stat_last_iteration_count = 0;
            float stat_last_average_predicted_density_error = 0.0f;

            void execute_simulation_step(Timepoint& timestep) override {
                FluidSolverBase<3, FS_SOLVER_IISPH_3D, SEARCH>::execute_simulation_step(timestep);
                stat_last_iteration_count = (size_t)this->last_stats.iterations;
                stat_last_average_predicted_density_error = this->last_stats.avg_density_error;
            }

          protected:
            void fill_settings(fs_params& p) override {
                p.max_density_error = settings.max_density_error_allowed;
                p.min_iterations = (int32_t)settings.min_number_of_iterations;
                p.max_iterations = (int32_t)settings.max_number_of_iterations;
                p.omega = settings.omega;
                p.gamma = settings.gamma;
                p.viscosity = settings.viscosity;
                p.single_layer_boundary = settings.single_layer_boundary ? 1 : 0;
                p.single_layer_gamma_1 = settings.single_layer_boundary_gamma_1;
            }
            void settings_acknowledge() override { settings.acknowledge_data_change(); }
        };

        // SESPHFluidSolver3D (SESPHFluidSolver3D.hpp:12-339)
        template <int SEARCH = FS_SEARCH_HASHED_3D>
        class SESPHFluidSolver3D : public FluidSolverBase<3, FS_SOLVER_SESPH_3D, SEARCH> {
          public:
            SESPHSettings3D settings;

          protected:
            void fill_settings(fs_params& p) override {
                p.stiffness = settings.StiffnessK;
                p.viscosity = settings.Viscosity;
                p.single_layer_boundary = settings.single_layer_boundary ? 1 : 0;
                p.single_layer_gamma_1 = settings.single_layer_boundary_gamma_1;
                p.single_layer_gamma_2 = settings.single_layer_boundary_gamma_2;
            }
            void settings_acknowledge() override { settings.acknowledge_data_change(); }
        };

        // IISPHFluidSolver, 2D (IISPHFluidSolver.hpp:21-548)
        template <int SEARCH = FS_SEARCH_QUADRATIC_2D>
        class IISPHFluidSolver : public FluidSolverBase<2, FS_SOLVER_IISPH_2D, SEARCH> {
          public:
            IISPHSettings settings;

          protected:
            void fill_settings(fs_params& p) override {
                p.max_density_error = settings.MaxDensityErrorAllowed;
                p.min_iterations = (int32_t)settings.MinNumberOfIterations;
                p.max_iterations = (int32_t)settings.MaxNumberOfIterations;
                p.omega = settings.Omega;
                p.gamma = settings.Gamma;
                p.viscosity = settings.Viscosity;
            }
            void settings_acknowledge() override { settings.acknowledge_data_change(); }
        };

        // SESPHFluidSolver, 2D (SESPHFluidSolver.hpp:12-299)
        template <int SEARCH = FS_SEARCH_QUADRATIC_2D>
        class SESPHFluidSolver : public FluidSolverBase<2, FS_SOLVER_SESPH_2D, SEARCH> {
          public:
            SESPHSettings settings;

          protected:
            void fill_settings(fs_params& p) override {
                p.stiffness = settings.StiffnessK;
                p.viscosity = settings.Viscosity;
            }
            void settings_acknowledge() override { settings.acknowledge_data_change(); }
        };

        // BoundaryPreprocessor (entities/BoundaryPreprocessor.hpp:7-28) for a drop-in solver: the
        // same entity, executed before the solver, on the device state of `solver`
        template <class Solver>
        class BoundaryPreprocessor final : public SimulationEntity {
          public:
            explicit BoundaryPreprocessor(Solver& s) : solver(s) {
                settings.execution_point = EntityExecutionPoint::BeforeSolver;
            }
            void execute_simulation_step(const Timepoint&, bool before_solver) override {
                if (!before_solver)
                    throw Error(FS_ERR_INVALID, "It makes only sense to execute the preprocessor before the solver!");
                solver.boundary_preprocess();
            }
            void initialize() override {}
            void create_compatibility_report(CompatibilityReport& report) override {
                report.begin_scope("Cuda::BoundaryPreprocessor");
                if (solver.parameters.particle_size <= 0.0f) report.add_issue("Particle size is smaller or equal to zero!");
                report.end_scope();
            }

          private:
            Solver& solver;
        };

    } // namespace Cuda
} // namespace LibFluid
