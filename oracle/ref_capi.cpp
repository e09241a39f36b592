// C entry points over the reference UniformCPU engine, compiled from the reference's own
// sources (FluidSim/UniformCPU/FluidGridCPU.cpp, PressureMultigrid.cpp) by oracle/Makefile.
//
// Test infrastructure only: used to pin the C restatement (fluid_oracle.c), to generate the
// golden fixtures under tests/golden/, and as the timed CPU baseline of bench.py.
#include "UniformCPU/FluidGridCPU.h"
#include "UniformCPU/PressureMultigrid.h"
#include "UniformCPU/FluidSurfaceTensionCPU.h"
#include <bitloop/core/threads.h>
#include <chrono>
#include <cstring>
#include <exception>

using fluid::FluidGridCPU;

namespace fluid
{
// FluidField is only bound through setAccelerationField, which the oracle never calls; the
// reference implementation needs WebGPU, so these link stubs refuse to run.
const FluidField::Layout& FluidField::layout() const { std::terminate(); }
bool FluidField::isWebGPU() const { std::terminate(); }
std::span<const float> FluidField::values() const { std::terminate(); }
std::span<float> FluidField::values() { std::terminate(); }
}

// FluidGridCPU::applySurfaceTension is private. An explicit template instantiation may name a
// private member ([temp.explicit]), which hands its address to a friend function here, so the
// oracle can run the reference's own force code on a given state.
namespace
{
struct TensionMember
{
    using type = void (FluidGridCPU::*)(double);
};
template <typename Tag, typename Tag::type Member> struct Expose
{
    friend typename Tag::type member_of(Tag) { return Member; }
};
TensionMember::type member_of(TensionMember);
template struct Expose<TensionMember, &FluidGridCPU::applySurfaceTension>;
}

extern "C" {

struct ref_result
{
    int iterations;
    int converged;
    double max_divergence;
    double elapsed_ms;
};

void* ref_create(int width, int height, double cell_size)
{
    try
    {
        return new FluidGridCPU(width, height, cell_size);
    }
    catch (...)
    {
        return nullptr;
    }
}

void ref_destroy(void* handle) { delete static_cast<FluidGridCPU*>(handle); }

void ref_set_threads(int count) { bl::Thread::setMaxThreads(count); }

// One liquid and one gas component with the given densities (the reference test fixture).
void ref_configure(void* handle, double liquid_density, double gas_density)
{
    auto& grid = *static_cast<FluidGridCPU*>(handle);
    grid.substances = {};
    const auto water = grid.substances.add({"Water", {0.0f, 0.0f, 1.0f}});
    const auto air = grid.substances.add({"Air", {0.0f, 0.0f, 0.0f}});
    grid.liquid_mixture.components = {{water, liquid_density}};
    grid.gas_mixture.components = {{air, gas_density}};
}

void ref_set_gravity(void* handle, double gravity) { static_cast<FluidGridCPU*>(handle)->gravity_y = gravity; }

void ref_set_preconditioner(void* handle, int multigrid)
{
    static_cast<FluidGridCPU*>(handle)->pressure_preconditioner =
        multigrid ? FluidGridCPU::PressurePreconditioner::Multigrid : FluidGridCPU::PressurePreconditioner::Diagonal;
}

// Upload; any pointer may be null (zero field). Returns 0 or -1 on a rejected upload.
int ref_upload(void* handle, const double* fraction, const double* u, const double* v, const double* pressure,
    const double* liquid_mass, const double* gas_mass)
{
    auto& grid = *static_cast<FluidGridCPU*>(handle);
    const size_t n = size_t(grid.width) * grid.height;
    FluidGridCPU::State state;
    auto take = [](std::vector<double>& out, const double* values, size_t count)
    {
        if (values)
            out.assign(values, values + count);
    };
    take(state.liquid_fraction, fraction, n);
    take(state.u, u, size_t(grid.width + 1) * grid.height);
    take(state.v, v, size_t(grid.width) * (grid.height + 1));
    take(state.pressure, pressure, n);
    if (liquid_mass || gas_mass)
    {
        state.liquid_mass.assign(1, std::vector<double>(n, 0.0));
        state.gas_mass.assign(1, std::vector<double>(n, 0.0));
        take(state.liquid_mass[0], liquid_mass, n);
        take(state.gas_mass[0], gas_mass, n);
    }
    try
    {
        grid.upload(state);
    }
    catch (...)
    {
        return -1;
    }
    return 0;
}

void ref_download(void* handle, double* fraction, double* u, double* v, double* pressure)
{
    const auto& grid = *static_cast<FluidGridCPU*>(handle);
    auto put = [](double* out, const std::vector<double>& values)
    {
        if (out)
            std::memcpy(out, values.data(), values.size() * sizeof(double));
    };
    put(fraction, grid.liquid_fraction);
    put(u, grid.u);
    put(v, grid.v);
    put(pressure, grid.pressure);
}

static ref_result timed(auto&& call)
{
    const auto start = std::chrono::steady_clock::now();
    const fluid::FluidProjectionResult r = call();
    const auto stop = std::chrono::steady_clock::now();
    return {r.iterations, r.converged ? 1 : 0, r.max_divergence,
        std::chrono::duration<double, std::milli>(stop - start).count()};
}

ref_result ref_project(void* handle, double dt, int max_iterations, double tolerance)
{
    auto& grid = *static_cast<FluidGridCPU*>(handle);
    return timed([&] { return grid.project(dt, max_iterations, tolerance); });
}

void ref_apply_gravity(void* handle, double dt) { static_cast<FluidGridCPU*>(handle)->applyGravity(dt); }

ref_result ref_step(void* handle, double dt, int max_iterations, double tolerance)
{
    auto& grid = *static_cast<FluidGridCPU*>(handle);
    return timed([&] { return grid.step(dt, max_iterations, tolerance); });
}

void ref_set_surface_tension(void* handle, double sigma) { static_cast<FluidGridCPU*>(handle)->setSurfaceTension(sigma); }

double ref_capillary_step_limit(void* handle) { return static_cast<FluidGridCPU*>(handle)->capillaryStepLimit(); }

// FluidGridCPU::applySurfaceTension(dt) on the uploaded state.
void ref_apply_surface_tension(void* handle, double dt)
{
    auto& grid = *static_cast<FluidGridCPU*>(handle);
    (grid.*member_of(TensionMember{}))(dt);
}

// FluidSurfaceTensionCPU's three sweeps on a fraction field: completed curvature and validity.
void ref_surface_curvature(int width, int height, double cell_size, const double* fraction, double* curvature,
    unsigned char* valid)
{
    fluid::FluidSurfaceTensionCPU geometry(width, height);
    geometry.liquid = std::span<const double>(fraction, size_t(width) * height);
    geometry.cell_size = cell_size;
    for (int y = 0; y < height; ++y)
        for (int x = 0; x < width; ++x)
            geometry.buildHeight(x, y);
    for (int y = 0; y < height; ++y)
        for (int x = 0; x < width; ++x)
            geometry.buildCurvature(x, y);
    for (int y = 0; y < height; ++y)
        for (int x = 0; x < width; ++x)
            geometry.completeCurvature(x, y);
    for (size_t i = 0; i < size_t(width) * height; ++i)
    {
        curvature[i] = geometry.curvature[i].valid ? geometry.curvature[i].value : 0.0;
        valid[i] = geometry.curvature[i].valid ? 1 : 0;
    }
}

// FluidGridCPU::advect(dt) (FluidGridCPU.cpp:362-463) on the uploaded state.
void ref_advect(void* handle, double dt) { static_cast<FluidGridCPU*>(handle)->advect(dt); }

// Component masses of the single liquid and gas components.
void ref_masses(void* handle, double* liquid, double* gas)
{
    const auto& grid = *static_cast<FluidGridCPU*>(handle);
    std::memcpy(liquid, grid.liquid_mass[0].data(), grid.liquid_mass[0].size() * sizeof(double));
    std::memcpy(gas, grid.gas_mass[0].data(), grid.gas_mass[0].size() * sizeof(double));
}

void ref_set_origin(void* handle, double x, double y) { static_cast<FluidGridCPU*>(handle)->setOrigin({x, y}); }

// FluidGridCPU::sampleVelocity at interleaved (x, y) world positions.
void ref_sample_velocity(void* handle, int count, const double* positions, double* velocities)
{
    const auto& grid = *static_cast<FluidGridCPU*>(handle);
    for (int n = 0; n < count; ++n)
    {
        const bl::DVec2 v = grid.sampleVelocity({positions[2 * n], positions[2 * n + 1]});
        velocities[2 * n] = v.x;
        velocities[2 * n + 1] = v.y;
    }
}

double ref_max_divergence(void* handle) { return static_cast<FluidGridCPU*>(handle)->maxDivergence(); }

// Face weights as the engine caches them (valid after a projection).
void ref_coefficients(void* handle, double* inv_u, double* inv_v, double* inv_diagonal)
{
    const auto& grid = *static_cast<FluidGridCPU*>(handle);
    std::memcpy(inv_u, grid.inv_density_u.data(), grid.inv_density_u.size() * sizeof(double));
    std::memcpy(inv_v, grid.inv_density_v.data(), grid.inv_density_v.size() * sizeof(double));
    std::memcpy(inv_diagonal, grid.inv_pressure_diagonal.data(), grid.inv_pressure_diagonal.size() * sizeof(double));
}

// Standalone V-cycle of the reference preconditioner: rebuild from face weights, then apply.
int ref_mg_apply(int width, int height, const double* inv_u, const double* inv_v, const double* residual,
    double residual_mean, double* correction)
{
    fluid::PressureMultigrid mg(width, height);
    std::vector<double> u(inv_u, inv_u + size_t(width + 1) * height);
    std::vector<double> v(inv_v, inv_v + size_t(width) * (height + 1));
    if (!mg.rebuild(u, v))
        return -1;
    std::vector<double> r(residual, residual + size_t(width) * height), z;
    mg.apply(r, z, residual_mean);
    std::memcpy(correction, z.data(), z.size() * sizeof(double));
    return 0;
}
}
