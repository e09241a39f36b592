// fluid::FluidGridCUDA: the UniformCUDA engine behind FluidSim's engine contract.
//
// Header-only adapter from fluid::FluidGridBase (FluidSim/FluidGridBase.h:20-147) to the C ABI
// in fluidcuda.h. A FluidSim build adds it as one more backend of FluidGrid::selectBackend
// (FluidSim/FluidGrid.cpp:37-90), next to the CPU and WebGPU branches. Status codes
// become the reference's exception types: std::invalid_argument, std::logic_error,
// std::runtime_error; a non-converged projection is a result, not an exception.
//
// Lifecycle as the reference's engines have it (UniformWebGPU/FluidGridWebGPU.cpp:145-165):
// destroy() releases the device grid; the configuration (materials, gravity, origin, transport)
// stays on the host, and the next upload() builds a new device grid from it. Any other use of
// device state between destroy() and upload() throws std::logic_error.
#pragma once

#include "FluidGridBase.h"
#include "fluidcuda.h"

#include <cmath>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace fluid
{

class FluidGridCUDA final : public FluidGridBase
{
public:
    // Identifies the backend kind for selection code (0 = unknown, 1 = UniformCUDA).
    static constexpr int kind() { return 1; }

    FluidGridCUDA(int width, int height, double cell_size, int precision = FC_PRECISION_FP32)
        : width(width), height(height), cell_size(cell_size), precision(precision)
    {
        check(fc_create(width, height, cell_size, precision, &grid));
    }

    ~FluidGridCUDA() override
    {
        if (grid)
            fc_destroy(grid);
    }

    FluidGridCUDA(const FluidGridCUDA&) = delete;
    FluidGridCUDA& operator=(const FluidGridCUDA&) = delete;

    int getWidth() const override { return width; }

    int getHeight() const override { return height; }

    double getCellSize() const override { return cell_size; }

    bl::DVec2 getOrigin() const override { return origin; }

    void setOrigin(bl::DVec2 position) override
    {
        origin = position;
        if (grid)
            check(fc_set_origin(grid, position.x, position.y));
    }

    bool requiresRenderThread() const override { return false; }

    void configureMaterials(SubstanceCatalogue catalogue, FluidMixture liquid, FluidMixture gas) override
    {
        std::vector<double> ld, lv, gd, gv;
        for (const auto& c : liquid.components)
            ld.push_back(c.density), lv.push_back(c.dynamic_viscosity);
        for (const auto& c : gas.components)
            gd.push_back(c.density), gv.push_back(c.dynamic_viscosity);
        if (grid)
            check(fc_configure_materials(grid, int(ld.size()), ld.data(), lv.data(), int(gd.size()), gd.data(), gv.data()));
        substances = std::move(catalogue);
        liquid_mixture = std::move(liquid);
        gas_mixture = std::move(gas);
    }

    // setComponentViscosity (FluidGridBase.h:47-52): a coefficient edit; membership stays fixed.
    void setComponentViscosity(Phase phase, size_t component, double coefficient) override
    {
        if (grid)
            check(fc_set_component_viscosity(grid, phase == Phase::Liquid ? 0 : 1, int(component), coefficient));
        else if (!std::isfinite(coefficient) || coefficient < 0.0)
            throw std::invalid_argument("FluidGridCUDA viscosity must be finite and non-negative");
        auto& mixture = phase == Phase::Liquid ? liquid_mixture : gas_mixture;
        mixture.components.at(component).dynamic_viscosity = coefficient;
    }

    const SubstanceCatalogue& getSubstances() const override { return substances; }

    const FluidMixture& getLiquidMixture() const override { return liquid_mixture; }

    const FluidMixture& getGasMixture() const override { return gas_mixture; }

    double getGravityY() const override { return gravity; }

    void setGravityY(double acceleration) override
    {
        if (grid)
            check(fc_set_gravity(grid, acceleration));
        else if (!std::isfinite(acceleration))
            throw std::invalid_argument("FluidGridCUDA gravity must be finite");
        gravity = acceleration;
    }

    // The material transport of step(): FC_TRANSPORT_SEMI_LAGRANGIAN (the default) or
    // FC_TRANSPORT_PLIC, the reference UniformCPU engine's conservative transport.
    void setTransport(int scheme)
    {
        if (grid)
            check(fc_set_transport(grid, scheme));
        else if (scheme != FC_TRANSPORT_SEMI_LAGRANGIAN && scheme != FC_TRANSPORT_PLIC)
            throw std::invalid_argument("FluidGridCUDA transport scheme is unknown");
        transport = scheme;
    }

    void upload(const State& state) override
    {
        const size_t cells = size_t(width) * height;
        auto sized = [](const std::vector<double>& values, size_t count)
        {
            if (!values.empty() && values.size() != count)
                throw std::invalid_argument("FluidGridCUDA upload dimensions do not match the grid");
            return values.empty() ? nullptr : values.data();
        };
        const double* f = sized(state.liquid_fraction, cells);
        const double* u = sized(state.u, size_t(width + 1) * height);
        const double* v = sized(state.v, size_t(width) * (height + 1));
        const double* p = sized(state.pressure, cells);
        auto components = [&](const std::vector<std::vector<double>>& masses, size_t expected)
        {
            std::vector<const double*> ptrs;
            if (masses.empty())
                return ptrs;
            if (masses.size() != expected)
                throw std::invalid_argument("FluidGridCUDA upload component count does not match the mixture");
            for (const auto& m : masses)
                ptrs.push_back(sized(m, cells));
            return ptrs;
        };
        const auto lm = components(state.liquid_mass, liquid_mixture.components.size());
        const auto gm = components(state.gas_mass, gas_mixture.components.size());
        check(fc_upload(rebuilt(), f, u, v, p, lm.empty() ? nullptr : lm.data(), gm.empty() ? nullptr : gm.data()));
    }

    State download() const override
    {
        const size_t cells = size_t(width) * height;
        State s;
        s.liquid_fraction.resize(cells);
        s.u.resize(size_t(width + 1) * height);
        s.v.resize(size_t(width) * (height + 1));
        s.pressure.resize(cells);
        s.liquid_mass.assign(liquid_mixture.components.size(), std::vector<double>(cells));
        s.gas_mass.assign(gas_mixture.components.size(), std::vector<double>(cells));
        std::vector<double*> lm, gm;
        for (auto& m : s.liquid_mass)
            lm.push_back(m.data());
        for (auto& m : s.gas_mass)
            gm.push_back(m.data());
        check(fc_download(live(), s.liquid_fraction.data(), s.u.data(), s.v.data(), s.pressure.data(),
            lm.empty() ? nullptr : lm.data(), gm.empty() ? nullptr : gm.data()));
        return s;
    }

    void destroy() override
    {
        if (grid)
            fc_destroy(grid);
        grid = nullptr;
    }

    ProjectionResult step(double dt, int max_iterations = 200, double divergence_tolerance = 1e-6,
        StepTimings* timings = nullptr) override
    {
        // Stage timings make every stage wait for its kernels; without them the substeps are
        // enqueued and only the projection waits.
        fc_result r{};
        fc_timings t{};
        check(fc_step(live(), dt, max_iterations, divergence_tolerance, &r, timings ? &t : nullptr));
        if (timings)
        {
            *timings = {};
            timings->transport_ms = t.transport_ms;
            timings->viscosity_ms = t.viscosity_ms;
            timings->forces_ms = t.forces_ms;
            timings->pressure_ms = t.pressure_ms;
        }
        return convert(r);
    }

    // FluidGridCPU::project (UniformCPU/FluidGridCPU.h:125): one projection without forces.
    ProjectionResult project(double dt, int max_iterations = 200, double divergence_tolerance = 1e-6)
    {
        fc_result r{};
        check(fc_project(live(), dt, max_iterations, divergence_tolerance, &r));
        return convert(r);
    }

    double maxDivergence() const override
    {
        double value = 0.0;
        check(fc_max_divergence(live(), &value));
        return value;
    }

    // Display colour of each cell from its component volumes (FluidGridCPU.cpp:1826-1860).
    void writeColorPixels(std::vector<float>& pixels, bool liquid_fraction_alpha = false) const override
    {
        const State s = download();
        const size_t cells = size_t(width) * height;
        const double volume = cell_size * cell_size;
        pixels.assign(cells * 4, 0.0f);
        for (size_t i = 0; i < cells; ++i)
        {
            float* pixel = pixels.data() + i * 4;
            pixel[3] = liquid_fraction_alpha ? float(s.liquid_fraction[i]) : 1.0f;
            auto add = [&](const FluidMixture& mixture, const std::vector<std::vector<double>>& masses)
            {
                for (size_t k = 0; k < mixture.components.size(); ++k)
                {
                    const auto& component = mixture.components[k];
                    const auto& color = substances[component.substance].color;
                    const double fraction = masses[k][i] / (component.density * volume);
                    for (int c = 0; c < 3; ++c)
                        pixel[c] += float(fraction * color[c]);
                }
            };
            add(liquid_mixture, s.liquid_mass);
            add(gas_mixture, s.gas_mass);
        }
    }

    // saveCheckpoint (FluidGridBase.h:123): the engine's "cuda-uniform" metadata and payload,
    // plus the host-side substance catalogue and mixture membership under "host".
    bool saveCheckpoint(FluidCheckpoint& checkpoint) const override
    {
        size_t meta_bytes = 0, payload_bytes = 0;
        check(fc_save_checkpoint(live(), nullptr, 0, &meta_bytes, nullptr, 0, &payload_bytes));
        std::string meta(meta_bytes, '\0');
        checkpoint.data.resize(payload_bytes);
        check(fc_save_checkpoint(grid, meta.data(), meta_bytes, &meta_bytes, checkpoint.data.data(), payload_bytes,
            &payload_bytes));
        auto metadata = bl::JSON::json::parse(meta.c_str());
        auto& host = metadata["host"];
        host["substances"] = bl::JSON::json::array();
        for (SubstanceId id = 0; id < substances.size(); ++id)
            host["substances"].push_back({{"name", substances[id].name}, {"color", substances[id].color}});
        for (const char* phase : {"liquid", "gas"})
        {
            auto& ids = host[std::string(phase) + "_substances"] = bl::JSON::json::array();
            for (const auto& c : (phase[0] == 'l' ? liquid_mixture : gas_mixture).components)
                ids.push_back(c.substance);
        }
        checkpoint.metadata = std::move(metadata);
        return true;
    }

    // loadCheckpoint (FluidGridBase.h:125): validated by the engine before anything changes.
    bool loadCheckpoint(const FluidCheckpoint& checkpoint) override
    {
        const auto& metadata = checkpoint.metadata;
        check(fc_load_checkpoint(rebuilt(), metadata.dump().c_str(), checkpoint.data.data(), checkpoint.data.size()));
        if (metadata.contains("gravity_y"))
            gravity = metadata["gravity_y"].template get<double>();
        if (metadata.contains("host"))
        {
            const auto& host = metadata["host"];
            SubstanceCatalogue catalogue;
            for (const auto& entry : host["substances"])
                catalogue.add({entry["name"].template get<std::string>(), entry["color"].template get<std::array<float, 3>>()});
            auto mixture = [&](const char* key, const char* phase)
            {
                FluidMixture out;
                const auto& ids = host[std::string(phase) + "_substances"];
                size_t k = 0;
                for (const auto& c : metadata[key])
                {
                    out.components.push_back({ids.at(k++).template get<SubstanceId>(), c["density"].template get<double>(),
                        c["dynamic_viscosity"].template get<double>()});
                }
                return out;
            };
            liquid_mixture = mixture("liquid_mixture", "liquid");
            gas_mixture = mixture("gas_mixture", "gas");
            substances = std::move(catalogue);
        }
        return true;
    }

    fc_grid* native() const { return grid; }

protected:
    // Material replacements (FluidGridCPU.cpp:256-290): a host round trip; edits are rare.
    void commitEdits(detail::CellEditBatch& batch) override
    {
        if (batch.velocity)
            throw std::invalid_argument("Material edit velocity requires uniform WebGPU");
        batch.prepare(width, height, cell_size * cell_size, liquid_mixture, gas_mixture);
        State s = download();
        const size_t liquids = s.liquid_mass.size();
        for (const auto& cell : batch.cells)
        {
            const size_t i = size_t(cell.y) * width + cell.x;
            const bool liquid = cell.component < liquids;
            s.liquid_fraction[i] = liquid ? 1.0 : 0.0;
            for (auto& m : s.liquid_mass)
                m[i] = 0.0;
            for (auto& m : s.gas_mass)
                m[i] = 0.0;
            if (liquid)
                s.liquid_mass[cell.component][i] = cell.mass;
            else
                s.gas_mass[cell.component - liquids][i] = cell.mass;
        }
        upload(s);
    }

private:
    static void check(int status)
    {
        if (status == FC_OK)
            return;
        const std::string message = fc_last_error();
        if (status == FC_ERR_INVALID_ARGUMENT)
            throw std::invalid_argument(message);
        if (status == FC_ERR_LIFECYCLE)
            throw std::logic_error(message);
        throw std::runtime_error(message);
    }

    fc_grid* live() const
    {
        if (!grid)
            throw std::logic_error("FluidGridCUDA: upload a state after destroy() before using the grid");
        return grid;
    }

    // The device grid for an upload: after destroy(), a new one with the host-side
    // configuration applied (the reference's re-initialisation by upload).
    fc_grid* rebuilt()
    {
        if (grid)
            return grid;
        fc_grid* fresh = nullptr;
        check(fc_create(width, height, cell_size, precision, &fresh));
        try
        {
            std::vector<double> ld, lv, gd, gv;
            for (const auto& c : liquid_mixture.components)
                ld.push_back(c.density), lv.push_back(c.dynamic_viscosity);
            for (const auto& c : gas_mixture.components)
                gd.push_back(c.density), gv.push_back(c.dynamic_viscosity);
            if (!ld.empty() || !gd.empty())
                check(fc_configure_materials(fresh, int(ld.size()), ld.data(), lv.data(), int(gd.size()), gd.data(),
                    gv.data()));
            check(fc_set_gravity(fresh, gravity));
            check(fc_set_origin(fresh, origin.x, origin.y));
            check(fc_set_transport(fresh, transport));
        }
        catch (...)
        {
            fc_destroy(fresh);
            throw;
        }
        grid = fresh;
        return grid;
    }

    static ProjectionResult convert(const fc_result& r)
    {
        ProjectionResult out;
        out.iterations = r.iterations;
        out.max_divergence = r.max_divergence;
        out.converged = r.converged != 0;
        out.physical_steps = r.physical_steps;
        out.transport_steps = r.transport_steps;
        out.relaxed = r.relaxed != 0;
        out.max_volume_error = r.max_volume_error;
        out.rms_volume_error = r.rms_volume_error;
        out.viscosity_iterations = r.viscosity_iterations;
        out.precision_limited = r.precision_limited != 0;
        return out;
    }

    fc_grid* grid = nullptr;
    int width;
    int height;
    double cell_size;
    int precision;
    double gravity = 0.0;
    int transport = FC_TRANSPORT_SEMI_LAGRANGIAN;
    bl::DVec2 origin{};
    SubstanceCatalogue substances;
    FluidMixture liquid_mixture;
    FluidMixture gas_mixture;
};

}
