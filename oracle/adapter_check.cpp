// Run-time check of the C++ drop-in, fluid::FluidGridCUDA (include/FluidGridCUDA.h), against
// the reference's own UniformCPU engine, both driven through fluid::FluidGridBase&.
//
// Test infrastructure only: built by oracle/Makefile (target `adapter`) from the reference's
// headers, linked with the reference engine (oracle/_ref/libfluidref.so) and the CUDA library
// (fluidsim_b200/libfluidcuda.so); run by tests/test_adapter_gpu.py on a GPU.
//
// The scenario restates the reference's facade test (tests/FluidGridAPITests.cpp:36-80, the
// sloped two-liquid/two-gas set-up, and :186-229, 64 steps with a gravity change at step 32, a
// zero-iteration step, destroy and re-upload), then adds what the CUDA engine must show on its
// own: the checkpoint round trip continues bit for bit, and status codes arrive as the
// reference's exception types. The CUDA grid runs the reference's PLIC transport so that the
// two engines take the same steps.
//
// Usage: adapter_check [fp64|fp32]. Prints one line per check and exits non-zero on a failure.
#include "FluidGridCUDA.h"
#include "UniformCPU/FluidGridCPU.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>

using namespace fluid;

namespace
{
int failures = 0;

void expect(bool ok, const std::string& what)
{
    std::printf("%s %s\n", ok ? "ok  " : "FAIL", what.c_str());
    if (!ok)
        ++failures;
}

double max_abs(const std::vector<double>& a)
{
    double m = 0.0;
    for (double x : a)
        m = std::max(m, std::abs(x));
    return m;
}

double max_diff(const std::vector<double>& a, const std::vector<double>& b)
{
    if (a.size() != b.size())
        return INFINITY;
    double m = 0.0;
    for (size_t i = 0; i < a.size(); ++i)
        m = std::max(m, std::abs(a[i] - b[i]));
    return m;
}

// Largest difference of two states relative to each field's scale: velocities to the larger
// velocity scale (at least 1), fraction and component masses to their own largest value.
double state_error(const FluidGridBase::State& a, const FluidGridBase::State& b)
{
    const double vs = std::max({1.0, max_abs(b.u), max_abs(b.v)});
    double e = std::max(max_diff(a.u, b.u), max_diff(a.v, b.v)) / vs;
    e = std::max(e, max_diff(a.liquid_fraction, b.liquid_fraction));
    for (size_t k = 0; k < b.liquid_mass.size(); ++k)
        e = std::max(e, max_diff(a.liquid_mass[k], b.liquid_mass[k]) / std::max(1e-300, max_abs(b.liquid_mass[k])));
    for (size_t k = 0; k < b.gas_mass.size(); ++k)
        e = std::max(e, max_diff(a.gas_mass[k], b.gas_mass[k]) / std::max(1e-300, max_abs(b.gas_mass[k])));
    return e;
}

bool identical(const FluidGridBase::State& a, const FluidGridBase::State& b)
{
    return a.liquid_fraction == b.liquid_fraction && a.u == b.u && a.v == b.v && a.pressure == b.pressure &&
           a.liquid_mass == b.liquid_mass && a.gas_mass == b.gas_mass;
}

// Two liquids (densities 100 and 300) and two gases (0.1 each) over a sloped interface: the
// reference facade test's set-up. Returns the uploaded state.
FluidGridBase::State configure(FluidGridBase& grid)
{
    SubstanceCatalogue substances;
    const SubstanceId water = substances.add({"Water", {0.1f, 0.35f, 1.0f}});
    const SubstanceId red = substances.add({"Red", {0.95f, 0.25f, 0.15f}});
    const SubstanceId air = substances.add({"Air", {0.015f, 0.025f, 0.06f}});
    const SubstanceId cloud = substances.add({"Cloud", {0.0f, 1.0f, 1.0f}});
    FluidMixture liquid, gas;
    liquid.components = {{water, 100.0}, {red, 300.0}};
    gas.components = {{air, 0.1}, {cloud, 0.1}};
    grid.configureMaterials(std::move(substances), liquid, gas);
    grid.setOrigin({-7.0, 11.0});
    grid.setGravityY(80.0);

    const int w = grid.getWidth(), h = grid.getHeight();
    const double area = grid.getCellSize() * grid.getCellSize();
    FluidGridBase::State s;
    s.liquid_fraction.assign(size_t(w) * h, 0.0);
    s.liquid_mass.assign(2, std::vector<double>(size_t(w) * h));
    s.gas_mass.assign(2, std::vector<double>(size_t(w) * h));
    for (int y = 0; y < h; ++y)
        for (int x = 0; x < w; ++x)
        {
            const size_t i = size_t(y) * w + x;
            const double f = std::clamp(y + 1.0 - (x + 0.5 * h), 0.0, 1.0);
            const double red_share = x < w / 4 ? 1.0 : 0.0;
            const double cloud_share = 0.15 + 0.1 * std::sin(0.2 * x);
            s.liquid_fraction[i] = f;
            s.liquid_mass[0][i] = 100.0 * f * area * (1.0 - red_share);
            s.liquid_mass[1][i] = 300.0 * f * area * red_share;
            s.gas_mass[0][i] = 0.1 * (1.0 - f) * area * (1.0 - cloud_share);
            s.gas_mass[1][i] = 0.1 * (1.0 - f) * area * cloud_share;
        }
    grid.upload(s);
    return s;
}

template <typename E, typename F> bool throws(F&& body)
{
    try
    {
        body();
    }
    catch (const E&)
    {
        return true;
    }
    catch (...)
    {
        return false;
    }
    return false;
}
}

int run(int argc, char** argv)
{
    const bool fp64 = argc < 2 || std::strcmp(argv[1], "fp32") != 0;
    const int precision = fp64 ? FC_PRECISION_FP64 : FC_PRECISION_FP32;
    // FP64: the reference's arithmetic with another reduction order, 1e-8 of each field's
    // scale over 64 steps. FP32 storage of the working arrays and face velocities: 1e-4.
    const double bar = fp64 ? 1e-8 : 1e-4;
    std::printf("adapter check, %s, bar %.0e\n", fp64 ? "fp64" : "fp32", bar);

    FluidGridCPU cpu(33, 25, 2.5);
    FluidGridCUDA cuda(33, 25, 2.5, precision);
    cuda.setTransport(FC_TRANSPORT_PLIC);
    FluidGridBase& direct = cpu;
    FluidGridBase& api = cuda;
    const FluidGridBase::State initial = configure(direct);
    configure(api);

    expect(api.getWidth() == 33 && api.getHeight() == 25 && api.getCellSize() == 2.5, "geometry");
    expect(api.getOrigin().x == -7.0 && api.getOrigin().y == 11.0 && api.getGravityY() == 80.0, "origin and gravity");
    expect(api.getLiquidMixture().components.size() == 2 && api.getGasMixture().components.size() == 2,
        "mixtures kept on the host");
    const double upload_error = state_error(api.download(), direct.download());
    expect(fp64 ? identical(api.download(), direct.download()) : upload_error <= 1e-7,
        "upload then download equals the reference's" + std::string(fp64 ? " bit for bit" : " to float rounding"));

    {
        const auto a = direct.step(0.0), b = api.step(0.0);
        expect(a.iterations == b.iterations && a.converged == b.converged && !b.converged,
            "a zero time step reports no convergence, as the reference does");
    }

    double worst = 0.0;
    int worst_iterations = 0;
    bool all_converged = true;
    for (int step = 0; step < 64; ++step)
    {
        if (step == 32)
        {
            direct.setGravityY(110.0);
            api.setGravityY(110.0);
        }
        const auto expected = direct.step(0.004, 2000, 1e-8);
        const auto actual = api.step(0.004, 2000, 1e-8);
        all_converged &= expected.converged && (fp64 ? actual.converged : actual.accepted());
        worst_iterations = std::max(worst_iterations, std::abs(expected.iterations - actual.iterations));
        worst = std::max(worst, state_error(api.download(), direct.download()));
    }
    std::printf("     64 steps: worst state error %.3e, worst iteration difference %d\n", worst, worst_iterations);
    expect(all_converged, "every step converged (FP32: accepted) on both engines");
    expect(worst <= bar, "64 steps agree with the reference within the bar");
    if (fp64)
        expect(worst_iterations <= 2, "iterations within two of the reference's on every step");
    expect(api.getGravityY() == 110.0, "gravity change applied");
    expect(fp64 ? api.maxDivergence() <= 1e-8 : std::isfinite(api.maxDivergence()),
        "maxDivergence after the steps");

    {
        const auto a = direct.step(0.01, 0, 1e-12), b = api.step(0.01, 0, 1e-12);
        expect(!a.converged && !b.converged, "a zero-iteration step does not claim convergence");
    }

    // Destroy and re-upload: the reference re-initialises from the uploaded state.
    direct.destroy();
    api.destroy();
    expect(throws<std::logic_error>([&] { api.download(); }), "use between destroy() and upload() is a logic_error");
    direct.upload(initial);
    api.upload(initial);
    expect(fp64 ? identical(api.download(), direct.download()) : state_error(api.download(), direct.download()) <= 1e-7,
        "re-upload after destroy() gives the reference's state");
    expect(api.getGravityY() == 110.0 && api.getOrigin().x == -7.0, "configuration survives destroy()");

    // Checkpoint round trip: a new grid loaded from the checkpoint continues bit for bit.
    api.step(0.004, 2000, 1e-8);
    FluidCheckpoint checkpoint;
    expect(api.saveCheckpoint(checkpoint), "saveCheckpoint supported");
    FluidGridCUDA restored(33, 25, 2.5, precision);
    FluidGridBase& copy = restored;
    expect(copy.loadCheckpoint(checkpoint), "loadCheckpoint supported");
    expect(identical(copy.download(), api.download()), "loaded state equals the saved one bit for bit");
    expect(copy.getGravityY() == api.getGravityY() && copy.getLiquidMixture().components.size() == 2,
        "loaded configuration equals the saved one");
    restored.setTransport(FC_TRANSPORT_PLIC);
    for (int k = 0; k < 3; ++k)
    {
        const auto a = api.step(0.004, 2000, 1e-8), b = copy.step(0.004, 2000, 1e-8);
        expect(a.iterations == b.iterations && a.max_divergence == b.max_divergence, "continued step " + std::to_string(k));
    }
    expect(identical(copy.download(), api.download()), "three continued steps agree bit for bit");

    // Status codes arrive as the reference's exception types, before any state changes.
    const auto before = api.download();
    FluidGridBase::State bad = initial;
    bad.u.assign(size_t(33 + 1) * 25 - 1, 0.0); // one face short (an empty u means all zero)
    expect(throws<std::invalid_argument>([&] { direct.upload(bad); }) &&
               throws<std::invalid_argument>([&] { api.upload(bad); }),
        "a mis-sized upload is invalid_argument on both engines");
    expect(identical(api.download(), before), "a rejected upload changes nothing");
    FluidCheckpoint broken = checkpoint;
    broken.data.resize(broken.data.size() - 8);
    expect(throws<std::invalid_argument>([&] { api.loadCheckpoint(broken); }), "a truncated checkpoint is rejected");
    expect(identical(api.download(), before), "a rejected checkpoint changes nothing");
    FluidGridCUDA fresh(8, 8, 1.0, precision);
    FluidGridBase& unused = fresh;
    expect(throws<std::logic_error>([&] { unused.step(0.01); }), "stepping before upload is a logic_error");
    expect(throws<std::invalid_argument>([&] { FluidGridCUDA(0, 8, 1.0, precision); }),
        "an empty grid is invalid_argument");
    FluidMixture negative;
    negative.components = {{0, -1.0}};
    expect(throws<std::invalid_argument>([&] { unused.configureMaterials({}, negative, FluidMixture{}); }),
        "a negative density is invalid_argument");

    std::printf("%s: %d failure(s)\n", failures ? "FAILED" : "PASSED", failures);
    return failures ? 1 : 0;
}

int main(int argc, char** argv)
{
    // Unbuffered: every check's line is out before a later failure ends the process.
    std::setvbuf(stdout, nullptr, _IONBF, 0);
    try
    {
        return run(argc, argv);
    }
    catch (const std::exception& e)
    {
        std::printf("FAIL uncaught exception: %s\n", e.what());
        return 2;
    }
}
