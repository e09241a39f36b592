// Serving loop of libfluidcuda.so: continuous batching of independent simulations on one GPU.
//
// Host runtime over the public C ABI (fluidcuda.h). The reference drives one grid per scene
// from FluidScene::sceneProcess (FluidScene.inl:328-420): step, check accepted(), repeat. Here a
// worker thread drives many grids at once. Each tick:
//   1. admit queued simulations in arrival order while their device bytes fit the budget and a
//      slot is free (create, configure, upload);
//   2. run one physical (sub)step of transport and forces on every active grid;
//   3. project all active grids in one batched solve (one launch per kernel for the batch);
//   4. retire finished simulations: copy their final state to host memory, free the grid.
// Substeps follow fc_step exactly (capillary subdivision, stop on a non-converged projection),
// and the batched solve computes bit for bit what a single-grid solve computes, so a
// simulation's result does not depend on what it was batched with.
#include "fc_errors.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <deque>
#include <limits>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

namespace fc
{
namespace
{

using Clock = std::chrono::steady_clock;

double ms_between(Clock::time_point a, Clock::time_point b)
{
    return std::chrono::duration<double, std::milli>(b - a).count();
}

// A submitted simulation: owned copies of its description and state, then its live grid.
struct Sim
{
    long long id = 0;
    fc_sim_desc desc{};
    std::vector<double> liquid_densities, gas_densities;
    std::vector<unsigned char> solid;
    std::vector<double> fraction, u, v, pressure;
    std::vector<std::vector<double>> liquid_mass, gas_mass;
    size_t bytes = 0;

    fc_grid* grid = nullptr;
    int substeps = 1;      // physical steps per time step
    int substep = 0;       // next substep of the current time step
    double sub_dt = 0.0;
    fc_sim_status status{};
    Clock::time_point submitted, admitted, step_started;
    bool has_state = false; // final state held in the vectors above
};

void status_check(int status, const char* what)
{
    if (status != FC_OK)
        fail(status, "%s: %s", what, fc_last_error());
}

std::vector<const double*> pointers(const std::vector<std::vector<double>>& arrays)
{
    std::vector<const double*> out;
    for (const auto& a : arrays)
        out.push_back(a.empty() ? nullptr : a.data());
    return out;
}

} // namespace

struct Server
{
    size_t budget = 0;
    int max_active = 0;
    int device = 0;

    std::mutex mutex;
    std::condition_variable wake;     // the worker: new work or stop
    std::condition_variable changed;  // waiters: a simulation finished
    bool stop = false;
    long long next_id = 1;
    std::deque<Sim*> queue;
    std::map<long long, std::unique_ptr<Sim>> sims;
    size_t in_use = 0;

    // Worker-owned. Grids are batched by what one batched solve must share: precision,
    // iteration cap and tolerance. Each group keeps its plan while its membership holds.
    struct Group
    {
        int precision;
        int max_iterations;
        double tolerance;
        fc_batch* batch = nullptr;
        std::vector<Sim*> members;
    };
    std::vector<Sim*> active;
    std::vector<Group> groups;

    // Statistics (guarded by mutex).
    fc_server_stats stats{};
    std::vector<double> latencies;
    bool busy = false;
    Clock::time_point busy_since;

    std::thread worker;

    void run();
    bool admit();
    void tick();
    bool project(std::vector<Sim*>& members, std::vector<fc_result>& results);
    void retire(Sim* s, int error);
    void release_groups();
};

void Server::retire(Sim* s, int error)
{
    // Called by the worker with the mutex released. A batch plan that holds this grid goes
    // first: batches are destroyed before their grids, and no later membership may match it.
    for (Group& g : groups)
        if (std::find(g.members.begin(), g.members.end(), s) != g.members.end())
        {
            if (g.batch)
                fc_batch_destroy(g.batch);
            g.batch = nullptr;
            g.members.clear();
        }
    if (error == FC_OK && s->grid)
    {
        const size_t cells = size_t(s->desc.width) * s->desc.height;
        s->fraction.assign(cells, 0.0);
        s->u.assign(size_t(s->desc.width + 1) * s->desc.height, 0.0);
        s->v.assign(size_t(s->desc.width) * (s->desc.height + 1), 0.0);
        s->pressure.assign(cells, 0.0);
        for (auto& m : s->liquid_mass)
            m.assign(cells, 0.0);
        for (auto& m : s->gas_mass)
            m.assign(cells, 0.0);
        std::vector<double*> lm, gm;
        for (auto& m : s->liquid_mass)
            lm.push_back(m.data());
        for (auto& m : s->gas_mass)
            gm.push_back(m.data());
        const int rc = fc_download(s->grid, s->fraction.data(), s->u.data(), s->v.data(), s->pressure.data(),
            lm.empty() ? nullptr : lm.data(), gm.empty() ? nullptr : gm.data());
        if (rc != FC_OK)
            error = rc;
        else
            s->has_state = true;
    }
    if (s->grid)
        fc_destroy(s->grid);
    s->grid = nullptr;
    std::lock_guard<std::mutex> lock(mutex);
    s->status.state = error == FC_OK ? FC_SIM_DONE : FC_SIM_FAILED;
    s->status.error = error;
    s->status.run_ms = ms_between(s->admitted, Clock::now());
    in_use -= s->bytes;
    changed.notify_all();
}

void Server::release_groups()
{
    for (Group& g : groups)
        if (g.batch)
            fc_batch_destroy(g.batch);
    groups.clear();
}

// One batched solve for a set of grids that share precision, cap and tolerance; the group's
// plan is rebuilt when its membership changed. Returns false on a failed solve.
bool Server::project(std::vector<Sim*>& members, std::vector<fc_result>& results)
{
    const fc_sim_desc& d = members.front()->desc;
    Group* group = nullptr;
    for (Group& g : groups)
        if (g.precision == d.precision && g.max_iterations == d.max_iterations && g.tolerance == d.divergence_tolerance)
            group = &g;
    if (!group)
    {
        groups.push_back({d.precision, d.max_iterations, d.divergence_tolerance, nullptr, {}});
        group = &groups.back();
    }
    if (group->members != members)
    {
        if (group->batch)
            fc_batch_destroy(group->batch);
        group->batch = nullptr;
        group->members.clear();
        std::vector<fc_grid*> grids;
        for (Sim* s : members)
            grids.push_back(s->grid);
        if (fc_batch_create(grids.data(), int(grids.size()), &group->batch) != FC_OK)
            return false;
        group->members = members;
        std::lock_guard<std::mutex> lock(mutex);
        ++stats.batch_rebuilds;
    }
    std::vector<double> dts;
    for (Sim* s : members)
        dts.push_back(s->sub_dt);
    results.assign(members.size(), fc_result{});
    if (fc_batch_project(group->batch, dts.data(), d.max_iterations, d.divergence_tolerance, 0.0, results.data()) != FC_OK)
    {
        fc_batch_destroy(group->batch);
        group->batch = nullptr;
        group->members.clear();
        return false;
    }
    return true;
}

// Moves queued simulations to the active set while they fit. Returns whether any is active.
bool Server::admit()
{
    for (;;)
    {
        Sim* s = nullptr;
        {
            std::unique_lock<std::mutex> lock(mutex);
            if (active.empty() && queue.empty())
            {
                if (busy)
                {
                    stats.busy_ms += ms_between(busy_since, Clock::now());
                    busy = false;
                }
                wake.wait(lock, [&] { return stop || !queue.empty(); });
            }
            if (stop)
                return false;
            if (queue.empty() || int(active.size()) >= max_active || in_use + queue.front()->bytes > budget)
                return !active.empty();
            s = queue.front();
            queue.pop_front();
            in_use += s->bytes;
            stats.peak_bytes = std::max(stats.peak_bytes, in_use);
            if (!busy)
            {
                busy = true;
                busy_since = Clock::now();
            }
        }
        s->admitted = Clock::now();
        const fc_sim_desc& d = s->desc;
        const int rc = guarded([&]
        {
            status_check(fc_create(d.width, d.height, d.cell_size, d.precision, &s->grid), "create");
            status_check(fc_configure_materials(s->grid, int(s->liquid_densities.size()), s->liquid_densities.data(),
                             nullptr, int(s->gas_densities.size()), s->gas_densities.data(), nullptr),
                "configure");
            status_check(fc_set_gravity(s->grid, d.gravity_y), "gravity");
            status_check(fc_set_surface_tension(s->grid, d.surface_tension), "surface tension");
            if (!s->solid.empty())
                status_check(fc_set_obstacles(s->grid, s->solid.data()), "obstacles");
            const auto lm = pointers(s->liquid_mass), gm = pointers(s->gas_mass);
            status_check(fc_upload(s->grid, s->fraction.empty() ? nullptr : s->fraction.data(),
                             s->u.empty() ? nullptr : s->u.data(), s->v.empty() ? nullptr : s->v.data(),
                             s->pressure.empty() ? nullptr : s->pressure.data(), lm.empty() ? nullptr : lm.data(),
                             gm.empty() ? nullptr : gm.data()),
                "upload");
            // fc_step's subdivision (capillary limit) of every time step.
            double limit = 0.0;
            status_check(fc_capillary_step_limit(s->grid, &limit), "capillary limit");
            const double count = d.surface_tension > 0.0 ? std::max(1.0, std::ceil(d.dt / limit)) : 1.0;
            if (count > double(std::numeric_limits<int>::max()))
                fail(FC_ERR_UNSUPPORTED, "Surface tension requires too many physical substeps for this timestep");
            s->substeps = int(count);
            s->sub_dt = d.dt / s->substeps;
        });
        // The host copies of the initial state are no longer needed.
        s->fraction.clear();
        s->u.clear();
        s->v.clear();
        s->pressure.clear();
        for (auto& m : s->liquid_mass)
            std::vector<double>().swap(m);
        for (auto& m : s->gas_mass)
            std::vector<double>().swap(m);
        {
            std::lock_guard<std::mutex> lock(mutex);
            s->status.queued_ms = ms_between(s->submitted, s->admitted);
            s->status.state = FC_SIM_RUNNING;
            s->status.device_bytes = s->bytes;
        }
        if (rc != FC_OK)
        {
            retire(s, rc);
            continue;
        }
        if (d.steps <= 0)
        {
            retire(s, FC_OK);
            continue;
        }
        active.push_back(s);
        std::lock_guard<std::mutex> lock(mutex);
        stats.peak_active = std::max(stats.peak_active, int(active.size()));
    }
}

void Server::tick()
{
    const Clock::time_point start = Clock::now();
    // Transport and forces of the next physical step of every active grid (fc_step order).
    for (size_t i = 0; i < active.size();)
    {
        Sim* s = active[i];
        if (s->substep == 0)
            s->step_started = start;
        const int rc = guarded([&]
        {
            status_check(fc_advect(s->grid, s->sub_dt), "advect");
            status_check(fc_apply_gravity(s->grid, s->sub_dt), "gravity");
            if (s->desc.surface_tension > 0.0)
                status_check(fc_apply_surface_tension(s->grid, s->sub_dt), "surface tension");
        });
        if (rc != FC_OK)
        {
            retire(s, rc);
            active.erase(active.begin() + i);
            continue;
        }
        ++i;
    }
    if (active.empty())
        return;

    // One batched projection per group of grids that can share a solve.
    std::vector<std::vector<Sim*>> parts;
    for (Sim* s : active)
    {
        auto same = [&](const std::vector<Sim*>& p)
        {
            const fc_sim_desc& a = p.front()->desc;
            return a.precision == s->desc.precision && a.max_iterations == s->desc.max_iterations &&
                   a.divergence_tolerance == s->desc.divergence_tolerance;
        };
        auto it = std::find_if(parts.begin(), parts.end(), same);
        if (it == parts.end())
            parts.push_back({s});
        else
            it->push_back(s);
    }
    // Plans of groups that no longer have members are released.
    for (size_t g = 0; g < groups.size();)
    {
        const bool used = std::any_of(parts.begin(), parts.end(), [&](const std::vector<Sim*>& p)
        {
            const fc_sim_desc& a = p.front()->desc;
            return a.precision == groups[g].precision && a.max_iterations == groups[g].max_iterations &&
                   a.divergence_tolerance == groups[g].tolerance;
        });
        if (used)
            ++g;
        else
        {
            if (groups[g].batch)
                fc_batch_destroy(groups[g].batch);
            groups.erase(groups.begin() + g);
        }
    }
    std::vector<std::pair<Sim*, fc_result>> done;
    std::vector<Sim*> failed;
    for (auto& part : parts)
    {
        std::vector<fc_result> results;
        if (project(part, results))
            for (size_t i = 0; i < part.size(); ++i)
                done.push_back({part[i], results[i]});
        else
            failed.insert(failed.end(), part.begin(), part.end());
    }
    const Clock::time_point end = Clock::now();
    const int failure = failed.empty() ? FC_OK : FC_ERR_CUDA;

    std::vector<Sim*> finished;
    {
        std::lock_guard<std::mutex> lock(mutex);
        ++stats.ticks;
        for (auto& [s, r] : done)
        {
            s->status.iterations += r.iterations;
            s->status.physical_steps += 1;
            s->status.max_divergence = r.max_divergence;
            if (!r.converged)
                s->status.converged = 0;
            ++stats.physical_steps;
            // A time step ends after its last substep, or early at a non-converged projection.
            if (++s->substep == s->substeps || !r.converged)
            {
                s->substep = 0;
                ++s->status.steps_done;
                ++stats.steps;
                stats.cell_steps += double(s->desc.width) * s->desc.height;
                latencies.push_back(ms_between(s->step_started, end));
                if (s->status.steps_done == s->desc.steps)
                    finished.push_back(s);
            }
        }
    }
    for (Sim* s : failed)
    {
        active.erase(std::find(active.begin(), active.end(), s));
        retire(s, failure);
    }
    for (Sim* s : finished)
    {
        active.erase(std::find(active.begin(), active.end(), s));
        retire(s, FC_OK);
    }
}

void Server::run()
{
    cudaSetDevice(device);
    while (admit())
        tick();
    release_groups();
    for (Sim* s : active)
        if (s->grid)
            fc_destroy(s->grid);
    active.clear();
}

} // namespace fc

struct fc_server
{
    fc::Server impl;
};

using fc::fail;
using fc::guarded;

extern "C" {

int fc_server_create(size_t device_budget_bytes, int max_active, fc_server** out)
{
    return guarded([&]
    {
        if (!out || device_budget_bytes == 0 || max_active <= 0)
            fail(FC_ERR_INVALID_ARGUMENT, "server needs a positive budget and slot count");
        *out = nullptr;
        auto server = std::make_unique<fc_server>();
        fc::Server& s = server->impl;
        s.budget = device_budget_bytes;
        s.max_active = max_active;
        if (cudaGetDevice(&s.device) != cudaSuccess)
        {
            cudaGetLastError();
            fail(FC_ERR_CUDA, "no CUDA device");
        }
        s.worker = std::thread([&s] { s.run(); });
        *out = server.release();
    });
}

int fc_server_destroy(fc_server* server)
{
    return guarded([&]
    {
        if (!server)
            return;
        {
            std::lock_guard<std::mutex> lock(server->impl.mutex);
            server->impl.stop = true;
        }
        server->impl.wake.notify_all();
        if (server->impl.worker.joinable())
            server->impl.worker.join();
        delete server;
    });
}

int fc_server_submit(fc_server* server, const fc_sim_desc* desc, long long* id)
{
    return guarded([&]
    {
        if (!server || !desc || !id)
            fail(FC_ERR_INVALID_ARGUMENT, "null argument");
        const fc_sim_desc& d = *desc;
        if (d.width <= 0 || d.height <= 0 || !(d.cell_size > 0.0) || !std::isfinite(d.cell_size))
            fail(FC_ERR_INVALID_ARGUMENT, "grid geometry must be positive and finite");
        if (d.liquid_count < 0 || d.gas_count < 0 || (d.liquid_count && !d.liquid_densities) ||
            (d.gas_count && !d.gas_densities))
            fail(FC_ERR_INVALID_ARGUMENT, "invalid material description");
        if (!(d.dt > 0.0) || !std::isfinite(d.dt) || d.steps < 0 || d.max_iterations < 0)
            fail(FC_ERR_INVALID_ARGUMENT, "invalid step description");
        if (!std::isfinite(d.surface_tension) || d.surface_tension < 0.0)
            fail(FC_ERR_INVALID_ARGUMENT, "Surface tension must be finite and nonnegative");
        size_t bytes = 0;
        const int components = d.liquid_count + d.gas_count;
        const int rc = fc_grid_device_bytes(d.width, d.height, d.precision, components, d.surface_tension > 0.0, &bytes);
        if (rc != FC_OK)
            fail(rc, "%s", fc_last_error());
        fc::Server& s = server->impl;
        if (bytes > s.budget)
            fail(FC_ERR_INVALID_ARGUMENT, "simulation needs %zu device bytes, more than the whole budget of %zu", bytes,
                s.budget);

        auto sim = std::make_unique<fc::Sim>();
        sim->desc = d;
        sim->bytes = bytes;
        const size_t cells = size_t(d.width) * d.height;
        sim->liquid_densities.assign(d.liquid_densities, d.liquid_densities + d.liquid_count);
        sim->gas_densities.assign(d.gas_densities, d.gas_densities + d.gas_count);
        if (d.solid)
            sim->solid.assign(d.solid, d.solid + cells);
        auto copy = [](std::vector<double>& to, const double* from, size_t n)
        {
            if (from)
                to.assign(from, from + n);
        };
        copy(sim->fraction, d.liquid_fraction, cells);
        copy(sim->u, d.u, size_t(d.width + 1) * d.height);
        copy(sim->v, d.v, size_t(d.width) * (d.height + 1));
        copy(sim->pressure, d.pressure, cells);
        sim->liquid_mass.resize(d.liquid_count);
        sim->gas_mass.resize(d.gas_count);
        for (int k = 0; k < d.liquid_count; ++k)
            copy(sim->liquid_mass[k], d.liquid_mass ? d.liquid_mass[k] : nullptr, cells);
        for (int k = 0; k < d.gas_count; ++k)
            copy(sim->gas_mass[k], d.gas_mass ? d.gas_mass[k] : nullptr, cells);
        // The description's pointers belong to the caller: keep only owned copies.
        sim->desc.liquid_densities = sim->desc.gas_densities = nullptr;
        sim->desc.solid = nullptr;
        sim->desc.liquid_fraction = sim->desc.u = sim->desc.v = sim->desc.pressure = nullptr;
        sim->desc.liquid_mass = sim->desc.gas_mass = nullptr;
        sim->status.state = FC_SIM_QUEUED;
        sim->status.converged = 1;
        sim->submitted = fc::Clock::now();
        {
            std::lock_guard<std::mutex> lock(s.mutex);
            if (s.stop)
                fail(FC_ERR_LIFECYCLE, "server is stopping");
            sim->id = s.next_id++;
            *id = sim->id;
            s.queue.push_back(sim.get());
            s.sims.emplace(sim->id, std::move(sim));
        }
        s.wake.notify_all();
    });
}

namespace
{
fc::Sim* find_sim(fc::Server& s, long long id)
{
    const auto it = s.sims.find(id);
    if (it == s.sims.end())
        fail(FC_ERR_INVALID_ARGUMENT, "unknown simulation %lld", id);
    return it->second.get();
}
} // namespace

int fc_server_status(fc_server* server, long long id, fc_sim_status* status)
{
    return guarded([&]
    {
        if (!server || !status)
            fail(FC_ERR_INVALID_ARGUMENT, "null argument");
        std::lock_guard<std::mutex> lock(server->impl.mutex);
        *status = find_sim(server->impl, id)->status;
    });
}

int fc_server_wait(fc_server* server, long long id, double timeout_seconds, fc_sim_status* status)
{
    return guarded([&]
    {
        if (!server)
            fail(FC_ERR_INVALID_ARGUMENT, "null server");
        fc::Server& s = server->impl;
        std::unique_lock<std::mutex> lock(s.mutex);
        fc::Sim* sim = find_sim(s, id);
        const auto finished = [&] { return sim->status.state == FC_SIM_DONE || sim->status.state == FC_SIM_FAILED; };
        const auto limit = std::chrono::duration<double>(std::max(timeout_seconds, 0.0));
        if (!s.changed.wait_for(lock, limit, finished))
            fail(FC_ERR_TIMEOUT, "simulation %lld still running after %.3f s", id, timeout_seconds);
        if (status)
            *status = sim->status;
    });
}

int fc_server_download(fc_server* server, long long id, double* liquid_fraction, double* u, double* v,
    double* pressure, double* const* liquid_mass, double* const* gas_mass)
{
    return guarded([&]
    {
        if (!server)
            fail(FC_ERR_INVALID_ARGUMENT, "null server");
        std::lock_guard<std::mutex> lock(server->impl.mutex);
        fc::Sim* sim = find_sim(server->impl, id);
        if (sim->status.state != FC_SIM_DONE || !sim->has_state)
            fail(FC_ERR_LIFECYCLE, "simulation %lld has no final state", id);
        auto out = [](double* to, const std::vector<double>& from)
        {
            if (to)
                std::copy(from.begin(), from.end(), to);
        };
        out(liquid_fraction, sim->fraction);
        out(u, sim->u);
        out(v, sim->v);
        out(pressure, sim->pressure);
        for (size_t k = 0; liquid_mass && k < sim->liquid_mass.size(); ++k)
            out(liquid_mass[k], sim->liquid_mass[k]);
        for (size_t k = 0; gas_mass && k < sim->gas_mass.size(); ++k)
            out(gas_mass[k], sim->gas_mass[k]);
    });
}

int fc_server_release(fc_server* server, long long id)
{
    return guarded([&]
    {
        if (!server)
            fail(FC_ERR_INVALID_ARGUMENT, "null server");
        std::lock_guard<std::mutex> lock(server->impl.mutex);
        fc::Sim* sim = find_sim(server->impl, id);
        if (sim->status.state != FC_SIM_DONE && sim->status.state != FC_SIM_FAILED)
            fail(FC_ERR_LIFECYCLE, "simulation %lld is still queued or running", id);
        server->impl.sims.erase(id);
    });
}

int fc_server_get_stats(fc_server* server, fc_server_stats* stats)
{
    return guarded([&]
    {
        if (!server || !stats)
            fail(FC_ERR_INVALID_ARGUMENT, "null argument");
        fc::Server& s = server->impl;
        std::lock_guard<std::mutex> lock(s.mutex);
        *stats = s.stats;
        if (s.busy)
            stats->busy_ms += fc::ms_between(s.busy_since, fc::Clock::now());
        std::vector<double> sorted = s.latencies;
        std::sort(sorted.begin(), sorted.end());
        auto percentile = [&](double q)
        {
            if (sorted.empty())
                return 0.0;
            // Nearest rank.
            const size_t rank = size_t(std::ceil(q * sorted.size()));
            return sorted[std::min(sorted.size(), std::max<size_t>(rank, 1)) - 1];
        };
        stats->step_p50_ms = percentile(0.50);
        stats->step_p99_ms = percentile(0.99);
        stats->step_max_ms = sorted.empty() ? 0.0 : sorted.back();
    });
}

int fc_server_step_latencies(fc_server* server, double* ms, size_t capacity, size_t* count)
{
    return guarded([&]
    {
        if (!server || !count || (capacity && !ms))
            fail(FC_ERR_INVALID_ARGUMENT, "null argument");
        std::lock_guard<std::mutex> lock(server->impl.mutex);
        const auto& l = server->impl.latencies;
        *count = l.size();
        std::copy(l.begin(), l.begin() + std::min(capacity, l.size()), ms);
    });
}

} // extern "C"
