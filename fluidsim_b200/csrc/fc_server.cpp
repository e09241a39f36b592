// Serving loop of libfluidcuda.so: continuous batching of independent simulations on one GPU.
//
// Host runtime over the public C ABI (fluidcuda.h). The reference drives one grid per scene
// from FluidScene::sceneProcess (FluidScene.inl:328-420): step, check accepted(), repeat. Here
// simulations are sorted by grid size into classes (lanes), each driven by its own worker
// thread, so a small simulation's step latency does not wait on a large grid's projection and
// the GPU runs the classes' kernels side by side on their own streams. Each tick of a lane:
//   1. admit the lane's queued simulations in arrival order while their device bytes fit the
//      server's budget and a slot is free (create, configure, upload);
//   2. enqueue one physical (sub)step of transport and forces on every active grid of the lane;
//   3. project the lane's active grids in one batched solve (one launch per kernel for them);
//   4. retire finished simulations: copy their final state to host memory, free the grid.
// Substeps follow fc_step exactly (capillary subdivision, stop on a non-converged projection),
// and the batched solve computes bit for bit what a single-grid solve computes, so a
// simulation's result does not depend on what it was batched with or which lane ran it.
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
#include <string>
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
    std::string error_text; // fc_last_error() of the call that failed it
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
    std::condition_variable wake;     // the workers: new work, freed capacity or stop
    std::condition_variable changed;  // waiters: a simulation finished
    bool stop = false;
    long long next_id = 1;
    std::map<long long, std::unique_ptr<Sim>> sims;
    size_t in_use = 0;    // device bytes of admitted simulations (all lanes)
    int running = 0;      // admitted simulations not yet retired (all lanes)

    // Grids are batched by what one batched solve must share: precision, iteration cap and
    // tolerance. Each group keeps its plan while its membership holds.
    struct Group
    {
        int precision;
        int max_iterations;
        double tolerance;
        fc_batch* batch = nullptr;
        std::vector<Sim*> members;
    };
    // A size class of simulations with its own worker. queue, stats and latencies are guarded
    // by mutex; active and groups belong to the worker.
    struct Lane
    {
        long long max_cells = 0; // grids of at most this many cells (the last lane: any size)
        int priority = 0;        // CUDA stream priority of its grids and batches
        std::deque<Sim*> queue;
        std::vector<Sim*> active;
        std::vector<Group> groups;
        fc_server_stats stats{};
        std::vector<double> latencies;
        bool busy = false;
        Clock::time_point busy_since;
        std::thread worker;
    };
    std::vector<std::unique_ptr<Lane>> lanes;

    // Whole-server statistics (guarded by mutex): peaks and the wall time with work.
    int peak_active = 0;
    size_t peak_bytes = 0;
    int busy_lanes = 0;
    double busy_ms = 0.0;
    Clock::time_point busy_since;

    Lane& lane_for(long long cells)
    {
        for (auto& l : lanes)
            if (cells <= l->max_cells)
                return *l;
        return *lanes.back();
    }
    void set_busy(Lane& lane, bool busy); // with mutex held
    void run(Lane& lane);
    bool admit(Lane& lane);
    void tick(Lane& lane);
    bool project(Lane& lane, std::vector<Sim*>& members, std::vector<fc_result>& results);
    void retire(Lane& lane, Sim* s, int error);
};

void Server::set_busy(Lane& lane, bool busy)
{
    if (lane.busy == busy)
        return;
    const Clock::time_point now = Clock::now();
    lane.busy = busy;
    if (busy)
    {
        lane.busy_since = now;
        if (busy_lanes++ == 0)
            busy_since = now;
    }
    else
    {
        lane.stats.busy_ms += ms_between(lane.busy_since, now);
        if (--busy_lanes == 0)
            busy_ms += ms_between(busy_since, now);
    }
}

void Server::retire(Lane& lane, Sim* s, int error)
{
    // Called by the lane's worker with the mutex released, right after the failing call (if
    // any): its message is still this thread's last error. A batch plan that holds this grid
    // goes first: batches are destroyed before their grids, and no later membership may match.
    if (error != FC_OK)
        s->error_text = fc_last_error();
    for (Group& g : lane.groups)
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
    --running;
    changed.notify_all();
    wake.notify_all(); // freed capacity may admit another lane's queued simulation
}

// One batched solve for a set of grids that share precision, cap and tolerance; the group's
// plan is rebuilt when its membership changed. Returns false on a failed solve.
bool Server::project(Lane& lane, std::vector<Sim*>& members, std::vector<fc_result>& results)
{
    const fc_sim_desc& d = members.front()->desc;
    Group* group = nullptr;
    for (Group& g : lane.groups)
        if (g.precision == d.precision && g.max_iterations == d.max_iterations && g.tolerance == d.divergence_tolerance)
            group = &g;
    if (!group)
    {
        lane.groups.push_back({d.precision, d.max_iterations, d.divergence_tolerance, nullptr, {}});
        group = &lane.groups.back();
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
        ++lane.stats.batch_rebuilds;
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

// Moves the lane's queued simulations to its active set while they fit. Returns whether any is
// active; waits while the lane has nothing to run.
bool Server::admit(Lane& lane)
{
    for (;;)
    {
        Sim* s = nullptr;
        {
            std::unique_lock<std::mutex> lock(mutex);
            const auto fits = [&]
            {
                return !lane.queue.empty() && running < max_active && in_use + lane.queue.front()->bytes <= budget;
            };
            if (lane.active.empty())
            {
                set_busy(lane, false);
                wake.wait(lock, [&] { return stop || fits(); });
            }
            if (stop)
                return false;
            if (!fits())
                return !lane.active.empty();
            s = lane.queue.front();
            lane.queue.pop_front();
            in_use += s->bytes;
            ++running;
            peak_bytes = std::max(peak_bytes, in_use);
            peak_active = std::max(peak_active, running);
            lane.stats.peak_bytes = std::max(lane.stats.peak_bytes, in_use);
            set_busy(lane, true);
        }
        s->admitted = Clock::now();
        const fc_sim_desc& d = s->desc;
        const int rc = guarded([&]
        {
            status_check(fc_create(d.width, d.height, d.cell_size, d.precision, &s->grid), "create");
            // Smaller classes run at higher priority: their short kernels take SMs before the
            // large grids' next ones when both wait.
            status_check(fc_set_stream_priority(s->grid, lane.priority), "stream priority");
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
            retire(lane, s, rc);
            continue;
        }
        if (d.steps <= 0)
        {
            retire(lane, s, FC_OK);
            continue;
        }
        lane.active.push_back(s);
        std::lock_guard<std::mutex> lock(mutex);
        lane.stats.peak_active = std::max(lane.stats.peak_active, int(lane.active.size()));
    }
}

void Server::tick(Lane& lane)
{
    std::vector<Sim*>& active = lane.active;
    const Clock::time_point start = Clock::now();
    // Transport and forces of the next physical step of every active grid (fc_step order).
    for (size_t i = 0; i < active.size();)
    {
        Sim* s = active[i];
        if (s->substep == 0)
            s->step_started = start;
        // Enqueued on the grid's stream without waiting: the grids' substeps run side by side
        // and the batched projection waits for each member's stream.
        const int rc = guarded([&] { status_check(fc_advance_substep(s->grid, s->sub_dt, nullptr), "substep"); });
        if (rc != FC_OK)
        {
            retire(lane, s, rc);
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
    for (size_t g = 0; g < lane.groups.size();)
    {
        const Group& group = lane.groups[g];
        const bool used = std::any_of(parts.begin(), parts.end(), [&](const std::vector<Sim*>& p)
        {
            const fc_sim_desc& a = p.front()->desc;
            return a.precision == group.precision && a.max_iterations == group.max_iterations &&
                   a.divergence_tolerance == group.tolerance;
        });
        if (used)
            ++g;
        else
        {
            if (group.batch)
                fc_batch_destroy(group.batch);
            lane.groups.erase(lane.groups.begin() + g);
        }
    }
    std::vector<std::pair<Sim*, fc_result>> done;
    std::vector<Sim*> failed;
    for (auto& part : parts)
    {
        std::vector<fc_result> results;
        if (project(lane, part, results))
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
        fc_server_stats& st = lane.stats;
        ++st.ticks;
        for (auto& [s, r] : done)
        {
            s->status.iterations += r.iterations;
            s->status.physical_steps += 1;
            s->status.max_divergence = r.max_divergence;
            if (!r.converged)
                s->status.converged = 0;
            ++st.physical_steps;
            // A time step ends after its last substep, or early at a non-converged projection.
            if (++s->substep == s->substeps || !r.converged)
            {
                s->substep = 0;
                ++s->status.steps_done;
                ++st.steps;
                st.cell_steps += double(s->desc.width) * s->desc.height;
                lane.latencies.push_back(ms_between(s->step_started, end));
                if (s->status.steps_done == s->desc.steps)
                    finished.push_back(s);
            }
        }
    }
    for (Sim* s : failed)
    {
        active.erase(std::find(active.begin(), active.end(), s));
        retire(lane, s, failure);
    }
    for (Sim* s : finished)
    {
        active.erase(std::find(active.begin(), active.end(), s));
        retire(lane, s, FC_OK);
    }
}

void Server::run(Lane& lane)
{
    cudaSetDevice(device);
    while (admit(lane))
        tick(lane);
    for (Group& g : lane.groups)
        if (g.batch)
            fc_batch_destroy(g.batch);
    lane.groups.clear();
    for (Sim* s : lane.active)
        if (s->grid)
            fc_destroy(s->grid);
    lane.active.clear();
}

// Nearest-rank percentiles and the maximum of step latencies into a stats record.
void fill_latencies(std::vector<double> sorted, fc_server_stats& stats)
{
    std::sort(sorted.begin(), sorted.end());
    auto percentile = [&](double q)
    {
        if (sorted.empty())
            return 0.0;
        const size_t rank = size_t(std::ceil(q * sorted.size()));
        return sorted[std::min(sorted.size(), std::max<size_t>(rank, 1)) - 1];
    };
    stats.step_p50_ms = percentile(0.50);
    stats.step_p99_ms = percentile(0.99);
    stats.step_max_ms = sorted.empty() ? 0.0 : sorted.back();
}

} // namespace fc

struct fc_server
{
    fc::Server impl;
};

using fc::fail;
using fc::guarded;

extern "C" {

int fc_server_create_classes(size_t device_budget_bytes, int max_active, int classes, const long long* max_cells,
    fc_server** out)
{
    return guarded([&]
    {
        if (!out || device_budget_bytes == 0 || max_active <= 0)
            fail(FC_ERR_INVALID_ARGUMENT, "server needs a positive budget and slot count");
        if (classes < 1 || classes > 16 || (classes > 1 && !max_cells))
            fail(FC_ERR_INVALID_ARGUMENT, "between 1 and 16 size classes, with classes - 1 bounds");
        for (int k = 0; k + 1 < classes; ++k)
            if (max_cells[k] <= 0 || (k > 0 && max_cells[k] <= max_cells[k - 1]))
                fail(FC_ERR_INVALID_ARGUMENT, "size class bounds must be positive and increasing");
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
        int least = 0, greatest = 0;
        if (cudaDeviceGetStreamPriorityRange(&least, &greatest) != cudaSuccess)
        {
            cudaGetLastError();
            least = greatest = 0;
        }
        for (int k = 0; k < classes; ++k)
        {
            s.lanes.push_back(std::make_unique<fc::Server::Lane>());
            s.lanes.back()->max_cells = k + 1 < classes ? max_cells[k] : std::numeric_limits<long long>::max();
            s.lanes.back()->priority = std::max(greatest, least - (classes - 1 - k));
        }
        try
        {
            for (auto& lane : s.lanes)
            {
                fc::Server::Lane* l = lane.get();
                l->worker = std::thread([&s, l] { s.run(*l); });
            }
        }
        catch (...)
        {
            // A worker that could not start: stop and join the ones that did before the server
            // they point to goes away.
            {
                std::lock_guard<std::mutex> lock(s.mutex);
                s.stop = true;
            }
            s.wake.notify_all();
            for (auto& lane : s.lanes)
                if (lane->worker.joinable())
                    lane->worker.join();
            fail(FC_ERR_OUT_OF_MEMORY, "could not start the server's workers");
        }
        *out = server.release();
    });
}

int fc_server_create(size_t device_budget_bytes, int max_active, fc_server** out)
{
    const long long bounds[4] = {128LL * 128, 256LL * 256, 512LL * 512, 1024LL * 1024};
    return fc_server_create_classes(device_budget_bytes, max_active, 5, bounds, out);
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
        for (auto& lane : server->impl.lanes)
            if (lane->worker.joinable())
                lane->worker.join();
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
            s.lane_for((long long)cells).queue.push_back(sim.get());
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

int fc_server_error(fc_server* server, long long id, char* text, size_t capacity)
{
    return guarded([&]
    {
        if (!server || (capacity && !text))
            fail(FC_ERR_INVALID_ARGUMENT, "null argument");
        std::lock_guard<std::mutex> lock(server->impl.mutex);
        const fc::Sim* sim = find_sim(server->impl, id);
        if (capacity)
        {
            const size_t n = std::min(capacity - 1, sim->error_text.size());
            std::copy(sim->error_text.begin(), sim->error_text.begin() + n, text);
            text[n] = '\0';
        }
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
        fc_server_stats total{};
        std::vector<double> latencies;
        for (auto& lane : s.lanes)
        {
            total.ticks += lane->stats.ticks;
            total.steps += lane->stats.steps;
            total.physical_steps += lane->stats.physical_steps;
            total.cell_steps += lane->stats.cell_steps;
            total.batch_rebuilds += lane->stats.batch_rebuilds;
            latencies.insert(latencies.end(), lane->latencies.begin(), lane->latencies.end());
        }
        total.busy_ms = s.busy_ms + (s.busy_lanes > 0 ? fc::ms_between(s.busy_since, fc::Clock::now()) : 0.0);
        total.peak_active = s.peak_active;
        total.peak_bytes = s.peak_bytes;
        fc::fill_latencies(std::move(latencies), total);
        *stats = total;
    });
}

int fc_server_class_count(fc_server* server, int* classes)
{
    return guarded([&]
    {
        if (!server || !classes)
            fail(FC_ERR_INVALID_ARGUMENT, "null argument");
        *classes = int(server->impl.lanes.size());
    });
}

int fc_server_get_class_stats(fc_server* server, int size_class, fc_server_stats* stats, long long* max_cells)
{
    return guarded([&]
    {
        if (!server || !stats)
            fail(FC_ERR_INVALID_ARGUMENT, "null argument");
        fc::Server& s = server->impl;
        if (size_class < 0 || size_class >= int(s.lanes.size()))
            fail(FC_ERR_INVALID_ARGUMENT, "no size class %d", size_class);
        std::lock_guard<std::mutex> lock(s.mutex);
        const fc::Server::Lane& lane = *s.lanes[size_class];
        *stats = lane.stats;
        if (lane.busy)
            stats->busy_ms += fc::ms_between(lane.busy_since, fc::Clock::now());
        fc::fill_latencies(lane.latencies, *stats);
        if (max_cells)
            *max_cells = lane.max_cells;
    });
}

int fc_server_step_latencies(fc_server* server, double* ms, size_t capacity, size_t* count)
{
    return guarded([&]
    {
        if (!server || !count || (capacity && !ms))
            fail(FC_ERR_INVALID_ARGUMENT, "null argument");
        std::lock_guard<std::mutex> lock(server->impl.mutex);
        std::vector<double> all;
        for (auto& lane : server->impl.lanes)
            all.insert(all.end(), lane->latencies.begin(), lane->latencies.end());
        *count = all.size();
        std::copy(all.begin(), all.begin() + std::min(capacity, all.size()), ms);
    });
}

} // extern "C"
