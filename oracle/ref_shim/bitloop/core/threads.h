// Stand-in for <bitloop/core/threads.h>: an ordered batch runner over a persistent pool.
//
// forEachBatch(count, op, workers) splits [0, count) into `workers` contiguous batches,
// runs op(first, last) on each, and returns the per-batch results in batch order (the
// UniformCPU engine merges reductions in that order). Workers are persistent threads so
// that timing the reference is not dominated by thread creation.
#pragma once
#include <algorithm>
#include <condition_variable>
#include <functional>
#include <mutex>
#include <thread>
#include <type_traits>
#include <vector>

namespace bl::Thread
{
namespace detail
{
class Pool
{
public:
    static Pool& instance()
    {
        static Pool pool;
        return pool;
    }

    // Runs tasks[0..n) with task 0 on the caller; returns when all are done.
    void run(std::vector<std::function<void()>>& tasks)
    {
        if (tasks.empty())
            return;
        ensure(int(tasks.size()) - 1);
        {
            std::unique_lock lock(mutex);
            pending = tasks.data() + 1;
            pending_count = int(tasks.size()) - 1;
            next = 0;
            remaining = pending_count;
            ++generation;
        }
        wake.notify_all();
        tasks[0]();
        // The caller also drains queued tasks.
        for (;;)
        {
            std::function<void()>* task = nullptr;
            {
                std::unique_lock lock(mutex);
                if (next < pending_count)
                    task = pending + next++;
            }
            if (!task)
                break;
            (*task)();
            std::unique_lock lock(mutex);
            if (--remaining == 0)
                done.notify_all();
        }
        std::unique_lock lock(mutex);
        done.wait(lock, [&] { return remaining == 0; });
        pending = nullptr;
        pending_count = 0;
    }

    ~Pool()
    {
        {
            std::unique_lock lock(mutex);
            stopping = true;
        }
        wake.notify_all();
        for (auto& t : threads)
            t.join();
    }

private:
    void ensure(int count)
    {
        std::unique_lock lock(mutex);
        while (int(threads.size()) < count)
            threads.emplace_back([this] { loop(); });
    }

    void loop()
    {
        unsigned seen = 0;
        for (;;)
        {
            std::function<void()>* task = nullptr;
            {
                std::unique_lock lock(mutex);
                wake.wait(lock, [&] { return stopping || (generation != seen && next < pending_count); });
                if (stopping)
                    return;
                task = pending + next++;
                if (next >= pending_count)
                    seen = generation;
            }
            (*task)();
            std::unique_lock lock(mutex);
            if (--remaining == 0)
                done.notify_all();
        }
    }

    std::mutex mutex;
    std::condition_variable wake;
    std::condition_variable done;
    std::vector<std::thread> threads;
    std::function<void()>* pending = nullptr;
    int pending_count = 0;
    int next = 0;
    int remaining = 0;
    unsigned generation = 0;
    bool stopping = false;
};

inline int& maxThreads()
{
    static int value = int(std::max(1u, std::thread::hardware_concurrency()));
    return value;
}
}

inline unsigned threadCount() { return unsigned(detail::maxThreads()); }

inline void setMaxThreads(int count) { detail::maxThreads() = std::max(1, count); }

template <typename Operation> auto forEachBatch(int count, Operation&& operation, int workers = 0)
{
    using Result = std::invoke_result_t<Operation&, int, int>;
    if (workers <= 0)
        workers = int(threadCount());
    workers = std::max(1, std::min(workers, std::max(count, 1)));

    std::vector<std::function<void()>> tasks;
    tasks.reserve(workers);
    auto bounds = [&](int b) { return int((long long)count * b / workers); };

    if constexpr (std::is_void_v<Result>)
    {
        for (int b = 0; b < workers; ++b)
            tasks.emplace_back([&, b] { operation(bounds(b), bounds(b + 1)); });
        detail::Pool::instance().run(tasks);
    }
    else
    {
        std::vector<Result> results(workers);
        for (int b = 0; b < workers; ++b)
            tasks.emplace_back([&, b] { results[b] = operation(bounds(b), bounds(b + 1)); });
        detail::Pool::instance().run(tasks);
        return results;
    }
}
}
