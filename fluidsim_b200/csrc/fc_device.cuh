// Device-side layout, descriptors and reduction helpers of the UniformCUDA backend.
//
// Layout in HBM. Every cell-centred array of a grid level (face weights, multigrid rhs and
// solution, and on the fine level the PCG vectors r, z, d, q, p) is stored padded: cell (x, y)
// lives at index (y + 1) * S + (x + 2), with S = round_up(w + 3, 8) elements per row and
// h + 2 rows. Row 0, row h + 1 and the columns left of x = 0 and right of x = w - 1 stay zero,
// so stencils need no bounds tests and a closed wall reads as a zero weight.
//
// A cell stores the weight of its right face ("right", the u face at x + 1) and of its lower
// face ("down", the v face at y + 1). The left weight of a cell is right[i - 1] and its upper
// weight down[i - S]. On the fine level these are the reference's inv_density_u/v
// (FluidGridCPU.cpp:1154-1205); coarse levels hold the multigrid conductances
// (PressureMultigrid.cpp:142-202).
#pragma once

#include <cuda_fp16.h>

#include <cstdint>
#include <cuda_runtime.h>

namespace fc
{

constexpr int kMaxLevels = 16;
constexpr int kPadX = 2;   // column of x = 0 inside a padded row
// Tiles of the fine-level vector kernels: 64 x 64 cells, 256 threads. Thread (lane, warp) covers
// columns lane and lane + 32 of rows warp + 8m (kVecCells cells), or, in the strip kernels,
// columns 2 lane and 2 lane + 1 of rows 8 warp .. 8 warp + 7.
constexpr int kVecTileX = 64;
constexpr int kVecTileY = 64;
constexpr int kVecThreads = 256;
constexpr int kVecCells = 16;

__host__ __device__ inline int padded_stride(int w) { return ((w + 3) + 7) / 8 * 8; }
__host__ __device__ inline long long padded_index(int S, int x, int y) { return (long long)(y + 1) * S + x + kPadX; }

// Solver status codes shared with the C ABI (fc_result.status).
enum SolveStatus : int
{
    kRunning = 0,
    kConverged = 1,        // stop rule met on the true residual
    kIterationLimit = 2,   // max_iterations reached
    kStalled = 3,          // r.z or d.Ad lost positivity / finiteness (reference loop exit)
    kNoWork = 4,           // right-hand side already below tolerance
    kBreakdown = 5,        // coarsest factorisation failed
};

// Per-grid PCG scalars, resident on the device for the whole solve.
struct SolveState
{
    double rz;          // r . z of the current direction
    double dq;          // d . A d
    double beta;
    double mean_b;      // mean of the raw right-hand side
    double mean_r;      // mean of the current residual
    double mean_z;
    double mean_p;
    double sum_r, max_r, sumsq_r;
    double bmax, bsumsq;
    double tol_max;     // max-norm stop rule (pressure units); +inf when unused
    double tol_sumsq;   // L2 stop rule, squared; +inf when unused
    double inv_cells;   // 1 / cell count
    double div_max;     // post-projection max |div u|
    double div_excess;  // max(0, |div u| - local float rounding allowance)
    double div_sumsq;   // sum of div^2
    double res_max, res_sumsq;
    double refresh_max; // FP32: recurrence max-norm that triggers a refresh from the true residual (0: none)
    double dt;          // time step of the projection in flight
    double alpha_pending; // step length whose p += alpha d is still to be applied (p_pending)
    int iterations;
    int restarts;       // true-residual checks that failed and restarted the directions
    int refreshes;      // FP32 early restarts from the true residual (refresh_threshold)
    int max_iterations;
    int done;
    int status;
    int verify;
    int restart;
    int mg_valid;       // multigrid hierarchy and coarsest inverse are usable
    int use_mg;         // multigrid (1) or diagonal (0) preconditioner
    int nonfinite;
    int p_pending;      // the first iteration of a pair updated r but left p += alpha d to the second
};

// Linear interpolation from a fine axis position to the two nearest coarse centres
// (PressureMultigrid.cpp:64-102). weight belongs to `second`.
struct Interp
{
    int first;
    int second;
    double weight;
};

// Transpose of Interp: the fine cells that a coarse cell gathers from.
struct Gather
{
    int count;
    int index[4];
    double weight[4];
};

// Unknowns of the coarsest direct solve: every cell with an open face except the first one,
// which is pinned (the reference pins cell 0, PressureMultigrid.cpp:306-320; with no obstacle
// the two are the same). Written by the rebuild, read by every V-cycle.
struct CoarseInfo
{
    int n;       // unknowns
    int pinned;  // pinned cell, -1 when no cell is open
    int open;    // open cells (n + 1, or 0)
    int map[64]; // cell -> unknown index, -1 for the pinned and the closed cells
    int dirichlet; // Dirichlet air: unknowns only, nothing pinned, no mean and no gauge
};

struct LevelDesc
{
    int w, h, S;
    void* right;
    void* down;
    // Mixed precision: FP16 copies of right/down read by the smoothing kernels, stored divided
    // by wscale (a per-level scale that keeps every weight in FP16's normal range).
    const void* right_h;
    const void* down_h;
    float wscale;
    // Inverse diagonal of the levels the strip kernels smooth, in the working precision: 1 / the
    // sum of a cell's four face weights (as the kernels decode them), 0 for a cell with no open
    // face and in the padding. Written by the rebuild.
    void* inv;
    void* rhs;           // levels >= 1 (level 0 reads the PCG residual minus its mean)
    void* pre;           // pre-smoothed solution, read by the post-smoothing of the same level
    void* sol;           // final solution of the level (level 0: the PCG vector z)
    const double* cx;    // cell centres, in fine cells
    const double* cy;
    const Interp* px;    // fine level -> this level's coarse parent (valid for l < last)
    const Interp* py;
    const Gather* rx;    // coarse (l+1) cell -> fine cells of l
    const Gather* ry;
    // The same per coarse column / row as offset weights in the working precision
    // (RestrictAxis<T>, fc_smooth.cuh), built by the host from rx / ry.
    const void* rwx;
    const void* rwy;
};

struct GridDesc
{
    int W, H, S;
    int levels;          // multigrid levels, the last one solved directly
    int tail;            // first level handled by the one-block coarse tail
    int ncoarse;         // unknowns of the coarsest solve (cells - 1)
    double dx;
    LevelDesc lev[kMaxLevels];
    // fine-level vectors (padded layout)
    void* r;
    void* z;
    void* d[2];
    void* q;
    double* p;
    double* p_prev;
    double* b;
    // face velocities, unpadded: u is (W+1) x H, v is W x (H+1), row-major
    void* u;
    void* v;
    // coarsest inverse, up to ncoarse x ncoarse, row-major FP64, and its unknown map
    double* coarse_inverse;
    CoarseInfo* coarse;
    SolveState* state;
    double4* partial;        // one slot per tile of the largest reduction
    unsigned int* counter;   // arrival counter of the reduction in flight
    int vec_tiles;           // tiles of the fine vector kernels
    int post_tiles;          // tiles of the level-0 post-smoothing kernel (0 when tail == 0)
    unsigned char* solid;    // optional obstacle mask, W x H, unpadded (null: none)
    // Dirichlet air model (null: the reference's gas model): 1 where a cell is air held at
    // p = 0, neither solid nor liquid phase (f > 0.5). Written by k_coefficients from `fraction`.
    unsigned char* air;
    const double* fraction;  // liquid fraction, W x H, unpadded
    double* density;         // W x H, unpadded
    double* const* masses;   // device array of `components` W x H mass fields
    int components;
    const void* maps;        // TMA tensor maps of the smoothed levels (see fc_stage.cuh)
};

// One CTA of work: grid index, tile origin in cells, and the tile's index within its grid.
struct Tile
{
    int grid;
    int x0;
    int y0;
    int index;
};

// Correctly rounded reciprocal in the working precision.
__device__ __forceinline__ float reciprocal(float v) { return __frcp_rn(v); }
__device__ __forceinline__ double reciprocal(double v) { return 1.0 / v; }

__device__ __forceinline__ double warp_sum(double v)
{
    for (int o = 16; o > 0; o >>= 1)
        v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ float warp_sum(float v)
{
    for (int o = 16; o > 0; o >>= 1)
        v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ double warp_max(double v)
{
    for (int o = 16; o > 0; o >>= 1)
        v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Block reduction of up to four doubles; lane (component) c is summed, or maxed when
// (max_mask >> c) & 1. Result valid in thread 0. Fixed order: deterministic.
template <int NT> __device__ double4 block_reduce4(double4 v, int max_mask)
{
    __shared__ double4 slots[NT / 32];
    double a[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
    for (int c = 0; c < 4; ++c)
        a[c] = ((max_mask >> c) & 1) ? warp_max(a[c]) : warp_sum(a[c]);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __syncthreads();
    if (lane == 0)
        slots[warp] = make_double4(a[0], a[1], a[2], a[3]);
    __syncthreads();
    double4 out = make_double4(0, 0, 0, 0);
    if (threadIdx.x == 0)
    {
        out = slots[0];
        for (int w = 1; w < NT / 32; ++w)
        {
            const double4 s = slots[w];
            out.x = (max_mask & 1) ? fmax(out.x, s.x) : out.x + s.x;
            out.y = (max_mask & 2) ? fmax(out.y, s.y) : out.y + s.y;
            out.z = (max_mask & 4) ? fmax(out.z, s.z) : out.z + s.z;
            out.w = (max_mask & 8) ? fmax(out.w, s.w) : out.w + s.w;
        }
    }
    return out;
}

// The last block's fold of a grid's per-tile partials, in tile order (deterministic): each
// thread folds a contiguous run (loads batched ahead of the sums, read from L2), then the runs
// are combined by block_reduce4. Leaves the result in *total (thread 0's view) and resets the
// counter. Must be called by all threads of the block, after the arrival's fence.
template <int NT> __device__ void fold_partials(const GridDesc& g, int tiles, double4* total, int max_mask)
{
    double4 acc = make_double4(0, 0, 0, 0);
    const int per = (tiles + NT - 1) / NT;
    const int first = threadIdx.x * per;
    const int last = min(tiles, first + per);
    constexpr int kBatch = 4;
    const double2* slots = reinterpret_cast<const double2*>(g.partial);
    for (int t0 = first; t0 < last; t0 += kBatch)
    {
        double2 lo[kBatch], hi[kBatch];
#pragma unroll
        for (int u = 0; u < kBatch; ++u)
            if (t0 + u < last)
            {
                lo[u] = __ldcg(slots + 2 * (t0 + u));
                hi[u] = __ldcg(slots + 2 * (t0 + u) + 1);
            }
#pragma unroll
        for (int u = 0; u < kBatch; ++u)
            if (t0 + u < last)
            {
                acc.x = (max_mask & 1) ? fmax(acc.x, lo[u].x) : acc.x + lo[u].x;
                acc.y = (max_mask & 2) ? fmax(acc.y, lo[u].y) : acc.y + lo[u].y;
                acc.z = (max_mask & 4) ? fmax(acc.z, hi[u].x) : acc.z + hi[u].x;
                acc.w = (max_mask & 8) ? fmax(acc.w, hi[u].y) : acc.w + hi[u].y;
            }
    }
    const double4 out = block_reduce4<NT>(acc, max_mask);
    if (threadIdx.x == 0)
    {
        *total = out;
        *g.counter = 0u;
        __threadfence();
    }
    __syncthreads();
}

// Publishes this tile's partial and reports whether this block is the last of its grid to
// arrive; the last block then folds every partial (fold_partials). Must be called by all
// threads of the block.
template <int NT>
__device__ bool arrive_last(const GridDesc& g, int tile_index, int tiles, double4 mine, double4* total, int max_mask)
{
    __shared__ int is_last;
    if (threadIdx.x == 0)
    {
        g.partial[tile_index] = mine;
        __threadfence();
        const unsigned int ticket = atomicAdd(g.counter, 1u);
        is_last = ticket == unsigned(tiles - 1);
    }
    __syncthreads();
    if (!is_last)
        return false;
    __threadfence();
    fold_partials<NT>(g, tiles, total, max_mask);
    return true;
}

// Arrival of a persistent kernel's run of `run_tiles` tiles of one grid whose partials thread 0
// already wrote to g.partial[tile]: the CTA counts the run once instead of once per tile, and
// the last CTA to arrive folds all `tiles` partials (fold_partials). Must be called by all
// threads of the block.
template <int NT>
__device__ bool arrive_count(const GridDesc& g, int run_tiles, int tiles, double4* total, int max_mask)
{
    __shared__ int is_last;
    if (threadIdx.x == 0)
    {
        __threadfence(); // the partials before the count
        const unsigned int ticket = atomicAdd(g.counter, unsigned(run_tiles));
        is_last = ticket + unsigned(run_tiles) == unsigned(tiles);
    }
    __syncthreads();
    if (!is_last)
        return false;
    __threadfence();
    fold_partials<NT>(g, tiles, total, max_mask);
    return true;
}

// Arrival of a persistent kernel's run of `run_tiles` tiles of one grid whose partial pairs are
// already written to `pairs` (`entries` slots in all, indexed by tile). The CTA counts the run
// once instead of once per tile; the last CTA to arrive folds all pairs in slot order (each
// thread a contiguous run, loads batched; deterministic), leaves the sums in total->x, total->y
// (thread 0) and resets the counter. Must be called by all threads.
template <int NT>
__device__ bool arrive_run(const GridDesc& g, const double2* pairs, int run_tiles, int grid_tiles, int entries,
    double4* total)
{
    __shared__ int is_last;
    __threadfence(); // the writers' partials before the count
    __syncthreads();
    if (threadIdx.x == 0)
    {
        const unsigned int ticket = atomicAdd(g.counter, unsigned(run_tiles));
        is_last = ticket + unsigned(run_tiles) == unsigned(grid_tiles);
    }
    __syncthreads();
    if (!is_last)
        return false;
    __threadfence();
    const int per = (entries + NT - 1) / NT;
    const int first = threadIdx.x * per;
    const int last = min(entries, first + per);
    double sx = 0.0, sy = 0.0;
    constexpr int kBatch = 8;
    for (int e = first; e < last; e += kBatch)
    {
        double2 v[kBatch];
#pragma unroll
        for (int u = 0; u < kBatch; ++u)
            v[u] = e + u < last ? __ldcg(pairs + e + u) : make_double2(0.0, 0.0);
#pragma unroll
        for (int u = 0; u < kBatch; ++u)
            if (e + u < last)
            {
                sx += v[u].x;
                sy += v[u].y;
            }
    }
    const double4 out = block_reduce4<NT>(make_double4(sx, sy, 0.0, 0.0), 0);
    if (threadIdx.x == 0)
    {
        *total = out;
        *g.counter = 0u;
        __threadfence();
    }
    __syncthreads();
    return true;
}

__device__ __forceinline__ void stage_failed_at(SolveState* state)
{
    state->status = kBreakdown;
    state->done = 1;
}

// Whether a grid's solve was done already before this kernel's dependency wait, read from L2.
// Inside a projection the flag only rises (the set-up clears it with ordinary launches, which
// complete before any kernel of the loop starts; the timing and tuning entry points clear it
// with copies ordered before their launches), so a done flag read before the wait is still done
// after it. A flag read as running may be stale and is settled after the wait.
__device__ __forceinline__ bool done_before_wait(const SolveState* s) { return __ldcg(&s->done) != 0; }

// Records a failed wait (the staged data never arrived) on the tile's grid; returns true then.
__device__ __forceinline__ bool stage_failed(bool ok, SolveState* state)
{
    if (__syncthreads_or(!ok))
    {
        if (threadIdx.x == 0)
            stage_failed_at(state);
        return true;
    }
    return false;
}

// Programmatic dependent launch. The kernels of the PCG loop are launched so that each may
// start while its predecessor finishes: allow_dependents() lets the next kernel's CTAs be
// scheduled once every CTA of this one has started, and dependency_wait() blocks until every
// earlier kernel has completed and its writes are visible. Before the wait a kernel reads only
// data no kernel of the projection writes (tiles, descriptors, face weights, transfer tables).
__device__ __forceinline__ void dependency_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void allow_dependents() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
// Start of a kernel that reads earlier kernels' writes from its first instruction: its own
// successor may be scheduled at once, and it waits for its predecessors. Launched without
// programmatic serialization, both are no-ops.
__device__ __forceinline__ void dependent_start()
{
    allow_dependents();
    dependency_wait();
}

} // namespace fc
