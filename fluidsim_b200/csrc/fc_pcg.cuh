// Fine-level PCG kernels of the UniformCUDA projection.
//
// Every kernel takes the grid descriptors and a tile table, so one launch serves one grid or a
// batch of independent grids of uneven sizes (each CTA looks up its grid). A tile is 32 x 32
// cells worked by 256 threads, 4 rows each. Reductions are folded in FP64: each CTA writes one
// partial and the last CTA of a grid to arrive folds them in tile order, so results do not
// depend on which other grids share the launch.
//
// The per-iteration schedule follows FluidGridCPU::solvePressure (FluidGridCPU.cpp:1728-1824):
//   dir_op   d = (z - mean z) + beta d ; q = A d ; d.q            (operator :1507-1598)
//   update   p += alpha d ; r -= alpha q ; sum r, max |r|, sum r^2  (:1600-1641)
//   verify   on a met stop rule: r = b - A p, accept or restart     (:1795-1804, :1643-1683)
//   V-cycle  z = M r (fc_multigrid.cuh), then r.z and beta          (:1685-1726)
#pragma once

#include "fc_device.cuh"

namespace fc
{

template <typename T> __device__ __forceinline__ double dd(T v) { return double(v); }

// Arithmetic of the stop rule: max-norm (the reference rule) and/or squared L2 norm.
__device__ __forceinline__ bool stop_rule_met(const SolveState& s, double maximum, double sumsq)
{
    return maximum <= s.tol_max && sumsq <= s.tol_sumsq;
}

// The trigger for verifying the true residual. The operator's range is mean-free, so no
// iteration changes the mean of the recurrence residual: in FP64 it stays at rounding level,
// and the reference's rule (max |r| and sum r^2) applies unchanged. In FP32 the rounding of
// each update adds a mean that can exceed the tolerance after a large initial residual (a poor
// warm start) and would hold max |r| above it for good. FP32 therefore judges the mean-free
// part: max |r| - |mean| (max |r - mean| <= tol implies it) and sum (r - mean)^2 over the open
// cells (sum r^2 - sum * mean). The verification that follows recomputes b - A p in FP64 and
// accepts only under the reference's rule; a premature trigger costs one verification and a
// restart from the true residual.
template <typename T>
__device__ __forceinline__ bool recurrence_rule_met(const SolveState& s, double maximum, double sum, double sumsq)
{
    if constexpr (sizeof(T) == sizeof(double))
        return stop_rule_met(s, maximum, sumsq);
    else
    {
        const double mean = sum * s.inv_cells;
        return stop_rule_met(s, maximum - fabs(mean), sumsq - sum * mean);
    }
}

// Residual refresh of the FP32 solve. An FP32 recurrence residual tracks the true residual
// b - A p only to about 1e-6 of the residual it started from; past that it keeps falling while
// the true residual stalls, and a stop rule far below that level (the reference's absolute
// rule asks for a max-norm reduction of about 1e-9 on the dam breaks) is met only by the
// recurrence, so the verification fails and the solve restarts late. The FP32 solve therefore
// verifies early: when its stop rule lies more than kRefreshDepth below the residual of the
// last true-residual computation, the recurrence's max-norm falling by kRefreshRatio triggers
// one: r = b - A p in FP64 from the FP64 pressure, then a restart of the directions (iterative
// refinement with inner FP32 PCG solves). A refresh that meets the stop rule ends the solve
// like any verification. Measured on the 2048 x 2048 dam break under the reference's rule:
// 85 iterations without refreshes, 61 with a ratio of 1e-4 (63 at 1e-3 and 1e-5, 62 at 3e-3
// and 3e-4, 66 at 1e-6); keeping
// the directions across the refresh instead (residual replacement) gave 61 at 1e-4 and 111 at
// 1e-5, and 96 instead of 84 with 16 obstacles at 1024 x 1024. FP64 keeps the reference's
// schedule.
#ifndef FC_REFRESH_RATIO
#define FC_REFRESH_RATIO 1e-4
#endif
constexpr double kRefreshRatio = FC_REFRESH_RATIO;
constexpr double kRefreshDepth = 1e-6;

template <typename T> __device__ __forceinline__ double refresh_threshold(const SolveState& s, double maximum, double sumsq)
{
    if constexpr (sizeof(T) == sizeof(double))
        return 0.0;
    else
        return s.tol_max < kRefreshDepth * maximum || s.tol_sumsq < kRefreshDepth * kRefreshDepth * sumsq
            ? kRefreshRatio * maximum : 0.0;
}

__device__ __forceinline__ bool cell_solid(const GridDesc& g, int x, int y)
{
    return g.solid && g.solid[(long long)y * g.W + x];
}

// A cell that is no unknown of the pressure solve: solid, or air under the Dirichlet model
// (held at p = 0; its faces keep their weights, so its liquid neighbours see the zero).
__device__ __forceinline__ bool cell_held(const GridDesc& g, int x, int y)
{
    return cell_solid(g, x, y) || (g.air && g.air[(long long)y * g.W + x]);
}

// cell_held through the kernel's own copies of the masks: `restrict` tells the compiler that no
// store of the kernel writes them, so their loads may be issued ahead of its stores.
__device__ __forceinline__ bool held_at(const unsigned char* __restrict__ solid, const unsigned char* __restrict__ air,
    int W, int x, int y)
{
    const long long c = (long long)y * W + x;
    return (solid && solid[c]) || (air && air[c]);
}

#define FC_VEC_TILE_PROLOGUE                                                                       \
    const Tile t = tiles[blockIdx.x];                                                              \
    const GridDesc& g = grids[t.grid];                                                             \
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;

// Density from component masses: sum of liquid then gas masses, times 1/dx^2.
// FluidGridCPU.cpp:1399-1423 (rebuildDensity).
__global__ void k_density(const GridDesc* __restrict__ grids, const Tile* __restrict__ tiles)
{
    dependent_start();
    FC_VEC_TILE_PROLOGUE
    const double inv_area = 1.0 / (g.dx * g.dx);
    const int W = g.W, H = g.H, components = g.components;
    const double* const* __restrict__ masses = g.masses;
    double* __restrict__ density = g.density;
#pragma unroll
    for (int k = 0; k < kVecCells; ++k)
    {
        const int x = t.x0 + tx + 32 * (k & 1), y = t.y0 + ty + 8 * (k >> 1);
        if (x >= W || y >= H)
            continue;
        const long long i = (long long)y * W + x;
        double total = 0.0;
        for (int m = 0; m < components; ++m)
            total += masses[m][i];
        density[i] = total * inv_area;
    }
}

// Face weights 2/(rho_a + rho_b), zero on walls and around solid cells.
// FluidGridCPU.cpp:1154-1205 (rebuildPressureCoefficients).
template <typename T> __global__ void k_coefficients(const GridDesc* __restrict__ grids, const Tile* __restrict__ tiles)
{
    dependent_start();
    FC_VEC_TILE_PROLOGUE
    const double* __restrict__ density = g.density;
    T* __restrict__ right = static_cast<T*>(g.lev[0].right);
    T* __restrict__ down = static_cast<T*>(g.lev[0].down);
    const int W = g.W, H = g.H, S = g.S;
    const unsigned char* __restrict__ solid_mask = g.solid;
    unsigned char* __restrict__ air = g.air;
    const double* __restrict__ fraction = g.fraction;
    auto solid_at = [&](int sx, int sy) { return solid_mask && solid_mask[(long long)sy * W + sx]; };
#pragma unroll
    for (int k = 0; k < kVecCells; ++k)
    {
        const int x = t.x0 + tx + 32 * (k & 1), y = t.y0 + ty + 8 * (k >> 1);
        if (x >= W || y >= H)
            continue;
        const long long c = (long long)y * W + x;
        const long long i = padded_index(S, x, y);
        const bool solid = solid_at(x, y);
        if (air)
            air[c] = !solid && !(fraction[c] > 0.5); // FluidGridCPU.cpp:1321-1322: liquid is f > 0.5
        double wr = 0.0, wd = 0.0;
        if (x + 1 < W && !solid && !solid_at(x + 1, y))
            wr = 2.0 / (density[c] + density[c + 1]);
        if (y + 1 < H && !solid && !solid_at(x, y + 1))
            wd = 2.0 / (density[c] + density[c + W]);
        right[i] = T(wr);
        down[i] = T(wd);
    }
}

// Closed faces (outer walls, and faces of solid cells) read as zero; the thread of the cell on
// the low side of a face writes the zero. Returns the four face velocities of cell (x, y).
template <typename T>
__device__ __forceinline__ void cell_faces(T* __restrict__ u, T* __restrict__ v, const unsigned char* __restrict__ solid,
    int W, int H, int x, int y, bool write_closed, double& ul, double& ur, double& vu, double& vd)
{
    const long long iu = (long long)y * (W + 1) + x;
    const long long iv = (long long)y * W + x;
    auto solid_at = [&](int sx, int sy) { return solid && solid[(long long)sy * W + sx]; };
    const bool here = solid_at(x, y);
    const bool closed_l = x == 0 || here || solid_at(x - 1, y);
    const bool closed_r = x + 1 == W || here || solid_at(x + 1, y);
    const bool closed_u = y == 0 || here || solid_at(x, y - 1);
    const bool closed_d = y + 1 == H || here || solid_at(x, y + 1);
    ul = closed_l ? 0.0 : dd(u[iu]);
    ur = closed_r ? 0.0 : dd(u[iu + 1]);
    vu = closed_u ? 0.0 : dd(v[iv]);
    vd = closed_d ? 0.0 : dd(v[iv + W]);
    if (write_closed)
    {
        // Each closed face is zeroed by exactly one cell: the left/upper face by this cell when
        // it is the outer wall or this cell is solid; the right/lower face when it is the wall.
        if (closed_r)
            u[iu + 1] = T(0);
        if (closed_d)
            v[iv + W] = T(0);
        if (x == 0)
            u[iu] = T(0);
        if (y == 0)
            v[iv] = T(0);
    }
}

// b = -(du + dv)/dx * dx^2/dt with closed faces zeroed; sums b over open cells.
// FluidGridCPU.cpp:1050-1083.
template <typename T> __global__ void __launch_bounds__(kVecThreads) k_rhs(const GridDesc* __restrict__ grids, const Tile* __restrict__ tiles)
{
    dependent_start();
    FC_VEC_TILE_PROLOGUE
    const double dt = g.state->dt;
    const double dx = g.dx;
    const double scale = dx * dx / dt;
    const int W = g.W, H = g.H, S = g.S;
    T* __restrict__ u = static_cast<T*>(g.u);
    T* __restrict__ v = static_cast<T*>(g.v);
    const unsigned char* __restrict__ solid = g.solid;
    const unsigned char* __restrict__ air = g.air;
    double* __restrict__ rhs = g.b;
    double sum = 0.0;
#pragma unroll
    for (int k = 0; k < kVecCells; ++k)
    {
        const int x = t.x0 + tx + 32 * (k & 1), y = t.y0 + ty + 8 * (k >> 1);
        if (x >= W || y >= H)
            continue;
        double ul, ur, vu, vd;
        cell_faces<T>(u, v, solid, W, H, x, y, true, ul, ur, vu, vd);
        const double du = ur - ul;
        const double dv = vd - vu;
        double b = -(du + dv) / dx * scale;
        if (held_at(solid, air, W, x, y))
            b = 0.0;
        rhs[padded_index(S, x, y)] = b;
        sum += b;
    }
    __shared__ double4 total;
    if (arrive_last<kVecThreads>(g, t.index, g.vec_tiles, block_reduce4<kVecThreads>(make_double4(sum, 0, 0, 0), 0), &total, 0))
    {
        if (threadIdx.x == 0)
            g.state->mean_b = total.x * g.state->inv_cells;
    }
}

// max |b - mean| and sum (b - mean)^2; decides the early exit (FluidGridCPU.cpp:1731-1740).
template <typename T> __global__ void __launch_bounds__(kVecThreads) k_rhs_stats(const GridDesc* __restrict__ grids, const Tile* __restrict__ tiles)
{
    dependent_start();
    FC_VEC_TILE_PROLOGUE
    const double mean = g.state->mean_b;
    const int W = g.W, H = g.H, S = g.S;
    const unsigned char* __restrict__ solid = g.solid;
    const unsigned char* __restrict__ air = g.air;
    const double* __restrict__ rhs = g.b;
    double mx = 0.0, sq = 0.0;
#pragma unroll
    for (int k = 0; k < kVecCells; ++k)
    {
        const int x = t.x0 + tx + 32 * (k & 1), y = t.y0 + ty + 8 * (k >> 1);
        if (x >= W || y >= H || held_at(solid, air, W, x, y))
            continue;
        const double b = rhs[padded_index(S, x, y)] - mean;
        mx = fmax(mx, isfinite(b) ? fabs(b) : INFINITY);
        sq += b * b;
    }
    __shared__ double4 total;
    if (arrive_last<kVecThreads>(g, t.index, g.vec_tiles, block_reduce4<kVecThreads>(make_double4(mx, sq, 0, 0), 1), &total, 1))
    {
        if (threadIdx.x == 0)
        {
            SolveState& s = *g.state;
            s.bmax = total.x;
            s.bsumsq = total.y;
            if (s.tol_sumsq < 0.0) // relative rule requested: -tol_sumsq carries tol^2
                s.tol_sumsq = -s.tol_sumsq * total.y;
            if (stop_rule_met(s, total.x, total.y))
            {
                s.status = kNoWork;
                s.done = 1;
            }
        }
    }
}

// Warm start p = 2p - p_prev, or clear both when no solve is needed; sums the prediction.
// FluidGridCPU.cpp:1731-1753.
__global__ void __launch_bounds__(kVecThreads) k_warm_start(const GridDesc* __restrict__ grids, const Tile* __restrict__ tiles)
{
    dependent_start();
    FC_VEC_TILE_PROLOGUE
    const bool clear = g.state->status == kNoWork;
    const int W = g.W, H = g.H, S = g.S;
    const unsigned char* __restrict__ solid = g.solid;
    const unsigned char* __restrict__ air = g.air;
    double* __restrict__ p = g.p;
    double* __restrict__ p_prev = g.p_prev;
    double sum = 0.0;
#pragma unroll
    for (int k = 0; k < kVecCells; ++k)
    {
        const int x = t.x0 + tx + 32 * (k & 1), y = t.y0 + ty + 8 * (k >> 1);
        if (x >= W || y >= H)
            continue;
        const long long i = padded_index(S, x, y);
        if (clear || held_at(solid, air, W, x, y))
        {
            p[i] = 0.0;
            p_prev[i] = 0.0;
            continue;
        }
        const double latest = p[i];
        const double predicted = 2.0 * latest - p_prev[i];
        p[i] = predicted;
        p_prev[i] = latest;
        sum += predicted;
    }
    __shared__ double4 total;
    if (arrive_last<kVecThreads>(g, t.index, g.vec_tiles, block_reduce4<kVecThreads>(make_double4(sum, 0, 0, 0), 0), &total, 0))
    {
        if (threadIdx.x == 0)
            g.state->mean_p = total.x * g.state->inv_cells;
    }
}

// Pressure sum for the final mean removal.
__global__ void __launch_bounds__(kVecThreads) k_pressure_sum(const GridDesc* __restrict__ grids, const Tile* __restrict__ tiles)
{
    dependent_start();
    FC_VEC_TILE_PROLOGUE
    if (g.state->status == kBreakdown)
        return;
    const int W = g.W, H = g.H, S = g.S;
    const unsigned char* __restrict__ solid = g.solid;
    const unsigned char* __restrict__ air = g.air;
    const double* __restrict__ p = g.p;
    double sum = 0.0;
#pragma unroll
    for (int k = 0; k < kVecCells; ++k)
    {
        const int x = t.x0 + tx + 32 * (k & 1), y = t.y0 + ty + 8 * (k >> 1);
        if (x >= W || y >= H || held_at(solid, air, W, x, y))
            continue;
        sum += p[padded_index(S, x, y)];
    }
    __shared__ double4 total;
    if (arrive_last<kVecThreads>(g, t.index, g.vec_tiles, block_reduce4<kVecThreads>(make_double4(sum, 0, 0, 0), 0), &total, 0))
    {
        if (threadIdx.x == 0)
            g.state->mean_p = total.x * g.state->inv_cells;
    }
}

// p -= mean_p over open cells (FluidGridCPU.cpp:1466-1474, removeMean).
__global__ void k_remove_pressure_mean(const GridDesc* __restrict__ grids, const Tile* __restrict__ tiles)
{
    dependent_start();
    FC_VEC_TILE_PROLOGUE
    if (g.state->status == kBreakdown)
        return;
    const double mean = g.state->mean_p;
    const int W = g.W, H = g.H, S = g.S;
    const unsigned char* __restrict__ solid = g.solid;
    const unsigned char* __restrict__ air = g.air;
    double* __restrict__ p = g.p;
#pragma unroll
    for (int k = 0; k < kVecCells; ++k)
    {
        const int x = t.x0 + tx + 32 * (k & 1), y = t.y0 + ty + 8 * (k >> 1);
        if (x >= W || y >= H)
            continue;
        const long long i = padded_index(S, x, y);
        // Pressure inside obstacles (and in Dirichlet air) is held at zero.
        p[i] = held_at(solid, air, W, x, y) ? 0.0 : p[i] - mean;
    }
}

template <typename T>
__device__ __forceinline__ double apply_cell_fp64(const T* right, const T* down, const double* x, long long i, int S)
{
    const double c = x[i];
    return (dd(right[i - 1]) * (c - x[i - 1]) + dd(right[i]) * (c - x[i + 1])) +
           (dd(down[i - S]) * (c - x[i - S]) + dd(down[i]) * (c - x[i + S]));
}

// p + alpha d with one rounding (a fused multiply-add), the same wherever a pressure step is
// applied (k_update, k_flush_pressure) or read as pending (k_true_residual).
__device__ __forceinline__ double step_value(double p, double alpha, double d) { return __fma_rn(alpha, d, p); }

// A p at cell i with p + alpha d in place of p: the pressure with the pending step of a pair
// (k_update), each value formed exactly as k_update forms it.
template <typename T>
__device__ __forceinline__ double apply_cell_fp64_pending(const T* right, const T* down, const double* x, const T* d,
    double alpha, long long i, int S)
{
    auto at = [&](long long j) { return step_value(x[j], alpha, double(d[j])); };
    const double c = at(i);
    return (dd(right[i - 1]) * (c - at(i - 1)) + dd(right[i]) * (c - at(i + 1))) +
           (dd(down[i - S]) * (c - at(i - S)) + dd(down[i]) * (c - at(i + S)));
}

// True residual r = (b - mean b) - A p in FP64, stored in the working type, with its stats.
// `initial` selects the solve's first residual (FluidGridCPU.cpp:1754-1757) versus the
// convergence check inside the loop (:1795-1804).
template <typename T>
__global__ void __launch_bounds__(kVecThreads) k_true_residual(const GridDesc* __restrict__ grids, const Tile* __restrict__ tiles, int initial)
{
    allow_dependents();
    FC_VEC_TILE_PROLOGUE
    SolveState& s = *g.state;
    dependency_wait();
    if (s.done || (!initial && !s.verify))
        return;
    const T* __restrict__ right = static_cast<const T*>(g.lev[0].right);
    const T* __restrict__ down = static_cast<const T*>(g.lev[0].down);
    T* __restrict__ r = static_cast<T*>(g.r);
    const double* __restrict__ rhs = g.b;
    const double* __restrict__ p = g.p;
    const int W = g.W, H = g.H, S = g.S;
    const unsigned char* __restrict__ solid = g.solid;
    const unsigned char* __restrict__ air = g.air;
    const double mean_b = s.mean_b;
    // Inside a pair the pressure still lacks the first iteration's step (k_update).
    const bool pending = !initial && s.p_pending;
    const T* __restrict__ d0 = static_cast<const T*>(g.d[1]);
    const double alpha0 = s.alpha_pending;
    double sum = 0.0, mx = 0.0, sq = 0.0;
#pragma unroll
    for (int k = 0; k < kVecCells; ++k)
    {
        const int x = t.x0 + tx + 32 * (k & 1), y = t.y0 + ty + 8 * (k >> 1);
        if (x >= W || y >= H)
            continue;
        const long long i = padded_index(S, x, y);
        double value = 0.0;
        if (!held_at(solid, air, W, x, y))
            value = (rhs[i] - mean_b) - (pending ? apply_cell_fp64_pending(right, down, p, d0, alpha0, i, S)
                                                 : apply_cell_fp64(right, down, p, i, S));
        const T stored = T(value);
        r[i] = stored;
        const double rv = dd(stored);
        sum += rv;
        mx = fmax(mx, fabs(rv));
        sq += rv * rv;
    }
    __shared__ double4 total;
    if (arrive_last<kVecThreads>(g, t.index, g.vec_tiles, block_reduce4<kVecThreads>(make_double4(sum, mx, sq, 0), 2), &total, 2))
    {
        if (threadIdx.x == 0)
        {
            const double maximum = isfinite(total.x) ? total.y : INFINITY;
            s.sum_r = total.x;
            s.max_r = maximum;
            s.sumsq_r = total.z;
            s.res_max = maximum;
            s.res_sumsq = total.z;
            s.mean_r = total.x * s.inv_cells;
            const int refresh = s.verify == 2;
            s.verify = 0;
            s.refresh_max = refresh_threshold<T>(s, maximum, total.z);
            if (stop_rule_met(s, maximum, total.z))
            {
                s.status = kConverged;
                s.done = 1;
            }
            else if (s.iterations >= s.max_iterations)
            {
                s.status = kIterationLimit;
                s.done = 1;
            }
            else if (s.use_mg && !s.mg_valid)
            {
                s.status = kBreakdown;
                s.done = 1;
            }
            else
            {
                s.restart = 1;
                s.restarts += initial || refresh ? 0 : 1;
                s.refreshes += refresh;
            }
        }
    }
}

template <typename T> struct VecPair;
template <> struct VecPair<float>
{
    using type = float2;
};
template <> struct VecPair<double>
{
    using type = double2;
};

// d = (z - mean z) + beta d_old; q = A d; d.q through the grid's reduction. Warp w handles rows
// 8w .. 8w + 7 of the tile's 64 columns (lane = column pair) in four passes of two rows: all
// loads of a pass (four rows of z and d, two rows of weights) are issued first, then the
// directions and the operator are formed in registers; horizontal neighbours across pairs are
// warp shuffles, and lanes 0 and 31 fetch the columns just outside the warp. At 64 registers
// four CTAs fit an SM in FP32, which hides more load latency than passes of four rows at 80
// registers and three CTAs (31.5 -> 30.2 us at 2048 x 2048).
// Operator: FluidGridCPU.cpp:1507-1598.
template <typename T>
__global__ void __launch_bounds__(kVecThreads, sizeof(T) == 4 ? 4 : 1)
    k_direction_operator(const GridDesc* __restrict__ grids, const Tile* __restrict__ tiles, int parity)
{
    using P = typename VecPair<T>::type;
    constexpr int R = 2;
    allow_dependents();
    const Tile t = tiles[blockIdx.x];
    const GridDesc& g = grids[t.grid];
    SolveState& s = *g.state;
    dependency_wait();
    if (s.done)
        return;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const T* right = static_cast<const T*>(g.lev[0].right);
    const T* down = static_cast<const T*>(g.lev[0].down);
    const T* z = static_cast<const T*>(g.z);
    const T* d_old = static_cast<const T*>(g.d[parity]);
    T* d_new = static_cast<T*>(g.d[parity ^ 1]);
    T* q = static_cast<T*>(g.q);
    const T mz = T(s.mean_z), b = T(s.beta);
    const int S = g.S;
    const int gx = t.x0 + 2 * lane;
    const bool cols = gx < g.W; // the pair's first column lies in the grid
    const bool in_b = gx + 1 < g.W;
    // Column just outside the warp: left of the first pair for lane 0, right of the last for 31.
    const int edge_x = lane == 0 ? gx - 1 : gx + 2;
    const bool edge = (lane == 0 && cols) || (lane == 31 && gx + 2 + kPadX < S);
    P up_w = P{};
    if (cols)
        up_w = *reinterpret_cast<const P*>(down + padded_index(S, gx, t.y0 + 8 * warp - 1));
    double dot = 0.0;
#pragma unroll 1
    for (int pass = 0; pass < 8 / R; ++pass)
    {
        const int y0 = t.y0 + 8 * warp + R * pass;
        P zz[R + 2], dd0[R + 2], w[R], dn[R];
        T ez[R], ed[R], ew[R];
#pragma unroll
        for (int k = 0; k < R + 2; ++k)
        {
            const int y = y0 - 1 + k;
            zz[k] = P{};
            dd0[k] = P{};
            if (cols && y >= -1 && y <= g.H)
            {
                const long long i = padded_index(S, gx, y);
                zz[k] = *reinterpret_cast<const P*>(z + i);
                dd0[k] = *reinterpret_cast<const P*>(d_old + i);
            }
        }
#pragma unroll
        for (int k = 0; k < R; ++k)
        {
            const int y = y0 + k;
            w[k] = P{};
            dn[k] = P{};
            ez[k] = ed[k] = ew[k] = T(0);
            if (y < g.H)
            {
                const long long i = padded_index(S, gx, y);
                if (cols)
                {
                    w[k] = *reinterpret_cast<const P*>(right + i);
                    dn[k] = *reinterpret_cast<const P*>(down + i);
                }
                if (edge)
                {
                    const long long e = padded_index(S, edge_x, y);
                    ez[k] = z[e];
                    ed[k] = d_old[e];
                    ew[k] = right[e]; // lane 0: the face between gx - 1 and gx
                }
            }
        }
        // Directions in the working precision (the operator and the p update read exactly the
        // stored d); halo rows and padding columns read zero fields.
        P dir[R + 2];
#pragma unroll
        for (int k = 0; k < R + 2; ++k)
        {
            dir[k].x = (zz[k].x - mz) + b * dd0[k].x;
            dir[k].y = (zz[k].y - mz) + b * dd0[k].y;
        }
#pragma unroll
        for (int k = 0; k < R; ++k)
        {
            const int y = y0 + k;
            const P prev = dir[k], cur = dir[k + 1], next = dir[k + 2];
            T left = __shfl_up_sync(0xffffffffu, cur.y, 1);
            T right_d = __shfl_down_sync(0xffffffffu, cur.x, 1);
            T wl = __shfl_up_sync(0xffffffffu, w[k].y, 1);
            const T edge_dir = (ez[k] - mz) + b * ed[k];
            if (lane == 0)
            {
                left = edge_dir;
                wl = ew[k];
            }
            if (lane == 31)
                right_d = edge_dir;
            const P uw = k == 0 ? up_w : dn[k - 1];
            if (cols && y < g.H)
            {
                const long long i = padded_index(S, gx, y);
                const T ca = cur.x, cb = cur.y;
                T qa = (wl * (ca - left) + w[k].x * (ca - cb)) + (uw.x * (ca - prev.x) + dn[k].x * (ca - next.x));
                T qb = (w[k].x * (cb - ca) + w[k].y * (cb - right_d)) + (uw.y * (cb - prev.y) + dn[k].y * (cb - next.y));
                if (g.air)
                {
                    // Dirichlet air is no unknown: its direction is zero and its q stays zero,
                    // so its residual stays zero.
                    const unsigned char* air = g.air + (long long)y * g.W + gx;
                    qa = air[0] ? T(0) : qa;
                    qb = in_b && air[1] ? T(0) : qb;
                }
                if (in_b)
                {
                    *reinterpret_cast<P*>(d_new + i) = cur;
                    P qq;
                    qq.x = qa;
                    qq.y = qb;
                    *reinterpret_cast<P*>(q + i) = qq;
                    dot += double(ca) * double(qa) + double(cb) * double(qb);
                }
                else
                {
                    d_new[i] = ca;
                    q[i] = qa;
                    dot += double(ca) * double(qa);
                }
            }
        }
        up_w = dn[R - 1];
    }
    __shared__ double4 total;
    if (arrive_last<kVecThreads>(g, t.index, g.vec_tiles, block_reduce4<kVecThreads>(make_double4(dot, 0, 0, 0), 0), &total, 0))
    {
        if (threadIdx.x == 0)
        {
            s.dq = total.x;
            const double alpha = s.rz / total.x;
            if (!(total.x > 0.0) || !isfinite(total.x) || !isfinite(alpha))
            {
                s.status = kStalled;
                s.done = 1;
            }
        }
    }
}

// p += alpha d ; r -= alpha q ; residual stats. FluidGridCPU.cpp:1600-1641.
// The padded halo and row padding of d, q, r and p are zero, so the update runs over the whole
// padded array as one flat stream cut into one equal slice per vector tile. The kernel is
// persistent (two CTAs per SM walk the slices of every grid), each thread takes two quads of
// four cells per step with every load of the step issued before the arithmetic, and a CTA
// counts its slices of a grid once; the per-slice partials and their fold are those of one CTA
// per slice.
//
// The loop runs its iterations in pairs (parity 0, then 1). Nothing inside the loop reads p
// except the true residual, so the first iteration of a pair updates only r and leaves its
// p += alpha_0 d_0 pending (alpha_pending, p_pending); the second applies it and then its own,
// p = (p + alpha_0 d_0) + alpha_1 d_1, the same two roundings as two separate updates. That
// streams p (16 B per cell in FP64) once per pair instead of once per iteration. The true
// residual reads p + alpha_0 d_0 while an update is pending (k_true_residual), and the loop's
// exit applies a pending update (k_flush_pressure) before anything after the loop reads p.
template <typename T> struct Quad;
template <> struct Quad<float>
{
    using type = float4;
};
template <> struct Quad<double>
{
    using type = double4;
};

constexpr int kUpdateCtasPerSm = 2;

template <typename T>
__device__ __forceinline__ void add_step(double4& p, double alpha, const typename Quad<T>::type& d)
{
    p.x = step_value(p.x, alpha, double(d.x));
    p.y = step_value(p.y, alpha, double(d.y));
    p.z = step_value(p.z, alpha, double(d.z));
    p.w = step_value(p.w, alpha, double(d.w));
}

template <typename T>
__global__ void __launch_bounds__(kVecThreads, kUpdateCtasPerSm)
    k_update(const GridDesc* __restrict__ grids, const Tile* __restrict__ tiles, int count, int parity)
{
    using Q = typename Quad<T>::type;
    // Quads per thread and step (FP64 takes one: its quads are twice the registers). A thread
    // visits the same quads in the same order either way.
    constexpr int U = sizeof(T) == 4 ? 2 : 1;
    allow_dependents();
    dependency_wait();
    __shared__ double4 total;
    int run = 0; // slices of the current grid finished since the last count
    for (int i = blockIdx.x; i < count; i += gridDim.x)
    {
        const Tile t = tiles[i];
        const GridDesc& g = grids[t.grid];
        SolveState& s = *g.state;
        if (s.done)
            continue;
        const T* d = static_cast<const T*>(g.d[parity ^ 1]);
        const T* q = static_cast<const T*>(g.q);
        T* r = static_cast<T*>(g.r);
        const double alpha = s.rz / s.dq;
        // Second of a pair: the first's pending step (its direction is the other buffer).
        const bool update_p = parity == 1;
        const bool pending = update_p && s.p_pending;
        const double alpha0 = s.alpha_pending;
        const T* d0 = static_cast<const T*>(g.d[parity]);
        // The padded length S * (H + 2) is a multiple of 8; slices are whole quads.
        const long long quads = (long long)g.S * (g.H + 2) / 4;
        const long long per = (quads + g.vec_tiles - 1) / g.vec_tiles;
        const long long first = per * t.index;
        const long long last = min(quads, first + per);
        double sum = 0.0, mx = 0.0, sq = 0.0;
        for (long long base = first + threadIdx.x; base < last; base += (long long)kVecThreads * U)
        {
            Q dv[U], d0v[U], qv[U], rv[U];
            double4 pv[U];
#pragma unroll
            for (int u = 0; u < U; ++u)
            {
                const long long j = base + (long long)u * kVecThreads;
                if (j < last)
                {
                    qv[u] = reinterpret_cast<const Q*>(q)[j];
                    rv[u] = reinterpret_cast<const Q*>(r)[j];
                    if (update_p)
                    {
                        dv[u] = reinterpret_cast<const Q*>(d)[j];
                        pv[u] = reinterpret_cast<const double4*>(g.p)[j];
                        if (pending)
                            d0v[u] = reinterpret_cast<const Q*>(d0)[j];
                    }
                }
            }
#pragma unroll
            for (int u = 0; u < U; ++u)
            {
                const long long j = base + (long long)u * kVecThreads;
                if (j >= last)
                    continue;
                if (update_p)
                {
                    double4 pp = pv[u];
                    if (pending)
                        add_step<T>(pp, alpha0, d0v[u]);
                    add_step<T>(pp, alpha, dv[u]);
                    reinterpret_cast<double4*>(g.p)[j] = pp;
                }
                Q rr;
                rr.x = T(double(rv[u].x) - alpha * double(qv[u].x));
                rr.y = T(double(rv[u].y) - alpha * double(qv[u].y));
                rr.z = T(double(rv[u].z) - alpha * double(qv[u].z));
                rr.w = T(double(rv[u].w) - alpha * double(qv[u].w));
                reinterpret_cast<Q*>(r)[j] = rr;
                const double e[4] = {double(rr.x), double(rr.y), double(rr.z), double(rr.w)};
#pragma unroll
                for (int c = 0; c < 4; ++c)
                {
                    sum += e[c];
                    mx = fmax(mx, fabs(e[c]));
                    sq += e[c] * e[c];
                }
            }
        }
        const double4 part = block_reduce4<kVecThreads>(make_double4(sum, mx, sq, 0), 2);
        if (threadIdx.x == 0)
            g.partial[t.index] = part;
        ++run;
        const int next = i + gridDim.x;
        if (next >= count || tiles[next].grid != t.grid)
        {
            if (arrive_count<kVecThreads>(g, run, g.vec_tiles, &total, 2))
            {
                if (threadIdx.x == 0)
                {
                    // Every slice of the grid has read the pending state by now.
                    s.p_pending = update_p ? 0 : 1;
                    s.alpha_pending = update_p ? 0.0 : alpha;
                    s.iterations += 1;
                    const double maximum = isfinite(total.x) ? total.y : INFINITY;
                    s.sum_r = total.x;
                    s.max_r = maximum;
                    s.sumsq_r = total.z;
                    s.mean_r = total.x * s.inv_cells;
                    if (recurrence_rule_met<T>(s, maximum, total.x, total.z))
                        s.verify = 1;
                    else if (s.iterations >= s.max_iterations)
                    {
                        s.status = kIterationLimit;
                        s.done = 1;
                    }
                    else if (maximum - fabs(s.mean_r) <= s.refresh_max)
                        s.verify = 2; // FP32 refresh (refresh_threshold)
                }
            }
            run = 0;
        }
    }
}

// Applies a pair's pending p += alpha d at the loop's exit (see k_update), over the padded
// array as one flat stream; p is read only after this.
template <typename T> __global__ void __launch_bounds__(kVecThreads) k_flush_pressure(const GridDesc* __restrict__ grids, const Tile* __restrict__ tiles)
{
    dependent_start();
    using Q = typename Quad<T>::type;
    const Tile t = tiles[blockIdx.x];
    const GridDesc& g = grids[t.grid];
    const SolveState& s = *g.state;
    if (!s.p_pending)
        return;
    const T* d0 = static_cast<const T*>(g.d[1]);
    const double alpha0 = s.alpha_pending;
    const long long quads = (long long)g.S * (g.H + 2) / 4;
    const long long per = (quads + g.vec_tiles - 1) / g.vec_tiles;
    const long long first = per * t.index;
    const long long last = min(quads, first + per);
    for (long long j = first + threadIdx.x; j < last; j += kVecThreads)
    {
        double4 pp = reinterpret_cast<const double4*>(g.p)[j];
        add_step<T>(pp, alpha0, reinterpret_cast<const Q*>(d0)[j]);
        reinterpret_cast<double4*>(g.p)[j] = pp;
    }
}

// u -= (dp/dx) dt w on open interior faces; each cell updates its left and upper face.
// FluidGridCPU.cpp:1098-1118.
template <typename T> __global__ void k_velocity_update(const GridDesc* __restrict__ grids, const Tile* __restrict__ tiles)
{
    dependent_start();
    FC_VEC_TILE_PROLOGUE
    if (g.state->status == kBreakdown)
        return;
    const double dt = g.state->dt, dx = g.dx;
    const int W = g.W, H = g.H, S = g.S;
    T* __restrict__ u = static_cast<T*>(g.u);
    T* __restrict__ v = static_cast<T*>(g.v);
    const T* __restrict__ right = static_cast<const T*>(g.lev[0].right);
    const T* __restrict__ down = static_cast<const T*>(g.lev[0].down);
    const double* __restrict__ p = g.p;
#pragma unroll
    for (int k = 0; k < kVecCells; ++k)
    {
        const int x = t.x0 + tx + 32 * (k & 1), y = t.y0 + ty + 8 * (k >> 1);
        if (x >= W || y >= H)
            continue;
        const long long i = padded_index(S, x, y);
        const double pc = p[i];
        if (x > 0)
        {
            const double w = dd(right[i - 1]);
            if (w != 0.0)
            {
                const long long f = (long long)y * (W + 1) + x;
                u[f] = T(dd(u[f]) - ((pc - p[i - 1]) / dx) * dt * w);
            }
        }
        if (y > 0)
        {
            const double w = dd(down[i - S]);
            if (w != 0.0)
            {
                const long long f = (long long)y * W + x;
                v[f] = T(dd(v[f]) - ((pc - p[i - S]) / dx) * dt * w);
            }
        }
    }
}

// Storage rounding of one face velocity: one unit in the last place of the working type.
__device__ __forceinline__ double face_ulp(float value)
{
    const unsigned int bits = __float_as_uint(fabsf(value)) & 0x7f800000u;
    return double(__uint_as_float(bits)) * 1.1920928955078125e-7;
}

__device__ __forceinline__ double face_ulp(double value)
{
    const unsigned long long bits = __double_as_longlong(fabs(value)) & 0x7ff0000000000000ull;
    return __longlong_as_double(bits) * 2.220446049250313e-16;
}

// max |div u| (FluidGridCPU.cpp:1126-1152), its excess over the float rounding allowance of the
// four faces (as UniformWebGPU's velocity_stats, FluidUniformWebGPUKernels.h:166-213), and the
// sum of squares.
template <typename T> __global__ void __launch_bounds__(kVecThreads) k_divergence(const GridDesc* __restrict__ grids, const Tile* __restrict__ tiles)
{
    dependent_start();
    FC_VEC_TILE_PROLOGUE
    const T* __restrict__ u = static_cast<const T*>(g.u);
    const T* __restrict__ v = static_cast<const T*>(g.v);
    const int W = g.W, H = g.H;
    const double dx = g.dx;
    const bool dirichlet = g.air != nullptr;
    const unsigned char* __restrict__ solid = g.solid;
    const double* __restrict__ fraction = g.fraction;
    double mx = 0.0, excess = 0.0, sq = 0.0;
    int nonfinite = 0;
#pragma unroll
    for (int k = 0; k < kVecCells; ++k)
    {
        const int x = t.x0 + tx + 32 * (k & 1), y = t.y0 + ty + 8 * (k >> 1);
        if (x >= W || y >= H)
            continue;
        // Dirichlet air: only the liquid is held divergence-free (classified from the current
        // fraction, so a check between steps needs no coefficient rebuild).
        const long long iv = (long long)y * W + x;
        if (dirichlet && ((solid && solid[iv]) || !(fraction[iv] > 0.5)))
            continue;
        const long long iu = (long long)y * (W + 1) + x;
        const T ul = u[iu], ur = u[iu + 1], vu = v[iv], vd = v[iv + W];
        const double div = ((dd(ur) - dd(ul)) + (dd(vd) - dd(vu))) / dx;
        if (!isfinite(div))
        {
            nonfinite = 1;
            continue;
        }
        const double rounding = (face_ulp(ul) + face_ulp(ur) + face_ulp(vu) + face_ulp(vd)) / dx;
        mx = fmax(mx, fabs(div));
        excess = fmax(excess, fmax(0.0, fabs(div) - rounding));
        sq += div * div;
    }
    __shared__ double4 total;
    const double4 mine = make_double4(mx, excess, sq, double(nonfinite));
    if (arrive_last<kVecThreads>(g, t.index, g.vec_tiles, block_reduce4<kVecThreads>(mine, 1 | 2 | 8), &total, 1 | 2 | 8))
    {
        if (threadIdx.x == 0)
        {
            SolveState& s = *g.state;
            s.nonfinite = total.w != 0.0;
            s.div_max = s.nonfinite ? INFINITY : total.x;
            s.div_excess = s.nonfinite ? INFINITY : total.y;
            s.div_sumsq = total.z;
        }
    }
}

// Converts FP64 host-layout fields into the device working type (upload) ...
template <typename T> __global__ void k_from_f64(const double* src, T* dst, long long n)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        dst[i] = T(src[i]);
}

// ... and back (download).
template <typename T> __global__ void k_to_f64(const T* src, double* dst, long long n)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        dst[i] = double(src[i]);
}

// Unpadded W x H FP64 field <-> padded FP64 field (pressure).
__global__ void k_pad_f64(const double* src, double* dst, int W, int H, int S)
{
    const long long n = (long long)W * H;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    {
        const int x = int(i % W), y = int(i / W);
        dst[padded_index(S, x, y)] = src[i];
    }
}

__global__ void k_unpad_f64(const double* src, double* dst, int W, int H, int S)
{
    const long long n = (long long)W * H;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    {
        const int x = int(i % W), y = int(i / W);
        dst[i] = src[padded_index(S, x, y)];
    }
}

template <typename T> __global__ void k_unpad_t(const void* src, double* dst, int W, int H, int S)
{
    const long long n = (long long)W * H;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    {
        const int x = int(i % W), y = int(i / W);
        dst[i] = double(static_cast<const T*>(src)[padded_index(S, x, y)]);
    }
}

template <typename T> __global__ void k_pad_t(const double* src, void* dst, int W, int H, int S)
{
    const long long n = (long long)W * H;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    {
        const int x = int(i % W), y = int(i / W);
        static_cast<T*>(dst)[padded_index(S, x, y)] = T(src[i]);
    }
}

} // namespace fc
