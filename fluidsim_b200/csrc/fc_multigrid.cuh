// Multigrid preconditioner of the UniformCUDA projection: one fixed V-cycle, z = M r.
//
// Same preconditioner as the reference PressureMultigrid (PressureMultigrid.cpp): levels
// halve (rounding up) until at most 64 cells remain; conductances combine in series/parallel;
// four red-black Gauss-Seidel sweeps before (the first from zero) and after (colours reversed)
// the coarse correction; transpose-bilinear restriction, bilinear prolongation; the coarsest
// level is solved directly with one cell pinned, then given a mean-zero gauge.
//
// B200 mapping:
//  * k_mg_pre / k_mg_post: temporally blocked smoothing. A 256-thread CTA stages a 64 x 8K
//    region of one level, keeps each cell's coefficients in registers (thread = two adjacent
//    columns of K rows) and the solution in shared memory split by colour, so a half-sweep is
//    four conflict-free shared loads per cell. All eight half-sweeps of a smoothing run on-chip;
//    the region's halo (10 cells for pre, 8 for post) absorbs the dependency cone. The pre kernel
//    fuses the residual and the restriction (writes the coarse rhs directly); the post kernel
//    fuses the prolongation, and on the fine level the mean and r.z reductions of z.
//  * k_mg_tail: the coarse levels that fit in shared memory are cycled by one CTA per grid,
//    including the coarsest direct solve (explicit FP64 inverse of the pinned Cholesky system).
#pragma once

#include "fc_device.cuh"

namespace fc
{

// Finishes a preconditioner application: z's mean, r.(z - mean z) and beta.
// FluidGridCPU.cpp:1712-1726 (applyPreconditioner) and :1806-1818 (beta, loop condition).
__device__ __forceinline__ void finish_preconditioner(SolveState& s, double sum_z, double sum_rz)
{
    const double mean_z = sum_z * s.inv_cells;
    const double rz = sum_rz - mean_z * s.sum_r;
    const double beta = s.restart ? 0.0 : rz / s.rz;
    s.mean_z = mean_z;
    s.beta = beta;
    s.restart = 0;
    s.rz = rz;
    if (!isfinite(beta) || !(rz > 0.0) || !isfinite(rz))
    {
        s.status = kStalled;
        s.done = 1;
    }
}

// Diagonal (Jacobi) preconditioner: z = (r - mean r) / diag. FluidGridCPU.cpp:1691-1698.
template <typename T>
__global__ void __launch_bounds__(kVecThreads) k_precondition_diagonal(const GridDesc* grids, const Tile* tiles)
{
    const Tile t = tiles[blockIdx.x];
    const GridDesc& g = grids[t.grid];
    SolveState& s = *g.state;
    if (s.done)
        return;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const T* right = static_cast<const T*>(g.lev[0].right);
    const T* down = static_cast<const T*>(g.lev[0].down);
    const T* r = static_cast<const T*>(g.r);
    T* z = static_cast<T*>(g.z);
    const double mean_r = s.mean_r;
    double sz = 0.0, srz = 0.0;
    for (int k = 0; k < 4; ++k)
    {
        const int x = t.x0 + tx, y = t.y0 + ty + 8 * k;
        if (x >= g.W || y >= g.H)
            continue;
        const long long i = padded_index(g.S, x, y);
        const double sum = ((double(right[i - 1]) + double(right[i])) + double(down[i - g.S])) + double(down[i]);
        const double inv = sum > 0.0 ? 1.0 / sum : 0.0;
        const T value = T((double(r[i]) - mean_r) * inv);
        z[i] = value;
        if (g.solid && g.solid[(long long)y * g.W + x])
            continue;
        sz += double(value);
        srz += double(r[i]) * double(value);
    }
    __shared__ double4 total;
    if (arrive_last<kVecThreads>(g, t.index, g.vec_tiles, block_reduce4<kVecThreads>(make_double4(sz, srz, 0, 0), 0), &total, 0))
    {
        if (threadIdx.x == 0)
            finish_preconditioner(s, total.x, total.y);
    }
}

// ------------------------------------------------------------------------------------------
// Rebuild: coarse conductances and the coarsest inverse
// ------------------------------------------------------------------------------------------

// Coarse level `level + 1` from `level`. PressureMultigrid.cpp:142-202 (coarsen) and
// :104-117 (the diagonal is recomputed on the fly wherever it is needed).
template <typename T> __global__ void k_coarsen(const GridDesc* grids, const Tile* tiles, int level)
{
    const Tile t = tiles[blockIdx.x];
    const GridDesc& g = grids[t.grid];
    const LevelDesc& f = g.lev[level];
    const LevelDesc& c = g.lev[level + 1];
    const T* fr = static_cast<const T*>(f.right);
    const T* fd = static_cast<const T*>(f.down);
    T* cr = static_cast<T*>(c.right);
    T* cd = static_cast<T*>(c.down);
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    for (int k = 0; k < 4; ++k)
    {
        const int x = t.x0 + tx, y = t.y0 + ty + 8 * k;
        if (x >= c.w || y >= c.h)
            continue;
        double right = 0.0, down = 0.0;
        if (x + 1 < c.w)
        {
            const int e = 2 * x + 2;
            const double a = (f.cx[e - 1] - c.cx[x]) / (f.cx[e - 1] - f.cx[e - 2]);
            const double b = e + 1 < f.w ? (c.cx[x + 1] - f.cx[e]) / (f.cx[e + 1] - f.cx[e]) : 0.0;
            const int fy_end = min(2 * y + 2, f.h);
            for (int fy = 2 * y; fy < fy_end; ++fy)
            {
                const long long i = padded_index(f.S, e - 1, fy); // fine cell 2x+1: its right face is the coarse face
                double resistance = a / double(fr[i - 1]) + 1.0 / double(fr[i]);
                if (b != 0.0)
                    resistance += b / double(fr[i + 1]);
                right += 1.0 / resistance;
            }
        }
        if (y + 1 < c.h)
        {
            const int e = 2 * y + 2;
            const double a = (f.cy[e - 1] - c.cy[y]) / (f.cy[e - 1] - f.cy[e - 2]);
            const double b = e + 1 < f.h ? (c.cy[y + 1] - f.cy[e]) / (f.cy[e + 1] - f.cy[e]) : 0.0;
            const int fx_end = min(2 * x + 2, f.w);
            for (int fx = 2 * x; fx < fx_end; ++fx)
            {
                const long long i = padded_index(f.S, fx, e - 1); // fine cell 2y+1: its lower face is the coarse face
                double resistance = a / double(fd[i - f.S]) + 1.0 / double(fd[i]);
                if (b != 0.0)
                    resistance += b / double(fd[i + f.S]);
                down += 1.0 / resistance;
            }
        }
        const long long ci = padded_index(c.S, x, y);
        cr[ci] = T(right);
        cd[ci] = T(down);
    }
}

// Dense pinned operator of the coarsest level, its Cholesky factor and the explicit inverse,
// in FP64; one CTA per grid. PressureMultigrid.cpp:300-345 (factorCoarsest). A non-positive
// or non-finite pivot marks the preconditioner invalid (the reference's breakdown, :334-335).
constexpr int kMaxCoarse = 64;

template <typename T> __global__ void __launch_bounds__(256) k_coarse_inverse(const GridDesc* grids)
{
    const GridDesc& g = grids[blockIdx.x];
    const int last = g.levels - 1;
    const LevelDesc& l = g.lev[last];
    const int cells = l.w * l.h;
    __shared__ double a[kMaxCoarse * kMaxCoarse];
    __shared__ int map[kMaxCoarse];
    __shared__ int failed, n_shared, pinned_shared;
    const T* right = static_cast<const T*>(l.right);
    const T* down = static_cast<const T*>(l.down);
    if (threadIdx.x == 0)
    {
        // Unknowns in cell order: open cells after the first one (pinned).
        int n = 0, pinned = -1;
        for (int cell = 0; cell < cells; ++cell)
        {
            const long long i = padded_index(l.S, cell % l.w, cell / l.w);
            const double diag = ((double(right[i - 1]) + double(right[i])) + double(down[i - l.S])) + double(down[i]);
            map[cell] = -1;
            if (!(diag > 0.0))
                continue;
            if (pinned < 0)
                pinned = cell;
            else
                map[cell] = n++;
        }
        failed = 0;
        n_shared = n;
        pinned_shared = pinned;
    }
    __syncthreads();
    const int n = n_shared;
    for (int i = threadIdx.x; i < n * n; i += blockDim.x)
        a[i] = 0.0;
    __syncthreads();
    for (int cell = threadIdx.x; cell < cells; cell += blockDim.x)
    {
        const int row = map[cell];
        if (row < 0)
            continue;
        const int x = cell % l.w, y = cell / l.w;
        const long long i = padded_index(l.S, x, y);
        a[row * n + row] = ((double(right[i - 1]) + double(right[i])) + double(down[i - l.S])) + double(down[i]);
        if (x > 0 && map[cell - 1] >= 0)
            a[row * n + map[cell - 1]] = -double(right[i - 1]);
        if (y > 0 && map[cell - l.w] >= 0)
            a[row * n + map[cell - l.w]] = -double(down[i - l.S]);
    }
    __syncthreads();
    // Cholesky of the lower triangle, column by column (same arithmetic as row by row).
    for (int col = 0; col < n; ++col)
    {
        if (threadIdx.x == 0)
        {
            double value = a[col * n + col];
            for (int k = 0; k < col; ++k)
                value -= a[col * n + k] * a[col * n + k];
            if (!(value > 0.0) || !isfinite(value))
                failed = 1;
            a[col * n + col] = sqrt(value);
        }
        __syncthreads();
        const double pivot = a[col * n + col];
        for (int row = col + 1 + threadIdx.x; row < n; row += blockDim.x)
        {
            double value = a[row * n + col];
            for (int k = 0; k < col; ++k)
                value -= a[row * n + k] * a[col * n + k];
            a[row * n + col] = value / pivot;
        }
        __syncthreads();
    }
    // inverse = L^-T L^-1, one column of the identity per thread.
    for (int c = threadIdx.x; c < n; c += blockDim.x)
    {
        double y[kMaxCoarse];
        for (int row = 0; row < n; ++row)
        {
            double value = row == c ? 1.0 : 0.0;
            for (int k = 0; k < row; ++k)
                value -= a[row * n + k] * y[k];
            y[row] = value / a[row * n + row];
        }
        for (int row = n - 1; row >= 0; --row)
        {
            double value = y[row];
            for (int k = row + 1; k < n; ++k)
                value -= a[k * n + row] * y[k];
            y[row] = value / a[row * n + row];
        }
        for (int row = 0; row < n; ++row)
            g.coarse_inverse[row * n + c] = y[row];
    }
    for (int cell = threadIdx.x; cell < kMaxCoarse; cell += blockDim.x)
        g.coarse->map[cell] = cell < cells ? map[cell] : -1;
    if (threadIdx.x == 0)
    {
        g.coarse->n = n;
        g.coarse->pinned = pinned_shared;
        g.coarse->open = pinned_shared < 0 ? 0 : n + 1;
        g.state->mg_valid = failed ? 0 : 1;
    }
}

// ------------------------------------------------------------------------------------------
// Temporally blocked red-black smoothing tiles
// ------------------------------------------------------------------------------------------

template <bool PRE> struct TileHalo
{
    // Pre: 8 half-sweeps (the first needs no neighbours) leave cells >= 7 from the region edge
    // exact; the residual needs 8 and the restriction stencil (fine cells 2C-1 .. 2C+2) 9;
    // rounded up to 10 to keep the region origin even. Post: 8 half-sweeps need 8.
    static constexpr int value = PRE ? 10 : 8;
};

template <typename T, int K, bool PRE> struct TileShape
{
    static constexpr int RX = 64;
    static constexpr int RY = 8 * K;
    static constexpr int HALO = TileHalo<PRE>::value;
    static constexpr int OX = RX - 2 * HALO;
    static constexpr int OY = RY - 2 * HALO;
};

// Per-thread cell coefficients: cell (row warp + 8k, colour c) of the region.
template <typename T, int K> struct TileCells
{
    T rhs[K][2];
    T wl[K][2], wr[K][2], wu[K][2], wd[K][2];
    T inv[K][2];
};

template <typename T, int K>
__device__ __forceinline__ void tile_half_sweep(T (&sol)[2][8 * K + 2][34], const TileCells<T, K>& cells, int colour,
    bool from_zero, int lane, int warp)
{
    const int other = colour ^ 1;
#pragma unroll
    for (int k = 0; k < K; ++k)
    {
        const int y = warp + 8 * k;
        const int s = (colour + y) & 1;
        T acc = cells.rhs[k][colour];
        if (!from_zero)
        {
            const T sl = sol[other][y + 1][lane + s];
            const T sr = sol[other][y + 1][lane + 1 + s];
            const T su = sol[other][y][lane + 1];
            const T sd = sol[other][y + 2][lane + 1];
            acc = acc + ((cells.wl[k][colour] * sl + cells.wr[k][colour] * sr) +
                            (cells.wu[k][colour] * su + cells.wd[k][colour] * sd));
        }
        sol[colour][y + 1][lane + 1] = acc * cells.inv[k][colour];
    }
    __syncthreads();
}

// Loads the region's coefficients (zero outside the level) into registers.
template <typename T, int K>
__device__ __forceinline__ void tile_load_cells(TileCells<T, K>& cells, const GridDesc& g, const LevelDesc& L,
    int level, int X0, int Y0, int lane, int warp, double mean_r)
{
    const T* right = static_cast<const T*>(L.right);
    const T* down = static_cast<const T*>(L.down);
    const T* rhs = level == 0 ? static_cast<const T*>(g.r) : static_cast<const T*>(L.rhs);
#pragma unroll
    for (int k = 0; k < K; ++k)
    {
#pragma unroll
        for (int c = 0; c < 2; ++c)
        {
            const int y = warp + 8 * k;
            const int x = 2 * lane + ((c + y) & 1);
            const int gx = X0 + x, gy = Y0 + y;
            T b = T(0), wl = T(0), wr = T(0), wu = T(0), wd = T(0), inv = T(0);
            if (gx >= 0 && gx < L.w && gy >= 0 && gy < L.h)
            {
                const long long i = padded_index(L.S, gx, gy);
                wl = right[i - 1];
                wr = right[i];
                wu = down[i - L.S];
                wd = down[i];
                const T diag = ((wl + wr) + wu) + wd;
                inv = diag > T(0) ? T(1) / diag : T(0);
                // A cell without an open face takes no part (rhs 0): inside obstacles, or a 1x1 grid.
                b = diag > T(0) ? (level == 0 ? T(double(rhs[i]) - mean_r) : rhs[i]) : T(0);
            }
            cells.rhs[k][c] = b;
            cells.wl[k][c] = wl;
            cells.wr[k][c] = wr;
            cells.wu[k][c] = wu;
            cells.wd[k][c] = wd;
            cells.inv[k][c] = inv;
        }
    }
}

// Pre-smoothing (4 sweeps, the first from zero), residual and restriction of one tile.
// PressureMultigrid.cpp:398-402 (cycle), :204-231 (smooth), :233-276 (restrictResidual).
template <typename T, int K>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 2 : 1) k_mg_pre(const GridDesc* grids, const Tile* tiles, int level)
{
    using Shape = TileShape<T, K, true>;
    const Tile t = tiles[blockIdx.x];
    const GridDesc& g = grids[t.grid];
    if (g.state->done)
        return;
    const LevelDesc& L = g.lev[level];
    const LevelDesc& C = g.lev[level + 1];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int X0 = t.x0 - Shape::HALO, Y0 = t.y0 - Shape::HALO;

    __shared__ T sol[2][Shape::RY + 2][34];
    for (int i = threadIdx.x; i < 2 * (Shape::RY + 2) * 34; i += 256)
        (&sol[0][0][0])[i] = T(0);

    TileCells<T, K> cells;
    tile_load_cells<T, K>(cells, g, L, level, X0, Y0, lane, warp, level == 0 ? g.state->mean_r : 0.0);
    __syncthreads();

    tile_half_sweep<T, K>(sol, cells, 0, true, lane, warp);
    tile_half_sweep<T, K>(sol, cells, 1, false, lane, warp);
#pragma unroll 1
    for (int sweep = 1; sweep < 4; ++sweep)
    {
        tile_half_sweep<T, K>(sol, cells, 0, false, lane, warp);
        tile_half_sweep<T, K>(sol, cells, 1, false, lane, warp);
    }

    // Residual of every owned cell, and the pre-smoothed solution of the tile's output cells.
    T* pre = static_cast<T*>(L.pre);
    T res[K][2];
#pragma unroll
    for (int k = 0; k < K; ++k)
    {
#pragma unroll
        for (int c = 0; c < 2; ++c)
        {
            const int y = warp + 8 * k;
            const int s = (c + y) & 1;
            const int other = c ^ 1;
            const T center = sol[c][y + 1][lane + 1];
            const T sl = sol[other][y + 1][lane + s];
            const T sr = sol[other][y + 1][lane + 1 + s];
            const T su = sol[other][y][lane + 1];
            const T sd = sol[other][y + 2][lane + 1];
            const T product = (cells.wl[k][c] * (center - sl) + cells.wr[k][c] * (center - sr)) +
                              (cells.wu[k][c] * (center - su) + cells.wd[k][c] * (center - sd));
            res[k][c] = cells.rhs[k][c] - product;
            const int x = 2 * lane + s;
            const int gx = X0 + x, gy = Y0 + y;
            if (x >= Shape::HALO && x < Shape::HALO + Shape::OX && y >= Shape::HALO && y < Shape::HALO + Shape::OY &&
                gx < L.w && gy < L.h)
                pre[padded_index(L.S, gx, gy)] = center;
        }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < K; ++k)
    {
#pragma unroll
        for (int c = 0; c < 2; ++c)
            sol[c][warp + 8 * k + 1][lane + 1] = res[k][c];
    }
    __syncthreads();

    // Transpose-bilinear restriction onto the tile's coarse cells.
    T* crhs = static_cast<T*>(C.rhs);
    constexpr int OCX = Shape::OX / 2, OCY = Shape::OY / 2;
    const int cx0 = t.x0 / 2, cy0 = t.y0 / 2;
    for (int q = threadIdx.x; q < OCX * OCY; q += 256)
    {
        const int cx = cx0 + q % OCX, cy = cy0 + q / OCX;
        if (cx >= C.w || cy >= C.h)
            continue;
        const Gather gx = L.rx[cx];
        const Gather gy = L.ry[cy];
        double value = 0.0;
        for (int iy = 0; iy < gy.count; ++iy)
        {
            const int y = gy.index[iy] - Y0;
            double line = 0.0;
            for (int ix = 0; ix < gx.count; ++ix)
            {
                const int x = gx.index[ix] - X0;
                line += gx.weight[ix] * double(sol[(x + y) & 1][y + 1][(x >> 1) + 1]);
            }
            value += gy.weight[iy] * line;
        }
        crhs[padded_index(C.S, cx, cy)] = T(value);
    }
}

// Prolongation of the coarse correction, then 4 sweeps in reversed colour order; on the fine
// level also sum(z) and sum(r z). PressureMultigrid.cpp:403-407 (cycle), :278-298
// (prolongCorrection); FluidGridCPU.cpp:1712-1726 (z mean and r.z).
template <typename T, int K>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 2 : 1) k_mg_post(const GridDesc* grids, const Tile* tiles, int level)
{
    using Shape = TileShape<T, K, false>;
    const Tile t = tiles[blockIdx.x];
    const GridDesc& g = grids[t.grid];
    SolveState& state = *g.state;
    if (state.done)
        return;
    const LevelDesc& L = g.lev[level];
    const LevelDesc& C = g.lev[level + 1];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int X0 = t.x0 - Shape::HALO, Y0 = t.y0 - Shape::HALO;

    __shared__ T sol[2][Shape::RY + 2][34];
    for (int i = threadIdx.x; i < 2 * (Shape::RY + 2) * 34; i += 256)
        (&sol[0][0][0])[i] = T(0);

    TileCells<T, K> cells;
    tile_load_cells<T, K>(cells, g, L, level, X0, Y0, lane, warp, level == 0 ? state.mean_r : 0.0);
    __syncthreads();

    const T* pre = static_cast<const T*>(L.pre);
    const T* coarse = static_cast<const T*>(C.sol);
#pragma unroll
    for (int k = 0; k < K; ++k)
    {
#pragma unroll
        for (int c = 0; c < 2; ++c)
        {
            const int y = warp + 8 * k;
            const int x = 2 * lane + ((c + y) & 1);
            const int gx = X0 + x, gy = Y0 + y;
            if (gx < 0 || gx >= L.w || gy < 0 || gy >= L.h)
                continue;
            const Interp px = L.px[gx];
            const Interp py = L.py[gy];
            const long long top = padded_index(C.S, 0, py.first);
            const long long bottom = padded_index(C.S, 0, py.second);
            const double a = (1.0 - px.weight) * double(coarse[top + px.first]) + px.weight * double(coarse[top + px.second]);
            const double b =
                (1.0 - px.weight) * double(coarse[bottom + px.first]) + px.weight * double(coarse[bottom + px.second]);
            const double value = double(pre[padded_index(L.S, gx, gy)]) + ((1.0 - py.weight) * a + py.weight * b);
            sol[c][y + 1][lane + 1] = T(value);
        }
    }
    __syncthreads();

#pragma unroll 1
    for (int sweep = 0; sweep < 4; ++sweep)
    {
        tile_half_sweep<T, K>(sol, cells, 1, false, lane, warp);
        tile_half_sweep<T, K>(sol, cells, 0, false, lane, warp);
    }

    T* out = static_cast<T*>(L.sol);
    const T* r = static_cast<const T*>(g.r);
    double sz = 0.0, srz = 0.0;
#pragma unroll
    for (int k = 0; k < K; ++k)
    {
#pragma unroll
        for (int c = 0; c < 2; ++c)
        {
            const int y = warp + 8 * k;
            const int x = 2 * lane + ((c + y) & 1);
            const int gx = X0 + x, gy = Y0 + y;
            if (x < Shape::HALO || x >= Shape::HALO + Shape::OX || y < Shape::HALO || y >= Shape::HALO + Shape::OY ||
                gx >= L.w || gy >= L.h)
                continue;
            const long long i = padded_index(L.S, gx, gy);
            const T value = sol[c][y + 1][lane + 1];
            out[i] = value;
            if (level == 0 && !(g.solid && g.solid[(long long)gy * g.W + gx]))
            {
                sz += double(value);
                srz += double(r[i]) * double(value);
            }
        }
    }
    if (level != 0)
        return;
    __shared__ double4 total;
    if (arrive_last<256>(g, t.index, g.post_tiles, block_reduce4<256>(make_double4(sz, srz, 0, 0), 0), &total, 0))
    {
        if (threadIdx.x == 0)
            finish_preconditioner(state, total.x, total.y);
    }
}

// ------------------------------------------------------------------------------------------
// Coarse tail: the remaining levels cycled by one CTA in shared memory
// ------------------------------------------------------------------------------------------

constexpr int kTailThreads = 512;

template <typename T> struct TailLevel
{
    int w, h, s; // s = w + 2, one zero halo cell
    T *right, *down, *inv, *rhs, *sol, *res;
    __device__ int at(int x, int y) const { return (y + 1) * s + x + 1; }
};

// Shared-memory bytes of the tail of a grid starting at `first` (host and device agree).
__host__ __device__ inline size_t tail_bytes(const int* w, const int* h, int first, int levels, size_t elem)
{
    size_t cells = 0;
    for (int l = first; l < levels; ++l)
        cells += size_t(w[l] + 2) * (h[l] + 2);
    return cells * 6 * elem + 2 * kMaxCoarse * sizeof(double) + 64;
}

template <typename T> __device__ void tail_smooth(const TailLevel<T>& L, bool reverse, bool from_zero)
{
    const int half = (L.w + 1) / 2;
    for (int pass = 0; pass < 2; ++pass)
    {
        const int colour = reverse ? 1 - pass : pass;
        for (int q = threadIdx.x; q < half * L.h; q += blockDim.x)
        {
            const int y = q / half;
            const int x = 2 * (q % half) + ((colour + y) & 1);
            if (x >= L.w)
                continue;
            const int i = L.at(x, y);
            T value = L.rhs[i];
            if (!(from_zero && pass == 0))
                value = value + ((L.right[i - 1] * L.sol[i - 1] + L.right[i] * L.sol[i + 1]) +
                                    (L.down[i - L.s] * L.sol[i - L.s] + L.down[i] * L.sol[i + L.s]));
            L.sol[i] = value * L.inv[i];
        }
        __syncthreads();
    }
}

template <typename T>
__device__ void tail_restrict(const TailLevel<T>& F, const TailLevel<T>& Cl, const LevelDesc& fine_desc)
{
    for (int q = threadIdx.x; q < F.w * F.h; q += blockDim.x)
    {
        const int x = q % F.w, y = q / F.w;
        const int i = F.at(x, y);
        const T center = F.sol[i];
        const T product = (F.right[i - 1] * (center - F.sol[i - 1]) + F.right[i] * (center - F.sol[i + 1])) +
                          (F.down[i - F.s] * (center - F.sol[i - F.s]) + F.down[i] * (center - F.sol[i + F.s]));
        // Cells without an open face pass no residual down (keeps the cycle symmetric).
        F.res[i] = F.inv[i] > T(0) ? F.rhs[i] - product : T(0);
    }
    __syncthreads();
    for (int q = threadIdx.x; q < Cl.w * Cl.h; q += blockDim.x)
    {
        const int cx = q % Cl.w, cy = q / Cl.w;
        const Gather gx = fine_desc.rx[cx];
        const Gather gy = fine_desc.ry[cy];
        double value = 0.0;
        for (int iy = 0; iy < gy.count; ++iy)
        {
            double line = 0.0;
            for (int ix = 0; ix < gx.count; ++ix)
                line += gx.weight[ix] * double(F.res[F.at(gx.index[ix], gy.index[iy])]);
            value += gy.weight[iy] * line;
        }
        Cl.rhs[Cl.at(cx, cy)] = T(value);
    }
    __syncthreads();
}

template <typename T>
__device__ void tail_prolong(const TailLevel<T>& Cl, const TailLevel<T>& F, const LevelDesc& fine_desc)
{
    for (int q = threadIdx.x; q < F.w * F.h; q += blockDim.x)
    {
        const int x = q % F.w, y = q / F.w;
        const Interp px = fine_desc.px[x];
        const Interp py = fine_desc.py[y];
        const double a = (1.0 - px.weight) * double(Cl.sol[Cl.at(px.first, py.first)]) +
                         px.weight * double(Cl.sol[Cl.at(px.second, py.first)]);
        const double b = (1.0 - px.weight) * double(Cl.sol[Cl.at(px.first, py.second)]) +
                         px.weight * double(Cl.sol[Cl.at(px.second, py.second)]);
        const int i = F.at(x, y);
        F.sol[i] = T(double(F.sol[i]) + ((1.0 - py.weight) * a + py.weight * b));
    }
    __syncthreads();
}

// Mean-free rhs, explicit inverse, mean-zero gauge over the open cells.
// PressureMultigrid.cpp:347-384 (solveCoarsest).
template <typename T>
__device__ void tail_solve_coarsest(const TailLevel<T>& L, const double* inverse, const CoarseInfo& info, double* b,
    double* z)
{
    __shared__ double mean_shared;
    const int cells = L.w * L.h, n = info.n;
    double part = 0.0;
    for (int q = threadIdx.x; q < cells; q += blockDim.x)
        if (q == info.pinned || info.map[q] >= 0)
            part += double(L.rhs[L.at(q % L.w, q / L.w)]);
    const double4 total = block_reduce4<kTailThreads>(make_double4(part, 0, 0, 0), 0);
    if (threadIdx.x == 0)
        mean_shared = info.open > 0 ? total.x / info.open : 0.0;
    __syncthreads();
    const double mean = mean_shared;
    for (int q = threadIdx.x; q < cells; q += blockDim.x)
    {
        const int k = info.map[q];
        if (k >= 0)
            b[k] = double(L.rhs[L.at(q % L.w, q / L.w)]) - mean;
    }
    __syncthreads();
    for (int row = threadIdx.x; row < n; row += blockDim.x)
    {
        double value = 0.0;
        for (int col = 0; col < n; ++col)
            value += inverse[row * n + col] * b[col];
        z[row] = value;
    }
    __syncthreads();
    double zpart = 0.0;
    for (int k = threadIdx.x; k < n; k += blockDim.x)
        zpart += z[k];
    const double4 ztotal = block_reduce4<kTailThreads>(make_double4(zpart, 0, 0, 0), 0);
    if (threadIdx.x == 0)
        mean_shared = info.open > 0 ? ztotal.x / info.open : 0.0;
    __syncthreads();
    const double zmean = mean_shared;
    for (int q = threadIdx.x; q < cells; q += blockDim.x)
    {
        const int k = info.map[q];
        double value = 0.0;
        if (k >= 0)
            value = z[k] - zmean;
        else if (q == info.pinned)
            value = -zmean;
        L.sol[L.at(q % L.w, q / L.w)] = T(value);
    }
    __syncthreads();
}

template <typename T> __global__ void __launch_bounds__(kTailThreads) k_mg_tail(const GridDesc* grids)
{
    const GridDesc& g = grids[blockIdx.x];
    SolveState& state = *g.state;
    if (state.done)
        return;
    extern __shared__ __align__(16) unsigned char tail_smem[];
    const int first = g.tail, last = g.levels - 1;
    TailLevel<T> lv[kMaxLevels];
    size_t offset = 0;
    T* base = reinterpret_cast<T*>(tail_smem);
    for (int l = first; l <= last; ++l)
    {
        TailLevel<T>& L = lv[l];
        L.w = g.lev[l].w;
        L.h = g.lev[l].h;
        L.s = L.w + 2;
        const size_t cells = size_t(L.s) * (L.h + 2);
        T** arrays[6] = {&L.right, &L.down, &L.inv, &L.rhs, &L.sol, &L.res};
        for (int a = 0; a < 6; ++a)
        {
            *arrays[a] = base + offset;
            offset += cells;
        }
    }
    double* b = reinterpret_cast<double*>(tail_smem + ((offset * sizeof(T) + 15) / 16) * 16);
    double* z = b + kMaxCoarse;
    for (size_t i = threadIdx.x; i < offset; i += blockDim.x)
        base[i] = T(0);
    __syncthreads();

    // Coefficients of every tail level and the first level's right-hand side.
    const double mean_r = first == 0 ? state.mean_r : 0.0;
    for (int l = first; l <= last; ++l)
    {
        const TailLevel<T>& L = lv[l];
        const LevelDesc& D = g.lev[l];
        const T* right = static_cast<const T*>(D.right);
        const T* down = static_cast<const T*>(D.down);
        const T* rhs = first == 0 ? static_cast<const T*>(g.r) : static_cast<const T*>(D.rhs);
        for (int q = threadIdx.x; q < L.w * L.h; q += blockDim.x)
        {
            const int x = q % L.w, y = q / L.w;
            const long long i = padded_index(D.S, x, y);
            const int j = L.at(x, y);
            L.right[j] = right[i];
            L.down[j] = down[i];
            if (l == first)
                L.rhs[j] = first == 0 ? T(double(rhs[i]) - mean_r) : rhs[i];
        }
    }
    __syncthreads();
    for (int l = first; l <= last; ++l)
    {
        const TailLevel<T>& L = lv[l];
        for (int q = threadIdx.x; q < L.w * L.h; q += blockDim.x)
        {
            const int j = L.at(q % L.w, q / L.w);
            const T diag = ((L.right[j - 1] + L.right[j]) + L.down[j - L.s]) + L.down[j];
            L.inv[j] = diag > T(0) ? T(1) / diag : T(0);
            if (l == first && !(diag > T(0)))
                L.rhs[j] = T(0);
        }
    }
    __syncthreads();

    for (int l = first; l < last; ++l)
    {
        tail_smooth(lv[l], false, true);
        for (int sweep = 1; sweep < 4; ++sweep)
            tail_smooth(lv[l], false, false);
        tail_restrict(lv[l], lv[l + 1], g.lev[l]);
    }
    tail_solve_coarsest(lv[last], g.coarse_inverse, *g.coarse, b, z);
    for (int l = last - 1; l >= first; --l)
    {
        tail_prolong(lv[l + 1], lv[l], g.lev[l]);
        for (int sweep = 0; sweep < 4; ++sweep)
            tail_smooth(lv[l], true, false);
    }

    // Hand the first tail level's solution to the finer post-smoothing (or to z).
    const TailLevel<T>& F = lv[first];
    const LevelDesc& D = g.lev[first];
    T* out = static_cast<T*>(D.sol);
    const T* r = static_cast<const T*>(g.r);
    double sz = 0.0, srz = 0.0;
    for (int q = threadIdx.x; q < F.w * F.h; q += blockDim.x)
    {
        const int x = q % F.w, y = q / F.w;
        const long long i = padded_index(D.S, x, y);
        const T value = F.sol[F.at(x, y)];
        out[i] = value;
        if (first == 0 && !(g.solid && g.solid[(long long)y * g.W + x]))
        {
            sz += double(value);
            srz += double(r[i]) * double(value);
        }
    }
    if (first != 0)
        return;
    const double4 total = block_reduce4<kTailThreads>(make_double4(sz, srz, 0, 0), 0);
    if (threadIdx.x == 0)
        finish_preconditioner(state, total.x, total.y);
}

} // namespace fc
