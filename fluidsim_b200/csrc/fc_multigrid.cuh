// Multigrid preconditioner of the UniformCUDA projection: one fixed V-cycle, z = M r.
//
// Same preconditioner as the reference PressureMultigrid (PressureMultigrid.cpp): levels
// halve (rounding up) until at most 64 cells remain; conductances combine in series/parallel;
// four red-black Gauss-Seidel sweeps before (the first from zero) and after (colours reversed)
// the coarse correction; transpose-bilinear restriction, bilinear prolongation; the coarsest
// level is solved directly with one cell pinned, then given a mean-zero gauge.
//
// B200 mapping:
//  * k_smooth_pre / k_smooth_post (fc_stage.cuh): temporally blocked smoothing of one level per launch,
//    with the residual and restriction fused into the pre kernel and the prolongation and the
//    fine-level z reductions fused into the post kernel.
//  * k_mg_tail: the coarse levels of at most 64 x 64 cells that fit in shared memory are cycled
//    by one CTA per grid as register strips, their inputs bulk-copied in before the dependency
//    wait, including the coarsest direct solve (explicit FP64 inverse of the pinned Cholesky
//    system).
//  * The rebuild: k_coarsen (one coarse cell per thread), k_inverse_diagonal, k_weights_half
//    (mixed precision) and k_coarse_inverse (right-looking factor, the reference's arithmetic).
#pragma once

#include "fc_device.cuh"
#include "fc_smooth.cuh"
#include "fc_tma.cuh"

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
    allow_dependents();
    const Tile t = tiles[blockIdx.x];
    const GridDesc& g = grids[t.grid];
    SolveState& s = *g.state;
    dependency_wait();
    if (s.done)
        return;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const T* right = static_cast<const T*>(g.lev[0].right);
    const T* down = static_cast<const T*>(g.lev[0].down);
    const T* r = static_cast<const T*>(g.r);
    T* z = static_cast<T*>(g.z);
    const double mean_r = s.mean_r;
    double sz = 0.0, srz = 0.0;
    for (int k = 0; k < kVecCells; ++k)
    {
        const int x = t.x0 + tx + 32 * (k & 1), y = t.y0 + ty + 8 * (k >> 1);
        if (x >= g.W || y >= g.H)
            continue;
        const long long i = padded_index(g.S, x, y);
        const double sum = ((double(right[i - 1]) + double(right[i])) + double(down[i - g.S])) + double(down[i]);
        const double inv = sum > 0.0 ? 1.0 / sum : 0.0;
        const T value = g.air && g.air[(long long)y * g.W + x] ? T(0) : T((double(r[i]) - mean_r) * inv);
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

// Mixed precision: FP16 copies of a level's face weights for the strip kernels, divided by
// the level's scale and saturated at the largest finite FP16 value (blockIdx.y = grid).
__global__ void k_weights_half(const GridDesc* __restrict__ grids, int level)
{
    dependent_start();
    const GridDesc& g = grids[blockIdx.y];
    if (level < 1 || level >= g.tail)
        return;
    const LevelDesc& L = g.lev[level];
    const int n = L.S * (L.h + 2);
    const float inv = 1.0f / L.wscale;
    const float* right = static_cast<const float*>(L.right);
    const float* down = static_cast<const float*>(L.down);
    __half* rh = static_cast<__half*>(const_cast<void*>(L.right_h));
    __half* dh = static_cast<__half*>(const_cast<void*>(L.down_h));
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    {
        rh[i] = __float2half_rn(fminf(right[i] * inv, 65504.0f));
        dh[i] = __float2half_rn(fminf(down[i] * inv, 65504.0f));
    }
}

// Dirichlet air (no reference counterpart): a cell held at zero. On the fine level the air
// cells; on a coarse level the cells none of whose fine cells (2x .. 2x+1, 2y .. 2y+1 of the
// level above, whose inverse diagonal is final) is an unknown. A held cell keeps its face
// weights, so the unknowns beside it see the zero: the p = 0 boundary on every level.
template <typename T> __device__ __forceinline__ bool held_cell(const GridDesc& g, int level, int x, int y)
{
    if (level == 0)
        return g.air[(long long)y * g.W + x] != 0;
    const LevelDesc& F = g.lev[level - 1];
    const T* inv = static_cast<const T*>(F.inv);
    for (int dy = 0; dy < 2; ++dy)
        for (int dx = 0; dx < 2; ++dx)
        {
            const int fx = 2 * x + dx, fy = 2 * y + dy;
            if (fx < F.w && fy < F.h && inv[padded_index(F.S, fx, fy)] > T(0))
                return false;
        }
    return true;
}

// Inverse diagonal of a level the strip kernels smooth (blockIdx.y = grid): for each cell
// 1 / (((left + right) + up) + down) over its face weights, decoded as the kernels decode them
// (the FP16 copies times the level scale on mixed-precision coarse levels), 0 where the sum is
// not positive and in the padding. The kernels formed it per region before; the sum and the
// reciprocal are the same, so the smoothing is unchanged (PressureMultigrid.cpp:104-117).
template <typename T> __global__ void k_inverse_diagonal(const GridDesc* __restrict__ grids, int level)
{
    dependent_start();
    const GridDesc& g = grids[blockIdx.y];
    if (level + 1 >= g.levels)
        return;
    const LevelDesc& L = g.lev[level];
    const int n = L.S * (L.h + 2);
    T* inv = static_cast<T*>(L.inv);
    bool half = false;
    if constexpr (sizeof(T) == 4)
        half = L.right_h != nullptr && level >= 1 && level < g.tail;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    {
        const int x = i % L.S - kPadX, y = i / L.S - 1;
        T value = T(0);
        if (x >= 0 && x < L.w && y >= 0 && y < L.h)
        {
            T wl, wr, wu, wd;
            if constexpr (sizeof(T) == 4)
            {
                if (half)
                {
                    const __half* rh = static_cast<const __half*>(L.right_h);
                    const __half* dh = static_cast<const __half*>(L.down_h);
                    wl = __half2float(rh[i - 1]) * L.wscale;
                    wr = __half2float(rh[i]) * L.wscale;
                    wu = __half2float(dh[i - L.S]) * L.wscale;
                    wd = __half2float(dh[i]) * L.wscale;
                }
            }
            if (!half)
            {
                const T* right = static_cast<const T*>(L.right);
                const T* down = static_cast<const T*>(L.down);
                wl = right[i - 1];
                wr = right[i];
                wu = down[i - L.S];
                wd = down[i];
            }
            const T diag = ((wl + wr) + wu) + wd;
            value = diag > T(0) ? reciprocal(diag) : T(0);
            if (g.air && held_cell<T>(g, level, x, y))
                value = T(0);
        }
        inv[i] = value;
    }
}

// Coarse level `level + 1` from `level`. PressureMultigrid.cpp:142-202 (coarsen) and
// :104-117 (the diagonal is recomputed on the fly wherever it is needed).
// One thread per coarse cell (blockIdx.y = grid): the FP64 divisions of a cell form a long
// dependent chain, so the kernel needs many cells in flight rather than many cells per thread.
template <typename T> __global__ void k_coarsen(const GridDesc* __restrict__ grids, int level)
{
    dependent_start();
    const GridDesc& g = grids[blockIdx.y];
    if (level + 1 >= g.levels)
        return;
    const LevelDesc& f = g.lev[level];
    const LevelDesc& c = g.lev[level + 1];
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= c.w * c.h)
        return;
    const int x = q % c.w, y = q / c.w;
    const T* fr = static_cast<const T*>(f.right);
    const T* fd = static_cast<const T*>(f.down);
    T* cr = static_cast<T*>(c.right);
    T* cd = static_cast<T*>(c.down);
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

// Dense pinned operator of the coarsest level, its Cholesky factor and the explicit inverse,
// in FP64; one CTA per grid. PressureMultigrid.cpp:300-345 (factorCoarsest). A non-positive
// or non-finite pivot marks the preconditioner invalid (the reference's breakdown, :334-335).
//
// The factor is formed right-looking: every entry receives the same subtractions in the same
// order as the reference's column-by-column loop (products of columns 0, 1, ... in turn, then
// the division by the pivot), so it is the same factor bit for bit, with the work of each step
// spread over the CTA. Y = L^-1 by forward substitution (likewise right-looking, each entry
// keeping the left-looking order), and the inverse A^-1 = Y^T Y as independent dot products.
constexpr int kMaxCoarse = 64;
constexpr int kCoarseThreads = 512;
// Dynamic shared memory: the factor L and Y, n x n doubles each.
constexpr size_t kCoarseInverseSmem = 2 * size_t(kMaxCoarse) * kMaxCoarse * sizeof(double);

template <typename T> __global__ void __launch_bounds__(kCoarseThreads) k_coarse_inverse(const GridDesc* grids)
{
    dependent_start();
    const GridDesc& g = grids[blockIdx.x];
    const int last = g.levels - 1;
    const LevelDesc& l = g.lev[last];
    const int cells = l.w * l.h;
    extern __shared__ double coarse_smem[];
    double* a = coarse_smem;                         // operator, then its factor (lower triangle)
    double* yi = coarse_smem + kMaxCoarse * kMaxCoarse; // L^-1 (lower triangle)
    __shared__ int map[kMaxCoarse];
    __shared__ unsigned char open[kMaxCoarse];
    __shared__ int failed, n_shared, pinned_shared;
    const T* right = static_cast<const T*>(l.right);
    const T* down = static_cast<const T*>(l.down);
    // Unknowns in cell order: open cells after the first one (pinned). The cells' diagonals
    // are read in parallel, the numbering is one pass over the flags.
    const bool dirichlet = g.air != nullptr;
    for (int cell = threadIdx.x; cell < cells; cell += blockDim.x)
    {
        const long long i = padded_index(l.S, cell % l.w, cell / l.w);
        const double diag = ((double(right[i - 1]) + double(right[i])) + double(down[i - l.S])) + double(down[i]);
        open[cell] = diag > 0.0 && !(dirichlet && held_cell<T>(g, last, cell % l.w, cell / l.w)) ? 1 : 0;
    }
    __syncthreads();
    if (threadIdx.x == 0)
    {
        int n = 0, pinned = -1;
        for (int cell = 0; cell < cells; ++cell)
        {
            map[cell] = -1;
            if (!open[cell])
                continue;
            // Dirichlet air makes the system non-singular: nothing is pinned.
            if (pinned < 0 && !dirichlet)
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
    {
        a[i] = 0.0;
        yi[i] = (i / n == i % n) ? 1.0 : 0.0;
    }
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
    // Cholesky, right-looking: at step k the pivot and column k are final; the trailing lower
    // triangle then takes its k-th product. Every thread forms the pivot itself (the same
    // correctly rounded square root), so a step needs two barriers: one after the column is
    // scaled, one after the trailing update. The threads cover the trailing triangle as rows of
    // 64 columns (kMaxCoarse), 512 / 64 rows at a time, with no index divisions; each entry takes
    // the same operations in the same order as in the reference's column loop.
    //
    // Y = L^-1 by right-looking forward substitution runs in the same steps: row k of Y has all
    // its products once step k starts (steps j < k gave them), takes its division by the pivot
    // with column k's scaling, and the rows below take its product with the trailing update.
    // Each entry of L and Y sees the same operations in the same order as in two separate loops.
    constexpr int kCols = kMaxCoarse, kRows = kCoarseThreads / kMaxCoarse;
    const int trow = threadIdx.x / kCols, tcol = threadIdx.x % kCols;
    for (int k = 0; k < n; ++k)
    {
        const double value = a[k * n + k];
        const double pivot = sqrt(value);
        if (threadIdx.x == 0 && (!(value > 0.0) || !isfinite(value)))
            failed = 1;
        for (int row = k + 1 + threadIdx.x; row < n; row += blockDim.x)
            a[row * n + k] = a[row * n + k] / pivot;
        // Y's row k on other threads than column k's scaling (those with index >= kMaxCoarse).
        for (int col = int(threadIdx.x) - kMaxCoarse; col >= 0 && col <= k; col += blockDim.x - kMaxCoarse)
            yi[k * n + col] = yi[k * n + col] / pivot;
        __syncthreads();
        if (threadIdx.x == 0)
            a[k * n + k] = pivot;
        const int col = k + 1 + tcol;
        for (int row = k + 1 + trow; row < n; row += kRows)
            if (col <= row)
                a[row * n + col] -= a[row * n + k] * a[col * n + k];
        if (tcol <= k)
            for (int row = k + 1 + trow; row < n; row += kRows)
                yi[row * n + tcol] -= a[row * n + k] * yi[k * n + tcol];
        __syncthreads();
    }
    // A^-1 = Y^T Y: entry (r, c) sums Y[k][r] Y[k][c] over k >= max(r, c).
    for (int e = threadIdx.x; e < n * n; e += blockDim.x)
    {
        const int r = e / n, c = e % n;
        double value = 0.0;
        for (int k = max(r, c); k < n; ++k)
            value += yi[k * n + r] * yi[k * n + c];
        g.coarse_inverse[e] = value;
    }
    for (int cell = threadIdx.x; cell < kMaxCoarse; cell += blockDim.x)
        g.coarse->map[cell] = cell < cells ? map[cell] : -1;
    if (threadIdx.x == 0)
    {
        g.coarse->n = n;
        g.coarse->pinned = pinned_shared;
        g.coarse->open = dirichlet ? n : (pinned_shared < 0 ? 0 : n + 1);
        g.coarse->dirichlet = dirichlet ? 1 : 0;
        g.state->mg_valid = failed ? 0 : 1;
    }
}

// ------------------------------------------------------------------------------------------
// Coarse tail: the remaining levels cycled by one CTA in shared memory
// ------------------------------------------------------------------------------------------

constexpr int kTailThreads = 1024;
constexpr int kTailWarps = kTailThreads / 32;

// Dynamic shared memory of the tail kernel. Levels address it through element offsets so that
// every access is a shared-memory access.
extern __shared__ __align__(16) unsigned char tail_smem[];

// A tail level in shared memory: its arrays keep the global padded layout (stride s = the
// level's padded stride, halo row and columns of zeros), so that whole arrays arrive by bulk copy.
template <typename T> struct TailLevel
{
    int w, h, s;
    int right, down, inv, rhs, sol, res; // element offsets of the level's arrays
    int px, py, rx, ry;               // byte offsets of the transfer tables
    __device__ int at(int x, int y) const { return (y + 1) * s + x + kPadX; }
};

template <typename T> __device__ __forceinline__ T* tail_array() { return reinterpret_cast<T*>(tail_smem); }
template <typename E> __device__ __forceinline__ E* tail_table(int offset)
{
    return reinterpret_cast<E*>(tail_smem + offset);
}

__host__ __device__ inline size_t align16(size_t n) { return (n + 15) / 16 * 16; }
__host__ __device__ inline int padded_index32_tail(int S, int x, int y) { return (y + 1) * S + x + kPadX; }

// Shared-memory layout of the tail of a grid starting at level `first` (host and device
// agree): per level six padded arrays, then per smoothed level its four transfer tables (each
// 16-byte aligned), then the coarsest inverse and two vectors of the coarsest solve.
__host__ __device__ inline size_t tail_bytes(const int* w, const int* h, int first, int levels, size_t elem)
{
    size_t bytes = 0;
    for (int l = first; l < levels; ++l)
        bytes += align16(size_t(padded_stride(w[l])) * (h[l] + 2) * 6 * elem);
    for (int l = first; l + 1 < levels; ++l)
        bytes += align16(w[l] * sizeof(Interp)) + align16(h[l] * sizeof(Interp)) + align16(w[l + 1] * sizeof(Gather)) +
                 align16(h[l + 1] * sizeof(Gather));
    bytes += align16(size_t(kMaxCoarse) * kMaxCoarse * sizeof(double)) + 2 * kMaxCoarse * sizeof(double);
    return bytes;
}

// The tail smooths each level as register strips, the same arithmetic as the strip kernels
// (fc_smooth.cuh) with the whole level resident: warp w holds rows 2w and 2w + 1, lane j columns
// 2j and 2j + 1, so a level of up to 64 x 64 cells fits the 32 warps (the tail only takes such
// levels). Rows and columns outside the level hold zero weights, inverse diagonals and values,
// and the edge rows of the warps pass through shared memory once per half-sweep.
constexpr int kTailK = 2;
constexpr int kTailMaxSide = 2 * 32;
static_assert(kTailWarps * kTailK == kTailMaxSide, "tail strips cover 64 rows");

template <typename T> using TailEdges = Edges<T, kTailWarps>;

// Strip registers of level L: weights, inverse diagonals, masked right-hand side (less `mean`:
// the residual's mean on the fine level, zero elsewhere) and, for the post-smoothing, the
// pre-smoothed solution.
template <typename T>
__device__ __forceinline__ void tail_load_strip(const TailLevel<T>& L, Strip<T, kTailK>& s, bool with_solution,
    double mean, int lane, int warp)
{
    const T* m = tail_array<T>();
    const int x = 2 * lane;
    const bool col_a = x < L.w, col_b = x + 1 < L.w;
    const int y0 = kTailK * warp;
    s.ua = col_a && y0 < L.h ? m[L.down + L.at(x, y0 - 1)] : T(0);
    s.ub = col_b && y0 < L.h ? m[L.down + L.at(x + 1, y0 - 1)] : T(0);
#pragma unroll
    for (int k = 0; k < kTailK; ++k)
    {
        const int y = y0 + k;
        const bool in_a = col_a && y < L.h, in_b = col_b && y < L.h;
        const int i = in_a ? L.at(x, y) : 0;
        s.wm[k] = in_a ? m[L.right + i] : T(0);
        s.da[k] = in_a ? m[L.down + i] : T(0);
        s.ia[k] = in_a ? m[L.inv + i] : T(0);
        s.ra[k] = in_a && s.ia[k] > T(0) ? minus_mean(m[L.rhs + i], mean) : T(0);
        s.a[k] = in_a && with_solution ? m[L.sol + i] : T(0);
        s.wr[k] = in_b ? m[L.right + i + 1] : T(0);
        s.db[k] = in_b ? m[L.down + i + 1] : T(0);
        s.ib[k] = in_b ? m[L.inv + i + 1] : T(0);
        s.rb[k] = in_b && s.ib[k] > T(0) ? minus_mean(m[L.rhs + i + 1], mean) : T(0);
        s.b[k] = in_b && with_solution ? m[L.sol + i + 1] : T(0);
    }
}

template <typename T>
__device__ __forceinline__ void tail_store_solution(const TailLevel<T>& L, const Strip<T, kTailK>& s, int lane, int warp)
{
    T* m = tail_array<T>();
    const int x = 2 * lane;
#pragma unroll
    for (int k = 0; k < kTailK; ++k)
    {
        const int y = kTailK * warp + k;
        if (y >= L.h || x >= L.w)
            continue;
        const int i = L.at(x, y);
        m[L.sol + i] = s.a[k];
        if (x + 1 < L.w)
            m[L.sol + i + 1] = s.b[k];
    }
}

// Warps of the tail CTA that hold rows of level L, and the strips barrier for them: the whole
// CTA when every warp does, else named barrier 1 over those warps (the others wait for the
// level at the next CTA barrier). The last of them reads the row below its strip from the
// edge slot of the first idle warp, which a taller level may have written: it clears it.
template <typename T> struct TailWarps
{
    int active, threads;
    __device__ TailWarps(const TailLevel<T>& L)
    {
        active = (L.h + kTailK - 1) / kTailK;
        threads = active == kTailWarps ? 0 : active * 32;
    }
    __device__ void clear_below(TailEdges<T>& edges, int lane, int warp) const
    {
        if (warp == active - 1 && active < kTailWarps)
        {
            edges.top[0][active + 1][lane] = T(0);
            edges.top[1][active + 1][lane] = T(0);
        }
    }
};

// Pre-smoothing of tail level L: four red-black sweeps from zero, the residual, and its
// transpose-bilinear restriction into C's right-hand side (PressureMultigrid.cpp:398-402,
// 204-231, 233-276). The pre-smoothed solution stays in L.sol for the post-smoothing.
template <typename T>
__device__ void tail_pre(const TailLevel<T> L, const TailLevel<T> C, double mean, TailEdges<T>& edges, int lane, int warp)
{
    T* const m = tail_array<T>();
    const TailWarps<T> tw(L);
    if (warp < tw.active)
    {
    Strip<T, kTailK> s;
    tail_load_strip(L, s, false, mean, lane, warp);
    tw.clear_below(edges, lane, warp);
    strip_sweep<T, kTailK, kTailWarps>(s, edges, 0, true, 0, lane, warp, tw.threads);
    strip_sweep<T, kTailK, kTailWarps>(s, edges, 1, false, 1, lane, warp, tw.threads);
#pragma unroll 1
    for (int sweep = 1; sweep < 4; ++sweep)
    {
        strip_sweep<T, kTailK, kTailWarps>(s, edges, 0, false, 0, lane, warp, tw.threads);
        strip_sweep<T, kTailK, kTailWarps>(s, edges, 1, false, 1, lane, warp, tw.threads);
    }
    // Residual from registers; the edge buffers hold the final values (buffer 0 colour 0,
    // buffer 1 colour 1). Cells without an open face pass no residual down.
    const T above_a = edges.bottom[1][warp][lane], above_b = edges.bottom[0][warp][lane];
    const T below_a = edges.top[0][warp + 2][lane], below_b = edges.top[1][warp + 2][lane];
    const int x = 2 * lane;
#pragma unroll
    for (int k = 0; k < kTailK; ++k)
    {
        T left = __shfl_up_sync(0xffffffffu, s.b[k], 1);
        T right = __shfl_down_sync(0xffffffffu, s.a[k], 1);
        T wl = __shfl_up_sync(0xffffffffu, s.wr[k], 1);
        left = lane == 0 ? T(0) : left;
        right = lane == 31 ? T(0) : right;
        wl = lane == 0 ? T(0) : wl;
        const T ua = k == 0 ? above_a : s.a[k - 1];
        const T ub = k == 0 ? above_b : s.b[k - 1];
        const T na = k == kTailK - 1 ? below_a : s.a[k + 1];
        const T nb = k == kTailK - 1 ? below_b : s.b[k + 1];
        const T wua = k == 0 ? s.ua : s.da[k - 1];
        const T wub = k == 0 ? s.ub : s.db[k - 1];
        const T a = s.a[k], b = s.b[k];
        const T pa = (wl * (a - left) + s.wm[k] * (a - b)) + (wua * (a - ua) + s.da[k] * (a - na));
        const T pb = (s.wm[k] * (b - a) + s.wr[k] * (b - right)) + (wub * (b - ub) + s.db[k] * (b - nb));
        const int y = kTailK * warp + k;
        if (y >= L.h || x >= L.w)
            continue;
        const int i = L.at(x, y);
        m[L.sol + i] = a;
        m[L.res + i] = s.ia[k] > T(0) ? s.ra[k] - pa : T(0);
        if (x + 1 < L.w)
        {
            m[L.sol + i + 1] = b;
            m[L.res + i + 1] = s.ib[k] > T(0) ? s.rb[k] - pb : T(0);
        }
    }
    }
    __syncthreads();
    // Restriction: coarse cell (cx, cy) sums fine rows 2cy-1 .. 2cy+2 of the x-sums of fine
    // columns 2cx-1 .. 2cx+2 (only the offsets its tables list are read).
    const Gather* rx = tail_table<const Gather>(L.rx);
    const Gather* ry = tail_table<const Gather>(L.ry);
    for (int q = threadIdx.x; q < C.w * C.h; q += kTailThreads)
    {
        const int cx = q % C.w, cy = q / C.w;
        const RestrictAxis<T> ax = restrict_axis<T>(rx, cx), ay = restrict_axis<T>(ry, cy);
        T line[4];
#pragma unroll
        for (int p = 0; p < 4; ++p)
        {
            line[p] = T(0);
            if (ay.mask & (1u << p))
            {
                const int row = L.res + L.at(2 * cx - 1, 2 * cy - 1 + p);
                T v[4];
#pragma unroll
                for (int e = 0; e < 4; ++e)
                    v[e] = (ax.mask & (1u << e)) ? m[row + e] : T(0);
                line[p] = restrict_sum(ax, v[0], v[1], v[2], v[3]);
            }
        }
        m[C.rhs + C.at(cx, cy)] = restrict_sum(ay, line[0], line[1], line[2], line[3]);
    }
    __syncthreads();
}

// Post-smoothing of tail level L: the bilinear prolongation of C's solution added to the
// pre-smoothed solution, then four sweeps in reversed colour order (PressureMultigrid.cpp:
// 403-407, 278-298). The result replaces L.sol.
template <typename T>
__device__ void tail_post(const TailLevel<T> C, const TailLevel<T> L, double mean, TailEdges<T>& edges, int lane,
    int warp)
{
    const T* m = tail_array<T>();
    const TailWarps<T> tw(L);
    if (warp < tw.active)
    {
    Strip<T, kTailK> s;
    tail_load_strip(L, s, true, mean, lane, warp);
    tw.clear_below(edges, lane, warp);
    const Interp* px = tail_table<const Interp>(L.px);
    const Interp* py = tail_table<const Interp>(L.py);
    const int x = 2 * lane;
    const bool col_a = x < L.w, col_b = x + 1 < L.w;
    const Interp pa = col_a ? px[x] : Interp{0, 0, 0.0};
    const Interp pb = col_b ? px[x + 1] : Interp{0, 0, 0.0};
    const T wxa = T(pa.weight), wxb = T(pb.weight);
#pragma unroll
    for (int k = 0; k < kTailK; ++k)
    {
        const int y = kTailK * warp + k;
        if (y >= L.h)
            continue;
        const Interp iy = py[y];
        const T wy = T(iy.weight);
        const int top = C.sol + C.at(0, iy.first), bottom = C.sol + C.at(0, iy.second);
        if (col_a)
        {
            const T u = (T(1) - wxa) * m[top + pa.first] + wxa * m[top + pa.second];
            const T d = (T(1) - wxa) * m[bottom + pa.first] + wxa * m[bottom + pa.second];
            s.a[k] = s.a[k] + ((T(1) - wy) * u + wy * d);
        }
        if (col_b)
        {
            const T u = (T(1) - wxb) * m[top + pb.first] + wxb * m[top + pb.second];
            const T d = (T(1) - wxb) * m[bottom + pb.first] + wxb * m[bottom + pb.second];
            s.b[k] = s.b[k] + ((T(1) - wy) * u + wy * d);
        }
        // A cell that is no unknown keeps zero (Dirichlet air sees it; elsewhere such a cell
        // has no open face and its value is never read).
        s.a[k] = s.ia[k] > T(0) ? s.a[k] : T(0);
        s.b[k] = s.ib[k] > T(0) ? s.b[k] : T(0);
    }
    // The first half-sweep (colour 1) reads colour-0 edges from buffer 1.
    edges.top[1][warp + 1][lane] = s.a[0];
    edges.bottom[1][warp + 1][lane] = s.b[kTailK - 1];
    strips_barrier(tw.threads);
#pragma unroll 1
    for (int sweep = 0; sweep < 4; ++sweep)
    {
        strip_sweep<T, kTailK, kTailWarps>(s, edges, 1, false, 0, lane, warp, tw.threads);
        strip_sweep<T, kTailK, kTailWarps>(s, edges, 0, false, 1, lane, warp, tw.threads);
    }
    tail_store_solution(L, s, lane, warp);
    }
    __syncthreads();
}

// Mean-free rhs, explicit inverse, mean-zero gauge over the open cells.
// PressureMultigrid.cpp:347-384 (solveCoarsest).
template <typename T>
__device__ void tail_solve_coarsest(const TailLevel<T> L, int inverse_offset, int vectors_offset, const CoarseInfo& info)
{
    T* const m = tail_array<T>();
    const double* inverse = tail_table<const double>(inverse_offset);
    double* b = tail_table<double>(vectors_offset);
    double* z = b + kMaxCoarse;
    __shared__ double mean_shared;
    const int cells = L.w * L.h, n = info.n;
    // Single-warp reductions: the coarsest level has at most 64 cells.
    if (threadIdx.x < 32)
    {
        double part = 0.0;
        for (int q = threadIdx.x; q < cells; q += 32)
            if (q == info.pinned || info.map[q] >= 0)
                part += double(m[L.rhs + L.at(q % L.w, q / L.w)]);
        part = warp_sum(part);
        if (threadIdx.x == 0)
            mean_shared = info.open > 0 && !info.dirichlet ? part / info.open : 0.0;
    }
    __syncthreads();
    const double mean = mean_shared;
    for (int q = threadIdx.x; q < cells; q += blockDim.x)
    {
        const int k = info.map[q];
        if (k >= 0)
            b[k] = double(m[L.rhs + L.at(q % L.w, q / L.w)]) - mean;
    }
    __syncthreads();
    // z = inverse b: eight threads per row, then a shuffle fold within each group of eight.
    for (int base = 0; base < n; base += kTailThreads / 8)
    {
        const int row = base + int(threadIdx.x >> 3), part = threadIdx.x & 7;
        double value = 0.0;
        if (row < n)
            for (int col = part; col < n; col += 8)
                value += inverse[row * n + col] * b[col];
        value += __shfl_xor_sync(0xffffffffu, value, 1);
        value += __shfl_xor_sync(0xffffffffu, value, 2);
        value += __shfl_xor_sync(0xffffffffu, value, 4);
        if (row < n && part == 0)
            z[row] = value;
    }
    __syncthreads();
    if (threadIdx.x < 32)
    {
        double part = 0.0;
        for (int k = threadIdx.x; k < n; k += 32)
            part += z[k];
        part = warp_sum(part);
        if (threadIdx.x == 0)
            mean_shared = info.open > 0 && !info.dirichlet ? part / info.open : 0.0;
    }
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
        m[L.sol + L.at(q % L.w, q / L.w)] = T(value);
    }
    __syncthreads();
}

template <typename T> __global__ void __launch_bounds__(kTailThreads) k_mg_tail(const GridDesc* grids)
{
    allow_dependents();
    const GridDesc& g = grids[blockIdx.x];
    SolveState& state = *g.state;
    // In a batch (one CTA per grid), a grid whose solve is known to be done before the wait
    // copies nothing in. A single grid skips the check: its load would delay the copies.
    if (gridDim.x > 1 && done_before_wait(g.state))
        return;
    const int first = g.tail, last = g.levels - 1;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    T* const m = tail_array<T>();
    TailLevel<T> lv[kMaxLevels];
    int cursor = 0; // bytes
    for (int l = first; l <= last; ++l)
    {
        TailLevel<T>& L = lv[l];
        L.w = g.lev[l].w;
        L.h = g.lev[l].h;
        L.s = g.lev[l].S;
        const int cells = L.s * (L.h + 2);
        const int base = cursor / int(sizeof(T));
        L.right = base;
        L.down = base + cells;
        L.inv = base + 2 * cells;
        L.rhs = base + 3 * cells;
        L.sol = base + 4 * cells;
        L.res = base + 5 * cells;
        cursor += int(align16(size_t(cells) * 6 * sizeof(T)));
    }
    for (int l = first; l < last; ++l)
    {
        TailLevel<T>& L = lv[l];
        L.px = cursor;
        cursor += int(align16(L.w * sizeof(Interp)));
        L.py = cursor;
        cursor += int(align16(L.h * sizeof(Interp)));
        L.rx = cursor;
        cursor += int(align16(lv[l + 1].w * sizeof(Gather)));
        L.ry = cursor;
        cursor += int(align16(lv[l + 1].h * sizeof(Gather)));
    }
    const int inverse_offset = cursor;
    cursor += int(align16(size_t(kMaxCoarse) * kMaxCoarse * sizeof(double)));
    const int vectors_offset = cursor;

    // Everything the cycle reads except the right-hand side is written by no kernel of the
    // projection (weights, inverse diagonals, transfer tables, the coarsest inverse and its
    // unknown map), so it is copied in by bulk copies before waiting on the previous kernel. The
    // global arrays are 256-byte aligned slots of one allocation, so rounding a copy up to 16
    // bytes stays inside it; every shared region is rounded the same way. The arrays that no
    // copy fills are written before they are read (solutions, residuals, coarse right-hand
    // sides), and only their in-level cells are read.
    __shared__ uint64_t bar;
    __shared__ TailEdges<T> edges;
    __shared__ CoarseInfo info;
    if (threadIdx.x == 0)
    {
        mbarrier_init(&bar, 1);
        fence_async_shared();
    }
    edges_clear<T, kTailK, kTailWarps>(edges);
    if (threadIdx.x < int(sizeof(CoarseInfo) / sizeof(int)))
        reinterpret_cast<int*>(&info)[threadIdx.x] = reinterpret_cast<const int*>(g.coarse)[threadIdx.x];
    __syncthreads();
    // Bulk copies write 16-byte aligned shared addresses only: a misplaced buffer is reported.
    if ((smem_address(tail_smem) & 15u) != 0)
    {
        if (threadIdx.x == 0)
            stage_failed_at(g.state);
        return;
    }
    if (threadIdx.x == 0)
    {
        auto rounded = [](size_t bytes) { return unsigned(align16(bytes)); };
        unsigned total = 0;
        for (int l = first; l < last; ++l)
        {
            const size_t cells = size_t(lv[l].s) * (lv[l].h + 2);
            total += 3 * rounded(cells * sizeof(T));
            total += rounded(lv[l].w * sizeof(Interp)) + rounded(lv[l].h * sizeof(Interp)) +
                     rounded(lv[l + 1].w * sizeof(Gather)) + rounded(lv[l + 1].h * sizeof(Gather));
        }
        total += rounded(size_t(info.n) * info.n * sizeof(double));
        mbarrier_expect_tx(&bar, total);
        for (int l = first; l < last; ++l)
        {
            const TailLevel<T>& L = lv[l];
            const LevelDesc& D = g.lev[l];
            const unsigned bytes = rounded(size_t(L.s) * (L.h + 2) * sizeof(T));
            bulk_load(m + L.right, D.right, bytes, &bar);
            bulk_load(m + L.down, D.down, bytes, &bar);
            bulk_load(m + L.inv, D.inv, bytes, &bar);
            bulk_load(tail_smem + L.px, D.px, rounded(L.w * sizeof(Interp)), &bar);
            bulk_load(tail_smem + L.py, D.py, rounded(L.h * sizeof(Interp)), &bar);
            bulk_load(tail_smem + L.rx, D.rx, rounded(lv[l + 1].w * sizeof(Gather)), &bar);
            bulk_load(tail_smem + L.ry, D.ry, rounded(lv[l + 1].h * sizeof(Gather)), &bar);
        }
        if (info.n > 0)
            bulk_load(tail_smem + inverse_offset, g.coarse_inverse, rounded(size_t(info.n) * info.n * sizeof(double)), &bar);
    }
    if (stage_failed(mbarrier_wait(&bar, 0), g.state))
        return;

    // The right-hand side of the first tail level comes from the previous kernel.
    dependency_wait();
    if (state.done)
        return;
    const double mean_r = first == 0 ? state.mean_r : 0.0;
    {
        const TailLevel<T> L = lv[first];
        const LevelDesc& D = g.lev[first];
        const T* rhs = first == 0 ? static_cast<const T*>(g.r) : static_cast<const T*>(D.rhs);
        if (first < last)
        {
            // Raw; the strips mask it and take off the residual's mean (level 0).
            if (threadIdx.x == 0)
            {
                const unsigned bytes = unsigned(align16(size_t(L.s) * (L.h + 2) * sizeof(T)));
                mbarrier_expect_tx(&bar, bytes);
                bulk_load(m + L.rhs, rhs, bytes, &bar);
            }
            if (stage_failed(mbarrier_wait(&bar, 1), g.state))
                return;
        }
        else
        {
            // A grid of at most 64 cells: the coarsest solve reads the masked right-hand side.
            const T* right = static_cast<const T*>(D.right);
            const T* down = static_cast<const T*>(D.down);
            for (int q = threadIdx.x; q < L.w * L.h; q += kTailThreads)
            {
                const int x = q % L.w, y = q / L.w;
                const int i = padded_index32_tail(D.S, x, y);
                const T diag = ((right[i - 1] + right[i]) + down[i - D.S]) + down[i];
                m[L.rhs + L.at(x, y)] = diag > T(0) ? (first == 0 ? minus_mean(rhs[i], mean_r) : rhs[i]) : T(0);
            }
            __syncthreads();
        }
    }

    for (int l = first; l < last; ++l)
        tail_pre(lv[l], lv[l + 1], l == 0 ? mean_r : 0.0, edges, lane, warp);
    tail_solve_coarsest(lv[last], inverse_offset, vectors_offset, info);
    for (int l = last - 1; l >= first; --l)
        tail_post(lv[l + 1], lv[l], l == 0 ? mean_r : 0.0, edges, lane, warp);

    // Hand the first tail level's solution to the finer post-smoothing (or to z).
    const TailLevel<T> F = lv[first];
    const LevelDesc& D = g.lev[first];
    T* out = static_cast<T*>(D.sol);
    const T* r = static_cast<const T*>(g.r);
    double sz = 0.0, srz = 0.0;
    for (int y = warp; y < F.h; y += kTailWarps)
    {
        for (int x = lane; x < F.w; x += 32)
        {
            const int i = padded_index32_tail(D.S, x, y);
            const T value = m[F.sol + F.at(x, y)];
            out[i] = value;
            if (first == 0)
            {
                // Cells without an open face hold z = 0; the rest add to both sums.
                sz += double(value);
                srz += double(r[i]) * double(value);
            }
        }
    }
    if (first != 0)
        return;
    const double4 total = block_reduce4<kTailThreads>(make_double4(sz, srz, 0, 0), 0);
    if (threadIdx.x == 0)
        finish_preconditioner(state, total.x, total.y);
}

} // namespace fc
