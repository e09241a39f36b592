// Persistent, TMA-staged red-black smoothing of the multigrid levels (the V-cycle's hot kernels).
//
// Same arithmetic as the register strips of fc_smooth.cuh (a warp owns K rows x 64 columns,
// lane j columns 2j and 2j+1, every cell's values in registers, one shuffle per horizontal
// neighbour, edge rows through shared memory), but each CTA now walks a list of tiles and the
// inputs of its next tile stream into shared memory by TMA while the current tile computes:
//
//   wait for tile i's boxes -> load the strips from shared memory -> barrier ->
//   issue tile i+1's boxes -> sweep tile i from registers -> write tile i's outputs
//
// so the HBM latency of one tile hides behind the arithmetic of the previous one. The boxes are
// 2D tiles of the padded level arrays: weights, inverse diagonal, the level's vector (and for
// the post kernel the pre-smoothed solution and the coarse solution), 72 columns x WARPS*K+1
// rows (the strip rows and the row above, the column left of the region, rounded out to 16-byte
// alignment); coordinates outside an array read as zero, as the padded halo does. The post kernel
// also bulk-copies the region's rows and columns of the prolongation tables.
#pragma once

#include "fc_smooth.cuh"
#include "fc_tma.cuh"

namespace fc
{

// One padded level array's box, and the per-tile layout of the staging buffer.
template <typename T, typename W, int K, bool PRE, int WARPS = 8> struct Stage
{
    static constexpr int BW = 72;            // box columns (elements)
    static constexpr int BH = WARPS * K + 1; // strip rows plus the row above
    static constexpr int CBW = 40;           // coarse box (post): columns
    static constexpr int CBH = WARPS * K / 2 + 4; //   and rows
    static constexpr size_t round(size_t b) { return (b + 127) / 128 * 128; }
    static constexpr size_t WB = round(size_t(BW) * BH * sizeof(W));
    static constexpr size_t VB = round(size_t(BW) * BH * sizeof(T));
    static constexpr size_t CB = PRE ? 0 : round(size_t(CBW) * CBH * sizeof(T));
    // Post: the prolongation tables of the region's rows and columns (Interp, 16 bytes each).
    static constexpr size_t IY = PRE ? 0 : round(size_t(WARPS) * K * sizeof(Interp));
    static constexpr size_t IX = PRE ? 0 : round(64 * sizeof(Interp));
    // The inverse diagonal is staged rather than formed from the weights: a correctly rounded
    // FP32 reciprocal per cell cost more time (2,300 cycles a tile) than its box's copy.
    static constexpr size_t right = 0, down = WB, inv = 2 * WB, vec = 2 * WB + VB, pre = 2 * WB + 2 * VB;
    static constexpr size_t coarse = PRE ? pre : pre + VB;
    static constexpr size_t rows = coarse + CB, cols = rows + IY;
    static constexpr size_t bytes = cols + IX;
    // Bytes the boxes of one tile deliver (full boxes, zero-filled parts included).
    static constexpr unsigned tx = unsigned(2 * BW * BH * sizeof(W) + (PRE ? 2 : 3) * BW * BH * sizeof(T) +
                                            (PRE ? 0 : CBW * CBH * sizeof(T)));
};

// Tensor maps of a grid: per level, per region shape (kShapeTall, kShapeShort, kShapeWide),
// six maps.
enum RegionShape
{
    kShapeTall = 0,  // 8 warps of the larger strip height
    kShapeShort = 1, // 8 warps of the smaller strip height
    kShapeWide = 2,  // 16 warps of the larger strip height (FP32): twice the rows per region
    kShapes = 3
};

enum StageMap
{
    kMapRight = 0,
    kMapDown = 1,
    kMapVector = 2, // level 0: the PCG residual r; coarser levels: the restricted rhs
    kMapPre = 3,
    kMapCoarse = 4, // the next level's solution (post)
    kMapInverse = 5, // the level's inverse diagonal
    kMapsPerSet = 6
};
constexpr int kTensorMapBytes = 128;

__device__ __forceinline__ const void* stage_map(const char* maps, int level, int set, int which)
{
    return maps + size_t((level * kShapes + set) * kMapsPerSet + which) * kTensorMapBytes;
}

// What the issuing thread needs to start one tile's copies, read from the tile's grid
// descriptor a tile ahead: the issue then waits on no global load.
struct IssueArgs
{
    const char* maps;  // the grid's tensor maps
    const Interp* py;  // post: the level's prolongation tables
    const Interp* px;
    int w, h;          // the level's size
};

__device__ __forceinline__ IssueArgs issue_args(const GridDesc& g, int level)
{
    const LevelDesc& L = g.lev[level];
    return IssueArgs{static_cast<const char*>(g.maps), L.py, L.px, L.w, L.h};
}

// First box column of a region whose leftmost needed padded column is v: a TMA box must start
// at a multiple of 16 bytes, i.e. of 16 / sizeof(E) elements (4 for FP32, 8 for FP16).
template <typename E> __host__ __device__ __forceinline__ int box_start(int v)
{
    return sizeof(E) >= 4 ? (v & ~3) : (v & ~7);
}

// Issues the boxes of the tile whose region starts at (X0, Y0); one thread. The weights and the
// inverse diagonal are written by no kernel of the projection, so a kernel may issue them before
// waiting on its predecessor (stage_issue_weights); the other boxes follow (stage_issue_data). The barrier
// expects the bytes of all of them from the first call.
template <typename T, typename W, int K, bool PRE, int WARPS>
__device__ __forceinline__ void stage_issue_weights(const IssueArgs& g, int level, int set, int X0, int Y0, char* stage,
    uint64_t* bar)
{
    using S = Stage<T, W, K, PRE, WARPS>;
    // Padded coordinates: column gx + 2, row gy + 1. The region needs columns X0-1 .. X0+63 and
    // rows Y0-1 .. Y0+WARPS*K-1.
    const int bw = box_start<W>(X0 + 1), by = Y0;
    if constexpr (!PRE)
    {
        // The prolongation tables of the region's in-level rows and columns, by bulk copy into
        // slots indexed by region row / column (the kernel reads in-level slots only).
        const int r0 = max(Y0, 0), r1 = min(Y0 + WARPS * K, g.h);
        const int c0 = max(X0, 0), c1 = min(X0 + 64, g.w);
        const unsigned row_bytes = r1 > r0 ? unsigned(r1 - r0) * sizeof(Interp) : 0u;
        const unsigned col_bytes = c1 > c0 ? unsigned(c1 - c0) * sizeof(Interp) : 0u;
        mbarrier_expect_tx(bar, S::tx + row_bytes + col_bytes);
        if (row_bytes)
            bulk_load(stage + S::rows + size_t(r0 - Y0) * sizeof(Interp), g.py + r0, row_bytes, bar);
        if (col_bytes)
            bulk_load(stage + S::cols + size_t(c0 - X0) * sizeof(Interp), g.px + c0, col_bytes, bar);
    }
    else
        mbarrier_expect_tx(bar, S::tx);
    tma_load_2d(stage + S::right, stage_map(g.maps, level, set, kMapRight), bw, by, bar);
    tma_load_2d(stage + S::down, stage_map(g.maps, level, set, kMapDown), bw, by, bar);
    tma_load_2d(stage + S::inv, stage_map(g.maps, level, set, kMapInverse), box_start<T>(X0 + 1), by, bar);
}

template <typename T, typename W, int K, bool PRE, int WARPS>
__device__ __forceinline__ void stage_issue_data(const IssueArgs& g, int level, int set, int X0, int Y0, char* stage,
    uint64_t* bar)
{
    using S = Stage<T, W, K, PRE, WARPS>;
    const int bx = box_start<T>(X0 + 1), by = Y0;
    tma_load_2d(stage + S::vec, stage_map(g.maps, level, set, kMapVector), bx, by, bar);
    if (!PRE)
    {
        tma_load_2d(stage + S::pre, stage_map(g.maps, level, set, kMapPre), bx, by, bar);
        const int CX0 = X0 / 2 - 1, CY0 = Y0 / 2 - 1;
        tma_load_2d(stage + S::coarse, stage_map(g.maps, level, set, kMapCoarse), box_start<T>(CX0 + 2), CY0 + 1, bar);
    }
}

// Fetches the descriptors of the data maps ahead of the data copies (one thread): their first
// use after the dependency wait then costs only the copy.
template <bool PRE> __device__ __forceinline__ void stage_prefetch_data_maps(const IssueArgs& g, int level, int set)
{
    prefetch_tensormap(stage_map(g.maps, level, set, kMapVector));
    if (!PRE)
    {
        prefetch_tensormap(stage_map(g.maps, level, set, kMapPre));
        prefetch_tensormap(stage_map(g.maps, level, set, kMapCoarse));
    }
}

template <typename T, typename W, int K, bool PRE, int WARPS>
__device__ __forceinline__ void stage_issue(const IssueArgs& g, int level, int set, int X0, int Y0, char* stage,
    uint64_t* bar)
{
    stage_issue_weights<T, W, K, PRE, WARPS>(g, level, set, X0, Y0, stage, bar);
    stage_issue_data<T, W, K, PRE, WARPS>(g, level, set, X0, Y0, stage, bar);
}

template <typename W> __device__ __forceinline__ float2 weight_pair(const W* p, float scale);
template <> __device__ __forceinline__ float2 weight_pair<float>(const float* p, float)
{
    return *reinterpret_cast<const float2*>(p);
}
template <> __device__ __forceinline__ float2 weight_pair<__half>(const __half* p, float scale)
{
    const float2 v = __half22float2(*reinterpret_cast<const __half2*>(p));
    return make_float2(v.x * scale, v.y * scale);
}

// Strip registers from the staged boxes: weights, inverse diagonals and right-hand side.
template <typename T, typename W, int K, bool PRE, int WARPS>
__device__ __forceinline__ void stage_strip(Strip<T, K>& s, const char* stage, int X0, float wscale, int lane, int warp)
{
    using S = Stage<T, W, K, PRE, WARPS>;
    using P = typename Pair<T>::type;
    // Box columns of cell X0 + 2 lane in the vector and the weight boxes.
    const int c = (X0 + 2 - box_start<T>(X0 + 1)) + 2 * lane;
    const int cw = (X0 + 2 - box_start<W>(X0 + 1)) + 2 * lane;
    const W* right = reinterpret_cast<const W*>(stage + S::right);
    const W* down = reinterpret_cast<const W*>(stage + S::down);
    const T* vec = reinterpret_cast<const T*>(stage + S::vec);
    const T* inv = reinterpret_cast<const T*>(stage + S::inv);
#pragma unroll
    for (int k = 0; k < K; ++k)
    {
        const int r = (warp * K + k + 1) * S::BW + c;
        const int rw = (warp * K + k + 1) * S::BW + cw;
        if constexpr (sizeof(T) == 8)
        {
            const P w2 = *reinterpret_cast<const P*>(right + rw);
            const P d2 = *reinterpret_cast<const P*>(down + rw);
            s.wm[k] = w2.x;
            s.wr[k] = w2.y;
            s.da[k] = d2.x;
            s.db[k] = d2.y;
        }
        else
        {
            const float2 w2 = weight_pair<W>(right + rw, wscale);
            const float2 d2 = weight_pair<W>(down + rw, wscale);
            s.wm[k] = w2.x;
            s.wr[k] = w2.y;
            s.da[k] = d2.x;
            s.db[k] = d2.y;
        }
        const P r2 = *reinterpret_cast<const P*>(vec + r);
        s.ra[k] = r2.x;
        s.rb[k] = r2.y;
        const P i2 = *reinterpret_cast<const P*>(inv + r);
        s.ia[k] = i2.x;
        s.ib[k] = i2.y;
    }
    const int u = (warp * K) * S::BW + cw;
    if constexpr (sizeof(T) == 8)
    {
        const P u2 = *reinterpret_cast<const P*>(down + u);
        s.ua = u2.x;
        s.ub = u2.y;
    }
    else
    {
        const float2 u2 = weight_pair<W>(down + u, wscale);
        s.ua = u2.x;
        s.ub = u2.y;
    }
}

// (1 - w) lo + w hi with one explicit rounding order (a product, then a fused multiply-add),
// so that every path of the prolongation rounds a value the same way.
template <typename T> __device__ __forceinline__ T prolong_lerp(T w, T lo, T hi)
{
    return fma(w, hi, (T(1) - w) * lo);
}

// Pre-smoothing of `count` tiles (tiles[0 .. count)): four sweeps from zero, the residual, the
// pre-smoothed solution of the output cells and the transpose-bilinear restriction into the
// coarse right-hand side (PressureMultigrid.cpp:398-402, 204-231, 233-276).
//
// Descriptor fields a tile uses are copied into registers when the tile starts, and the next
// tile's entry and copy arguments are read one tile ahead: the kernel's global stores cannot
// alias them, but the compiler cannot know that and would reload them from memory after every
// store, which put dependent global loads on each tile's path.
//
// A tile whose grid's solve is done is neither computed nor copied in: the issuing thread
// completes its barrier phase with a plain arrival instead of the boxes and records its decision
// in `tile_live`, which every thread reads after the phase's wait. The loop's idle passes after
// convergence, and the finished grids of a batch, then stream nothing but the first tile's
// boxes of each CTA (issued before the dependency wait, when no decision is known yet).
template <typename T, int K, typename W, int WARPS>
__global__ void __launch_bounds__(32 * WARPS, (sizeof(T) == 4 && WARPS == 8) ? 2 : 1)
    k_smooth_pre(const GridDesc* __restrict__ grids, const Tile* __restrict__ tiles, int count, int level, int set)
{
    using Shape = TileShape<T, K, true, WARPS>;
    using S = Stage<T, W, K, true, WARPS>;
    extern __shared__ __align__(128) char stage[];
    __shared__ uint64_t bar;
    __shared__ Edges<T, WARPS> edges;
    constexpr int OCX = Shape::OX / 2, OCY = Shape::OY / 2;
    // The restriction runs in two passes. Along x, lane L sums fine columns 2L-1 .. 2L+2 of
    // every row from registers into lines[row][L]: that is coarse column L - HALO/2 of the
    // tile. Along y, coarse row q sums lines HALO-1+2q .. HALO+2+2q.
    static_assert(Shape::HALO % 2 == 0 && Shape::HALO / 2 >= 2 && OCX + Shape::HALO / 2 <= 31, "restriction lanes");
    __shared__ T lines[Shape::RY][32];
    __shared__ RestrictAxis<T> along_y[OCY];
    __shared__ int tile_live; // the issuing thread's decision on the tile it last started
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    allow_dependents();
    // TMA writes shared memory at 128-byte aligned addresses only; a misplaced staging buffer is
    // reported on the first tile's grid (after the wait) instead of being written.
    const bool misplaced = (smem_address(stage) & 127u) != 0;
    if (threadIdx.x == 0)
    {
        mbarrier_init(&bar, 1);
        fence_async_shared();
    }
    edges_clear<T, K, WARPS>(edges);
    __syncthreads();
    int i = blockIdx.x;
    Tile t = i < count ? tiles[i] : Tile{};
    // The first tile's weights stream in while the previous kernel finishes.
    if (threadIdx.x == 0 && i < count && !misplaced)
    {
        const IssueArgs first = issue_args(grids[t.grid], level);
        stage_issue_weights<T, W, K, true, WARPS>(first, level, set, t.x0 - Shape::HALO, t.y0 - Shape::HALO, stage, &bar);
        stage_prefetch_data_maps<true>(first, level, set);
    }
    dependency_wait();
    if (misplaced)
    {
        if (threadIdx.x == 0 && i < count)
            stage_failed_at(grids[t.grid].state);
        return;
    }
    // The first tile's boxes complete its phase whatever its grid's state (the weights are in
    // flight already); it only decides whether the tile is computed.
    if (threadIdx.x == 0 && i < count)
    {
        tile_live = grids[t.grid].state->done == 0;
        stage_issue_data<T, W, K, true, WARPS>(issue_args(grids[t.grid], level), level, set, t.x0 - Shape::HALO,
            t.y0 - Shape::HALO, stage, &bar);
    }
    unsigned parity = 0;
    for (; i < count; i += gridDim.x)
    {
        const int next = i + gridDim.x;
        const Tile n = next < count ? tiles[next] : Tile{};
        const GridDesc& g = grids[t.grid];
        SolveState* const state = g.state;
        const LevelDesc& Ld = g.lev[level];
        const LevelDesc& Cd = g.lev[level + 1];
        const int Lw = Ld.w, Lh = Ld.h, LS = Ld.S;
        const int Cw = Cd.w, Ch = Cd.h, CS = Cd.S;
        T* const pre = static_cast<T*>(Ld.pre);
        T* const crhs = static_cast<T*>(Cd.rhs);
        const float wscale = Ld.wscale;
        const int X0 = t.x0 - Shape::HALO, Y0 = t.y0 - Shape::HALO;
        const int cx0 = t.x0 / 2, cy0 = t.y0 / 2;
        // The restriction weights of the tile's coarse cells, while its boxes land.
        const int qx = lane - Shape::HALO / 2, cx = cx0 + qx;
        const bool column = qx >= 0 && qx < OCX && cx < Cw;
        // Plain loads first used after the sweeps, so their latency stays off the tile's path.
        RestrictAxis<T> along_x{};
        if (column)
            along_x = static_cast<const RestrictAxis<T>*>(Ld.rwx)[cx];
        RestrictAxis<T> row_weights{};
        if (threadIdx.x < OCY && cy0 + int(threadIdx.x) < Ch)
            row_weights = static_cast<const RestrictAxis<T>*>(Ld.rwy)[cy0 + threadIdx.x];
        const double mean_r = level == 0 ? state->mean_r : 0.0;
        // The next tile's copy arguments and whether its grid still solves, for the issuing thread.
        IssueArgs na{};
        bool next_live = false;
        if (threadIdx.x == 0 && next < count)
        {
            na = issue_args(grids[n.grid], level);
            next_live = grids[n.grid].state->done == 0;
        }
        const bool ok = mbarrier_wait(&bar, parity);
        if (stage_failed(ok, state))
            return;
        parity ^= 1u;
        // Written before the barrier inside stage_failed; rewritten only after the next one.
        const bool done = tile_live == 0;
        Strip<T, K> s;
        if (!done)
        {
            stage_strip<T, W, K, true, WARPS>(s, stage, X0, wscale, lane, warp);
            strip_finish<T, K>(s, level, mean_r);
        }
        __syncthreads();
        // The staging buffer is free: the next tile's boxes stream in while this one sweeps.
        if (threadIdx.x == 0 && next < count)
        {
            tile_live = next_live;
            if (next_live)
            {
                fence_async_shared();
                stage_issue<T, W, K, true, WARPS>(na, level, set, n.x0 - Shape::HALO, n.y0 - Shape::HALO, stage, &bar);
            }
            else
                mbarrier_arrive(&bar);
        }
        if (done)
        {
            t = n;
            continue;
        }
#pragma unroll
        for (int k = 0; k < K; ++k)
            s.a[k] = s.b[k] = T(0);
        strip_sweep<T, K, WARPS>(s, edges, 0, true, 0, lane, warp);
        strip_sweep<T, K, WARPS>(s, edges, 1, false, 1, lane, warp);
#pragma unroll 1
        for (int sweep = 1; sweep < 4; ++sweep)
        {
            strip_sweep<T, K, WARPS>(s, edges, 0, false, 0, lane, warp);
            strip_sweep<T, K, WARPS>(s, edges, 1, false, 1, lane, warp);
        }
        // Residual of every cell, summed along x into the lines; the edge buffers hold the final
        // values: buffer 0 colour 0, buffer 1 colour 1.
        const T above_a = edges.bottom[1][warp][lane], above_b = edges.bottom[0][warp][lane];
        const T below_a = edges.top[0][warp + 2][lane], below_b = edges.top[1][warp + 2][lane];
        const int gx = X0 + 2 * lane;
#pragma unroll
        for (int k = 0; k < K; ++k)
        {
            T left = __shfl_up_sync(0xffffffffu, s.b[k], 1);
            T right = __shfl_down_sync(0xffffffffu, s.a[k], 1);
            left = lane == 0 ? T(0) : left;
            right = lane == 31 ? T(0) : right;
            const T ua = k == 0 ? above_a : s.a[k - 1];
            const T ub = k == 0 ? above_b : s.b[k - 1];
            const T na_ = k == K - 1 ? below_a : s.a[k + 1];
            const T nb_ = k == K - 1 ? below_b : s.b[k + 1];
            const T wua = k == 0 ? s.ua : s.da[k - 1];
            const T wub = k == 0 ? s.ub : s.db[k - 1];
            const T a = s.a[k], b = s.b[k];
            // Lane 0's cells are halo columns whose residual neither the output nor the
            // restriction reads (its first lane, HALO/2, takes columns from HALO - 1 on).
            T wl = __shfl_up_sync(0xffffffffu, s.wr[k], 1); // every lane takes part
            wl = lane == 0 ? T(0) : wl;
            const T pa = (wl * (a - left) + s.wm[k] * (a - b)) + (wua * (a - ua) + s.da[k] * (a - na_));
            const T pb = (s.wm[k] * (b - a) + s.wr[k] * (b - right)) + (wub * (b - ub) + s.db[k] * (b - nb_));
            const int y = warp * K + k;
            const T res_a = s.ia[k] > T(0) ? s.ra[k] - pa : T(0);
            const T res_b = s.ib[k] > T(0) ? s.rb[k] - pb : T(0);
            // Lanes 0 and 31 hold no coarse column, so the wrapped shuffles are never summed.
            const T res_left = __shfl_up_sync(0xffffffffu, res_b, 1);
            const T res_right = __shfl_down_sync(0xffffffffu, res_a, 1);
            lines[y][lane] = restrict_sum(along_x, res_left, res_a, res_b, res_right);
            const int gy = Y0 + y;
            if (y >= Shape::HALO && y < Shape::HALO + Shape::OY && 2 * lane >= Shape::HALO &&
                2 * lane < Shape::HALO + Shape::OX && gy < Lh && gx < Lw)
            {
                const int idx = padded_index32(LS, gx, gy);
                if (gx + 1 < Lw)
                {
                    typename Pair<T>::type ab;
                    ab.x = a;
                    ab.y = b;
                    *reinterpret_cast<typename Pair<T>::type*>(pre + idx) = ab;
                }
                else
                    pre[idx] = a;
            }
        }
        if (threadIdx.x < OCY)
            along_y[threadIdx.x] = row_weights;
        __syncthreads();
        // Along y onto the tile's coarse cells: warp w takes coarse rows w, w + WARPS, ...
        // The next tile rewrites lines and along_y only after its first barrier, which every
        // thread reaches after finishing here.
        if (column)
        {
            for (int qy = warp; qy < OCY; qy += WARPS)
            {
                const int cy = cy0 + qy;
                if (cy >= Ch)
                    break;
                const int r = Shape::HALO - 1 + 2 * qy;
                crhs[padded_index32(CS, cx, cy)] =
                    restrict_sum(along_y[qy], lines[r][lane], lines[r + 1][lane], lines[r + 2][lane], lines[r + 3][lane]);
            }
        }
        t = n;
    }
}

// Post-smoothing of `count` tiles: the bilinear prolongation of the coarse solution added to
// the pre-smoothed one, four sweeps in reversed colour order, and on the fine level sum(z) and
// r.z for the PCG scalars (PressureMultigrid.cpp:403-407, 278-298; FluidGridCPU.cpp:1712-1726).
// Descriptor fields are held in registers and the next tile's entry read a tile ahead, as in
// k_smooth_pre.
template <typename T, int K, typename W, int WARPS>
__global__ void __launch_bounds__(32 * WARPS, (sizeof(T) == 4 && WARPS == 8) ? 2 : 1)
    k_smooth_post(const GridDesc* __restrict__ grids, const Tile* __restrict__ tiles, int count, int level, int set)
{
    using Shape = TileShape<T, K, false, WARPS>;
    using S = Stage<T, W, K, false, WARPS>;
    constexpr int NT = 32 * WARPS;
    extern __shared__ __align__(128) char stage[];
    __shared__ uint64_t bar;
    __shared__ Edges<T, WARPS> edges;
    __shared__ double4 total;
    __shared__ double2 warp_pairs[WARPS];
    __shared__ int tile_live; // the issuing thread's decision on the tile it last started (k_smooth_pre)
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    allow_dependents();
    // TMA writes shared memory at 128-byte aligned addresses only; a misplaced staging buffer is
    // reported on the first tile's grid (after the wait) instead of being written.
    const bool misplaced = (smem_address(stage) & 127u) != 0;
    if (threadIdx.x == 0)
    {
        mbarrier_init(&bar, 1);
        fence_async_shared();
    }
    edges_clear<T, K, WARPS>(edges);
    __syncthreads();
    int i = blockIdx.x;
    Tile t = i < count ? tiles[i] : Tile{};
    // The first tile's weights stream in while the previous kernel finishes.
    if (threadIdx.x == 0 && i < count && !misplaced)
    {
        const IssueArgs first = issue_args(grids[t.grid], level);
        stage_issue_weights<T, W, K, false, WARPS>(first, level, set, t.x0 - Shape::HALO, t.y0 - Shape::HALO, stage, &bar);
        stage_prefetch_data_maps<false>(first, level, set);
    }
    dependency_wait();
    if (misplaced)
    {
        if (threadIdx.x == 0 && i < count)
            stage_failed_at(grids[t.grid].state);
        return;
    }
    // The first tile's boxes complete its phase whatever its grid's state (the weights are in
    // flight already); it only decides whether the tile is computed.
    if (threadIdx.x == 0 && i < count)
    {
        tile_live = grids[t.grid].state->done == 0;
        stage_issue_data<T, W, K, false, WARPS>(issue_args(grids[t.grid], level), level, set, t.x0 - Shape::HALO,
            t.y0 - Shape::HALO, stage, &bar);
    }
    unsigned parity = 0;
    int run = 0; // level 0: tiles of the current grid finished since the last count
    for (; i < count; i += gridDim.x)
    {
        const int next = i + gridDim.x;
        const Tile n = next < count ? tiles[next] : Tile{};
        const GridDesc& g = grids[t.grid];
        SolveState* const state = g.state;
        const LevelDesc& Ld = g.lev[level];
        const int Lw = Ld.w, Lh = Ld.h, LS = Ld.S;
        T* const out = static_cast<T*>(Ld.sol);
        const float wscale = Ld.wscale;
        const int X0 = t.x0 - Shape::HALO, Y0 = t.y0 - Shape::HALO;
        const int CX0 = X0 / 2 - 1, CY0 = Y0 / 2 - 1;
        const int gx = X0 + 2 * lane;
        const bool in_a = gx >= 0 && gx < Lw, in_b = gx + 1 >= 0 && gx + 1 < Lw;
        const double mean_r = level == 0 ? state->mean_r : 0.0;
        IssueArgs na{};
        bool next_live = false;
        if (threadIdx.x == 0 && next < count)
        {
            na = issue_args(grids[n.grid], level);
            next_live = grids[n.grid].state->done == 0;
        }
        const bool ok = mbarrier_wait(&bar, parity);
        if (stage_failed(ok, state))
            return;
        parity ^= 1u;
        const bool done = tile_live == 0;
        Strip<T, K> s;
        if (!done)
        {
            stage_strip<T, W, K, false, WARPS>(s, stage, X0, wscale, lane, warp);
            // The pre-smoothed values of the strip.
            const T* pre = reinterpret_cast<const T*>(stage + S::pre);
            const int c = (X0 + 2 - box_start<T>(X0 + 1)) + 2 * lane;
#pragma unroll
            for (int k = 0; k < K; ++k)
            {
                const typename Pair<T>::type ab =
                    *reinterpret_cast<const typename Pair<T>::type*>(pre + (warp * K + k + 1) * S::BW + c);
                s.a[k] = ab.x;
                s.b[k] = ab.y;
            }
            strip_finish<T, K>(s, level, mean_r);
            // Add the prolonged coarse correction, in-level cells only; the tables arrived with
            // the tile's boxes.
            const Interp* interp_y = reinterpret_cast<const Interp*>(stage + S::rows);
            const Interp* interp_x = reinterpret_cast<const Interp*>(stage + S::cols);
            const T* coarse = reinterpret_cast<const T*>(stage + S::coarse);
            const int coff = CX0 + 2 - box_start<T>(CX0 + 2);
            const Interp pa = in_a ? interp_x[2 * lane] : Interp{CX0, CX0, 0.0};
            const Interp pb = in_b ? interp_x[2 * lane + 1] : Interp{CX0, CX0, 0.0};
            const T wxa = T(pa.weight), wxb = T(pb.weight);
            const int fa = pa.first - CX0 + coff, sa = pa.second - CX0 + coff;
            const int fb = pb.first - CX0 + coff, sb = pb.second - CX0 + coff;
            const int r0 = warp * K;
            // Each coarse row the warp's rows read is interpolated along x once: K / 2 + 2 rows
            // instead of 2K. The loads do not wait for the row tables: the box rows r0 / 2 ..
            // r0 / 2 + K / 2 + 1 are inside the coarse box whatever the tables say.
            T xa[K / 2 + 2], xb[K / 2 + 2];
#pragma unroll
            for (int j = 0; j < K / 2 + 2; ++j)
            {
                const T* row = coarse + (r0 / 2 + j) * S::CBW;
                xa[j] = prolong_lerp(wxa, row[fa], row[sa]);
                xb[j] = prolong_lerp(wxb, row[fb], row[sb]);
            }
            Interp py[K];
            bool regular = true;
#pragma unroll
            for (int k = 0; k < K; ++k)
            {
                const int gy = Y0 + r0 + k;
                regular = regular && gy >= 0 && gy < Lh;
                py[k] = regular ? interp_y[r0 + k] : Interp{CY0, CY0, 0.0};
                // Away from the level's edges, fine rows 2m and 2m + 1 (the region origin is
                // even) read coarse rows m - 1, m and m, m + 1: box rows r0 / 2 + (k + 1) / 2
                // and the one below.
                regular = regular && py[k].first - CY0 == r0 / 2 + (k + 1) / 2 && py[k].second == py[k].first + 1;
            }
            if (regular)
            {
#pragma unroll
                for (int k = 0; k < K; ++k)
                {
                    const T wy = T(py[k].weight);
                    const int f = (k + 1) / 2;
                    if (in_a)
                        s.a[k] = s.a[k] + prolong_lerp(wy, xa[f], xa[f + 1]);
                    if (in_b)
                        s.b[k] = s.b[k] + prolong_lerp(wy, xb[f], xb[f + 1]);
                }
            }
            else
            {
                // Rows at the level's edges: each fine row reads its two coarse rows.
#pragma unroll
                for (int k = 0; k < K; ++k)
                {
                    const int gy = Y0 + r0 + k;
                    if (gy < 0 || gy >= Lh)
                        continue;
                    const Interp q = interp_y[r0 + k];
                    const T* top = coarse + (q.first - CY0) * S::CBW;
                    const T* bottom = coarse + (q.second - CY0) * S::CBW;
                    const T wy = T(q.weight);
                    if (in_a)
                        s.a[k] = s.a[k] + prolong_lerp(wy, prolong_lerp(wxa, top[fa], top[sa]),
                                              prolong_lerp(wxa, bottom[fa], bottom[sa]));
                    if (in_b)
                        s.b[k] = s.b[k] + prolong_lerp(wy, prolong_lerp(wxb, top[fb], top[sb]),
                                              prolong_lerp(wxb, bottom[fb], bottom[sb]));
                }
            }
            // A cell that is no unknown keeps zero: Dirichlet air is read by its liquid
            // neighbours as p = 0; any other such cell has no open face and is never read.
#pragma unroll
            for (int k = 0; k < K; ++k)
            {
                s.a[k] = s.ia[k] > T(0) ? s.a[k] : T(0);
                s.b[k] = s.ib[k] > T(0) ? s.b[k] : T(0);
            }
        }
        __syncthreads();
        // The staging buffer is free: the next tile's boxes stream in while this one sweeps.
        if (threadIdx.x == 0 && next < count)
        {
            tile_live = next_live;
            if (next_live)
            {
                fence_async_shared();
                stage_issue<T, W, K, false, WARPS>(na, level, set, n.x0 - Shape::HALO, n.y0 - Shape::HALO, stage, &bar);
            }
            else
                mbarrier_arrive(&bar);
        }
        if (done)
        {
            t = n;
            continue;
        }
        // The first half-sweep (colour 1) reads colour-0 edges from buffer 1.
        edges.top[1][warp + 1][lane] = s.a[0];
        edges.bottom[1][warp + 1][lane] = s.b[K - 1];
        __syncthreads();
#pragma unroll 1
        for (int sweep = 0; sweep < 4; ++sweep)
        {
            strip_sweep<T, K, WARPS>(s, edges, 1, false, 0, lane, warp);
            strip_sweep<T, K, WARPS>(s, edges, 0, false, 1, lane, warp);
        }
        // Fine level: the thread's sums of z and r z over its output cells. FP32 sums its at
        // most 2K terms, and the warp's 32 threads, in FP32 and hands the warp's sums to the FP64
        // reduction (FP64 arithmetic and conversions per cell made this phase as long as the
        // sweeps); FP64 sums in FP64.
        T tz = T(0), trz = T(0);
        const bool cols_out = 2 * lane >= Shape::HALO && 2 * lane < Shape::HALO + Shape::OX;
#pragma unroll
        for (int k = 0; k < K; ++k)
        {
            const int y = warp * K + k;
            const int gy = Y0 + y;
            if (!cols_out || y < Shape::HALO || y >= Shape::HALO + Shape::OY || gy >= Lh || !in_a)
                continue;
            const int idx = padded_index32(LS, gx, gy);
            if (in_b)
            {
                typename Pair<T>::type ab;
                ab.x = s.a[k];
                ab.y = s.b[k];
                *reinterpret_cast<typename Pair<T>::type*>(out + idx) = ab;
            }
            else
                out[idx] = s.a[k];
            if (level == 0)
            {
                // Cells without an open face hold z = 0 and rhs = 0: they add nothing to either sum.
                tz += s.a[k];
                trz += s.ra[k] * s.a[k];
                if (in_b)
                {
                    tz += s.b[k];
                    trz += s.rb[k] * s.b[k];
                }
            }
        }
        if (level == 0)
        {
            // One (sum z, sum r z) pair per tile, the warps' sums added in warp order; the CTA
            // counts its tiles of this grid once, when its next tile belongs to another grid or
            // it has none left. warp_pairs is rewritten only after the next tile's barriers.
            double2* pairs = reinterpret_cast<double2*>(g.partial);
            // The warp's sums in the working precision (FP32: a fixed shuffle tree of 32 terms).
            const double wz = double(warp_sum(tz)), wrz = double(warp_sum(trz));
            if (lane == 0)
                warp_pairs[warp] = make_double2(wz, wrz);
            __syncthreads();
            if (threadIdx.x == 0)
            {
                double2 acc = warp_pairs[0];
#pragma unroll
                for (int w = 1; w < WARPS; ++w)
                {
                    acc.x += warp_pairs[w].x;
                    acc.y += warp_pairs[w].y;
                }
                pairs[t.index] = acc;
            }
            ++run;
            if (next >= count || n.grid != t.grid)
            {
                if (arrive_run<NT>(g, pairs, run, g.post_tiles, g.post_tiles, &total))
                {
                    // The strips hold r - mean r: sum r z = sum (r - mean r) z + mean r sum z.
                    if (threadIdx.x == 0)
                        finish_preconditioner(*state, total.x, total.y + state->mean_r * total.x);
                }
                run = 0;
            }
        }
        t = n;
    }
}

} // namespace fc
