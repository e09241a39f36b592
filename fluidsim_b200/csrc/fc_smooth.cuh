// Temporally blocked red-black smoothing of one multigrid level (the V-cycle's hot kernels).
//
// A 256-thread CTA stages a region of 64 columns x 8K rows of a level. Warp w owns the K rows
// [wK, wK + K) of all 64 columns; lane j owns columns 2j ("a") and 2j+1 ("b"). Every cell's
// solution, right-hand side, face weights and inverse diagonal live in registers:
//  * the upper/lower neighbours of a cell are the same thread's adjacent rows;
//  * the left/right neighbour across the column pair is one warp shuffle;
//  * only the first and last row of each warp's strip cross warps, through two small
//    double-buffered shared-memory edge arrays, with one barrier per half-sweep.
// A half-sweep is then four FMAs, one multiply and one shuffle per updated cell.
//
// Region origins are even and K is even, so column 2j of region row k has colour k & 1 in the
// level's red-black colouring (x + y) & 1 (PressureMultigrid.cpp:216).
//
// k_mg_pre: four sweeps (the first from zero), then the residual and its transpose-bilinear
// restriction straight into the coarse right-hand side (PressureMultigrid.cpp:398-402,
// 204-231, 233-276). k_mg_post: the bilinear prolongation of the coarse solution added to the
// pre-smoothed one, four sweeps in reversed colour order, and on the fine level sum(z) and r.z
// (PressureMultigrid.cpp:403-407, 278-298; FluidGridCPU.cpp:1712-1726).
#pragma once

#include "fc_device.cuh"

namespace fc
{

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
    static_assert(K % 2 == 0, "strip height must be even");
    static_assert(OY > 0, "strip too short for the halo");
};

template <typename T> struct Pair;
template <> struct Pair<float>
{
    using type = float2;
};
template <> struct Pair<double>
{
    using type = double2;
};

__device__ __forceinline__ float reciprocal(float v) { return __frcp_rn(v); }
__device__ __forceinline__ double reciprocal(double v) { return 1.0 / v; }

// r - mean in the working precision (FP64 keeps the reference's exact subtraction).
__device__ __forceinline__ float minus_mean(float r, double mean) { return r - float(mean); }
__device__ __forceinline__ double minus_mean(double r, double mean) { return r - mean; }

__host__ __device__ inline int padded_index32(int S, int x, int y) { return (y + 1) * S + x + kPadX; }

template <typename T, int K> struct Strip
{
    T a[K], b[K];   // solution at columns 2j, 2j+1
    T ra[K], rb[K]; // right-hand side (zero where a cell has no open face)
    T wl[K];        // face between columns 2j-1 and 2j
    T wm[K];        // face between 2j and 2j+1
    T wr[K];        // face between 2j+1 and 2j+2
    T da[K], db[K]; // lower faces (row k to k+1)
    T ua, ub;       // upper faces of row 0
    T ia[K], ib[K]; // inverse diagonals
};

// Shared edge rows of the strips: [buffer][warp + 1][lane]; warps -1 and 8 stay zero.
template <typename T> struct Edges
{
    T top[2][10][32];
    T bottom[2][10][32];
};

// Strip loading in three steps: strip_weights issues the face-weight loads (no kernel of the
// projection writes them, so before the wait on the previous kernel), strip_rhs issues the
// right-hand side loads (after the wait), strip_finish forms the left weights, inverse
// diagonals and the right-hand side once the loads have landed. Callers issue their other
// loads between strip_rhs and strip_finish so that all of them are in flight together.
template <typename T, int K> struct StripRaw
{
    T wl0[K];
};

// Face weights of the strip. With kHalf (mixed precision, T = float) they come from the level's
// FP16 copies and are scaled back by wscale; the arithmetic stays FP32.
template <typename T, int K, bool kHalf = false>
__device__ __forceinline__ void strip_weights(Strip<T, K>& s, StripRaw<T, K>& raw, const LevelDesc& L, int X0, int Y0,
    int lane, int warp)
{
    using P = typename Pair<T>::type;
    const int gx = X0 + 2 * lane;
    // The pair (gx, gx + 1) is either wholly inside the padded row [0, S) or wholly outside.
    const bool cols = gx + kPadX >= 0 && gx + kPadX + 1 < L.S;
    const bool left_col = gx + kPadX - 1 >= 0 && gx + kPadX - 1 < L.S;
    const int y0 = Y0 + warp * K;
    if constexpr (kHalf)
    {
        static_assert(sizeof(T) == 4, "FP16 weights feed FP32 smoothing");
        const __half* right = static_cast<const __half*>(L.right_h);
        const __half* down = static_cast<const __half*>(L.down_h);
        const float scale = L.wscale;
#pragma unroll
        for (int k = 0; k < K; ++k)
        {
            const int gy = y0 + k;
            const bool in = cols && gy >= -1 && gy <= L.h;
            const int i = padded_index32(L.S, gx, gy);
            float2 w2 = make_float2(0.f, 0.f), d2 = make_float2(0.f, 0.f);
            if (in)
            {
                w2 = __half22float2(*reinterpret_cast<const __half2*>(right + i));
                d2 = __half22float2(*reinterpret_cast<const __half2*>(down + i));
            }
            s.wm[k] = w2.x * scale;
            s.wr[k] = w2.y * scale;
            s.da[k] = d2.x * scale;
            s.db[k] = d2.y * scale;
            raw.wl0[k] = (lane == 0 && left_col && gy >= -1 && gy <= L.h) ? __half2float(right[i - 1]) * scale : T(0);
        }
        float2 u2 = make_float2(0.f, 0.f);
        if (cols && y0 - 1 >= -1 && y0 - 1 <= L.h)
            u2 = __half22float2(*reinterpret_cast<const __half2*>(down + padded_index32(L.S, gx, y0 - 1)));
        s.ua = u2.x * scale;
        s.ub = u2.y * scale;
    }
    else
    {
        const T* right = static_cast<const T*>(L.right);
        const T* down = static_cast<const T*>(L.down);
#pragma unroll
        for (int k = 0; k < K; ++k)
        {
            const int gy = y0 + k;
            const bool in = cols && gy >= -1 && gy <= L.h;
            const int i = padded_index32(L.S, gx, gy);
            P w2 = P{}, d2 = P{};
            if (in)
            {
                w2 = *reinterpret_cast<const P*>(right + i);
                d2 = *reinterpret_cast<const P*>(down + i);
            }
            s.wm[k] = w2.x;
            s.wr[k] = w2.y;
            s.da[k] = d2.x;
            s.db[k] = d2.y;
            raw.wl0[k] = (lane == 0 && left_col && gy >= -1 && gy <= L.h) ? right[i - 1] : T(0);
        }
        P u2 = P{};
        if (cols && y0 - 1 >= -1 && y0 - 1 <= L.h)
            u2 = *reinterpret_cast<const P*>(down + padded_index32(L.S, gx, y0 - 1));
        s.ua = u2.x;
        s.ub = u2.y;
    }
}

template <typename T, int K>
__device__ __forceinline__ void strip_rhs(Strip<T, K>& s, const GridDesc& g, const LevelDesc& L, int level, int X0,
    int Y0, int lane, int warp)
{
    using P = typename Pair<T>::type;
    const T* rhs = level == 0 ? static_cast<const T*>(g.r) : static_cast<const T*>(L.rhs);
    const int gx = X0 + 2 * lane;
    const bool cols = gx + kPadX >= 0 && gx + kPadX + 1 < L.S;
    const int y0 = Y0 + warp * K;
#pragma unroll
    for (int k = 0; k < K; ++k)
    {
        const int gy = y0 + k;
        P r2 = P{};
        if (cols && gy >= -1 && gy <= L.h)
            r2 = *reinterpret_cast<const P*>(rhs + padded_index32(L.S, gx, gy));
        s.ra[k] = r2.x;
        s.rb[k] = r2.y;
    }
}

template <typename T, int K>
__device__ __forceinline__ void strip_finish(Strip<T, K>& s, const StripRaw<T, K>& raw, int level, int lane, double mean_r)
{
#pragma unroll
    for (int k = 0; k < K; ++k)
    {
        const T shifted = __shfl_up_sync(0xffffffffu, s.wr[k], 1);
        s.wl[k] = lane == 0 ? raw.wl0[k] : shifted;
        const T up_a = k == 0 ? s.ua : s.da[k - 1];
        const T up_b = k == 0 ? s.ub : s.db[k - 1];
        const T diag_a = ((s.wl[k] + s.wm[k]) + up_a) + s.da[k];
        const T diag_b = ((s.wm[k] + s.wr[k]) + up_b) + s.db[k];
        s.ia[k] = diag_a > T(0) ? reciprocal(diag_a) : T(0);
        s.ib[k] = diag_b > T(0) ? reciprocal(diag_b) : T(0);
        // A cell with no open face takes no part (inside obstacles, a 1x1 grid, the padding).
        if (level == 0)
        {
            s.ra[k] = diag_a > T(0) ? minus_mean(s.ra[k], mean_r) : T(0);
            s.rb[k] = diag_b > T(0) ? minus_mean(s.rb[k], mean_r) : T(0);
        }
        else
        {
            s.ra[k] = diag_a > T(0) ? s.ra[k] : T(0);
            s.rb[k] = diag_b > T(0) ? s.rb[k] : T(0);
        }
    }
}

// One red-black half-sweep of colour c over the strip; publishes the strip's edge rows of that
// colour into buffer `buf` and reads the neighbours' edges from buffer buf ^ 1.
template <typename T, int K>
__device__ __forceinline__ void strip_sweep(Strip<T, K>& s, Edges<T>& e, int c, bool from_zero, int buf, int lane,
    int warp)
{
    const T above = from_zero ? T(0) : e.bottom[buf ^ 1][warp][lane];
    const T below = from_zero ? T(0) : e.top[buf ^ 1][warp + 2][lane];
#pragma unroll
    for (int k = 0; k < K; ++k)
    {
        if ((k & 1) == c)
        {
            if (from_zero)
                s.a[k] = s.ra[k] * s.ia[k];
            else
            {
                T left = __shfl_up_sync(0xffffffffu, s.b[k], 1);
                left = lane == 0 ? T(0) : left;
                const T up = k == 0 ? above : s.a[k - 1];
                const T dn = k == K - 1 ? below : s.a[k + 1];
                const T wu = k == 0 ? s.ua : s.da[k - 1];
                s.a[k] = (s.ra[k] + ((s.wl[k] * left + s.wm[k] * s.b[k]) + (wu * up + s.da[k] * dn))) * s.ia[k];
            }
        }
        else
        {
            if (from_zero)
                s.b[k] = s.rb[k] * s.ib[k];
            else
            {
                T right = __shfl_down_sync(0xffffffffu, s.a[k], 1);
                right = lane == 31 ? T(0) : right;
                const T up = k == 0 ? above : s.b[k - 1];
                const T dn = k == K - 1 ? below : s.b[k + 1];
                const T wu = k == 0 ? s.ub : s.db[k - 1];
                s.b[k] = (s.rb[k] + ((s.wm[k] * s.a[k] + s.wr[k] * right) + (wu * up + s.db[k] * dn))) * s.ib[k];
            }
        }
    }
    // Row 0 is even: colour c sits in a when c == 0. Row K-1 is odd: in a when c == 1.
    e.top[buf][warp + 1][lane] = c == 0 ? s.a[0] : s.b[0];
    e.bottom[buf][warp + 1][lane] = c == 1 ? s.a[K - 1] : s.b[K - 1];
    __syncthreads();
}

template <typename T, int K>
__device__ __forceinline__ void edges_clear(Edges<T>& e)
{
    T* flat = &e.top[0][0][0];
    for (int i = threadIdx.x; i < int(sizeof(Edges<T>) / sizeof(T)); i += blockDim.x)
        flat[i] = T(0);
}

template <typename T, int K, bool kHalf = false>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 2 : 1) k_mg_pre(const GridDesc* grids, const Tile* tiles, int level)
{
    using Shape = TileShape<T, K, true>;
    allow_dependents();
    const Tile t = tiles[blockIdx.x];
    const GridDesc& g = grids[t.grid];
    const LevelDesc& L = g.lev[level];
    const LevelDesc& C = g.lev[level + 1];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int X0 = t.x0 - Shape::HALO, Y0 = t.y0 - Shape::HALO;

    __shared__ Edges<T> edges;
    __shared__ T res[Shape::RY][Shape::RX];
    constexpr int OCX = Shape::OX / 2, OCY = Shape::OY / 2;
    __shared__ Gather gather_x[OCX], gather_y[OCY];
    const int cx0 = t.x0 / 2, cy0 = t.y0 / 2;
    // The restriction tables of the tile's coarse cells, fetched while the strips load.
    if (threadIdx.x < OCX)
    {
        const int cx = cx0 + threadIdx.x;
        if (cx < C.w)
            gather_x[threadIdx.x] = L.rx[cx];
    }
    else if (threadIdx.x < OCX + OCY)
    {
        const int cy = cy0 + int(threadIdx.x) - OCX;
        if (cy < C.h)
            gather_y[threadIdx.x - OCX] = L.ry[cy];
    }
    edges_clear<T, K>(edges);
    Strip<T, K> s;
    StripRaw<T, K> raw;
    strip_weights<T, K, kHalf>(s, raw, L, X0, Y0, lane, warp);
    dependency_wait();
    if (g.state->done)
        return;
    strip_rhs<T, K>(s, g, L, level, X0, Y0, lane, warp);
    strip_finish<T, K>(s, raw, level, lane, level == 0 ? g.state->mean_r : 0.0);
#pragma unroll
    for (int k = 0; k < K; ++k)
        s.a[k] = s.b[k] = T(0);
    __syncthreads();

    strip_sweep<T, K>(s, edges, 0, true, 0, lane, warp);
    strip_sweep<T, K>(s, edges, 1, false, 1, lane, warp);
#pragma unroll 1
    for (int sweep = 1; sweep < 4; ++sweep)
    {
        strip_sweep<T, K>(s, edges, 0, false, 0, lane, warp);
        strip_sweep<T, K>(s, edges, 1, false, 1, lane, warp);
    }

    // Residual of every cell (zero where the cell has no open face), into shared memory; the
    // edge buffers now hold the final values: buffer 0 colour 0, buffer 1 colour 1.
    const T above_a = edges.bottom[1][warp][lane], above_b = edges.bottom[0][warp][lane];
    const T below_a = edges.top[0][warp + 2][lane], below_b = edges.top[1][warp + 2][lane];
    T* pre = static_cast<T*>(L.pre);
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
        const T na = k == K - 1 ? below_a : s.a[k + 1];
        const T nb = k == K - 1 ? below_b : s.b[k + 1];
        const T wua = k == 0 ? s.ua : s.da[k - 1];
        const T wub = k == 0 ? s.ub : s.db[k - 1];
        const T a = s.a[k], b = s.b[k];
        const T pa = (s.wl[k] * (a - left) + s.wm[k] * (a - b)) + (wua * (a - ua) + s.da[k] * (a - na));
        const T pb = (s.wm[k] * (b - a) + s.wr[k] * (b - right)) + (wub * (b - ub) + s.db[k] * (b - nb));
        const int y = warp * K + k;
        typename Pair<T>::type rr;
        rr.x = s.ia[k] > T(0) ? s.ra[k] - pa : T(0);
        rr.y = s.ib[k] > T(0) ? s.rb[k] - pb : T(0);
        *reinterpret_cast<typename Pair<T>::type*>(&res[y][2 * lane]) = rr;
        // The pre-smoothed solution of the tile's output cells, for the post-smoothing.
        const int gy = Y0 + y;
        if (y >= Shape::HALO && y < Shape::HALO + Shape::OY && 2 * lane >= Shape::HALO &&
            2 * lane < Shape::HALO + Shape::OX && gy < L.h && gx < L.w)
        {
            const int i = padded_index32(L.S, gx, gy);
            if (gx + 1 < L.w)
            {
                typename Pair<T>::type ab;
                ab.x = a;
                ab.y = b;
                *reinterpret_cast<typename Pair<T>::type*>(pre + i) = ab;
            }
            else
                pre[i] = a;
        }
    }
    __syncthreads();

    // Transpose-bilinear restriction onto the tile's coarse cells.
    T* crhs = static_cast<T*>(C.rhs);
    for (int q = threadIdx.x; q < OCX * OCY; q += 256)
    {
        const int qx = q % OCX, qy = q / OCX;
        const int cx = cx0 + qx, cy = cy0 + qy;
        if (cx >= C.w || cy >= C.h)
            continue;
        const Gather& gxr = gather_x[qx];
        const Gather& gyr = gather_y[qy];
        T value = T(0);
        for (int iy = 0; iy < gyr.count; ++iy)
        {
            const int y = gyr.index[iy] - Y0;
            T line = T(0);
            for (int ix = 0; ix < gxr.count; ++ix)
                line += T(gxr.weight[ix]) * res[y][gxr.index[ix] - X0];
            value += T(gyr.weight[iy]) * line;
        }
        crhs[padded_index32(C.S, cx, cy)] = value;
    }
}

template <typename T, int K, bool kHalf = false>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 2 : 1) k_mg_post(const GridDesc* grids, const Tile* tiles, int level)
{
    using Shape = TileShape<T, K, false>;
    constexpr int CW = 36, CH = Shape::RY / 2 + 4;
    allow_dependents();
    const Tile t = tiles[blockIdx.x];
    const GridDesc& g = grids[t.grid];
    SolveState& state = *g.state;
    const LevelDesc& L = g.lev[level];
    const LevelDesc& C = g.lev[level + 1];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int X0 = t.x0 - Shape::HALO, Y0 = t.y0 - Shape::HALO;
    const int CX0 = X0 / 2 - 1, CY0 = Y0 / 2 - 1;

    __shared__ Edges<T> edges;
    __shared__ T coarse[CH][CW];
    __shared__ Interp interp_y[Shape::RY];
    // Tables and weights first (written by no kernel of the projection); after the wait the
    // right-hand side, the coarse solution under the region (cells outside the coarse level
    // read 0) and the pre-smoothed values are all requested before any of them is used.
    Interp iy{0, 0, 0.0};
    if (threadIdx.x < Shape::RY)
    {
        const int gy = Y0 + int(threadIdx.x);
        if (gy >= 0 && gy < L.h)
            iy = L.py[gy];
    }
    Strip<T, K> s;
    StripRaw<T, K> raw;
    strip_weights<T, K, kHalf>(s, raw, L, X0, Y0, lane, warp);
    dependency_wait();
    if (state.done)
        return;
    strip_rhs<T, K>(s, g, L, level, X0, Y0, lane, warp);
    const double mean_r = level == 0 ? state.mean_r : 0.0;
    const T* csol = static_cast<const T*>(C.sol);
    constexpr int STAGE = (CH * CW + 255) / 256;
    T staged[STAGE];
#pragma unroll
    for (int u = 0; u < STAGE; ++u)
    {
        const int q = threadIdx.x + 256 * u;
        const int cx = CX0 + q % CW, cy = CY0 + q / CW;
        staged[u] = (q < CH * CW && cx >= 0 && cx < C.w && cy >= 0 && cy < C.h) ? csol[padded_index32(C.S, cx, cy)] : T(0);
    }
    // The pre-smoothed values of the strip.
    const T* pre = static_cast<const T*>(L.pre);
    const int gx = X0 + 2 * lane;
    const bool in_a = gx >= 0 && gx < L.w, in_b = gx + 1 >= 0 && gx + 1 < L.w;
    Interp pa{0, 0, 0.0}, pb{0, 0, 0.0};
    if (in_a)
        pa = L.px[gx];
    if (in_b)
        pb = L.px[gx + 1];
#pragma unroll
    for (int k = 0; k < K; ++k)
    {
        const int gy = Y0 + warp * K + k;
        s.a[k] = s.b[k] = T(0);
        if (gy < 0 || gy >= L.h)
            continue;
        const int i = padded_index32(L.S, gx, gy);
        if (in_a)
            s.a[k] = pre[i];
        if (in_b)
            s.b[k] = pre[i + 1];
    }
    strip_finish<T, K>(s, raw, level, lane, mean_r);
#pragma unroll
    for (int u = 0; u < STAGE; ++u)
    {
        const int q = threadIdx.x + 256 * u;
        if (q < CH * CW)
            coarse[q / CW][q % CW] = staged[u];
    }
    if (threadIdx.x < Shape::RY)
        interp_y[threadIdx.x] = iy;
    edges_clear<T, K>(edges);
    __syncthreads();

    // Add the prolonged coarse correction, in-level cells only.
    const T wxa = T(pa.weight), wxb = T(pb.weight);
    const int fa = pa.first - CX0, sa = pa.second - CX0, fb = pb.first - CX0, sb = pb.second - CX0;
#pragma unroll
    for (int k = 0; k < K; ++k)
    {
        const int gy = Y0 + warp * K + k;
        if (gy < 0 || gy >= L.h)
            continue;
        const Interp& py = interp_y[warp * K + k];
        const int top = py.first - CY0, bottom = py.second - CY0;
        const T wy = T(py.weight);
        if (in_a)
        {
            const T u = (T(1) - wxa) * coarse[top][fa] + wxa * coarse[top][sa];
            const T d = (T(1) - wxa) * coarse[bottom][fa] + wxa * coarse[bottom][sa];
            s.a[k] = s.a[k] + ((T(1) - wy) * u + wy * d);
        }
        if (in_b)
        {
            const T u = (T(1) - wxb) * coarse[top][fb] + wxb * coarse[top][sb];
            const T d = (T(1) - wxb) * coarse[bottom][fb] + wxb * coarse[bottom][sb];
            s.b[k] = s.b[k] + ((T(1) - wy) * u + wy * d);
        }
    }
    // The first half-sweep (colour 1) reads colour-0 edges from buffer 1.
    edges.top[1][warp + 1][lane] = s.a[0];
    edges.bottom[1][warp + 1][lane] = s.b[K - 1];
    __syncthreads();

#pragma unroll 1
    for (int sweep = 0; sweep < 4; ++sweep)
    {
        strip_sweep<T, K>(s, edges, 1, false, 0, lane, warp);
        strip_sweep<T, K>(s, edges, 0, false, 1, lane, warp);
    }

    T* out = static_cast<T*>(L.sol);
    double sz = 0.0, srz = 0.0;
    const bool cols_out = 2 * lane >= Shape::HALO && 2 * lane < Shape::HALO + Shape::OX;
#pragma unroll
    for (int k = 0; k < K; ++k)
    {
        const int y = warp * K + k;
        const int gy = Y0 + y;
        if (!cols_out || y < Shape::HALO || y >= Shape::HALO + Shape::OY || gy >= L.h || !in_a)
            continue;
        const int i = padded_index32(L.S, gx, gy);
        if (in_b)
        {
            typename Pair<T>::type ab;
            ab.x = s.a[k];
            ab.y = s.b[k];
            *reinterpret_cast<typename Pair<T>::type*>(out + i) = ab;
        }
        else
            out[i] = s.a[k];
        if (level == 0)
        {
            // Cells without an open face hold z = 0 and rhs = 0: they add nothing to either sum.
            sz += double(s.a[k]);
            srz += double(s.ra[k]) * double(s.a[k]);
            if (in_b)
            {
                sz += double(s.b[k]);
                srz += double(s.rb[k]) * double(s.b[k]);
            }
        }
    }
    if (level != 0)
        return;
    __shared__ double4 total;
    if (arrive_last<256>(g, t.index, g.post_tiles, block_reduce4<256>(make_double4(sz, srz, 0, 0), 0), &total, 0))
    {
        // The strips hold r - mean r: sum r z = sum (r - mean r) z + mean r sum z.
        if (threadIdx.x == 0)
            finish_preconditioner(state, total.x, total.y + state.mean_r * total.x);
    }
}

} // namespace fc
