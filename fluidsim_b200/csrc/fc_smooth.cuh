// Register strips: the building blocks of the temporally blocked red-black smoothing kernels
// (k_smooth_pre / k_smooth_post in fc_stage.cuh).
//
// A 256-thread CTA works on a region of 64 columns x 8K rows of a level. Warp w owns the K rows
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
// The red-black sweep is PressureMultigrid.cpp:204-231.
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

template <typename T, int K, bool PRE, int WARPS = 8> struct TileShape
{
    static constexpr int RX = 64;
    static constexpr int RY = WARPS * K;
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


// r - mean in the working precision (FP64 keeps the reference's exact subtraction).
__device__ __forceinline__ float minus_mean(float r, double mean) { return r - float(mean); }
__device__ __forceinline__ double minus_mean(double r, double mean) { return r - mean; }

__host__ __device__ inline int padded_index32(int S, int x, int y) { return (y + 1) * S + x + kPadX; }

template <typename T, int K> struct Strip
{
    T a[K], b[K];   // solution at columns 2j, 2j+1
    T ra[K], rb[K]; // right-hand side (zero where a cell has no open face)
    // The face between columns 2j-1 and 2j is the left lane's wr: its products come from there
    // by shuffle, which keeps eight registers per strip free.
    T wm[K];        // face between 2j and 2j+1
    T wr[K];        // face between 2j+1 and 2j+2
    T da[K], db[K]; // lower faces (row k to k+1)
    T ua, ub;       // upper faces of row 0
    T ia[K], ib[K]; // inverse diagonals
};

// Shared edge rows of the strips: [buffer][warp + 1][lane]; warps -1 and 8 stay zero.
template <typename T, int WARPS = 8> struct Edges
{
    T top[2][WARPS + 2][32];
    T bottom[2][WARPS + 2][32];
};

// Strip assembly: the staged loads (fc_stage.cuh) fill the weights, inverse diagonals and
// right-hand side; strip_finish masks the right-hand side (and on the fine level subtracts the
// residual's mean).
template <typename T, int K>
__device__ __forceinline__ void strip_finish(Strip<T, K>& s, int level, double mean_r)
{
#pragma unroll
    for (int k = 0; k < K; ++k)
    {
        // A cell with no open face takes no part (inside obstacles, a 1x1 grid, the padding):
        // its inverse diagonal is zero.
        if (level == 0)
        {
            s.ra[k] = s.ia[k] > T(0) ? minus_mean(s.ra[k], mean_r) : T(0);
            s.rb[k] = s.ib[k] > T(0) ? minus_mean(s.rb[k], mean_r) : T(0);
        }
        else
        {
            s.ra[k] = s.ia[k] > T(0) ? s.ra[k] : T(0);
            s.rb[k] = s.ib[k] > T(0) ? s.rb[k] : T(0);
        }
    }
}

// Barrier of the warps that hold strips: the whole CTA (threads == 0), or, where only the first
// threads / 32 warps hold a level's rows, those warps alone on named barrier 1 (threads a multiple
// of 32; every one of them reaches each barrier).
__device__ __forceinline__ void strips_barrier(int threads)
{
    if (threads == 0)
        __syncthreads();
    else
        asm volatile("bar.sync 1, %0;" ::"r"(threads) : "memory");
}

// One red-black half-sweep of colour c over the strip; publishes the strip's edge rows of that
// colour into buffer `buf` and reads the neighbours' edges from buffer buf ^ 1. `threads` selects
// the barrier (strips_barrier).
template <typename T, int K, int WARPS = 8>
__device__ __forceinline__ void strip_sweep(Strip<T, K>& s, Edges<T, WARPS>& e, int c, bool from_zero, int buf, int lane,
    int warp, int threads = 0)
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
                // wl * left, formed on the left lane as its wr * b (zero left of the region).
                T left = __shfl_up_sync(0xffffffffu, s.wr[k] * s.b[k], 1);
                left = lane == 0 ? T(0) : left;
                const T up = k == 0 ? above : s.a[k - 1];
                const T dn = k == K - 1 ? below : s.a[k + 1];
                const T wu = k == 0 ? s.ua : s.da[k - 1];
                s.a[k] = (s.ra[k] + ((left + s.wm[k] * s.b[k]) + (wu * up + s.da[k] * dn))) * s.ia[k];
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
    strips_barrier(threads);
}

template <typename T, int K, int WARPS = 8>
__device__ __forceinline__ void edges_clear(Edges<T, WARPS>& e)
{
    T* flat = &e.top[0][0][0];
    for (int i = threadIdx.x; i < int(sizeof(Edges<T, WARPS>) / sizeof(T)); i += blockDim.x)
        flat[i] = T(0);
}

// One axis of the transpose-bilinear restriction for coarse cell c: the weights of fine cells
// 2c-1, 2c, 2c+1, 2c+2 (bit p of `mask` set when fine cell 2c-1+p contributes). The table lists
// its fine cells in ascending order, so summing by offset keeps the table's order; the host
// checks that no entry falls outside the four offsets. The strip kernels read these per coarse
// cell precomputed (LevelDesc::rwx, rwy); the tail forms them from its staged tables.
template <typename T> struct alignas(16) RestrictAxis
{
    T w[4];
    unsigned mask;
};

template <typename T> __device__ __forceinline__ RestrictAxis<T> restrict_axis(const Gather* table, int c)
{
    RestrictAxis<T> r;
    r.mask = 0;
    const Gather g = table[c];
#pragma unroll
    for (int p = 0; p < 4; ++p)
    {
        r.w[p] = T(0);
#pragma unroll
        for (int e = 0; e < 4; ++e)
            if (e < g.count && g.index[e] == 2 * c - 1 + p)
            {
                r.w[p] = T(g.weight[e]);
                r.mask |= 1u << p;
            }
    }
    return r;
}

// sum over the set offsets of w[p] * v[p], accumulated in offset order from zero.
template <typename T>
__device__ __forceinline__ T restrict_sum(const RestrictAxis<T>& r, T v0, T v1, T v2, T v3)
{
    T s = T(0);
    if (r.mask & 1u)
        s += r.w[0] * v0;
    if (r.mask & 2u)
        s += r.w[1] * v1;
    if (r.mask & 4u)
        s += r.w[2] * v2;
    if (r.mask & 8u)
        s += r.w[3] * v3;
    return s;
}

} // namespace fc
