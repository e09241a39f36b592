// Semi-Lagrangian transport of the UniformCUDA step.
//
// The reference moves material with conservative PLIC transport (FluidGridCPU.cpp:362-463);
// this backend's step advects by second-order (midpoint) semi-Lagrangian back-tracing instead.
// Its building block is the reference's clamped bilinear sampler on the staggered grid
// (FluidGridCPU.cpp:67-90 sampleScalar, :465-471 sampleVelocity): u is sampled at (x, y - 1/2)
// of a (W+1) x H array, v at (x - 1/2, y) of a W x (H+1) array, cell fields at
// (x - 1/2, y - 1/2) of a W x H array, positions in cells from the grid corner.
//
// For a sample point p, with s = dt / dx and V the sampled velocity:
//   mid  = p - (s / 2) V(p)
//   back = p - s V(mid)
//   q_new(p) = q(back)
// Velocities and cell fields are traced through the velocity at the start of the step. The
// wall-normal faces of the outer boundary are written as zero; obstacle faces are left to the
// projection.
//
// Every multiply and add is an explicitly rounded double operation (no fused multiply-add), so
// the results equal an IEEE evaluation of the same expressions on the host bit for bit.
#pragma once

#include "fc_device.cuh"

namespace fc
{

// std::lerp as specified by P0811R3 and implemented by libstdc++: exact at both ends, monotonic,
// and never beyond b for t <= 1. FluidGridCPU.cpp:86-89 blends with it.
__device__ __forceinline__ double lerp_exact(double a, double b, double t)
{
    if ((a <= 0.0 && b >= 0.0) || (a >= 0.0 && b <= 0.0))
        return __dadd_rn(__dmul_rn(t, b), __dmul_rn(__dsub_rn(1.0, t), a));
    if (t == 1.0)
        return b;
    const double x = __dadd_rn(a, __dmul_rn(t, __dsub_rn(b, a)));
    return (t > 1.0) == (b > a) ? (b < x ? x : b) : (b > x ? x : b);
}

// std::clamp(x, lo, hi) for lo <= hi.
__device__ __forceinline__ double clamp_exact(double x, double lo, double hi)
{
    const double m = x < lo ? lo : x;
    return hi < m ? hi : m;
}

// FluidGridCPU.cpp:67-90: clamped bilinear sample of a row-major w x h array at fractional
// array index (x, y).
template <typename T>
__device__ __forceinline__ double sample_clamped(const T* data, int w, int h, double x, double y)
{
    x = clamp_exact(x, 0.0, double(w - 1));
    y = clamp_exact(y, 0.0, double(h - 1));
    const int x0 = int(x), y0 = int(y);
    const int x1 = min(x0 + 1, w - 1), y1 = min(y0 + 1, h - 1);
    const double tx = __dsub_rn(x, double(x0)), ty = __dsub_rn(y, double(y0));
    const double a00 = double(data[(long long)y0 * w + x0]), a10 = double(data[(long long)y0 * w + x1]);
    const double a01 = double(data[(long long)y1 * w + x0]), a11 = double(data[(long long)y1 * w + x1]);
    return lerp_exact(lerp_exact(a00, a10, tx), lerp_exact(a01, a11, tx), ty);
}

// FluidGridCPU.cpp:465-471 in cell units: velocity at (x, y) cells from the grid corner.
template <typename T>
__device__ __forceinline__ void sample_velocity(const T* u, const T* v, int W, int H, double x, double y, double& vx,
    double& vy)
{
    vx = sample_clamped(u, W + 1, H, x, __dsub_rn(y, 0.5));
    vy = sample_clamped(v, W, H + 1, __dsub_rn(x, 0.5), y);
}

// Midpoint back-trace from (x, y); half = s / 2 and s = dt / dx, both computed on the host.
template <typename T>
__device__ __forceinline__ void trace_back(const T* u, const T* v, int W, int H, double s, double half, double x,
    double y, double& bx, double& by)
{
    double vx, vy;
    sample_velocity(u, v, W, H, x, y, vx, vy);
    const double mx = __dsub_rn(x, __dmul_rn(half, vx)), my = __dsub_rn(y, __dmul_rn(half, vy));
    sample_velocity(u, v, W, H, mx, my, vx, vy);
    bx = __dsub_rn(x, __dmul_rn(s, vx));
    by = __dsub_rn(y, __dmul_rn(s, vy));
}

// New face velocities into u_next / v_next. The tiles cover the (W+1) x (H+1) face index space:
// point (i, j) is u face (i, j) when j < H and v face (i, j) when i < W.
template <typename T>
__global__ void k_advect_velocity(const GridDesc* __restrict__ grids, const Tile* __restrict__ tiles, double s,
    double half, T* __restrict__ u_next, T* __restrict__ v_next)
{
    const Tile t = tiles[blockIdx.x];
    const GridDesc& g = grids[t.grid];
    // The current velocities are read only; the new ones go to other arrays.
    const T* __restrict__ u = static_cast<const T*>(g.u);
    const T* __restrict__ v = static_cast<const T*>(g.v);
    const int W = g.W, H = g.H;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    for (int k = 0; k < kVecCells; ++k)
    {
        const int i = t.x0 + tx + 32 * (k & 1), j = t.y0 + ty + 8 * (k >> 1);
        if (i <= W && j < H)
        {
            double value = 0.0;
            if (i > 0 && i < W)
            {
                double bx, by;
                trace_back(u, v, W, H, s, half, double(i), __dadd_rn(double(j), 0.5), bx, by);
                value = sample_clamped(u, W + 1, H, bx, __dsub_rn(by, 0.5));
            }
            u_next[(long long)j * (W + 1) + i] = T(value);
        }
        if (i < W && j <= H)
        {
            double value = 0.0;
            if (j > 0 && j < H)
            {
                double bx, by;
                trace_back(u, v, W, H, s, half, __dadd_rn(double(i), 0.5), double(j), bx, by);
                value = sample_clamped(v, W, H + 1, __dsub_rn(bx, 0.5), by);
            }
            v_next[(long long)j * W + i] = T(value);
        }
    }
}

// One cell-centred FP64 field (liquid fraction or a component mass) into `next`.
template <typename T>
__global__ void k_advect_cells(const GridDesc* __restrict__ grids, const Tile* __restrict__ tiles, double s, double half,
    const double* __restrict__ field, double* __restrict__ next)
{
    const Tile t = tiles[blockIdx.x];
    const GridDesc& g = grids[t.grid];
    const T* __restrict__ u = static_cast<const T*>(g.u);
    const T* __restrict__ v = static_cast<const T*>(g.v);
    const int W = g.W, H = g.H;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    for (int k = 0; k < kVecCells; ++k)
    {
        const int i = t.x0 + tx + 32 * (k & 1), j = t.y0 + ty + 8 * (k >> 1);
        if (i >= W || j >= H)
            continue;
        double bx, by;
        trace_back(u, v, W, H, s, half, __dadd_rn(double(i), 0.5), __dadd_rn(double(j), 0.5), bx, by);
        next[(long long)j * W + i] = sample_clamped(field, W, H, __dsub_rn(bx, 0.5), __dsub_rn(by, 0.5));
    }
}

// FluidGridCPU::sampleVelocity (FluidGridCPU.cpp:465-471) at world positions: positions and
// velocities are interleaved (x, y) pairs.
template <typename T>
__global__ void k_sample_velocity(const T* u, const T* v, int W, int H, double origin_x, double origin_y,
    double cell_size, int count, const double* positions, double* velocities)
{
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= count)
        return;
    const double x = __ddiv_rn(__dsub_rn(positions[2 * n], origin_x), cell_size);
    const double y = __ddiv_rn(__dsub_rn(positions[2 * n + 1], origin_y), cell_size);
    sample_velocity(u, v, W, H, x, y, velocities[2 * n], velocities[2 * n + 1]);
}

} // namespace fc
