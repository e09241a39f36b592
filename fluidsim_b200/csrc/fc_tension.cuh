// Surface tension of the UniformCUDA step: height-function curvature and the capillary face
// force, FP64 throughout.
//
// Follows FluidSim/UniformCPU/FluidSurfaceTensionCPU.h (three ordered sweeps: heights, local
// curvature, completion of missing curvature) and FluidGridCPU.cpp:890-926 (the face force
// u += dt w sigma kappa_f (f_R - f_L) / dx with the pressure face weights w). The MYC normal
// and the PLIC offset are those of FluidSim/Shared/Adaptive/FluidInterfaceGeometry.h:14-61.
// Each sweep is one kernel with one thread per cell; each reads only the previous sweep's
// output, so the three launches reproduce the reference's ordered passes.
#pragma once

#include "fc_device.cuh"

namespace fc
{

struct TensionArrays
{
    double2* height;        // height along x and along y, in cells (FluidSurfaceTensionCPU::Height)
    signed char* orient;    // 2 per cell: orientation_x, orientation_y in {-1, 0, 1}
    double* raw;            // curvature from the local sweep
    unsigned char* raw_ok;
    double* kappa;          // completed curvature
    unsigned char* kappa_ok;
};

struct Vec2d
{
    double x, y;
};

// Even reflection about the walls (FluidSurfaceTensionCPU.h:45-50).
__device__ __forceinline__ int mirror_cell(int i, int extent)
{
    const int period = 2 * extent;
    const int q = ((i % period) + period) % period;
    return q >= extent ? period - 1 - q : q;
}

// Fraction with walls mirrored and near-pure cells snapped (FluidSurfaceTensionCPU.h:52-67).
__device__ __forceinline__ double geometry_fraction(const double* f, int W, int H, int x, int y)
{
    const double value = f[(long long)mirror_cell(y, H) * W + mirror_cell(x, W)];
    const double roundoff = 32.0 * 2.220446049250313e-16; // 32 machine epsilons of double
    if (value <= roundoff)
        return 0.0;
    if (value >= 1.0 - roundoff)
        return 1.0;
    return value;
}

__device__ __forceinline__ bool interfacial_cell(const double* f, int W, int H, int x, int y)
{
    const double c = geometry_fraction(f, W, H, x, y);
    if (c > 0.0 && c < 1.0)
        return true;
    const double around[4] = {geometry_fraction(f, W, H, x - 1, y), geometry_fraction(f, W, H, x + 1, y),
        geometry_fraction(f, W, H, x, y - 1), geometry_fraction(f, W, H, x, y + 1)};
    for (double n : around)
        if ((c >= 1.0 && n <= 0.0) || (c <= 0.0 && n >= 1.0))
            return true;
    return false;
}

// MYC normal of the 3x3 stencil around (x, y) (FluidInterfaceGeometry.h:14-50): the centred
// height estimate, or Youngs' gradient where that is steeper.
__device__ __forceinline__ Vec2d myc_normal(const double* f, int W, int H, int x, int y)
{
    auto s = [&](int dx, int dy) { return geometry_fraction(f, W, H, x + dx, y + dy); };
    const double tl = s(-1, -1), t = s(0, -1), tr = s(1, -1);
    const double l = s(-1, 0), r = s(1, 0);
    const double bl = s(-1, 1), b = s(0, 1), br = s(1, 1);
    const double left = tl + l + bl, right = tr + r + br;
    const double top = tl + t + tr, bottom = bl + b + br;
    Vec2d centred{0.5 * (left - right), 0.5 * (top - bottom)};
    const Vec2d youngs{left + l - right - r, top + t - bottom - b};
    if (centred.x == 0.0 && centred.y == 0.0)
        return youngs.x == 0.0 && youngs.y == 0.0 ? Vec2d{1.0, 0.0} : youngs;
    if (fabs(centred.x) <= fabs(centred.y))
    {
        centred.y = copysign(1.0, centred.y);
        if (fabs(youngs.x) > fabs(centred.x * youngs.y))
            return youngs;
    }
    else
    {
        centred.x = copysign(1.0, centred.x);
        if (fabs(youngs.y) > fabs(centred.y * youngs.x))
            return youngs;
    }
    return centred;
}

// Unit outward normal (FluidSurfaceTensionCPU.h:88-100).
__device__ __forceinline__ Vec2d outward_normal(const double* f, int W, int H, int x, int y)
{
    Vec2d n = myc_normal(f, W, H, x, y);
    const double magnitude = fmax(fabs(n.x), fabs(n.y));
    n.x /= magnitude;
    n.y /= magnitude;
    const double length = sqrt(n.x * n.x + n.y * n.y);
    return {n.x / length, n.y / length};
}

// PLIC line offset for a normal and a fraction (FluidInterfaceGeometry.h:52-61).
__device__ __forceinline__ double plic_offset(Vec2d n, double fraction)
{
    const double a = fmin(fabs(n.x), fabs(n.y));
    const double b = fmax(fabs(n.x), fabs(n.y));
    const double triangle = 0.5 * a / b;
    const double cut = fraction < triangle ? sqrt(2.0 * a * b * fraction)
                       : fraction <= 1.0 - triangle ? b * fraction + 0.5 * a
                                                    : a + b - sqrt(2.0 * a * b * (1.0 - fraction));
    return fmin(n.x, 0.0) + fmin(n.y, 0.0) + cut;
}

// Height of the interface nearest to the cell along one axis, from a 9-cell column
// (FluidSurfaceTensionCPU.h:102-136). Returns the height and its orientation (+1 liquid below
// the interface along the axis, -1 above, 0 none).
__device__ __forceinline__ void column_height(const double* f, int W, int H, int x, int y, int ax, int ay, double& h,
    double& orientation)
{
    int start = -4;
    double base = geometry_fraction(f, W, H, x - 4 * ax, y - 4 * ay);
    bool have = base <= 0.0 || base >= 1.0;
    base = base >= 1.0 ? 1.0 : 0.0;
    double sum = 0.0, nearest = 10.0;
    h = 0.0;
    orientation = 0.0;
    for (int k = -3; k <= 4; ++k)
    {
        const double c = geometry_fraction(f, W, H, x + k * ax, y + k * ay);
        if (c <= 0.0 || c >= 1.0)
        {
            const double pure = c >= 1.0 ? 1.0 : 0.0;
            if (have && pure != base)
            {
                const double candidate = start + 0.5 + (base == 1.0 ? sum : (k - start - 1) - sum);
                if (fabs(candidate) < nearest)
                {
                    nearest = fabs(candidate);
                    h = candidate;
                    orientation = base == 1.0 ? 1.0 : -1.0;
                }
            }
            start = k;
            base = pure;
            have = true;
            sum = 0.0;
        }
        else
            sum += c;
    }
}

struct HeightSample
{
    double x, y, ox, oy;
};

// Height record of a possibly mirrored cell (FluidSurfaceTensionCPU.h:161-178).
__device__ __forceinline__ HeightSample height_at(const TensionArrays& a, int W, int H, int x, int y)
{
    const long long i = (long long)mirror_cell(y, H) * W + mirror_cell(x, W);
    const double2 h = a.height[i];
    HeightSample s{h.x, h.y, double(a.orient[2 * i]), double(a.orient[2 * i + 1])};
    if (x < 0 || x >= W)
    {
        s.x = -s.x;
        s.ox = -s.ox;
    }
    if (y < 0 || y >= H)
    {
        s.y = -s.y;
        s.oy = -s.oy;
    }
    return s;
}

__device__ __forceinline__ double clamp_range(double k, double lo, double hi)
{
    return k < lo ? lo : (hi < k ? hi : k);
}

// Curvature from three consistent heights across the tangent (FluidSurfaceTensionCPU.h:180-201).
__device__ __forceinline__ bool height_curvature(const TensionArrays& a, int W, int H, int x, int y, bool horizontal,
    double cell_size, double& kappa)
{
    const int tx = horizontal ? 0 : 1, ty = horizontal ? 1 : 0;
    const HeightSample p = height_at(a, W, H, x - tx, y - ty);
    const HeightSample q = height_at(a, W, H, x, y);
    const HeightSample r = height_at(a, W, H, x + tx, y + ty);
    const double orientation = horizontal ? q.ox : q.oy;
    if (orientation == 0.0 || (horizontal ? p.ox : p.oy) != orientation || (horizontal ? r.ox : r.oy) != orientation)
        return false;
    const double left = horizontal ? p.x : p.y;
    const double mid = horizontal ? q.x : q.y;
    const double right = horizontal ? r.x : r.y;
    const double slope = 0.5 * (right - left);
    const double second = (right - mid) - (mid - left);
    const double k = -orientation * second / pow(1.0 + slope * slope, 1.5);
    kappa = clamp_range(k, -1.0, 1.0) / cell_size;
    return true;
}

// Weighted least-squares parabola in the frame of the normal (FluidSurfaceTensionCPU.h:203-250).
struct ParabolaFit
{
    double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0, s4 = 0.0, y0 = 0.0, y1 = 0.0, y2 = 0.0;

    __device__ void add(double px, double py, Vec2d n, double weight)
    {
        const double x = -px * n.y + py * n.x;
        const double y = px * n.x + py * n.y;
        const double x2 = x * x;
        s0 += weight;
        s1 += weight * x;
        s2 += weight * x2;
        s3 += weight * x2 * x;
        s4 += weight * x2 * x2;
        y0 += weight * y;
        y1 += weight * x * y;
        y2 += weight * x2 * y;
    }

    __device__ bool evaluate(double cell_size, double& kappa) const
    {
        if (s0 == 0.0)
            return false;
        const double a = s2 - s1 * s1 / s0;
        const double b = s3 - s1 * s2 / s0;
        const double c = s4 - s2 * s2 / s0;
        const double d = y1 - s1 * y0 / s0;
        const double e = y2 - s2 * y0 / s0;
        const double determinant = a * c - b * b;
        if (determinant <= 1e-5 * fmax(a * c, 1e-12))
            return false;
        const double quadratic = (a * e - b * d) / determinant;
        const double slope = (c * d - b * e) / determinant;
        const double k = -2.0 * quadratic / pow(1.0 + slope * slope, 1.5);
        kappa = clamp_range(k, -2.0, 2.0) / cell_size;
        return true;
    }
};

// Centre and length of the PLIC segment of a cell, relative to the cell centre
// (FluidSurfaceTensionCPU.h:286-325). Returns length 0 when the line misses the cell.
__device__ __forceinline__ void plic_segment(const double* f, int W, int H, int x, int y, Vec2d n, double& sx,
    double& sy, double& length)
{
    const double offset = plic_offset(n, geometry_fraction(f, W, H, x, y));
    double low = 10.0, high = -10.0;
    for (int i = 0; i <= 1; ++i)
    {
        if (fabs(n.x) > 1e-7)
        {
            const double px = (offset - n.y * i) / n.x;
            if (px >= 0.0 && px <= 1.0)
            {
                const double s = -px * n.y + i * n.x;
                low = fmin(low, s);
                high = fmax(high, s);
            }
        }
        if (fabs(n.y) > 1e-7)
        {
            const double py = (offset - n.x * i) / n.y;
            if (py >= 0.0 && py <= 1.0)
            {
                const double s = -i * n.y + py * n.x;
                low = fmin(low, s);
                high = fmax(high, s);
            }
        }
    }
    if (high <= low)
    {
        sx = sy = length = 0.0;
        return;
    }
    const double middle = 0.5 * (low + high);
    sx = n.x * offset - n.y * middle - 0.5;
    sy = n.y * offset + n.x * middle - 0.5;
    length = high - low;
}

// Sweep 1: heights (FluidSurfaceTensionCPU.h:138-159).
__global__ void k_tension_heights(const double* f, int W, int H, TensionArrays a)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= W || y >= H)
        return;
    double low = 1.0, high = 0.0;
    for (int dy = -1; dy <= 1; ++dy)
        for (int dx = -1; dx <= 1; ++dx)
        {
            const double c = geometry_fraction(f, W, H, x + dx, y + dy);
            low = fmin(low, c);
            high = fmax(high, c);
        }
    double hx = 0.0, hy = 0.0, ox = 0.0, oy = 0.0;
    if (low != high)
    {
        column_height(f, W, H, x, y, 1, 0, hx, ox);
        column_height(f, W, H, x, y, 0, 1, hy, oy);
    }
    const long long i = (long long)y * W + x;
    a.height[i] = make_double2(hx, hy);
    a.orient[2 * i] = (signed char)ox;
    a.orient[2 * i + 1] = (signed char)oy;
}

// Sweep 2: curvature from heights, else a fit of neighbouring heights
// (FluidSurfaceTensionCPU.h:252-284).
__global__ void k_tension_curvature(const double* f, int W, int H, double cell_size, TensionArrays a)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= W || y >= H)
        return;
    const long long i = (long long)y * W + x;
    double kappa = 0.0;
    bool ok = false;
    if (interfacial_cell(f, W, H, x, y))
    {
        const Vec2d n = outward_normal(f, W, H, x, y);
        const bool horizontal = fabs(n.x) > fabs(n.y);
        ok = height_curvature(a, W, H, x, y, horizontal, cell_size, kappa);
        if (!ok)
            ok = height_curvature(a, W, H, x, y, !horizontal, cell_size, kappa);
        if (!ok)
        {
            ParabolaFit fit;
            for (int j = -1; j <= 1; ++j)
            {
                const HeightSample hx = height_at(a, W, H, x, y + j);
                const HeightSample hy = height_at(a, W, H, x + j, y);
                if (hx.ox * n.x > 0.0)
                    fit.add(hx.x, j, n, 1.0);
                if (hy.oy * n.y > 0.0)
                    fit.add(j, hy.y, n, 1.0);
            }
            ok = fit.evaluate(cell_size, kappa);
        }
    }
    a.raw[i] = ok ? kappa : 0.0;
    a.raw_ok[i] = ok ? 1 : 0;
}

// Sweep 3: interface cells without a curvature take the mean of valid neighbours, else a fit
// of neighbouring PLIC segments (FluidSurfaceTensionCPU.h:327-378).
__global__ void k_tension_complete(const double* f, int W, int H, double cell_size, TensionArrays a)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= W || y >= H)
        return;
    const long long i = (long long)y * W + x;
    double kappa = a.raw[i];
    bool ok = a.raw_ok[i] != 0;
    if (!ok && interfacial_cell(f, W, H, x, y))
    {
        double sum = 0.0;
        int count = 0;
        for (int dy = -1; dy <= 1; ++dy)
            for (int dx = -1; dx <= 1; ++dx)
            {
                const long long j = (long long)mirror_cell(y + dy, H) * W + mirror_cell(x + dx, W);
                if (a.raw_ok[j])
                {
                    sum += a.raw[j];
                    ++count;
                }
            }
        if (count > 0)
        {
            kappa = sum / count;
            ok = true;
        }
        else
        {
            const Vec2d n = outward_normal(f, W, H, x, y);
            ParabolaFit fit;
            for (int dy = -1; dy <= 1; ++dy)
                for (int dx = -1; dx <= 1; ++dx)
                {
                    const double c = geometry_fraction(f, W, H, x + dx, y + dy);
                    if (c <= 0.0 || c >= 1.0)
                        continue;
                    const Vec2d nq = outward_normal(f, W, H, x + dx, y + dy);
                    if (n.x * nq.x + n.y * nq.y <= 0.0)
                        continue;
                    double sx, sy, length;
                    plic_segment(f, W, H, x + dx, y + dy, nq, sx, sy, length);
                    if (length > 0.0)
                        fit.add(sx + dx, sy + dy, n, length);
                }
            ok = fit.evaluate(cell_size, kappa);
        }
    }
    a.kappa[i] = ok ? kappa : 0.0;
    a.kappa_ok[i] = ok ? 1 : 0;
}

// Face curvature: mean of the valid sides (FluidSurfaceTensionCPU.h:380-388).
__device__ __forceinline__ double face_curvature(const TensionArrays& a, long long left, long long right)
{
    const bool lo = a.kappa_ok[left] != 0, ro = a.kappa_ok[right] != 0;
    if (!lo)
        return ro ? a.kappa[right] : 0.0;
    return ro ? 0.5 * (a.kappa[left] + a.kappa[right]) : a.kappa[left];
}

// Capillary face force (FluidGridCPU.cpp:906-925) with the pressure face weights of level 0:
// right[(x-1, y)] weighs u face (x, y) and down[(x, y-1)] weighs v face (x, y).
template <typename T>
__global__ void k_tension_force(const GridDesc* grids, int grid, const double* f, TensionArrays a, double sigma,
    double dt)
{
    const GridDesc& g = grids[grid];
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= g.W || y >= g.H)
        return;
    const T* right = static_cast<const T*>(g.lev[0].right);
    const T* down = static_cast<const T*>(g.lev[0].down);
    T* u = static_cast<T*>(g.u);
    T* v = static_cast<T*>(g.v);
    const long long cell = (long long)y * g.W + x;
    if (x >= 1)
    {
        const double jump = sigma * face_curvature(a, cell - 1, cell) * (f[cell] - f[cell - 1]);
        const double w = double(right[padded_index(g.S, x - 1, y)]);
        const long long face = (long long)y * (g.W + 1) + x;
        u[face] = T(double(u[face]) + dt * w * jump / g.dx);
    }
    if (y >= 1)
    {
        const double jump = sigma * face_curvature(a, cell - g.W, cell) * (f[cell] - f[cell - g.W]);
        const double w = double(down[padded_index(g.S, x, y - 1)]);
        v[cell] = T(double(v[cell]) + dt * w * jump / g.dx);
    }
}

} // namespace fc
