// Conservative PLIC transport (UniformCPU's advect), FP64.
//
// FluidSim/UniformCPU/FluidGridCPU.cpp:362-463 moves the liquid fraction, every component mass
// and the face momenta through the faces, X pass then Y pass, in CFL substeps that export at
// most half a cell per substep. Each face's liquid volume comes from the donor cell's PLIC line
// (MYC normal and offset, :473-531, 93-167), each component follows its mixture's share of that
// volume (:1251-1325), momentum moves with the transported mass (:560-712), corrections keep a
// directional pass from compressing or expanding the selected phase (:1327-1397), and the
// velocities are recovered from momentum and the new densities (:714-757).
//
// Every multiply, add and divide below is an explicitly rounded IEEE operation (no fused
// multiply-add), in the order the reference writes it, so the device reproduces a
// contraction-free host build of the reference.
#pragma once

#include "fc_device.cuh"

namespace fc
{
namespace plic
{

__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double div(double a, double b) { return __ddiv_rn(a, b); }
// std::min / std::max / std::clamp semantics.
__device__ __forceinline__ double smin(double a, double b) { return b < a ? b : a; }
__device__ __forceinline__ double smax(double a, double b) { return a < b ? b : a; }
__device__ __forceinline__ double sclamp(double v, double lo, double hi) { return v < lo ? lo : (hi < v ? hi : v); }

// liquidArea (FluidGridCPU.cpp:93-137): liquid area of an axis-aligned rectangle below a line.
__device__ inline double liquid_area(double nx, double ny, double offset, double x0, double y0, double x1, double y1)
{
    const double width = sub(x1, x0);
    const double height = sub(y1, y0);
    const double area = mul(width, height);
    const double min_projection = add(mul(nx, nx >= 0.0 ? x0 : x1), mul(ny, ny >= 0.0 ? y0 : y1));
    const double cut = sub(offset, min_projection);
    const double span_x = mul(fabs(nx), width);
    const double span_y = mul(fabs(ny), height);
    const double small_span = smin(span_x, span_y);
    const double large_span = smax(span_x, span_y);
    if (cut <= 0.0)
        return 0.0;
    if (cut >= add(small_span, large_span))
        return area;
    if (small_span == 0.0)
        return div(mul(area, cut), large_span);
    if (cut < small_span)
        return div(mul(mul(area, cut), cut), mul(mul(2.0, small_span), large_span));
    if (cut < large_span)
        return div(mul(area, sub(cut, mul(0.5, small_span))), large_span);
    const double dry_cut = sub(add(small_span, large_span), cut);
    return mul(area, sub(1.0, div(mul(dry_cut, dry_cut), mul(mul(2.0, small_span), large_span))));
}

// interfaceOffset (FluidGridCPU.cpp:139-167).
__device__ inline double interface_offset(double nx, double ny, double fraction)
{
    const double min_projection = add(smin(nx, 0.0), smin(ny, 0.0));
    const double span_x = fabs(nx), span_y = fabs(ny);
    const double small_span = smin(span_x, span_y);
    const double large_span = smax(span_x, span_y);
    const double triangle_fraction = div(mul(0.5, small_span), large_span);
    double cut;
    if (fraction < triangle_fraction)
        cut = __dsqrt_rn(mul(mul(mul(2.0, small_span), large_span), fraction));
    else if (fraction <= sub(1.0, triangle_fraction))
        cut = add(mul(large_span, fraction), mul(0.5, small_span));
    else
        cut = sub(add(small_span, large_span), __dsqrt_rn(mul(mul(mul(2.0, small_span), large_span), sub(1.0, fraction))));
    return add(min_projection, cut);
}

// interfaceNormal (FluidGridCPU.cpp:473-513): MYC normal from the 3x3 fractions, neighbours
// outside the grid clamped to the nearest boundary cell.
__device__ inline double2 interface_normal(const double* f, int W, int H, int x, int y)
{
    const int lx = max(x - 1, 0), rx = min(x + 1, W - 1);
    const double* above = f + (long long)max(y - 1, 0) * W;
    const double* row = f + (long long)y * W;
    const double* below = f + (long long)min(y + 1, H - 1) * W;
    const double tl = above[lx], t = above[x], tr = above[rx];
    const double l = row[lx], r = row[rx];
    const double bl = below[lx], b = below[x], br = below[rx];
    const double left_sum = add(add(tl, l), bl);
    const double right_sum = add(add(tr, r), br);
    const double top_sum = add(add(tl, t), tr);
    const double bottom_sum = add(add(bl, b), br);
    double cx = mul(0.5, sub(left_sum, right_sum)), cy = mul(0.5, sub(top_sum, bottom_sum));
    const double yx = sub(sub(add(left_sum, l), right_sum), r);
    const double yy = sub(sub(add(top_sum, t), bottom_sum), b);
    if (cx == 0.0 && cy == 0.0)
        return yx == 0.0 && yy == 0.0 ? make_double2(1.0, 0.0) : make_double2(yx, yy);
    if (fabs(cx) <= fabs(cy))
    {
        cy = copysign(1.0, cy);
        if (fabs(yx) > fabs(mul(cx, yy)))
            return make_double2(yx, yy);
    }
    else
    {
        cx = copysign(1.0, cx);
        if (fabs(yy) > fabs(mul(cy, yx)))
            return make_double2(yx, yy);
    }
    return make_double2(cx, cy);
}

// componentMassTransfer (FluidGridCPU.cpp:533-541).
__device__ __forceinline__ double component_transfer(double volume_transfer, double donor_fraction, double donor_mass)
{
    if (donor_fraction <= 0.0)
        return 0.0;
    return mul(donor_mass, div(volume_transfer, donor_fraction));
}

// momentumTransfer (FluidGridCPU.cpp:543-548).
__device__ __forceinline__ double momentum_transfer(double mass, double before, double after)
{
    return mul(mass, mass >= 0.0 ? before : after);
}

// Work arrays of one grid's transport (all FP64).
struct PlicArrays
{
    double *mom_u, *mom_v;   // face momenta
    double *next_u, *next_v; // evolving face velocities
    double *lt_u, *lt_v;     // liquid volume through each face (cell-volume units)
    double *mt_u, *mt_v;     // transported mass per cell volume through each face
    double2* normal;         // PLIC normals of interface cells
    double* offset;          // PLIC offsets of interface cells
    unsigned char* split;    // 1: the liquid phase fills at least half the cell (frozen)
    double* corr;            // components x cells: correction weights (frozen)
    double* mcorr;           // cells: their density counterpart
    double* fnext;           // next liquid fraction
    double* mnext;           // components x cells: next masses
    unsigned long long* outflow; // largest cell outflow, as ordered bits of a nonnegative double
};

__device__ __forceinline__ int face_count(int W, int H) { return (W + 1) * (H + 1); }

// rebuildMomentum (FluidGridCPU.cpp:1425-1475): face momentum of the current velocity and
// density; the walls hold zero.
template <typename T>
__global__ void k_plic_begin(int W, int H, const T* u, const T* v, const double* density, PlicArrays a)
{
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= face_count(W, H))
        return;
    const int x = n % (W + 1), y = n / (W + 1);
    if (y < H)
    {
        const long long face = (long long)y * (W + 1) + x;
        if (x == 0 || x == W)
            a.mom_u[face] = a.next_u[face] = 0.0;
        else
        {
            const long long cell = (long long)y * W + x;
            const double fd = mul(0.5, add(density[cell - 1], density[cell]));
            a.mom_u[face] = mul(fd, double(u[face]));
            a.next_u[face] = double(u[face]);
        }
    }
    if (x < W)
    {
        const long long face = (long long)y * W + x;
        if (y == 0 || y == H)
            a.mom_v[face] = a.next_v[face] = 0.0;
        else
        {
            const double fd = mul(0.5, add(density[face - W], density[face]));
            a.mom_v[face] = mul(fd, double(v[face]));
            a.next_v[face] = double(v[face]);
        }
    }
}

// Largest cell outflow (FluidGridCPU.cpp:366-385); nonnegative doubles order as their bits.
template <typename T> __global__ void k_plic_outflow(int W, int H, const T* u, const T* v, PlicArrays a)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= W * H)
        return;
    const int x = i % W, y = i / W;
    const T* horizontal = u + (long long)y * (W + 1);
    const T* vertical = v + (long long)y * W;
    const double outflow = add(add(add(smax(double(horizontal[x + 1]), 0.0), smax(-double(horizontal[x]), 0.0)),
                                   smax(double(vertical[x + W]), 0.0)),
        smax(-double(vertical[x]), 0.0));
    atomicMax(a.outflow, __double_as_longlong(outflow) < 0 ? 0ull : (unsigned long long)__double_as_longlong(outflow));
}

// freezeComponentCorrections (FluidGridCPU.cpp:1291-1325).
__global__ void k_plic_freeze(int W, int H, const double* f, const double* const* masses, int liquids, int components,
    double inverse_volume, PlicArrays a)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int cells = W * H;
    if (i >= cells)
        return;
    const double fraction = f[i];
    const bool selected = fraction > 0.5;
    a.split[i] = selected ? 1 : 0;
    const double inverse = div(1.0, selected ? fraction : sub(1.0, fraction));
    double total = 0.0;
    for (int k = 0; k < components; ++k)
    {
        const bool active = (k < liquids) == selected;
        const double w = active ? mul(masses[k][i], inverse) : 0.0;
        a.corr[(long long)k * cells + i] = w;
        total = add(total, mul(w, inverse_volume));
    }
    a.mcorr[i] = total;
}

// rebuildInterfaces (FluidGridCPU.cpp:515-531).
__global__ void k_plic_interfaces(int W, int H, const double* f, PlicArrays a)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= W * H)
        return;
    const double fraction = f[i];
    if (fraction <= 0.0 || fraction >= 1.0)
        return;
    const double2 n = interface_normal(f, W, H, i % W, i / W);
    a.normal[i] = n;
    a.offset[i] = interface_offset(n.x, n.y, fraction);
}

// Axis helpers: kX passes move through u faces ((W+1) x H), kY passes through v faces (W x (H+1)).
// A face's "before" cell is left (X) or above (Y); faces on the outer walls are closed.
template <int AXIS> struct Axis;
template <> struct Axis<0>
{
    __device__ static bool face(int W, int H, int n, int& x, int& y, long long& f)
    {
        x = n % (W + 1);
        y = n / (W + 1);
        f = (long long)y * (W + 1) + x;
        return y < H;
    }
    __device__ static bool wall(int W, int H, int x, int y) { return x == 0 || x == W; }
    __device__ static long long before_cell(int W, int x, int y) { return (long long)y * W + x - 1; }
    __device__ static long long after_cell(int W, int x, int y) { return (long long)y * W + x; }
    // Faces before and after cell (x, y).
    __device__ static long long face_before(int W, int x, int y) { return (long long)y * (W + 1) + x; }
    __device__ static long long face_after(int W, int x, int y) { return (long long)y * (W + 1) + x + 1; }
};
template <> struct Axis<1>
{
    __device__ static bool face(int W, int H, int n, int& x, int& y, long long& f)
    {
        x = n % (W + 1);
        y = n / (W + 1);
        f = (long long)y * W + x;
        return x < W;
    }
    __device__ static bool wall(int W, int H, int x, int y) { return y == 0 || y == H; }
    __device__ static long long before_cell(int W, int x, int y) { return (long long)(y - 1) * W + x; }
    __device__ static long long after_cell(int W, int x, int y) { return (long long)y * W + x; }
    __device__ static long long face_before(int W, int x, int y) { return (long long)y * W + x; }
    __device__ static long long face_after(int W, int x, int y) { return (long long)(y + 1) * W + x; }
};

// liquidTransferX / liquidTransferY (FluidGridCPU.cpp:759-833).
template <typename T, int AXIS>
__global__ void k_plic_transfer(int W, int H, const T* flow, const double* f, double scale, PlicArrays a, double* lt)
{
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= face_count(W, H))
        return;
    int x, y;
    long long face;
    if (!Axis<AXIS>::face(W, H, n, x, y, face))
        return;
    double value = 0.0;
    const double speed = double(flow[face]);
    if (!Axis<AXIS>::wall(W, H, x, y) && speed != 0.0)
    {
        const long long donor = speed > 0.0 ? Axis<AXIS>::before_cell(W, x, y) : Axis<AXIS>::after_cell(W, x, y);
        const double fraction = f[donor];
        if (fraction > 0.0)
        {
            const double volume = mul(speed, scale);
            const double strip = fabs(volume);
            if (fraction >= 1.0)
                value = volume;
            else
            {
                const double2 nrm = a.normal[donor];
                double area;
                if (AXIS == 0)
                    area = liquid_area(nrm.x, nrm.y, a.offset[donor], speed > 0.0 ? sub(1.0, strip) : 0.0, 0.0,
                        speed > 0.0 ? 1.0 : strip, 1.0);
                else
                    area = liquid_area(nrm.x, nrm.y, a.offset[donor], 0.0, speed > 0.0 ? sub(1.0, strip) : 0.0, 1.0,
                        speed > 0.0 ? 1.0 : strip);
                const double bounded = sclamp(area, smax(0.0, sub(strip, sub(1.0, fraction))), smin(strip, fraction));
                value = speed > 0.0 ? bounded : -bounded;
            }
        }
    }
    lt[face] = value;
}

// The mass a component moves through a face (rebuildComponentTransfersX/Y,
// FluidGridCPU.cpp:1235-1289); zero on the walls.
template <typename T, int AXIS>
__device__ __forceinline__ double face_component_transfer(int W, int H, int x, int y, long long face, const T* flow,
    const double* f, const double* lt, const double* mass, bool is_liquid, double scale)
{
    if (Axis<AXIS>::wall(W, H, x, y))
        return 0.0;
    const double speed = double(flow[face]);
    const long long donor = speed > 0.0 ? Axis<AXIS>::before_cell(W, x, y) : Axis<AXIS>::after_cell(W, x, y);
    const double total = mul(speed, scale);
    const double liquid = lt[face];
    const double fraction = f[donor];
    return component_transfer(is_liquid ? liquid : sub(total, liquid), is_liquid ? fraction : sub(1.0, fraction), mass[donor]);
}

// mass_transfer (per cell volume) of every face: the sum over the components, liquids first.
template <typename T, int AXIS>
__global__ void k_plic_mass_transfer(int W, int H, const T* flow, const double* f, const double* lt,
    const double* const* masses, int liquids, int components, double scale, double inverse_volume, double* mt)
{
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= face_count(W, H))
        return;
    int x, y;
    long long face;
    if (!Axis<AXIS>::face(W, H, n, x, y, face))
        return;
    double total = 0.0;
    if (!Axis<AXIS>::wall(W, H, x, y))
        for (int k = 0; k < components; ++k)
            total = add(total, mul(face_component_transfer<T, AXIS>(W, H, x, y, face, flow, f, lt, masses[k], k < liquids,
                                       scale),
                                   inverse_volume));
    mt[face] = total;
}

// advectComponents (FluidGridCPU.cpp:1351-1397): every component's next mass.
template <typename T, int AXIS>
__global__ void k_plic_components(int W, int H, const T* flow, const double* f, const double* lt,
    const double* const* masses, int liquids, int components, double scale, PlicArrays a)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int cells = W * H;
    if (i >= cells)
        return;
    const int x = i % W, y = i / W;
    const long long fb = Axis<AXIS>::face_before(W, x, y), fa = Axis<AXIS>::face_after(W, x, y);
    // Face (x, y) for the before face, (x + 1, y) or (x, y + 1) for the after face.
    const int ax = AXIS == 0 ? x + 1 : x, ay = AXIS == 0 ? y : y + 1;
    const double net_fluid = mul(scale, sub(double(flow[fa]), double(flow[fb])));
    for (int k = 0; k < components; ++k)
    {
        const bool liquid = k < liquids;
        const double before = face_component_transfer<T, AXIS>(W, H, x, y, fb, flow, f, lt, masses[k], liquid, scale);
        const double after = face_component_transfer<T, AXIS>(W, H, ax, ay, fa, flow, f, lt, masses[k], liquid, scale);
        const double w = a.corr[(long long)k * cells + i];
        a.mnext[(long long)k * cells + i] = add(masses[k][i], add(sub(before, after), mul(w, net_fluid)));
    }
}

// advectMomentumX / advectMomentumY (FluidGridCPU.cpp:560-712): every u and v face's momentum
// after the pass. Transfers between neighbouring samples carry the donor's velocity; the frozen
// correction accounts for the pass's compression.
template <typename T, int AXIS>
__global__ void k_plic_momentum(int W, int H, const T* u, const T* v, const double* mt, double scale, PlicArrays a)
{
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= face_count(W, H))
        return;
    const int x = n % (W + 1), y = n / (W + 1);
    const int su = W + 1;
    // The density counterpart of the frozen correction of cell (cx, cy) for this pass.
    auto correction = [&](int cx, int cy)
    {
        const long long cell = (long long)cy * W + cx;
        const double flow = AXIS == 0 ? sub(double(u[(long long)cy * su + cx + 1]), double(u[(long long)cy * su + cx]))
                                      : sub(double(v[(long long)(cy + 1) * W + cx]), double(v[(long long)cy * W + cx]));
        return mul(mul(a.mcorr[cell], scale), flow);
    };
    if (y < H)
    {
        // u face (x, y).
        const long long face = (long long)y * su + x;
        if (x == 0 || x == W)
            a.mom_u[face] = 0.0;
        else
        {
            double before_m, after_m;
            if (AXIS == 0)
            {
                const double left_mass = mul(0.5, add(mt[face - 1], mt[face]));
                const double right_mass = mul(0.5, add(mt[face], mt[face + 1]));
                before_m = momentum_transfer(left_mass, a.next_u[face - 1], a.next_u[face]);
                after_m = momentum_transfer(right_mass, a.next_u[face], a.next_u[face + 1]);
            }
            else
            {
                const long long left_top = (long long)y * W + x - 1, right_top = (long long)y * W + x;
                const double top_mass = mul(0.5, add(mt[left_top], mt[right_top]));
                const double bottom_mass = mul(0.5, add(mt[left_top + W], mt[right_top + W]));
                before_m = y > 0 ? momentum_transfer(top_mass, a.next_u[face - su], a.next_u[face]) : 0.0;
                after_m = y + 1 < H ? momentum_transfer(bottom_mass, a.next_u[face], a.next_u[face + su]) : 0.0;
            }
            const double c = mul(0.5, add(correction(x - 1, y), correction(x, y)));
            a.mom_u[face] = add(a.mom_u[face], add(sub(before_m, after_m), mul(double(u[face]), c)));
        }
    }
    if (x < W)
    {
        // v face (x, y).
        const long long face = (long long)y * W + x;
        if (y == 0 || y == H)
            a.mom_v[face] = 0.0;
        else
        {
            double before_m, after_m;
            if (AXIS == 0)
            {
                const long long above_left = (long long)(y - 1) * su + x, below_left = (long long)y * su + x;
                const double left_mass = mul(0.5, add(mt[above_left], mt[below_left]));
                const double right_mass = mul(0.5, add(mt[above_left + 1], mt[below_left + 1]));
                before_m = x > 0 ? momentum_transfer(left_mass, a.next_v[face - 1], a.next_v[face]) : 0.0;
                after_m = x + 1 < W ? momentum_transfer(right_mass, a.next_v[face], a.next_v[face + 1]) : 0.0;
            }
            else
            {
                const double top_mass = mul(0.5, add(mt[face - W], mt[face]));
                const double bottom_mass = mul(0.5, add(mt[face], mt[face + W]));
                before_m = momentum_transfer(top_mass, a.next_v[face - W], a.next_v[face]);
                after_m = momentum_transfer(bottom_mass, a.next_v[face], a.next_v[face + W]);
            }
            const double c = mul(0.5, add(correction(x, y - 1), correction(x, y)));
            a.mom_v[face] = add(a.mom_v[face], add(sub(before_m, after_m), mul(double(v[face]), c)));
        }
    }
}

// The fraction after a pass (FluidGridCPU.cpp:408-427, 438-455).
template <typename T, int AXIS>
__global__ void k_plic_fraction(int W, int H, const T* flow, const double* f, const double* lt, double scale,
    PlicArrays a)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= W * H)
        return;
    const int x = i % W, y = i / W;
    const long long fb = Axis<AXIS>::face_before(W, x, y), fa = Axis<AXIS>::face_after(W, x, y);
    const double net_liquid = sub(lt[fa], lt[fb]);
    const double net_fluid = mul(scale, sub(double(flow[fa]), double(flow[fb])));
    a.fnext[i] = add(sub(f[i], net_liquid), mul(double(a.split[i]), net_fluid));
}

// recoverVelocity (FluidGridCPU.cpp:714-757): velocity from momentum and the new density.
__global__ void k_plic_recover(int W, int H, const double* density, PlicArrays a)
{
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= face_count(W, H))
        return;
    const int x = n % (W + 1), y = n / (W + 1);
    if (y < H)
    {
        const long long face = (long long)y * (W + 1) + x;
        if (x == 0 || x == W)
            a.next_u[face] = 0.0;
        else
        {
            const long long cell = (long long)y * W + x;
            a.next_u[face] = div(a.mom_u[face], mul(0.5, add(density[cell - 1], density[cell])));
        }
    }
    if (x < W)
    {
        const long long face = (long long)y * W + x;
        if (y == 0 || y == H)
            a.next_v[face] = 0.0;
        else
            a.next_v[face] = div(a.mom_v[face], mul(0.5, add(density[face - W], density[face])));
    }
}

// Density of every cell from its component masses (FluidGridCPU.cpp:1399-1423).
__global__ void k_plic_density(int cells, const double* const* masses, int components, double inverse_volume,
    double* density)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= cells)
        return;
    double total = 0.0;
    for (int k = 0; k < components; ++k)
        total = add(total, masses[k][i]);
    density[i] = mul(total, inverse_volume);
}

// The face velocities after transport (advect's final swap, FluidGridCPU.cpp:461-462).
template <typename T> __global__ void k_plic_finish(int W, int H, PlicArrays a, T* u, T* v)
{
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= face_count(W, H))
        return;
    const int x = n % (W + 1), y = n / (W + 1);
    if (y < H)
        u[(long long)y * (W + 1) + x] = T(a.next_u[(long long)y * (W + 1) + x]);
    if (x < W)
        v[(long long)y * W + x] = T(a.next_v[(long long)y * W + x]);
}

} // namespace plic
} // namespace fc
