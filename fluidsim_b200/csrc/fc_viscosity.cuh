// Implicit viscosity of the UniformCUDA step: backward Euler
//   m (v - v0) = -dt K v,   K = the Hessian of the strain energy sum mu (normal^2 + shear^2),
// solved by CG with a damped-Jacobi multigrid preconditioner.
//
// Follows the reference's GPU solver (FluidSim/UniformWebGPU/ViscosityKernels.h:8-400 and
// ViscositySolverGPU.cpp:61-294): the same operator, diagonal, smoother, transfers, V-cycle,
// CG recurrences and 4-iteration true-residual check. Vectors are in the working precision;
// every reduction and CG scalar is FP64.
//
// Layout: the (w+1) x (h+1) node lattice of a level, row-major; node p holds u face p (x) and v
// face p (y) as one 2-vector, and 4 coefficients (cell mu, vertex mu, u-face mass, v-face mass).
// Reads outside a field clamp to its edge, as the reference's field accessor does. One thread
// per node, 1D blocks of kViscThreads. The V-cycle and CG kernels are launched as programmatic
// dependents of their predecessor and wait for it (dependency_wait) before their first memory
// access, so only the launch itself overlaps the kernel before.
#pragma once

#include "fc_device.cuh"

namespace fc
{

constexpr int kViscThreads = 256;
constexpr int kViscCoarseNodes = 256; // the coarsest level fits one block
// Nodes per thread of the kernels that end in a grid reduction: a block covers this many runs
// of kViscThreads consecutive nodes, so the per-block reduction, fence and atomic are paid a
// quarter as often.
constexpr int kViscReduceNodes = 4;

template <typename T> struct Vec;
template <> struct Vec<float>
{
    using two = float2;
    using four = float4;
};
template <> struct Vec<double>
{
    using two = double2;
    using four = double4;
};

// CG state of one solve (device). Written by the last block of each reduction.
struct ViscState
{
    double rz, alpha, beta;
    double target;     // tol^2 |x0|^2_M + 1e-12 total mass
    double rnorm;      // recurrence residual, sum r.r / m
    double truth;      // true residual of the last check
    double energy;     // |x0|^2_M (twice the initial kinetic energy)
    double total_mass;
    int count;         // alpha updates since the last (re)start
    int stopped;       // recurrence residual reached the target
    int breakdown;     // non-positive curvature or non-finite value
    int pad;
};

struct ViscLevel
{
    int w, h;
    double dx;
    const void* material; // 2 per cell (density, viscosity)
    const void* coeff;    // 4 per node
    void* x;
    void* next;
    void* rhs;
    void* res;
};

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

__device__ __forceinline__ bool valid_u_face(int w, int h, int x, int y) { return x > 0 && x < w && y < h; }
__device__ __forceinline__ bool valid_v_face(int w, int h, int x, int y) { return y > 0 && y < h && x < w; }

// Faces of obstacle cells are closed on the finest level (no reference counterpart: the
// reference has only the outer walls).
__device__ __forceinline__ bool solid_at(const unsigned char* solid, int w, int x, int y)
{
    return solid && solid[(long long)y * w + x];
}

template <typename T> struct Nodes
{
    using T2 = typename Vec<T>::two;
    using T4 = typename Vec<T>::four;
    int w, h;
    __device__ long long at(int x, int y) const { return (long long)clampi(y, 0, h) * (w + 1) + clampi(x, 0, w); }
    __device__ T2 load(const void* f, int x, int y) const { return static_cast<const T2*>(f)[at(x, y)]; }
    __device__ T4 coeff(const void* c, int x, int y) const { return static_cast<const T4*>(c)[at(x, y)]; }
};

// Deterministic two-level reduction. Blocks arrive in fixed groups of NT consecutive blocks:
// the last block of a group to arrive folds the group's partials (one per thread, then
// block_reduce4's fixed tree) into a group sum, and the last group to finish folds the group
// sums (each thread a contiguous run, in index order). No serial chain is longer than two
// loads per thread, and the order of every sum is set by the block indices, not by arrival.
// partial holds blocks + groups slots; counter[0] counts finished groups and counter[1 + g] the
// arrivals in group g (viscosity_layout sizes both).
template <int NT>
__device__ bool visc_arrive_last(double4* partial, unsigned int* counter, int index, int blocks, double4 mine,
    double4* total, int max_mask)
{
    __shared__ int is_last;
    const int group = index / NT, groups = (blocks + NT - 1) / NT;
    const int first = group * NT, members = min(NT, blocks - first);
    if (threadIdx.x == 0)
    {
        partial[index] = mine;
        __threadfence();
        is_last = atomicAdd(counter + 1 + group, 1u) == unsigned(members - 1);
    }
    __syncthreads();
    if (!is_last)
        return false;
    __threadfence();
    const double2* slots = reinterpret_cast<const double2*>(partial);
    double4 v = make_double4(0, 0, 0, 0);
    if (int(threadIdx.x) < members)
    {
        const double2 lo = __ldcg(slots + 2 * (first + threadIdx.x)), hi = __ldcg(slots + 2 * (first + threadIdx.x) + 1);
        v = make_double4(lo.x, lo.y, hi.x, hi.y);
    }
    const double4 group_total = block_reduce4<NT>(v, max_mask);
    if (threadIdx.x == 0)
    {
        partial[blocks + group] = group_total;
        counter[1 + group] = 0u;
        __threadfence();
        is_last = atomicAdd(counter, 1u) == unsigned(groups - 1);
    }
    __syncthreads();
    if (!is_last)
        return false;
    __threadfence();
    const int per = (groups + NT - 1) / NT;
    const int a = threadIdx.x * per, b = min(groups, a + per);
    double4 acc = make_double4(0, 0, 0, 0);
    for (int t = a; t < b; ++t)
    {
        const double2 lo = __ldcg(slots + 2 * (blocks + t)), hi = __ldcg(slots + 2 * (blocks + t) + 1);
        acc.x = (max_mask & 1) ? fmax(acc.x, lo.x) : acc.x + lo.x;
        acc.y = (max_mask & 2) ? fmax(acc.y, lo.y) : acc.y + lo.y;
        acc.z = (max_mask & 4) ? fmax(acc.z, hi.x) : acc.z + hi.x;
        acc.w = (max_mask & 8) ? fmax(acc.w, hi.y) : acc.w + hi.y;
    }
    const double4 out = block_reduce4<NT>(acc, max_mask);
    if (threadIdx.x == 0)
    {
        *total = out;
        *counter = 0u;
        __threadfence();
    }
    __syncthreads();
    return true;
}

// ---------------------------------------------------------------------------------------------
// Set-up: material, coarse material, coefficients
// ---------------------------------------------------------------------------------------------

// Cell density sum m / dx^2 and volume-weighted viscosity sum(m mu/rho) / sum(m / rho)
// (FluidGridGPU.cpp:172-217, 987-1037); comp[k] = (mu_k / rho_k, 1 / rho_k). A cell without
// mass gets viscosity 0.
template <typename T>
__global__ void k_visc_material(const double* const* masses, int components, const double2* comp, int cells,
    double inv_area, void* material)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= cells)
        return;
    double total = 0.0, weighted = 0.0, volume = 0.0;
    for (int k = 0; k < components; ++k)
    {
        const double m = masses[k][i];
        total += m;
        weighted += m * comp[k].x;
        volume += m * comp[k].y;
    }
    using T2 = typename Vec<T>::two;
    T2 out;
    out.x = T(total * inv_area);
    out.y = T(volume > 0.0 ? weighted / volume : 0.0);
    static_cast<T2*>(material)[i] = out;
}

// Mean of the existing fine cells of each 2x2 block (ViscosityKernels.h "coarse material").
template <typename T>
__global__ void k_visc_coarsen(const void* fine, int fw, int fh, void* coarse, int cw, int ch)
{
    using T2 = typename Vec<T>::two;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= cw * ch)
        return;
    const int x = i % cw, y = i / cw;
    T a = 0, b = 0, n = 0;
    for (int j = 0; j < 2; ++j)
        for (int k = 0; k < 2; ++k)
        {
            const int qx = 2 * x + k, qy = 2 * y + j;
            if (qx < fw && qy < fh)
            {
                const T2 m = static_cast<const T2*>(fine)[(long long)qy * fw + qx];
                a += m.x;
                b += m.y;
                n += T(1);
            }
        }
    T2 out;
    out.x = a / n;
    out.y = b / n;
    static_cast<T2*>(coarse)[i] = out;
}

// Node coefficients (ViscosityKernels.h "viscosity coefficients"): cell mu, the mean mu of the
// four cells around an interior vertex, and the face masses rho_face dx^2.
template <typename T>
__global__ void k_visc_coefficients(const void* material, int w, int h, double dx, void* coeff)
{
    using T2 = typename Vec<T>::two;
    using T4 = typename Vec<T>::four;
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= (w + 1) * (h + 1))
        return;
    const int x = n % (w + 1), y = n / (w + 1);
    const T2* m = static_cast<const T2*>(material);
    auto at = [&](int cx, int cy) { return m[(long long)clampi(cy, 0, h - 1) * w + clampi(cx, 0, w - 1)]; };
    const T2 c = at(x, y);
    T mu = 0;
    if (x > 0 && y > 0 && x < w && y < h)
        mu = T(0.25) * (c.y + at(x - 1, y).y + at(x, y - 1).y + at(x - 1, y - 1).y);
    const T area = T(dx * dx);
    T4 out;
    out.x = c.y;
    out.y = mu;
    out.z = T(0.5) * area * (c.x + at(x - 1, y).x);
    out.w = T(0.5) * area * (c.x + at(x, y - 1).x);
    static_cast<T4*>(coeff)[n] = out;
}

// ---------------------------------------------------------------------------------------------
// Operator (ViscosityKernels.h:8-75)
// ---------------------------------------------------------------------------------------------

template <typename T>
__device__ __forceinline__ T shear_term(const Nodes<T>& L, const void* f, const void* c, int x, int y)
{
    const auto p = L.load(f, x, y);
    return L.coeff(c, x, y).y * ((p.x - L.load(f, x, y - 1).x) + (p.y - L.load(f, x - 1, y).y));
}

// mass f(p) + dt stress(f)(p) for both components of node p, before the valid-face mask.
template <typename T>
__device__ __forceinline__ void operator_at(const Nodes<T>& L, const void* f, const void* coeff, T dt, int x, int y,
    T& ax, T& ay)
{
    const auto c = L.load(f, x, y);
    const auto a = L.coeff(coeff, x, y);
    const T t = shear_term<T>(L, f, coeff, x, y);
    const T nx = T(2) * (L.coeff(coeff, x - 1, y).x * (c.x - L.load(f, x - 1, y).x) + a.x * (c.x - L.load(f, x + 1, y).x));
    const T ny = T(2) * (L.coeff(coeff, x, y - 1).x * (c.y - L.load(f, x, y - 1).y) + a.x * (c.y - L.load(f, x, y + 1).y));
    ax = a.z * c.x + dt * (nx + (t - shear_term<T>(L, f, coeff, x, y + 1)));
    ay = a.w * c.y + dt * (ny + (t - shear_term<T>(L, f, coeff, x + 1, y)));
}

template <typename T>
__device__ __forceinline__ void diagonal_at(const Nodes<T>& L, const void* coeff, T dt, int x, int y, T& dx_, T& dy_)
{
    const auto c = L.coeff(coeff, x, y);
    dx_ = c.z + dt * (T(2) * (c.x + L.coeff(coeff, x - 1, y).x) + c.y + L.coeff(coeff, x, y + 1).y);
    dy_ = c.w + dt * (T(2) * (c.x + L.coeff(coeff, x, y - 1).x) + c.y + L.coeff(coeff, x + 1, y).y);
}

struct FaceMask
{
    bool u, v;
};

__device__ __forceinline__ FaceMask face_mask(int w, int h, int x, int y, const unsigned char* solid)
{
    FaceMask m{valid_u_face(w, h, x, y), valid_v_face(w, h, x, y)};
    if (solid)
    {
        if (m.u && (solid_at(solid, w, x - 1, y) || solid_at(solid, w, x, y)))
            m.u = false;
        if (m.v && (solid_at(solid, w, x, y - 1) || solid_at(solid, w, x, y)))
            m.v = false;
    }
    return m;
}

__device__ __forceinline__ bool visc_stopped(const ViscState* s) { return s->stopped || s->breakdown; }

// out = A f on valid faces (ViscosityKernels.h "apply"); with dq, also d.Ad reduced into the CG
// step length alpha (ViscosityKernels.h "scalar" mode 2).
template <typename T, bool kDot>
__global__ void __launch_bounds__(kViscThreads) k_visc_apply(ViscLevel lv, double dt, const unsigned char* solid,
    const void* f, void* out, ViscState* state, double4* partial, unsigned int* counter)
{
    allow_dependents();
    dependency_wait();
    using T2 = typename Vec<T>::two;
    constexpr int kNodes = kDot ? kViscReduceNodes : 1;
    const Nodes<T> L{lv.w, lv.h};
    const bool stopped = visc_stopped(state);
    double dq = 0.0;
#pragma unroll 1
    for (int k = 0; k < kNodes; ++k)
    {
        const int n = (blockIdx.x * kNodes + k) * blockDim.x + threadIdx.x;
        if (n >= (lv.w + 1) * (lv.h + 1))
            break;
        const int x = n % (lv.w + 1), y = n / (lv.w + 1);
        T2 r;
        r.x = r.y = T(0);
        if (!stopped)
        {
            const FaceMask m = face_mask(lv.w, lv.h, x, y, solid);
            T ax, ay;
            operator_at<T>(L, f, lv.coeff, T(dt), x, y, ax, ay);
            r.x = m.u ? ax : T(0);
            r.y = m.v ? ay : T(0);
            const T2 d = static_cast<const T2*>(f)[n];
            dq += double(d.x) * double(r.x) + double(d.y) * double(r.y);
        }
        static_cast<T2*>(out)[n] = r;
    }
    if (!kDot)
        return;
    double4 total;
    const int blocks = gridDim.x;
    if (visc_arrive_last<kViscThreads>(partial, counter, blockIdx.x, blocks,
            block_reduce4<kViscThreads>(make_double4(dq, 0, 0, 0), 0), &total, 0))
    {
        if (threadIdx.x == 0 && !stopped)
        {
            if (!(total.x > 0.0) || !isfinite(total.x))
                state->breakdown = 1;
            else
            {
                state->alpha = state->rz / total.x;
                state->count += 1;
            }
        }
    }
}

// Damped Jacobi (ViscosityKernels.h "smooth"): x + (b - A x) / (2 D), or b / (2 D) from zero.
template <typename T>
__global__ void __launch_bounds__(kViscThreads) k_visc_smooth(ViscLevel lv, double dt, const unsigned char* solid,
    const void* b, int zero, const ViscState* state)
{
    allow_dependents();
    dependency_wait();
    using T2 = typename Vec<T>::two;
    const Nodes<T> L{lv.w, lv.h};
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= (lv.w + 1) * (lv.h + 1))
        return;
    const int x = n % (lv.w + 1), y = n / (lv.w + 1);
    T2 out;
    out.x = out.y = T(0);
    if (!visc_stopped(state))
    {
        const FaceMask m = face_mask(lv.w, lv.h, x, y, solid);
        T dxx, dyy;
        diagonal_at<T>(L, lv.coeff, T(dt), x, y, dxx, dyy);
        const T2 bb = static_cast<const T2*>(b)[n];
        T vx, vy;
        if (zero)
        {
            vx = T(0.5) * bb.x / dxx;
            vy = T(0.5) * bb.y / dyy;
        }
        else
        {
            T ax, ay;
            operator_at<T>(L, lv.x, lv.coeff, T(dt), x, y, ax, ay);
            const T2 c = static_cast<const T2*>(lv.x)[n];
            vx = c.x + T(0.5) * (bb.x - ax) / dxx;
            vy = c.y + T(0.5) * (bb.y - ay) / dyy;
        }
        out.x = m.u ? vx : T(0);
        out.y = m.v ? vy : T(0);
    }
    static_cast<T2*>(lv.next)[n] = out;
}

// Statistics a residual pass can reduce (ViscosityKernels.h "first_reduce" modes 0 and 3).
enum ViscResidualMode
{
    kResidualPlain = 0,   // multigrid residual, no reduction
    kResidualInitial = 1, // |r|^2_M, |x|^2_M, total mass; sets the target
    kResidualTruth = 2    // |r|^2_M into state->truth
};

// out = b - A f on valid faces.
template <typename T, int kMode>
__global__ void __launch_bounds__(kViscThreads) k_visc_residual(ViscLevel lv, double dt, const unsigned char* solid,
    const void* f, const void* b, void* out, ViscState* state, double4* partial, unsigned int* counter,
    double tolerance)
{
    allow_dependents();
    dependency_wait();
    using T2 = typename Vec<T>::two;
    constexpr int kNodes = kMode == kResidualPlain ? 1 : kViscReduceNodes;
    const Nodes<T> L{lv.w, lv.h};
    if (kMode == kResidualPlain && visc_stopped(state))
    {
        const int n = blockIdx.x * blockDim.x + threadIdx.x;
        if (n < (lv.w + 1) * (lv.h + 1))
            static_cast<T2*>(out)[n] = T2{T(0), T(0)};
        return;
    }
    double4 mine = make_double4(0, 0, 0, 0);
#pragma unroll 1
    for (int k = 0; k < kNodes; ++k)
    {
        const int n = (blockIdx.x * kNodes + k) * blockDim.x + threadIdx.x;
        if (n >= (lv.w + 1) * (lv.h + 1))
            break;
        const int x = n % (lv.w + 1), y = n / (lv.w + 1);
        const FaceMask m = face_mask(lv.w, lv.h, x, y, solid);
        T ax, ay;
        operator_at<T>(L, f, lv.coeff, T(dt), x, y, ax, ay);
        const T2 bb = static_cast<const T2*>(b)[n];
        T2 r;
        r.x = m.u ? bb.x - ax : T(0);
        r.y = m.v ? bb.y - ay : T(0);
        static_cast<T2*>(out)[n] = r;
        if (kMode != kResidualPlain)
        {
            const auto c = L.coeff(lv.coeff, x, y);
            const double rx = r.x, ry = r.y;
            mine.x += rx / double(c.z) * rx + ry / double(c.w) * ry;
            if (kMode == kResidualInitial)
            {
                const T2 v = static_cast<const T2*>(f)[n];
                mine.y += double(c.z) * double(v.x) * double(v.x) + double(c.w) * double(v.y) * double(v.y);
                mine.z += double(c.z) + double(c.w);
            }
        }
    }
    if (kMode == kResidualPlain)
        return;
    double4 total;
    if (visc_arrive_last<kViscThreads>(partial, counter, blockIdx.x, gridDim.x, block_reduce4<kViscThreads>(mine, 0),
            &total, 0))
    {
        if (threadIdx.x == 0)
        {
            const bool finite = isfinite(total.x) && isfinite(total.y) && isfinite(total.z);
            if (kMode == kResidualInitial)
            {
                // A new solve: earlier flags are cleared.
                state->breakdown = finite ? 0 : 1;
                state->rz = state->alpha = state->beta = 0.0;
                state->count = 0;
                state->stopped = 0;
                state->energy = total.y;
                state->total_mass = total.z;
                state->target = tolerance * tolerance * total.y + 1e-12 * total.z;
                state->rnorm = total.x;
                state->truth = total.x;
            }
            else
            {
                if (!finite)
                    state->breakdown = 1;
                state->truth = total.x;
            }
        }
    }
}

// ---------------------------------------------------------------------------------------------
// Transfers (ViscosityKernels.h:290-400): bilinear interpolation at face locations and its
// exact transpose, with the reference's tangential clamps.
// ---------------------------------------------------------------------------------------------


__device__ __forceinline__ void transfer_clamp(int bx, int by, int component, int cw, int ch, int& cx, int& cy)
{
    cx = clampi(bx, 0, cw - (component == 1 ? 1 : 0));
    cy = clampi(by, 0, ch - (component == 1 ? 0 : 1));
}

// Coarse coordinate of fine index f along an axis with face offset `half` (0 or 1/2):
// l = (f + half) / 2 - half, returned as b = floor(l) and t = l - b. Both are exact in integer
// arithmetic: t is 0 or 1/2 without the offset, 3/4 or 1/4 with it.
__device__ __forceinline__ void transfer_axis(int f, bool half, int& b, double& t)
{
    if (half)
    {
        b = (f - 1) >> 1; // arithmetic shift: floor((f - 1) / 2)
        t = (f & 1) ? 0.25 : 0.75;
    }
    else
    {
        b = f >> 1;
        t = (f & 1) ? 0.5 : 0.0;
    }
}

__device__ __forceinline__ double transfer_weight(int fx, int fy, int px, int py, int component, int cw, int ch)
{
    int bx, by;
    double tx, ty;
    transfer_axis(fx, component == 1, bx, tx);
    transfer_axis(fy, component == 0, by, ty);
    double result = 0.0;
    for (int y = 0; y < 2; ++y)
        for (int x = 0; x < 2; ++x)
        {
            int cx, cy;
            transfer_clamp(bx + x, by + y, component, cw, ch, cx, cy);
            if (cx == px && cy == py)
                result += (x == 1 ? tx : 1.0 - tx) * (y == 1 ? ty : 1.0 - ty);
        }
    return result;
}

// Coarse right-hand side: transpose of the prolongation applied to the fine residual.
template <typename T>
__global__ void __launch_bounds__(kViscThreads) k_visc_restrict(ViscLevel fine, ViscLevel coarse, const ViscState* state)
{
    allow_dependents();
    dependency_wait();
    using T2 = typename Vec<T>::two;
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= (coarse.w + 1) * (coarse.h + 1))
        return;
    const int px = n % (coarse.w + 1), py = n / (coarse.w + 1);
    double value[2] = {0.0, 0.0};
    if (!visc_stopped(state))
    {
        // The 4 x 4 fine nodes 2p - 1 .. 2p + 2 cover both components' stencils; they are loaded
        // together (indices clamped into the lattice, the clamped copies unused), then summed in
        // the stencil's row order, skipping nodes outside the lattice.
        const T2* res = static_cast<const T2*>(fine.res);
        T2 q[4][4];
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int i = 0; i < 4; ++i)
            {
                const int qx = clampi(2 * px + i - 1, 0, fine.w), qy = clampi(2 * py + j - 1, 0, fine.h);
                q[j][i] = res[(long long)qy * (fine.w + 1) + qx];
            }
        if (px >= 2 && py >= 2 && px <= coarse.w - 3 && py <= coarse.h - 3)
        {
            // No clamp reaches a node two or more from every edge: each stencil weight is the
            // product of the 1D weights (1/2, 1, 1/2) along the face's own axis and
            // (1/4, 3/4, 3/4, 1/4) across it, exactly transfer_weight's value.
            constexpr double kNear[3] = {0.5, 1.0, 0.5};
            constexpr double kFar[4] = {0.25, 0.75, 0.75, 0.25};
#pragma unroll
            for (int y = 0; y < 4; ++y)
#pragma unroll
                for (int x = 0; x < 3; ++x)
                    value[0] += kNear[x] * kFar[y] * double(q[y][x].x);
#pragma unroll
            for (int y = 0; y < 3; ++y)
#pragma unroll
                for (int x = 0; x < 4; ++x)
                    value[1] += kFar[x] * kNear[y] * double(q[y][x].y);
        }
        else
#pragma unroll
        for (int component = 0; component < 2; ++component)
        {
            if ((component == 0 && (px == 0 || px == coarse.w || py == coarse.h)) ||
                (component == 1 && (py == 0 || py == coarse.h || px == coarse.w)))
                continue;
            const int ex = component == 1 ? 2 : 1, ey = component == 1 ? 1 : 2;
#pragma unroll
            for (int y = -1; y <= 2; ++y)
#pragma unroll
                for (int x = -1; x <= 2; ++x)
                {
                    const int qx = 2 * px + x, qy = 2 * py + y;
                    if (x > ex || y > ey || qx < 0 || qy < 0 || qx > fine.w || qy > fine.h)
                        continue;
                    const T2 r = q[y + 1][x + 1];
                    value[component] += transfer_weight(qx, qy, px, py, component, coarse.w, coarse.h) *
                                        double(component == 0 ? r.x : r.y);
                }
        }
    }
    T2 out;
    out.x = T(value[0]);
    out.y = T(value[1]);
    static_cast<T2*>(coarse.rhs)[n] = out;
}

// Fine x += bilinear interpolation of the coarse correction, on valid faces (into fine.next).
template <typename T>
__global__ void __launch_bounds__(kViscThreads) k_visc_prolong(ViscLevel fine, ViscLevel coarse,
    const unsigned char* solid, const ViscState* state)
{
    allow_dependents();
    dependency_wait();
    using T2 = typename Vec<T>::two;
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= (fine.w + 1) * (fine.h + 1))
        return;
    const int px = n % (fine.w + 1), py = n / (fine.w + 1);
    T2 out;
    out.x = out.y = T(0);
    if (!visc_stopped(state))
    {
        const T2 own = static_cast<const T2*>(fine.x)[n];
        const T2* c = static_cast<const T2*>(coarse.x);
        T value[2] = {own.x, own.y};
#pragma unroll
        for (int component = 0; component < 2; ++component)
        {
            int bx, by;
            double tx, ty;
            transfer_axis(px, component == 1, bx, tx);
            transfer_axis(py, component == 0, by, ty);
#pragma unroll
            for (int y = 0; y < 2; ++y)
#pragma unroll
                for (int x = 0; x < 2; ++x)
                {
                    int cx, cy;
                    transfer_clamp(bx + x, by + y, component, coarse.w, coarse.h, cx, cy);
                    const T2 v = c[(long long)cy * (coarse.w + 1) + cx];
                    value[component] += T((x == 1 ? tx : 1.0 - tx) * (y == 1 ? ty : 1.0 - ty)) * (component == 0 ? v.x : v.y);
                }
        }
        const FaceMask m = face_mask(fine.w, fine.h, px, py, solid);
        out.x = m.u ? value[0] : T(0);
        out.y = m.v ? value[1] : T(0);
    }
    static_cast<T2*>(fine.next)[n] = out;
}

// Coarsest level: 16 damped-Jacobi sweeps from zero in one block's shared memory
// (ViscosityKernels.h "coarse_smooth").
template <typename T>
__global__ void __launch_bounds__(kViscCoarseNodes) k_visc_coarse(ViscLevel lv, double dt, const unsigned char* solid,
    const ViscState* state)
{
    allow_dependents();
    dependency_wait();
    using T2 = typename Vec<T>::two;
    using T4 = typename Vec<T>::four;
    __shared__ T2 sx[kViscCoarseNodes];
    __shared__ T4 sc[kViscCoarseNodes];
    const int nodes = (lv.w + 1) * (lv.h + 1);
    const int n = threadIdx.x;
    const bool mine = n < nodes;
    const bool stopped = visc_stopped(state);
    const int x = mine ? n % (lv.w + 1) : 0, y = mine ? n / (lv.w + 1) : 0;
    T2 b;
    b.x = b.y = T(0);
    if (mine)
    {
        sx[n] = T2{T(0), T(0)};
        sc[n] = static_cast<const T4*>(lv.coeff)[n];
        b = static_cast<const T2*>(lv.rhs)[n];
    }
    __syncthreads();
    // Shared-memory views of the level with the clamped accessors of Nodes.
    auto at = [&](int px, int py) { return clampi(py, 0, lv.h) * (lv.w + 1) + clampi(px, 0, lv.w); };
    const FaceMask m = face_mask(lv.w, lv.h, x, y, solid);
    for (int sweep = 0; sweep < 16 && !stopped; ++sweep)
    {
        T2 value;
        value.x = value.y = T(0);
        if (mine)
        {
            const T dtt = T(dt);
            auto shear = [&](int px, int py)
            {
                const T2 p = sx[at(px, py)];
                return sc[at(px, py)].y * ((p.x - sx[at(px, py - 1)].x) + (p.y - sx[at(px - 1, py)].y));
            };
            const T2 c = sx[at(x, y)];
            const T4 a = sc[at(x, y)];
            const T t = shear(x, y);
            const T nx = T(2) * (sc[at(x - 1, y)].x * (c.x - sx[at(x - 1, y)].x) + a.x * (c.x - sx[at(x + 1, y)].x));
            const T ny = T(2) * (sc[at(x, y - 1)].x * (c.y - sx[at(x, y - 1)].y) + a.x * (c.y - sx[at(x, y + 1)].y));
            const T ax = a.z * c.x + dtt * (nx + (t - shear(x, y + 1)));
            const T ay = a.w * c.y + dtt * (ny + (t - shear(x + 1, y)));
            const T dxx = a.z + dtt * (T(2) * (a.x + sc[at(x - 1, y)].x) + a.y + sc[at(x, y + 1)].y);
            const T dyy = a.w + dtt * (T(2) * (a.x + sc[at(x, y - 1)].x) + a.y + sc[at(x + 1, y)].y);
            value.x = m.u ? c.x + T(0.5) * (b.x - ax) / dxx : T(0);
            value.y = m.v ? c.y + T(0.5) * (b.y - ay) / dyy : T(0);
        }
        __syncthreads();
        if (mine)
            sx[n] = value;
        __syncthreads();
    }
    if (mine)
        static_cast<T2*>(lv.x)[n] = stopped ? T2{T(0), T(0)} : sx[n];
}

// ---------------------------------------------------------------------------------------------
// CG on the finest level (ViscosityKernels.h "scalar", "direction", "update", "pack", "unpack")
// ---------------------------------------------------------------------------------------------

// r.z and |r|^2_M; sets beta, or stops when the recurrence residual reaches the target.
template <typename T>
__global__ void __launch_bounds__(kViscThreads) k_visc_dot_rz(int nodes, const void* coeff, const void* r, const void* z,
    ViscState* state, double4* partial, unsigned int* counter)
{
    allow_dependents();
    dependency_wait();
    using T2 = typename Vec<T>::two;
    using T4 = typename Vec<T>::four;
    double4 mine = make_double4(0, 0, 0, 0);
    if (!visc_stopped(state))
    {
        T2 a[kViscReduceNodes], b[kViscReduceNodes];
        T4 c[kViscReduceNodes];
#pragma unroll
        for (int k = 0; k < kViscReduceNodes; ++k)
        {
            const int n = (blockIdx.x * kViscReduceNodes + k) * blockDim.x + threadIdx.x;
            if (n < nodes)
            {
                a[k] = static_cast<const T2*>(r)[n];
                b[k] = static_cast<const T2*>(z)[n];
                c[k] = static_cast<const T4*>(coeff)[n];
            }
        }
#pragma unroll
        for (int k = 0; k < kViscReduceNodes; ++k)
        {
            const int n = (blockIdx.x * kViscReduceNodes + k) * blockDim.x + threadIdx.x;
            if (n < nodes)
            {
                mine.x += double(a[k].x) * double(b[k].x) + double(a[k].y) * double(b[k].y);
                mine.y += double(a[k].x) / double(c[k].z) * double(a[k].x) + double(a[k].y) / double(c[k].w) * double(a[k].y);
            }
        }
    }
    double4 total;
    if (visc_arrive_last<kViscThreads>(partial, counter, blockIdx.x, gridDim.x, block_reduce4<kViscThreads>(mine, 0),
            &total, 0))
    {
        if (threadIdx.x == 0 && !visc_stopped(state))
        {
            state->rnorm = total.y;
            if (!isfinite(total.y))
                state->breakdown = 1;
            else if (total.y <= state->target)
                state->stopped = 1;
            else if (!(total.x > 0.0) || !isfinite(total.x))
                state->breakdown = 1;
            else
            {
                state->beta = state->count > 0 ? total.x / state->rz : 0.0;
                state->rz = total.x;
            }
        }
    }
}

// d = z + beta d.
template <typename T>
__global__ void __launch_bounds__(kViscThreads) k_visc_direction(int nodes, const void* z, void* d, const ViscState* state)
{
    allow_dependents();
    dependency_wait();
    using T2 = typename Vec<T>::two;
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= nodes || visc_stopped(state))
        return;
    const T2 c = static_cast<const T2*>(z)[n];
    T2 out = c;
    if (state->count > 0)
    {
        const T beta = T(state->beta);
        const T2 p = static_cast<const T2*>(d)[n];
        out.x = c.x + beta * p.x;
        out.y = c.y + beta * p.y;
    }
    static_cast<T2*>(d)[n] = out;
}

// x += alpha d, r -= alpha q.
template <typename T>
__global__ void __launch_bounds__(kViscThreads) k_visc_update(int nodes, void* x, void* r, const void* d, const void* q,
    const ViscState* state)
{
    allow_dependents();
    dependency_wait();
    using T2 = typename Vec<T>::two;
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= nodes || visc_stopped(state))
        return;
    const T alpha = T(state->alpha);
    T2 a = static_cast<T2*>(x)[n], b = static_cast<T2*>(r)[n];
    const T2 dd = static_cast<const T2*>(d)[n], qq = static_cast<const T2*>(q)[n];
    a.x += alpha * dd.x;
    a.y += alpha * dd.y;
    b.x -= alpha * qq.x;
    b.y -= alpha * qq.y;
    static_cast<T2*>(x)[n] = a;
    static_cast<T2*>(r)[n] = b;
}

// solution = face velocities on valid faces, rhs = mass * solution.
template <typename T>
__global__ void __launch_bounds__(kViscThreads) k_visc_pack(int w, int h, const void* u, const void* v, const void* coeff,
    const unsigned char* solid, void* solution, void* rhs)
{
    using T2 = typename Vec<T>::two;
    using T4 = typename Vec<T>::four;
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= (w + 1) * (h + 1))
        return;
    const int x = n % (w + 1), y = n / (w + 1);
    const FaceMask m = face_mask(w, h, x, y, solid);
    T2 s;
    s.x = m.u ? static_cast<const T*>(u)[(long long)y * (w + 1) + x] : T(0);
    s.y = m.v ? static_cast<const T*>(v)[(long long)y * w + x] : T(0);
    const T4 c = static_cast<const T4*>(coeff)[n];
    static_cast<T2*>(solution)[n] = s;
    static_cast<T2*>(rhs)[n] = T2{c.z * s.x, c.w * s.y};
}

// Every face velocity from the solution (walls and closed faces receive zero).
template <typename T>
__global__ void __launch_bounds__(kViscThreads) k_visc_unpack(int w, int h, const void* solution, void* u, void* v)
{
    using T2 = typename Vec<T>::two;
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= (w + 1) * (h + 1))
        return;
    const int x = n % (w + 1), y = n / (w + 1);
    const T2 s = static_cast<const T2*>(solution)[n];
    if (y < h)
        static_cast<T*>(u)[(long long)y * (w + 1) + x] = s.x;
    if (x < w)
        static_cast<T*>(v)[(long long)y * w + x] = s.y;
}

// Restart from the true residual after the recurrence claimed convergence too early.
template <typename T>
__global__ void __launch_bounds__(kViscThreads) k_visc_refresh(int nodes, const void* truth, void* r, ViscState* state)
{
    allow_dependents();
    dependency_wait();
    using T2 = typename Vec<T>::two;
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n < nodes)
        static_cast<T2*>(r)[n] = static_cast<const T2*>(truth)[n];
    if (n == 0)
    {
        state->rz = state->alpha = state->beta = 0.0;
        state->count = 0;
        state->stopped = 0;
        state->rnorm = state->truth;
    }
}

} // namespace fc
