// UniformCUDA engine: device memory, multigrid hierarchy, launch plans, CUDA graphs, C ABI.
//
// One grid = one arena of device memory holding every field of the projection. A Plan is the
// launch schedule of a set of grids (one grid, or a batch of uneven grids): tile tables per
// kernel and level, a device array of grid descriptors, and one CUDA graph that runs a whole
// projection: set-up, a conditional WHILE node around the PCG iterations, the velocity update
// and the divergence check. The loop condition is computed on the device, so a projection is
// one graph launch plus one small read-back of the per-grid results.
#include "fc_device.cuh"
#include "fc_multigrid.cuh"
#include "fc_pcg.cuh"
#include "fc_smooth.cuh"
#include "fc_stage.cuh"
#include "fc_json.h"
#include "fc_advect.cuh"
#include "fc_tension.cuh"
#include "fc_viscosity.cuh"
#include "fc_plic.cuh"
#include "fc_errors.h"

#include "../../include/fluidcuda.h"

#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <limits>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <type_traits>
#include <vector>

namespace fc
{

// ------------------------------------------------------------------------------------------
// Errors and launches
// ------------------------------------------------------------------------------------------

thread_local std::string last_error;
std::atomic<long long> launch_count{0};
// Launches made by the calling thread: graph capture counts its captured kernels from this, so
// kernels launched by other threads meanwhile are not counted as captured.
thread_local long long thread_launches = 0;

[[noreturn]] void fail(int status, const char* format, ...)
{
    char buffer[512];
    va_list args;
    va_start(args, format);
    vsnprintf(buffer, sizeof(buffer), format, args);
    va_end(args);
    last_error = buffer;
    throw Failure{status};
}

void check(cudaError_t err, const char* what)
{
    if (err != cudaSuccess)
    {
        cudaGetLastError();
        fail(err == cudaErrorMemoryAllocation ? FC_ERR_OUT_OF_MEMORY : FC_ERR_CUDA, "%s: %s", what,
            cudaGetErrorString(err));
    }
}

// Device memory of grids and plans comes from the device's stream-ordered pool: allocations and
// frees are ordered on the owner's stream and never synchronise the device, so tearing down one
// grid does not wait for other threads' work (the serving loop retires simulations while other
// size classes run; a plain free waited up to 1.4 s there). The pool keeps freed memory for
// reuse instead of returning it at every synchronisation.
void device_pool_setup()
{
    static std::mutex lock;
    static bool done[64] = {};
    int device = 0;
    check(cudaGetDevice(&device), "device");
    std::lock_guard<std::mutex> guard(lock);
    if (device < 0 || device >= 64 || done[device])
        return;
    cudaMemPool_t pool;
    check(cudaDeviceGetDefaultMemPool(&pool, device), "memory pool");
    unsigned long long keep = ~0ull;
    check(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep), "memory pool threshold");
    done[device] = true;
}

template <typename P> void device_alloc(P** ptr, size_t bytes, cudaStream_t s, const char* what)
{
    device_pool_setup();
    void* p = nullptr;
    check(cudaMallocAsync(&p, bytes, s), what);
    *ptr = static_cast<P*>(p);
}

void device_free(void* ptr, cudaStream_t s)
{
    if (ptr)
        cudaFreeAsync(ptr, s);
}

inline long long launch_size(long long blocks) { return blocks; }
inline long long launch_size(dim3 blocks) { return (long long)blocks.x * blocks.y * blocks.z; }

#define FC_LAUNCH(kernel, blocks, threads, smem, stream, ...)                                      \
    do                                                                                             \
    {                                                                                              \
        if (::fc::launch_size(blocks) > 0)                                                         \
        {                                                                                          \
            kernel<<<(blocks), (threads), (smem), (stream)>>>(__VA_ARGS__);                        \
            check(cudaGetLastError(), #kernel);                                                    \
            ::fc::launch_count.fetch_add(1, std::memory_order_relaxed);                            \
            ++::fc::thread_launches;                                                               \
        }                                                                                          \
    } while (0)

// Launch with programmatic stream serialization: the kernel may be scheduled before its
// predecessor completes and orders itself with dependency_wait() (fc_device.cuh).
template <typename Blocks, typename... Params, typename... Args>
void launch_dependent(const char* name, void (*kernel)(Params...), Blocks blocks, int threads, size_t smem,
    cudaStream_t stream, Args... args)
{
    if (launch_size(blocks) <= 0)
        return;
    cudaLaunchConfig_t config = {};
    config.gridDim = dim3(blocks);
    config.blockDim = dim3(threads);
    config.dynamicSmemBytes = smem;
    config.stream = stream;
    cudaLaunchAttribute attribute[1];
    attribute[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attribute[0].val.programmaticStreamSerializationAllowed = 1;
    config.attrs = attribute;
    config.numAttrs = 1;
    check(cudaLaunchKernelEx(&config, kernel, static_cast<Params>(args)...), name);
    launch_count.fetch_add(1, std::memory_order_relaxed);
    ++thread_launches;
}

#define FC_LAUNCH_DEP(kernel, blocks, threads, smem, stream, ...) \
    launch_dependent(#kernel, kernel, (blocks), (threads), (smem), (stream), __VA_ARGS__)

int ceil_div(int a, int b) { return (a + b - 1) / b; }

// ------------------------------------------------------------------------------------------
// Multigrid hierarchy (host side)
// ------------------------------------------------------------------------------------------

struct HostLevel
{
    int w = 0, h = 0, S = 0;
    std::vector<double> cx, cy;
    std::vector<Interp> px, py; // this level -> next
    std::vector<Gather> rx, ry; // next level's cells -> this level
    std::vector<unsigned char> rwx, rwy; // rx, ry as RestrictAxis<T> of the grid's precision
};

// Offset weights of a restriction table (what restrict_axis forms on the device).
template <typename T> std::vector<unsigned char> restrict_weights(const std::vector<Gather>& table)
{
    std::vector<unsigned char> bytes(table.size() * sizeof(RestrictAxis<T>));
    RestrictAxis<T>* out = reinterpret_cast<RestrictAxis<T>*>(bytes.data());
    for (size_t c = 0; c < table.size(); ++c)
    {
        RestrictAxis<T> r{};
        for (int p = 0; p < 4; ++p)
            for (int e = 0; e < table[c].count; ++e)
                if (table[c].index[e] == 2 * int(c) - 1 + p)
                {
                    r.w[p] = T(table[c].weight[e]);
                    r.mask |= 1u << p;
                }
        out[c] = r;
    }
    return bytes;
}

// Halving until at most 64 cells; cell centres keep a shorter last cell on odd sizes.
// PressureMultigrid.cpp:24-62.
std::vector<HostLevel> build_levels(int W, int H)
{
    std::vector<HostLevel> levels;
    int w = W, h = H, spacing = 1;
    for (;;)
    {
        HostLevel l;
        l.w = w;
        l.h = h;
        l.S = padded_stride(w);
        l.cx.resize(w);
        l.cy.resize(h);
        for (int x = 0; x < w; ++x)
            l.cx[x] = 0.5 * (double(x) * spacing + std::min((x + 1) * spacing, W));
        for (int y = 0; y < h; ++y)
            l.cy[y] = 0.5 * (double(y) * spacing + std::min((y + 1) * spacing, H));
        levels.push_back(std::move(l));
        if (w * h <= 64)
            break;
        w = (w + 1) / 2;
        h = (h + 1) / 2;
        spacing *= 2;
    }
    if (int(levels.size()) > kMaxLevels)
        fail(FC_ERR_INVALID_ARGUMENT, "grid %dx%d needs more than %d multigrid levels", W, H, kMaxLevels);
    // Linear interpolation between neighbouring coarse centres, clamped at the ends; the
    // restriction is its transpose. PressureMultigrid.cpp:64-102.
    auto axis = [](const std::vector<double>& fine, const std::vector<double>& coarse, std::vector<Interp>& p,
                    std::vector<Gather>& r)
    {
        const int nf = int(fine.size()), nc = int(coarse.size());
        p.assign(nf, Interp{});
        r.assign(nc, Gather{});
        for (int f = 0; f < nf; ++f)
        {
            const int parent = f / 2;
            const int first = std::max(0, parent - int(fine[f] < coarse[parent]));
            const int second = std::min(first + 1, nc - 1);
            const double weight =
                first == second ? 0.0 : std::clamp((fine[f] - coarse[first]) / (coarse[second] - coarse[first]), 0.0, 1.0);
            p[f] = {first, second, weight};
            const int target[2] = {first, second};
            const double value[2] = {1.0 - weight, weight};
            for (int k = 0; k < 2; ++k)
            {
                if (value[k] == 0.0)
                    continue;
                Gather& g = r[target[k]];
                // The smoothing kernels sum coarse cell c over fine cells 2c-1 .. 2c+2 only.
                if (g.count >= 4 || f < 2 * target[k] - 1 || f > 2 * target[k] + 2)
                    fail(FC_ERR_CUDA, "restriction stencil outside fine cells 2c-1 .. 2c+2");
                g.index[g.count] = f;
                g.weight[g.count] = value[k];
                ++g.count;
            }
        }
    };
    for (size_t i = 0; i + 1 < levels.size(); ++i)
    {
        axis(levels[i].cx, levels[i + 1].cx, levels[i].px, levels[i].rx);
        axis(levels[i].cy, levels[i + 1].cy, levels[i].py, levels[i].ry);
    }
    return levels;
}

// ------------------------------------------------------------------------------------------
// Grid
// ------------------------------------------------------------------------------------------

struct Plan;

struct Grid
{
    int W = 0, H = 0, S = 0;
    double dx = 1.0;
    double origin_x = 0.0, origin_y = 0.0;
    int precision = FC_PRECISION_FP32;
    size_t elem = 4;
    int device = 0;
    int preconditioner = FC_PRECONDITIONER_MULTIGRID;
    double gravity_y = 100.0; // FluidGridCPU.h:37
    double surface_tension = 0.0;
    std::vector<double> liquid_density, gas_density, liquid_viscosity, gas_viscosity;
    bool configured = false;
    bool uploaded = false;
    bool coefficients_dirty = true;
    bool has_solid = false;

    std::vector<HostLevel> levels;
    int tail = 0;
    size_t tail_smem = 0;
    int tail_cells = 1024; // largest level the one-CTA tail takes (autotuned)

    cudaStream_t stream = nullptr;
    int stream_priority = 0; // CUDA stream priority (lower runs first); batches take their members' highest
    char* arena = nullptr;
    size_t arena_bytes = 0;
    GridDesc desc{};
    double* fraction = nullptr;
    double* masses = nullptr;     // components x W*H
    double** mass_ptrs = nullptr; // device array of component pointers
    double* staging = nullptr;    // FP64 staging for upload/download conversions
    void* u_next = nullptr;       // advection outputs (working precision)
    void* v_next = nullptr;
    size_t staging_count = 0;
    unsigned char* solid = nullptr;
    unsigned char* mask = nullptr;
    size_t cells = 0, faces_u = 0, faces_v = 0;
    int mass_capacity = 0;
    char* tension_arena = nullptr; // curvature sweeps, allocated on first use
    TensionArrays tension{};
    char* visc_arena = nullptr;    // viscosity solver workspace, allocated on first use
    size_t visc_bytes = 0;
    int transport = FC_TRANSPORT_SEMI_LAGRANGIAN;
    int air_model = FC_AIR_GAS;
    unsigned char* air = nullptr;  // Dirichlet air cells (written by k_coefficients)
    unsigned char* air_faces = nullptr; // extension layers of the u then v faces (Dirichlet air)
    char* plic_arena = nullptr;    // PLIC transport workspace, allocated on first use
    size_t plic_bytes = 0;

    std::unique_ptr<Plan> plan; // single-grid plan, built lazily

    int components() const { return int(liquid_density.size() + gas_density.size()); }
    ~Grid();
};

// Strip heights of the smoothing kernels: tall strips (less halo overhead) on levels with
// enough tiles to fill the GPU twice, short ones (half the per-CTA latency) below that, and the
// strips of the 16-warp wide regions (FP32 only).
template <typename T> struct Tiling;
template <> struct Tiling<float>
{
    static constexpr int big = 8;
    static constexpr int small = 4;
    static constexpr int wide = 8;
};
template <> struct Tiling<double>
{
    static constexpr int big = 6;
    static constexpr int small = 4;
    static constexpr int wide = 6;
};

struct TileSizes
{
    int pre_x, pre_y, post_x, post_y;
};

template <typename T, int K, int WARPS> TileSizes tile_sizes_of()
{
    return {TileShape<T, K, true, WARPS>::OX, TileShape<T, K, true, WARPS>::OY, TileShape<T, K, false, WARPS>::OX,
        TileShape<T, K, false, WARPS>::OY};
}

// Output region of the smoothing kernels for a region shape (kShapeTall/Short/Wide).
TileSizes tile_sizes(int precision, int shape)
{
    if (precision == FC_PRECISION_FP64)
        return shape == kShapeShort ? tile_sizes_of<double, Tiling<double>::small, 8>()
                                    : tile_sizes_of<double, Tiling<double>::big, 8>();
    if (shape == kShapeShort)
        return tile_sizes_of<float, Tiling<float>::small, 8>();
    if (shape == kShapeWide)
        return tile_sizes_of<float, Tiling<float>::wide, 16>();
    return tile_sizes_of<float, Tiling<float>::big, 8>();
}

// The coarse tail starts at the first level of at most g.tail_cells cells (and 1024 in FP64)
// whose shared-memory footprint fits one CTA.
void choose_tail(Grid& g)
{
    const int limit_cells = g.elem == 4 ? g.tail_cells : std::min(g.tail_cells, 1024);
    // Dynamic shared memory of the tail, within the 227 KB a CTA may hold beside its static
    // shared memory (the register strips' edge rows: 19 KB in FP32, 36 KB in FP64).
    const size_t limit_bytes = (g.elem == 4 ? 208 : 188) * 1024;
    std::vector<int> w, h;
    for (auto& l : g.levels)
        w.push_back(l.w), h.push_back(l.h);
    const int n = int(g.levels.size());
    for (int l = 0; l < n; ++l)
    {
        const size_t bytes = tail_bytes(w.data(), h.data(), l, n, g.elem);
        // The tail's register strips hold levels of up to kTailMaxSide x kTailMaxSide cells (the
        // coarsest level, at most 64 cells, always fits).
        if (w[l] * h[l] <= limit_cells && w[l] <= kTailMaxSide && h[l] <= kTailMaxSide && bytes <= limit_bytes)
        {
            g.tail = l;
            g.tail_smem = bytes;
            return;
        }
    }
    g.tail = n - 1;
    g.tail_smem = tail_bytes(w.data(), h.data(), n - 1, n, g.elem);
}

// ------------------------------------------------------------------------------------------
// TMA tensor maps of the smoothed levels
// ------------------------------------------------------------------------------------------

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link against libcuda).
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, []
    {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
        else
            cudaGetLastError();
    });
    if (!fn)
        fail(FC_ERR_CUDA, "cuTensorMapEncodeTiled is not available");
    return fn;
}

// A 2D map over a padded level array (S columns, rows rows) with a box_w x box_h box.
void encode_box(CUtensorMap& map, const void* base, CUtensorMapDataType type, size_t elem, int S, int rows, int box_w,
    int box_h)
{
    const cuuint64_t dims[2] = {cuuint64_t(S), cuuint64_t(rows)};
    const cuuint64_t strides[1] = {cuuint64_t(S) * elem};
    const cuuint32_t box[2] = {cuuint32_t(box_w), cuuint32_t(box_h)};
    const cuuint32_t element_strides[2] = {1, 1};
    const CUresult r = tensor_map_encoder()(&map, type, 2, const_cast<void*>(base), dims, strides, box, element_strides,
        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS)
        fail(FC_ERR_CUDA, "tensor map encoding failed (%d)", int(r));
}

// Maps of every level the strip kernels smooth (levels below the tail), for both strip heights:
// weights (FP16 copies on coarse levels in mixed precision), the level's input vector, its
// pre-smoothed solution and the next level's solution.
void encode_stage_maps(Grid& g)
{
    const bool fp64 = g.precision == FC_PRECISION_FP64;
    const CUtensorMapDataType vt = fp64 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
    const int big = fp64 ? Tiling<double>::big : Tiling<float>::big;
    const int small = fp64 ? Tiling<double>::small : Tiling<float>::small;
    const int wide = fp64 ? Tiling<double>::wide : Tiling<float>::wide;
    // Strip rows of a region per shape: warps x strip height.
    const int rows[kShapes] = {8 * big, 8 * small, 16 * wide};
    std::vector<CUtensorMap> maps(g.levels.size() * kShapes * kMapsPerSet);
    std::memset(maps.data(), 0, maps.size() * sizeof(CUtensorMap));
    const GridDesc& d = g.desc;
    // Every level that has a coarser one: the tail threshold may move after allocation.
    for (int l = 0; l + 1 < int(g.levels.size()); ++l)
    {
        const LevelDesc& L = d.lev[l];
        const LevelDesc& C = d.lev[l + 1];
        const bool half = g.precision == FC_PRECISION_MIXED && l >= 1;
        for (int set = 0; set < kShapes; ++set)
        {
            const int bh = rows[set] + 1;
            CUtensorMap* m = &maps[(l * kShapes + set) * kMapsPerSet];
            if (half)
            {
                encode_box(m[kMapRight], L.right_h, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 2, L.S, L.h + 2, 72, bh);
                encode_box(m[kMapDown], L.down_h, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 2, L.S, L.h + 2, 72, bh);
            }
            else
            {
                encode_box(m[kMapRight], L.right, vt, g.elem, L.S, L.h + 2, 72, bh);
                encode_box(m[kMapDown], L.down, vt, g.elem, L.S, L.h + 2, 72, bh);
            }
            encode_box(m[kMapVector], l == 0 ? d.r : L.rhs, vt, g.elem, L.S, L.h + 2, 72, bh);
            encode_box(m[kMapInverse], L.inv, vt, g.elem, L.S, L.h + 2, 72, bh);
            encode_box(m[kMapPre], L.pre, vt, g.elem, L.S, L.h + 2, 72, bh);
            encode_box(m[kMapCoarse], C.sol, vt, g.elem, C.S, C.h + 2, 40, rows[set] / 2 + 4);
        }
    }
    check(cudaMemcpyAsync(const_cast<void*>(d.maps), maps.data(), maps.size() * sizeof(CUtensorMap),
              cudaMemcpyHostToDevice, g.stream),
        "tensor maps");
    // The host vector must outlive the copy.
    check(cudaStreamSynchronize(g.stream), "tensor maps");
}

// Lays out every device field of a grid in one allocation and fills the descriptor. With
// allocate false it only returns the arena size (no CUDA calls).
size_t allocate_grid(Grid& g, bool allocate = true)
{
    const int W = g.W, H = g.H;
    g.levels = build_levels(W, H);
    choose_tail(g);
    g.S = g.levels[0].S;
    g.cells = size_t(W) * H;
    g.faces_u = size_t(W + 1) * H;
    g.faces_v = size_t(W) * (H + 1);
    g.staging_count = std::max(g.faces_u, g.faces_v);

    struct Slot
    {
        void** where;
        size_t bytes;
    };
    std::vector<Slot> slots;
    const size_t elem = g.elem;
    GridDesc& d = g.desc;
    d = GridDesc{};
    d.W = W;
    d.H = H;
    d.S = g.S;
    d.dx = g.dx;
    d.levels = int(g.levels.size());
    d.tail = g.tail;
    const HostLevel& last = g.levels.back();
    d.ncoarse = last.w * last.h - 1;
    d.vec_tiles = ceil_div(W, kVecTileX) * ceil_div(H, kVecTileY);
    // The level-0 post kernel writes one (sum z, sum r z) pair per tile: slots for the most
    // tiles any region shape gives (two pairs to a double4 slot).
    const TileSizes ts = tile_sizes(g.precision, kShapeShort);
    d.post_tiles = g.tail > 0 ? ceil_div(W, ts.post_x) * ceil_div(H, ts.post_y) : 0;
    long long post_pairs = 0;
    for (int shape = 0; shape < kShapes && g.tail > 0; ++shape)
    {
        const TileSizes t = tile_sizes(g.precision, shape);
        post_pairs = std::max(post_pairs, (long long)ceil_div(W, t.post_x) * ceil_div(H, t.post_y));
    }

    const size_t padded0 = size_t(g.S) * (H + 2);
    auto add = [&](void** where, size_t bytes) { slots.push_back({where, bytes}); };
    add(&d.r, padded0 * elem);
    add(&d.z, padded0 * elem);
    add(&d.d[0], padded0 * elem);
    add(&d.d[1], padded0 * elem);
    add(&d.q, padded0 * elem);
    add((void**)&d.p, padded0 * sizeof(double));
    add((void**)&d.p_prev, padded0 * sizeof(double));
    add((void**)&d.b, padded0 * sizeof(double));
    add(&d.u, g.faces_u * elem);
    add(&d.v, g.faces_v * elem);
    // Up to every coarsest cell is an unknown (Dirichlet air pins none).
    add((void**)&d.coarse_inverse, size_t(std::max(1, (d.ncoarse + 1) * (d.ncoarse + 1))) * sizeof(double));
    add((void**)&d.coarse, sizeof(CoarseInfo));
    add((void**)&d.state, sizeof(SolveState));
    add((void**)&d.partial, size_t(std::max<long long>(std::max<long long>(d.vec_tiles, (post_pairs + 1) / 2), 1)) *
                                sizeof(double4));
    add((void**)&d.counter, sizeof(unsigned int) * 4);
    add((void**)&d.density, g.cells * sizeof(double));
    add((void**)&g.fraction, g.cells * sizeof(double));
    add((void**)&g.staging, g.staging_count * sizeof(double));
    add(&g.u_next, g.faces_u * elem);
    add(&g.v_next, g.faces_v * elem);
    add((void**)&g.solid, g.cells);
    add((void**)&g.mask, g.cells);
    add((void**)&g.air, g.cells);
    add((void**)&g.air_faces, g.faces_u + g.faces_v);
    add((void**)&d.lev[0].pre, padded0 * elem);
    std::vector<void*> cx(g.levels.size()), cy(g.levels.size()), px(g.levels.size()), py(g.levels.size()),
        rx(g.levels.size()), ry(g.levels.size()), rwx(g.levels.size()), rwy(g.levels.size());
    for (size_t l = 0; l < g.levels.size(); ++l)
    {
        const HostLevel& L = g.levels[l];
        LevelDesc& ld = d.lev[l];
        ld.w = L.w;
        ld.h = L.h;
        ld.S = L.S;
        const size_t padded = size_t(L.S) * (L.h + 2);
        add(&ld.right, padded * elem);
        add(&ld.down, padded * elem);
        if (l + 1 < g.levels.size())
            add(&ld.inv, padded * elem);
        // Mixed precision: FP16 copies of the weights of the coarse levels the strip kernels
        // smooth (the fine level keeps FP32 weights).
        if (g.precision == FC_PRECISION_MIXED && l >= 1 && l + 1 < g.levels.size())
        {
            add(const_cast<void**>(&ld.right_h), padded * sizeof(__half));
            add(const_cast<void**>(&ld.down_h), padded * sizeof(__half));
        }
        if (l > 0)
        {
            add(&ld.rhs, padded * elem);
            add(&ld.pre, padded * elem);
            add(&ld.sol, padded * elem);
        }
        add(&cx[l], L.cx.size() * sizeof(double));
        add(&cy[l], L.cy.size() * sizeof(double));
        if (l + 1 < g.levels.size())
        {
            add(&px[l], L.px.size() * sizeof(Interp));
            add(&py[l], L.py.size() * sizeof(Interp));
            add(&rx[l], L.rx.size() * sizeof(Gather));
            add(&ry[l], L.ry.size() * sizeof(Gather));
            HostLevel& H = g.levels[l];
            H.rwx = g.elem == 8 ? restrict_weights<double>(L.rx) : restrict_weights<float>(L.rx);
            H.rwy = g.elem == 8 ? restrict_weights<double>(L.ry) : restrict_weights<float>(L.ry);
            add(&rwx[l], H.rwx.size());
            add(&rwy[l], H.rwy.size());
        }
    }
    // TMA maps: per level, kShapes region shapes, kMapsPerSet maps of 128 bytes.
    add(const_cast<void**>(&d.maps), g.levels.size() * kShapes * kMapsPerSet * sizeof(CUtensorMap));
    size_t total = 0;
    std::vector<size_t> offsets;
    for (auto& s : slots)
    {
        offsets.push_back(total);
        total += (s.bytes + 255) / 256 * 256;
    }
    if (!allocate)
        return total;
    device_alloc(&g.arena, total, g.stream, "grid allocation");
    g.arena_bytes = total;
    check(cudaMemsetAsync(g.arena, 0, total, g.stream), "grid clear");
    for (size_t i = 0; i < slots.size(); ++i)
        *slots[i].where = g.arena + offsets[i];
    d.lev[0].sol = d.z;
    for (size_t l = 0; l < g.levels.size(); ++l)
    {
        const HostLevel& L = g.levels[l];
        LevelDesc& ld = d.lev[l];
        check(cudaMemcpyAsync(cx[l], L.cx.data(), L.cx.size() * sizeof(double), cudaMemcpyHostToDevice, g.stream), "centres");
        check(cudaMemcpyAsync(cy[l], L.cy.data(), L.cy.size() * sizeof(double), cudaMemcpyHostToDevice, g.stream), "centres");
        ld.cx = static_cast<const double*>(cx[l]);
        ld.cy = static_cast<const double*>(cy[l]);
        if (l + 1 < g.levels.size())
        {
            check(cudaMemcpyAsync(px[l], L.px.data(), L.px.size() * sizeof(Interp), cudaMemcpyHostToDevice, g.stream), "tables");
            check(cudaMemcpyAsync(py[l], L.py.data(), L.py.size() * sizeof(Interp), cudaMemcpyHostToDevice, g.stream), "tables");
            check(cudaMemcpyAsync(rx[l], L.rx.data(), L.rx.size() * sizeof(Gather), cudaMemcpyHostToDevice, g.stream), "tables");
            check(cudaMemcpyAsync(ry[l], L.ry.data(), L.ry.size() * sizeof(Gather), cudaMemcpyHostToDevice, g.stream), "tables");
            ld.px = static_cast<const Interp*>(px[l]);
            ld.py = static_cast<const Interp*>(py[l]);
            ld.rx = static_cast<const Gather*>(rx[l]);
            ld.ry = static_cast<const Gather*>(ry[l]);
            check(cudaMemcpyAsync(rwx[l], L.rwx.data(), L.rwx.size(), cudaMemcpyHostToDevice, g.stream), "tables");
            check(cudaMemcpyAsync(rwy[l], L.rwy.data(), L.rwy.size(), cudaMemcpyHostToDevice, g.stream), "tables");
            ld.rwx = rwx[l];
            ld.rwy = rwy[l];
        }
    }
    d.solid = nullptr;
    encode_stage_maps(g);
    check(cudaStreamSynchronize(g.stream), "grid set-up");
    return total;
}

// Bytes of the surface-tension sweeps of a grid (ensure_tension lays them out this way).
void tension_layout(size_t cells, size_t sizes[6])
{
    auto round = [](size_t b) { return (b + 255) / 256 * 256; };
    sizes[0] = round(cells * sizeof(double2));
    sizes[1] = round(2 * cells);
    sizes[2] = round(cells * sizeof(double));
    sizes[3] = round(cells);
    sizes[4] = round(cells * sizeof(double));
    sizes[5] = round(cells);
}

size_t tension_bytes(size_t cells)
{
    size_t sizes[6], total = 0;
    tension_layout(cells, sizes);
    for (size_t b : sizes)
        total += b;
    return total;
}

// Device bytes of a single-grid plan: descriptors, tile tables, solve states and parameters.
size_t plan_bytes(int W, int H)
{
    const size_t tiles = size_t(ceil_div(W, 16) + 1) * (ceil_div(H, 4) + 1) * 6;
    return (1u << 20) + tiles * 16;
}

// Component masses live in their own allocation (their count follows configureMaterials).
void allocate_masses(Grid& g)
{
    const int k = g.components();
    if (k == g.mass_capacity && g.masses)
        return;
    device_free(g.masses, g.stream);
    device_free(g.mass_ptrs, g.stream);
    g.masses = nullptr;
    g.mass_ptrs = nullptr;
    g.mass_capacity = k;
    if (k > 0)
    {
        device_alloc(&g.masses, size_t(k) * g.cells * sizeof(double), g.stream, "mass allocation");
        device_alloc(&g.mass_ptrs, size_t(k) * sizeof(double*), g.stream, "mass pointers");
        std::vector<double*> ptrs(k);
        for (int i = 0; i < k; ++i)
            ptrs[i] = g.masses + size_t(i) * g.cells;
        // On the grid's stream: its kernels and uploads are ordered after both. (A copy or set on
        // the legacy default stream is not ordered with the grid's non-blocking stream, and a
        // pageable copy may return before its data lands.)
        check(cudaMemcpyAsync(g.mass_ptrs, ptrs.data(), k * sizeof(double*), cudaMemcpyHostToDevice, g.stream),
            "mass pointers");
        check(cudaMemsetAsync(g.masses, 0, size_t(k) * g.cells * sizeof(double), g.stream), "mass clear");
    }
    g.desc.masses = g.mass_ptrs;
    g.desc.components = k;
}

// ------------------------------------------------------------------------------------------
// Plan: tile tables + descriptors + graph for a set of grids
// ------------------------------------------------------------------------------------------

struct Range
{
    int offset = 0;
    int count = 0;
};

struct ProjectParams
{
    double dt;
    double tol_max;
    double tol_sumsq; // negative: relative rule carrying -tol^2
    int max_iterations;
    int use_mg;
};

__global__ void k_init_states(const GridDesc* grids, int n, const ProjectParams* params, int* body_count)
{
    dependent_start();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0)
        *body_count = 0;
    if (i >= n)
        return;
    const GridDesc& g = grids[i];
    SolveState& s = *g.state;
    const ProjectParams p = params[i];
    const int mg_valid = s.mg_valid;
    s = SolveState{};
    s.mg_valid = mg_valid;
    s.use_mg = p.use_mg;
    s.tol_max = p.tol_max;
    s.tol_sumsq = p.tol_sumsq;
    s.max_iterations = p.max_iterations;
    s.restart = 1;
    s.rz = 1.0;
    s.dq = 1.0;
    s.dt = p.dt;
    // Dirichlet air: a non-singular system with no mean to take; a zero factor makes every mean
    // of the solve (right-hand side, pressure, residual, preconditioned residual) zero.
    s.inv_cells = g.air ? 0.0 : 1.0 / (double(g.W) * double(g.H));
    g.counter[0] = 0u;
}

// Open (non-solid) cells define the mean-free subspace of the solve.
__global__ void __launch_bounds__(kVecThreads) k_count_open(const GridDesc* __restrict__ grids, const Tile* __restrict__ tiles)
{
    dependent_start();
    const Tile t = tiles[blockIdx.x];
    const GridDesc& g = grids[t.grid];
    if (!g.solid || g.air)
        return;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    double open = 0.0;
    for (int k = 0; k < kVecCells; ++k)
    {
        const int x = t.x0 + tx + 32 * (k & 1), y = t.y0 + ty + 8 * (k >> 1);
        if (x >= g.W || y >= g.H)
            continue;
        open += g.solid[(long long)y * g.W + x] ? 0.0 : 1.0;
    }
    __shared__ double4 total;
    if (arrive_last<kVecThreads>(g, t.index, g.vec_tiles, block_reduce4<kVecThreads>(make_double4(open, 0, 0, 0), 0), &total, 0))
    {
        if (threadIdx.x == 0)
            g.state->inv_cells = total.x > 0.0 ? 1.0 / total.x : 0.0;
    }
}

__global__ void k_loop_condition(const GridDesc* grids, int n, int* body_count, int cap, cudaGraphConditionalHandle handle)
{
    allow_dependents();
    dependency_wait();
    int running = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x)
        running |= grids[i].state->done == 0;
    running = __syncthreads_or(running);
    if (threadIdx.x == 0)
    {
        const int bodies = ++*body_count;
        cudaGraphSetConditional(handle, (running && bodies < cap) ? 1u : 0u);
    }
}

__global__ void k_gather_states(const GridDesc* grids, int n, SolveState* out)
{
    dependent_start();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        out[i] = *grids[i].state;
}

// v += g dt on interior horizontal faces (FluidGridCPU.cpp:987-996): every cell below the top
// row updates its upper face.
template <typename T> __global__ void k_gravity(const GridDesc* grids, const Tile* tiles, double increment)
{
    const Tile t = tiles[blockIdx.x];
    const GridDesc& g = grids[t.grid];
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    T* v = static_cast<T*>(g.v);
    for (int k = 0; k < kVecCells; ++k)
    {
        const int x = t.x0 + tx + 32 * (k & 1), y = t.y0 + ty + 8 * (k >> 1);
        if (x >= g.W || y >= g.H || y == 0)
            continue;
        const long long f = (long long)y * g.W + x;
        v[f] = T(double(v[f]) + increment);
    }
}

// ------------------------------------------------------------------------------------------
// Velocity extension into Dirichlet air (no reference counterpart)
// ------------------------------------------------------------------------------------------
//
// Under Dirichlet air nothing constrains the face velocities between air cells: gravity keeps
// accelerating them, and transport, which samples and moves the velocity field on both sides
// of the surface, would carry that into the liquid. Before each substep the liquid's velocity
// is therefore extended into the air layer by layer (the constant extrapolation of R. Bridson,
// Fluid Simulation for Computer Graphics, 2nd ed., sec. 4.5): a face known to layer k - 1 keeps
// its value, an unknown face beside known ones takes their mean and joins layer k, and after
// kAirLayers layers the faces still unknown are set to zero. Faces of liquid cells, solid faces
// and the walls form layer 0.
constexpr int kAirLayers = 4;
constexpr unsigned char kAirUnknown = 255;

__device__ __forceinline__ bool liquid_cell(const GridDesc& g, int x, int y)
{
    const long long c = (long long)y * g.W + x;
    return !(g.solid && g.solid[c]) && g.fraction[c] > 0.5;
}

__device__ __forceinline__ bool solid_cell(const GridDesc& g, int x, int y)
{
    return g.solid && g.solid[(long long)y * g.W + x];
}

// Layer 0 over the face tiles ((W + 1) x (H + 1) positions: u face (x, y) for y < H, v face
// (x, y) for x < W).
__global__ void k_air_faces_init(const GridDesc* grids, const Tile* tiles, unsigned char* known_u, unsigned char* known_v)
{
    const Tile t = tiles[blockIdx.x];
    const GridDesc& g = grids[t.grid];
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    for (int k = 0; k < kVecCells; ++k)
    {
        const int x = t.x0 + tx + 32 * (k & 1), y = t.y0 + ty + 8 * (k >> 1);
        if (x <= g.W && y < g.H)
        {
            const bool known = x == 0 || x == g.W || solid_cell(g, x - 1, y) || solid_cell(g, x, y) ||
                               liquid_cell(g, x - 1, y) || liquid_cell(g, x, y);
            known_u[(long long)y * (g.W + 1) + x] = known ? 0 : kAirUnknown;
        }
        if (x < g.W && y <= g.H)
        {
            const bool known = y == 0 || y == g.H || solid_cell(g, x, y - 1) || solid_cell(g, x, y) ||
                               liquid_cell(g, x, y - 1) || liquid_cell(g, x, y);
            known_v[(long long)y * g.W + x] = known ? 0 : kAirUnknown;
        }
    }
}

// Layer `layer` of one face array (nx x ny faces). Faces written in this pass were unknown and
// are read by none of this pass's faces (they read faces of layers < `layer` only), so the
// update is in place and independent of the order in which faces run.
template <typename T>
__device__ __forceinline__ void extend_face(T* value, unsigned char* known, int nx, int ny, int x, int y, int layer)
{
    const long long f = (long long)y * nx + x;
    if (known[f] != kAirUnknown)
        return;
    double sum = 0.0;
    int count = 0;
    const int dx[4] = {-1, 1, 0, 0}, dy[4] = {0, 0, -1, 1};
#pragma unroll
    for (int n = 0; n < 4; ++n)
    {
        const int qx = x + dx[n], qy = y + dy[n];
        if (qx < 0 || qx >= nx || qy < 0 || qy >= ny)
            continue;
        const long long q = (long long)qy * nx + qx;
        if (known[q] < layer)
        {
            sum += double(value[q]);
            ++count;
        }
    }
    if (count > 0)
    {
        value[f] = T(sum / count);
        known[f] = (unsigned char)layer;
    }
    else if (layer == kAirLayers)
        value[f] = T(0);
}

template <typename T>
__global__ void k_air_faces_extend(const GridDesc* grids, const Tile* tiles, unsigned char* known_u, unsigned char* known_v,
    int layer)
{
    const Tile t = tiles[blockIdx.x];
    const GridDesc& g = grids[t.grid];
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    for (int k = 0; k < kVecCells; ++k)
    {
        const int x = t.x0 + tx + 32 * (k & 1), y = t.y0 + ty + 8 * (k >> 1);
        if (x <= g.W && y < g.H)
            extend_face(static_cast<T*>(g.u), known_u, g.W + 1, g.H, x, y, layer);
        if (x < g.W && y <= g.H)
            extend_face(static_cast<T*>(g.v), known_v, g.W, g.H + 1, x, y, layer);
    }
}

__global__ void k_classify(const GridDesc* grids, const Tile* tiles, const double* fraction, unsigned char* mask)
{
    const Tile t = tiles[blockIdx.x];
    const GridDesc& g = grids[t.grid];
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    for (int k = 0; k < kVecCells; ++k)
    {
        const int x = t.x0 + tx + 32 * (k & 1), y = t.y0 + ty + 8 * (k >> 1);
        if (x >= g.W || y >= g.H)
            continue;
        const long long i = (long long)y * g.W + x;
        unsigned char m = 0;
        if (g.solid && g.solid[i])
            m = 4;
        else
        {
            const double f = fraction[i];
            if (f > 0.5)
                m |= 1;
            if (f > 0.0 && f < 1.0)
                m |= 2;
        }
        mask[i] = m;
    }
}

struct Plan
{
    std::vector<Grid*> grids;
    int precision = FC_PRECISION_FP32;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    GridDesc* d_desc = nullptr;
    Tile* d_tiles = nullptr;
    ProjectParams* d_params = nullptr;
    ProjectParams* h_params = nullptr; // host copies (pageable)
    SolveState* d_states = nullptr;
    SolveState* h_states = nullptr;
    int* d_body_count = nullptr;
    Range vec;
    Range faces; // tiles over the (W+1) x (H+1) face index space
    Range pre[kMaxLevels];
    Range post[kMaxLevels];
    // Region shape (RegionShape) of each level's pre- and post-smoothing kernels.
    int shape_pre[kMaxLevels] = {};
    int shape_post[kMaxLevels] = {};
    // The fine level's post-smoothing folds each grid's z sums per region, so its regions take
    // each grid's own shape (the one the grid would have alone): results then do not depend on
    // which grids share the plan. post0[shape] holds the regions of the grids of that shape.
    Range post0[kShapes];
    std::vector<int> post0_shape; // per grid
    int max_levels = 0;
    int max_tail = 0;
    int padded_max[kMaxLevels] = {}; // largest padded level array of any grid, per level
    size_t tail_smem = 0;
    cudaGraphExec_t exec = nullptr;
    cudaGraph_t graph = nullptr;
    int graph_cap = -1;
    int graph_use_mg = -1;
    int h_bodies = 0;       // loop bodies the last projection ran
    int setup_kernels = 0;  // kernels outside the loop in the captured graph
    int body_kernels = 0;   // kernels of one loop body
    int rebuild_kernels = 0;

    ~Plan()
    {
        if (exec)
            cudaGraphExecDestroy(exec);
        if (graph)
            cudaGraphDestroy(graph);
        for (void* ptr : {(void*)d_desc, (void*)d_tiles, (void*)d_params, (void*)d_states, (void*)d_body_count})
            device_free(ptr, stream);
        delete[] h_params;
        delete[] h_states;
        if (own_stream && stream)
            cudaStreamDestroy(stream);
    }

    const Tile* at(const Range& r) const { return d_tiles + r.offset; }
    int n() const { return int(grids.size()); }
};

Grid::~Grid()
{
    plan.reset();
    for (void* ptr : {(void*)masses, (void*)mass_ptrs, (void*)tension_arena, (void*)visc_arena, (void*)plic_arena,
             (void*)arena})
        device_free(ptr, stream);
    if (stream)
        cudaStreamDestroy(stream);
}

void append_tiles(std::vector<Tile>& tiles, int grid, int w, int h, int tx, int ty)
{
    int index = 0;
    for (int y = 0; y < h; y += ty)
        for (int x = 0; x < w; x += tx)
            tiles.push_back({grid, x, y, index++});
}

void upload_descriptors(Plan& plan)
{
    std::vector<GridDesc> descs(plan.n());
    for (int i = 0; i < plan.n(); ++i)
    {
        descs[i] = plan.grids[i]->desc;
        // Level-0 post regions of this grid (its own shape): the count its z reduction waits for.
        const Grid& g = *plan.grids[i];
        const int shape = i < int(plan.post0_shape.size()) ? plan.post0_shape[i] : kShapeShort;
        const TileSizes ts = tile_sizes(plan.precision, shape);
        descs[i].post_tiles = g.tail > 0 ? ceil_div(g.W, ts.post_x) * ceil_div(g.H, ts.post_y) : 0;
    }
    check(cudaMemcpyAsync(plan.d_desc, descs.data(), descs.size() * sizeof(GridDesc), cudaMemcpyHostToDevice, plan.stream),
        "plan descriptors");
    check(cudaStreamSynchronize(plan.stream), "plan descriptors");
}

// Region shape of a level from its region counts in the tall and wide shapes: tall regions once
// there is one for every other SM (a tall region costs less than the two short ones it
// replaces: the per-region latency is paid once, with less halo); short strips, which halve
// each CTA's latency, on the smaller levels; in FP32 the wide shape (one 16-warp CTA per SM,
// the least halo per output cell) for levels with four waves of regions.
int region_shape(int precision, long long tall_regions, long long wide_regions, int sms)
{
    if (precision != FC_PRECISION_FP64 && wide_regions >= 4LL * sms)
        return kShapeWide;
    return 2 * tall_regions >= sms ? kShapeTall : kShapeShort;
}

std::unique_ptr<Plan> make_plan(const std::vector<Grid*>& grids, cudaStream_t stream)
{
    auto plan = std::make_unique<Plan>();
    plan->grids = grids;
    plan->precision = grids.front()->precision;
    if (stream)
        plan->stream = stream;
    else
    {
        int priority = 0;
        for (const Grid* g : grids)
            priority = std::min(priority, g->stream_priority);
        check(cudaStreamCreateWithPriority(&plan->stream, cudaStreamNonBlocking, priority), "plan stream");
        plan->own_stream = true;
    }
    const int n = plan->n();
    std::vector<Tile> tiles;
    auto add = [&](Range& r, auto&& body)
    {
        r.offset = int(tiles.size());
        body();
        r.count = int(tiles.size()) - r.offset;
    };
    add(plan->vec, [&]
    {
        for (int i = 0; i < n; ++i)
            append_tiles(tiles, i, grids[i]->W, grids[i]->H, kVecTileX, kVecTileY);
    });
    add(plan->faces, [&]
    {
        for (int i = 0; i < n; ++i)
            append_tiles(tiles, i, grids[i]->W + 1, grids[i]->H + 1, kVecTileX, kVecTileY);
    });
    for (Grid* g : grids)
    {
        plan->max_levels = std::max(plan->max_levels, int(g->levels.size()));
        plan->max_tail = std::max(plan->max_tail, g->tail);
        plan->tail_smem = std::max(plan->tail_smem, g->tail_smem);
        for (size_t l = 0; l < g->levels.size(); ++l)
            plan->padded_max[l] = std::max(plan->padded_max[l], g->levels[l].S * (g->levels[l].h + 2));
    }
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, grids.front()->device);
    for (int l = 0; l < plan->max_tail; ++l)
    {
        auto tiles_of = [&](int shape, int only)
        {
            const TileSizes t = tile_sizes(plan->precision, shape);
            long long count = 0;
            for (int i = 0; i < n; ++i)
                if (l < grids[i]->tail && (only < 0 || i == only))
                    count += (long long)ceil_div(grids[i]->levels[l].w, t.pre_x) * ceil_div(grids[i]->levels[l].h, t.pre_y);
            return count;
        };
        const int shape = region_shape(plan->precision, tiles_of(kShapeTall, -1), tiles_of(kShapeWide, -1), sms);
        if (l == 0)
        {
            plan->post0_shape.assign(n, kShapeShort);
            for (int i = 0; i < n; ++i)
                plan->post0_shape[i] = region_shape(plan->precision, tiles_of(kShapeTall, i), tiles_of(kShapeWide, i), sms);
            for (int set = 0; set < kShapes; ++set)
            {
                const TileSizes tq = tile_sizes(plan->precision, set);
                add(plan->post0[set], [&]
                {
                    for (int i = 0; i < n; ++i)
                        if (grids[i]->tail > 0 && plan->post0_shape[i] == set)
                            append_tiles(tiles, i, grids[i]->W, grids[i]->H, tq.post_x, tq.post_y);
                });
            }
        }
        plan->shape_pre[l] = shape;
        plan->shape_post[l] = shape;
        const TileSizes tp = tile_sizes(plan->precision, plan->shape_pre[l]);
        const TileSizes tq = tile_sizes(plan->precision, plan->shape_post[l]);
        add(plan->pre[l], [&]
        {
            for (int i = 0; i < n; ++i)
                if (l < grids[i]->tail)
                    append_tiles(tiles, i, grids[i]->levels[l].w, grids[i]->levels[l].h, tp.pre_x, tp.pre_y);
        });
        if (l > 0)
            add(plan->post[l], [&]
            {
                for (int i = 0; i < n; ++i)
                    if (l < grids[i]->tail)
                        append_tiles(tiles, i, grids[i]->levels[l].w, grids[i]->levels[l].h, tq.post_x, tq.post_y);
            });
    }
    device_alloc(&plan->d_tiles, std::max<size_t>(1, tiles.size()) * sizeof(Tile), plan->stream, "plan tiles");
    // On the plan's stream, which every kernel reading the tiles runs on (a copy on the legacy
    // default stream is not ordered with it and may return before its data lands).
    check(cudaMemcpyAsync(plan->d_tiles, tiles.data(), tiles.size() * sizeof(Tile), cudaMemcpyHostToDevice, plan->stream),
        "plan tiles");
    device_alloc(&plan->d_desc, n * sizeof(GridDesc), plan->stream, "plan descriptors");
    device_alloc(&plan->d_params, n * sizeof(ProjectParams), plan->stream, "plan params");
    device_alloc(&plan->d_states, n * sizeof(SolveState), plan->stream, "plan states");
    device_alloc(&plan->d_body_count, sizeof(int), plan->stream, "plan counter");
    // Host copies in pageable memory: the copies into them complete before their call returns,
    // and pinned memory would need a freeing call that synchronises the device.
    plan->h_params = new ProjectParams[n]();
    plan->h_states = new SolveState[n]();
    upload_descriptors(*plan);
    return plan;
}

// ------------------------------------------------------------------------------------------
// Launch sequences
// ------------------------------------------------------------------------------------------

// Density, face weights, multigrid conductances and the coarsest inverse of every grid.
// The kernels are launched with programmatic serialization: each starts with dependent_start(),
// so its launch overlaps the end of its predecessor.
template <typename T> void launch_rebuild(Plan& p)
{
    cudaStream_t s = p.stream;
    FC_LAUNCH_DEP(k_density, p.vec.count, kVecThreads, 0, s, p.d_desc, p.at(p.vec));
    FC_LAUNCH_DEP(k_coefficients<T>, p.vec.count, kVecThreads, 0, s, p.d_desc, p.at(p.vec));
    for (int l = 0; l + 1 < p.max_levels; ++l)
        FC_LAUNCH_DEP(k_coarsen<T>, dim3(ceil_div(p.padded_max[l + 1], 256), p.n()), 256, 0, s, p.d_desc, l);
    static const bool inverse_configured = [&]
    {
        check(cudaFuncSetAttribute(k_coarse_inverse<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kCoarseInverseSmem)),
            "coarse inverse shared memory");
        return true;
    }();
    (void)inverse_configured;
    if (p.precision == FC_PRECISION_MIXED)
        for (int l = 1; l < p.max_tail; ++l)
            FC_LAUNCH_DEP(k_weights_half, dim3(ceil_div(p.padded_max[l], 256), p.n()), 256, 0, s, p.d_desc, l);
    // Level by level: under Dirichlet air a coarse level's held cells follow from the finer
    // level's inverse diagonal, and the coarsest factor from the level above it.
    for (int l = 0; l + 1 < p.max_levels; ++l)
        FC_LAUNCH_DEP(k_inverse_diagonal<T>, dim3(ceil_div(p.padded_max[l], 256), p.n()), 256, 0, s, p.d_desc, l);
    FC_LAUNCH_DEP(k_coarse_inverse<T>, p.n(), kCoarseThreads, kCoarseInverseSmem, s, p.d_desc);
}

// Resident CTAs of the persistent smoothing kernels: two per SM in FP32, one in FP64 (their
// launch bounds and shared-memory staging).
int sm_count()
{
    static int sms = 0;
    if (!sms)
    {
        int device = 0;
        check(cudaGetDevice(&device), "device");
        check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device), "SM count");
    }
    return sms;
}

int smoothing_ctas(bool fp64) { return sm_count() * (fp64 ? 1 : 2); }

template <typename T, int K, typename W, bool PRE, int WARPS>
void launch_smooth_kernel(Plan& p, const Range& r, int level, int set, bool dependent, cudaStream_t s)
{
    using St = Stage<T, W, K, PRE, WARPS>;
    if (r.count <= 0)
        return;
    auto kernel = PRE ? k_smooth_pre<T, K, W, WARPS> : k_smooth_post<T, K, W, WARPS>;
    static const bool configured = [&]
    {
        check(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(St::bytes)),
            "smoothing shared memory");
        return true;
    }();
    (void)configured;
    // Resident CTAs: two per SM for 8-warp FP32 regions, one otherwise.
    const int ctas = std::min(r.count, smoothing_ctas(sizeof(T) == 8 || WARPS > 8));
    if (dependent)
        FC_LAUNCH_DEP(kernel, ctas, 32 * WARPS, St::bytes, s, p.d_desc, p.at(r), r.count, level, set);
    else
        FC_LAUNCH(kernel, ctas, 32 * WARPS, St::bytes, s, p.d_desc, p.at(r), r.count, level, set);
}

template <typename T, typename W, bool PRE>
void launch_smooth_shape(Plan& p, const Range& r, int level, int shape, bool dependent, cudaStream_t s)
{
    constexpr int KB = Tiling<T>::big, KS = Tiling<T>::small, KW = Tiling<T>::wide;
    if constexpr (sizeof(T) == 4)
    {
        if (shape == kShapeWide)
            return launch_smooth_kernel<T, KW, W, PRE, 16>(p, r, level, shape, dependent, s);
    }
    if (shape == kShapeShort)
        launch_smooth_kernel<T, KS, W, PRE, 8>(p, r, level, shape, dependent, s);
    else
        launch_smooth_kernel<T, KB, W, PRE, 8>(p, r, level, shape, dependent, s);
}

// The pre- or post-smoothing kernel of one level in the plan's region shape, with FP16 weights
// on the coarse levels of a mixed-precision plan.
template <typename T> void launch_smooth(Plan& p, int level, bool pre, bool dependent, cudaStream_t s)
{
    if (!pre && level == 0)
    {
        // One launch per region shape the plan's grids take on the fine level.
        for (int shape = 0; shape < kShapes; ++shape)
            launch_smooth_shape<T, T, false>(p, p.post0[shape], 0, shape, dependent, s);
        return;
    }
    const Range& r = pre ? p.pre[level] : p.post[level];
    const int shape = pre ? p.shape_pre[level] : p.shape_post[level];
    if constexpr (sizeof(T) == 4)
    {
        if (p.precision == FC_PRECISION_MIXED && level >= 1)
        {
            pre ? launch_smooth_shape<T, __half, true>(p, r, level, shape, dependent, s)
                : launch_smooth_shape<T, __half, false>(p, r, level, shape, dependent, s);
            return;
        }
    }
    pre ? launch_smooth_shape<T, T, true>(p, r, level, shape, dependent, s)
        : launch_smooth_shape<T, T, false>(p, r, level, shape, dependent, s);
}

// One application of the preconditioner to r: z, mean z, r.z and beta.
template <typename T> void launch_precondition(Plan& p, bool use_mg)
{
    cudaStream_t s = p.stream;
    if (!use_mg)
    {
        FC_LAUNCH_DEP(k_precondition_diagonal<T>, p.vec.count, kVecThreads, 0, s, p.d_desc, p.at(p.vec));
        return;
    }
    for (int l = 0; l < p.max_tail; ++l)
        launch_smooth<T>(p, l, true, true, s);
    FC_LAUNCH_DEP(k_mg_tail<T>, p.n(), kTailThreads, p.tail_smem, s, p.d_desc);
    for (int l = p.max_tail - 1; l >= 0; --l)
        launch_smooth<T>(p, l, false, true, s);
}

template <typename T> void launch_iteration(Plan& p, bool use_mg, int parity)
{
    cudaStream_t s = p.stream;
    FC_LAUNCH_DEP(k_direction_operator<T>, p.vec.count, kVecThreads, 0, s, p.d_desc, p.at(p.vec), parity);
    FC_LAUNCH_DEP(k_update<T>, std::min(p.vec.count, kUpdateCtasPerSm * sm_count()), kVecThreads, 0, s, p.d_desc,
        p.at(p.vec), p.vec.count, parity);
    FC_LAUNCH_DEP(k_true_residual<T>, p.vec.count, kVecThreads, 0, s, p.d_desc, p.at(p.vec), 0);
    launch_precondition<T>(p, use_mg);
}

template <typename T> void set_kernel_attributes(Plan& p)
{
    // Always opted in: the tail's static edge rows count against the 48 KB default as well.
    // The limit only ever rises (to the largest tail any plan has launched), so plans driven
    // from several threads never lower it under one another's launches.
    static std::mutex lock;
    static size_t opted = 0;
    std::lock_guard<std::mutex> guard(lock);
    if (p.tail_smem > opted)
    {
        check(cudaFuncSetAttribute(k_mg_tail<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(p.tail_smem)),
            "tail shared memory");
        opted = p.tail_smem;
    }
}

// Projection set-up: states, right-hand side, warm start, first residual, first z.
template <typename T> void launch_setup(Plan& p, bool use_mg)
{
    cudaStream_t s = p.stream;
    // The first launch follows a copy (or starts the graph); the others follow a kernel.
    FC_LAUNCH(k_init_states, ceil_div(p.n(), 128), 128, 0, s, p.d_desc, p.n(), p.d_params, p.d_body_count);
    FC_LAUNCH_DEP(k_count_open, p.vec.count, kVecThreads, 0, s, p.d_desc, p.at(p.vec));
    FC_LAUNCH_DEP(k_rhs<T>, p.vec.count, kVecThreads, 0, s, p.d_desc, p.at(p.vec));
    FC_LAUNCH_DEP(k_rhs_stats<T>, p.vec.count, kVecThreads, 0, s, p.d_desc, p.at(p.vec));
    FC_LAUNCH_DEP(k_warm_start, p.vec.count, kVecThreads, 0, s, p.d_desc, p.at(p.vec));
    FC_LAUNCH_DEP(k_remove_pressure_mean, p.vec.count, kVecThreads, 0, s, p.d_desc, p.at(p.vec));
    FC_LAUNCH_DEP(k_true_residual<T>, p.vec.count, kVecThreads, 0, s, p.d_desc, p.at(p.vec), 1);
    launch_precondition<T>(p, use_mg);
}

// After the solve: final mean removal, velocity update, divergence, results gathered.
template <typename T> void launch_finish(Plan& p)
{
    cudaStream_t s = p.stream;
    // The first launch follows the loop (a conditional node in the graph); the others follow a
    // kernel.
    FC_LAUNCH(k_flush_pressure<T>, p.vec.count, kVecThreads, 0, s, p.d_desc, p.at(p.vec));
    FC_LAUNCH_DEP(k_pressure_sum, p.vec.count, kVecThreads, 0, s, p.d_desc, p.at(p.vec));
    FC_LAUNCH_DEP(k_velocity_update<T>, p.vec.count, kVecThreads, 0, s, p.d_desc, p.at(p.vec));
    FC_LAUNCH_DEP(k_remove_pressure_mean, p.vec.count, kVecThreads, 0, s, p.d_desc, p.at(p.vec));
    FC_LAUNCH_DEP(k_divergence<T>, p.vec.count, kVecThreads, 0, s, p.d_desc, p.at(p.vec));
    FC_LAUNCH_DEP(k_gather_states, ceil_div(p.n(), 128), 128, 0, s, p.d_desc, p.n(), p.d_states);
}

// Launch mechanism of the PCG loop: one CUDA graph with a device-side WHILE node (default), or
// host-driven launches that poll the per-grid done flags (for per-kernel profilers, and where
// conditional graph nodes are unavailable). Both run the same kernels in the same order.
std::atomic<int> launch_mode{FC_LAUNCH_GRAPH};

// Captures the projection: set-up, WHILE { 2 iterations, condition }, velocity, divergence.
template <typename T> void capture_projection(Plan& p, bool use_mg, int cap)
{
    if (p.exec)
    {
        cudaGraphExecDestroy(p.exec);
        p.exec = nullptr;
    }
    if (p.graph)
    {
        cudaGraphDestroy(p.graph);
        p.graph = nullptr;
    }
    set_kernel_attributes<T>(p);
    cudaStream_t s = p.stream;
    cudaGraph_t graph;
    check(cudaGraphCreate(&graph, 0), "graph create");
    p.graph = graph;

    // Set-up, captured into the outer graph.
    const long long before_setup = thread_launches;
    check(cudaStreamBeginCaptureToGraph(s, graph, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal), "capture");
    launch_setup<T>(p, use_mg);

    // The conditional node depends on everything captured so far.
    cudaStreamCaptureStatus status;
    const cudaGraphNode_t* deps = nullptr;
    size_t ndeps = 0;
    check(cudaStreamGetCaptureInfo(s, &status, nullptr, nullptr, &deps, &ndeps), "capture info");
    std::vector<cudaGraphNode_t> dependencies(deps, deps + ndeps);
    cudaGraphConditionalHandle handle;
    check(cudaGraphConditionalHandleCreate(&handle, graph, 1, cudaGraphCondAssignDefault), "conditional handle");
    cudaGraphNodeParams params = {};
    params.type = cudaGraphNodeTypeConditional;
    params.conditional.handle = handle;
    params.conditional.type = cudaGraphCondTypeWhile;
    params.conditional.size = 1;
    cudaGraphNode_t loop;
    check(cudaGraphAddNode(&loop, graph, dependencies.data(), dependencies.size(), &params), "while node");
    cudaGraph_t body = params.conditional.phGraph_out[0];
    check(cudaStreamUpdateCaptureDependencies(s, &loop, 1, cudaStreamSetCaptureDependencies), "capture deps");

    // Finishing kernels after the loop, in the outer graph.
    launch_finish<T>(p);
    cudaGraph_t captured;
    check(cudaStreamEndCapture(s, &captured), "end capture");
    p.setup_kernels = int(thread_launches - before_setup);
    const long long before_body = thread_launches;

    // Loop body: two iterations (the direction buffers alternate) and the condition.
    cudaStream_t side;
    check(cudaStreamCreateWithFlags(&side, cudaStreamNonBlocking), "body stream");
    check(cudaStreamBeginCaptureToGraph(side, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal), "body capture");
    {
        Plan& q = p;
        cudaStream_t saved = q.stream;
        q.stream = side;
        launch_iteration<T>(q, use_mg, 0);
        launch_iteration<T>(q, use_mg, 1);
        FC_LAUNCH_DEP(k_loop_condition, 1, 256, 0, side, q.d_desc, q.n(), q.d_body_count, cap, handle);
        q.stream = saved;
    }
    cudaGraph_t body_captured;
    check(cudaStreamEndCapture(side, &body_captured), "body end capture");
    cudaStreamDestroy(side);
    p.body_kernels = int(thread_launches - before_body);
    // Captured launches are not executions: take them back out of the process counter, which
    // then advances by the executed kernels after each projection.
    launch_count.fetch_sub(p.setup_kernels + p.body_kernels);

    check(cudaGraphInstantiate(&p.exec, graph, 0), "graph instantiate");
    p.graph_cap = cap;
    p.graph_use_mg = use_mg ? 1 : 0;
}

// Runs one projection of every grid of the plan; returns the kernels executed on the device.
template <typename T> long long run_projection(Plan& p, bool use_mg, int max_iterations)
{
    const int cap = (std::max(max_iterations, 0) + 1) / 2 + 8;
    if (launch_mode.load() == FC_LAUNCH_STREAM)
    {
        set_kernel_attributes<T>(p);
        const long long before = thread_launches;
        check(cudaMemcpyAsync(p.d_params, p.h_params, p.n() * sizeof(ProjectParams), cudaMemcpyHostToDevice, p.stream),
            "params");
        launch_setup<T>(p, use_mg);
        int bodies = 0;
        for (;;)
        {
            launch_iteration<T>(p, use_mg, 0);
            launch_iteration<T>(p, use_mg, 1);
            ++bodies;
            FC_LAUNCH(k_gather_states, ceil_div(p.n(), 128), 128, 0, p.stream, p.d_desc, p.n(), p.d_states);
            check(cudaMemcpyAsync(p.h_states, p.d_states, p.n() * sizeof(SolveState), cudaMemcpyDeviceToHost, p.stream),
                "poll");
            check(cudaStreamSynchronize(p.stream), "poll");
            bool all_done = true;
            for (int i = 0; i < p.n(); ++i)
                all_done &= p.h_states[i].done != 0;
            if (all_done || bodies >= cap)
                break;
        }
        launch_finish<T>(p);
        check(cudaMemcpyAsync(p.h_states, p.d_states, p.n() * sizeof(SolveState), cudaMemcpyDeviceToHost, p.stream),
            "results");
        check(cudaStreamSynchronize(p.stream), "projection");
        p.h_bodies = bodies;
        return thread_launches - before;
    }
    if (!p.exec || p.graph_cap != cap || p.graph_use_mg != (use_mg ? 1 : 0))
        capture_projection<T>(p, use_mg, cap);
    check(cudaMemcpyAsync(p.d_params, p.h_params, p.n() * sizeof(ProjectParams), cudaMemcpyHostToDevice, p.stream),
        "params");
    check(cudaGraphLaunch(p.exec, p.stream), "graph launch");
    check(cudaMemcpyAsync(p.h_states, p.d_states, p.n() * sizeof(SolveState), cudaMemcpyDeviceToHost, p.stream),
        "results");
    check(cudaMemcpyAsync(&p.h_bodies, p.d_body_count, sizeof(int), cudaMemcpyDeviceToHost, p.stream), "results");
    check(cudaStreamSynchronize(p.stream), "projection");
    const long long executed = p.setup_kernels + (long long)p.h_bodies * p.body_kernels;
    launch_count.fetch_add(executed);
    return executed;
}

void fill_result(const Grid& g, const SolveState& s, double divergence_tolerance, fc_result* out)
{
    fc_result r{};
    r.physical_steps = 1;
    r.solve_status = s.status;
    if (s.status == kBreakdown)
    {
        // The reference returns a default result on a coarse breakdown (FluidGridCPU.cpp:1095-1096).
        r.iterations = 0;
        r.max_divergence = INFINITY;
        r.converged = 0;
    }
    else
    {
        r.iterations = s.iterations;
        r.max_divergence = s.div_max;
        r.converged = s.div_max <= divergence_tolerance;
        r.precision_limited =
            !r.converged && (s.status == kConverged || s.status == kNoWork) && s.div_excess <= divergence_tolerance;
    }
    r.residual_max = s.res_max;
    r.residual_l2 = std::sqrt(s.res_sumsq);
    r.rhs_l2 = std::sqrt(s.bsumsq);
    r.divergence_excess = s.div_excess;
    r.divergence_l2 = std::sqrt(s.div_sumsq);
    r.restarts = s.restarts;
    r.refreshes = s.refreshes;
    if (s.status == kNoWork)
    {
        r.residual_max = s.bmax;
        r.residual_l2 = std::sqrt(s.bsumsq);
    }
    *out = r;
}

// ------------------------------------------------------------------------------------------
// Grid operations
// ------------------------------------------------------------------------------------------

Plan& single_plan(Grid& g)
{
    if (!g.plan)
        g.plan = make_plan({&g}, g.stream);
    return *g.plan;
}

template <typename F> void dispatch(int precision, F&& body)
{
    if (precision == FC_PRECISION_FP64)
        body(double{});
    else
        body(float{});
}

// Per-level scale of the FP16 weights: a fine weight 2 / (rho_a + rho_b) is at most 1 / rho_min,
// and each coarsening at most doubles the largest weight (two parallel rows of series faces),
// so level l's weights divided by 2^l / rho_min lie in (0, 1].
void set_weight_scales(Grid& g)
{
    double rho_min = 0.0;
    for (const auto* set : {&g.liquid_density, &g.gas_density})
        for (double rho : *set)
            rho_min = rho_min == 0.0 ? rho : std::min(rho_min, rho);
    for (size_t l = 0; l < g.levels.size(); ++l)
        g.desc.lev[l].wscale = float(rho_min > 0.0 ? std::ldexp(1.0 / rho_min, int(l)) : 1.0);
}

void refresh_descriptor(Grid& g)
{
    set_weight_scales(g);
    g.desc.solid = g.has_solid ? g.solid : nullptr;
    g.desc.air = g.air_model == FC_AIR_DIRICHLET ? g.air : nullptr;
    g.desc.fraction = g.fraction;
    g.desc.masses = g.mass_ptrs;
    g.desc.components = g.components();
    if (g.plan)
        upload_descriptors(*g.plan);
}

void rebuild_if_dirty(Plan& p)
{
    bool dirty = false;
    for (Grid* g : p.grids)
        dirty |= g->coefficients_dirty;
    if (!dirty)
        return;
    const long long before = thread_launches;
    dispatch(p.precision, [&](auto zero)
    {
        using T = decltype(zero);
        launch_rebuild<T>(p);
    });
    p.rebuild_kernels = int(thread_launches - before);
    for (Grid* g : p.grids)
        g->coefficients_dirty = false;
}

void require_uploaded(const Grid& g)
{
    if (!g.uploaded)
        fail(FC_ERR_LIFECYCLE, "upload the grid state before stepping");
}

void project_plan(Plan& p, const double* dts, int max_iterations, double divergence_tolerance, double relative_tolerance,
    fc_result* results)
{
    p.rebuild_kernels = 0;
    for (Grid* g : p.grids)
        require_uploaded(*g);
    const bool use_mg = p.grids.front()->preconditioner == FC_PRECONDITIONER_MULTIGRID;
    for (Grid* g : p.grids)
        if ((g->preconditioner == FC_PRECONDITIONER_MULTIGRID) != use_mg)
            fail(FC_ERR_INVALID_ARGUMENT, "a batch needs one preconditioner for all grids");
    rebuild_if_dirty(p);
    for (int i = 0; i < p.n(); ++i)
    {
        const Grid& g = *p.grids[i];
        ProjectParams& q = p.h_params[i];
        q.dt = dts[i];
        const double scale = g.dx * g.dx / dts[i];
        if (relative_tolerance > 0.0)
        {
            q.tol_max = INFINITY;
            q.tol_sumsq = -(relative_tolerance * relative_tolerance);
        }
        else
        {
            q.tol_max = divergence_tolerance * scale;
            q.tol_sumsq = INFINITY;
        }
        q.max_iterations = max_iterations;
        q.use_mg = use_mg ? 1 : 0;
    }
    long long executed = p.rebuild_kernels;
    dispatch(p.precision, [&](auto zero)
    {
        using T = decltype(zero);
        executed += run_projection<T>(p, use_mg, max_iterations);
    });
    for (int i = 0; i < p.n(); ++i)
    {
        const SolveState& s = p.h_states[i];
        if (!s.done)
            fail(FC_ERR_TIMEOUT, "pressure loop stopped at its iteration cap before grid %d finished", i);
        fill_result(*p.grids[i], s, divergence_tolerance, &results[i]);
        results[i].kernels = int(executed);
    }
}

int project_one(Grid& g, double dt, int max_iterations, double divergence_tolerance, double relative_tolerance,
    fc_result* out)
{
    return guarded([&]
    {
        if (!out)
            fail(FC_ERR_INVALID_ARGUMENT, "null result");
        // FluidGridCPU::project returns a default result for these (FluidGridCPU.cpp:1032-1035).
        if (!(dt > 0.0) || max_iterations < 0)
        {
            *out = fc_result{};
            out->max_divergence = INFINITY;
            out->physical_steps = 1;
            return;
        }
        project_plan(single_plan(g), &dt, max_iterations, divergence_tolerance, relative_tolerance, out);
    });
}

template <typename T> void upload_velocity(Grid& g, const double* host, void* device, size_t count)
{
    if (!host)
    {
        check(cudaMemsetAsync(device, 0, count * sizeof(T), g.stream), "upload clear");
        return;
    }
    check(cudaMemcpyAsync(g.staging, host, count * sizeof(double), cudaMemcpyHostToDevice, g.stream), "upload");
    FC_LAUNCH(k_from_f64<T>, std::min<int>(ceil_div(int(std::min<size_t>(count, 1 << 30)), 256), 4096), 256, 0, g.stream,
        g.staging, static_cast<T*>(device), (long long)count);
}

template <typename T> void download_velocity(Grid& g, double* host, const void* device, size_t count)
{
    if (!host)
        return;
    FC_LAUNCH(k_to_f64<T>, std::min<int>(ceil_div(int(std::min<size_t>(count, 1 << 30)), 256), 4096), 256, 0, g.stream,
        static_cast<const T*>(device), g.staging, (long long)count);
    // Stream order keeps the staging buffer's next writer behind this copy; the caller waits
    // for the host buffers.
    check(cudaMemcpyAsync(host, g.staging, count * sizeof(double), cudaMemcpyDeviceToHost, g.stream), "download");
}

int blocks_for(size_t n) { return int(std::min<size_t>((n + 255) / 256, 4096)); }

void upload(Grid& g, const double* fraction, const double* u, const double* v, const double* pressure,
    const double* const* liquid_mass, const double* const* gas_mass)
{
    if (!g.configured)
        fail(FC_ERR_LIFECYCLE, "configure materials before uploading");
    allocate_masses(g);
    refresh_descriptor(g);
    const size_t n = g.cells;
    if (fraction)
        check(cudaMemcpyAsync(g.fraction, fraction, n * sizeof(double), cudaMemcpyHostToDevice, g.stream), "fraction");
    else
        check(cudaMemsetAsync(g.fraction, 0, n * sizeof(double), g.stream), "fraction");
    const int nl = int(g.liquid_density.size()), ng = int(g.gas_density.size());
    for (int k = 0; k < nl + ng; ++k)
    {
        const double* src = k < nl ? (liquid_mass ? liquid_mass[k] : nullptr) : (gas_mass ? gas_mass[k - nl] : nullptr);
        double* dst = g.masses + size_t(k) * n;
        if (src)
            check(cudaMemcpyAsync(dst, src, n * sizeof(double), cudaMemcpyHostToDevice, g.stream), "masses");
        else
            check(cudaMemsetAsync(dst, 0, n * sizeof(double), g.stream), "masses");
    }
    dispatch(g.precision, [&](auto zero)
    {
        using T = decltype(zero);
        upload_velocity<T>(g, u, g.desc.u, g.faces_u);
        upload_velocity<T>(g, v, g.desc.v, g.faces_v);
    });
    const size_t padded = size_t(g.S) * (g.H + 2);
    check(cudaMemsetAsync(g.desc.p, 0, padded * sizeof(double), g.stream), "pressure");
    if (pressure)
    {
        check(cudaMemcpyAsync(g.staging, pressure, n * sizeof(double), cudaMemcpyHostToDevice, g.stream), "pressure");
        FC_LAUNCH(k_pad_f64, blocks_for(n), 256, 0, g.stream, g.staging, g.desc.p, g.W, g.H, g.S);
    }
    // The warm-start history restarts from the uploaded pressure (FluidGridCPU.cpp:251).
    check(cudaMemcpyAsync(g.desc.p_prev, g.desc.p, padded * sizeof(double), cudaMemcpyDeviceToDevice, g.stream), "history");
    check(cudaStreamSynchronize(g.stream), "upload");
    g.uploaded = true;
    g.coefficients_dirty = true;
}

void download(Grid& g, double* fraction, double* u, double* v, double* pressure, double* const* liquid_mass,
    double* const* gas_mass)
{
    require_uploaded(g);
    const size_t n = g.cells;
    if (fraction)
        check(cudaMemcpyAsync(fraction, g.fraction, n * sizeof(double), cudaMemcpyDeviceToHost, g.stream), "fraction");
    const int nl = int(g.liquid_density.size()), ng = int(g.gas_density.size());
    for (int k = 0; k < nl + ng; ++k)
    {
        double* dst = k < nl ? (liquid_mass ? liquid_mass[k] : nullptr) : (gas_mass ? gas_mass[k - nl] : nullptr);
        if (dst)
            check(cudaMemcpyAsync(dst, g.masses + size_t(k) * n, n * sizeof(double), cudaMemcpyDeviceToHost, g.stream), "masses");
    }
    dispatch(g.precision, [&](auto zero)
    {
        using T = decltype(zero);
        download_velocity<T>(g, u, g.desc.u, g.faces_u);
        download_velocity<T>(g, v, g.desc.v, g.faces_v);
    });
    if (pressure)
    {
        FC_LAUNCH(k_unpad_f64, blocks_for(n), 256, 0, g.stream, g.desc.p, g.staging, g.W, g.H, g.S);
        check(cudaMemcpyAsync(pressure, g.staging, n * sizeof(double), cudaMemcpyDeviceToHost, g.stream), "pressure");
    }
    check(cudaStreamSynchronize(g.stream), "download");
}

// Semi-Lagrangian transport of the velocities, the liquid fraction and every component mass
// through the velocity at the start of the step (fc_advect.cuh). Masses change, so the
// pressure coefficients are rebuilt at the next projection.
void advect_semi_lagrangian(Grid& g, double dt, bool wait)
{
    require_uploaded(g);
    Plan& p = single_plan(g);
    const double scale = dt / g.dx, half = 0.5 * scale;
    cudaStream_t s = p.stream;
    dispatch(g.precision, [&](auto zero)
    {
        using T = decltype(zero);
        const int fields = 1 + g.components();
        for (int k = 0; k < fields; ++k)
        {
            double* field = k == 0 ? g.fraction : g.masses + size_t(k - 1) * g.cells;
            FC_LAUNCH(k_advect_cells<T>, p.vec.count, kVecThreads, 0, s, p.d_desc, p.at(p.vec), scale, half, field,
                g.staging);
            check(cudaMemcpyAsync(field, g.staging, g.cells * sizeof(double), cudaMemcpyDeviceToDevice, s), "advect");
        }
        FC_LAUNCH(k_advect_velocity<T>, p.faces.count, kVecThreads, 0, s, p.d_desc, p.at(p.faces), scale, half,
            static_cast<T*>(g.u_next), static_cast<T*>(g.v_next));
        check(cudaMemcpyAsync(g.desc.u, g.u_next, g.faces_u * sizeof(T), cudaMemcpyDeviceToDevice, s), "advect");
        check(cudaMemcpyAsync(g.desc.v, g.v_next, g.faces_v * sizeof(T), cudaMemcpyDeviceToDevice, s), "advect");
    });
    if (wait)
        check(cudaStreamSynchronize(s), "advect");
    g.coefficients_dirty = true;
}

// FluidGridCPU::sampleVelocity at `count` world positions (host arrays of (x, y) pairs).
void sample_velocity(Grid& g, int count, const double* positions, double* velocities)
{
    require_uploaded(g);
    Plan& p = single_plan(g);
    const size_t bytes = size_t(count) * 2 * sizeof(double);
    double* d = nullptr;
    device_alloc(&d, 2 * bytes, p.stream, "sample allocation");
    try
    {
        check(cudaMemcpyAsync(d, positions, bytes, cudaMemcpyHostToDevice, p.stream), "sample upload");
        dispatch(g.precision, [&](auto zero)
        {
            using T = decltype(zero);
            FC_LAUNCH(k_sample_velocity<T>, (count + 255) / 256, 256, 0, p.stream, static_cast<const T*>(g.desc.u),
                static_cast<const T*>(g.desc.v), g.W, g.H, g.origin_x, g.origin_y, g.dx, count, d, d + 2 * count);
        });
        check(cudaMemcpyAsync(velocities, d + 2 * count, bytes, cudaMemcpyDeviceToHost, p.stream), "sample download");
        check(cudaStreamSynchronize(p.stream), "sample");
    }
    catch (...)
    {
        device_free(d, p.stream);
        throw;
    }
    device_free(d, p.stream);
}

// FluidGridCPU::capillaryStepLimit (FluidGridCPU.cpp:843-860): half the period of the
// shortest resolved capillary wave, from the lightest liquid and gas components.
double capillary_step_limit(const Grid& g)
{
    if (g.surface_tension == 0.0 || g.liquid_density.empty() || g.gas_density.empty())
        return INFINITY;
    const double liquid = *std::min_element(g.liquid_density.begin(), g.liquid_density.end());
    const double gas = *std::min_element(g.gas_density.begin(), g.gas_density.end());
    constexpr double pi = 3.14159265358979323846;
    return 0.5 * std::sqrt((liquid + gas) * g.dx * g.dx * g.dx / (2.0 * pi * g.surface_tension));
}

void ensure_tension(Grid& g)
{
    if (g.tension_arena)
        return;
    size_t sizes[6], total = 0;
    tension_layout(g.cells, sizes);
    for (size_t b : sizes)
        total += b;
    device_alloc(&g.tension_arena, total, g.stream, "surface tension allocation");
    char* at = g.tension_arena;
    void* ptrs[6];
    for (int i = 0; i < 6; ++i)
    {
        ptrs[i] = at;
        at += sizes[i];
    }
    g.tension = {static_cast<double2*>(ptrs[0]), static_cast<signed char*>(ptrs[1]), static_cast<double*>(ptrs[2]),
        static_cast<unsigned char*>(ptrs[3]), static_cast<double*>(ptrs[4]), static_cast<unsigned char*>(ptrs[5])};
}

// The three curvature sweeps of FluidSurfaceTensionCPU on the current liquid fraction.
void launch_curvature(Grid& g, cudaStream_t s)
{
    ensure_tension(g);
    const dim3 block(32, 8), grid_dim((g.W + 31) / 32, (g.H + 7) / 8);
    FC_LAUNCH(k_tension_heights, grid_dim, block, 0, s, g.fraction, g.W, g.H, g.tension);
    FC_LAUNCH(k_tension_curvature, grid_dim, block, 0, s, g.fraction, g.W, g.H, g.dx, g.tension);
    FC_LAUNCH(k_tension_complete, grid_dim, block, 0, s, g.fraction, g.W, g.H, g.dx, g.tension);
}

// FluidGridCPU::applySurfaceTension (FluidGridCPU.cpp:862-926): curvature, then the capillary
// force on every interior face with the pressure face weights of the current densities.
void apply_surface_tension(Grid& g, double dt, bool wait = true)
{
    require_uploaded(g);
    if (g.surface_tension == 0.0)
        return;
    Plan& p = single_plan(g);
    rebuild_if_dirty(p);
    launch_curvature(g, p.stream);
    const dim3 block(32, 8), grid_dim((g.W + 31) / 32, (g.H + 7) / 8);
    dispatch(g.precision, [&](auto zero)
    {
        using T = decltype(zero);
        FC_LAUNCH(k_tension_force<T>, grid_dim, block, 0, p.stream, p.d_desc, 0, g.fraction, g.tension, g.surface_tension,
            dt);
    });
    if (wait)
        check(cudaStreamSynchronize(p.stream), "surface tension");
}

// Completed curvature per cell and its validity, for inspection.
void surface_curvature(Grid& g, double* values, unsigned char* valid)
{
    require_uploaded(g);
    Plan& p = single_plan(g);
    launch_curvature(g, p.stream);
    if (values)
        check(cudaMemcpyAsync(values, g.tension.kappa, g.cells * sizeof(double), cudaMemcpyDeviceToHost, p.stream),
            "curvature download");
    if (valid)
        check(cudaMemcpyAsync(valid, g.tension.kappa_ok, g.cells, cudaMemcpyDeviceToHost, p.stream), "curvature download");
    check(cudaStreamSynchronize(p.stream), "curvature");
}

// ------------------------------------------------------------------------------------------
// Implicit viscosity (fc_viscosity.cuh)
// ------------------------------------------------------------------------------------------

bool has_viscosity(const Grid& g)
{
    for (double mu : g.liquid_viscosity)
        if (mu != 0.0)
            return true;
    for (double mu : g.gas_viscosity)
        if (mu != 0.0)
            return true;
    return false;
}

// Level sizes of the viscosity hierarchy (ViscositySolverGPU.cpp:74-86): halve, rounding up,
// until a level has at most 64 cells.
std::vector<std::pair<int, int>> viscosity_levels(int w, int h)
{
    std::vector<std::pair<int, int>> out;
    for (;;)
    {
        out.push_back({w, h});
        if ((long long)w * h <= 64 || out.size() == size_t(kMaxLevels))
            break;
        w = (w + 1) / 2;
        h = (h + 1) / 2;
    }
    return out;
}

struct ViscWork
{
    std::vector<ViscLevel> lev;
    void *solution, *rhs, *residual, *direction, *product, *truth;
    ViscState* state;
    double4* partial;
    unsigned int* counter;
    double2* comp;
};

// Lays out (and with allocate, allocates) the viscosity workspace of a grid.
size_t viscosity_layout(const Grid& g, ViscWork* work, char* base)
{
    const size_t e = g.elem;
    const auto sizes = viscosity_levels(g.W, g.H);
    size_t total = 0;
    auto take = [&](size_t bytes) -> void*
    {
        void* p = base ? base + total : nullptr;
        total += (bytes + 255) / 256 * 256;
        return p;
    };
    const size_t nodes0 = size_t(g.W + 1) * (g.H + 1);
    if (work)
        work->lev.assign(sizes.size(), ViscLevel{});
    for (size_t l = 0; l < sizes.size(); ++l)
    {
        const int w = sizes[l].first, h = sizes[l].second;
        const size_t nodes = size_t(w + 1) * (h + 1);
        ViscLevel v{};
        v.w = w;
        v.h = h;
        v.dx = std::ldexp(g.dx, int(l));
        v.material = take(size_t(w) * h * 2 * e);
        v.coeff = take(nodes * 4 * e);
        v.x = take(nodes * 2 * e);
        v.next = take(nodes * 2 * e);
        v.rhs = take(nodes * 2 * e);
        v.res = take(nodes * 2 * e);
        if (work)
            work->lev[l] = v;
    }
    void* vecs[6];
    for (void*& p : vecs)
        p = take(nodes0 * 2 * e);
    void* state = take(sizeof(ViscState));
    // visc_arrive_last: one partial per block and per group of kViscThreads blocks, a counter
    // per group and one for the groups.
    const int blocks = ceil_div(int(nodes0), kViscThreads);
    const int groups = ceil_div(blocks, kViscThreads);
    void* partial = take(size_t(blocks + groups) * sizeof(double4));
    void* counter = take(sizeof(unsigned int) * (1 + groups));
    void* comp = take(size_t(std::max(g.components(), 1)) * sizeof(double2));
    if (work)
    {
        work->solution = vecs[0];
        work->rhs = vecs[1];
        work->residual = vecs[2];
        work->direction = vecs[3];
        work->product = vecs[4];
        work->truth = vecs[5];
        work->state = static_cast<ViscState*>(state);
        work->partial = static_cast<double4*>(partial);
        work->counter = static_cast<unsigned int*>(counter);
        work->comp = static_cast<double2*>(comp);
    }
    return total;
}

ViscWork viscosity_workspace(Grid& g, cudaStream_t s)
{
    const size_t bytes = viscosity_layout(g, nullptr, nullptr);
    if (!g.visc_arena || g.visc_bytes < bytes)
    {
        device_free(g.visc_arena, s);
        g.visc_arena = nullptr;
        g.visc_bytes = 0;
        device_alloc(&g.visc_arena, bytes, s, "viscosity allocation");
        g.visc_bytes = bytes;
        check(cudaMemsetAsync(g.visc_arena, 0, bytes, s), "viscosity clear");
    }
    ViscWork w;
    viscosity_layout(g, &w, g.visc_arena);
    return w;
}

template <typename T> void viscosity_cycle(ViscWork& w, size_t l, void* b, double dt, const unsigned char* solid,
    cudaStream_t s)
{
    ViscLevel& L = w.lev[l];
    const unsigned char* mask = l == 0 ? solid : nullptr;
    const int blocks = ceil_div((L.w + 1) * (L.h + 1), kViscThreads);
    if (l + 1 == w.lev.size())
    {
        ViscLevel c = L;
        c.rhs = b;
        FC_LAUNCH_DEP(k_visc_coarse<T>, 1, kViscCoarseNodes, 0, s, c, dt, mask, w.state);
        return;
    }
    auto smooth = [&](int zero)
    {
        FC_LAUNCH_DEP(k_visc_smooth<T>, blocks, kViscThreads, 0, s, L, dt, mask, b, zero, w.state);
        std::swap(L.x, L.next);
    };
    smooth(1);
    smooth(0);
    FC_LAUNCH_DEP((k_visc_residual<T, kResidualPlain>), blocks, kViscThreads, 0, s, L, dt, mask, L.x, b, L.res, w.state,
        w.partial, w.counter, 0.0);
    ViscLevel& C = w.lev[l + 1];
    FC_LAUNCH_DEP(k_visc_restrict<T>, ceil_div((C.w + 1) * (C.h + 1), kViscThreads), kViscThreads, 0, s, L, C, w.state);
    viscosity_cycle<T>(w, l + 1, C.rhs, dt, solid, s);
    FC_LAUNCH_DEP(k_visc_prolong<T>, blocks, kViscThreads, 0, s, L, C, mask, w.state);
    std::swap(L.x, L.next);
    smooth(0);
    smooth(0);
}

struct ViscResult
{
    int iterations;
    double relative_residual;
};

// Backward-Euler viscosity solve of the grid's face velocities (ViscositySolverGPU.cpp:170-294):
// CG preconditioned by the V-cycle, the true residual checked every 4 iterations, the
// velocities written only on success. max_iterations < 0 means no cap.
template <typename T> ViscResult viscosity_solve(Grid& g, double dt, double tolerance, int max_iterations)
{
    Plan& p = single_plan(g);
    cudaStream_t s = p.stream;
    ViscWork w = viscosity_workspace(g, s);
    // Per-component (mu / rho, 1 / rho), liquid components first, as the masses are stored.
    std::vector<double2> comp;
    for (size_t k = 0; k < g.liquid_density.size(); ++k)
        comp.push_back(make_double2(g.liquid_viscosity[k] / g.liquid_density[k], 1.0 / g.liquid_density[k]));
    for (size_t k = 0; k < g.gas_density.size(); ++k)
        comp.push_back(make_double2(g.gas_viscosity[k] / g.gas_density[k], 1.0 / g.gas_density[k]));
    if (!comp.empty())
        check(cudaMemcpyAsync(w.comp, comp.data(), comp.size() * sizeof(double2), cudaMemcpyHostToDevice, s), "viscosity");
    const int cells = g.W * g.H;
    FC_LAUNCH(k_visc_material<T>, ceil_div(cells, kViscThreads), kViscThreads, 0, s, g.desc.masses, g.components(),
        w.comp, cells, 1.0 / (g.dx * g.dx), const_cast<void*>(w.lev[0].material));
    for (size_t l = 0; l < w.lev.size(); ++l)
    {
        const ViscLevel& L = w.lev[l];
        if (l > 0)
        {
            const ViscLevel& F = w.lev[l - 1];
            FC_LAUNCH(k_visc_coarsen<T>, ceil_div(L.w * L.h, kViscThreads), kViscThreads, 0, s, F.material, F.w, F.h,
                const_cast<void*>(L.material), L.w, L.h);
        }
        FC_LAUNCH(k_visc_coefficients<T>, ceil_div((L.w + 1) * (L.h + 1), kViscThreads), kViscThreads, 0, s,
            L.material, L.w, L.h, L.dx, const_cast<void*>(L.coeff));
    }
    const unsigned char* solid = g.has_solid ? g.solid : nullptr;
    const int nodes = (g.W + 1) * (g.H + 1);
    const int blocks = ceil_div(nodes, kViscThreads);
    const int reduce_blocks = ceil_div(nodes, kViscThreads * kViscReduceNodes);
    ViscLevel& L0 = w.lev[0];
    FC_LAUNCH(k_visc_pack<T>, blocks, kViscThreads, 0, s, g.W, g.H, g.desc.u, g.desc.v, L0.coeff, solid, w.solution, w.rhs);
    FC_LAUNCH((k_visc_residual<T, kResidualInitial>), reduce_blocks, kViscThreads, 0, s, L0, dt, solid, w.solution, w.rhs,
        w.residual, w.state, w.partial, w.counter, tolerance);
    ViscState h{};
    auto read_state = [&]
    {
        check(cudaMemcpyAsync(&h, w.state, sizeof(ViscState), cudaMemcpyDeviceToHost, s), "viscosity state");
        check(cudaStreamSynchronize(s), "viscosity");
    };
    read_state();
    if (h.breakdown)
        fail(FC_ERR_NONFINITE, "Viscosity received nonfinite velocity/material state");
    ViscResult result{0, std::sqrt(h.rnorm / std::max(h.energy, 1e-30))};
    if (h.rnorm <= h.target)
        return result;
    for (;;)
    {
        if (max_iterations >= 0 && result.iterations >= max_iterations)
            fail(FC_ERR_TIMEOUT, "Implicit viscosity did not converge; relative residual %g", result.relative_residual);
        const int batch = max_iterations < 0 ? 4 : std::min(4, max_iterations - result.iterations);
        for (int i = 0; i < batch; ++i)
        {
            viscosity_cycle<T>(w, 0, w.residual, dt, solid, s);
            FC_LAUNCH_DEP(k_visc_dot_rz<T>, reduce_blocks, kViscThreads, 0, s, nodes, L0.coeff, w.residual, L0.x, w.state,
                w.partial, w.counter);
            FC_LAUNCH_DEP(k_visc_direction<T>, blocks, kViscThreads, 0, s, nodes, L0.x, w.direction, w.state);
            FC_LAUNCH_DEP((k_visc_apply<T, true>), reduce_blocks, kViscThreads, 0, s, L0, dt, solid, w.direction, w.product,
                w.state, w.partial, w.counter);
            FC_LAUNCH_DEP(k_visc_update<T>, blocks, kViscThreads, 0, s, nodes, w.solution, w.residual, w.direction,
                w.product, w.state);
        }
        result.iterations += batch;
        FC_LAUNCH_DEP((k_visc_residual<T, kResidualTruth>), reduce_blocks, kViscThreads, 0, s, L0, dt, solid, w.solution, w.rhs,
            w.truth, w.state, w.partial, w.counter, tolerance);
        read_state();
        result.relative_residual = std::sqrt(h.truth / std::max(h.energy, 1e-30));
        if (h.breakdown)
            fail(FC_ERR_BREAKDOWN, "Implicit viscosity solver breakdown");
        if (h.truth <= h.target)
            break;
        if (h.stopped)
            FC_LAUNCH_DEP(k_visc_refresh<T>, blocks, kViscThreads, 0, s, nodes, w.truth, w.residual, w.state);
    }
    FC_LAUNCH(k_visc_unpack<T>, blocks, kViscThreads, 0, s, g.W, g.H, w.solution, g.desc.u, g.desc.v);
    check(cudaStreamSynchronize(s), "viscosity");
    return result;
}

// FluidGridGPU::applyViscosity (FluidGridGPU.cpp:987-1045): tolerance 1e-4 relative, no cap in
// the reference; max_iterations bounds it here when >= 0.
ViscResult apply_viscosity(Grid& g, double dt, double tolerance, int max_iterations)
{
    require_uploaded(g);
    if (!(dt > 0.0) || !has_viscosity(g))
        return {0, 0.0};
    ViscResult r{};
    dispatch(g.precision, [&](auto zero)
    {
        using T = decltype(zero);
        r = viscosity_solve<T>(g, dt, tolerance, max_iterations);
    });
    return r;
}

// ------------------------------------------------------------------------------------------
// Conservative PLIC transport (fc_plic.cuh)
// ------------------------------------------------------------------------------------------

size_t plic_layout(const Grid& g, plic::PlicArrays* a, char* base)
{
    const size_t cells = g.cells, k = size_t(g.components());
    size_t total = 0;
    auto take = [&](size_t bytes) -> char*
    {
        char* p = base ? base + total : nullptr;
        total += (bytes + 255) / 256 * 256;
        return p;
    };
    plic::PlicArrays t{};
    t.mom_u = reinterpret_cast<double*>(take(g.faces_u * 8));
    t.mom_v = reinterpret_cast<double*>(take(g.faces_v * 8));
    t.next_u = reinterpret_cast<double*>(take(g.faces_u * 8));
    t.next_v = reinterpret_cast<double*>(take(g.faces_v * 8));
    t.lt_u = reinterpret_cast<double*>(take(g.faces_u * 8));
    t.lt_v = reinterpret_cast<double*>(take(g.faces_v * 8));
    t.mt_u = reinterpret_cast<double*>(take(g.faces_u * 8));
    t.mt_v = reinterpret_cast<double*>(take(g.faces_v * 8));
    t.normal = reinterpret_cast<double2*>(take(cells * 16));
    t.offset = reinterpret_cast<double*>(take(cells * 8));
    t.split = reinterpret_cast<unsigned char*>(take(cells));
    t.corr = reinterpret_cast<double*>(take(std::max<size_t>(k, 1) * cells * 8));
    t.mcorr = reinterpret_cast<double*>(take(cells * 8));
    t.fnext = reinterpret_cast<double*>(take(cells * 8));
    t.mnext = reinterpret_cast<double*>(take(std::max<size_t>(k, 1) * cells * 8));
    t.outflow = reinterpret_cast<unsigned long long*>(take(8));
    if (a)
        *a = t;
    return total;
}

plic::PlicArrays plic_workspace(Grid& g, cudaStream_t s)
{
    const size_t bytes = plic_layout(g, nullptr, nullptr);
    if (!g.plic_arena || g.plic_bytes < bytes)
    {
        device_free(g.plic_arena, s);
        g.plic_arena = nullptr;
        g.plic_bytes = 0;
        device_alloc(&g.plic_arena, bytes, s, "transport allocation");
        g.plic_bytes = bytes;
        check(cudaMemsetAsync(g.plic_arena, 0, bytes, s), "transport clear");
    }
    plic::PlicArrays a{};
    plic_layout(g, &a, g.plic_arena);
    return a;
}

// FluidGridCPU::advect (FluidGridCPU.cpp:362-463): CFL substeps of an X pass and a Y pass.
template <typename T> void advect_plic_t(Grid& g, double dt)
{
    using namespace plic;
    Plan& p = single_plan(g);
    cudaStream_t s = p.stream;
    PlicArrays a = plic_workspace(g, s);
    const int W = g.W, H = g.H, cells = int(g.cells), K = g.components(), L = int(g.liquid_density.size());
    const double inverse_volume = 1.0 / (g.dx * g.dx);
    T* u = static_cast<T*>(g.desc.u);
    T* v = static_cast<T*>(g.desc.v);
    double* const* masses = g.desc.masses;
    const int cell_blocks = ceil_div(cells, 256), face_blocks = ceil_div((W + 1) * (H + 1), 256);

    FC_LAUNCH(k_plic_density, cell_blocks, 256, 0, s, cells, masses, K, inverse_volume, g.desc.density);
    FC_LAUNCH(k_plic_begin<T>, face_blocks, 256, 0, s, W, H, u, v, g.desc.density, a);
    check(cudaMemsetAsync(a.outflow, 0, 8, s), "transport");
    FC_LAUNCH(k_plic_outflow<T>, cell_blocks, 256, 0, s, W, H, u, v, a);
    unsigned long long bits = 0;
    check(cudaMemcpyAsync(&bits, a.outflow, 8, cudaMemcpyDeviceToHost, s), "transport");
    check(cudaStreamSynchronize(s), "transport");
    double max_outflow;
    std::memcpy(&max_outflow, &bits, 8);
    if (!std::isfinite(max_outflow))
        fail(FC_ERR_NONFINITE, "transport received a non-finite velocity");
    // Limit transport so no cell exports more than half its volume per substep.
    const double max_step = max_outflow > 0.0 ? 0.5 * g.dx / max_outflow : dt;
    if (dt / max_step > 1e6)
        fail(FC_ERR_UNSUPPORTED, "transport would need more than a million substeps");

    auto pass = [&](auto axis, double step)
    {
        constexpr int AXIS = decltype(axis)::value;
        const double scale = step / g.dx;
        const T* flow = AXIS == 0 ? u : v;
        double* lt = AXIS == 0 ? a.lt_u : a.lt_v;
        double* mt = AXIS == 0 ? a.mt_u : a.mt_v;
        FC_LAUNCH(k_plic_interfaces, cell_blocks, 256, 0, s, W, H, g.fraction, a);
        FC_LAUNCH((k_plic_transfer<T, AXIS>), face_blocks, 256, 0, s, W, H, flow, g.fraction, scale, a, lt);
        FC_LAUNCH((k_plic_mass_transfer<T, AXIS>), face_blocks, 256, 0, s, W, H, flow, g.fraction, lt, masses, L, K,
            scale, inverse_volume, mt);
        FC_LAUNCH((k_plic_components<T, AXIS>), cell_blocks, 256, 0, s, W, H, flow, g.fraction, lt, masses, L, K, scale, a);
        FC_LAUNCH((k_plic_momentum<T, AXIS>), face_blocks, 256, 0, s, W, H, u, v, mt, scale, a);
        FC_LAUNCH((k_plic_fraction<T, AXIS>), cell_blocks, 256, 0, s, W, H, flow, g.fraction, lt, scale, a);
        check(cudaMemcpyAsync(g.fraction, a.fnext, size_t(cells) * 8, cudaMemcpyDeviceToDevice, s), "transport");
        if (K > 0)
            check(cudaMemcpyAsync(g.masses, a.mnext, size_t(K) * cells * 8, cudaMemcpyDeviceToDevice, s), "transport");
        FC_LAUNCH(k_plic_density, cell_blocks, 256, 0, s, cells, masses, K, inverse_volume, g.desc.density);
        FC_LAUNCH(k_plic_recover, face_blocks, 256, 0, s, W, H, g.desc.density, a);
    };
    double remaining = dt;
    while (remaining > 0.0)
    {
        const double step = max_step < remaining ? max_step : remaining;
        // Frozen for both passes of the substep.
        FC_LAUNCH(k_plic_freeze, cell_blocks, 256, 0, s, W, H, g.fraction, masses, L, K, inverse_volume, a);
        pass(std::integral_constant<int, 0>{}, step);
        pass(std::integral_constant<int, 1>{}, step);
        remaining -= step;
    }
    FC_LAUNCH(k_plic_finish<T>, face_blocks, 256, 0, s, W, H, a, u, v);
    check(cudaStreamSynchronize(s), "transport");
}

void advect_plic(Grid& g, double dt)
{
    require_uploaded(g);
    dispatch(g.precision, [&](auto zero)
    {
        using T = decltype(zero);
        advect_plic_t<T>(g, dt);
    });
    g.coefficients_dirty = true;
}

// Transport of one step. With wait false the semi-Lagrangian kernels are only enqueued on the
// grid's stream (PLIC transport reads back its CFL substeps and always waits).
void advect(Grid& g, double dt, bool wait = true)
{
    if (g.transport == FC_TRANSPORT_PLIC)
        advect_plic(g, dt);
    else
        advect_semi_lagrangian(g, dt, wait);
}

// One preconditioner application to a given residual (PressureMultigrid::apply,
// PressureMultigrid.cpp:410-434, or the diagonal at FluidGridCPU.cpp:1691-1698); the
// correction is returned without its mean removed, as the reference's apply returns it.
void apply_preconditioner(Grid& g, const double* residual, double residual_mean, double* correction)
{
    require_uploaded(g);
    Plan& p = single_plan(g);
    rebuild_if_dirty(p);
    const bool use_mg = g.preconditioner == FC_PRECONDITIONER_MULTIGRID;
    SolveState s;
    check(cudaMemcpyAsync(&s, g.desc.state, sizeof(s), cudaMemcpyDeviceToHost, p.stream), "state");
    check(cudaStreamSynchronize(p.stream), "state");
    if (use_mg && !s.mg_valid)
        fail(FC_ERR_BREAKDOWN, "coarsest multigrid factorisation failed");
    const int mg_valid = s.mg_valid;
    s = SolveState{};
    s.mg_valid = mg_valid;
    s.use_mg = use_mg ? 1 : 0;
    s.mean_r = residual_mean;
    s.restart = 1;
    s.rz = 1.0;
    s.inv_cells = g.air_model == FC_AIR_DIRICHLET ? 0.0 : 1.0 / double(g.cells);
    check(cudaMemcpyAsync(g.desc.state, &s, sizeof(s), cudaMemcpyHostToDevice, p.stream), "state");
    check(cudaMemcpyAsync(g.staging, residual, g.cells * sizeof(double), cudaMemcpyHostToDevice, p.stream), "residual");
    dispatch(g.precision, [&](auto zero)
    {
        using T = decltype(zero);
        set_kernel_attributes<T>(p);
        FC_LAUNCH(k_pad_t<T>, blocks_for(g.cells), 256, 0, p.stream, g.staging, g.desc.r, g.W, g.H, g.S);
        launch_precondition<T>(p, use_mg);
        FC_LAUNCH(k_unpad_t<T>, blocks_for(g.cells), 256, 0, p.stream, g.desc.z, g.staging, g.W, g.H, g.S);
    });
    check(cudaMemcpyAsync(correction, g.staging, g.cells * sizeof(double), cudaMemcpyDeviceToHost, p.stream), "correction");
    check(cudaStreamSynchronize(p.stream), "preconditioner");
}

double time_kernel(Grid& g, int kernel, int repeats)
{
    require_uploaded(g);
    Plan& p = single_plan(g);
    if (kernel < 0 || kernel > 3 || repeats <= 0)
        fail(FC_ERR_INVALID_ARGUMENT, "unknown kernel or repeat count");
    if ((kernel == 0 || kernel == 1) && g.tail == 0)
        fail(FC_ERR_INVALID_ARGUMENT, "grid too small for the fine-level smoothing kernels");
    rebuild_if_dirty(p);
    SolveState saved;
    check(cudaMemcpyAsync(&saved, g.desc.state, sizeof(saved), cudaMemcpyDeviceToHost, p.stream), "state");
    check(cudaStreamSynchronize(p.stream), "state");
    SolveState running = saved;
    running.done = 0;
    running.restart = 1;
    check(cudaMemcpyAsync(g.desc.state, &running, sizeof(running), cudaMemcpyHostToDevice, p.stream), "state");
    // One event pair per launch: the state reset between launches stays outside the timing.
    std::vector<cudaEvent_t> marks(2 * size_t(repeats));
    for (cudaEvent_t& e : marks)
        check(cudaEventCreate(&e), "event");
    dispatch(g.precision, [&](auto zero)
    {
        using T = decltype(zero);
        set_kernel_attributes<T>(p);
        auto launch = [&]
        {
            switch (kernel)
            {
            case 0: launch_smooth<T>(p, 0, true, false, p.stream); break;
            case 1: launch_smooth<T>(p, 0, false, false, p.stream); break;
            case 2: FC_LAUNCH(k_direction_operator<T>, p.vec.count, kVecThreads, 0, p.stream, p.d_desc, p.at(p.vec), 0); break;
            default: FC_LAUNCH(k_mg_tail<T>, p.n(), kTailThreads, p.tail_smem, p.stream, p.d_desc); break;
            }
        };
        launch(); // warm
        for (int i = 0; i < repeats; ++i)
        {
            // The level-0 post kernel folds a reduction that may mark the solve done.
            check(cudaMemcpyAsync(&g.desc.state->done, &running.done, sizeof(int), cudaMemcpyHostToDevice, p.stream), "state");
            check(cudaEventRecord(marks[2 * i], p.stream), "event");
            launch();
            check(cudaEventRecord(marks[2 * i + 1], p.stream), "event");
        }
    });
    check(cudaEventSynchronize(marks.back()), "event");
    double ms = 0.0;
    for (int i = 0; i < repeats; ++i)
    {
        float one = 0.0f;
        check(cudaEventElapsedTime(&one, marks[2 * i], marks[2 * i + 1]), "event");
        ms += one;
    }
    for (cudaEvent_t e : marks)
        cudaEventDestroy(e);
    check(cudaMemcpyAsync(g.desc.state, &saved, sizeof(saved), cudaMemcpyHostToDevice, p.stream), "state");
    check(cudaStreamSynchronize(p.stream), "state");
    return double(ms) / repeats;
}

// ------------------------------------------------------------------------------------------
// Autotuning of the multigrid schedule
// ------------------------------------------------------------------------------------------
//
// The tail threshold (the largest level the one-CTA tail cycles in shared memory; the levels
// above it run the strip kernels) changes which kernels run, not the arithmetic: both apply
// the same red-black sweeps, transfers and coarsest solve. The tuner times V-cycles of a plan
// under each candidate and keeps the fastest.

// Applies a tail threshold to a grid. The grid's single-grid plan is rebuilt on next use; the
// caller rebuilds any batch plan holding it.
void set_tail_cells(Grid& g, int cells)
{
    g.tail_cells = cells;
    choose_tail(g);
    g.desc.tail = g.tail;
    g.plan.reset();
    g.coefficients_dirty = true; // mixed precision: FP16 copies of the newly smoothed levels
}

// Mean time of one V-cycle of a plan, in ms, over `repeats` after two warm-up cycles. The
// solve states are saved before and restored after, so timing leaves the grids as they were.
double time_vcycles(Plan& p, int repeats)
{
    rebuild_if_dirty(p);
    std::vector<SolveState> saved(p.n());
    for (int i = 0; i < p.n(); ++i)
        check(cudaMemcpyAsync(&saved[i], p.grids[i]->desc.state, sizeof(SolveState), cudaMemcpyDeviceToHost, p.stream),
            "state");
    check(cudaStreamSynchronize(p.stream), "state");
    cudaEvent_t start = nullptr, stop = nullptr;
    check(cudaEventCreate(&start), "event");
    check(cudaEventCreate(&stop), "event");
    float ms = 0.0f;
    try
    {
        auto cycle = [&]
        {
            for (int i = 0; i < p.n(); ++i)
            {
                SolveState running = saved[i];
                running.done = 0;
                check(cudaMemcpyAsync(p.grids[i]->desc.state, &running, sizeof(running), cudaMemcpyHostToDevice, p.stream),
                    "state");
            }
            dispatch(p.precision, [&](auto zero)
            {
                using T = decltype(zero);
                set_kernel_attributes<T>(p);
                launch_precondition<T>(p, true);
            });
        };
        cycle();
        cycle();
        check(cudaEventRecord(start, p.stream), "event");
        for (int r = 0; r < repeats; ++r)
            cycle();
        check(cudaEventRecord(stop, p.stream), "event");
        check(cudaEventSynchronize(stop), "event");
        check(cudaEventElapsedTime(&ms, start, stop), "event");
    }
    catch (...)
    {
        cudaEventDestroy(start);
        cudaEventDestroy(stop);
        throw;
    }
    cudaEventDestroy(start);
    cudaEventDestroy(stop);
    for (int i = 0; i < p.n(); ++i)
        check(cudaMemcpyAsync(p.grids[i]->desc.state, &saved[i], sizeof(SolveState), cudaMemcpyHostToDevice, p.stream),
            "state");
    check(cudaStreamSynchronize(p.stream), "state");
    return double(ms) / repeats;
}

constexpr int kTailCandidates[] = {256, 1024, 4096};

struct TuneResult
{
    int tail_cells;
    double ms;
};

// Tries every tail threshold on the grids of a plan; `remake` rebuilds the plan after a change.
template <typename Remake> TuneResult autotune_plan(std::vector<Grid*> grids, Remake&& remake, int repeats)
{
    TuneResult best{grids.front()->tail_cells, INFINITY};
    for (int cells : kTailCandidates)
    {
        for (Grid* g : grids)
            set_tail_cells(*g, cells);
        const double ms = time_vcycles(remake(), repeats);
        if (ms < best.ms)
            best = {cells, ms};
    }
    for (Grid* g : grids)
        set_tail_cells(*g, best.tail_cells);
    remake();
    return best;
}

// ------------------------------------------------------------------------------------------
// Checkpoints: the "cuda-uniform" native format
// ------------------------------------------------------------------------------------------
//
// Modelled on the reference's "webgpu-uniform" checkpoint (UniformWebGPU/FluidGridGPU.cpp:
// 567-892): JSON metadata (backend, version, scalar types, byte order, geometry, materials,
// solver settings) and a payload of the physical state and solver history in a fixed order:
// liquid fraction, u, v, pressure, previous pressure, component masses (liquid then gas), then
// the obstacle mask when there is one. Each field keeps its device precision, so a loaded grid
// continues bit for bit. Loading validates everything before it changes any state.

constexpr int kCheckpointVersion = 1;

struct PayloadLayout
{
    size_t fraction, u, v, pressure, previous, masses, solid, total;
};

PayloadLayout payload_layout(const Grid& g, int components, bool solid)
{
    PayloadLayout l{};
    size_t at = 0;
    l.fraction = at;
    at += g.cells * sizeof(double);
    l.u = at;
    at += g.faces_u * g.elem;
    l.v = at;
    at += g.faces_v * g.elem;
    l.pressure = at;
    at += g.cells * sizeof(double);
    l.previous = at;
    at += g.cells * sizeof(double);
    l.masses = at;
    at += size_t(components) * g.cells * sizeof(double);
    l.solid = at;
    if (solid)
        at += g.cells;
    l.total = at;
    return l;
}

std::string checkpoint_metadata(const Grid& g)
{
    using json::number;
    using json::quoted;
    auto mixture = [](const std::vector<double>& density, const std::vector<double>& viscosity)
    {
        std::string out = "[";
        for (size_t i = 0; i < density.size(); ++i)
        {
            if (i)
                out += ", ";
            out += "{\"density\": " + number(density[i]) + ", \"dynamic_viscosity\": " + number(viscosity[i]) + "}";
        }
        return out + "]";
    };
    const bool little = [] { const unsigned one = 1; return *reinterpret_cast<const unsigned char*>(&one) == 1; }();
    const PayloadLayout layout = payload_layout(g, g.components(), g.has_solid);
    std::string m = "{";
    m += "\"backend\": " + quoted("cuda-uniform");
    m += ", \"version\": " + std::to_string(kCheckpointVersion);
    m += ", \"scalar\": " + quoted(g.elem == 8 ? "float64" : "float32");
    m += ", \"state_scalar\": " + quoted("float64");
    m += ", \"byte_order\": " + quoted(little ? "little" : "big");
    m += ", \"precision\": " + std::to_string(g.precision);
    m += ", \"width\": " + std::to_string(g.W) + ", \"height\": " + std::to_string(g.H);
    m += ", \"cell_size\": " + number(g.dx);
    m += ", \"origin\": [" + number(g.origin_x) + ", " + number(g.origin_y) + "]";
    m += ", \"gravity_y\": " + number(g.gravity_y);
    m += ", \"surface_tension\": " + number(g.surface_tension);
    m += ", \"transport\": " + std::to_string(g.transport);
    m += ", \"air_model\": " + std::to_string(g.air_model);
    m += ", \"preconditioner\": " + std::to_string(g.preconditioner);
    m += ", \"liquid_mixture\": " + mixture(g.liquid_density, g.liquid_viscosity);
    m += ", \"gas_mixture\": " + mixture(g.gas_density, g.gas_viscosity);
    m += ", \"obstacles\": " + std::string(g.has_solid ? "true" : "false");
    m += ", \"payload_bytes\": " + std::to_string(layout.total);
    m += ", \"fields\": [\"liquid_fraction\", \"u\", \"v\", \"pressure\", \"previous_pressure\", \"component_masses\"" +
         std::string(g.has_solid ? ", \"solid\"" : "") + "]";
    return m + "}";
}

void save_checkpoint(Grid& g, char* metadata, size_t metadata_capacity, size_t* metadata_bytes, void* payload,
    size_t payload_capacity, size_t* payload_bytes)
{
    require_uploaded(g);
    const std::string text = checkpoint_metadata(g);
    const PayloadLayout layout = payload_layout(g, g.components(), g.has_solid);
    if (metadata_bytes)
        *metadata_bytes = text.size() + 1;
    if (payload_bytes)
        *payload_bytes = layout.total;
    if (!metadata && !payload)
        return; // size query
    if (!metadata || metadata_capacity < text.size() + 1 || !payload || payload_capacity < layout.total)
        fail(FC_ERR_INVALID_ARGUMENT, "checkpoint buffers too small (%zu and %zu bytes needed)", text.size() + 1,
            layout.total);
    std::memcpy(metadata, text.c_str(), text.size() + 1);
    char* out = static_cast<char*>(payload);
    cudaStream_t s = g.stream;
    check(cudaStreamSynchronize(s), "checkpoint");
    check(cudaMemcpyAsync(out + layout.fraction, g.fraction, g.cells * sizeof(double), cudaMemcpyDeviceToHost, s), "checkpoint");
    check(cudaMemcpyAsync(out + layout.u, g.desc.u, g.faces_u * g.elem, cudaMemcpyDeviceToHost, s), "checkpoint");
    check(cudaMemcpyAsync(out + layout.v, g.desc.v, g.faces_v * g.elem, cudaMemcpyDeviceToHost, s), "checkpoint");
    if (g.components() > 0)
        check(cudaMemcpyAsync(out + layout.masses, g.masses, size_t(g.components()) * g.cells * sizeof(double),
                  cudaMemcpyDeviceToHost, s), "checkpoint");
    if (g.has_solid)
        check(cudaMemcpyAsync(out + layout.solid, g.solid, g.cells, cudaMemcpyDeviceToHost, s), "checkpoint");
    const double* fields[2] = {g.desc.p, g.desc.p_prev};
    const size_t offsets[2] = {layout.pressure, layout.previous};
    for (int k = 0; k < 2; ++k)
    {
        FC_LAUNCH(k_unpad_f64, blocks_for(g.cells), 256, 0, s, fields[k], g.staging, g.W, g.H, g.S);
        check(cudaMemcpyAsync(out + offsets[k], g.staging, g.cells * sizeof(double), cudaMemcpyDeviceToHost, s), "checkpoint");
        check(cudaStreamSynchronize(s), "checkpoint");
    }
}

void load_checkpoint(Grid& g, const char* metadata, const void* payload, size_t payload_bytes)
{
    if (!metadata || !payload)
        fail(FC_ERR_INVALID_ARGUMENT, "null checkpoint");
    json::Value m;
    try
    {
        m = json::Parser(metadata).parse();
    }
    catch (const std::exception& e)
    {
        fail(FC_ERR_INVALID_ARGUMENT, "checkpoint metadata is not valid JSON: %s", e.what());
    }
    auto need = [&](const char* key, json::Value::Kind kind) -> const json::Value&
    {
        const json::Value* v = m.kind == json::Value::Object ? m.find(key) : nullptr;
        if (!v || v->kind != kind)
            fail(FC_ERR_INVALID_ARGUMENT, "checkpoint metadata lacks a valid \"%s\"", key);
        return *v;
    };
    // A number the loader casts to an integer: finite, integral and within [lo, hi] first, so
    // no out-of-range value reaches a cast.
    auto integer = [&](const char* key, double lo, double hi) -> long long
    {
        const double x = need(key, json::Value::Number).number;
        if (!std::isfinite(x) || x != std::floor(x) || x < lo || x > hi)
            fail(FC_ERR_INVALID_ARGUMENT, "checkpoint \"%s\" is not an integer in range", key);
        return (long long)x;
    };
    auto finite = [&](const json::Value& v, const char* what) -> double
    {
        if (v.kind != json::Value::Number || !std::isfinite(v.number))
            fail(FC_ERR_INVALID_ARGUMENT, "checkpoint %s is not a finite number", what);
        return v.number;
    };
    if (need("backend", json::Value::String).text != "cuda-uniform")
        fail(FC_ERR_INVALID_ARGUMENT, "checkpoint was written by another backend");
    if (integer("version", 0, 1e6) != kCheckpointVersion)
        fail(FC_ERR_INVALID_ARGUMENT, "unsupported checkpoint version");
    const bool little = [] { const unsigned one = 1; return *reinterpret_cast<const unsigned char*>(&one) == 1; }();
    if (need("byte_order", json::Value::String).text != (little ? "little" : "big"))
        fail(FC_ERR_INVALID_ARGUMENT, "checkpoint byte order differs from this host");
    if (need("scalar", json::Value::String).text != (g.elem == 8 ? "float64" : "float32") ||
        integer("precision", 0, 16) != g.precision)
        fail(FC_ERR_INVALID_ARGUMENT, "checkpoint precision differs from the grid's");
    if (integer("width", 1, 1 << 30) != g.W || integer("height", 1, 1 << 30) != g.H ||
        need("cell_size", json::Value::Number).number != g.dx)
        fail(FC_ERR_INVALID_ARGUMENT, "checkpoint geometry differs from the grid's");
    const json::Value& origin = need("origin", json::Value::Array);
    if (origin.items.size() != 2)
        fail(FC_ERR_INVALID_ARGUMENT, "checkpoint origin is malformed");
    const double origin_x = finite(origin.items[0], "origin"), origin_y = finite(origin.items[1], "origin");
    auto mixture = [&](const char* key, std::vector<double>& density, std::vector<double>& viscosity)
    {
        density.clear();
        viscosity.clear();
        for (const json::Value& c : need(key, json::Value::Array).items)
        {
            const json::Value* d = c.find("density");
            const json::Value* mu = c.find("dynamic_viscosity");
            if (!d || d->kind != json::Value::Number || !(d->number > 0.0) || !std::isfinite(d->number))
                fail(FC_ERR_INVALID_ARGUMENT, "checkpoint mixture component is malformed");
            density.push_back(d->number);
            viscosity.push_back(mu && mu->kind == json::Value::Number ? mu->number : 0.0);
        }
    };
    std::vector<double> ld, lv, gd, gv;
    mixture("liquid_mixture", ld, lv);
    mixture("gas_mixture", gd, gv);
    for (double mu : lv)
        if (!std::isfinite(mu) || mu < 0.0)
            fail(FC_ERR_INVALID_ARGUMENT, "Invalid saved material viscosity");
    for (double mu : gv)
        if (!std::isfinite(mu) || mu < 0.0)
            fail(FC_ERR_INVALID_ARGUMENT, "Invalid saved material viscosity");
    const long long preconditioner = integer("preconditioner", -1e6, 1e6);
    if (preconditioner != FC_PRECONDITIONER_DIAGONAL && preconditioner != FC_PRECONDITIONER_MULTIGRID)
        fail(FC_ERR_INVALID_ARGUMENT, "checkpoint preconditioner is unknown");
    const bool solid = need("obstacles", json::Value::Bool).boolean;
    const double gravity = finite(need("gravity_y", json::Value::Number), "gravity_y");
    // Older checkpoints carry no surface tension: zero, the engine default.
    double tension = 0.0;
    if (const json::Value* st = m.find("surface_tension"))
    {
        if (st->kind != json::Value::Number || !std::isfinite(st->number) || st->number < 0.0)
            fail(FC_ERR_INVALID_ARGUMENT, "checkpoint surface tension is malformed");
        tension = st->number;
    }
    // Older checkpoints carry no transport scheme: semi-Lagrangian, the engine default.
    int transport = FC_TRANSPORT_SEMI_LAGRANGIAN;
    if (const json::Value* tr = m.find("transport"))
    {
        if (tr->kind != json::Value::Number || (tr->number != FC_TRANSPORT_SEMI_LAGRANGIAN && tr->number != FC_TRANSPORT_PLIC))
            fail(FC_ERR_INVALID_ARGUMENT, "checkpoint transport scheme is unknown");
        transport = int(tr->number);
    }
    // Older checkpoints carry no air model: the gas model, the engine default.
    int air_model = FC_AIR_GAS;
    if (const json::Value* am = m.find("air_model"))
    {
        if (am->kind != json::Value::Number || (am->number != FC_AIR_GAS && am->number != FC_AIR_DIRICHLET))
            fail(FC_ERR_INVALID_ARGUMENT, "checkpoint air model is unknown");
        air_model = int(am->number);
    }
    const PayloadLayout layout = payload_layout(g, int(ld.size() + gd.size()), solid);
    if (integer("payload_bytes", 0, 9.0e15) != (long long)layout.total || payload_bytes != layout.total)
        fail(FC_ERR_INVALID_ARGUMENT, "checkpoint payload has %zu bytes, %zu expected", payload_bytes, layout.total);

    // Validated: apply.
    g.liquid_density = ld;
    g.liquid_viscosity = lv;
    g.gas_density = gd;
    g.gas_viscosity = gv;
    g.configured = true;
    g.preconditioner = int(preconditioner);
    g.gravity_y = gravity;
    g.surface_tension = tension;
    g.transport = transport;
    g.air_model = air_model;
    g.origin_x = origin_x;
    g.origin_y = origin_y;
    allocate_masses(g);
    g.has_solid = solid;
    const char* in = static_cast<const char*>(payload);
    cudaStream_t s = g.stream;
    check(cudaStreamSynchronize(s), "checkpoint");
    check(cudaMemcpyAsync(g.fraction, in + layout.fraction, g.cells * sizeof(double), cudaMemcpyHostToDevice, s), "checkpoint");
    check(cudaMemcpyAsync(g.desc.u, in + layout.u, g.faces_u * g.elem, cudaMemcpyHostToDevice, s), "checkpoint");
    check(cudaMemcpyAsync(g.desc.v, in + layout.v, g.faces_v * g.elem, cudaMemcpyHostToDevice, s), "checkpoint");
    if (g.components() > 0)
        check(cudaMemcpyAsync(g.masses, in + layout.masses, size_t(g.components()) * g.cells * sizeof(double),
                  cudaMemcpyHostToDevice, s), "checkpoint");
    if (solid)
        check(cudaMemcpyAsync(g.solid, in + layout.solid, g.cells, cudaMemcpyHostToDevice, s), "checkpoint");
    double* fields[2] = {g.desc.p, g.desc.p_prev};
    const size_t offsets[2] = {layout.pressure, layout.previous};
    for (int k = 0; k < 2; ++k)
    {
        check(cudaMemcpyAsync(g.staging, in + offsets[k], g.cells * sizeof(double), cudaMemcpyHostToDevice, s), "checkpoint");
        FC_LAUNCH(k_pad_f64, blocks_for(g.cells), 256, 0, s, g.staging, fields[k], g.W, g.H, g.S);
        check(cudaStreamSynchronize(s), "checkpoint");
    }
    refresh_descriptor(g);
    g.uploaded = true;
    g.coefficients_dirty = true;
}

// ------------------------------------------------------------------------------------------
// Divergence statistics for callers that cannot allocate device memory
// ------------------------------------------------------------------------------------------
//
// Some callers cannot call cudaMalloc: a host whose allocator owns every byte of device memory
// (a game engine or a simulation framework with its own pool), a process held to a fixed
// device-memory budget, or a real-time loop that must never stall in the driver (cudaMalloc can
// synchronise the device). fc_divergence_noalloc serves them: the caller passes the face
// velocities and a device buffer for the result, and the reduction's scratch lives in the
// fixed array below instead of a per-grid allocation. Every GPU that loads this library holds
// the array until the process exits.

constexpr int kNoAllocTile = 32;       // tiles of 32 x 32 cells
constexpr int kNoAllocMaxTiles = 4096; // at most 4,194,304 cells
constexpr size_t kNoAllocCounterOffset = size_t(kNoAllocMaxTiles) * sizeof(double4);
static __device__ __align__(256) unsigned char noalloc_scratch[kNoAllocCounterOffset + 256];

// Same statistics as k_divergence, over a caller's unpadded face arrays; tile t covers the
// 32 x 32 cells at (t % tiles_x, t / tiles_x). The last tile to arrive folds the partials in
// tile order and resets the arrival counter.
template <typename T>
__global__ void __launch_bounds__(kVecThreads) k_divergence_noalloc(const T* u, const T* v, int W, int H, double dx,
    unsigned char* scratch, double* out)
{
    double4* partial = reinterpret_cast<double4*>(scratch);
    unsigned int* counter = reinterpret_cast<unsigned int*>(scratch + kNoAllocCounterOffset);
    const int tiles_x = (W + kNoAllocTile - 1) / kNoAllocTile;
    const int x0 = (blockIdx.x % tiles_x) * kNoAllocTile, y0 = (blockIdx.x / tiles_x) * kNoAllocTile;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    double mx = 0.0, excess = 0.0, sq = 0.0;
    int nonfinite = 0;
    for (int k = 0; k < 4; ++k)
    {
        const int x = x0 + tx, y = y0 + ty + 8 * k;
        if (x >= W || y >= H)
            continue;
        const long long iu = (long long)y * (W + 1) + x;
        const long long iv = (long long)y * W + x;
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
    const double4 mine = block_reduce4<kVecThreads>(make_double4(mx, excess, sq, double(nonfinite)), 1 | 2 | 8);
    __shared__ int is_last;
    if (threadIdx.x == 0)
    {
        partial[blockIdx.x] = mine;
        __threadfence();
        is_last = atomicAdd(counter, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!is_last)
        return;
    __threadfence();
    double4 acc = make_double4(0, 0, 0, 0);
    const int per = (int(gridDim.x) + kVecThreads - 1) / kVecThreads;
    const int first = threadIdx.x * per, last = min(int(gridDim.x), first + per);
    for (int t = first; t < last; ++t)
    {
        const volatile double* slot = reinterpret_cast<const volatile double*>(&partial[t]);
        acc.x = fmax(acc.x, slot[0]);
        acc.y = fmax(acc.y, slot[1]);
        acc.z += slot[2];
        acc.w = fmax(acc.w, slot[3]);
    }
    const double4 total = block_reduce4<kVecThreads>(acc, 1 | 2 | 8);
    if (threadIdx.x == 0)
    {
        out[0] = total.w != 0.0 ? INFINITY : total.x;
        out[1] = total.w != 0.0 ? INFINITY : total.y;
        out[2] = total.z;
        *counter = 0u;
    }
}

// Device address of the scratch array on the current device. Outside stream capture it is
// looked up on every call, so a device or primary-context reset by the host (which unloads the
// module and with it the array) never leaves a stale address behind. During capture the last
// address looked up on that device is used, as a capture must not load modules; the header
// asks for one call before any capture.
void* noalloc_address(cudaStream_t stream)
{
    static std::mutex lock;
    static void* addresses[64] = {};
    int device = 0;
    check(cudaGetDevice(&device), "current device");
    if (device < 0 || device >= 64)
        fail(FC_ERR_UNSUPPORTED, "device index %d out of range", device);
    int stream_device = device;
    check(cudaStreamGetDevice(stream, &stream_device), "stream device");
    if (stream_device != device)
        fail(FC_ERR_INVALID_ARGUMENT, "the stream belongs to device %d, but device %d is current; make the stream's "
            "device current before the call", stream_device, device);
    cudaStreamCaptureStatus capture = cudaStreamCaptureStatusNone;
    check(cudaStreamIsCapturing(stream, &capture), "stream capture status");
    std::lock_guard<std::mutex> guard(lock);
    if (capture == cudaStreamCaptureStatusNone || !addresses[device])
    {
        void* address = nullptr;
        check(cudaGetSymbolAddress(&address, noalloc_scratch), "scratch symbol address");
        addresses[device] = address;
    }
    return addresses[device];
}

// Gravity on the vertical faces (FluidGridCPU.cpp:835-841 order: after transport).
void apply_gravity(Grid& g, double dt, bool wait)
{
    require_uploaded(g);
    Plan& p = single_plan(g);
    dispatch(g.precision, [&](auto zero)
    {
        using T = decltype(zero);
        FC_LAUNCH(k_gravity<T>, p.vec.count, kVecThreads, 0, p.stream, p.d_desc, p.at(p.vec), g.gravity_y * dt);
    });
    if (wait)
        check(cudaStreamSynchronize(p.stream), "gravity");
}

// Dirichlet air: the liquid's face velocities extended into the air (k_air_faces_extend).
void extend_air_velocity(Grid& g, bool wait)
{
    require_uploaded(g);
    Plan& p = single_plan(g);
    unsigned char* known_u = g.air_faces;
    unsigned char* known_v = g.air_faces + g.faces_u;
    FC_LAUNCH(k_air_faces_init, p.faces.count, kVecThreads, 0, p.stream, p.d_desc, p.at(p.faces), known_u, known_v);
    dispatch(g.precision, [&](auto zero)
    {
        using T = decltype(zero);
        for (int layer = 1; layer <= kAirLayers; ++layer)
            FC_LAUNCH(k_air_faces_extend<T>, p.faces.count, kVecThreads, 0, p.stream, p.d_desc, p.at(p.faces), known_u,
                known_v, layer);
    });
    if (wait)
        check(cudaStreamSynchronize(p.stream), "air velocity extension");
}

// The reference's step runs the viscosity solve without an iteration cap; this bound only turns
// a solve that cannot converge into an error instead of an endless loop.
constexpr int kViscosityCap = 20000;

// fc_step's physical substep before its projection (FluidGridCPU.cpp:300-360 order): the air
// extension under Dirichlet air, transport, implicit viscosity when a component is viscous
// (FluidGridGPU.cpp:1139-1146, 1e-4 relative), gravity and surface tension. With wait false the
// kernels are only enqueued on the grid's stream; the viscosity solve and PLIC transport read
// values back and wait regardless. Returns the viscosity iterations.
int advance_substep(Grid& g, double dt, bool wait)
{
    if (g.air_model == FC_AIR_DIRICHLET)
        extend_air_velocity(g, wait);
    advect(g, dt, wait);
    int viscous = 0;
    if (has_viscosity(g))
    {
        const ViscResult r = apply_viscosity(g, dt, 1e-4, kViscosityCap);
        viscous = r.iterations;
    }
    apply_gravity(g, dt, wait);
    if (g.surface_tension > 0.0)
        apply_surface_tension(g, dt, wait);
    return viscous;
}

} // namespace fc

// ==========================================================================================
// C ABI
// ==========================================================================================

using fc::Grid;
using fc::guarded;
using fc::fail;
using fc::check;

struct fc_grid
{
    Grid impl;
};

struct fc_batch
{
    std::vector<fc_grid*> grids;
    std::unique_ptr<fc::Plan> plan;
};

extern "C" {

int fc_abi_version(void) { return FC_ABI_VERSION; }

const char* fc_last_error(void) { return fc::last_error.c_str(); }

const char* fc_status_string(int status)
{
    switch (status)
    {
    case FC_OK: return "ok";
    case FC_ERR_INVALID_ARGUMENT: return "invalid argument";
    case FC_ERR_LIFECYCLE: return "lifecycle";
    case FC_ERR_CUDA: return "cuda";
    case FC_ERR_OUT_OF_MEMORY: return "out of memory";
    case FC_ERR_NONFINITE: return "non-finite";
    case FC_ERR_BREAKDOWN: return "breakdown";
    case FC_ERR_UNSUPPORTED: return "unsupported";
    case FC_ERR_TIMEOUT: return "timeout";
    default: return "unknown";
    }
}

long long fc_kernel_launches(void) { return fc::launch_count.load(); }

int fc_set_launch_mode(int mode)
{
    return guarded([&]
    {
        if (mode != FC_LAUNCH_GRAPH && mode != FC_LAUNCH_STREAM)
            fail(FC_ERR_INVALID_ARGUMENT, "unknown launch mode %d", mode);
        fc::launch_mode.store(mode);
    });
}

int fc_create(int width, int height, double cell_size, int precision, fc_grid** out)
{
    return guarded([&]
    {
        if (!out)
            fail(FC_ERR_INVALID_ARGUMENT, "null output handle");
        *out = nullptr;
        if (width <= 0 || height <= 0 || !(cell_size > 0.0) || !std::isfinite(cell_size))
            fail(FC_ERR_INVALID_ARGUMENT, "grid geometry must be positive and finite");
        if ((long long)width * height > (1ll << 30))
            fail(FC_ERR_INVALID_ARGUMENT, "grid too large");
        if (precision != FC_PRECISION_FP32 && precision != FC_PRECISION_FP64 && precision != FC_PRECISION_MIXED)
            fail(FC_ERR_INVALID_ARGUMENT, "unknown precision %d", precision);
        auto handle = std::make_unique<fc_grid>();
        Grid& g = handle->impl;
        g.W = width;
        g.H = height;
        g.dx = cell_size;
        g.precision = precision;
        g.elem = precision == FC_PRECISION_FP64 ? 8 : 4;
        check(cudaGetDevice(&g.device), "device");
        check(cudaStreamCreateWithFlags(&g.stream, cudaStreamNonBlocking), "stream");
        fc::allocate_grid(g);
        *out = handle.release();
    });
}

int fc_grid_device_bytes(int width, int height, int precision, int components, int surface_tension, size_t* bytes)
{
    return guarded([&]
    {
        if (!bytes || width <= 0 || height <= 0 || components < 0 || (long long)width * height > (1ll << 30))
            fail(FC_ERR_INVALID_ARGUMENT, "invalid grid description");
        if (precision != FC_PRECISION_FP32 && precision != FC_PRECISION_FP64 && precision != FC_PRECISION_MIXED)
            fail(FC_ERR_INVALID_ARGUMENT, "unknown precision %d", precision);
        fc::Grid g;
        g.W = width;
        g.H = height;
        g.precision = precision;
        g.elem = precision == FC_PRECISION_FP64 ? 8 : 4;
        size_t total = fc::allocate_grid(g, false);
        total += size_t(components) * g.cells * sizeof(double) + 256 + size_t(std::max(components, 1)) * sizeof(double*);
        if (surface_tension)
            total += fc::tension_bytes(g.cells);
        total += fc::plan_bytes(width, height);
        *bytes = total;
    });
}

int fc_get_device_bytes(const fc_grid* grid, size_t* bytes)
{
    return guarded([&]
    {
        if (!grid || !bytes)
            fail(FC_ERR_INVALID_ARGUMENT, "null argument");
        const Grid& g = grid->impl;
        size_t total = g.arena_bytes + size_t(g.mass_capacity) * g.cells * sizeof(double);
        if (g.tension_arena)
            total += fc::tension_bytes(g.cells);
        total += g.visc_bytes;
        total += fc::plan_bytes(g.W, g.H);
        *bytes = total;
    });
}

int fc_destroy(fc_grid* grid)
{
    return guarded([&]
    {
        if (grid)
        {
            cudaStreamSynchronize(grid->impl.stream);
            delete grid;
        }
    });
}

int fc_get_geometry(const fc_grid* grid, int* width, int* height, double* cell_size)
{
    return guarded([&]
    {
        if (!grid)
            fail(FC_ERR_INVALID_ARGUMENT, "null grid");
        if (width)
            *width = grid->impl.W;
        if (height)
            *height = grid->impl.H;
        if (cell_size)
            *cell_size = grid->impl.dx;
    });
}

int fc_get_origin(const fc_grid* grid, double* x, double* y)
{
    return guarded([&]
    {
        if (!grid || !x || !y)
            fail(FC_ERR_INVALID_ARGUMENT, "null argument");
        *x = grid->impl.origin_x;
        *y = grid->impl.origin_y;
    });
}

int fc_set_origin(fc_grid* grid, double x, double y)
{
    return guarded([&]
    {
        if (!grid)
            fail(FC_ERR_INVALID_ARGUMENT, "null grid");
        grid->impl.origin_x = x;
        grid->impl.origin_y = y;
    });
}

int fc_get_precision(const fc_grid* grid, int* precision)
{
    return guarded([&]
    {
        if (!grid || !precision)
            fail(FC_ERR_INVALID_ARGUMENT, "null argument");
        *precision = grid->impl.precision;
    });
}

int fc_configure_materials(fc_grid* grid, int liquid_count, const double* liquid_densities,
    const double* liquid_viscosities, int gas_count, const double* gas_densities, const double* gas_viscosities)
{
    return guarded([&]
    {
        if (!grid || liquid_count < 0 || gas_count < 0 || (liquid_count && !liquid_densities) || (gas_count && !gas_densities))
            fail(FC_ERR_INVALID_ARGUMENT, "invalid material description");
        Grid& g = grid->impl;
        auto take = [](std::vector<double>& out, int n, const double* values)
        {
            out.assign(n, 0.0);
            for (int i = 0; i < n && values; ++i)
                out[i] = values[i];
        };
        for (int i = 0; i < liquid_count; ++i)
            if (!(liquid_densities[i] > 0.0) || !std::isfinite(liquid_densities[i]))
                fail(FC_ERR_INVALID_ARGUMENT, "component densities must be positive and finite");
        for (int i = 0; i < gas_count; ++i)
            if (!(gas_densities[i] > 0.0) || !std::isfinite(gas_densities[i]))
                fail(FC_ERR_INVALID_ARGUMENT, "component densities must be positive and finite");
        // FluidGridGPU.cpp:381-382.
        for (int i = 0; i < liquid_count && liquid_viscosities; ++i)
            if (!std::isfinite(liquid_viscosities[i]) || liquid_viscosities[i] < 0.0)
                fail(FC_ERR_INVALID_ARGUMENT, "Material viscosity must be finite and nonnegative");
        for (int i = 0; i < gas_count && gas_viscosities; ++i)
            if (!std::isfinite(gas_viscosities[i]) || gas_viscosities[i] < 0.0)
                fail(FC_ERR_INVALID_ARGUMENT, "Material viscosity must be finite and nonnegative");
        take(g.liquid_density, liquid_count, liquid_densities);
        take(g.gas_density, gas_count, gas_densities);
        take(g.liquid_viscosity, liquid_count, liquid_viscosities);
        take(g.gas_viscosity, gas_count, gas_viscosities);
        g.configured = true;
        // Changing mixtures requires another upload (FluidGridBase.h:41).
        g.uploaded = false;
    });
}

int fc_get_gravity(const fc_grid* grid, double* gravity_y)
{
    return guarded([&]
    {
        if (!grid || !gravity_y)
            fail(FC_ERR_INVALID_ARGUMENT, "null argument");
        *gravity_y = grid->impl.gravity_y;
    });
}

int fc_set_gravity(fc_grid* grid, double gravity_y)
{
    return guarded([&]
    {
        if (!grid)
            fail(FC_ERR_INVALID_ARGUMENT, "null grid");
        grid->impl.gravity_y = gravity_y;
    });
}

int fc_get_surface_tension(const fc_grid* grid, double* coefficient)
{
    return guarded([&]
    {
        if (!grid || !coefficient)
            fail(FC_ERR_INVALID_ARGUMENT, "null argument");
        *coefficient = grid->impl.surface_tension;
    });
}

int fc_set_surface_tension(fc_grid* grid, double coefficient)
{
    return guarded([&]
    {
        if (!grid)
            fail(FC_ERR_INVALID_ARGUMENT, "null grid");
        if (!std::isfinite(coefficient) || coefficient < 0.0)
            fail(FC_ERR_INVALID_ARGUMENT, "Surface tension must be finite and nonnegative");
        grid->impl.surface_tension = coefficient;
    });
}

int fc_capillary_step_limit(const fc_grid* grid, double* limit)
{
    return guarded([&]
    {
        if (!grid || !limit)
            fail(FC_ERR_INVALID_ARGUMENT, "null argument");
        *limit = fc::capillary_step_limit(grid->impl);
    });
}

int fc_apply_viscosity(fc_grid* grid, double dt, double tolerance, int max_iterations, int* iterations,
    double* relative_residual)
{
    return guarded([&]
    {
        if (!grid)
            fail(FC_ERR_INVALID_ARGUMENT, "null grid");
        if (!std::isfinite(dt) || !(tolerance >= 0.0))
            fail(FC_ERR_INVALID_ARGUMENT, "invalid viscosity time step or tolerance");
        const fc::ViscResult r = fc::apply_viscosity(grid->impl, dt, tolerance, max_iterations);
        if (iterations)
            *iterations = r.iterations;
        if (relative_residual)
            *relative_residual = r.relative_residual;
    });
}

int fc_set_component_viscosity(fc_grid* grid, int phase, int component, double coefficient)
{
    return guarded([&]
    {
        if (!grid)
            fail(FC_ERR_INVALID_ARGUMENT, "null grid");
        if (!std::isfinite(coefficient) || coefficient < 0.0)
            fail(FC_ERR_INVALID_ARGUMENT, "Material viscosity must be finite and nonnegative");
        Grid& g = grid->impl;
        std::vector<double>& mu = phase == 0 ? g.liquid_viscosity : g.gas_viscosity;
        if ((phase != 0 && phase != 1) || component < 0 || size_t(component) >= mu.size())
            fail(FC_ERR_INVALID_ARGUMENT, "no such material component");
        mu[component] = coefficient;
    });
}

int fc_apply_surface_tension(fc_grid* grid, double dt)
{
    return guarded([&]
    {
        if (!grid)
            fail(FC_ERR_INVALID_ARGUMENT, "null grid");
        if (!std::isfinite(dt))
            fail(FC_ERR_INVALID_ARGUMENT, "time step must be finite");
        fc::apply_surface_tension(grid->impl, dt);
    });
}

int fc_surface_curvature(fc_grid* grid, double* curvature, unsigned char* valid)
{
    return guarded([&]
    {
        if (!grid)
            fail(FC_ERR_INVALID_ARGUMENT, "null grid");
        fc::surface_curvature(grid->impl, curvature, valid);
    });
}

int fc_set_preconditioner(fc_grid* grid, int preconditioner)
{
    return guarded([&]
    {
        if (!grid || (preconditioner != FC_PRECONDITIONER_DIAGONAL && preconditioner != FC_PRECONDITIONER_MULTIGRID))
            fail(FC_ERR_INVALID_ARGUMENT, "unknown preconditioner");
        grid->impl.preconditioner = preconditioner;
    });
}

int fc_set_obstacles(fc_grid* grid, const unsigned char* solid)
{
    return guarded([&]
    {
        if (!grid)
            fail(FC_ERR_INVALID_ARGUMENT, "null grid");
        Grid& g = grid->impl;
        if (solid)
        {
            std::vector<unsigned char> flags(g.cells);
            for (size_t i = 0; i < g.cells; ++i)
                flags[i] = solid[i] ? 1 : 0;
            check(cudaMemcpyAsync(g.solid, flags.data(), g.cells, cudaMemcpyHostToDevice, g.stream), "obstacles");
            check(cudaStreamSynchronize(g.stream), "obstacles");
            g.has_solid = true;
        }
        else
            g.has_solid = false;
        fc::refresh_descriptor(g);
        g.coefficients_dirty = true;
    });
}

int fc_upload(fc_grid* grid, const double* liquid_fraction, const double* u, const double* v, const double* pressure,
    const double* const* liquid_mass, const double* const* gas_mass)
{
    return guarded([&]
    {
        if (!grid)
            fail(FC_ERR_INVALID_ARGUMENT, "null grid");
        fc::upload(grid->impl, liquid_fraction, u, v, pressure, liquid_mass, gas_mass);
    });
}

int fc_download(fc_grid* grid, double* liquid_fraction, double* u, double* v, double* pressure,
    double* const* liquid_mass, double* const* gas_mass)
{
    return guarded([&]
    {
        if (!grid)
            fail(FC_ERR_INVALID_ARGUMENT, "null grid");
        fc::download(grid->impl, liquid_fraction, u, v, pressure, liquid_mass, gas_mass);
    });
}

int fc_copy_state(fc_grid* dst, const fc_grid* src)
{
    return guarded([&]
    {
        if (!dst || !src)
            fail(FC_ERR_INVALID_ARGUMENT, "null grid");
        Grid& d = dst->impl;
        const Grid& s = src->impl;
        if (d.W != s.W || d.H != s.H || d.precision != s.precision || d.components() != s.components())
            fail(FC_ERR_INVALID_ARGUMENT, "grids differ in geometry, precision or materials");
        fc::require_uploaded(s);
        if (!d.configured)
            fail(FC_ERR_LIFECYCLE, "configure the destination's materials first");
        fc::allocate_masses(d);
        fc::refresh_descriptor(d);
        const size_t padded = size_t(d.S) * (d.H + 2);
        check(cudaStreamSynchronize(s.stream), "copy source");
        auto copy = [&](void* to, const void* from, size_t bytes)
        { check(cudaMemcpyAsync(to, from, bytes, cudaMemcpyDeviceToDevice, d.stream), "state copy"); };
        copy(d.fraction, s.fraction, d.cells * sizeof(double));
        if (d.components() > 0)
            copy(d.masses, s.masses, size_t(d.components()) * d.cells * sizeof(double));
        copy(d.desc.u, s.desc.u, d.faces_u * d.elem);
        copy(d.desc.v, s.desc.v, d.faces_v * d.elem);
        copy(d.desc.p, s.desc.p, padded * sizeof(double));
        copy(d.desc.p_prev, s.desc.p_prev, padded * sizeof(double));
        check(cudaStreamSynchronize(d.stream), "state copy");
        d.uploaded = true;
        d.coefficients_dirty = true;
    });
}

int fc_project(fc_grid* grid, double dt, int max_iterations, double divergence_tolerance, fc_result* result)
{
    if (!grid)
        return FC_ERR_INVALID_ARGUMENT;
    return fc::project_one(grid->impl, dt, max_iterations, divergence_tolerance, 0.0, result);
}

int fc_project_relative(fc_grid* grid, double dt, int max_iterations, double relative_tolerance,
    double divergence_tolerance, fc_result* result)
{
    if (!grid || !(relative_tolerance > 0.0))
        return FC_ERR_INVALID_ARGUMENT;
    return fc::project_one(grid->impl, dt, max_iterations, divergence_tolerance, relative_tolerance, result);
}

int fc_advect(fc_grid* grid, double dt)
{
    return guarded([&]
    {
        if (!grid)
            fail(FC_ERR_INVALID_ARGUMENT, "null grid");
        if (!(dt > 0.0) || !std::isfinite(dt))
            fail(FC_ERR_INVALID_ARGUMENT, "time step must be positive and finite");
        fc::advect(grid->impl, dt);
    });
}

int fc_set_transport(fc_grid* grid, int transport)
{
    return guarded([&]
    {
        if (!grid)
            fail(FC_ERR_INVALID_ARGUMENT, "null grid");
        if (transport != FC_TRANSPORT_SEMI_LAGRANGIAN && transport != FC_TRANSPORT_PLIC)
            fail(FC_ERR_INVALID_ARGUMENT, "unknown transport scheme %d", transport);
        grid->impl.transport = transport;
    });
}

int fc_set_air_model(fc_grid* grid, int model)
{
    return guarded([&]
    {
        if (!grid)
            fail(FC_ERR_INVALID_ARGUMENT, "null grid");
        if (model != FC_AIR_GAS && model != FC_AIR_DIRICHLET)
            fail(FC_ERR_INVALID_ARGUMENT, "unknown air model %d", model);
        Grid& g = grid->impl;
        if (g.air_model == model)
            return;
        g.air_model = model;
        g.coefficients_dirty = true;
        fc::refresh_descriptor(g);
    });
}

int fc_set_stream_priority(fc_grid* grid, int priority)
{
    return guarded([&]
    {
        if (!grid)
            fail(FC_ERR_INVALID_ARGUMENT, "null grid");
        int least = 0, greatest = 0;
        check(cudaDeviceGetStreamPriorityRange(&least, &greatest), "stream priority range");
        if (priority > least || priority < greatest)
            fail(FC_ERR_INVALID_ARGUMENT, "stream priority %d outside [%d, %d]", priority, greatest, least);
        Grid& g = grid->impl;
        if (priority == g.stream_priority)
            return;
        // The grid's single-grid plan runs on its stream: both are remade (the device state is
        // kept); batches made later take the new priority.
        check(cudaStreamSynchronize(g.stream), "stream priority");
        g.plan.reset();
        cudaStream_t fresh = nullptr;
        check(cudaStreamCreateWithPriority(&fresh, cudaStreamNonBlocking, priority), "stream");
        cudaStreamDestroy(g.stream);
        g.stream = fresh;
        g.stream_priority = priority;
    });
}

int fc_get_air_model(const fc_grid* grid, int* model)
{
    return guarded([&]
    {
        if (!grid || !model)
            fail(FC_ERR_INVALID_ARGUMENT, "null argument");
        *model = grid->impl.air_model;
    });
}

int fc_get_transport(const fc_grid* grid, int* transport)
{
    return guarded([&]
    {
        if (!grid || !transport)
            fail(FC_ERR_INVALID_ARGUMENT, "null argument");
        *transport = grid->impl.transport;
    });
}

int fc_sample_velocity(fc_grid* grid, int count, const double* positions, double* velocities)
{
    return guarded([&]
    {
        if (!grid || count < 0 || (count > 0 && (!positions || !velocities)))
            fail(FC_ERR_INVALID_ARGUMENT, "invalid sample arguments");
        if (count > 0)
            fc::sample_velocity(grid->impl, count, positions, velocities);
    });
}

int fc_apply_gravity(fc_grid* grid, double dt)
{
    return guarded([&]
    {
        if (!grid)
            fail(FC_ERR_INVALID_ARGUMENT, "null grid");
        fc::apply_gravity(grid->impl, dt, true);
    });
}

// Dirichlet air: the liquid's face velocities extended into the air (k_air_faces_extend).
int fc_extend_air_velocity(fc_grid* grid)
{
    return guarded([&]
    {
        if (!grid)
            fail(FC_ERR_INVALID_ARGUMENT, "null grid");
        fc::extend_air_velocity(grid->impl, true);
    });
}

int fc_advance_substep(fc_grid* grid, double dt, int* viscosity_iterations)
{
    return guarded([&]
    {
        if (!grid)
            fail(FC_ERR_INVALID_ARGUMENT, "null grid");
        if (!(dt > 0.0) || !std::isfinite(dt))
            fail(FC_ERR_INVALID_ARGUMENT, "time step must be positive and finite");
        const int viscous = fc::advance_substep(grid->impl, dt, false);
        if (viscosity_iterations)
            *viscosity_iterations = viscous;
    });
}

int fc_step(fc_grid* grid, double dt, int max_iterations, double divergence_tolerance, fc_result* result,
    fc_timings* timings)
{
    if (!grid)
        return FC_ERR_INVALID_ARGUMENT;
    using Clock = std::chrono::steady_clock;
    if (timings)
        *timings = fc_timings{};
    if (!(dt > 0.0))
    {
        // FluidGridCPU::step: dt <= 0 returns {0, inf, false, 0, 0} (FluidGridCPU.cpp:306-307).
        if (result)
        {
            *result = fc_result{};
            result->max_divergence = INFINITY;
        }
        return FC_OK;
    }
    // Capillary subdivisions (FluidGridCPU.cpp:309-320): each advances transport, forces and
    // the projection together.
    const bool tension = grid->impl.surface_tension > 0.0;
    const double subdivisions = tension ? std::max(1.0, std::ceil(dt / fc::capillary_step_limit(grid->impl))) : 1.0;
    // The reference throws std::runtime_error here.
    if (subdivisions > double(std::numeric_limits<int>::max()))
        return guarded([] { fail(FC_ERR_UNSUPPORTED, "Surface tension requires too many physical substeps for this timestep"); });
    const int count = int(subdivisions);
    const double step = dt / count;
    fc_result total{};
    fc_result one{};
    int status = FC_OK;
    auto previous = Clock::now();
    auto elapsed = [&]
    {
        const auto now = Clock::now();
        const double ms = std::chrono::duration<double, std::milli>(now - previous).count();
        previous = now;
        return ms;
    };
    for (int i = 0; i < count; ++i)
    {
        if (!timings)
        {
            // The substep's kernels are enqueued without waiting; the projection orders after
            // them on the grid's stream.
            int viscous = 0;
            if ((status = guarded([&] { viscous = fc::advance_substep(grid->impl, step, false); })) != FC_OK)
                return status;
            total.viscosity_iterations += viscous;
        }
        else
        {
            // Timed: every stage waits for its kernels, so its time is its own.
            // Dirichlet air: transport sees the liquid's velocity extended into the air.
            if (grid->impl.air_model == FC_AIR_DIRICHLET && (status = fc_extend_air_velocity(grid)) != FC_OK)
                return status;
            if ((status = fc_advect(grid, step)) != FC_OK)
                return status;
            timings->transport_ms += elapsed();
            // Implicit viscosity after transport (FluidGridGPU.cpp:1139-1146), 1e-4 relative.
            if (fc::has_viscosity(grid->impl))
            {
                int viscous = 0;
                if ((status = fc_apply_viscosity(grid, step, 1e-4, fc::kViscosityCap, &viscous, nullptr)) != FC_OK)
                    return status;
                total.viscosity_iterations += viscous;
                timings->viscosity_ms += elapsed();
            }
            if ((status = fc_apply_gravity(grid, step)) != FC_OK)
                return status;
            if (tension && (status = fc_apply_surface_tension(grid, step)) != FC_OK)
                return status;
            timings->forces_ms += elapsed();
        }
        if ((status = fc_project(grid, step, max_iterations, divergence_tolerance, &one)) != FC_OK)
            return status;
        if (timings)
            timings->pressure_ms += elapsed();
        const int iterations = total.iterations + one.iterations;
        const int restarts = total.restarts + one.restarts;
        const int kernels = total.kernels + one.kernels;
        const int steps = total.physical_steps + 1;
        const int viscous = total.viscosity_iterations;
        total = one;
        total.viscosity_iterations = viscous;
        total.iterations = iterations;
        total.restarts = restarts;
        total.kernels = kernels;
        total.physical_steps = steps;
        if (!one.converged)
            break;
    }
    if (result)
        *result = total;
    return FC_OK;
}

int fc_max_divergence(fc_grid* grid, double* out)
{
    return guarded([&]
    {
        if (!grid || !out)
            fail(FC_ERR_INVALID_ARGUMENT, "null argument");
        Grid& g = grid->impl;
        fc::require_uploaded(g);
        fc::Plan& p = fc::single_plan(g);
        fc::dispatch(g.precision, [&](auto zero)
        {
            using T = decltype(zero);
            FC_LAUNCH(fc::k_divergence<T>, p.vec.count, fc::kVecThreads, 0, p.stream, p.d_desc, p.at(p.vec));
        });
        fc::SolveState s;
        check(cudaMemcpyAsync(&s, g.desc.state, sizeof(s), cudaMemcpyDeviceToHost, p.stream), "divergence");
        check(cudaStreamSynchronize(p.stream), "divergence");
        *out = s.div_max;
    });
}

int fc_classify(fc_grid* grid, unsigned char* mask)
{
    return guarded([&]
    {
        if (!grid || !mask)
            fail(FC_ERR_INVALID_ARGUMENT, "null argument");
        Grid& g = grid->impl;
        fc::require_uploaded(g);
        fc::Plan& p = fc::single_plan(g);
        FC_LAUNCH(fc::k_classify, p.vec.count, fc::kVecThreads, 0, p.stream, p.d_desc, p.at(p.vec), g.fraction, g.mask);
        check(cudaMemcpyAsync(mask, g.mask, g.cells, cudaMemcpyDeviceToHost, p.stream), "classify");
        check(cudaStreamSynchronize(p.stream), "classify");
    });
}

int fc_download_coefficients(fc_grid* grid, double* inv_u, double* inv_v, double* inv_diagonal)
{
    return guarded([&]
    {
        if (!grid || !inv_u || !inv_v)
            fail(FC_ERR_INVALID_ARGUMENT, "null argument");
        Grid& g = grid->impl;
        fc::require_uploaded(g);
        fc::Plan& p = fc::single_plan(g);
        fc::rebuild_if_dirty(p);
        const fc::LevelDesc& L = g.desc.lev[0];
        if (inv_diagonal && !L.inv)
            fail(FC_ERR_UNSUPPORTED, "a single-level grid keeps no inverse diagonal");
        const size_t padded = size_t(g.S) * (g.H + 2);
        std::vector<double> right(padded), down(padded), inv(inv_diagonal ? padded : 0);
        auto fetch = [&](const void* device, std::vector<double>& host)
        {
            if (g.elem == 8)
            {
                check(cudaMemcpyAsync(host.data(), device, padded * sizeof(double), cudaMemcpyDeviceToHost, p.stream),
                    "coefficients");
                return;
            }
            std::vector<float> f(padded);
            check(cudaMemcpyAsync(f.data(), device, padded * sizeof(float), cudaMemcpyDeviceToHost, p.stream),
                "coefficients");
            check(cudaStreamSynchronize(p.stream), "coefficients");
            for (size_t i = 0; i < padded; ++i)
                host[i] = double(f[i]);
        };
        fetch(L.right, right);
        fetch(L.down, down);
        if (inv_diagonal)
            fetch(L.inv, inv);
        check(cudaStreamSynchronize(p.stream), "coefficients");
        // A cell stores the weights of its right and lower faces (padded layout); the reference's
        // arrays hold every face, walls included (FluidGridTypes.h:10-20).
        const int W = g.W, H = g.H;
        for (int y = 0; y < H; ++y)
        {
            inv_u[size_t(y) * (W + 1)] = 0.0;
            for (int x = 0; x < W; ++x)
            {
                const size_t i = size_t(fc::padded_index(g.S, x, y));
                inv_u[size_t(y) * (W + 1) + x + 1] = right[i];
                inv_v[size_t(y + 1) * W + x] = down[i];
                if (inv_diagonal)
                    inv_diagonal[size_t(y) * W + x] = inv[i];
            }
        }
        for (int x = 0; x < W; ++x)
            inv_v[x] = 0.0;
    });
}

int fc_autotune(fc_grid* grid, int repeats, int* tail_cells, double* vcycle_ms)
{
    return guarded([&]
    {
        if (!grid || repeats <= 0)
            fail(FC_ERR_INVALID_ARGUMENT, "invalid autotune arguments");
        Grid& g = grid->impl;
        fc::require_uploaded(g);
        if (g.preconditioner != FC_PRECONDITIONER_MULTIGRID)
            fail(FC_ERR_INVALID_ARGUMENT, "autotuning needs the multigrid preconditioner");
        const fc::TuneResult r = fc::autotune_plan({&g}, [&]() -> fc::Plan& { return fc::single_plan(g); }, repeats);
        if (tail_cells)
            *tail_cells = r.tail_cells;
        if (vcycle_ms)
            *vcycle_ms = r.ms;
    });
}

int fc_set_tail_cells(fc_grid* grid, int cells)
{
    return guarded([&]
    {
        if (!grid || cells < 1)
            fail(FC_ERR_INVALID_ARGUMENT, "tail threshold must be positive");
        fc::set_tail_cells(grid->impl, cells);
    });
}

int fc_time_kernel(fc_grid* grid, int kernel, int repeats, double* mean_ms)
{
    return guarded([&]
    {
        if (!grid || !mean_ms)
            fail(FC_ERR_INVALID_ARGUMENT, "null argument");
        *mean_ms = fc::time_kernel(grid->impl, kernel, repeats);
    });
}

int fc_divergence_noalloc(const void* u, const void* v, int width, int height, double cell_size, int precision,
    double* stats, void* stream)
{
    return guarded([&]
    {
        if (!u || !v || !stats)
            fail(FC_ERR_INVALID_ARGUMENT, "null argument");
        if (width <= 0 || height <= 0 || !(cell_size > 0.0) || !std::isfinite(cell_size))
            fail(FC_ERR_INVALID_ARGUMENT, "grid geometry must be positive and finite");
        if (precision != FC_PRECISION_FP32 && precision != FC_PRECISION_FP64)
            fail(FC_ERR_INVALID_ARGUMENT, "precision must be FP32 or FP64");
        const long long tiles = (long long)fc::ceil_div(width, fc::kNoAllocTile) * fc::ceil_div(height, fc::kNoAllocTile);
        if (tiles > fc::kNoAllocMaxTiles)
            fail(FC_ERR_INVALID_ARGUMENT,
                "a %dx%d grid needs %lld tiles of 32x32 cells; the no-allocation path holds at most %d "
                "(4,194,304 cells)", width, height, tiles, fc::kNoAllocMaxTiles);
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        unsigned char* scratch = static_cast<unsigned char*>(fc::noalloc_address(s));
        // The arrival counter must start at zero; the partial slots are overwritten.
        check(cudaMemsetAsync(scratch + fc::kNoAllocCounterOffset, 0, sizeof(unsigned int), s), "scratch clear");
        if (precision == FC_PRECISION_FP64)
            FC_LAUNCH(fc::k_divergence_noalloc<double>, int(tiles), fc::kVecThreads, 0, s,
                static_cast<const double*>(u), static_cast<const double*>(v), width, height, cell_size, scratch, stats);
        else
            FC_LAUNCH(fc::k_divergence_noalloc<float>, int(tiles), fc::kVecThreads, 0, s,
                static_cast<const float*>(u), static_cast<const float*>(v), width, height, cell_size, scratch, stats);
    });
}

int fc_velocity_pointers(fc_grid* grid, void** u, void** v)
{
    return guarded([&]
    {
        if (!grid)
            fail(FC_ERR_INVALID_ARGUMENT, "null grid");
        if (u)
            *u = grid->impl.desc.u;
        if (v)
            *v = grid->impl.desc.v;
    });
}

int fc_get_stream(const fc_grid* grid, void** stream)
{
    return guarded([&]
    {
        if (!grid || !stream)
            fail(FC_ERR_INVALID_ARGUMENT, "null argument");
        *stream = grid->impl.stream;
    });
}

int fc_synchronize(fc_grid* grid)
{
    return guarded([&]
    {
        if (!grid)
            fail(FC_ERR_INVALID_ARGUMENT, "null grid");
        check(cudaStreamSynchronize(grid->impl.stream), "synchronize");
    });
}

int fc_apply_preconditioner(fc_grid* grid, const double* residual, double residual_mean, double* correction)
{
    return guarded([&]
    {
        if (!grid || !residual || !correction)
            fail(FC_ERR_INVALID_ARGUMENT, "null argument");
        fc::apply_preconditioner(grid->impl, residual, residual_mean, correction);
    });
}

int fc_save_checkpoint(fc_grid* grid, char* metadata, size_t metadata_capacity, size_t* metadata_bytes, void* payload,
    size_t payload_capacity, size_t* payload_bytes)
{
    return guarded([&]
    {
        if (!grid)
            fail(FC_ERR_INVALID_ARGUMENT, "null grid");
        fc::save_checkpoint(grid->impl, metadata, metadata_capacity, metadata_bytes, payload, payload_capacity,
            payload_bytes);
    });
}

int fc_load_checkpoint(fc_grid* grid, const char* metadata, const void* payload, size_t payload_bytes)
{
    return guarded([&]
    {
        if (!grid)
            fail(FC_ERR_INVALID_ARGUMENT, "null grid");
        fc::load_checkpoint(grid->impl, metadata, payload, payload_bytes);
    });
}

int fc_batch_create(fc_grid* const* grids, int count, fc_batch** out)
{
    return guarded([&]
    {
        if (!grids || count <= 0 || !out)
            fail(FC_ERR_INVALID_ARGUMENT, "empty batch");
        *out = nullptr;
        std::vector<Grid*> members;
        for (int i = 0; i < count; ++i)
        {
            if (!grids[i])
                fail(FC_ERR_INVALID_ARGUMENT, "null grid in batch");
            if (grids[i]->impl.precision != grids[0]->impl.precision)
                fail(FC_ERR_INVALID_ARGUMENT, "a batch needs one precision");
            for (int j = 0; j < i; ++j)
                if (grids[j] == grids[i])
                    fail(FC_ERR_INVALID_ARGUMENT, "grid listed twice in a batch");
            members.push_back(&grids[i]->impl);
        }
        auto batch = std::make_unique<fc_batch>();
        batch->grids.assign(grids, grids + count);
        batch->plan = fc::make_plan(members, nullptr);
        *out = batch.release();
    });
}

int fc_batch_destroy(fc_batch* batch)
{
    return guarded([&]
    {
        if (batch)
        {
            cudaStreamSynchronize(batch->plan->stream);
            delete batch;
        }
    });
}

int fc_batch_project(fc_batch* batch, const double* dts, int max_iterations, double divergence_tolerance,
    double relative_tolerance, fc_result* results)
{
    return guarded([&]
    {
        if (!batch || !dts || !results)
            fail(FC_ERR_INVALID_ARGUMENT, "null argument");
        if (max_iterations < 0)
            fail(FC_ERR_INVALID_ARGUMENT, "max_iterations must be non-negative");
        for (size_t i = 0; i < batch->grids.size(); ++i)
            if (!(dts[i] > 0.0))
                fail(FC_ERR_INVALID_ARGUMENT, "time steps must be positive");
        fc::Plan& p = *batch->plan;
        // Grids may have changed (obstacles, materials) since the batch was made.
        for (Grid* g : p.grids)
        {
            g->desc.solid = g->has_solid ? g->solid : nullptr;
            g->desc.masses = g->mass_ptrs;
            g->desc.components = g->components();
            check(cudaStreamSynchronize(g->stream), "batch member");
        }
        fc::upload_descriptors(p);
        fc::project_plan(p, dts, max_iterations, divergence_tolerance, relative_tolerance, results);
    });
}

int fc_batch_autotune(fc_batch* batch, int repeats, int* tail_cells, double* vcycle_ms)
{
    return guarded([&]
    {
        if (!batch || repeats <= 0)
            fail(FC_ERR_INVALID_ARGUMENT, "invalid autotune arguments");
        std::vector<Grid*> grids;
        for (fc_grid* g : batch->grids)
        {
            fc::require_uploaded(g->impl);
            if (g->impl.preconditioner != FC_PRECONDITIONER_MULTIGRID)
                fail(FC_ERR_INVALID_ARGUMENT, "autotuning needs the multigrid preconditioner");
            grids.push_back(&g->impl);
        }
        cudaStream_t stream = batch->plan->stream;
        const fc::TuneResult r = fc::autotune_plan(grids, [&]() -> fc::Plan&
        {
            batch->plan.reset();
            batch->plan = fc::make_plan(grids, nullptr);
            (void)stream;
            return *batch->plan;
        }, repeats);
        if (tail_cells)
            *tail_cells = r.tail_cells;
        if (vcycle_ms)
            *vcycle_ms = r.ms;
    });
}

int fc_batch_get_stream(const fc_batch* batch, void** stream)
{
    return guarded([&]
    {
        if (!batch || !stream)
            fail(FC_ERR_INVALID_ARGUMENT, "null argument");
        *stream = batch->plan->stream;
    });
}

} // extern "C"
