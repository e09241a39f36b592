/*
 * fluidcuda: C ABI of the UniformCUDA backend for FluidSim's uniform MAC grid (B200, sm_100a).
 *
 * This is the drop-in boundary for FluidSim's engine contract fluid::FluidGridBase
 * (FluidSim/FluidGridBase.h:20-147), reached through FluidGrid::selectBackend
 * (FluidSim/FluidGrid.cpp:37-90). include/FluidGridCUDA.h wraps these functions into a
 * FluidGridBase implementation; each entry point below names the reference member it replaces.
 *
 * Conventions
 *  - Every function returns an fc_status code; 0 is success. No C++ exception crosses the ABI.
 *    fc_last_error() returns a message for the last failure on the calling thread.
 *  - Host arrays are FP64 in the reference's layouts (FluidSim/FluidGridTypes.h:10-20):
 *    cell fields are width*height, row-major (index y*width + x); u faces are (width+1)*height
 *    (index y*(width+1) + x); v faces are width*(height+1) (index y*width + x).
 *  - A grid owns its device memory and one CUDA stream; calls on one grid come from one thread
 *    (the reference's simulation-owner rule, FluidGridBase.h:37-39).
 *  - Device state is converted to the working precision on upload and back to FP64 on download
 *    (the reference converts the same way, UniformWebGPU/FluidGridWebGPU.cpp:134-137).
 */
#ifndef FLUIDCUDA_H
#define FLUIDCUDA_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FC_ABI_VERSION 2

typedef enum fc_status
{
    FC_OK = 0,
    FC_ERR_INVALID_ARGUMENT = 1, /* the reference throws std::invalid_argument */
    FC_ERR_LIFECYCLE = 2,        /* std::logic_error: wrong call order (e.g. step before upload) */
    FC_ERR_CUDA = 3,             /* std::runtime_error: device failure */
    FC_ERR_OUT_OF_MEMORY = 4,
    FC_ERR_NONFINITE = 5,
    FC_ERR_BREAKDOWN = 6,
    FC_ERR_UNSUPPORTED = 7,
    FC_ERR_TIMEOUT = 8           /* a device loop hit its iteration cap without finishing */
} fc_status;

typedef enum fc_precision
{
    FC_PRECISION_FP32 = 0,  /* plain FP32 working arrays; FP64 pressure, dots and coarse solve */
    FC_PRECISION_FP64 = 1,  /* everything FP64: the reference's arithmetic */
    FC_PRECISION_MIXED = 2  /* FP32, with the coarse multigrid levels' face weights stored in FP16 */
} fc_precision;

/* How a projection's PCG loop is launched (process-wide). */
typedef enum fc_transport
{
    FC_TRANSPORT_SEMI_LAGRANGIAN = 0, /* midpoint back-tracing on the staggered sampler (default) */
    FC_TRANSPORT_PLIC = 1             /* UniformCPU's conservative PLIC/MYC transport */
} fc_transport;

/* What the pressure solve makes of air. */
typedef enum fc_air_model
{
    FC_AIR_GAS = 0,      /* the reference's two-phase model: air is a light gas component of the
                            closed, mean-free system (FluidGridCPU.cpp:1063-1090); default */
    FC_AIR_DIRICHLET = 1 /* free surface: cells neither solid nor liquid phase (f > 0.5) are held
                            at p = 0 and only the liquid is made divergence-free */
} fc_air_model;

typedef enum fc_launch_mode
{
    FC_LAUNCH_GRAPH = 0, /* one CUDA graph per projection with a device-side loop (default) */
    FC_LAUNCH_STREAM = 1 /* host-driven launches polling the done flags: same kernels, for
                            per-kernel profilers and drivers without conditional graph nodes */
} fc_launch_mode;

typedef enum fc_preconditioner
{
    FC_PRECONDITIONER_DIAGONAL = 0, /* FluidGridCPU::PressurePreconditioner::Diagonal */
    FC_PRECONDITIONER_MULTIGRID = 1 /* ::Multigrid (default) */
} fc_preconditioner;

/* Why a pressure solve stopped. */
typedef enum fc_solve_status
{
    FC_SOLVE_RUNNING = 0,
    FC_SOLVE_CONVERGED = 1,       /* stop rule met on the true residual */
    FC_SOLVE_ITERATION_LIMIT = 2,
    FC_SOLVE_STALLED = 3,         /* r.z or d.Ad lost positivity or finiteness */
    FC_SOLVE_NO_WORK = 4,         /* right-hand side already below tolerance */
    FC_SOLVE_BREAKDOWN = 5        /* coarsest factorisation failed */
} fc_solve_status;

/* Mirrors fluid::FluidProjectionResult field for field (FluidSim/FluidGridTypes.h:59-79), then
 * adds the solver's own measurements. */
typedef struct fc_result
{
    int iterations;
    double max_divergence; /* max |div u| over cells, 1/s; +inf when non-finite */
    int converged;         /* max_divergence <= divergence tolerance */
    int physical_steps;
    int transport_steps;
    int relaxed;
    double max_volume_error;
    double rms_volume_error;
    int viscosity_iterations;
    int precision_limited; /* solve converged; only float velocity rounding exceeds tolerance */
    /* additions */
    int solve_status;          /* fc_solve_status */
    double residual_max;       /* final true residual b - A p, max norm (pressure units) */
    double residual_l2;        /* its L2 norm */
    double rhs_l2;             /* L2 norm of the mean-free right-hand side */
    double divergence_excess;  /* max over cells of |div u| minus its float rounding allowance */
    double divergence_l2;      /* L2 norm of div u over cells */
    int restarts;              /* recurrences that drifted and were restarted from b - A p */
    int kernels;               /* kernels the projection launched on the device */
    int refreshes;             /* FP32: early restarts from b - A p once the recurrence fell 1e-4 */
} fc_result;

/* Mirrors fluid::FluidStepTimings (FluidSim/FluidGridTypes.h:49-57); milliseconds. */
typedef struct fc_timings
{
    double transport_ms;
    double viscosity_ms;
    double forces_ms;
    double pressure_ms;
    double selection_ms;
    double regrid_ms;
} fc_timings;

typedef struct fc_grid fc_grid;
typedef struct fc_batch fc_batch;

int fc_abi_version(void);
const char* fc_last_error(void);
const char* fc_status_string(int status);
/* Number of kernels this library has launched in the calling process (a launch counter). */
long long fc_kernel_launches(void);
/* Selects the launch mechanism of subsequent projections (fc_launch_mode). */
int fc_set_launch_mode(int mode);

/* FluidGridCPU::FluidGridCPU(w, h, cell_size) (UniformCPU/FluidGridCPU.h:63); the device is
 * the calling thread's current CUDA device. */
int fc_create(int width, int height, double cell_size, int precision, fc_grid** out);
/* FluidGridBase::destroy (FluidGridBase.h:129) and the destructor. */
int fc_destroy(fc_grid* grid);

/* getWidth/getHeight/getCellSize (FluidGridBase.h:31-33). */
int fc_get_geometry(const fc_grid* grid, int* width, int* height, double* cell_size);
/* getOrigin/setOrigin (FluidGridBase.h:34-35). */
int fc_get_origin(const fc_grid* grid, double* x, double* y);
int fc_set_origin(fc_grid* grid, double x, double y);
int fc_get_precision(const fc_grid* grid, int* precision);

/* configureMaterials (FluidGridBase.h:42): component densities of the liquid and the gas
 * mixture, in order. Viscosities may be null (all zero). Must precede fc_upload. */
int fc_configure_materials(fc_grid* grid, int liquid_count, const double* liquid_densities,
    const double* liquid_viscosities, int gas_count, const double* gas_densities, const double* gas_viscosities);

/* getGravityY/setGravityY (FluidGridBase.h:70-71). */
int fc_get_gravity(const fc_grid* grid, double* gravity_y);
int fc_set_gravity(fc_grid* grid, double gravity_y);

/* FluidGridCPU::pressure_preconditioner (UniformCPU/FluidGridCPU.h:39-44). */
int fc_set_preconditioner(fc_grid* grid, int preconditioner);

/* Solid obstacle cells (width*height bytes, nonzero = solid; null clears). Their faces close
 * like the outer walls. No reference counterpart: the reference has only the four walls. */
int fc_set_obstacles(fc_grid* grid, const unsigned char* solid);

/* upload (FluidGridBase.h:118; FluidGridCPU.cpp:198-254). Null arrays mean zero. liquid_mass
 * and gas_mass point to one array per configured component (may be null: all zero). */
int fc_upload(fc_grid* grid, const double* liquid_fraction, const double* u, const double* v, const double* pressure,
    const double* const* liquid_mass, const double* const* gas_mass);
/* download (FluidGridBase.h:119). Null outputs are skipped. */
int fc_download(fc_grid* grid, double* liquid_fraction, double* u, double* v, double* pressure,
    double* const* liquid_mass, double* const* gas_mass);

/* Device-side copy of the complete physical state and solver history between two grids of
 * the same geometry, precision and materials (no host traffic). */
int fc_copy_state(fc_grid* dst, const fc_grid* src);

/* FluidGridCPU::project(dt, max_iterations, tolerance) (FluidGridCPU.cpp:1030-1124): closes the
 * walls, forms the mean-free divergence, solves the pressure by PCG to the reference's rule
 * max |r| <= tolerance * dx^2 / dt, updates the face velocities. */
int fc_project(fc_grid* grid, double dt, int max_iterations, double divergence_tolerance, fc_result* result);
/* The same projection stopped by the relative rule ||r||_2 <= relative_tolerance * ||b||_2. */
int fc_project_relative(fc_grid* grid, double dt, int max_iterations, double relative_tolerance, double divergence_tolerance,
    fc_result* result);

/* step (FluidGridBase.h:133-134; FluidGridCPU.cpp:300-360): transport (fc_advect), forces
 * (gravity on interior v faces, FluidGridCPU.cpp:987-996), then the projection. */
int fc_step(fc_grid* grid, double dt, int max_iterations, double divergence_tolerance, fc_result* result,
    fc_timings* timings);
/* FluidGridCPU::advect (UniformCPU/FluidGridCPU.h:121): this backend transports by second-order
 * semi-Lagrangian back-tracing instead of the reference's PLIC (FluidGridCPU.cpp:362-463),
 * sampling with the reference's staggered bilinear sampler (FluidGridCPU.cpp:67-90, 465-471).
 * Face velocities, the liquid fraction and every component mass are traced through the
 * velocity at the start of the step. */
int fc_advect(fc_grid* grid, double dt);
/* Transport scheme of fc_advect and fc_step. FC_TRANSPORT_PLIC is FluidGridCPU::advect
 * (UniformCPU/FluidGridCPU.cpp:362-463): conservative, directionally split PLIC/MYC transport of
 * the liquid fraction, every component mass and the face momenta in CFL substeps, evaluated in
 * FP64 whatever the grid's precision. */
int fc_set_transport(fc_grid* grid, int transport);
int fc_get_transport(const fc_grid* grid, int* transport);
/* Air model of the pressure solve (fc_air_model). No counterpart in the reference, whose air is
 * always a gas component; FC_AIR_DIRICHLET replaces the closure of FluidGridCPU.cpp:1063-1090 by
 * p = 0 in the air: no mean is removed, the liquid beside air sees the zero across the face (the
 * face weight 2 / (rho_liquid + rho_air) and the velocity update stay the two-phase ones), every
 * multigrid level holds the cells that cover no unknown at zero, the coarsest system pins no
 * cell, and max_divergence runs over the liquid only. A grid without air cells then has a
 * singular system: its coarsest factor breaks down. Set it before a batch holds the grid. */
int fc_set_air_model(fc_grid* grid, int model);
/* Priority of the grid's CUDA stream (cudaDeviceGetStreamPriorityRange: lower numbers run
 * first when kernels of several streams wait for the same SMs; 0 is the default). Waits for the
 * grid's work, then gives the grid a new stream of that priority (fc_get_stream returns it; the
 * old handle is destroyed). Batches made afterwards run at the highest priority among their
 * members. */
int fc_set_stream_priority(fc_grid* grid, int priority);
int fc_get_air_model(const fc_grid* grid, int* model);
/* Under Dirichlet air nothing constrains the velocity between air cells, so fc_step extends the
 * liquid's face velocities into the air before each substep's transport: faces of liquid cells,
 * solid faces and walls are known; for 4 layers each unknown face beside known ones takes their
 * mean; the faces left unknown are set to zero. No counterpart in the reference (its air is a
 * gas the projection constrains). Exposed for checks; fc_step calls it itself. */
int fc_extend_air_velocity(fc_grid* grid);
/* One physical substep of fc_step before its projection (FluidGridCPU.cpp:300-360 order): the
 * air extension under Dirichlet air, transport, implicit viscosity when a component is viscous,
 * gravity and surface tension. The kernels are enqueued on the grid's stream and the call
 * returns without waiting for them (the viscosity solve and PLIC transport read values back and
 * wait); the next projection of the grid (fc_project, fc_batch_project) runs after them, and
 * errors of the enqueued kernels surface at the next call that waits. viscosity_iterations may
 * be NULL. fc_step runs its substeps this way unless it is asked for stage timings. */
int fc_advance_substep(fc_grid* grid, double dt, int* viscosity_iterations);
/* FluidGridCPU::sampleVelocity (UniformCPU/FluidGridCPU.h:132, FluidGridCPU.cpp:465-471): the
 * staggered bilinear velocity at `count` world positions. positions and velocities are host
 * arrays of interleaved (x, y) pairs. */
int fc_sample_velocity(fc_grid* grid, int count, const double* positions, double* velocities);
/* Surface tension coefficient (FluidGridBase.h get/setSurfaceTension; FluidGridCPU.cpp:835-841:
 * negative or non-finite values are rejected). fc_step subdivides dt by the capillary limit
 * (FluidGridCPU.cpp:309-320) and applies the capillary force after gravity. */
int fc_get_surface_tension(const fc_grid* grid, double* coefficient);
int fc_set_surface_tension(fc_grid* grid, double coefficient);
/* FluidGridCPU::capillaryStepLimit (FluidGridCPU.cpp:843-860); +inf without tension. */
int fc_capillary_step_limit(const fc_grid* grid, double* limit);
/* FluidGridCPU::applySurfaceTension (FluidGridCPU.cpp:862-926): height-function curvature
 * (UniformCPU/FluidSurfaceTensionCPU.h) and the capillary face force. No-op when the
 * coefficient is zero. */
int fc_apply_surface_tension(fc_grid* grid, double dt);
/* The completed curvature of every cell (1/length) and its validity flag (1 = valid), computed
 * from the current liquid fraction; either output may be NULL. No reference counterpart: it
 * exposes FluidSurfaceTensionCPU::curvature for inspection. */
int fc_surface_curvature(fc_grid* grid, double* curvature, unsigned char* valid);
/* FluidGridGPU::applyViscosity (UniformWebGPU/FluidGridGPU.cpp:987-1045) and
 * ViscositySolverGPU::solve (UniformWebGPU/ViscositySolverGPU.cpp:170-294): backward-Euler
 * viscosity on the face velocities, with the cell viscosity the volume-weighted mean of the
 * component viscosities. CG with a multigrid preconditioner stops when the true residual, checked
 * every 4 iterations, satisfies |r|^2_M <= tolerance^2 |v0|^2_M + 1e-12 total mass. No-op for
 * dt <= 0 or when no component is viscous. max_iterations < 0: no cap; reaching a cap returns
 * FC_ERR_TIMEOUT with the velocities unchanged. Outputs may be NULL. fc_step calls this after
 * transport with tolerance 1e-4. */
int fc_apply_viscosity(fc_grid* grid, double dt, double tolerance, int max_iterations, int* iterations,
    double* relative_residual);
/* setComponentViscosity (FluidGridBase.h:48-52): phase 0 liquid, 1 gas. */
int fc_set_component_viscosity(fc_grid* grid, int phase, int component, double coefficient);
/* FluidGridCPU::applyGravity (FluidGridCPU.cpp:987-996). */
int fc_apply_gravity(fc_grid* grid, double dt);

/* maxDivergence (FluidGridBase.h:135; FluidGridCPU.cpp:1126-1152). */
int fc_max_divergence(fc_grid* grid, double* out);

/* Cell classes from the reference thresholds (liquid f > 0.5, FluidGridCPU.cpp:1321-1322;
 * interface 0 < f < 1, FluidGridCPU.cpp:531-533) and the obstacle mask: bit 1 liquid,
 * bit 2 interface, bit 4 solid (a solid cell carries only bit 4). width*height bytes. */
int fc_classify(fc_grid* grid, unsigned char* mask);

/* One application of the grid's pressure preconditioner to `residual` (width*height, minus
 * residual_mean), as PressureMultigrid::apply (UniformCPU/PressureMultigrid.h:43,
 * PressureMultigrid.cpp:410-434) or the diagonal (FluidGridCPU.cpp:1691-1698). The correction
 * keeps its constant component, like the reference's apply. Rebuilds coefficients if needed. */
int fc_apply_preconditioner(fc_grid* grid, const double* residual, double residual_mean, double* correction);

/* The fine level's face weights and inverse diagonal as the projection uses them, in the
 * reference's layout: inv_u (width+1)*height, inv_v width*(height+1), inv_diagonal
 * width*height (may be null), each in the grid's working precision widened to double. The
 * coefficients are rebuilt from the current state first if it changed. Replaces reading
 * FluidGridCPU's inv_density_u/v and inv_pressure_diagonal (FluidGridCPU.cpp:1154-1205) for
 * parity checks. A single-level grid keeps no inverse diagonal: FC_ERR_UNSUPPORTED. */
int fc_download_coefficients(fc_grid* grid, double* inv_u, double* inv_v, double* inv_diagonal);

/* Times one kernel of the projection with CUDA events on the grid's stream, on the grid's
 * current data, and returns the mean duration of `repeats` launches in milliseconds. Kernels:
 * 0 fine-level pre-smoothing + restriction, 1 fine-level prolongation + post-smoothing,
 * 2 direction update + operator, 3 coarse tail. They write only solver scratch (the multigrid
 * levels, z, d, q), so the physical state is unchanged. Profiling aid. */
int fc_time_kernel(fc_grid* grid, int kernel, int repeats, double* mean_ms);

/* Divergence statistics of caller-owned face velocities, for callers that cannot allocate
 * device memory: a host whose own allocator owns all of the device's memory (a game engine or
 * a framework with its own pool), a process held to a fixed device-memory budget, or a
 * real-time loop that must not stall in the driver, where cudaMalloc can synchronise the
 * device. No counterpart in the reference.
 *
 * u and v are device arrays in the reference layout ((width+1)*height and width*(height+1)),
 * float for FC_PRECISION_FP32 or double for FC_PRECISION_FP64. stats is a device array of 3
 * doubles receiving max |div u| (1/s; +inf if any cell is non-finite), the largest excess of
 * |div u| over the cell's float rounding allowance, and the sum of div u squared. The work is
 * queued on `stream` (a cudaStream_t, 0 for the legacy stream); the call does not wait. The
 * stream must belong to the current device; another device's stream is rejected with
 * FC_ERR_INVALID_ARGUMENT.
 *
 * This entry point allocates nothing: its scratch is a fixed 128 KiB device array that every
 * GPU loading this library keeps until process exit. Grids are limited to 4096 tiles of 32x32
 * cells (4,194,304 cells, e.g. 2048x2048); larger ones are rejected with
 * FC_ERR_INVALID_ARGUMENT. Each call outside stream capture looks up the array's device
 * address (so a device reset by the host leaves nothing stale); a call during capture reuses
 * the last address looked up on that device, so make one call before any stream capture, and
 * again after a device reset. All calls share the one array, so calls
 * whose work overlaps on the GPU race: order them on one stream or synchronise between them. */
int fc_divergence_noalloc(const void* u, const void* v, int width, int height, double cell_size, int precision,
    double* stats, void* stream);

/* Device pointers of the face velocities (working precision), for zero-copy producers. */
int fc_velocity_pointers(fc_grid* grid, void** u, void** v);
/* The grid's stream (cudaStream_t) and a wait for all of its work. */
int fc_get_stream(const fc_grid* grid, void** stream);
int fc_synchronize(fc_grid* grid);

/* saveCheckpoint (FluidGridBase.h:123): the "cuda-uniform" native checkpoint, modelled on the
 * reference's "webgpu-uniform" one (UniformWebGPU/FluidGridGPU.cpp:567-695). JSON metadata
 * (NUL-terminated) and a binary payload: liquid fraction, u, v, pressure, previous pressure,
 * component masses, then the obstacle mask, each in the grid's device precision. With both
 * buffers null the call only reports the sizes needed. */
int fc_save_checkpoint(fc_grid* grid, char* metadata, size_t metadata_capacity, size_t* metadata_bytes, void* payload,
    size_t payload_capacity, size_t* payload_bytes);
/* loadCheckpoint (FluidGridBase.h:125; FluidGridGPU.cpp:697-892): restores materials, settings
 * and state. Every field is validated before any state changes; a checkpoint of another
 * backend, version, precision or geometry is rejected with FC_ERR_INVALID_ARGUMENT. */
int fc_load_checkpoint(fc_grid* grid, const char* metadata, const void* payload, size_t payload_bytes);

/* Batched projection: many independent grids of one precision, uneven sizes allowed, solved
 * together (one launch per kernel for all grids; per-grid convergence). No reference
 * counterpart: the reference steps scenes one after another (FluidSim.cpp:90-93, 120-131). */
/* Device bytes a grid of this description holds once created, configured with `components`
 * material components and (surface_tension != 0) the curvature sweeps, including its
 * single-grid solve plan. Host arithmetic only: no device call. No reference counterpart (the
 * serving loop admits simulations by this figure). */
int fc_grid_device_bytes(int width, int height, int precision, int components, int surface_tension, size_t* bytes);
/* Device bytes a live grid holds, counted the same way. */
int fc_get_device_bytes(const fc_grid* grid, size_t* bytes);

int fc_batch_create(fc_grid* const* grids, int count, fc_batch** out);
int fc_batch_destroy(fc_batch* batch);
/* dts: one time step per grid. relative_tolerance > 0 selects the relative rule. */
int fc_batch_project(fc_batch* batch, const double* dts, int max_iterations, double divergence_tolerance,
    double relative_tolerance, fc_result* results);
int fc_batch_get_stream(const fc_batch* batch, void** stream);

/* Autotuning of the multigrid schedule (no reference counterpart). The tail threshold is the
 * largest level the one-block tail cycles in shared memory; larger levels run the strip
 * kernels. It changes which kernels run, not the arithmetic. fc_autotune and fc_batch_autotune
 * time `repeats` V-cycles of the grid's (or the batch's) plan under each candidate threshold
 * (256, 1024, 4096 cells) and keep the fastest; the grids' states are left as they were.
 * Outputs may be NULL. fc_set_tail_cells sets the threshold directly (default 1024). */
int fc_autotune(fc_grid* grid, int repeats, int* tail_cells, double* vcycle_ms);
int fc_batch_autotune(fc_batch* batch, int repeats, int* tail_cells, double* vcycle_ms);
int fc_set_tail_cells(fc_grid* grid, int cells);

/* ---- Serving: continuous batching of many simulations on one GPU ----------------------------
 * A request loop in the spirit of FluidScene::sceneProcess (FluidScene.inl:328-420) for many
 * independent simulations. A worker thread owns every grid. Each tick it admits queued
 * simulations in arrival order while their device bytes (fc_grid_device_bytes) fit the budget
 * and a slot is free, runs one physical (sub)step of transport and forces per active grid, then
 * projects all active grids in one batched solve, and retires the simulations that finished
 * (their final state is copied to host memory and their device memory freed). State stays
 * device-resident between steps. Every simulation computes exactly what fc_step would compute
 * on it alone. */
typedef struct fc_server fc_server;

typedef struct fc_sim_desc
{
    int width, height;
    double cell_size;
    int precision;
    int liquid_count;
    const double* liquid_densities;
    int gas_count;
    const double* gas_densities;
    double gravity_y;
    double surface_tension;
    const unsigned char* solid;      /* width*height obstacle cells, or NULL */
    const double* liquid_fraction;   /* initial state as for fc_upload; NULL arrays mean zero */
    const double* u;
    const double* v;
    const double* pressure;
    const double* const* liquid_mass;
    const double* const* gas_mass;
    int steps;                       /* time steps to run */
    double dt;
    int max_iterations;
    double divergence_tolerance;     /* the max-norm rule of fc_project */
} fc_sim_desc;

typedef enum fc_sim_state
{
    FC_SIM_QUEUED = 0,
    FC_SIM_RUNNING = 1,
    FC_SIM_DONE = 2,
    FC_SIM_FAILED = 3
} fc_sim_state;

typedef struct fc_sim_status
{
    int state;               /* fc_sim_state */
    int error;               /* fc_status of a failure, else FC_OK */
    int steps_done;
    int physical_steps;      /* capillary subdivisions included */
    long long iterations;    /* PCG iterations over all steps */
    int converged;           /* every projection converged */
    double max_divergence;   /* after the last projection */
    double queued_ms;        /* submission to admission */
    double run_ms;           /* admission to completion */
    size_t device_bytes;     /* charged against the budget while running */
} fc_sim_status;

typedef struct fc_server_stats
{
    long long ticks;
    long long steps;            /* completed time steps over all simulations */
    long long physical_steps;
    double cell_steps;          /* sum over completed steps of the grid's cells */
    double busy_ms;             /* wall time with at least one simulation running */
    double step_p50_ms;         /* latency of a time step: its first tick's start to its last tick's end */
    double step_p99_ms;
    double step_max_ms;
    int peak_active;
    size_t peak_bytes;
    long long batch_rebuilds;   /* batched solve plans built (one per change of membership) */
} fc_server_stats;

/* device_budget_bytes: device memory the simulations may hold together; max_active: slots
 * (both shared by all size classes). Simulations are sorted by cells into size classes, each
 * stepped by its own worker thread in its own batched solves, so a small grid's step latency
 * does not wait on a large grid's. fc_server_create uses five classes: up to 128 x 128 cells,
 * up to 256 x 256, 512 x 512, 1024 x 1024, and larger. fc_server_create_classes takes `classes` classes with
 * classes - 1 increasing bounds: class k holds grids of more than max_cells[k - 1] and at most
 * max_cells[k] cells; the last class holds the rest. One class steps every simulation in
 * lockstep. Within a class, simulations are admitted in arrival order. */
int fc_server_create(size_t device_budget_bytes, int max_active, fc_server** out);
int fc_server_create_classes(size_t device_budget_bytes, int max_active, int classes, const long long* max_cells,
    fc_server** out);
/* Stops the workers; simulations still queued or running are dropped. */
int fc_server_destroy(fc_server* server);
/* Copies the description and initial state; never blocks on the GPU. A simulation that could
 * never fit the budget is rejected with FC_ERR_INVALID_ARGUMENT. */
int fc_server_submit(fc_server* server, const fc_sim_desc* desc, long long* id);
int fc_server_status(fc_server* server, long long id, fc_sim_status* status);
/* Waits until the simulation is done or failed; FC_ERR_TIMEOUT after timeout_seconds. */
int fc_server_wait(fc_server* server, long long id, double timeout_seconds, fc_sim_status* status);
/* Final state of a finished simulation (as fc_download; NULL outputs are skipped). */
int fc_server_download(fc_server* server, long long id, double* liquid_fraction, double* u, double* v,
    double* pressure, double* const* liquid_mass, double* const* gas_mass);
/* The message of the call that failed a simulation (empty while it has not failed), truncated
 * to capacity - 1 characters and terminated. */
int fc_server_error(fc_server* server, long long id, char* text, size_t capacity);
/* Forgets a finished simulation and its host copy of the final state. */
int fc_server_release(fc_server* server, long long id);
/* Statistics over all size classes (ticks: the sum of the classes' ticks). */
int fc_server_get_stats(fc_server* server, fc_server_stats* stats);
int fc_server_class_count(fc_server* server, int* classes);
/* Statistics of one size class; max_cells (may be NULL) receives its upper bound in cells. */
int fc_server_get_class_stats(fc_server* server, int size_class, fc_server_stats* stats, long long* max_cells);
/* Latency of every completed time step, class by class in completion order; count receives
 * the total. */
int fc_server_step_latencies(fc_server* server, double* ms, size_t capacity, size_t* count);

#ifdef __cplusplus
}
#endif
#endif
