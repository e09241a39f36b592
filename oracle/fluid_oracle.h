/*
 * CPU restatement of the FluidSim UniformCPU pressure projection, in plain C and FP64.
 *
 * TEST INFRASTRUCTURE ONLY. This is the parity oracle for the CUDA backend: it is linked by
 * tests/, __graft_entry__.smoke() and the cpu_baseline leg of bench.py, never by the product.
 * It is pinned against the reference engine itself (oracle/_ref, compiled from the reference
 * sources by oracle/Makefile) and against the golden fixtures in tests/golden/.
 *
 * Reference files (paths inside the FluidSim project):
 *   FluidSim/UniformCPU/FluidGridCPU.cpp   project, coefficients, operator, PCG driver
 *   FluidSim/UniformCPU/PressureMultigrid.cpp  V-cycle preconditioner
 */
#ifndef FLUID_ORACLE_H
#define FLUID_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct or_grid or_grid;
typedef struct or_mg or_mg;

typedef struct or_result
{
    int iterations;        /* PCG iterations; -1 on coarse factor breakdown */
    int converged;         /* max |div u| <= tolerance after the update */
    double max_divergence; /* max |(du + dv)/dx| over cells, 1/s; +inf if non-finite */
    double residual_max;   /* final true residual, max norm (pressure units) */
    double residual_l2;    /* final true residual, L2 norm */
    double rhs_l2;         /* L2 norm of the mean-free right-hand side */
} or_result;

enum { OR_PRECONDITIONER_DIAGONAL = 0, OR_PRECONDITIONER_MULTIGRID = 1 };

/* Grid lifecycle. The grid owns u ((w+1)*h), v (w*(h+1)), pressure and previous pressure (w*h). */
or_grid* or_grid_create(int width, int height, double cell_size);
void or_grid_destroy(or_grid* grid);
void or_grid_set_preconditioner(or_grid* grid, int which);
/* Solid obstacle cells (no reference counterpart): their faces close like walls and they are
 * excluded from every mean. NULL clears. Call after upload (it rebuilds the coefficients). */
void or_grid_set_solid(or_grid* grid, const unsigned char* solid);

/* Dirichlet air (no reference counterpart): cells of `air` hold p = 0 (the free-surface
 * boundary), only the other cells are unknowns and divergence-free, and no mean is removed.
 * NULL returns to the reference's gas model. Call after upload. or_air_mask classifies air as
 * the cells that are neither solid nor liquid phase (f > 0.5, FluidGridCPU.cpp:1321-1322). */
void or_grid_set_air(or_grid* grid, const unsigned char* air);
void or_air_mask(int cells, const double* fraction, const unsigned char* solid, unsigned char* air);

/* Upload: density per cell, face velocities and pressure (null = zero). Resets the warm-start
 * history to the uploaded pressure, like FluidGridCPU::upload. */
void or_grid_upload(or_grid* grid, const double* density, const double* u, const double* v, const double* pressure);
void or_grid_download(const or_grid* grid, double* u, double* v, double* pressure);

/* v += g*dt on interior horizontal faces (FluidGridCPU::applyGravity). */
void or_grid_apply_gravity(or_grid* grid, double gravity, double dt);

/* One projection (FluidGridCPU::project). Stop rule: when relative_tolerance > 0, the L2 rule
 * ||r|| <= relative_tolerance * ||b|| is used, else the reference's max-norm rule
 * max |r| <= divergence_tolerance * dx^2 / dt. */
or_result or_grid_project(
    or_grid* grid, double dt, int max_iterations, double divergence_tolerance, double relative_tolerance);
double or_grid_max_divergence(const or_grid* grid);

/* Stand-alone pieces, used by the unit tests. */
void or_density(int cells, int components, const double* const* masses, double cell_size, double* density);
void or_coefficients(int width, int height, const double* density, double* inv_u, double* inv_v, double* inv_diagonal);
void or_diagonal(int width, int height, const double* inv_u, const double* inv_v, double* inv_diagonal);
double or_operator(int width, int height, const double* inv_u, const double* inv_v, const double* x, double* y);
void or_rhs(int width, int height, double cell_size, double dt, double* u, double* v, double* rhs);
void or_face_flags(int width, int height, const unsigned char* solid, double* inv_u, double* inv_v);
void or_classify(int cells, const double* fraction, const unsigned char* solid, unsigned char* mask);

/* Multigrid preconditioner (PressureMultigrid). */
or_mg* or_mg_create(int width, int height);
void or_mg_destroy(or_mg* mg);
int or_mg_levels(const or_mg* mg);
void or_mg_set_sweeps(or_mg* mg, int pre, int post);
void or_grid_set_sweeps(or_grid* grid, int pre, int post);
int or_mg_rebuild(or_mg* mg, const double* inv_u, const double* inv_v); /* 1 ok, 0 breakdown */
void or_mg_apply(or_mg* mg, const double* residual, double* correction, double residual_mean);

/* Semi-Lagrangian transport on the reference's staggered bilinear sampler
 * (FluidGridCPU.cpp:67-90, 465-471). s = dt / cell_size. u_out, v_out and out[k] must not alias
 * the inputs. Wall-normal boundary faces are written as zero. */
double or_sample_scalar(const double* data, int width, int height, double x, double y);
void or_sample_velocity(int width, int height, double cell_size, double origin_x, double origin_y, const double* u,
    const double* v, int count, const double* positions, double* velocities);
void or_advect(int width, int height, double s, const double* u, const double* v, int fields,
    const double* const* in, double* const* out, double* u_out, double* v_out);

/* Implicit viscosity restated in FP64 (UniformWebGPU/ViscosityKernels.h,
 * UniformWebGPU/ViscositySolverGPU.cpp). Node fields hold 2 values per node of the
 * (w+1) x (h+1) lattice: u face p and v face p. */
typedef struct or_visc or_visc;
or_visc* or_visc_create(int width, int height);
void or_visc_destroy(or_visc* solver);
int or_visc_levels(const or_visc* solver);
void or_visc_setup(or_visc* solver, const double* material, double dt, double cell_size);
void or_visc_apply(or_visc* solver, int level, double dt, const double* field, double* out);
void or_visc_precondition(or_visc* solver, const double* residual, double* correction);
int or_visc_solve(or_visc* solver, double* u, double* v, const double* material, double dt, double cell_size,
    double tolerance, int max_iterations, double* relative_residual);
void or_visc_material(int cells, int components, const double* const* masses, const double* densities,
    const double* viscosities, double cell_size, double* material);

#ifdef __cplusplus
}
#endif
#endif
