/*
 * CPU restatement of the FluidSim UniformCPU pressure projection (FP64, single thread).
 *
 * TEST INFRASTRUCTURE ONLY: the parity oracle for the CUDA backend. Only tests/, the smoke
 * check and the cpu_baseline leg of bench.py load it. Each function names the reference
 * code it follows (paths inside the FluidSim project).
 *
 * Additions that have no reference counterpart (solid obstacle cells, the L2 stop rule,
 * the cell classification mask) are marked as such; with no solid cells and the max-norm
 * rule the arithmetic is the reference's.
 */
#include "fluid_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define OR_MAX_LEVELS 16

/* ------------------------------------------------------------------------------------------ */
/* Materials and coefficients                                                                  */
/* ------------------------------------------------------------------------------------------ */

/* Density = total component mass / cell area. FluidGridCPU.cpp:1399-1423 (rebuildDensity). */
void or_density(int cells, int components, const double* const* masses, double cell_size, double* density)
{
    const double inverse_area = 1.0 / (cell_size * cell_size);
    for (int i = 0; i < cells; ++i)
    {
        double total = 0.0;
        for (int k = 0; k < components; ++k)
            total += masses[k][i];
        density[i] = total * inverse_area;
    }
}

/* Face weights 2/(rho_a + rho_b), zero on the four walls, and the inverse diagonal.
 * FluidGridCPU.cpp:1154-1205 (rebuildPressureCoefficients). u faces are (w+1) x h, row-major
 * with index y*(w+1)+x; v faces are w x (h+1) with index y*w+x. */
void or_coefficients(int w, int h, const double* rho, double* inv_u, double* inv_v, double* inv_diagonal)
{
    for (int y = 0; y < h; ++y)
    {
        double* hu = inv_u + (size_t)y * (w + 1);
        hu[0] = 0.0;
        hu[w] = 0.0;
        for (int x = 1; x < w; ++x)
            hu[x] = 2.0 / (rho[y * w + x - 1] + rho[y * w + x]);
        for (int x = 0; x < w; ++x)
            inv_v[(size_t)y * w + x] = y == 0 ? 0.0 : 2.0 / (rho[(y - 1) * w + x] + rho[y * w + x]);
    }
    for (int x = 0; x < w; ++x)
        inv_v[(size_t)h * w + x] = 0.0;

    if (!inv_diagonal)
        return;
    for (int y = 0; y < h; ++y)
    {
        for (int x = 0; x < w; ++x)
        {
            const double sum = inv_u[(size_t)y * (w + 1) + x] + inv_u[(size_t)y * (w + 1) + x + 1] +
                               inv_v[(size_t)y * w + x] + inv_v[(size_t)(y + 1) * w + x];
            inv_diagonal[(size_t)y * w + x] = sum > 0.0 ? 1.0 / sum : 0.0;
        }
    }
}

/* Inverse diagonal from face weights (the second pass of FluidGridCPU.cpp:1188-1202). */
void or_diagonal(int w, int h, const double* inv_u, const double* inv_v, double* inv_diagonal)
{
    for (int y = 0; y < h; ++y)
    {
        for (int x = 0; x < w; ++x)
        {
            const double sum = inv_u[(size_t)y * (w + 1) + x] + inv_u[(size_t)y * (w + 1) + x + 1] +
                               inv_v[(size_t)y * w + x] + inv_v[(size_t)(y + 1) * w + x];
            inv_diagonal[(size_t)y * w + x] = sum > 0.0 ? 1.0 / sum : 0.0;
        }
    }
}

/* Solid obstacle cells close their four faces, as the reference closes its outer walls
 * (FluidGridCPU.cpp:1170-1185). No reference counterpart: the reference has no obstacles. */
void or_face_flags(int w, int h, const unsigned char* solid, double* inv_u, double* inv_v)
{
    if (!solid)
        return;
    for (int y = 0; y < h; ++y)
    {
        for (int x = 0; x < w; ++x)
        {
            if (!solid[y * w + x])
                continue;
            inv_u[(size_t)y * (w + 1) + x] = 0.0;
            inv_u[(size_t)y * (w + 1) + x + 1] = 0.0;
            inv_v[(size_t)y * w + x] = 0.0;
            inv_v[(size_t)(y + 1) * w + x] = 0.0;
        }
    }
}

/* Cell classes from the reference thresholds: liquid phase f > 0.5 (FluidGridCPU.cpp:1321-1322),
 * interface 0 < f < 1 (FluidGridCPU.cpp:531-533); solid from the obstacle mask (no reference
 * counterpart). Bits: 1 liquid, 2 interface, 4 solid; a solid cell carries only bit 4. */
void or_classify(int cells, const double* f, const unsigned char* solid, unsigned char* mask)
{
    for (int i = 0; i < cells; ++i)
    {
        if (solid && solid[i])
        {
            mask[i] = 4;
            continue;
        }
        unsigned char m = 0;
        if (f[i] > 0.5)
            m |= 1;
        if (f[i] > 0.0 && f[i] < 1.0)
            m |= 2;
        mask[i] = m;
    }
}

/* (A x)_i = sum over the cell's faces of weight * (x_i - x_neighbour); returns x . Ax.
 * FluidGridCPU.cpp:1507-1598 (applyPressureOperator); same pairing of the four terms. */
double or_operator(int w, int h, const double* inv_u, const double* inv_v, const double* x, double* y)
{
    double dot = 0.0;
    for (int j = 0; j < h; ++j)
    {
        for (int i = 0; i < w; ++i)
        {
            const int c = j * w + i;
            const double center = x[c];
            const double wl = inv_u[(size_t)j * (w + 1) + i];
            const double wr = inv_u[(size_t)j * (w + 1) + i + 1];
            const double wu = inv_v[(size_t)j * w + i];
            const double wd = inv_v[(size_t)(j + 1) * w + i];
            const double xl = i > 0 ? x[c - 1] : center;
            const double xr = i + 1 < w ? x[c + 1] : center;
            const double xu = j > 0 ? x[c - w] : center;
            const double xd = j + 1 < h ? x[c + w] : center;
            const double value = (wl * (center - xl) + wr * (center - xr)) + (wu * (center - xu) + wd * (center - xd));
            y[c] = value;
            dot += center * value;
        }
    }
    return dot;
}

/* Zero the wall normal velocities and form b = -(du + dv)/dx * dx^2/dt (not yet mean-free).
 * FluidGridCPU.cpp:1050-1083. */
void or_rhs(int w, int h, double dx, double dt, double* u, double* v, double* b)
{
    const double scale = dx * dx / dt;
    for (int y = 0; y < h; ++y)
    {
        u[(size_t)y * (w + 1)] = 0.0;
        u[(size_t)y * (w + 1) + w] = 0.0;
    }
    for (int x = 0; x < w; ++x)
    {
        v[x] = 0.0;
        v[(size_t)h * w + x] = 0.0;
    }
    for (int y = 0; y < h; ++y)
    {
        for (int x = 0; x < w; ++x)
        {
            const double du = u[(size_t)y * (w + 1) + x + 1] - u[(size_t)y * (w + 1) + x];
            const double dv = v[(size_t)(y + 1) * w + x] - v[(size_t)y * w + x];
            b[y * w + x] = -(du + dv) / dx * scale;
        }
    }
}

/* ------------------------------------------------------------------------------------------ */
/* Multigrid preconditioner: PressureMultigrid.cpp                                              */
/* ------------------------------------------------------------------------------------------ */

typedef struct
{
    int first, second;
    double weight; /* weight of `second`; `first` gets 1 - weight */
} or_interp;

typedef struct
{
    int count;
    int index[4];
    double weight[4];
} or_gather;

typedef struct
{
    int w, h, s; /* s = w + 2: one zero halo cell on every side */
    double *cx, *cy;
    double *right, *down, *invd, *rhs, *sol, *res;
    or_interp *px, *py;  /* fine cell -> two coarse cells (used on the fine level) */
    or_gather *rx, *ry;  /* coarse cell -> fine cells: the transpose of px, py */
} or_level;

struct or_mg
{
    int pre_sweeps, post_sweeps; /* 4 and 4 in the reference (PressureMultigrid.cpp:396) */
    /* Dirichlet air (no reference counterpart): cells of `air` hold p = 0 on the fine level;
     * a coarse cell is held at zero when none of its fine cells is an unknown. Not owned. */
    int dirichlet;
    const unsigned char* air;
    int count;
    or_level* lev;
    int n;          /* coarsest unknowns: open cells - 1 (one pinned) */
    int pinned;     /* the pinned cell, -1 when no cell is open */
    int* map;       /* coarsest cell -> unknown index, -1 when pinned or closed */
    double* factor; /* dense n x n Cholesky factor, lower triangle */
    double* work;
};

/* Level geometry; cell centres with a shorter last cell on odd sizes. PressureMultigrid.cpp:24-36. */
static void level_init(or_level* l, int w, int h, int spacing, int domain_w, int domain_h)
{
    memset(l, 0, sizeof(*l));
    l->w = w;
    l->h = h;
    l->s = w + 2;
    const size_t count = (size_t)l->s * (h + 2);
    double** arrays[] = {&l->right, &l->down, &l->invd, &l->rhs, &l->sol, &l->res};
    for (int a = 0; a < 6; ++a)
        *arrays[a] = (double*)calloc(count, sizeof(double));
    l->cx = (double*)calloc(w, sizeof(double));
    l->cy = (double*)calloc(h, sizeof(double));
    for (int x = 0; x < w; ++x)
    {
        const int end = (x + 1) * spacing < domain_w ? (x + 1) * spacing : domain_w;
        l->cx[x] = 0.5 * (x * spacing + end);
    }
    for (int y = 0; y < h; ++y)
    {
        const int end = (y + 1) * spacing < domain_h ? (y + 1) * spacing : domain_h;
        l->cy[y] = 0.5 * (y * spacing + end);
    }
}

/* Linear interpolation between the two nearest coarse centres, clamped at the ends; the
 * restriction is its exact transpose. PressureMultigrid.cpp:64-102 (buildTransfers). */
static void build_axis(int nf, const double* fc, int nc, const double* cc, or_interp* p, or_gather* r)
{
    for (int c = 0; c < nc; ++c)
        r[c].count = 0;
    for (int f = 0; f < nf; ++f)
    {
        const int parent = f / 2;
        int first = parent - (fc[f] < cc[parent] ? 1 : 0);
        if (first < 0)
            first = 0;
        const int second = first + 1 < nc ? first + 1 : nc - 1;
        double weight = 0.0;
        if (first != second)
        {
            weight = (fc[f] - cc[first]) / (cc[second] - cc[first]);
            weight = weight < 0.0 ? 0.0 : (weight > 1.0 ? 1.0 : weight);
        }
        p[f].first = first;
        p[f].second = second;
        p[f].weight = weight;
        const int targets[2] = {first, second};
        const double values[2] = {1.0 - weight, weight};
        for (int k = 0; k < 2; ++k)
        {
            if (values[k] == 0.0)
                continue;
            or_gather* g = &r[targets[k]];
            g->index[g->count] = f;
            g->weight[g->count] = values[k];
            g->count++;
        }
    }
}

/* Halve (rounding up) until the level has at most 64 cells. PressureMultigrid.cpp:38-62. */
or_mg* or_mg_create(int width, int height)
{
    or_mg* mg = (or_mg*)calloc(1, sizeof(or_mg));
    mg->pre_sweeps = 4;
    mg->post_sweeps = 4;
    int w = width, h = height, spacing = 1, count = 0, cap = 4;
    mg->lev = (or_level*)calloc(cap, sizeof(or_level));
    for (;;)
    {
        if (count == cap)
        {
            cap *= 2;
            mg->lev = (or_level*)realloc(mg->lev, cap * sizeof(or_level));
        }
        level_init(&mg->lev[count++], w, h, spacing, width, height);
        if (w * h <= 64)
            break;
        w = (w + 1) / 2;
        h = (h + 1) / 2;
        spacing *= 2;
    }
    mg->count = count;
    for (int i = 0; i + 1 < count; ++i)
    {
        or_level* f = &mg->lev[i];
        or_level* c = &mg->lev[i + 1];
        f->px = (or_interp*)calloc(f->w, sizeof(or_interp));
        f->py = (or_interp*)calloc(f->h, sizeof(or_interp));
        f->rx = (or_gather*)calloc(c->w, sizeof(or_gather));
        f->ry = (or_gather*)calloc(c->h, sizeof(or_gather));
        build_axis(f->w, f->cx, c->w, c->cx, f->px, f->rx);
        build_axis(f->h, f->cy, c->h, c->cy, f->py, f->ry);
    }
    const or_level* last = &mg->lev[count - 1];
    const int cells = last->w * last->h;
    mg->n = cells - 1;
    mg->map = (int*)calloc(cells, sizeof(int));
    mg->factor = (double*)calloc((size_t)cells * cells, sizeof(double));
    mg->work = (double*)calloc(cells, sizeof(double));
    return mg;
}

void or_mg_destroy(or_mg* mg)
{
    if (!mg)
        return;
    for (int i = 0; i < mg->count; ++i)
    {
        or_level* l = &mg->lev[i];
        free(l->right), free(l->down), free(l->invd), free(l->rhs), free(l->sol), free(l->res);
        free(l->cx), free(l->cy), free(l->px), free(l->py), free(l->rx), free(l->ry);
    }
    free(mg->lev);
    free(mg->map);
    free(mg->factor);
    free(mg->work);
    free(mg);
}

int or_mg_levels(const or_mg* mg) { return mg->count; }

/* Sweep counts of the V-cycle (the reference's 4 and 4 by default); at least one pre-sweep. */
void or_mg_set_sweeps(or_mg* mg, int pre, int post)
{
    mg->pre_sweeps = pre < 1 ? 1 : pre;
    mg->post_sweeps = post < 0 ? 0 : post;
}

/* PressureMultigrid.cpp:104-117 (rebuildDiagonal). */
static void level_diagonal(or_level* l)
{
    for (int y = 0; y < l->h; ++y)
    {
        for (int x = 0; x < l->w; ++x)
        {
            const int i = (y + 1) * l->s + x + 1;
            const double d = l->right[i - 1] + l->right[i] + l->down[i - l->s] + l->down[i];
            l->invd[i] = d > 0.0 ? 1.0 / d : 0.0;
        }
    }
}

/* Coarse conductances: fine faces crossing a coarse face add in parallel; along the path
 * between coarse centres each crossed fine face adds in series, weighted by the fraction of
 * the fine spacing that the path covers. PressureMultigrid.cpp:142-202 (coarsen). */
static void level_coarsen(const or_level* f, or_level* c)
{
    for (int y = 0; y < c->h; ++y)
    {
        for (int x = 0; x + 1 < c->w; ++x)
        {
            const int e = 2 * x + 2;
            const double a = (f->cx[e - 1] - c->cx[x]) / (f->cx[e - 1] - f->cx[e - 2]);
            const double b = e + 1 < f->w ? (c->cx[x + 1] - f->cx[e]) / (f->cx[e + 1] - f->cx[e]) : 0.0;
            double g = 0.0;
            const int fy_end = 2 * y + 2 < f->h ? 2 * y + 2 : f->h;
            for (int fy = 2 * y; fy < fy_end; ++fy)
            {
                const int i = (fy + 1) * f->s + e;
                double resistance = a / f->right[i - 1] + 1.0 / f->right[i];
                if (b != 0.0)
                    resistance += b / f->right[i + 1];
                g += 1.0 / resistance;
            }
            c->right[(y + 1) * c->s + x + 1] = g;
        }
    }
    for (int y = 0; y + 1 < c->h; ++y)
    {
        for (int x = 0; x < c->w; ++x)
        {
            const int e = 2 * y + 2;
            const double a = (f->cy[e - 1] - c->cy[y]) / (f->cy[e - 1] - f->cy[e - 2]);
            const double b = e + 1 < f->h ? (c->cy[y + 1] - f->cy[e]) / (f->cy[e + 1] - f->cy[e]) : 0.0;
            double g = 0.0;
            const int fx_end = 2 * x + 2 < f->w ? 2 * x + 2 : f->w;
            for (int fx = 2 * x; fx < fx_end; ++fx)
            {
                const int i = e * f->s + fx + 1;
                double resistance = a / f->down[i - f->s] + 1.0 / f->down[i];
                if (b != 0.0)
                    resistance += b / f->down[i + f->s];
                g += 1.0 / resistance;
            }
            c->down[(y + 1) * c->s + x + 1] = g;
        }
    }
    level_diagonal(c);
}

/* Dirichlet air: a coarse cell none of whose fine cells is an unknown (inverse diagonal > 0)
 * is held at zero, like the air cells it covers; its faces to the unknowns stay in their
 * diagonals, which is the p = 0 boundary seen from the coarse level. No reference counterpart. */
static void level_fix(const or_level* f, or_level* c)
{
    for (int y = 0; y < c->h; ++y)
    {
        for (int x = 0; x < c->w; ++x)
        {
            int unknown = 0;
            for (int dy = 0; dy < 2; ++dy)
                for (int dx = 0; dx < 2; ++dx)
                {
                    const int fx = 2 * x + dx, fy = 2 * y + dy;
                    if (fx < f->w && fy < f->h && f->invd[(fy + 1) * f->s + fx + 1] > 0.0)
                        unknown = 1;
                }
            if (!unknown)
                c->invd[(y + 1) * c->s + x + 1] = 0.0;
        }
    }
}

/* Dense Cholesky of the coarsest operator with one cell pinned to zero.
 * PressureMultigrid.cpp:300-345 (factorCoarsest). The reference pins cell 0; here the pinned
 * cell is the first cell with an open face and cells without one (inside obstacles) are left
 * out of the system, which is the same system when no cell is closed. Returns 0 on a
 * non-positive pivot. */
static int factor_coarsest(or_mg* mg)
{
    const or_level* l = &mg->lev[mg->count - 1];
    const int cells = l->w * l->h;
    int* map = mg->map;
    int n = 0;
    mg->pinned = -1;
    for (int cell = 0; cell < cells; ++cell)
    {
        const int x = cell % l->w, y = cell / l->w;
        const int i = (y + 1) * l->s + x + 1;
        const double diag = l->right[i - 1] + l->right[i] + l->down[i - l->s] + l->down[i];
        map[cell] = -1;
        if (!(diag > 0.0))
            continue;
        if (mg->dirichlet)
        {
            /* Dirichlet air: the held cells leave the system and nothing is pinned. */
            if (l->invd[i] > 0.0)
                map[cell] = n++;
        }
        else if (mg->pinned < 0)
            mg->pinned = cell;
        else
            map[cell] = n++;
    }
    mg->n = n;
    double* a = mg->factor;
    if (n <= 0)
        return 1;
    memset(a, 0, sizeof(double) * (size_t)n * n);
    for (int cell = 0; cell < cells; ++cell)
    {
        const int row = map[cell];
        if (row < 0)
            continue;
        const int x = cell % l->w, y = cell / l->w;
        const int i = (y + 1) * l->s + x + 1;
        a[row * n + row] = l->right[i - 1] + l->right[i] + l->down[i - l->s] + l->down[i];
        if (x > 0 && map[cell - 1] >= 0)
            a[row * n + map[cell - 1]] = -l->right[i - 1];
        if (y > 0 && map[cell - l->w] >= 0)
            a[row * n + map[cell - l->w]] = -l->down[i - l->s];
    }
    for (int row = 0; row < n; ++row)
    {
        for (int col = 0; col <= row; ++col)
        {
            double value = a[row * n + col];
            for (int k = 0; k < col; ++k)
                value -= a[row * n + k] * a[col * n + k];
            if (row == col)
            {
                if (!(value > 0.0) || !isfinite(value))
                    return 0;
                a[row * n + col] = sqrt(value);
            }
            else
                a[row * n + col] = value / a[col * n + col];
        }
    }
    return 1;
}

/* PressureMultigrid.cpp:119-140 (rebuild). */
int or_mg_rebuild(or_mg* mg, const double* inv_u, const double* inv_v)
{
    or_level* f = &mg->lev[0];
    for (int y = 0; y < f->h; ++y)
    {
        for (int x = 0; x < f->w; ++x)
        {
            const int i = (y + 1) * f->s + x + 1;
            f->right[i] = inv_u[(size_t)y * (f->w + 1) + x + 1];
            f->down[i] = inv_v[(size_t)(y + 1) * f->w + x];
        }
    }
    level_diagonal(f);
    if (mg->dirichlet && mg->air)
        for (int y = 0; y < f->h; ++y)
            for (int x = 0; x < f->w; ++x)
                if (mg->air[y * f->w + x])
                    f->invd[(y + 1) * f->s + x + 1] = 0.0;
    for (int i = 0; i + 1 < mg->count; ++i)
    {
        level_coarsen(&mg->lev[i], &mg->lev[i + 1]);
        if (mg->dirichlet)
            level_fix(&mg->lev[i], &mg->lev[i + 1]);
    }
    return factor_coarsest(mg);
}

/* One red-black Gauss-Seidel sweep: colour (x + y) & 1 == c is updated from the other
 * colour; `reverse` runs colour 1 first; `from_zero` treats the first colour's neighbours as
 * zero. PressureMultigrid.cpp:204-231 (smooth). */
static void level_smooth(or_level* l, int reverse, int from_zero)
{
    const int s = l->s;
    for (int pass = 0; pass < 2; ++pass)
    {
        const int colour = reverse ? 1 - pass : pass;
        for (int y = 0; y < l->h; ++y)
        {
            for (int x = (colour ^ (y & 1)); x < l->w; x += 2)
            {
                const int i = (y + 1) * s + x + 1;
                double value = l->rhs[i];
                if (!(from_zero && pass == 0))
                    value += (l->right[i - 1] * l->sol[i - 1] + l->right[i] * l->sol[i + 1]) +
                             (l->down[i - s] * l->sol[i - s] + l->down[i] * l->sol[i + s]);
                l->sol[i] = value * l->invd[i];
            }
        }
    }
}

/* Fine residual, then its transpose-interpolation onto the coarse rhs.
 * PressureMultigrid.cpp:233-276 (restrictResidual). */
static void level_restrict(or_level* f, or_level* c)
{
    const int s = f->s;
    for (int y = 0; y < f->h; ++y)
    {
        for (int x = 0; x < f->w; ++x)
        {
            const int i = (y + 1) * s + x + 1;
            const double center = f->sol[i];
            const double product = (f->right[i - 1] * (center - f->sol[i - 1]) + f->right[i] * (center - f->sol[i + 1])) +
                                   (f->down[i - s] * (center - f->sol[i - s]) + f->down[i] * (center - f->sol[i + s]));
            /* A cell without an open face (possible only inside obstacles) passes no residual
             * down, which keeps the cycle symmetric; otherwise this is the reference's residual. */
            f->res[i] = f->invd[i] > 0.0 ? f->rhs[i] - product : 0.0;
        }
    }
    for (int y = 0; y < c->h; ++y)
    {
        for (int x = 0; x < c->w; ++x)
        {
            const or_gather* gx = &f->rx[x];
            const or_gather* gy = &f->ry[y];
            double value = 0.0;
            for (int j = 0; j < gy->count; ++j)
            {
                const double* row = f->res + (size_t)(gy->index[j] + 1) * s + 1;
                double line = 0.0;
                for (int k = 0; k < gx->count; ++k)
                    line += gx->weight[k] * row[gx->index[k]];
                value += gy->weight[j] * line;
            }
            c->rhs[(y + 1) * c->s + x + 1] = value;
        }
    }
}

/* Bilinear interpolation of the coarse correction, added to the fine solution.
 * PressureMultigrid.cpp:278-298 (prolongCorrection). */
static void level_prolong(const or_level* c, or_level* f, int dirichlet)
{
    for (int y = 0; y < f->h; ++y)
    {
        const or_interp* py = &f->py[y];
        const double* top = c->sol + (size_t)(py->first + 1) * c->s + 1;
        const double* bottom = c->sol + (size_t)(py->second + 1) * c->s + 1;
        for (int x = 0; x < f->w; ++x)
        {
            const or_interp* px = &f->px[x];
            const double a = (1.0 - px->weight) * top[px->first] + px->weight * top[px->second];
            const double b = (1.0 - px->weight) * bottom[px->first] + px->weight * bottom[px->second];
            f->sol[(y + 1) * f->s + x + 1] += (1.0 - py->weight) * a + py->weight * b;
            /* Dirichlet air: cells held at zero stay at zero (the prolongation is masked, and the
             * restriction, which passes no residual from them, is its transpose). */
            if (dirichlet && !(f->invd[(y + 1) * f->s + x + 1] > 0.0))
                f->sol[(y + 1) * f->s + x + 1] = 0.0;
        }
    }
}

/* Forward/back substitution on the mean-free coarse rhs, then a mean-zero gauge.
 * PressureMultigrid.cpp:347-384 (solveCoarsest); means run over the open cells. */
static void solve_coarsest(or_mg* mg)
{
    or_level* l = &mg->lev[mg->count - 1];
    const int n = mg->n, cells = l->w * l->h;
    const double* a = mg->factor;
    double* z = mg->work;
    double mean = 0.0;
    int open = 0;
    for (int cell = 0; cell < cells; ++cell)
    {
        if (cell != mg->pinned && mg->map[cell] < 0)
            continue;
        mean += l->rhs[(cell / l->w + 1) * l->s + cell % l->w + 1];
        ++open;
    }
    for (int cell = 0; cell < cells; ++cell)
        l->sol[(cell / l->w + 1) * l->s + cell % l->w + 1] = 0.0;
    if (open == 0)
        return;
    /* Dirichlet air: a non-singular system, solved as it stands (no mean, no gauge). */
    mean = mg->dirichlet ? 0.0 : mean / open;
    for (int cell = 0; cell < cells; ++cell)
    {
        const int row = mg->map[cell];
        if (row < 0)
            continue;
        double value = l->rhs[(cell / l->w + 1) * l->s + cell % l->w + 1] - mean;
        for (int col = 0; col < row; ++col)
            value -= a[row * n + col] * z[col];
        z[row] = value / a[row * n + row];
    }
    for (int row = n - 1; row >= 0; --row)
    {
        double value = z[row];
        for (int col = row + 1; col < n; ++col)
            value -= a[col * n + row] * z[col];
        z[row] = value / a[row * n + row];
    }
    double sum = 0.0;
    for (int k = 0; k < n; ++k)
        sum += z[k];
    mean = mg->dirichlet ? 0.0 : sum / open;
    if (mg->pinned >= 0)
        l->sol[(mg->pinned / l->w + 1) * l->s + mg->pinned % l->w + 1] = -mean;
    for (int cell = 0; cell < cells; ++cell)
        if (mg->map[cell] >= 0)
            l->sol[(cell / l->w + 1) * l->s + cell % l->w + 1] = z[mg->map[cell]] - mean;
}

/* Four pre-sweeps (the first from zero), restrict, recurse, prolong, four post-sweeps in the
 * reversed colour order. PressureMultigrid.cpp:386-408 (cycle). */
static void mg_cycle(or_mg* mg, int index)
{
    if (index + 1 == mg->count)
    {
        solve_coarsest(mg);
        return;
    }
    or_level* f = &mg->lev[index];
    or_level* c = &mg->lev[index + 1];
    level_smooth(f, 0, 1);
    for (int sweep = 1; sweep < mg->pre_sweeps; ++sweep)
        level_smooth(f, 0, 0);
    level_restrict(f, c);
    mg_cycle(mg, index + 1);
    level_prolong(c, f, mg->dirichlet);
    for (int sweep = 0; sweep < mg->post_sweeps; ++sweep)
        level_smooth(f, 1, 0);
}

/* PressureMultigrid.cpp:410-434 (apply). */
void or_mg_apply(or_mg* mg, const double* residual, double* correction, double residual_mean)
{
    or_level* f = &mg->lev[0];
    /* Cells without an open face (inside obstacles) take no part; with none closed this is
     * the reference's rhs = residual - mean. */
    for (int y = 0; y < f->h; ++y)
        for (int x = 0; x < f->w; ++x)
        {
            const int i = (y + 1) * f->s + x + 1;
            f->rhs[i] = f->invd[i] > 0.0 ? residual[y * f->w + x] - residual_mean : 0.0;
        }
    mg_cycle(mg, 0);
    for (int y = 0; y < f->h; ++y)
        memcpy(correction + (size_t)y * f->w, f->sol + (size_t)(y + 1) * f->s + 1, sizeof(double) * f->w);
}

/* ------------------------------------------------------------------------------------------ */
/* Grid and projection: FluidGridCPU.cpp                                                        */
/* ------------------------------------------------------------------------------------------ */

struct or_grid
{
    int w, h, n;
    int open;              /* cells outside obstacles */
    unsigned char* solid;  /* obstacle mask or NULL (no reference counterpart) */
    unsigned char* air;    /* Dirichlet air cells (p = 0) or NULL: the gas model (no reference counterpart) */
    double dx;
    int preconditioner;
    double *density, *u, *v, *p, *p_prev;
    double *inv_u, *inv_v, *inv_diag;
    double *b, *r, *z, *d, *q;
    or_mg* mg;
    int mg_valid;
};

or_grid* or_grid_create(int width, int height, double cell_size)
{
    or_grid* g = (or_grid*)calloc(1, sizeof(or_grid));
    g->w = width;
    g->h = height;
    g->n = width * height;
    g->dx = cell_size;
    g->open = g->n;
    g->preconditioner = OR_PRECONDITIONER_MULTIGRID;
    const size_t n = (size_t)g->n, nu = (size_t)(width + 1) * height, nv = (size_t)width * (height + 1);
    g->density = (double*)calloc(n, sizeof(double));
    g->u = (double*)calloc(nu, sizeof(double));
    g->v = (double*)calloc(nv, sizeof(double));
    g->p = (double*)calloc(n, sizeof(double));
    g->p_prev = (double*)calloc(n, sizeof(double));
    g->inv_u = (double*)calloc(nu, sizeof(double));
    g->inv_v = (double*)calloc(nv, sizeof(double));
    g->inv_diag = (double*)calloc(n, sizeof(double));
    double** vectors[] = {&g->b, &g->r, &g->z, &g->d, &g->q};
    for (int k = 0; k < 5; ++k)
        *vectors[k] = (double*)calloc(n, sizeof(double));
    g->mg = or_mg_create(width, height);
    return g;
}

/* Dirichlet air: the held cells take no part (inverse diagonal 0); their faces keep their
 * weights, so the unknowns beside them see p = 0. */
static void apply_air(or_grid* g)
{
    if (!g->air)
        return;
    for (int i = 0; i < g->n; ++i)
        if (g->air[i])
            g->inv_diag[i] = 0.0;
    g->mg->dirichlet = 1;
    g->mg->air = g->air;
}

void or_air_mask(int cells, const double* fraction, const unsigned char* solid, unsigned char* air)
{
    for (int i = 0; i < cells; ++i)
        air[i] = !(solid && solid[i]) && !(fraction[i] > 0.5);
}

void or_grid_set_air(or_grid* g, const unsigned char* air)
{
    free(g->air);
    g->air = NULL;
    g->mg->dirichlet = 0;
    g->mg->air = NULL;
    if (air)
    {
        g->air = (unsigned char*)malloc((size_t)g->n);
        for (int i = 0; i < g->n; ++i)
            g->air[i] = air[i] ? 1 : 0;
    }
    or_coefficients(g->w, g->h, g->density, g->inv_u, g->inv_v, g->inv_diag);
    or_face_flags(g->w, g->h, g->solid, g->inv_u, g->inv_v);
    or_diagonal(g->w, g->h, g->inv_u, g->inv_v, g->inv_diag);
    apply_air(g);
    g->mg_valid = 0;
}

void or_grid_set_solid(or_grid* g, const unsigned char* solid)
{
    free(g->solid);
    g->solid = NULL;
    g->open = g->n;
    if (solid)
    {
        g->solid = (unsigned char*)malloc((size_t)g->n);
        g->open = 0;
        for (int i = 0; i < g->n; ++i)
        {
            g->solid[i] = solid[i] ? 1 : 0;
            g->open += !g->solid[i];
        }
    }
    or_coefficients(g->w, g->h, g->density, g->inv_u, g->inv_v, g->inv_diag);
    or_face_flags(g->w, g->h, g->solid, g->inv_u, g->inv_v);
    or_diagonal(g->w, g->h, g->inv_u, g->inv_v, g->inv_diag);
    apply_air(g);
    g->mg_valid = 0;
}

void or_grid_destroy(or_grid* g)
{
    if (!g)
        return;
    free(g->solid);
    free(g->air);
    free(g->density), free(g->u), free(g->v), free(g->p), free(g->p_prev);
    free(g->inv_u), free(g->inv_v), free(g->inv_diag);
    free(g->b), free(g->r), free(g->z), free(g->d), free(g->q);
    or_mg_destroy(g->mg);
    free(g);
}

void or_grid_set_preconditioner(or_grid* g, int which) { g->preconditioner = which; }

void or_grid_set_sweeps(or_grid* g, int pre, int post) { or_mg_set_sweeps(g->mg, pre, post); }

/* FluidGridCPU.cpp:198-254 (upload): fields replaced, history reset, caches invalidated. */
void or_grid_upload(or_grid* g, const double* density, const double* u, const double* v, const double* p)
{
    const size_t n = (size_t)g->n, nu = (size_t)(g->w + 1) * g->h, nv = (size_t)g->w * (g->h + 1);
    if (density)
        memcpy(g->density, density, n * sizeof(double));
    else
        memset(g->density, 0, n * sizeof(double));
    if (u)
        memcpy(g->u, u, nu * sizeof(double));
    else
        memset(g->u, 0, nu * sizeof(double));
    if (v)
        memcpy(g->v, v, nv * sizeof(double));
    else
        memset(g->v, 0, nv * sizeof(double));
    if (p)
        memcpy(g->p, p, n * sizeof(double));
    else
        memset(g->p, 0, n * sizeof(double));
    memcpy(g->p_prev, g->p, n * sizeof(double));
    or_coefficients(g->w, g->h, g->density, g->inv_u, g->inv_v, g->inv_diag);
    if (g->solid)
    {
        or_face_flags(g->w, g->h, g->solid, g->inv_u, g->inv_v);
        or_diagonal(g->w, g->h, g->inv_u, g->inv_v, g->inv_diag);
    }
    apply_air(g);
    g->mg_valid = 0;
}

void or_grid_download(const or_grid* g, double* u, double* v, double* p)
{
    if (u)
        memcpy(u, g->u, (size_t)(g->w + 1) * g->h * sizeof(double));
    if (v)
        memcpy(v, g->v, (size_t)g->w * (g->h + 1) * sizeof(double));
    if (p)
        memcpy(p, g->p, (size_t)g->n * sizeof(double));
}

/* Interior horizontal faces only. FluidGridCPU.cpp:987-996 (applyGravity). */
void or_grid_apply_gravity(or_grid* g, double gravity, double dt)
{
    for (int i = g->w; i < g->w * g->h; ++i)
        g->v[i] += gravity * dt;
}

static double sum_of(const double* x, int n)
{
    double s = 0.0;
    for (int i = 0; i < n; ++i)
        s += x[i];
    return s;
}

/* FluidGridCPU.cpp:1466-1474 (removeMean); obstacle cells are held at zero and excluded. */
static void remove_mean(const or_grid* g, double* x)
{
    if (g->air)
    {
        /* Dirichlet air: a non-singular system; air cells hold zero. */
        for (int i = 0; i < g->n; ++i)
            if (g->air[i] || (g->solid && g->solid[i]))
                x[i] = 0.0;
        return;
    }
    double sum = 0.0;
    for (int i = 0; i < g->n; ++i)
        if (!g->solid || !g->solid[i])
            sum += x[i];
    const double mean = sum / g->open;
    for (int i = 0; i < g->n; ++i)
        x[i] = (g->solid && g->solid[i]) ? 0.0 : x[i] - mean;
}

typedef struct
{
    double sum, max, sumsq;
} or_stats;

static or_stats stats_of(const double* r, int n)
{
    or_stats s = {0.0, 0.0, 0.0};
    for (int i = 0; i < n; ++i)
    {
        s.sum += r[i];
        const double a = fabs(r[i]);
        if (a > s.max)
            s.max = a;
        s.sumsq += r[i] * r[i];
    }
    if (!isfinite(s.sum))
        s.max = INFINITY;
    return s;
}

/* r = b - A p with its stats. FluidGridCPU.cpp:1643-1683 (rebuildPressureResidual). */
static or_stats true_residual(or_grid* g)
{
    or_operator(g->w, g->h, g->inv_u, g->inv_v, g->p, g->q);
    for (int i = 0; i < g->n; ++i)
        g->r[i] = g->air && g->air[i] ? 0.0 : g->b[i] - g->q[i];
    return stats_of(g->r, g->n);
}

/* Preconditioner, then z's mean removed and r . z returned. FluidGridCPU.cpp:1685-1726. */
static double precondition(or_grid* g, double residual_mean)
{
    if (g->preconditioner == OR_PRECONDITIONER_MULTIGRID)
        or_mg_apply(g->mg, g->r, g->z, residual_mean);
    else
        for (int i = 0; i < g->n; ++i)
            g->z[i] = (g->r[i] - residual_mean) * g->inv_diag[i];
    double zsum = 0.0;
    for (int i = 0; i < g->n; ++i)
        if (!g->solid || !g->solid[i])
            zsum += g->z[i];
    const double mean = g->air ? 0.0 : zsum / g->open;
    double dot = 0.0;
    for (int i = 0; i < g->n; ++i)
    {
        g->z[i] = (g->solid && g->solid[i]) ? 0.0 : g->z[i] - mean;
        dot += g->r[i] * g->z[i];
    }
    return dot;
}

static int met(or_stats s, double tol_max, double tol_sumsq)
{
    return s.max <= tol_max && s.sumsq <= tol_sumsq;
}

/* PCG with warm start, lazy preconditioner, restart on drift.
 * FluidGridCPU.cpp:1728-1824 (solvePressure). */
static int solve_pressure(or_grid* g, int max_iterations, double tol_max, double tol_sumsq)
{
    const int n = g->n;
    double bmax = 0.0, bsq = 0.0;
    for (int i = 0; i < n; ++i)
    {
        const double a = isfinite(g->b[i]) ? fabs(g->b[i]) : INFINITY;
        bmax = a > bmax ? a : bmax;
        bsq += g->b[i] * g->b[i];
    }
    if (bmax <= tol_max && bsq <= tol_sumsq)
    {
        memset(g->p, 0, n * sizeof(double));
        memset(g->p_prev, 0, n * sizeof(double));
        return 0;
    }
    for (int i = 0; i < n; ++i)
    {
        const double latest = g->p[i];
        g->p[i] = 2.0 * latest - g->p_prev[i];
        g->p_prev[i] = latest;
    }
    remove_mean(g, g->p);
    or_stats initial = true_residual(g);
    if (met(initial, tol_max, tol_sumsq) || max_iterations == 0)
        return 0;
    if (g->preconditioner == OR_PRECONDITIONER_MULTIGRID && !g->mg_valid)
    {
        g->mg_valid = or_mg_rebuild(g->mg, g->inv_u, g->inv_v);
        if (!g->mg_valid)
            return -1;
    }
    double residual_mean = g->air ? 0.0 : initial.sum / g->open;
    double rz = precondition(g, residual_mean);
    memcpy(g->d, g->z, n * sizeof(double));
    int iterations = 0;
    while (iterations < max_iterations && rz > 0.0 && isfinite(rz))
    {
        const double dq = or_operator(g->w, g->h, g->inv_u, g->inv_v, g->d, g->q);
        if (g->air)
            for (int i = 0; i < n; ++i)
                if (g->air[i])
                    g->q[i] = 0.0; /* air cells are no unknowns: their residual stays zero */
        if (dq <= 0.0 || !isfinite(dq))
            break;
        const double alpha = rz / dq;
        if (!isfinite(alpha))
            break;
        for (int i = 0; i < n; ++i)
        {
            g->p[i] += alpha * g->d[i];
            g->r[i] -= alpha * g->q[i];
        }
        or_stats s = stats_of(g->r, n);
        residual_mean = g->air ? 0.0 : s.sum / g->open;
        ++iterations;
        int restart = 0;
        if (met(s, tol_max, tol_sumsq))
        {
            const or_stats actual = true_residual(g);
            if (met(actual, tol_max, tol_sumsq))
                break;
            residual_mean = g->air ? 0.0 : actual.sum / g->open;
            restart = 1;
        }
        const double next = precondition(g, residual_mean);
        const double beta = restart ? 0.0 : next / rz;
        if (!isfinite(beta))
            break;
        for (int i = 0; i < n; ++i)
            g->d[i] = g->z[i] + beta * g->d[i];
        rz = next;
    }
    remove_mean(g, g->p);
    return iterations;
}

/* FluidGridCPU.cpp:1126-1152 (maxDivergence). */
double or_grid_max_divergence(const or_grid* g)
{
    double maximum = 0.0;
    for (int y = 0; y < g->h; ++y)
    {
        for (int x = 0; x < g->w; ++x)
        {
            /* Dirichlet air: only the liquid is held divergence-free. */
            if (g->air && (g->air[y * g->w + x] || (g->solid && g->solid[y * g->w + x])))
                continue;
            const double div = ((g->u[(size_t)y * (g->w + 1) + x + 1] - g->u[(size_t)y * (g->w + 1) + x]) +
                                   (g->v[(size_t)(y + 1) * g->w + x] - g->v[(size_t)y * g->w + x])) /
                               g->dx;
            if (!isfinite(div))
                return INFINITY;
            if (fabs(div) > maximum)
                maximum = fabs(div);
        }
    }
    return maximum;
}

/* FluidGridCPU.cpp:1030-1124 (project). */
or_result or_grid_project(
    or_grid* g, double dt, int max_iterations, double divergence_tolerance, double relative_tolerance)
{
    or_result result = {0, 0, INFINITY, 0.0, 0.0, 0.0};
    if (dt <= 0.0 || g->w <= 0 || g->h <= 0 || max_iterations < 0)
        return result;
    const int w = g->w, h = g->h, n = g->n;
    const double scale = g->dx * g->dx / dt;
    if (g->solid)
    {
        /* Faces of obstacle cells close like walls (no reference counterpart). */
        for (int y = 0; y < h; ++y)
            for (int x = 0; x < w; ++x)
                if (g->solid[y * w + x])
                {
                    g->u[(size_t)y * (w + 1) + x] = 0.0;
                    g->u[(size_t)y * (w + 1) + x + 1] = 0.0;
                    g->v[(size_t)y * w + x] = 0.0;
                    g->v[(size_t)(y + 1) * w + x] = 0.0;
                }
    }
    or_rhs(w, h, g->dx, dt, g->u, g->v, g->b);
    remove_mean(g, g->b); /* Dirichlet air: b = 0 on air and solid cells, no mean taken */
    double bsq = 0.0;
    for (int i = 0; i < n; ++i)
        bsq += g->b[i] * g->b[i];
    result.rhs_l2 = sqrt(bsq);

    double tol_max = divergence_tolerance * scale, tol_sumsq = INFINITY;
    if (relative_tolerance > 0.0)
    {
        tol_max = INFINITY;
        tol_sumsq = relative_tolerance * relative_tolerance * bsq;
    }
    result.iterations = solve_pressure(g, max_iterations, tol_max, tol_sumsq);
    if (result.iterations < 0)
        return result;

    const or_stats final_residual = true_residual(g);
    result.residual_max = final_residual.max;
    result.residual_l2 = sqrt(final_residual.sumsq);

    /* u -= dp/dx * dt * w on interior faces. FluidGridCPU.cpp:1098-1118. */
    for (int y = 0; y < h; ++y)
    {
        const double* row = g->p + (size_t)y * w;
        for (int x = 1; x < w; ++x)
            g->u[(size_t)y * (w + 1) + x] -= ((row[x] - row[x - 1]) / g->dx) * dt * g->inv_u[(size_t)y * (w + 1) + x];
        if (y == 0)
            continue;
        for (int x = 0; x < w; ++x)
            g->v[(size_t)y * w + x] -= ((row[x] - row[x - w]) / g->dx) * dt * g->inv_v[(size_t)y * w + x];
    }
    result.max_divergence = or_grid_max_divergence(g);
    result.converged = result.max_divergence <= divergence_tolerance;
    return result;
}

/* ------------------------------------------------------------------------------------------ */
/* Semi-Lagrangian transport. The reference has no semi-Lagrangian step (its UniformCPU step   */
/* transports with PLIC, FluidGridCPU.cpp:362-463); this restates the UniformCUDA transport   */
/* on the reference's sampler, FluidGridCPU.cpp:67-90 (sampleScalar) and :465-471            */
/* (sampleVelocity). Compiled without multiply-add contraction, like the device code.         */
/* ------------------------------------------------------------------------------------------ */

/* std::lerp (P0811R3, as libstdc++ implements it): the blend FluidGridCPU.cpp:86-89 uses. */
static double or_lerp(double a, double b, double t)
{
    if ((a <= 0.0 && b >= 0.0) || (a >= 0.0 && b <= 0.0))
        return t * b + (1.0 - t) * a;
    if (t == 1.0)
        return b;
    const double x = a + t * (b - a);
    return ((t > 1.0) == (b > a)) ? (b < x ? x : b) : (b > x ? x : b);
}

/* std::clamp(x, lo, hi), lo <= hi. */
static double or_clamp(double x, double lo, double hi)
{
    const double m = x < lo ? lo : x;
    return hi < m ? hi : m;
}

/* FluidGridCPU.cpp:67-90. */
double or_sample_scalar(const double* data, int w, int h, double x, double y)
{
    x = or_clamp(x, 0.0, (double)(w - 1));
    y = or_clamp(y, 0.0, (double)(h - 1));
    const int x0 = (int)x, y0 = (int)y;
    const int x1 = x0 + 1 < w - 1 ? x0 + 1 : w - 1;
    const int y1 = y0 + 1 < h - 1 ? y0 + 1 : h - 1;
    const double tx = x - x0, ty = y - y0;
    const double a = or_lerp(data[(size_t)y0 * w + x0], data[(size_t)y0 * w + x1], tx);
    const double b = or_lerp(data[(size_t)y1 * w + x0], data[(size_t)y1 * w + x1], tx);
    return or_lerp(a, b, ty);
}

/* FluidGridCPU.cpp:465-471 in cell units. */
static void or_velocity_at(int W, int H, const double* u, const double* v, double x, double y, double* vx, double* vy)
{
    *vx = or_sample_scalar(u, W + 1, H, x, y - 0.5);
    *vy = or_sample_scalar(v, W, H + 1, x - 0.5, y);
}

void or_sample_velocity(int W, int H, double cell_size, double origin_x, double origin_y, const double* u,
    const double* v, int count, const double* positions, double* velocities)
{
    for (int n = 0; n < count; ++n)
    {
        const double x = (positions[2 * n] - origin_x) / cell_size;
        const double y = (positions[2 * n + 1] - origin_y) / cell_size;
        or_velocity_at(W, H, u, v, x, y, velocities + 2 * n, velocities + 2 * n + 1);
    }
}

/* Midpoint back-trace: mid = p - (s/2) V(p), back = p - s V(mid). */
static void or_trace(int W, int H, const double* u, const double* v, double s, double x, double y, double* bx,
    double* by)
{
    const double half = 0.5 * s;
    double vx, vy;
    or_velocity_at(W, H, u, v, x, y, &vx, &vy);
    const double mx = x - half * vx, my = y - half * vy;
    or_velocity_at(W, H, u, v, mx, my, &vx, &vy);
    *bx = x - s * vx;
    *by = y - s * vy;
}

void or_advect(int W, int H, double s, const double* u, const double* v, int fields, const double* const* in,
    double* const* out, double* u_out, double* v_out)
{
    for (int j = 0; j < H; ++j)
        for (int i = 0; i <= W; ++i)
        {
            double value = 0.0;
            if (i > 0 && i < W)
            {
                double bx, by;
                or_trace(W, H, u, v, s, (double)i, j + 0.5, &bx, &by);
                value = or_sample_scalar(u, W + 1, H, bx, by - 0.5);
            }
            u_out[(size_t)j * (W + 1) + i] = value;
        }
    for (int j = 0; j <= H; ++j)
        for (int i = 0; i < W; ++i)
        {
            double value = 0.0;
            if (j > 0 && j < H)
            {
                double bx, by;
                or_trace(W, H, u, v, s, i + 0.5, (double)j, &bx, &by);
                value = or_sample_scalar(v, W, H + 1, bx - 0.5, by);
            }
            v_out[(size_t)j * W + i] = value;
        }
    for (int j = 0; j < H; ++j)
        for (int i = 0; i < W; ++i)
        {
            double bx, by;
            or_trace(W, H, u, v, s, i + 0.5, j + 0.5, &bx, &by);
            for (int k = 0; k < fields; ++k)
                out[k][(size_t)j * W + i] = or_sample_scalar(in[k], W, H, bx - 0.5, by - 0.5);
        }
}

/* ------------------------------------------------------------------------------------------ */
/* Implicit viscosity. The reference solves it only on the GPU (WGSL, FP32); this restates     */
/* its algorithm in FP64:                                                                      */
/*   operator, diagonal, smoother, transfers  UniformWebGPU/ViscosityKernels.h:8-400           */
/*   levels and V-cycle                       UniformWebGPU/ViscositySolverGPU.cpp:61-167      */
/*   CG with the true-residual check          UniformWebGPU/ViscositySolverGPU.cpp:170-294     */
/*   cell viscosity blend                     UniformWebGPU/FluidGridGPU.cpp:172-217, 987-1037 */
/* Fields live on the (w+1) x (h+1) node lattice: node p carries u face p (x component) and   */
/* v face p (y component). Reads outside a field clamp to its edge, as the reference's field   */
/* accessor does.                                                                              */
/* ------------------------------------------------------------------------------------------ */

typedef struct
{
    int w, h;
    double dx;
    double* material; /* 2 per cell: density, viscosity */
    double* coeff;    /* 4 per node: cell mu, vertex mu, u-face mass, v-face mass */
    double *x, *next, *rhs, *res;
} or_vlevel;

struct or_visc
{
    int w, h, levels;
    or_vlevel lev[OR_MAX_LEVELS];
    double *solution, *rhs, *residual, *direction, *product, *truth;
    double dt;
};

static int vclampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

static const double* vmat(const or_vlevel* L, int x, int y)
{
    return L->material + 2 * ((size_t)vclampi(y, 0, L->h - 1) * L->w + vclampi(x, 0, L->w - 1));
}

static const double* vco(const or_vlevel* L, int x, int y)
{
    return L->coeff + 4 * ((size_t)vclampi(y, 0, L->h) * (L->w + 1) + vclampi(x, 0, L->w));
}

static const double* vsrc(const or_vlevel* L, const double* f, int x, int y)
{
    return f + 2 * ((size_t)vclampi(y, 0, L->h) * (L->w + 1) + vclampi(x, 0, L->w));
}

static int valid_u(const or_vlevel* L, int x, int y) { return x > 0 && x < L->w && y < L->h; }
static int valid_v(const or_vlevel* L, int x, int y) { return y > 0 && y < L->h && x < L->w; }

or_visc* or_visc_create(int width, int height)
{
    or_visc* s = (or_visc*)calloc(1, sizeof(or_visc));
    s->w = width;
    s->h = height;
    int w = width, h = height;
    for (;;)
    {
        or_vlevel* L = &s->lev[s->levels++];
        const size_t nodes = (size_t)(w + 1) * (h + 1);
        L->w = w;
        L->h = h;
        L->material = (double*)calloc(2 * (size_t)w * h, sizeof(double));
        L->coeff = (double*)calloc(4 * nodes, sizeof(double));
        L->x = (double*)calloc(2 * nodes, sizeof(double));
        L->next = (double*)calloc(2 * nodes, sizeof(double));
        L->rhs = (double*)calloc(2 * nodes, sizeof(double));
        L->res = (double*)calloc(2 * nodes, sizeof(double));
        if (w * h <= 64 || s->levels == OR_MAX_LEVELS)
            break;
        w = (w + 1) / 2;
        h = (h + 1) / 2;
    }
    const size_t nodes = (size_t)(width + 1) * (height + 1);
    double** v[] = {&s->solution, &s->rhs, &s->residual, &s->direction, &s->product, &s->truth};
    for (int k = 0; k < 6; ++k)
        *v[k] = (double*)calloc(2 * nodes, sizeof(double));
    return s;
}

void or_visc_destroy(or_visc* s)
{
    if (!s)
        return;
    for (int l = 0; l < s->levels; ++l)
    {
        or_vlevel* L = &s->lev[l];
        free(L->material);
        free(L->coeff);
        free(L->x);
        free(L->next);
        free(L->rhs);
        free(L->res);
    }
    double* v[] = {s->solution, s->rhs, s->residual, s->direction, s->product, s->truth};
    for (int k = 0; k < 6; ++k)
        free(v[k]);
    free(s);
}

int or_visc_levels(const or_visc* s) { return s->levels; }

/* Coefficients of one level (ViscosityKernels.h "viscosity coefficients"). */
static void visc_coefficients(or_vlevel* L)
{
    for (int y = 0; y <= L->h; ++y)
        for (int x = 0; x <= L->w; ++x)
        {
            const double* m = vmat(L, x, y);
            double mu = 0.0;
            if (x > 0 && y > 0 && x < L->w && y < L->h)
                mu = 0.25 * (m[1] + vmat(L, x - 1, y)[1] + vmat(L, x, y - 1)[1] + vmat(L, x - 1, y - 1)[1]);
            double* c = L->coeff + 4 * ((size_t)y * (L->w + 1) + x);
            c[0] = m[1];
            c[1] = mu;
            c[2] = 0.5 * L->dx * L->dx * (m[0] + vmat(L, x - 1, y)[0]);
            c[3] = 0.5 * L->dx * L->dx * (m[0] + vmat(L, x, y - 1)[0]);
        }
}

/* 2x2 mean of the existing fine cells (ViscosityKernels.h "viscosity coarse material"). */
static void visc_coarsen(const or_vlevel* F, or_vlevel* C)
{
    for (int y = 0; y < C->h; ++y)
        for (int x = 0; x < C->w; ++x)
        {
            double a = 0.0, b = 0.0, n = 0.0;
            for (int j = 0; j < 2; ++j)
                for (int i = 0; i < 2; ++i)
                {
                    const int qx = 2 * x + i, qy = 2 * y + j;
                    if (qx < F->w && qy < F->h)
                    {
                        a += F->material[2 * ((size_t)qy * F->w + qx)];
                        b += F->material[2 * ((size_t)qy * F->w + qx) + 1];
                        n += 1.0;
                    }
                }
            C->material[2 * ((size_t)y * C->w + x)] = a / n;
            C->material[2 * ((size_t)y * C->w + x) + 1] = b / n;
        }
}

static double shear_at(const or_vlevel* L, const double* f, int x, int y)
{
    return vco(L, x, y)[1] * ((vsrc(L, f, x, y)[0] - vsrc(L, f, x, y - 1)[0]) + (vsrc(L, f, x, y)[1] - vsrc(L, f, x - 1, y)[1]));
}

/* (A f)(p) = mass f(p) + dt * stress(f)(p) on valid faces, zero elsewhere
 * (ViscosityKernels.h "stressProduct" and "product"). */
static void visc_product(const or_vlevel* L, double dt, const double* f, int x, int y, double out[2])
{
    const double* c = vsrc(L, f, x, y);
    const double* a = vco(L, x, y);
    const double t = shear_at(L, f, x, y);
    const double nx = 2.0 * (vco(L, x - 1, y)[0] * (c[0] - vsrc(L, f, x - 1, y)[0]) + a[0] * (c[0] - vsrc(L, f, x + 1, y)[0]));
    const double ny = 2.0 * (vco(L, x, y - 1)[0] * (c[1] - vsrc(L, f, x, y - 1)[1]) + a[0] * (c[1] - vsrc(L, f, x, y + 1)[1]));
    const double sx = nx + (t - shear_at(L, f, x, y + 1));
    const double sy = ny + (t - shear_at(L, f, x + 1, y));
    out[0] = valid_u(L, x, y) ? a[2] * c[0] + dt * sx : 0.0;
    out[1] = valid_v(L, x, y) ? a[3] * c[1] + dt * sy : 0.0;
}

static void visc_diagonal(const or_vlevel* L, double dt, int x, int y, double d[2])
{
    const double* c = vco(L, x, y);
    d[0] = c[2] + dt * (2.0 * (c[0] + vco(L, x - 1, y)[0]) + c[1] + vco(L, x, y + 1)[1]);
    d[1] = c[3] + dt * (2.0 * (c[0] + vco(L, x, y - 1)[0]) + c[1] + vco(L, x + 1, y)[1]);
}

void or_visc_apply(or_visc* s, int level, double dt, const double* f, double* out)
{
    const or_vlevel* L = &s->lev[level];
    for (int y = 0; y <= L->h; ++y)
        for (int x = 0; x <= L->w; ++x)
            visc_product(L, dt, f, x, y, out + 2 * ((size_t)y * (L->w + 1) + x));
}

/* Residual b - A f on valid faces. */
static void visc_residual(const or_vlevel* L, double dt, const double* f, const double* b, double* out)
{
    for (int y = 0; y <= L->h; ++y)
        for (int x = 0; x <= L->w; ++x)
        {
            const size_t i = 2 * ((size_t)y * (L->w + 1) + x);
            double a[2];
            visc_product(L, dt, f, x, y, a);
            out[i] = valid_u(L, x, y) ? b[i] - a[0] : 0.0;
            out[i + 1] = valid_v(L, x, y) ? b[i + 1] - a[1] : 0.0;
        }
}

/* Damped Jacobi x <- x + (b - A x) / (2 D), or b / (2 D) from zero. */
static void visc_smooth(or_vlevel* L, double dt, const double* b, int zero)
{
    for (int y = 0; y <= L->h; ++y)
        for (int x = 0; x <= L->w; ++x)
        {
            const size_t i = 2 * ((size_t)y * (L->w + 1) + x);
            double d[2], a[2] = {0.0, 0.0}, v[2];
            visc_diagonal(L, dt, x, y, d);
            if (zero)
            {
                v[0] = 0.5 * b[i] / d[0];
                v[1] = 0.5 * b[i + 1] / d[1];
            }
            else
            {
                visc_product(L, dt, L->x, x, y, a);
                v[0] = L->x[i] + 0.5 * (b[i] - a[0]) / d[0];
                v[1] = L->x[i + 1] + 0.5 * (b[i + 1] - a[1]) / d[1];
            }
            L->next[i] = valid_u(L, x, y) ? v[0] : 0.0;
            L->next[i + 1] = valid_v(L, x, y) ? v[1] : 0.0;
        }
    double* t = L->x;
    L->x = L->next;
    L->next = t;
}

/* Bilinear transfer between levels on face locations (ViscosityKernels.h transfer). */
static double voffset_x(int component) { return component == 1 ? 0.5 : 0.0; }
static double voffset_y(int component) { return component == 1 ? 0.0 : 0.5; }

static void coarse_point(int bx, int by, int component, int sw, int sh, int* cx, int* cy)
{
    *cx = vclampi(bx, 0, sw - (component == 1 ? 1 : 0));
    *cy = vclampi(by, 0, sh - (component == 1 ? 0 : 1));
}

static double transfer_weight(int fx, int fy, int px, int py, int component, int sw, int sh)
{
    const double lx = (fx + voffset_x(component)) * 0.5 - voffset_x(component);
    const double ly = (fy + voffset_y(component)) * 0.5 - voffset_y(component);
    const int bx = (int)floor(lx), by = (int)floor(ly);
    const double tx = lx - bx, ty = ly - by;
    double result = 0.0;
    for (int y = 0; y < 2; ++y)
        for (int x = 0; x < 2; ++x)
        {
            int cx, cy;
            coarse_point(bx + x, by + y, component, sw, sh, &cx, &cy);
            if (cx == px && cy == py)
                result += (x == 1 ? tx : 1.0 - tx) * (y == 1 ? ty : 1.0 - ty);
        }
    return result;
}

static void visc_restrict(const or_vlevel* F, or_vlevel* C)
{
    for (int py = 0; py <= C->h; ++py)
        for (int px = 0; px <= C->w; ++px)
        {
            double value[2] = {0.0, 0.0};
            for (int component = 0; component < 2; ++component)
            {
                if ((component == 0 && (px == 0 || px == C->w || py == C->h)) ||
                    (component == 1 && (py == 0 || py == C->h || px == C->w)))
                    continue;
                const int ex = component == 1 ? 2 : 1, ey = component == 1 ? 1 : 2;
                for (int y = -1; y <= ey; ++y)
                    for (int x = -1; x <= ex; ++x)
                    {
                        const int qx = 2 * px + x, qy = 2 * py + y;
                        if (qx < 0 || qy < 0 || qx > F->w || qy > F->h)
                            continue;
                        value[component] += transfer_weight(qx, qy, px, py, component, C->w, C->h) *
                                            F->res[2 * ((size_t)qy * (F->w + 1) + qx) + component];
                    }
            }
            C->rhs[2 * ((size_t)py * (C->w + 1) + px)] = value[0];
            C->rhs[2 * ((size_t)py * (C->w + 1) + px) + 1] = value[1];
        }
}

static void visc_prolong(or_vlevel* F, const or_vlevel* C)
{
    for (int py = 0; py <= F->h; ++py)
        for (int px = 0; px <= F->w; ++px)
        {
            const size_t i = 2 * ((size_t)py * (F->w + 1) + px);
            double value[2] = {F->x[i], F->x[i + 1]};
            for (int component = 0; component < 2; ++component)
            {
                const double lx = (px + voffset_x(component)) * 0.5 - voffset_x(component);
                const double ly = (py + voffset_y(component)) * 0.5 - voffset_y(component);
                const int bx = (int)floor(lx), by = (int)floor(ly);
                const double tx = lx - bx, ty = ly - by;
                for (int y = 0; y < 2; ++y)
                    for (int x = 0; x < 2; ++x)
                    {
                        int cx, cy;
                        coarse_point(bx + x, by + y, component, C->w, C->h, &cx, &cy);
                        value[component] += (x == 1 ? tx : 1.0 - tx) * (y == 1 ? ty : 1.0 - ty) *
                                            C->x[2 * ((size_t)cy * (C->w + 1) + cx) + component];
                    }
            }
            F->next[i] = valid_u(F, px, py) ? value[0] : 0.0;
            F->next[i + 1] = valid_v(F, px, py) ? value[1] : 0.0;
        }
    double* t = F->x;
    F->x = F->next;
    F->next = t;
}

/* V-cycle (ViscositySolverGPU.cpp:137-167): two Jacobi sweeps down (the first from zero),
 * residual, restriction, recursion, prolongation, two sweeps up; the coarsest level takes 16
 * Jacobi sweeps from zero. */
static void visc_cycle(or_visc* s, int level, const double* b)
{
    or_vlevel* L = &s->lev[level];
    const double dt = s->dt;
    if (level + 1 == s->levels)
    {
        memset(L->x, 0, 2 * (size_t)(L->w + 1) * (L->h + 1) * sizeof(double));
        for (int sweep = 0; sweep < 16; ++sweep)
            visc_smooth(L, dt, b, 0);
        return;
    }
    visc_smooth(L, dt, b, 1);
    visc_smooth(L, dt, b, 0);
    visc_residual(L, dt, L->x, b, L->res);
    or_vlevel* C = &s->lev[level + 1];
    visc_restrict(L, C);
    visc_cycle(s, level + 1, C->rhs);
    visc_prolong(L, C);
    visc_smooth(L, dt, b, 0);
    visc_smooth(L, dt, b, 0);
}

void or_visc_precondition(or_visc* s, const double* r, double* z)
{
    visc_cycle(s, 0, r);
    memcpy(z, s->lev[0].x, 2 * (size_t)(s->w + 1) * (s->h + 1) * sizeof(double));
}

/* Level materials and coefficients from cell density and viscosity (2 per cell). */
void or_visc_setup(or_visc* s, const double* material, double dt, double cell_size)
{
    s->dt = dt;
    memcpy(s->lev[0].material, material, 2 * (size_t)s->w * s->h * sizeof(double));
    for (int l = 0; l < s->levels; ++l)
    {
        s->lev[l].dx = ldexp(cell_size, l);
        if (l > 0)
            visc_coarsen(&s->lev[l - 1], &s->lev[l]);
        visc_coefficients(&s->lev[l]);
    }
}

/* Sum over nodes of a.a / mass and the other statistics of ViscosityKernels.h "first_reduce". */
static double visc_mass_norm(const or_visc* s, const double* a)
{
    const or_vlevel* L = &s->lev[0];
    double sum = 0.0;
    for (size_t n = 0; n < (size_t)(s->w + 1) * (s->h + 1); ++n)
        sum += a[2 * n] / L->coeff[4 * n + 2] * a[2 * n] + a[2 * n + 1] / L->coeff[4 * n + 3] * a[2 * n + 1];
    return sum;
}

static double visc_dot(const or_visc* s, const double* a, const double* b)
{
    double sum = 0.0;
    for (size_t n = 0; n < 2 * (size_t)(s->w + 1) * (s->h + 1); ++n)
        sum += a[n] * b[n];
    return sum;
}

/* Backward-Euler viscosity solve (ViscositySolverGPU.cpp:170-294). u, v: face velocities (in,
 * out); material: density and viscosity per cell. Returns the iteration count (a multiple of
 * the 4-iteration check interval), -1 on breakdown or non-finite state, -2 when max_iterations
 * (>= 0) is reached without convergence. relative_residual receives sqrt(|r|^2_M / |x0|^2_M). */
int or_visc_solve(or_visc* s, double* u, double* v, const double* material, double dt, double cell_size,
    double tolerance, int max_iterations, double* relative_residual)
{
    const int w = s->w, h = s->h;
    const size_t nodes = (size_t)(w + 1) * (h + 1);
    if (relative_residual)
        *relative_residual = 0.0;
    if (dt <= 0.0)
        return 0;
    or_visc_setup(s, material, dt, cell_size);
    const or_vlevel* L = &s->lev[0];
    /* Pack: solution = velocities on valid faces, rhs = mass * solution. */
    for (int y = 0; y <= h; ++y)
        for (int x = 0; x <= w; ++x)
        {
            const size_t n = (size_t)y * (w + 1) + x;
            s->solution[2 * n] = valid_u(L, x, y) ? u[(size_t)y * (w + 1) + x] : 0.0;
            s->solution[2 * n + 1] = valid_v(L, x, y) ? v[(size_t)y * w + x] : 0.0;
            s->rhs[2 * n] = L->coeff[4 * n + 2] * s->solution[2 * n];
            s->rhs[2 * n + 1] = L->coeff[4 * n + 3] * s->solution[2 * n + 1];
        }
    visc_residual(L, dt, s->solution, s->rhs, s->residual);
    double energy = 0.0, total_mass = 0.0;
    for (size_t n = 0; n < nodes; ++n)
    {
        energy += L->coeff[4 * n + 2] * s->solution[2 * n] * s->solution[2 * n] +
                  L->coeff[4 * n + 3] * s->solution[2 * n + 1] * s->solution[2 * n + 1];
        total_mass += L->coeff[4 * n + 2] + L->coeff[4 * n + 3];
    }
    double rnorm = visc_mass_norm(s, s->residual);
    if (!isfinite(rnorm) || !isfinite(energy) || !isfinite(total_mass))
        return -1;
    const double target = tolerance * tolerance * energy + 1e-12 * total_mass;
    if (relative_residual)
        *relative_residual = sqrt(rnorm / fmax(energy, 1e-30));
    if (rnorm <= target)
        return 0;

    double rz = 0.0, alpha = 0.0, beta = 0.0;
    int count = 0, iterations = 0, stopped = 0;
    double* z = s->lev[0].x;
    for (;;)
    {
        if (max_iterations >= 0 && iterations >= max_iterations)
            return -2;
        const int batch = max_iterations < 0 ? 4 : (max_iterations - iterations < 4 ? max_iterations - iterations : 4);
        for (int i = 0; i < batch; ++i)
        {
            if (stopped)
                break;
            visc_cycle(s, 0, s->residual);
            z = s->lev[0].x;
            const double rz_new = visc_dot(s, s->residual, z);
            rnorm = visc_mass_norm(s, s->residual);
            if (rnorm <= target)
            {
                stopped = 1;
                break;
            }
            if (!(rz_new > 0.0) || !isfinite(rz_new))
                return -1;
            beta = count > 0 ? rz_new / rz : 0.0;
            rz = rz_new;
            for (size_t n = 0; n < 2 * nodes; ++n)
                s->direction[n] = z[n] + (count > 0 ? beta * s->direction[n] : 0.0);
            or_visc_apply(s, 0, dt, s->direction, s->product);
            const double dq = visc_dot(s, s->direction, s->product);
            if (!(dq > 0.0) || !isfinite(dq))
                return -1;
            alpha = rz / dq;
            ++count;
            for (size_t n = 0; n < 2 * nodes; ++n)
            {
                s->solution[n] += alpha * s->direction[n];
                s->residual[n] -= alpha * s->product[n];
            }
        }
        iterations += batch;
        visc_residual(L, dt, s->solution, s->rhs, s->truth);
        const double truth = visc_mass_norm(s, s->truth);
        if (relative_residual)
            *relative_residual = sqrt(truth / fmax(energy, 1e-30));
        if (!isfinite(truth))
            return -1;
        if (truth <= target)
            break;
        if (stopped)
        {
            /* The recurrence claimed convergence: restart from the true residual. */
            memcpy(s->residual, s->truth, 2 * nodes * sizeof(double));
            rz = alpha = beta = 0.0;
            count = 0;
            stopped = 0;
        }
    }
    /* Unpack (ViscosityKernels.h "unpack"): every face of the solution. */
    for (int y = 0; y < h; ++y)
        for (int x = 0; x <= w; ++x)
            u[(size_t)y * (w + 1) + x] = s->solution[2 * ((size_t)y * (w + 1) + x)];
    for (int y = 0; y <= h; ++y)
        for (int x = 0; x < w; ++x)
            v[(size_t)y * w + x] = s->solution[2 * ((size_t)y * (w + 1) + x) + 1];
    return iterations;
}

/* Cell density and volume-weighted dynamic viscosity (FluidGridGPU.cpp:172-217, 987-1037):
 * rho = sum m_k / dx^2, mu = sum (m_k mu_k / rho_k) / sum (m_k / rho_k); a cell without mass
 * gets mu = 0. material receives 2 values per cell. */
void or_visc_material(int cells, int components, const double* const* masses, const double* densities,
    const double* viscosities, double cell_size, double* material)
{
    const double inv_area = 1.0 / (cell_size * cell_size);
    for (int i = 0; i < cells; ++i)
    {
        double total = 0.0, weighted = 0.0, volume = 0.0;
        for (int k = 0; k < components; ++k)
        {
            const double m = masses[k][i];
            total += m;
            weighted += m * (viscosities[k] / densities[k]);
            volume += m * (1.0 / densities[k]);
        }
        material[2 * i] = total * inv_area;
        material[2 * i + 1] = volume > 0.0 ? weighted / volume : 0.0;
    }
}
