/*
 * sph_oracle.c -- FP64 CPU restatement of pySurf's weakly compressible delta-SPH step.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity checker for the CUDA backend in
 * pysurf_b200/csrc: only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load
 * it.  Nothing in the product path links or calls it.
 *
 * Every sum is written in gather form (each particle sums over its own neighbour row), as the
 * reference's numba and Warp backends are, but in float64 throughout, so it reproduces the
 * reference's float64 array formulation (src/pysurf/sphSolver.py:527-1424) to rounding.  The
 * citations on each function name the reference lines it restates.  It is pinned against
 * golden vectors generated from the reference itself (tests/golden/make_golden.py).
 *
 * Conventions: positions and vectors are row-major (n, dim) float64 as numpy lays them out;
 * isFluid is one byte per particle; lengths is each particle's smoothing length h.  A periodic
 * axis is y (index 1) with period > 0, separations taken to the nearest image with
 * round-half-even, as numpy's np.round is (src/pysurf/sphSolver.py:1541-1543).
 *
 * Build: gcc -O2 -fopenmp -ffp-contract=off -shared -fPIC (see oracle/build.py).  Contraction
 * stays off so r^2 = dx*dx + dy*dy + dz*dz rounds term by term, as numba's does, which keeps
 * the neighbour sets bit-exact against src/pysurf/sphCompiled.py:70-98.
 */
#include <math.h>
#include <stddef.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define MAXD 3

/* ------------------------------------------------------------------------------------------ */
/* Kernels: src/pysurf/sphKernels.py:108-648 (cubic spline, Wendland C2), sphGpu.py:139-204     */
/* ------------------------------------------------------------------------------------------ */

/* sigma at h = 1: cubic 10/(7 pi) (2D), 1/pi (3D); Wendland 7/(4 pi) (2D), 21/(16 pi) (3D)
 * (src/pysurf/sphGpu.py:1431-1451). */
static double sigma_unit(int kind, int dim)
{
    if (kind == 1) return dim == 2 ? 7.0 / (4.0 * M_PI) : 21.0 / (16.0 * M_PI);
    return dim == 2 ? 10.0 / (7.0 * M_PI) : 1.0 / M_PI;
}

static double sigma_at(int kind, int dim, double h)
{
    double s = sigma_unit(kind, dim);
    return dim == 2 ? s / (h * h) : s / (h * h * h);
}

static double kernel_value(int kind, int dim, double r, double h)
{
    double q = r / h, sg = sigma_at(kind, dim, h);
    if (kind == 1) {
        if (q >= 2.0) return 0.0;
        double rest = 1.0 - 0.5 * q, sq = rest * rest;
        return sg * sq * sq * (2.0 * q + 1.0);
    }
    if (q < 1.0) return sg * (1.0 - 1.5 * q * q + 0.75 * q * q * q);
    if (q < 2.0) { double rest = 2.0 - q; return sg * 0.25 * rest * rest * rest; }
    return 0.0;
}

static double kernel_slope(int kind, int dim, double r, double h)
{
    double q = r / h, sg = sigma_at(kind, dim, h);
    if (q < 1e-12) return 0.0;
    if (kind == 1) {
        if (q >= 2.0) return 0.0;
        double rest = 1.0 - 0.5 * q;
        return -5.0 * sg * q * rest * rest * rest / h;
    }
    if (q < 1.0) return sg * (-3.0 * q + 2.25 * q * q) / h;
    if (q < 2.0) { double rest = 2.0 - q; return sg * (-0.75 * rest * rest) / h; }
    return 0.0;
}

/* ------------------------------------------------------------------------------------------ */
/* Geometry helpers                                                                           */
/* ------------------------------------------------------------------------------------------ */

/* r_i - r_j, the periodic y component to its nearest image (src/pysurf/sphCompiled.py:70-85). */
static void separation(const double *x, int dim, long i, long j, double period, double d[MAXD])
{
    d[2] = 0.0;
    for (int a = 0; a < dim; ++a) d[a] = x[i * dim + a] - x[j * dim + a];
    if (period > 0.0) d[1] -= period * rint(d[1] / period);
}

static double norm_sq(const double d[MAXD], int dim)
{
    double s = d[0] * d[0] + d[1] * d[1];
    if (dim == 3) s = s + d[2] * d[2];
    return s;
}

static double det_n(const double *m, int dim)
{
    if (dim == 2) return m[0] * m[3] - m[1] * m[2];
    return m[0] * (m[4] * m[8] - m[5] * m[7]) - m[1] * (m[3] * m[8] - m[5] * m[6])
         + m[2] * (m[3] * m[7] - m[4] * m[6]);
}

static void inverse_n(const double *m, int dim, double *out)
{
    double det = det_n(m, dim);
    if (dim == 2) {
        out[0] = m[3] / det; out[1] = -m[1] / det; out[2] = -m[2] / det; out[3] = m[0] / det;
        return;
    }
    out[0] = (m[4] * m[8] - m[5] * m[7]) / det;
    out[1] = (m[2] * m[7] - m[1] * m[8]) / det;
    out[2] = (m[1] * m[5] - m[2] * m[4]) / det;
    out[3] = (m[5] * m[6] - m[3] * m[8]) / det;
    out[4] = (m[0] * m[8] - m[2] * m[6]) / det;
    out[5] = (m[2] * m[3] - m[0] * m[5]) / det;
    out[6] = (m[3] * m[7] - m[4] * m[6]) / det;
    out[7] = (m[1] * m[6] - m[0] * m[7]) / det;
    out[8] = (m[0] * m[4] - m[1] * m[3]) / det;
}

/* ------------------------------------------------------------------------------------------ */
/* Cell key: src/pysurf/sphSolver.py:1379-1408 (cellOrderKey)                                  */
/* ------------------------------------------------------------------------------------------ */

static int64_t pymod(int64_t a, int64_t b) { int64_t r = a % b; return r < 0 ? r + b : r; }

void or_cell_order_key(const double *x, long n, int dim, double width, const int64_t *shape, int64_t *keys)
{
    #pragma omp parallel for schedule(static)
    for (long i = 0; i < n; ++i) {
        int64_t cx = pymod((int64_t)floor(x[i * dim] / width), shape[0]);
        int64_t cy = pymod((int64_t)floor(x[i * dim + 1] / width), shape[1]);
        int64_t cz = dim == 3 ? pymod((int64_t)floor(x[i * dim + 2] / width), shape[2]) : 0;
        keys[i] = (cz * shape[1] + cy) * shape[0] + cx;
    }
}

/* ------------------------------------------------------------------------------------------ */
/* Neighbour rows: src/pysurf/sphCompiled.py:133-234 (neighborList), the same cells, the same   */
/* scan order and the same float64 test, so rows match the reference's element for element.    */
/* ------------------------------------------------------------------------------------------ */

typedef struct {
    double lower[3], size[3];
    int64_t cells[3];
    int64_t *start, *order, *cellOf;
    int64_t steps[3][3], stepCount[3];
} CellList;

static void cells_build(CellList *c, const double *x, long n, int dim, double radius, double period)
{
    const int pa = 1;
    for (int a = 0; a < 3; ++a) { c->cells[a] = 1; c->size[a] = radius; c->lower[a] = 0.0; }
    for (int a = 0; a < dim; ++a) {
        double lo = x[a], hi = x[a];
        for (long i = 0; i < n; ++i) { double v = x[i * dim + a]; lo = v < lo ? v : lo; hi = v > hi ? v : hi; }
        if (period > 0.0 && a == pa) {
            c->lower[a] = 0.0;
            int64_t k = (int64_t)floor(period / radius);
            c->cells[a] = k > 1 ? k : 1;
            c->size[a] = period / (double)c->cells[a];
        } else {
            c->lower[a] = lo;
            c->cells[a] = (int64_t)floor((hi - lo) / radius) + 1;
        }
    }
    c->cellOf = (int64_t *)malloc(sizeof(int64_t) * (n > 0 ? n : 1));
    for (long i = 0; i < n; ++i) {
        int64_t index = 0;
        for (int a = 0; a < 3; ++a) {
            int64_t cc = 0;
            if (a < dim) {
                double value = x[i * dim + a] - c->lower[a];
                if (period > 0.0 && a == pa) value = value - period * floor(value / period);
                cc = (int64_t)(value / c->size[a]);
                if (cc < 0) cc = 0;
                if (cc > c->cells[a] - 1) cc = c->cells[a] - 1;
            }
            index = index * c->cells[a] + cc;
        }
        c->cellOf[i] = index;
    }
    int64_t total = c->cells[0] * c->cells[1] * c->cells[2];
    c->start = (int64_t *)calloc((size_t)total + 1, sizeof(int64_t));
    for (long i = 0; i < n; ++i) c->start[c->cellOf[i] + 1] += 1;
    for (int64_t k = 0; k < total; ++k) c->start[k + 1] += c->start[k];
    int64_t *fill = (int64_t *)malloc(sizeof(int64_t) * (size_t)(total + 1));
    memcpy(fill, c->start, sizeof(int64_t) * (size_t)total);
    c->order = (int64_t *)malloc(sizeof(int64_t) * (n > 0 ? n : 1));
    for (long i = 0; i < n; ++i) c->order[fill[c->cellOf[i]]++] = i;
    free(fill);
    for (int a = 0; a < 3; ++a) {
        if (a >= dim) { c->stepCount[a] = 1; c->steps[a][0] = 0; continue; }
        if (period > 0.0 && a == pa && c->cells[a] < 3) {
            c->stepCount[a] = c->cells[a];
            for (int k = 0; k < c->cells[a]; ++k) c->steps[a][k] = k;
        } else {
            c->stepCount[a] = 3; c->steps[a][0] = -1; c->steps[a][1] = 0; c->steps[a][2] = 1;
        }
    }
}

static void cells_free(CellList *c) { free(c->start); free(c->order); free(c->cellOf); }

static long cells_scan(const CellList *c, const double *x, int dim, long i, double r2max, double period,
                       int32_t *out)
{
    const int pa = 1;
    int64_t home = c->cellOf[i];
    int64_t c2 = home % c->cells[2], c1 = (home / c->cells[2]) % c->cells[1], c0 = home / (c->cells[2] * c->cells[1]);
    long found = 0;
    for (int a = 0; a < c->stepCount[0]; ++a) {
        int64_t n0 = c0 + c->steps[0][a];
        if (period > 0.0 && pa == 0) n0 = pymod(n0, c->cells[0]);
        else if (n0 < 0 || n0 >= c->cells[0]) continue;
        for (int b = 0; b < c->stepCount[1]; ++b) {
            int64_t n1 = c1 + c->steps[1][b];
            if (period > 0.0 && pa == 1) n1 = pymod(n1, c->cells[1]);
            else if (n1 < 0 || n1 >= c->cells[1]) continue;
            for (int e = 0; e < c->stepCount[2]; ++e) {
                int64_t n2 = c2 + c->steps[2][e];
                if (n2 < 0 || n2 >= c->cells[2]) continue;
                int64_t cell = (n0 * c->cells[1] + n1) * c->cells[2] + n2;
                for (int64_t k = c->start[cell]; k < c->start[cell + 1]; ++k) {
                    long j = (long)c->order[k];
                    if (j == i) continue;
                    double d[MAXD];
                    separation(x, dim, i, j, period, d);
                    /* numba: dx*dx + dy*dy + dz*dz with dz = 0 in 2D */
                    double s = d[0] * d[0] + d[1] * d[1];
                    s = s + d[2] * d[2];
                    if (s < r2max) { if (out) out[found] = (int32_t)j; ++found; }
                }
            }
        }
    }
    return found;
}

/* Count pass (neighbors == NULL: offsets filled, returns the total) or fill pass. */
long or_neighbor_list(const double *x, long n, int dim, double radius, double period, int64_t *offsets,
                      int32_t *neighbors)
{
    CellList c;
    cells_build(&c, x, n, dim, radius, period);
    double r2 = radius * radius;
    if (!neighbors) {
        int64_t *counts = (int64_t *)malloc(sizeof(int64_t) * (n > 0 ? n : 1));
        #pragma omp parallel for schedule(dynamic, 256)
        for (long i = 0; i < n; ++i) counts[i] = cells_scan(&c, x, dim, i, r2, period, NULL);
        offsets[0] = 0;
        for (long i = 0; i < n; ++i) offsets[i + 1] = offsets[i] + counts[i];
        free(counts);
    } else {
        #pragma omp parallel for schedule(dynamic, 256)
        for (long i = 0; i < n; ++i) cells_scan(&c, x, dim, i, r2, period, neighbors + offsets[i]);
    }
    cells_free(&c);
    return (long)offsets[n];
}

/* ------------------------------------------------------------------------------------------ */
/* The sums, over neighbour rows built at radius 2 max(h): each pair at h_ij = (h_i + h_j) / 2, */
/* kept when r < 2 h_ij (src/pysurf/sphSolver.py:1547-1555; src/pysurf/sphGpu.py:52-56, 362).   */
/* ------------------------------------------------------------------------------------------ */

typedef struct {
    int dim, kind;
    double period;
    const double *x;          /* (n, dim) */
    const double *h;          /* (n,) smoothing lengths */
    const uint8_t *fluid;     /* (n,) */
    const double *m;          /* (n,) */
    const int64_t *off;       /* (n + 1,) */
    const int32_t *nbr;
} Sys;

/* One pair's geometry; returns 0 when the pair is outside h_ij's support or coincident. */
static int pair_geom(const Sys *s, long i, long j, double d[MAXD], double *r, double *hij, int skipCoincident)
{
    separation(s->x, s->dim, i, j, s->period, d);
    *r = sqrt(norm_sq(d, s->dim));
    *hij = 0.5 * (s->h[i] + s->h[j]);
    if (*r >= 2.0 * *hij) return 0;
    if (skipCoincident && *r < 1e-12) return 0;
    return 1;
}

/* Tait pressure B((rho/rho0)^7 - 1), clamped at zero unless tension is allowed in the fluid
 * (src/pysurf/sphSolver.py:541-558, 1576-1585; src/pysurf/sphGpu.py:1058-1070). */
void or_equation_of_state(long n, const double *rho, const uint8_t *fluid, double rho0, double c0, int tension,
                          double *p)
{
    double B = rho0 * c0 * c0 / 7.0;
    for (long i = 0; i < n; ++i) {
        double ratio = rho[i] / rho0, sq = ratio * ratio;
        double v = B * (sq * sq * sq * ratio - 1.0);
        if (!tension || !fluid[i]) v = v > 0.0 ? v : 0.0;
        p[i] = v;
    }
}

/* src/pysurf/sphSolver.py:1045-1106 (extrapolatedWallPressure); src/pysurf/sphGpu.py:804-854.
 * Boundary rows take p_w = max(sum W (p_f + rho_f g . r_wf) / sum W, 0) and rho_w = Tait^-1(p_w);
 * fluid rows are copied. */
void or_wall_pressure(const Sys *s, long n, const double *rho, const double *p, const double *g, double rho0,
                      double c0, double *pOut, double *rhoOut)
{
    double B = rho0 * c0 * c0 / 7.0;
    #pragma omp parallel for schedule(dynamic, 128)
    for (long i = 0; i < n; ++i) {
        pOut[i] = p[i];
        if (rhoOut) rhoOut[i] = rho[i];
        if (s->fluid[i]) continue;
        double weight = 0.0, total = 0.0;
        for (int64_t k = s->off[i]; k < s->off[i + 1]; ++k) {
            long j = s->nbr[k];
            if (!s->fluid[j]) continue;
            double d[MAXD], r, hij;
            if (!pair_geom(s, i, j, d, &r, &hij, 0)) continue;
            double w = kernel_value(s->kind, s->dim, r, hij);
            double gd = 0.0;
            for (int a = 0; a < s->dim; ++a) gd += g[a] * d[a];
            weight += w;
            total += w * (p[j] + rho[j] * gd);
        }
        double pw = 0.0;
        if (weight > 0.0) { pw = total / weight; pw = pw > 0.0 ? pw : 0.0; }
        pOut[i] = pw;
        if (rhoOut) rhoOut[i] = rho0 * pow(1.0 + pw / B, 1.0 / 7.0);
    }
}

/* src/pysurf/sphSolver.py:1151-1190 (velocityGradients); src/pysurf/sphGpu.py:643-697.
 * G_i = S_i M_i^-1 over fluid neighbours, zero on the boundary and where det M < 0.25^dim. */
void or_velocity_gradients(const Sys *s, long n, const double *v, const double *rho, double *G)
{
    int dim = s->dim, dd = dim * dim;
    double floorDet = pow(0.25, dim);
    #pragma omp parallel for schedule(dynamic, 128)
    for (long i = 0; i < n; ++i) {
        double S[9] = {0}, M[9] = {0}, inv[9];
        for (int a = 0; a < dd; ++a) G[i * dd + a] = 0.0;
        if (!s->fluid[i]) continue;
        for (int64_t k = s->off[i]; k < s->off[i + 1]; ++k) {
            long j = s->nbr[k];
            if (!s->fluid[j]) continue;
            double d[MAXD], r, hij;
            if (!pair_geom(s, i, j, d, &r, &hij, 1)) continue;
            double w = s->m[j] / rho[j] * kernel_slope(s->kind, dim, r, hij) / r;
            for (int a = 0; a < dim; ++a)
                for (int b = 0; b < dim; ++b) {
                    S[a * dim + b] += w * (v[j * dim + a] - v[i * dim + a]) * d[b];
                    M[a * dim + b] += -w * d[a] * d[b];
                }
        }
        if (det_n(M, dim) >= floorDet) {
            inverse_n(M, dim, inv);
            for (int a = 0; a < dim; ++a)
                for (int b = 0; b < dim; ++b) {
                    double t = 0.0;
                    for (int c = 0; c < dim; ++c) t += S[a * dim + c] * inv[c * dim + b];
                    G[i * dd + a * dim + b] = t;
                }
        }
    }
}

/* src/pysurf/sphSolver.py:656-689 (correctionMatrices); src/pysurf/sphGpu.py:593-641.
 * L_i = M_i^-1 over every neighbour; the identity on the boundary and where det M < 0.25^dim. */
void or_correction_matrices(const Sys *s, long n, const double *rho, double *L)
{
    int dim = s->dim, dd = dim * dim;
    double floorDet = pow(0.25, dim);
    #pragma omp parallel for schedule(dynamic, 128)
    for (long i = 0; i < n; ++i) {
        double M[9] = {0};
        for (int a = 0; a < dim; ++a)
            for (int b = 0; b < dim; ++b) L[i * dd + a * dim + b] = a == b ? 1.0 : 0.0;
        if (!s->fluid[i]) continue;
        for (int64_t k = s->off[i]; k < s->off[i + 1]; ++k) {
            long j = s->nbr[k];
            double d[MAXD], r, hij;
            if (!pair_geom(s, i, j, d, &r, &hij, 1)) continue;
            double w = s->m[j] / rho[j] * kernel_slope(s->kind, dim, r, hij) / r;
            for (int a = 0; a < dim; ++a)
                for (int b = 0; b < dim; ++b) M[a * dim + b] += -w * d[a] * d[b];
        }
        if (det_n(M, dim) >= floorDet) inverse_n(M, dim, L + i * dd);
    }
}

/* src/pysurf/sphSolver.py:691-716 (renormalizedDensityGradient); src/pysurf/sphGpu.py:547-591.
 * grad rho_i = L_i sum_j V_j (rho_j - rho_i) grad W_ij over every neighbour; zero on the boundary. */
void or_density_gradients(const Sys *s, long n, const double *rho, const double *L, double *out)
{
    int dim = s->dim, dd = dim * dim;
    #pragma omp parallel for schedule(dynamic, 128)
    for (long i = 0; i < n; ++i) {
        double t[MAXD] = {0};
        for (int a = 0; a < dim; ++a) out[i * dim + a] = 0.0;
        if (!s->fluid[i]) continue;
        for (int64_t k = s->off[i]; k < s->off[i + 1]; ++k) {
            long j = s->nbr[k];
            double d[MAXD], r, hij;
            if (!pair_geom(s, i, j, d, &r, &hij, 1)) continue;
            double w = s->m[j] / rho[j] * (rho[j] - rho[i]) * kernel_slope(s->kind, dim, r, hij) / r;
            for (int a = 0; a < dim; ++a) t[a] += w * d[a];
        }
        for (int a = 0; a < dim; ++a) {
            double u = 0.0;
            for (int b = 0; b < dim; ++b) u += L[i * dd + a * dim + b] * t[b];
            out[i * dim + a] = u;
        }
    }
}

typedef struct {
    double c0, alpha, boundaryFactor, g[3];
    int limited;
    int closure;                /* the delta-LES-SPH viscous term on fluid pairs */
    double waterTerm, rho0;     /* 2 (dim + 2) nu / c0, and rho0 */
    const double *alphas;       /* each particle's alpha_i (or_closure_coefficients) */
    double *parts;              /* energy budget: each fluid row's pressure and viscosity from fluid and
                                   from boundary neighbours (n x 4 x dim), or NULL */
} AccelParams;

static double harmonic_mean(double a, double b)
{
    double both = a + b;
    return both > 0.0 ? 2.0 * a * b / both : 0.0;
}

/* The energy budget's elastic energy, src/pysurf/sphEnergy.py:100-139 (elasticEnergy): e(rho) per
 * unit mass = (c0^2 / 7) x^2 (21 + 35 x + 35 x^2 + 21 x^3 + 7 x^4 + x^5) / (6 (1 + x)), x = rho / rho0 - 1,
 * zero below rho0 unless the fluid carries tension.  scale = c0^2 / 7. */
static double elastic_energy(double rho, double rho0, double scale, int tension)
{
    double x = rho / rho0 - 1.0;
    double poly = 21.0 + x * (35.0 + x * (35.0 + x * (21.0 + x * (7.0 + x))));
    double e = scale * x * x * poly / (6.0 * (1.0 + x));
    return (!tension && x < 0.0) ? 0.0 : e;
}

/* src/pysurf/sphEnergy.py:141-160 (elasticSlope): the secant (e(after) - e(before)) / (after - before),
 * or p / rho^2 at the midpoint for a change under 1e-10 rho0. */
static double elastic_slope(double before, double after, double rho0, double scale, int tension)
{
    double change = after - before, mid = 0.5 * (before + after), ratio = mid / rho0;
    double p = scale * rho0 * (pow(ratio, 7.0) - 1.0);
    if (!tension && p < 0.0) p = 0.0;
    if (fabs(change) > 1e-10 * rho0)
        return (elastic_energy(after, rho0, scale, tension) - elastic_energy(before, rho0, scale, tension)) / change;
    return p / (mid * mid);
}

void or_elastic_energy(long n, const double *rho, double rho0, double c0, int tension, double *out)
{
    for (long i = 0; i < n; ++i) out[i] = elastic_energy(rho[i], rho0, c0 * c0 / 7.0, tension);
}

void or_elastic_slope(long n, const double *before, const double *after, double rho0, double c0, int tension,
                      double *out)
{
    for (long i = 0; i < n; ++i) out[i] = elastic_slope(before[i], after[i], rho0, c0 * c0 / 7.0, tension);
}

/* The fluid's kinetic, potential (-m g . x) and elastic energy [J] (src/pysurf/sphParticles.py:236-255,
 * src/pysurf/sphSolver.py:2156-2161), summed in particle order. */
void or_fluid_energy(long n, int dim, const double *x, const double *v, const double *rho, const double *m,
                     const uint8_t *fluid, const double *g, double rho0, double c0, int tension, double out[3])
{
    double k = 0.0, p = 0.0, e = 0.0;
    for (long i = 0; i < n; ++i) {
        if (!fluid[i]) continue;
        double v2 = 0.0, gx = 0.0;
        for (int c = 0; c < dim; ++c) { v2 += v[i * dim + c] * v[i * dim + c]; gx += g[c] * x[i * dim + c]; }
        k += 0.5 * m[i] * v2;
        p -= m[i] * gx;
        e += m[i] * elastic_energy(rho[i], rho0, c0 * c0 / 7.0, tension);
    }
    out[0] = k; out[1] = p; out[2] = e;
}

/* src/pysurf/sphSolver.py:1232-1274 (closureCoefficients): ||D|| = sqrt(2 D:D), D = (G + G^T) / 2,
 * alpha_i = 2 (dim + 2) (C_S l)^2 ||D|| / (c0 h), delta_i = (C_delta l)^2 ||D|| / (c0 h), l = 2 h,
 * C_S 0.12, C_delta 1.5, each at most 0.2; zero on the boundary. */
void or_closure_coefficients(const Sys *s, long n, const double *G, double c0, double *alphas, double *deltas)
{
    int dim = s->dim, dd = dim * dim;
    for (long i = 0; i < n; ++i) {
        alphas[i] = deltas[i] = 0.0;
        if (!s->fluid[i]) continue;
        double sum = 0.0;
        for (int a = 0; a < dim; ++a)
            for (int b = 0; b < dim; ++b) {
                double e = 0.5 * (G[i * dd + a * dim + b] + G[i * dd + b * dim + a]);
                sum += e * e;
            }
        double norm = sqrt(2.0 * sum), h = s->h[i], width = 2.0 * h;
        double al = 2.0 * (dim + 2) * (0.12 * width) * (0.12 * width) * norm / (c0 * h);
        double de = (1.5 * width) * (1.5 * width) * norm / (c0 * h);
        alphas[i] = al < 0.2 ? al : 0.2;
        deltas[i] = de < 0.2 ? de : 0.2;
    }
}

/* src/pysurf/sphSolver.py:1122-1149 (artificialViscosity), 1192-1230 (limitedVelocityDifference),
 * 1328-1356 (pairAccelerations), 1610-1643 (_computeRates); src/pysurf/sphGpu.py:303-414.
 * a_i = -sum_j m_j (p_i/rho_i^2 + p_j/rho_j^2 + Pi_ij) grad W_ij + g on the fluid, zero on the
 * boundary. */
void or_accelerations(const Sys *s, long n, const double *v, const double *rho, const double *p,
                      const double *G, const AccelParams *ap, double *a)
{
    int dim = s->dim, dd = dim * dim;
    #pragma omp parallel for schedule(dynamic, 128)
    for (long i = 0; i < n; ++i) {
        for (int c = 0; c < dim; ++c) a[i * dim + c] = 0.0;
        if (!s->fluid[i]) continue;
        double own = p[i] / (rho[i] * rho[i]);
        double tot[MAXD] = {0}, part[4][MAXD] = {{0}};
        for (int64_t k = s->off[i]; k < s->off[i + 1]; ++k) {
            long j = s->nbr[k];
            double d[MAXD], r, h;
            if (!pair_geom(s, i, j, d, &r, &h, 1)) continue;
            double rel[MAXD] = {0}, approach = 0.0;
            for (int c = 0; c < dim; ++c) { rel[c] = v[i * dim + c] - v[j * dim + c]; approach += rel[c] * d[c]; }
            double visc = 0.0;
            if (approach < 0.0 && ap->limited && s->fluid[j]) {
                double rampI[MAXD] = {0}, rampJ[MAXD] = {0}, slopeI = 0.0, slopeJ = 0.0;
                for (int c = 0; c < dim; ++c) {
                    for (int b = 0; b < dim; ++b) {
                        rampI[c] += G[i * dd + c * dim + b] * d[b];
                        rampJ[c] += G[j * dd + c * dim + b] * d[b];
                    }
                    slopeI += d[c] * rampI[c];
                    slopeJ += d[c] * rampJ[c];
                }
                double lim = 0.0;
                if (slopeI * slopeJ > 0.0) {
                    double ratio = slopeI / slopeJ;
                    lim = 4.0 * ratio / ((1.0 + ratio) * (1.0 + ratio));
                    lim = lim < 1.0 ? lim : 1.0;
                    double eta = r / h;
                    if (eta < 0.3) { double f = (eta - 0.3) / 0.2; lim *= exp(-f * f); }
                }
                approach = 0.0;
                for (int c = 0; c < dim; ++c) approach += (rel[c] - 0.5 * lim * (rampI[c] + rampJ[c])) * d[c];
            }
            if (approach < 0.0) {
                double mu = h * approach / (r * r + 0.01 * h * h);
                visc = -ap->alpha * ap->c0 * mu / (0.5 * (rho[i] + rho[j]));
                if (!s->fluid[j]) visc *= ap->boundaryFactor;
            }
            if (ap->closure && s->fluid[j]) {
                /* src/pysurf/sphSolver.py:1283-1326 (closureViscosity): every fluid pair, the plain v_ij . r_ij */
                double plain = 0.0;
                for (int c = 0; c < dim; ++c) plain += rel[c] * d[c];
                double pairAlpha = ap->waterTerm / h + harmonic_mean(ap->alphas[i], ap->alphas[j]);
                visc += -pairAlpha * ap->c0 * h * ap->rho0 * plain / (r * r * rho[i] * rho[j]);
            }
            double coef = -(own + p[j] / (rho[j] * rho[j]) + visc) * s->m[j];
            double grad = kernel_slope(s->kind, dim, r, h) / r, f = coef * grad;
            for (int c = 0; c < dim; ++c) tot[c] += f * d[c];
            if (ap->parts) {
                /* src/pysurf/sphGpu.py:400-409: pressure and viscosity, from fluid or boundary j */
                int wall = s->fluid[j] ? 0 : 2;
                double fp = -(own + p[j] / (rho[j] * rho[j])) * s->m[j] * grad, fv = -visc * s->m[j] * grad;
                for (int c = 0; c < dim; ++c) { part[wall][c] += fp * d[c]; part[wall + 1][c] += fv * d[c]; }
            }
        }
        for (int c = 0; c < dim; ++c) a[i * dim + c] = tot[c] + ap->g[c];
        if (ap->parts)
            for (int q = 0; q < 4; ++q)
                for (int c = 0; c < dim; ++c) ap->parts[(i * 4 + q) * dim + c] = part[q][c];
    }
}

typedef struct {
    int mode;              /* 0 none, 1 molteni, 2 hydrostatic, 3 antuono */
    double delta, c0, rho0, gravity;
    int corrected;
    int closure;           /* the pair's delta is the harmonic mean of the two particles' (closure) */
    const double *deltas;
    double *parts;         /* energy budget: each fluid row's plain sum over fluid and over boundary
                              neighbours, the correction's part and the diffusion (n x 4), or NULL */
} ContinuityParams;

/* src/pysurf/sphSolver.py:623-654 (continuityRate), 718-822 (hydrostaticDensityDifference,
 * densityDiffusionRate); src/pysurf/sphGpu.py:430-545.  Pairs of two boundary particles add
 * nothing; the diffusive term acts on fluid pairs. */
void or_continuity(const Sys *s, long n, const double *v, const double *rho, const double *L,
                   const double *gradRho, const ContinuityParams *cp, double *out)
{
    int dim = s->dim, dd = dim * dim;
    #pragma omp parallel for schedule(dynamic, 128)
    for (long i = 0; i < n; ++i) {
        int boundaryI = !s->fluid[i];
        int diffuses = cp->mode != 0 && !boundaryI;
        double total = 0.0, plainF = 0.0, plainW = 0.0, diffusive = 0.0;
        for (int64_t k = s->off[i]; k < s->off[i + 1]; ++k) {
            long j = s->nbr[k];
            if (boundaryI && !s->fluid[j]) continue;
            double d[MAXD], r, h;
            if (!pair_geom(s, i, j, d, &r, &h, 1)) continue;
            double slope = kernel_slope(s->kind, dim, r, h);
            double Ld[MAXD];
            for (int a = 0; a < dim; ++a) {
                Ld[a] = d[a];
                if (cp->corrected && !boundaryI) {
                    Ld[a] = 0.0;
                    for (int b = 0; b < dim; ++b) Ld[a] += L[i * dd + a * dim + b] * d[b];
                }
            }
            double dot = 0.0, plainDot = 0.0;
            for (int a = 0; a < dim; ++a) {
                dot += (v[i * dim + a] - v[j * dim + a]) * Ld[a];
                plainDot += (v[i * dim + a] - v[j * dim + a]) * d[a];
            }
            total += s->m[j] * dot * slope / r;
            /* src/pysurf/sphGpu.py:508-515: the uncorrected sum, split by the neighbour's kind */
            if (s->fluid[j]) plainF += s->m[j] * plainDot * slope / r;
            else plainW += s->m[j] * plainDot * slope / r;
            if (diffuses && s->fluid[j]) {
                double diff = rho[j] - rho[i];
                if (cp->mode == 2) {
                    double ratio = 0.5 * (rho[i] + rho[j]) / cp->rho0;
                    diff -= cp->rho0 * cp->gravity / (cp->c0 * cp->c0) * d[dim - 1] * pow(ratio, -5.0);
                } else if (cp->mode == 3) {
                    double t = 0.0;
                    for (int a = 0; a < dim; ++a) t += (gradRho[i * dim + a] + gradRho[j * dim + a]) * d[a];
                    diff += 0.5 * t;
                }
                double outward = -slope * r;
                double delta = cp->closure ? harmonic_mean(cp->deltas[i], cp->deltas[j]) : cp->delta;
                double term = 2.0 * delta * h * cp->c0 * diff * outward / (r * r + 0.01 * h * h) * s->m[j] / rho[j];
                total += term;
                diffusive += term;
            }
        }
        out[i] = total;
        if (cp->parts) {
            double *q = cp->parts + i * 4;
            q[0] = boundaryI ? 0.0 : plainF;
            q[1] = boundaryI ? 0.0 : plainW;
            q[2] = boundaryI || !cp->corrected ? 0.0 : total - diffusive - plainF - plainW;
            q[3] = boundaryI ? 0.0 : diffusive;
        }
    }
}

/* Particle shifting, src/pysurf/sphSolver.py:824-887 (shiftingFields): over every neighbour of a
 * fluid particle, grad C = sum V_j [1 + 0.2 (W_ij / W(dx))^4] grad W_ij, grad C0 = sum V_j grad W_ij,
 * div r = -sum V_j r_ij . grad W_ij, grad rho = sum (rho_j - rho_i) V_j grad W_ij.  Boundary rows
 * get zeros and a divergence of 1e6 (never a free surface). */
void or_shifting_fields(const Sys *s, long n, const double *rho, double spacingKernel, double *grad, double *plain,
                        double *div, double *rhoGrad)
{
    int dim = s->dim;
    #pragma omp parallel for schedule(dynamic, 128)
    for (long i = 0; i < n; ++i) {
        double g[MAXD] = {0}, c[MAXD] = {0}, rg[MAXD] = {0}, total = 0.0;
        if (s->fluid[i]) {
            for (int64_t k = s->off[i]; k < s->off[i + 1]; ++k) {
                long j = s->nbr[k];
                double d[MAXD], r, h;
                if (!pair_geom(s, i, j, d, &r, &h, 1)) continue;
                double volume = s->m[j] / rho[j];
                double slope = kernel_slope(s->kind, dim, r, h);
                double ratio = kernel_value(s->kind, dim, r, h) / spacingKernel, square = ratio * ratio;
                for (int a = 0; a < dim; ++a) {
                    double weighted = volume * slope / r * d[a];
                    c[a] += weighted;
                    g[a] += (1.0 + 0.2 * square * square) * weighted;
                    rg[a] += (rho[j] - rho[i]) * weighted;
                }
                total -= volume * slope * r;
            }
        } else {
            total = 1.0e6;
        }
        for (int a = 0; a < dim; ++a) { grad[i * dim + a] = g[a]; plain[i * dim + a] = c[a]; rhoGrad[i * dim + a] = rg[a]; }
        div[i] = total;
    }
}

/* src/pysurf/sphSolver.py:889-979 (freeSurface, shiftingDisplacement) and 981-1010
 * (shiftedVelocityChange).  A fluid particle is on the free surface when div r < threshold or
 * h |grad C0| > lopsidedness; it and the boundary do not shift.  Next to a surface particle (one
 * within 2h) the shift -size_i grad C loses its part along n, the kernel-weighted mean of the
 * surface neighbours' outward normals -grad C0 / |grad C0|, or is zero where h |grad C| > 0.03;
 * elsewhere it is whole.  The density change is shift . grad rho; the velocity change
 * sum_j V_j (v_j - v_i) (grad W_ij . shift) over fluid neighbours. */
void or_shift(const Sys *s, long n, const double *rho, const double *v, const double *grad, const double *plain,
              const double *div, const double *rhoGrad, const double *size, double threshold, double lopsidedness,
              double *shift, double *drho, double *dv)
{
    int dim = s->dim;
    uint8_t *surface = (uint8_t *)malloc((size_t)n);
    for (long i = 0; i < n; ++i) {
        double length = 0.0;
        for (int a = 0; a < dim; ++a) length += plain[i * dim + a] * plain[i * dim + a];
        length = sqrt(length);
        surface[i] = s->fluid[i] && (div[i] < threshold || s->h[i] * length > lopsidedness);
    }
    #pragma omp parallel for schedule(dynamic, 128)
    for (long i = 0; i < n; ++i) {
        double sh[MAXD] = {0}, nrm[MAXD] = {0};
        int vicinity = 0;
        for (int64_t k = s->off[i]; k < s->off[i + 1]; ++k) {
            long j = s->nbr[k];
            if (!surface[j]) continue;
            double d[MAXD], r, h;
            if (!pair_geom(s, i, j, d, &r, &h, 0)) continue;
            vicinity = 1;
            double length = 0.0;
            for (int a = 0; a < dim; ++a) length += plain[j * dim + a] * plain[j * dim + a];
            length = sqrt(length);
            double w = kernel_value(s->kind, dim, r, h);
            for (int a = 0; a < dim; ++a) nrm[a] += w * (-plain[j * dim + a] / length);
        }
        double gl = 0.0;
        for (int a = 0; a < dim; ++a) { sh[a] = -size[i] * grad[i * dim + a]; gl += grad[i * dim + a] * grad[i * dim + a]; }
        gl = sqrt(gl);
        if (vicinity) {
            double weight = 0.0;
            for (int a = 0; a < dim; ++a) weight += nrm[a] * nrm[a];
            weight = sqrt(weight);
            if (weight > 0.0) {
                double dot = 0.0;
                for (int a = 0; a < dim; ++a) { nrm[a] /= weight; dot += sh[a] * nrm[a]; }
                for (int a = 0; a < dim; ++a) sh[a] -= dot * nrm[a];
            }
        }
        if (surface[i] || !s->fluid[i] || (vicinity && s->h[i] * gl > 0.03))
            for (int a = 0; a < dim; ++a) sh[a] = 0.0;
        double change = 0.0, vc[MAXD] = {0};
        for (int a = 0; a < dim; ++a) change += sh[a] * rhoGrad[i * dim + a];
        if (s->fluid[i]) {
            for (int64_t k = s->off[i]; k < s->off[i + 1]; ++k) {
                long j = s->nbr[k];
                if (!s->fluid[j]) continue;
                double d[MAXD], r, h;
                if (!pair_geom(s, i, j, d, &r, &h, 1)) continue;
                double dot = 0.0;
                for (int a = 0; a < dim; ++a) dot += d[a] * sh[a];
                double f = s->m[j] / rho[j] * kernel_slope(s->kind, dim, r, h) / r * dot;
                for (int a = 0; a < dim; ++a) vc[a] += f * (v[j * dim + a] - v[i * dim + a]);
            }
        }
        for (int a = 0; a < dim; ++a) { shift[i * dim + a] = sh[a]; dv[i * dim + a] = vc[a]; }
        drho[i] = change;
    }
    free(surface);
}

/* src/pysurf/sphSolver.py:1358-1377 (xsphVelocity over fluid pairs); src/pysurf/sphGpu.py:725-766. */
void or_xsph(const Sys *s, long n, const double *v, const double *rho, double eps, double *out)
{
    int dim = s->dim;
    #pragma omp parallel for schedule(dynamic, 128)
    for (long i = 0; i < n; ++i) {
        double c[MAXD] = {0};
        for (int a = 0; a < dim; ++a) out[i * dim + a] = v[i * dim + a];
        if (!s->fluid[i]) continue;
        for (int64_t k = s->off[i]; k < s->off[i + 1]; ++k) {
            long j = s->nbr[k];
            if (!s->fluid[j]) continue;
            double d[MAXD], r, h;
            if (!pair_geom(s, i, j, d, &r, &h, 0)) continue;
            double w = s->m[j] * kernel_value(s->kind, dim, r, h) / (0.5 * (rho[i] + rho[j]));
            for (int a = 0; a < dim; ++a) c[a] += w * (v[j * dim + a] - v[i * dim + a]);
        }
        for (int a = 0; a < dim; ++a) out[i * dim + a] = v[i * dim + a] + eps * c[a];
    }
}

/* src/pysurf/sphSolver.py:1011-1032 (shepardDensity); src/pysurf/sphGpu.py:768-802. */
void or_shepard(const Sys *s, long n, const double *rho, double *out)
{
    int dim = s->dim;
    #pragma omp parallel for schedule(dynamic, 128)
    for (long i = 0; i < n; ++i) {
        double own = sigma_at(s->kind, dim, s->h[i]);
        double num = s->m[i] * own, den = s->m[i] / rho[i] * own;
        for (int64_t k = s->off[i]; k < s->off[i + 1]; ++k) {
            long j = s->nbr[k];
            double d[MAXD], r, h;
            if (!pair_geom(s, i, j, d, &r, &h, 0)) continue;
            double w = kernel_value(s->kind, dim, r, h);
            num += s->m[j] * w;
            den += s->m[j] / rho[j] * w;
        }
        out[i] = num / den;
    }
}

/* ------------------------------------------------------------------------------------------ */
/* Boundary enforcement: src/pysurf/sphBoundaries.py:126-147, 295-344, 597-640;                */
/* src/pysurf/sphGpu.py:1197-1419 (the device kernels' arithmetic).                            */
/* ------------------------------------------------------------------------------------------ */

void or_enforce_container(long n, int dim, double *x, double *v, const uint8_t *fluid, const double *lower,
                          const double *upper, int openTop)
{
    for (long i = 0; i < n; ++i) {
        if (!fluid[i]) continue;
        for (int a = 0; a < dim; ++a) {
            if (x[i * dim + a] < lower[a]) { x[i * dim + a] = lower[a]; if (v[i * dim + a] < 0.0) v[i * dim + a] = 0.0; }
            if (a < dim - 1 || !openTop)
                if (x[i * dim + a] > upper[a]) { x[i * dim + a] = upper[a]; if (v[i * dim + a] > 0.0) v[i * dim + a] = 0.0; }
        }
    }
}

typedef struct {
    const double *bedX, *bedZ;
    long count;
    double clearance;
    int sideWalls;
    double width;
    int offshoreWall;
    double wallX, pistonSpeed, endLimit;
} BedParams;

static long bed_segment(double x, const double *bx, long count)
{
    long lo = 0, hi = count - 1;
    while (hi - lo > 1) {
        long mid = (lo + hi) / 2;
        if (bx[mid] <= x) lo = mid; else hi = mid;
    }
    return lo;
}

void or_enforce_bed(long n, int dim, double *x, double *v, const uint8_t *fluid, const BedParams *bp)
{
    int vert = dim - 1;
    for (long i = 0; i < n; ++i) {
        if (!fluid[i]) continue;
        double *xi = x + i * dim, *vi = v + i * dim;
        long k = bed_segment(xi[0], bp->bedX, bp->count);
        double run = bp->bedX[k + 1] - bp->bedX[k], rise = bp->bedZ[k + 1] - bp->bedZ[k];
        double share = (xi[0] - bp->bedX[k]) / run;
        share = share < 0.0 ? 0.0 : (share > 1.0 ? 1.0 : share);
        double bed = bp->bedZ[k] + share * rise;
        if (xi[vert] < bed + bp->clearance) {
            xi[vert] = bed + bp->clearance;
            double slope = rise / run, len = sqrt(1.0 + slope * slope);
            double nx = -slope / len, nz = 1.0 / len;
            double inward = vi[0] * nx + vi[vert] * nz;
            if (inward < 0.0) { vi[0] -= inward * nx; vi[vert] -= inward * nz; }
        }
        if (bp->sideWalls) {
            if (xi[1] < bp->clearance) { xi[1] = bp->clearance; if (vi[1] < 0.0) vi[1] = 0.0; }
            if (xi[1] > bp->width - bp->clearance) { xi[1] = bp->width - bp->clearance; if (vi[1] > 0.0) vi[1] = 0.0; }
        }
        if (bp->offshoreWall && xi[0] < bp->wallX + bp->clearance) {
            xi[0] = bp->wallX + bp->clearance;
            if (vi[0] < bp->pistonSpeed) vi[0] = bp->pistonSpeed;
        }
        if (xi[0] > bp->endLimit) { xi[0] = bp->endLimit; if (vi[0] > 0.0) vi[0] = 0.0; }
    }
}

typedef struct {
    const double *table;     /* (ny, nx) */
    long nx, ny;
    double originX, originY, stepX, stepY, clearance, lowY, highY;
    int offshoreWall;
    double lowX, highX;
} FieldParams;

/* Cubic convolution weights (Keys 1981, a = -1/2): src/pysurf/bathymetry.py:310-334. */
static void conv_weights(double u, double w[4])
{
    double u2 = u * u, u3 = u2 * u;
    w[0] = -0.5 * u3 + u2 - 0.5 * u; w[1] = 1.5 * u3 - 2.5 * u2 + 1.0;
    w[2] = -1.5 * u3 + 2.0 * u2 + 0.5 * u; w[3] = 0.5 * u3 - 0.5 * u2;
}

static void conv_slope_weights(double u, double w[4])
{
    double u2 = u * u;
    w[0] = -1.5 * u2 + 2.0 * u - 0.5; w[1] = 4.5 * u2 - 5.0 * u;
    w[2] = -4.5 * u2 + 4.0 * u + 0.5; w[3] = 1.5 * u2 - u;
}

static long clampl(long a, long lo, long hi) { return a < lo ? lo : (a > hi ? hi : a); }

void or_enforce_heightfield(long n, double *x, double *v, const uint8_t *fluid, const FieldParams *fp)
{
    for (long i = 0; i < n; ++i) {
        if (!fluid[i]) continue;
        double *xi = x + i * 3, *vi = v + i * 3;
        double rawX = (xi[0] - fp->originX) / fp->stepX, rawY = (xi[1] - fp->originY) / fp->stepY;
        double fx = rawX < 0.0 ? 0.0 : (rawX > (double)(fp->nx - 1) ? (double)(fp->nx - 1) : rawX);
        double fy = rawY < 0.0 ? 0.0 : (rawY > (double)(fp->ny - 1) ? (double)(fp->ny - 1) : rawY);
        long ix = (long)floor(fx), iy = (long)floor(fy);
        double wx[4], wy[4], sx[4], sy[4];
        conv_weights(fx - (double)ix, wx); conv_weights(fy - (double)iy, wy);
        conv_slope_weights(fx - (double)ix, sx); conv_slope_weights(fy - (double)iy, sy);
        double bed = 0.0, slopeX = 0.0, slopeY = 0.0;
        for (int a = 0; a < 4; ++a) {
            long row = clampl(iy - 1 + a, 0, fp->ny - 1);
            double along = 0.0, alongSlope = 0.0;
            for (int b = 0; b < 4; ++b) {
                double value = fp->table[row * fp->nx + clampl(ix - 1 + b, 0, fp->nx - 1)];
                along += wx[b] * value;
                alongSlope += sx[b] * value;
            }
            bed += wy[a] * along; slopeX += wy[a] * alongSlope; slopeY += sy[a] * along;
        }
        slopeX /= fp->stepX; slopeY /= fp->stepY;
        if (rawX < 0.0 || rawX > (double)(fp->nx - 1)) slopeX = 0.0;
        if (rawY < 0.0 || rawY > (double)(fp->ny - 1)) slopeY = 0.0;
        if (xi[2] < bed + fp->clearance) {
            xi[2] = bed + fp->clearance;
            double len = sqrt(slopeX * slopeX + slopeY * slopeY + 1.0);
            double nrm[3] = {-slopeX / len, -slopeY / len, 1.0 / len};
            double inward = vi[0] * nrm[0] + vi[1] * nrm[1] + vi[2] * nrm[2];
            if (inward < 0.0) for (int a = 0; a < 3; ++a) vi[a] -= inward * nrm[a];
        }
        if (xi[1] < fp->lowY) { xi[1] = fp->lowY; if (vi[1] < 0.0) vi[1] = 0.0; }
        if (xi[1] > fp->highY) { xi[1] = fp->highY; if (vi[1] > 0.0) vi[1] = 0.0; }
        if (fp->offshoreWall && xi[0] < fp->lowX) { xi[0] = fp->lowX; if (vi[0] < 0.0) vi[0] = 0.0; }
        if (xi[0] > fp->highX) { xi[0] = fp->highX; if (vi[0] > 0.0) vi[0] = 0.0; }
    }
}

/* ------------------------------------------------------------------------------------------ */
/* One device-resident step: src/pysurf/sphGpu.py:2237-2315 (residentRates, residentIntegrate) */
/* and src/pysurf/sphSolver.py:1941-1991 (advance), 1410-1424 (cflTimeStep).                   */
/* ------------------------------------------------------------------------------------------ */

typedef struct {
    int dim, kind;
    double period, hMax, hMin;
    double rho0, c0, alpha, boundaryFactor, g[3], xsphEpsilon, densityFloor;
    int diffusion; double delta;
    int wallExtrapolated, tension, corrected, limited;
    double cfl, maxTimeStep;
    int filterDensity;                          /* this step filters (Shepard) */
    int boundaryKind;                            /* 0 none, 1 container, 2 bed, 3 height field */
    double lower[3], upper[3]; int openTop;     /* container */
    BedParams bed;
    FieldParams field;
    int closure;                                 /* delta-LES-SPH closure, with the water's viscosity */
    double viscosity;
    int shifting, shiftLocal;                    /* particle shifting: size c0 dt / h Ma (2h)^2, or 2 h |v| dt */
    double shiftMach, spacingKernel, shiftThreshold, lopsidedness;
    double *energy;                              /* the energy budget's 14 running totals, or NULL */
} StepParams;

static double cfl_time_step(double h, double c0, double vmax, double amax, double cfl, double maxdt)
{
    double dt = cfl * h / (c0 + vmax);
    if (amax > 1e-12) { double f = cfl * sqrt(h / amax); dt = f < dt ? f : dt; }
    return dt < maxdt ? dt : maxdt;
}

/* Advances the state in place by one step.  x, v, rho are the float64 state; p and a come back
 * as the step's pressures and accelerations.  Returns the step size. */
double or_step(const StepParams *sp, long n, double *x, double *v, double *rho, const double *m, const double *h,
               const uint8_t *fluid, double *p, double *a)
{
    int dim = sp->dim;
    int64_t *off = (int64_t *)malloc(sizeof(int64_t) * (size_t)(n + 1));
    long total = or_neighbor_list(x, n, dim, 2.0 * sp->hMax, sp->period, off, NULL);
    int32_t *nbr = (int32_t *)malloc(sizeof(int32_t) * (size_t)(total > 0 ? total : 1));
    or_neighbor_list(x, n, dim, 2.0 * sp->hMax, sp->period, off, nbr);
    Sys s = {dim, sp->kind, sp->period, x, h, fluid, m, off, nbr};

    double *tmp = (double *)malloc(sizeof(double) * (size_t)n * 9);
    double *G = NULL, *L = NULL, *gr = NULL;
    /* The energy budget (src/pysurf/sphGpu.py:1046-1186, 1189-1230): each term's energy, in the
     * order pressureFluid, viscosityFluid, pressureWall, viscosityWall, gravityWork, continuityFluid,
     * continuityWall, correction, diffusion, floor, drift, clamp, shifting, filter. */
    double *E = sp->energy, scale = sp->c0 * sp->c0 / 7.0;
    double *accParts = E ? (double *)calloc((size_t)n * 4 * dim, sizeof(double)) : NULL;
    double *rateParts = E ? (double *)calloc((size_t)n * 4, sizeof(double)) : NULL;
    if (sp->filterDensity) {
        or_shepard(&s, n, rho, tmp);
        for (long i = 0; i < n; ++i) {
            if (!fluid[i]) continue;
            if (E) E[13] += m[i] * (elastic_energy(tmp[i], sp->rho0, scale, sp->tension)
                                    - elastic_energy(rho[i], sp->rho0, scale, sp->tension));
            rho[i] = tmp[i];
        }
    }
    or_equation_of_state(n, rho, fluid, sp->rho0, sp->c0, sp->tension, p);
    if (sp->wallExtrapolated) {
        double *pw = (double *)malloc(sizeof(double) * (size_t)n), *rw = (double *)malloc(sizeof(double) * (size_t)n);
        or_wall_pressure(&s, n, rho, p, sp->g, sp->rho0, sp->c0, pw, rw);
        memcpy(p, pw, sizeof(double) * (size_t)n);
        memcpy(rho, rw, sizeof(double) * (size_t)n);
        free(pw); free(rw);
    }
    double *alphas = NULL, *deltas = NULL;
    if (sp->limited || sp->closure) {
        G = (double *)malloc(sizeof(double) * (size_t)n * dim * dim);
        or_velocity_gradients(&s, n, v, rho, G);
    }
    if (sp->closure) {
        /* the coefficients come from the step's starting velocities; the diffusion reuses them */
        alphas = (double *)malloc(sizeof(double) * (size_t)n);
        deltas = (double *)malloc(sizeof(double) * (size_t)n);
        or_closure_coefficients(&s, n, G, sp->c0, alphas, deltas);
    }
    AccelParams ap = {sp->c0, sp->alpha, sp->boundaryFactor, {sp->g[0], sp->g[1], sp->g[2]}, sp->limited,
                      sp->closure, 2.0 * (dim + 2) * sp->viscosity / sp->c0, sp->rho0, alphas, accParts};
    or_accelerations(&s, n, v, rho, p, G, &ap, a);
    double vmax = 0.0, amax = 0.0;
    for (long i = 0; i < n; ++i) {
        if (!fluid[i]) continue;
        double sv = 0.0, sa = 0.0;
        for (int c = 0; c < dim; ++c) { sv += v[i * dim + c] * v[i * dim + c]; sa += a[i * dim + c] * a[i * dim + c]; }
        sv = sqrt(sv); sa = sqrt(sa);
        vmax = sv > vmax ? sv : vmax; amax = sa > amax ? sa : amax;
    }
    double dt = cfl_time_step(sp->hMin, sp->c0, vmax, amax, sp->cfl, sp->maxTimeStep);
    for (long i = 0; i < n; ++i) {
        if (!fluid[i]) continue;
        double mean[MAXD];
        for (int c = 0; c < dim; ++c) {
            double start = v[i * dim + c];
            v[i * dim + c] += a[i * dim + c] * dt;
            mean[c] = 0.5 * (start + v[i * dim + c]);
        }
        if (!E) continue;
        /* work m a . (v + v') / 2 dt of each part of a, and of gravity */
        for (int q = 0; q < 4; ++q) {
            double w = 0.0;
            for (int c = 0; c < dim; ++c) w += accParts[(i * 4 + q) * dim + c] * mean[c];
            E[q] += m[i] * w * dt;
        }
        double w = 0.0;
        for (int c = 0; c < dim; ++c) w += sp->g[c] * mean[c];
        E[4] += m[i] * w * dt;
    }
    int renormalized = sp->diffusion == 3;
    if (sp->corrected || renormalized) {
        L = (double *)malloc(sizeof(double) * (size_t)n * dim * dim);
        or_correction_matrices(&s, n, rho, L);
    }
    if (renormalized) {
        gr = (double *)malloc(sizeof(double) * (size_t)n * dim);
        or_density_gradients(&s, n, rho, L, gr);
    }
    ContinuityParams cp = {sp->diffusion, sp->delta, sp->c0, sp->rho0, fabs(sp->g[dim - 1]), sp->corrected,
                           sp->closure, deltas, rateParts};
    or_continuity(&s, n, v, rho, L, gr, &cp, tmp);
    for (long i = 0; i < n; ++i) {
        double start = rho[i];
        rho[i] += tmp[i] * dt;
        double unfloored = rho[i];
        if (sp->densityFloor > 0.0 && fluid[i] && rho[i] < sp->densityFloor) rho[i] = sp->densityFloor;
        if (E && fluid[i]) {
            /* each part of the rate over the secant slope of e, and the floor's change */
            double slope = elastic_slope(start, unfloored, sp->rho0, scale, sp->tension);
            for (int q = 0; q < 4; ++q) E[5 + q] += m[i] * slope * rateParts[i * 4 + q] * dt;
            E[9] += m[i] * (elastic_energy(rho[i], sp->rho0, scale, sp->tension)
                            - elastic_energy(unfloored, sp->rho0, scale, sp->tension));
        }
    }
    const double *transport = v;
    double *xs = NULL;
    if (sp->xsphEpsilon > 0.0) {
        xs = (double *)malloc(sizeof(double) * (size_t)n * dim);
        or_xsph(&s, n, v, rho, sp->xsphEpsilon, xs);
        transport = xs;
    }
    double *start = NULL, *shift = NULL, *drho = NULL, *dvel = NULL;
    if (sp->shifting) {
        /* the shift takes the step's starting geometry (the pairs of its grid), the updated densities
         * and the kicked velocities (src/pysurf/sphSolver.py:1760-1785) */
        start = (double *)malloc(sizeof(double) * (size_t)n * dim);
        memcpy(start, x, sizeof(double) * (size_t)n * dim);
    }
    for (long i = 0; i < n; ++i) {
        if (!fluid[i]) continue;
        double gx = 0.0;
        for (int c = 0; c < dim; ++c) {
            double start = x[i * dim + c];
            x[i * dim + c] += transport[i * dim + c] * dt;
            gx += sp->g[c] * (x[i * dim + c] - start);
        }
        if (E) E[10] -= m[i] * gx;
    }
    if (sp->shifting) {
        Sys s0 = {dim, sp->kind, sp->period, start, h, fluid, m, off, nbr};
        double *grad = (double *)malloc(sizeof(double) * (size_t)n * dim * 3), *plain = grad + (size_t)n * dim;
        double *rg = plain + (size_t)n * dim, *div = (double *)malloc(sizeof(double) * (size_t)n * 2);
        double *size = div + n;
        shift = (double *)malloc(sizeof(double) * (size_t)n * dim * 2);
        dvel = shift + (size_t)n * dim;
        drho = (double *)malloc(sizeof(double) * (size_t)n);
        or_shifting_fields(&s0, n, rho, sp->spacingKernel, grad, plain, div, rg);
        for (long i = 0; i < n; ++i) {
            double speed = 0.0;
            for (int c = 0; c < dim; ++c) speed += v[i * dim + c] * v[i * dim + c];
            size[i] = sp->shiftLocal ? 2.0 * h[i] * sqrt(speed) * dt
                                     : (sp->c0 * dt / h[i]) * sp->shiftMach * (2.0 * h[i]) * (2.0 * h[i]);
        }
        or_shift(&s0, n, rho, v, grad, plain, div, rg, size, sp->shiftThreshold, sp->lopsidedness, shift, drho, dvel);
        for (long i = 0; i < n; ++i) {
            if (!fluid[i]) continue;
            double k0 = 0.0, k1 = 0.0, gs = 0.0, rho0i = rho[i];
            for (int c = 0; c < dim; ++c) {
                k0 += v[i * dim + c] * v[i * dim + c];
                x[i * dim + c] += shift[i * dim + c];
                v[i * dim + c] += dvel[i * dim + c];
                k1 += v[i * dim + c] * v[i * dim + c];
                gs += sp->g[c] * shift[i * dim + c];
            }
            rho[i] += drho[i];
            if (E) E[12] += m[i] * (0.5 * (k1 - k0) + elastic_energy(rho[i], sp->rho0, scale, sp->tension)
                                    - elastic_energy(rho0i, sp->rho0, scale, sp->tension) - gs);
        }
        free(grad); free(div);
    }
    for (long i = 0; i < n; ++i)
        if (fluid[i] && sp->period > 0.0) x[i * dim + 1] -= sp->period * floor(x[i * dim + 1] / sp->period);
    double *before = NULL;
    if (E && sp->boundaryKind) {
        before = (double *)malloc(sizeof(double) * (size_t)n * dim * 2);
        memcpy(before, x, sizeof(double) * (size_t)n * dim);
        memcpy(before + (size_t)n * dim, v, sizeof(double) * (size_t)n * dim);
    }
    if (sp->boundaryKind == 1) or_enforce_container(n, dim, x, v, fluid, sp->lower, sp->upper, sp->openTop);
    else if (sp->boundaryKind == 2) or_enforce_bed(n, dim, x, v, fluid, &sp->bed);
    else if (sp->boundaryKind == 3) or_enforce_heightfield(n, x, v, fluid, &sp->field);
    if (before) {
        /* the enforcement's change of kinetic and potential energy (clampEnergy) */
        const double *x0 = before, *v0 = before + (size_t)n * dim;
        for (long i = 0; i < n; ++i) {
            if (!fluid[i]) continue;
            double dk = 0.0, gx = 0.0;
            for (int c = 0; c < dim; ++c) {
                long k = i * dim + c;
                dk += v[k] * v[k] - v0[k] * v0[k];
                gx += sp->g[c] * (x[k] - x0[k]);
            }
            E[11] += m[i] * (0.5 * dk - gx);
        }
        free(before);
    }
    free(accParts); free(rateParts);
    free(off); free(nbr); free(tmp); free(G); free(L); free(gr); free(xs); free(alphas); free(deltas);
    free(start); free(shift); free(drho);
    return dt;
}

/* Thin exported wrappers that take a Sys by fields, for ctypes. */
#define SYS_ARGS int dim, int kind, double period, const double *x, const double *h, const uint8_t *fluid, \
                 const double *m, const int64_t *off, const int32_t *nbr
#define SYS_MAKE Sys s = {dim, kind, period, x, h, fluid, m, off, nbr}

void orx_wall_pressure(SYS_ARGS, long n, const double *rho, const double *p, const double *g, double rho0, double c0,
                       double *pOut, double *rhoOut)
{ SYS_MAKE; or_wall_pressure(&s, n, rho, p, g, rho0, c0, pOut, rhoOut); }

void orx_velocity_gradients(SYS_ARGS, long n, const double *v, const double *rho, double *G)
{ SYS_MAKE; or_velocity_gradients(&s, n, v, rho, G); }

void orx_correction_matrices(SYS_ARGS, long n, const double *rho, double *L)
{ SYS_MAKE; or_correction_matrices(&s, n, rho, L); }

void orx_density_gradients(SYS_ARGS, long n, const double *rho, const double *L, double *out)
{ SYS_MAKE; or_density_gradients(&s, n, rho, L, out); }

void orx_accelerations(SYS_ARGS, long n, const double *v, const double *rho, const double *p, const double *G,
                       double c0, double alpha, double boundaryFactor, const double *g, int limited, int closure,
                       double waterTerm, double rho0, const double *alphas, double *a)
{
    SYS_MAKE;
    AccelParams ap = {c0, alpha, boundaryFactor, {g[0], g[1], dim == 3 ? g[2] : 0.0}, limited, closure, waterTerm,
                      rho0, alphas};
    or_accelerations(&s, n, v, rho, p, G, &ap, a);
}

void orx_continuity(SYS_ARGS, long n, const double *v, const double *rho, const double *L, const double *gradRho,
                    int mode, double delta, double c0, double rho0, double gravity, int corrected, int closure,
                    const double *deltas, double *out)
{
    SYS_MAKE;
    ContinuityParams cp = {mode, delta, c0, rho0, gravity, corrected, closure, deltas};
    or_continuity(&s, n, v, rho, L, gradRho, &cp, out);
}

void orx_closure_coefficients(SYS_ARGS, long n, const double *G, double c0, double *alphas, double *deltas)
{ SYS_MAKE; or_closure_coefficients(&s, n, G, c0, alphas, deltas); }

double orx_kernel_value(int kind, int dim, double r, double h) { return kernel_value(kind, dim, r, h); }

void orx_shifting_fields(SYS_ARGS, long n, const double *rho, double spacingKernel, double *grad, double *plain,
                         double *div, double *rhoGrad)
{ SYS_MAKE; or_shifting_fields(&s, n, rho, spacingKernel, grad, plain, div, rhoGrad); }

void orx_shift(SYS_ARGS, long n, const double *rho, const double *v, const double *grad, const double *plain,
               const double *div, const double *rhoGrad, const double *size, double threshold, double lopsidedness,
               double *shift, double *drho, double *dv)
{ SYS_MAKE; or_shift(&s, n, rho, v, grad, plain, div, rhoGrad, size, threshold, lopsidedness, shift, drho, dv); }

void orx_xsph(SYS_ARGS, long n, const double *v, const double *rho, double eps, double *out)
{ SYS_MAKE; or_xsph(&s, n, v, rho, eps, out); }

void orx_shepard(SYS_ARGS, long n, const double *rho, double *out)
{ SYS_MAKE; or_shepard(&s, n, rho, out); }

long orx_step_size(void) { return (long)sizeof(StepParams); }
long orx_bed_offset(void) { return (long)offsetof(StepParams, bed); }
long orx_field_offset(void) { return (long)offsetof(StepParams, field); }
