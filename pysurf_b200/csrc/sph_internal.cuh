// sph_internal.cuh -- shared types and device helpers of the B200 delta-SPH backend.
//
// Layout in HBM (all arrays in the current sort order, slot s = 0..n-1):
//   master float64 state, double-buffered so a re-sort is one gather:
//     x[a], v[a] (a < dim), rho            integrated in float64, as the reference integrates
//   per-particle constants carried through each re-sort:
//     m, h (float64), fluid (uint8), orig (int32: the caller's index of the slot)
//   the sweeps' float32 frame, rebuilt from the master each step:
//     pa   float4  2D (hx, hy, lx, ly)      3D (hx, hy, hz, hs)
//     pb   float4  2D (m, hs, dev, V)       3D (lx, ly, lz, m)
//     kin  float4  2D (vx, vy, rho, P2)     3D (vx, vy, vz, rho)
//     aux  float4  3D (P2, dev, V, -)
//     low  float4  (vlx, vly, vlz, devLo): the float32 remainders of the float64 velocity and deviation
//     pres float   the pressure p
//   hi + lo is each float64 coordinate split into a float32 point and its float32 remainder, so a
//   separation (hi_i - hi_j) + (lo_i - lo_j) keeps the float64 positions' digits without float64
//   arithmetic (src/pysurf/sphGpu.py:227-242 states the same split).  hs is +h for a fluid
//   particle and -h for a boundary particle; dev is rho - rho0 in float32, taken in float64
//   (src/pysurf/sphGpu.py:1031-1038), so neighbours' density differences keep their digits.
//   The continuity sweep takes velocity and deviation differences from the float32 values and their
//   remainders, (v_i - v_j) + (vl_i - vl_j), so they keep float64's digits: continuity sums terms
//   that cancel (the velocity's divergence next to a wall, the hydrostatic subtraction near rest),
//   where a float32 value's rounding would otherwise dominate the rate.
//   V = m / rho and P2 = p / rho^2 are each particle's own, taken once per step instead of once per
//   pair: the same float32 quotients the pair sums would take.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace sph {

constexpr int kBlock = 128;                 // threads per sweep block
#ifndef SPH_SWEEP_MIN_BLOCKS
#define SPH_SWEEP_MIN_BLOCKS 8
#endif
#ifndef SPH_SWEEP_MIN_BLOCKS_3D
#define SPH_SWEEP_MIN_BLOCKS_3D 6
#endif
// Resident sweep blocks an SM, which caps a sweep's registers: in 2D 8 blocks of 128 (64 registers)
// give the warps that hide the neighbours' load latency; the 3D sweeps' 3 x 3 sums want about 105
// registers, and 6 blocks (80 registers, a few spilled) ran faster than 4 (none spilled) or 5.
template <int D>
constexpr int sweepMinBlocks() { return D == 2 ? SPH_SWEEP_MIN_BLOCKS : SPH_SWEEP_MIN_BLOCKS_3D; }
constexpr float kViscositySoftening = 0.01f;   // mu_ij's r^2 + 0.01 h^2 (src/pysurf/sphSolver.py:213)
constexpr float kCloseDistance = 0.3f;      // limiter fade (src/pysurf/sphSolver.py:220-221)
constexpr float kFoldWidth = 0.2f;
constexpr float kCandidateMargin = 1.0001f; // on r^2, as the reference's coarse test (src/pysurf/sphGpu.py:99)

// Error flags the device raises; the host reads them after each call that syncs.
enum DeviceError : int {
    kErrNonFinite = 1,      // a position, velocity or density stopped being finite
    kErrTimeStep = 2,       // the step collapsed (dt not positive and finite)
};

// Everything a sweep needs besides the arrays; passed by value.
struct Params {
    int n;                  // particles
    int dim;
    int kind;               // 0 cubic spline, 1 Wendland C2
    int mixedH;             // particles carry different smoothing lengths
    float hMax;             // longest smoothing length, sizes the cells
    float sigmaUnit;        // kernel sigma at h = 1
    // grid: cell c = (cz * ny + cy) * nx + cx, x fastest; coordinates clamped onto the grid
    double origin[3];
    double cellWidth;
    int nc[3];
    int ncs;                // cells per support: the stencil is +-ncs cells
    int precise;            // separations from point + remainder (1) or the float32 points alone (0)
    // the fine level, for mixed smoothing lengths: a particle whose h is below fineBelow is sorted
    // into a second grid of fineWidth-wide cells (ncs to the fine level's longest h, fineMax),
    // numbered from fineFirst after the coarse grid's; a particle searches each grid only as far as
    // that grid's particles reach.  levels is 1 when no particle is on the fine level.
    int levels;
    double fineOrigin[3];
    double fineWidth;
    int fineNc[3];
    int fineFirst;
    int cells;              // both grids' cells
    float fineMax;
    double fineBelow;
    double period;          // periodic y axis length, 0 for none
    float periodF;
    // physics
    float c0, alpha, boundaryFactor;
    float g[3];
    double rho0, stiffness, densityFloor;  // the equation of state's rho0 and B = rho0 c0^2 / 7
    double devReference;    // the diffusion's rho0: deviations are rho - devReference
    float halfInvRho0;      // 0.5 / devReference: a pair's mean deviation over rho0
    int tension;            // the fluid may carry negative pressure
    int diffusion;          // 0 none, 1 molteni, 2 hydrostatic, 3 antuono
    float diffusionFactor;  // 2 delta c0
    float hydrostaticSlope; // rho0 g / c0^2, rounded once from float64: the hydrostatic density's slope in z
    int corrected;          // continuity takes L_i grad W
    int limited;            // viscosity limiter
    int wallExtrapolated;
    float xsphEpsilon;
    double gravity64[3];
    // delta-LES-SPH closure (src/pysurf/sphSolver.py:1232-1326): the eddy coefficients from the
    // velocity gradients, a viscous term on every fluid pair, the pair's diffusion coefficient
    int closure;
    float waterTerm;        // 2 (dim + 2) nu / c0: the water's own viscosity as an alpha times h
    float closureRho0;
    float closureC0;        // the closure's sound speed: its coefficients and its diffusion's 2 c0
    // particle shifting (src/pysurf/sphSolver.py:824-1010): W(dx) for the anti-clumping weight, the
    // free surface's divergence and lopsidedness thresholds, the size CFL Ma (2h)^2 or 2 h |v| dt
    int shifting, shiftLocal;
    float spacingKernel, shiftThreshold, lopsidedness;
    double shiftScale;      // c0 Ma 4 h: the size CFL Ma (2h)^2 = shiftScale dt
    double shiftDt;         // the host-step call's dt (the device steps take ctl->dt)
    // neighbour table: up to listCap entries a particle (a multiple of 4), entry k of slot i at
    // 4 ((k / 4) listStride + i) + k % 4; listCap 0: no table, the sweeps walk the cells
    int listCap;
    int listStride;
    // energy budget (src/pysurf/sphEnergy.py): each particle's running total of each term, by caller
    // index, column t at t * energyStride; the momentum sweep's parts of a at q * energyStride + slot
    int budget;
    int energyStride;
    // the momentum and continuity sums compensated (never with the budget: its sweeps keep plain sums)
    int compensated;
};

// The float32 frame and the float64 master state, current buffers.
struct Frame {
    float4 *pa, *pb, *kin, *aux;
    float4 *low;            // remainders: velocity (xyz) and deviation (w)
    float *pres;            // pressure
    int *cell;              // sorted cell index of each slot
    const int *cellStart;   // lower bound of each cell in the sorted order, numCells + 1 entries
    float4 *G0, *G1, *G2;   // velocity gradient rows (2D: G0 = (G00, G01, G10, G11))
    float4 *L0, *L1, *L2;   // correction matrix rows, same packing
    float4 *gradRho;        // renormalized density gradient
    float4 *acc;            // acceleration (w: unused)
    float *rate;            // d rho / dt
    float *scalar;          // scratch per particle (Shepard, wall pressure outputs)
    float4 *vec;            // scratch per particle (XSPH transport velocity)
    float2 *eddy;           // closure: each particle's (alpha_i, delta_i)
    // shifting: grad C (w unused), grad C0 (w: div r, -1 where the support is lopsided, 1e6 on the
    // boundary), grad rho; the shift (w: the density change) and the velocity change
    float4 *shiftGrad, *shiftPlain, *shiftRhoGrad, *shift, *shiftDv;
    double *energy;         // energy budget: kEnergyTerms columns, by caller index
    float4 *parts;          // energy budget: pressure and viscosity of a from fluid and from boundary neighbours
    int *nbr;               // neighbour table (chunks of four), top bit: a pair across the periodic seam
    int *ncount;            // each slot's neighbour count (may exceed the table's capacity)
    // master (current buffers)
    double *x[3], *v[3], *rho, *m, *h;
    uint8_t *fluid;
    int *orig;
};

// Step control on the device: the time step is taken from the step's own maxima on the device,
// so a run of steps needs no host round trip (src/pysurf/sphSolver.py:1410-1424, 1980-1989).
struct Control {
    double time, untilTime, dt;
    long long step, lastStep;
    double vmax, amax;          // this step's fluid maxima
    double hMin, cfl, maxTimeStep, soundSpeed;   // the CFL step's inputs, float64 as the host takes them
    int active;                 // this step runs
    int hostDt;                 // dt comes from the host (residentIntegrate), not the maxima
    int filterNow;              // host-driven steps: this step filters the density (Shepard)
    long long filterInterval;   // device loop: filter every this many steps, 0 for none
    unsigned int ticket;        // last-warp-done counter of the maxima reduction
    int error;                  // DeviceError flags
    // the maxima reduction's running values: the bits of non-negative doubles, which order as the
    // doubles do, so an integer atomicMax takes their maximum in any order; zero between steps
    unsigned long long vmaxBits, amaxBits;
};

// ------------------------------------------------------------------------------------------
// Kernels W and (dW/dr) / r: src/pysurf/sphKernels.py:108-648; src/pysurf/sphGpu.py:139-204.
// The pair sums only ever take dW/dr divided by r (grad W = (dW/dr) r_ij / r), which for the
// Wendland C2 is -5 sigma (1 - q/2)^3 / h^2 with no division by r, and for the cubic spline
// sigma (2.25 q - 3) / h^2 inside q < 1.  The constants depend on h alone, so with one smoothing
// length they are taken once per thread.
// ------------------------------------------------------------------------------------------

struct KernelAt {
    float invH;     // 1 / h
    float sigma;    // sigma at h
    float gradC;    // Wendland: -5 sigma / h^2; cubic: sigma / h^2
    float soft;     // the viscosity's and the diffusion's softening 0.01 h^2
};

template <int K, int D>
__device__ __forceinline__ KernelAt kernelAt(float unit, float h)
{
    KernelAt k;
    k.invH = 1.0f / h;
    float s = unit * k.invH * k.invH;
    if (D == 3) s *= k.invH;
    k.sigma = s;
    k.gradC = (K == 1 ? -5.0f : 1.0f) * s * k.invH * k.invH;
    k.soft = kViscositySoftening * h * h;
    return k;
}

// A pair's kernel constants at h_ij: one set a thread when every particle has the same smoothing
// length (then h_ij = hMax), else taken per pair.  HOLD (mixed lengths): the set is held at the
// particle's own length instead, which every pair with a neighbour of the same length has
// (0.5 (h + h) = h exactly), so those pairs, all but the few across a refinement zone's edge, take
// the held set and the rest take theirs per pair, with the same bits either way.  It pays where a
// sweep has registers to spare (measured: the refined 3D ridge's gradients 10.2 -> 9.7 ms, while
// continuity, at its register cap, went 11.5 -> 12.2).
template <int K, int D, bool HOLD = false>
struct Smoothing {
    KernelAt fixed;
    float held;     // the length `fixed` is taken at
    float unit;
    bool mixed;
    __device__ __forceinline__ static float heldLength(const Params &P, float own)
    {
        return HOLD && P.mixedH && own > 0.0f ? own : P.hMax;
    }
    // own: the particle's smoothing length (HOLD only)
    __device__ __forceinline__ explicit Smoothing(const Params &P, float own = 0.0f)
        : fixed(kernelAt<K, D>(P.sigmaUnit, heldLength(P, own))), held(heldLength(P, own)), unit(P.sigmaUnit),
          mixed(P.mixedH != 0) {}
    __device__ __forceinline__ KernelAt at(float h) const
    {
        if constexpr (HOLD) {
            if (h == held) return fixed;
            return kernelAt<K, D>(unit, h);
        } else {
            return mixed ? kernelAt<K, D>(unit, h) : fixed;
        }
    }
};

// W(q h), q < 2.
template <int K>
__device__ __forceinline__ float kernelValue(float q, const KernelAt &k)
{
    if (K == 1) {
        float rest = 1.0f - 0.5f * q, sq = rest * rest;
        return k.sigma * sq * sq * (2.0f * q + 1.0f);
    }
    if (q < 1.0f) return k.sigma * (1.0f - 1.5f * q * q + 0.75f * q * q * q);
    float rest = 2.0f - q;
    return k.sigma * 0.25f * rest * rest * rest;
}

// (dW/dr) / r at r = q h, 0 < q < 2.
template <int K>
__device__ __forceinline__ float kernelGradient(float q, const KernelAt &k)
{
    if (K == 1) {
        float rest = 1.0f - 0.5f * q;
        return k.gradC * rest * rest * rest;
    }
    if (q < 1.0f) return k.gradC * (2.25f * q - 3.0f);
    float rest = 2.0f - q;
    return __fdividef(-0.75f * k.gradC * rest * rest, q);
}

// (dW/dr) / r in float64 at a pair's float64 distance r, with the pair's (float32) kernel constants:
// the continuity sweep's wall pairs, whose terms cancel across a particle's neighbours, so each
// term's own rounding must stay well below float32's.
template <int K>
__device__ __forceinline__ double kernelGradient64(double r, const KernelAt &k)
{
    const double q = r * (double)k.invH;
    if (K == 1) {
        const double rest = 1.0 - 0.5 * q;
        return (double)k.gradC * rest * rest * rest;
    }
    if (q < 1.0) return (double)k.gradC * (2.25 * q - 3.0);
    const double rest = 2.0 - q;
    return -0.75 * (double)k.gradC * rest * rest / q;
}

__device__ __forceinline__ float sigmaAt(float unit, float h, int dim)
{
    return dim == 2 ? unit / (h * h) : unit / (h * h * h);
}

__device__ __forceinline__ int clampi(int a, int lo, int hi) { return a < lo ? lo : (a > hi ? hi : a); }

// Tait pressure B ((rho / rho0)^7 - 1), the power as three multiplies, clamped at zero unless the
// fluid may carry tension (src/pysurf/sphGpu.py:1058-1070).
__device__ __forceinline__ double taitPressure(const Params &P, double rho, bool fluid)
{
    double ratio = rho / P.rho0, sq = ratio * ratio;
    double p = P.stiffness * (sq * sq * sq * ratio - 1.0);
    if (!P.tension || !fluid) p = p > 0.0 ? p : 0.0;
    return p;
}

// The energy budget's terms, the columns of F.energy (src/pysurf/sphEnergy.py:92-98, deviceTerms).
enum EnergyTerm {
    kPressureFluid, kViscosityFluid, kPressureWall, kViscosityWall, kGravityWork, kContinuityFluid,
    kContinuityWall, kCorrection, kDiffusion, kFloor, kDrift, kClamp, kShifting, kFilter, kEnergyTerms
};

// e(rho), the Tait equation of state's elastic energy per unit mass (src/pysurf/sphEnergy.py:100-139):
// (c0^2 / 7) x^2 (21 + 35 x + 35 x^2 + 21 x^3 + 7 x^4 + x^5) / (6 (1 + x)), x = rho / rho0 - 1, so no
// digits cancel near rho0; zero below rho0 unless the fluid carries tension.
__device__ __forceinline__ double elasticEnergy(const Params &P, double rho)
{
    const double x = rho / P.rho0 - 1.0;
    if (!P.tension && x < 0.0) return 0.0;
    const double poly = 21.0 + x * (35.0 + x * (35.0 + x * (21.0 + x * (7.0 + x))));
    return (P.stiffness / P.rho0) * x * x * poly / (6.0 * (1.0 + x));
}

// The secant slope (e(after) - e(before)) / (after - before), or p / rho^2 at the midpoint for a
// change under 1e-10 rho0, where the two energies would lose their digits (src/pysurf/sphEnergy.py:141-160).
__device__ __forceinline__ double elasticSlope(const Params &P, double before, double after)
{
    const double change = after - before;
    if (fabs(change) > 1e-10 * P.rho0) return (elasticEnergy(P, after) - elasticEnergy(P, before)) / change;
    const double middle = 0.5 * (before + after);
    return taitPressure(P, middle, true) / (middle * middle);
}

// Adds to a fluid slot's running total of one term of the budget.
__device__ __forceinline__ void addEnergy(const Params &P, const Frame &F, int i, int term, double value)
{
    F.energy[(size_t)term * P.energyStride + F.orig[i]] += value;
}

// Cell coordinate of a float64 coordinate along an axis, clamped onto the grid.  Clamping is
// monotone and never parts two cells further than they were, so the +-ncs stencil still finds
// every neighbour of a particle outside the grid; only its candidates grow.
__device__ __forceinline__ int cellCoordinate(double value, double origin, double width, int count)
{
    double f = floor((value - origin) / width);
    if (!(f >= 0.0)) return 0;      // below the grid, or not a number: never an index outside it
    if (f > (double)(count - 1)) return count - 1;
    return (int)f;
}

// A box of cells of one grid around a centre cell, clamped to the grid: rows (y, z) of the
// x range [x0, x1]; the grid's cells are numbered from `first`, x fastest.
struct CellBox {
    int first, nx, ny;
    int cx, cy, cz;
    int x0, x1, y0, y1, z0, z1;
};

// The half-width in cells of a particle's search of a level's grid: the coarse grid's ncs (its
// cells are 2 hMax / ncs wide, and no pair reaches past 2 hMax), the fine grid's as many cells as
// hI + fineMax, the farthest a fine neighbour can be, spans.
__device__ __forceinline__ int searchCells(const Params &P, int level, float hI)
{
    if (level == 0) return P.ncs;
    return (int)ceil(((double)hI + (double)P.fineMax) / P.fineWidth - 1e-9);
}

// The box of +-n cells of a level's grid (0 coarse, 1 fine) around the cell holding pos; in the
// particle's own grid the centre is its sorted cell ownCell (y taken from pos when `image`, the
// search of a periodic image).  single: there is one level, so the own grid is the searched one.
__device__ __forceinline__ CellBox cellBox(const Params &P, int level, int ownCell, const double pos[3], bool image,
                                           int dim, int n, bool single = false)
{
    CellBox B;
    const bool fine = level == 1;
    B.nx = fine ? P.fineNc[0] : P.nc[0];
    B.ny = fine ? P.fineNc[1] : P.nc[1];
    const int nz = fine ? P.fineNc[2] : P.nc[2];
    B.first = fine ? P.fineFirst : 0;
    const double width = fine ? P.fineWidth : P.cellWidth;
    const double *origin = fine ? P.fineOrigin : P.origin;
    if (single || (ownCell >= P.fineFirst) == fine) {
        const int local = ownCell - B.first;
        B.cx = local % B.nx;
        B.cy = (local / B.nx) % B.ny;
        B.cz = local / (B.nx * B.ny);
        if (image) B.cy = cellCoordinate(pos[1], origin[1], width, B.ny);
    } else {
        B.cx = cellCoordinate(pos[0], origin[0], width, B.nx);
        B.cy = cellCoordinate(pos[1], origin[1], width, B.ny);
        B.cz = dim == 3 ? cellCoordinate(pos[2], origin[2], width, nz) : 0;
    }
    B.x0 = max(B.cx - n, 0);
    B.x1 = min(B.cx + n, B.nx - 1);
    B.y0 = max(B.cy - n, 0);
    B.y1 = min(B.cy + n, B.ny - 1);
    B.z0 = dim == 3 ? max(B.cz - n, 0) : 0;
    B.z1 = dim == 3 ? min(B.cz + n, nz - 1) : 0;
    return B;
}

// ------------------------------------------------------------------------------------------
// Frame access per dimension.
// ------------------------------------------------------------------------------------------

// A particle's signed smoothing length (+h fluid, -h boundary).
template <int D> __device__ __forceinline__ float signedLength(const Frame &F, int j);
template <> __device__ __forceinline__ float signedLength<2>(const Frame &F, int j) { return __ldg(&F.pb[j].y); }
template <> __device__ __forceinline__ float signedLength<3>(const Frame &F, int j) { return __ldg(&F.pa[j].w); }

template <int D> __device__ __forceinline__ float massOf(const Frame &F, int j);
template <> __device__ __forceinline__ float massOf<2>(const Frame &F, int j) { return __ldg(&F.pb[j].x); }
template <> __device__ __forceinline__ float massOf<3>(const Frame &F, int j) { return __ldg(&F.pb[j].w); }

template <int D> __device__ __forceinline__ float pressureOf(const Frame &F, int j) { return __ldg(&F.pres[j]); }

// p / rho^2
template <int D> __device__ __forceinline__ float pressureRatioOf(const Frame &F, int j);
template <> __device__ __forceinline__ float pressureRatioOf<2>(const Frame &F, int j) { return __ldg(&F.kin[j].w); }
template <> __device__ __forceinline__ float pressureRatioOf<3>(const Frame &F, int j) { return __ldg(&F.aux[j].x); }

template <int D> __device__ __forceinline__ float deviationOf(const Frame &F, int j);
template <> __device__ __forceinline__ float deviationOf<2>(const Frame &F, int j) { return __ldg(&F.pb[j].z); }
template <> __device__ __forceinline__ float deviationOf<3>(const Frame &F, int j) { return __ldg(&F.aux[j].y); }

// m / rho
template <int D> __device__ __forceinline__ float volumeOf(const Frame &F, int j);
template <> __device__ __forceinline__ float volumeOf<2>(const Frame &F, int j) { return __ldg(&F.pb[j].w); }
template <> __device__ __forceinline__ float volumeOf<3>(const Frame &F, int j) { return __ldg(&F.aux[j].z); }

template <int D> __device__ __forceinline__ float densityOf(const Frame &F, int j);
template <> __device__ __forceinline__ float densityOf<2>(const Frame &F, int j) { return __ldg(&F.kin[j].z); }
template <> __device__ __forceinline__ float densityOf<3>(const Frame &F, int j) { return __ldg(&F.kin[j].w); }

// A neighbour's values from its rows, each row loaded once a pair: pa (A), pb (B), kin (K) and, in
// 3D, aux (X).
template <int D> __device__ __forceinline__ float4 auxRow(const Frame &F, int j)
{
    return D == 3 ? __ldg(&F.aux[j]) : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
}
template <int D> __device__ __forceinline__ float signedLengthIn(const float4 &A, const float4 &B)
{ return D == 2 ? B.y : A.w; }
template <int D> __device__ __forceinline__ float massIn(const float4 &B) { return D == 2 ? B.x : B.w; }
template <int D> __device__ __forceinline__ float volumeIn(const float4 &B, const float4 &X)
{ return D == 2 ? B.w : X.z; }
template <int D> __device__ __forceinline__ float deviationIn(const float4 &B, const float4 &X)
{ return D == 2 ? B.z : X.y; }
template <int D> __device__ __forceinline__ float densityIn(const float4 &K) { return D == 2 ? K.z : K.w; }
template <int D> __device__ __forceinline__ float pressureRatioIn(const float4 &K, const float4 &X)
{ return D == 2 ? K.w : X.x; }
template <int D> __device__ __forceinline__ void pointIn(const float4 &A, float p[3])
{
    p[0] = A.x; p[1] = A.y; p[2] = D == 3 ? A.z : 0.0f;
}
template <int D> __device__ __forceinline__ void remainderIn(const float4 &A, const float4 &B, float l[3])
{
    if (D == 2) { l[0] = A.z; l[1] = A.w; l[2] = 0.0f; }
    else { l[0] = B.x; l[1] = B.y; l[2] = B.z; }
}
template <int D> __device__ __forceinline__ void velocityIn(const float4 &K, float v[3])
{
    v[0] = K.x; v[1] = K.y; v[2] = D == 3 ? K.z : 0.0f;
}

// Write a slot's density-derived fields: rho, rho - rho0, V = m / rho, p, p / rho^2.
template <int D>
__device__ __forceinline__ void storeDensity(const Frame &F, int i, float m, double rho64, double devReference, float p)
{
    const double dev64 = rho64 - devReference;
    const float rho = (float)rho64, dev = (float)dev64;
    const float volume = m / rho, ratio = p / (rho * rho);
    F.pres[i] = p;
    F.low[i].w = (float)(dev64 - (double)dev);
    if (D == 2) {
        F.kin[i].z = rho; F.kin[i].w = ratio;
        F.pb[i].z = dev; F.pb[i].w = volume;
    } else {
        F.kin[i].w = rho;
        F.aux[i] = make_float4(ratio, dev, volume, 0.0f);
    }
}

// Velocity (float32) of slot j.
template <int D> __device__ __forceinline__ void velocityOf(const Frame &F, int j, float v[3])
{
    float4 k = __ldg(&F.kin[j]);
    v[0] = k.x; v[1] = k.y; v[2] = D == 3 ? k.z : 0.0f;
}

// Candidate coordinates (the float32 points alone) and the remainders.
template <int D> __device__ __forceinline__ void pointOf(const Frame &F, int j, float p[3]);
template <> __device__ __forceinline__ void pointOf<2>(const Frame &F, int j, float p[3])
{
    float4 a = __ldg(&F.pa[j]); p[0] = a.x; p[1] = a.y; p[2] = 0.0f;
}
template <> __device__ __forceinline__ void pointOf<3>(const Frame &F, int j, float p[3])
{
    float4 a = __ldg(&F.pa[j]); p[0] = a.x; p[1] = a.y; p[2] = a.z;
}

template <int D> __device__ __forceinline__ void remainderOf(const Frame &F, int j, float l[3]);
template <> __device__ __forceinline__ void remainderOf<2>(const Frame &F, int j, float l[3])
{
    float4 a = __ldg(&F.pa[j]); l[0] = a.z; l[1] = a.w; l[2] = 0.0f;
}
template <> __device__ __forceinline__ void remainderOf<3>(const Frame &F, int j, float l[3])
{
    float4 b = __ldg(&F.pb[j]); l[0] = b.x; l[1] = b.y; l[2] = b.z;
}

// Matrix rows (dim x dim) packed in float4 rows.
template <int D> __device__ __forceinline__ void loadMatrix(const float4 *R0, const float4 *R1, const float4 *R2,
                                                            int j, float M[3][3]);
template <> __device__ __forceinline__ void loadMatrix<2>(const float4 *R0, const float4 *, const float4 *, int j,
                                                          float M[3][3])
{
    float4 a = __ldg(&R0[j]);
    M[0][0] = a.x; M[0][1] = a.y; M[1][0] = a.z; M[1][1] = a.w;
}
template <> __device__ __forceinline__ void loadMatrix<3>(const float4 *R0, const float4 *R1, const float4 *R2, int j,
                                                          float M[3][3])
{
    float4 a = __ldg(&R0[j]), b = __ldg(&R1[j]), c = __ldg(&R2[j]);
    M[0][0] = a.x; M[0][1] = a.y; M[0][2] = a.z;
    M[1][0] = b.x; M[1][1] = b.y; M[1][2] = b.z;
    M[2][0] = c.x; M[2][1] = c.y; M[2][2] = c.z;
}

template <int D> __device__ __forceinline__ void storeMatrix(float4 *R0, float4 *R1, float4 *R2, int j,
                                                             const float M[3][3]);
template <> __device__ __forceinline__ void storeMatrix<2>(float4 *R0, float4 *, float4 *, int j, const float M[3][3])
{
    R0[j] = make_float4(M[0][0], M[0][1], M[1][0], M[1][1]);
}
template <> __device__ __forceinline__ void storeMatrix<3>(float4 *R0, float4 *R1, float4 *R2, int j,
                                                           const float M[3][3])
{
    R0[j] = make_float4(M[0][0], M[0][1], M[0][2], 0.0f);
    R1[j] = make_float4(M[1][0], M[1][1], M[1][2], 0.0f);
    R2[j] = make_float4(M[2][0], M[2][1], M[2][2], 0.0f);
}

template <int D, class R> __device__ __forceinline__ R determinant(const R M[3][3])
{
    if (D == 2) return M[0][0] * M[1][1] - M[0][1] * M[1][0];
    return M[0][0] * (M[1][1] * M[2][2] - M[1][2] * M[2][1]) - M[0][1] * (M[1][0] * M[2][2] - M[1][2] * M[2][0])
         + M[0][2] * (M[1][0] * M[2][1] - M[1][1] * M[2][0]);
}

template <int D, class R> __device__ __forceinline__ void inverse(const R M[3][3], R out[3][3])
{
    R det = determinant<D>(M);
    R s = R(1) / det;
    if (D == 2) {
        out[0][0] = M[1][1] * s; out[0][1] = -M[0][1] * s;
        out[1][0] = -M[1][0] * s; out[1][1] = M[0][0] * s;
        return;
    }
    out[0][0] = (M[1][1] * M[2][2] - M[1][2] * M[2][1]) * s;
    out[0][1] = (M[0][2] * M[2][1] - M[0][1] * M[2][2]) * s;
    out[0][2] = (M[0][1] * M[1][2] - M[0][2] * M[1][1]) * s;
    out[1][0] = (M[1][2] * M[2][0] - M[1][0] * M[2][2]) * s;
    out[1][1] = (M[0][0] * M[2][2] - M[0][2] * M[2][0]) * s;
    out[1][2] = (M[0][2] * M[1][0] - M[0][0] * M[1][2]) * s;
    out[2][0] = (M[1][0] * M[2][1] - M[1][1] * M[2][0]) * s;
    out[2][1] = (M[0][1] * M[2][0] - M[0][0] * M[2][1]) * s;
    out[2][2] = (M[0][0] * M[1][1] - M[0][1] * M[1][0]) * s;
}

}  // namespace sph
