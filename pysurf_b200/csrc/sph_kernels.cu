// sph_kernels.cu -- the B200 kernels of the delta-SPH step.
//
//   cell list      counting sort by cell, each cell's slots in caller-index order -> cell lower
//                  bounds -> one gather that permutes the float64 master and builds the float32
//                  frame (with the Tait pressure, the density deviation, m / rho and p / rho^2)
//   sweeps         A  wall pressure      boundary rows over fluid neighbours
//                  B  gradients          fluid rows: velocity gradient G, correction L, grad rho
//                  C  momentum           fluid rows: pressure, limited viscosity, gravity; the
//                                        fluid maxima reduced per block, the last block takes the
//                                        time step in float64
//                  D  continuity         every row: corrected continuity + delta-SPH diffusion;
//                                        the epilogue advances the density, drifts and enforces
//                  X  XSPH               transport velocity, drift and enforcement (epsilon > 0)
//                  S  Shepard            filtered density (when a filter step is due)
//   pointwise      kick (v += a dt), enforcement, scatter to the caller's order
//
// No float atomics: every sum is a gather in a fixed order (the sorted order of (cell, caller
// index)), so a run is bit-for-bit repeatable and a resumed run follows the uninterrupted one.
#include <math.h>

#include "sph_enforce.cuh"
#include "sph_kernels.h"

namespace sph {

// ------------------------------------------------------------------------------------------
// Cell list
// ------------------------------------------------------------------------------------------

// A counting sort by cell, in four launches:
//   count  each slot's cell, and its place among the slots of that cell in the order the atomics
//          hand places out (an arbitrary order)
//   scan   the cells' lower bounds from the counts (two launches), which also clears the counts
//   place  each slot into its cell's range at that place, with its caller index
//   rank   within each cell, the slots in caller-index order: a slot's rank is the number of its
//          cellmates with a smaller caller index, so the sorted order is (cell, caller index), a
//          function of the state alone
// A cell holds a handful of slots, so the rank's loop over the cell is short; its cost grows with
// the square of a cell's count, as the sweeps' candidate tests over that cell already do.
// A slot whose h is below P.fineBelow goes to the fine grid's cells, numbered after the coarse grid's.
__global__ void cellCountKernel(Params P, int n, const double *x0, const double *x1, const double *x2,
                                const double *h, int *slotCell, int *slotWithin, int *cellCount, const Control *ctl)
{
    if (ctl && !ctl->active) return;
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const bool fine = P.levels > 1 && h[s] < P.fineBelow;
    const double width = fine ? P.fineWidth : P.cellWidth;
    const double *origin = fine ? P.fineOrigin : P.origin;
    const int *nc = fine ? P.fineNc : P.nc;
    int cx = cellCoordinate(x0[s], origin[0], width, nc[0]);
    int cy = cellCoordinate(x1[s], origin[1], width, nc[1]);
    int cz = P.dim == 3 ? cellCoordinate(x2[s], origin[2], width, nc[2]) : 0;
    int c = (fine ? P.fineFirst : 0) + (cz * nc[1] + cy) * nc[0] + cx;
    slotCell[s] = c;
    slotWithin[s] = atomicAdd(&cellCount[c], 1);
}

constexpr int kScanThreads = 1024;
constexpr int kScanItems = 4;
constexpr int kScanTile = kScanThreads * kScanItems;

// The block's sum of one value a thread (every thread gets it).
__device__ __forceinline__ int blockSumInt(int value, int *shared)
{
    for (int offset = 16; offset > 0; offset >>= 1) value += __shfl_xor_sync(0xFFFFFFFFu, value, offset);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) shared[warp] = value;
    __syncthreads();
    value = lane < (int)(blockDim.x >> 5) ? shared[lane] : 0;
    for (int offset = 16; offset > 0; offset >>= 1) value += __shfl_xor_sync(0xFFFFFFFFu, value, offset);
    return value;
}

// partials[b] = the sum of tile b's counts.
__global__ void __launch_bounds__(kScanThreads)
cellScanReduceKernel(const int *cellCount, int total, int *partials, const Control *ctl)
{
    if (ctl && !ctl->active) return;
    __shared__ int shared[32];
    const int base = blockIdx.x * kScanTile;
    int sum = 0;
    for (int k = 0; k < kScanItems; ++k) {
        int idx = base + k * kScanThreads + threadIdx.x;
        if (idx < total) sum += cellCount[idx];
    }
    sum = blockSumInt(sum, shared);
    if (threadIdx.x == 0) partials[blockIdx.x] = sum;
}

// cellStart[c] = the counts' exclusive prefix sum; the counts go back to zero for the next sort.
__global__ void __launch_bounds__(kScanThreads)
cellScanApplyKernel(int *cellCount, int total, const int *partials, int *cellStart, const Control *ctl)
{
    if (ctl && !ctl->active) return;
    __shared__ int shared[32];
    // the tiles before this one
    int before = 0;
    for (int b = threadIdx.x; b < (int)blockIdx.x; b += kScanThreads) before += partials[b];
    before = blockSumInt(before, shared);
    // thread t scans items base + 4t .. base + 4t + 3
    const int first = blockIdx.x * kScanTile + threadIdx.x * kScanItems;
    int item[kScanItems], sum = 0;
    for (int k = 0; k < kScanItems; ++k) {
        item[k] = first + k < total ? cellCount[first + k] : 0;
        sum += item[k];
    }
    // exclusive prefix of the threads' sums: within the warp, then over the warps
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int inclusive = sum;
    for (int offset = 1; offset < 32; offset <<= 1) {
        int up = __shfl_up_sync(0xFFFFFFFFu, inclusive, offset);
        if (lane >= offset) inclusive += up;
    }
    __syncthreads();
    if (lane == 31) shared[warp] = inclusive;
    __syncthreads();
    if (warp == 0) {
        int w = lane < kScanThreads / 32 ? shared[lane] : 0, wi = w;
        for (int offset = 1; offset < 32; offset <<= 1) {
            int up = __shfl_up_sync(0xFFFFFFFFu, wi, offset);
            if (lane >= offset) wi += up;
        }
        if (lane < kScanThreads / 32) shared[lane] = wi - w;
    }
    __syncthreads();
    int running = before + shared[warp] + inclusive - sum;
    for (int k = 0; k < kScanItems; ++k) {
        if (first + k < total) {
            cellStart[first + k] = running;
            cellCount[first + k] = 0;
        }
        running += item[k];
    }
}

__global__ void cellPlaceKernel(int n, const int *slotCell, const int *slotWithin, const int *orig,
                                const int *cellStart, int2 *bucket, const Control *ctl)
{
    if (ctl && !ctl->active) return;
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    bucket[cellStart[slotCell[s]] + slotWithin[s]] = make_int2(orig[s], s);
}

// perm[k] = the old slot of sorted slot k; sortedCell[k] = its cell.
__global__ void cellRankKernel(int n, const int2 *bucket, const int *slotCell, const int *cellStart, int *perm,
                               int *sortedCell, const Control *ctl)
{
    if (ctl && !ctl->active) return;
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int2 e = bucket[k];
    const int c = slotCell[e.y];
    const int start = cellStart[c], end = cellStart[c + 1];
    // ties (never, with distinct caller indices) fall to the old slot, so the ranks stay a permutation
    int rank = 0;
    for (int q = start; q < end; ++q) {
        const int2 o = bucket[q];
        rank += o.x < e.x || (o.x == e.x && o.y < e.y);
    }
    perm[start + rank] = e.y;
    sortedCell[start + rank] = c;
}

// Permute the master into the new order (from the old buffers) and build the float32 frame:
// points and remainders (src/pysurf/sphGpu.py:1010-1019), float32 velocity and density
// (1021-1029), deviation (1031-1038) and the Tait pressure (1058-1070).
__global__ void gatherKernel(Params P, int n, const int *perm, MasterView from, MasterView to, Frame F,
                             const Control *ctl)
{
    if (ctl && !ctl->active) return;
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    int o = perm[s];
    double x[3] = {0.0, 0.0, 0.0}, v[3] = {0.0, 0.0, 0.0};
    for (int a = 0; a < P.dim; ++a) {
        x[a] = from.x[a][o];
        v[a] = from.v[a][o];
        to.x[a][s] = x[a];
        to.v[a][s] = v[a];
    }
    double rho = from.rho[o];
    double m64 = from.m[o], h64 = from.h[o];
    float m = (float)m64, h = (float)h64;
    uint8_t fl = from.fluid[o];
    to.rho[s] = rho;
    to.m[s] = m64;
    to.h[s] = h64;
    to.fluid[s] = fl;
    to.orig[s] = from.orig[o];
    float hi[3], lo[3];
    for (int a = 0; a < 3; ++a) {
        hi[a] = (float)x[a];
        lo[a] = (float)(x[a] - (double)hi[a]);
    }
    float hs = fl ? h : -h;
    float p = (float)taitPressure(P, rho, fl != 0);
    const double dev64 = rho - P.devReference;
    float dev = (float)dev64;
    float rhoF = (float)rho;
    float volume = m / rhoF, ratio = p / (rhoF * rhoF);
    float vf[3], vl[3];
    for (int a = 0; a < 3; ++a) {
        vf[a] = (float)v[a];
        vl[a] = (float)(v[a] - (double)vf[a]);
    }
    F.pres[s] = p;
    F.low[s] = make_float4(vl[0], vl[1], vl[2], (float)(dev64 - (double)dev));
    if (P.dim == 2) {
        F.pa[s] = make_float4(hi[0], hi[1], lo[0], lo[1]);
        F.pb[s] = make_float4(m, hs, dev, volume);
        F.kin[s] = make_float4(vf[0], vf[1], rhoF, ratio);
    } else {
        F.pa[s] = make_float4(hi[0], hi[1], hi[2], hs);
        F.pb[s] = make_float4(lo[0], lo[1], lo[2], m);
        F.kin[s] = make_float4(vf[0], vf[1], vf[2], rhoF);
        F.aux[s] = make_float4(ratio, dev, volume, 0.0f);
    }
}

// The frame's velocity, density, deviation and pressure from caller-order float64 arrays (the
// host-step sums take these from the caller each call), then V = m / rho and p / rho^2 from the
// frame's density and pressure.  Any of the arrays may be null.
__global__ void loadFieldsKernel(Params P, int n, const int *orig, const double *velocities, const double *densities,
                                 const double *pressures, double deviationReference, Frame F)
{
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    int o = orig[s];
    float4 k = F.kin[s];
    float4 low = F.low[s];
    if (velocities) {
        const double *v = velocities + (size_t)o * P.dim;
        k.x = (float)v[0];
        k.y = (float)v[1];
        low.x = (float)(v[0] - (double)k.x);
        low.y = (float)(v[1] - (double)k.y);
        if (P.dim == 3) {
            k.z = (float)v[2];
            low.z = (float)(v[2] - (double)k.z);
        }
    }
    float p = pressures ? (float)pressures[o] : F.pres[s];
    F.pres[s] = p;
    if (P.dim == 2) {
        float4 b = F.pb[s];
        if (densities) {
            const double dev = densities[o] - deviationReference;
            k.z = (float)densities[o];
            b.z = (float)dev;
            low.w = (float)(dev - (double)b.z);
        }
        b.w = b.x / k.z;
        k.w = p / (k.z * k.z);
        F.pb[s] = b;
    } else {
        float4 x = F.aux[s];
        if (densities) {
            const double dev = densities[o] - deviationReference;
            k.w = (float)densities[o];
            x.y = (float)dev;
            low.w = (float)(dev - (double)x.y);
        }
        x.z = F.pb[s].w / k.w;
        x.x = p / (k.w * k.w);
        F.aux[s] = x;
    }
    F.kin[s] = k;
    F.low[s] = low;
}

__global__ void refreshDensityKernel(int n, const double *rho, float *out)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = (float)rho[i];
}

// ------------------------------------------------------------------------------------------
// Pointwise
// ------------------------------------------------------------------------------------------

__global__ void enforceKernel(Params P, Frame F, Enforcement E)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.n || !F.fluid[i]) return;
    const int dim = P.dim;
    double x[3] = {0, 0, 0}, v[3] = {0, 0, 0};
    for (int a = 0; a < dim; ++a) { x[a] = F.x[a][i]; v[a] = F.v[a][i]; }
    enforceTracked(P, F, E, dim, i, x, v);
    for (int a = 0; a < dim; ++a) { F.x[a][i] = x[a]; F.v[a][i] = v[a]; }
}

// Column sums in a fixed order: block c sums column c (its rows `stride` doubles apart from the
// last column's) over rows 0 .. n - 1, each thread a strided share, then a tree in shared memory.
constexpr int kColumnSumThreads = 1024;
__global__ void __launch_bounds__(kColumnSumThreads) columnSumKernel(const double *columns, long long stride, int n,
                                                                     double *out)
{
    __shared__ double partial[kColumnSumThreads];
    const double *column = columns + (size_t)blockIdx.x * stride;
    double sum = 0.0;
    for (int k = threadIdx.x; k < n; k += kColumnSumThreads) sum += column[k];
    partial[threadIdx.x] = sum;
    __syncthreads();
    for (int width = kColumnSumThreads / 2; width > 0; width >>= 1) {
        if (threadIdx.x < width) partial[threadIdx.x] += partial[threadIdx.x + width];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[blockIdx.x] = partial[0];
}

// Each slot's kinetic m |v|^2 / 2, potential -m g . x and elastic m e(rho) energy (zero on the
// boundary) into three columns, `stride` doubles apart.
__global__ void fluidEnergyKernel(Params P, Frame F, double *columns, long long stride)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.n) return;
    double kinetic = 0.0, potential = 0.0, elastic = 0.0;
    if (F.fluid[i]) {
        const double m = F.m[i];
        double v2 = 0.0, gx = 0.0;
        for (int a = 0; a < P.dim; ++a) {
            v2 += F.v[a][i] * F.v[a][i];
            gx += P.gravity64[a] * F.x[a][i];
        }
        kinetic = 0.5 * m * v2;
        potential = -m * gx;
        elastic = m * elasticEnergy(P, F.rho[i]);
    }
    columns[i] = kinetic;
    columns[stride + i] = potential;
    columns[2 * stride + i] = elastic;
}

// The step's end: the clock advances, and the next step runs while t < untilTime and the step
// count allows (src/pysurf/sphSolver.py:1980-1989).
__global__ void stepEndKernel(Control *ctl)
{
    if (!ctl->active) return;
    ctl->time += ctl->dt;
    ctl->step += 1;
    ctl->active = ctl->time < ctl->untilTime && ctl->step < ctl->lastStep && ctl->error == 0;
}

// Caller-order float64 rows from the sorted master or frame.
// A pull's fields in one pass, so the copies out follow one launch.
template <int D>
__global__ void pullKernel(int n, MasterView M, Frame F, const float4 *acc, PullRows R)
{
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const size_t o = (size_t)M.orig[s];
    if (R.x) for (int a = 0; a < D; ++a) R.x[o * D + a] = M.x[a][s];
    if (R.v) for (int a = 0; a < D; ++a) R.v[o * D + a] = M.v[a][s];
    if (R.rho) R.rho[o] = M.rho[s];
    if (R.m) R.m[o] = M.m[s];
    if (R.h) R.h[o] = M.h[s];
    if (R.p) {
        if (R.framed) {
            R.p[o] = (double)pressureOf<D>(F, s);
        } else {
            Params P{};
            P.rho0 = R.rho0; P.stiffness = R.stiffness; P.tension = R.tension;
            R.p[o] = (double)(float)taitPressure(P, M.rho[s], M.fluid[s] != 0);
        }
    }
    if (R.a) {
        const float4 q = R.framed ? acc[s] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        const float c[3] = {q.x, q.y, q.z};
        for (int a = 0; a < D; ++a) R.a[o * D + a] = (double)c[a];
    }
    if (R.fluid) R.fluid[o] = M.fluid[s];
}

__global__ void scatterFloat4Kernel(int n, int dim, const int *orig, const float4 *values, double *out)
{
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    int o = orig[s];
    float4 q = values[s];
    float c[4] = {q.x, q.y, q.z, q.w};
    for (int a = 0; a < dim; ++a) out[o * dim + a] = (double)c[a];
}

// A frame of the run in caller order (src/pysurf/sphFrames.py:60-100): each particle's position in
// float32, its speed |v| taken in float64 as numpy's norm takes it ((vx^2 + vy^2) + vz^2, then the
// square root) and rounded to float32, and its fluid flag.
__global__ void frameKernel(int n, int dim, MasterView M, float *positions, float *speeds, uint8_t *fluid)
{
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const int o = M.orig[s];
    double v2 = __dmul_rn(M.v[0][s], M.v[0][s]);
    for (int a = 1; a < dim; ++a) v2 = __dadd_rn(v2, __dmul_rn(M.v[a][s], M.v[a][s]));
    speeds[o] = (float)sqrt(v2);
    for (int a = 0; a < dim; ++a) positions[(size_t)o * dim + a] = (float)M.x[a][s];
    fluid[o] = M.fluid[s];
}

__global__ void scatterFloatKernel(int n, const int *orig, const float *values, double *out)
{
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < n) out[orig[s]] = (double)values[s];
}

// dim x dim matrices from float4 rows into caller-order (n, dim, dim) rows.
__global__ void scatterMatrixKernel(int n, int dim, const int *orig, const float4 *R0, const float4 *R1,
                                    const float4 *R2, double *out)
{
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    int o = orig[s];
    if (dim == 2) {
        float4 a = R0[s];
        out[o * 4 + 0] = a.x; out[o * 4 + 1] = a.y; out[o * 4 + 2] = a.z; out[o * 4 + 3] = a.w;
    } else {
        const float4 *rows[3] = {R0, R1, R2};
        for (int a = 0; a < 3; ++a) {
            float4 q = rows[a][s];
            out[o * 9 + a * 3 + 0] = q.x; out[o * 9 + a * 3 + 1] = q.y; out[o * 9 + a * 3 + 2] = q.z;
        }
    }
}

// The frame's pressure of every slot, caller order.
template <int D>
__global__ void scatterPressureKernel(int n, const int *orig, Frame F, double *out)
{
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < n) out[orig[s]] = (double)pressureOf<D>(F, s);
}

// Master arrays from caller-order float64 rows (push / update): slot s = caller index s.
__global__ void loadMasterKernel(int n, int dim, const double *positions, const double *velocities,
                                 const double *densities, const double *masses, const uint8_t *fluid,
                                 const double *lengths, double hDefault, MasterView M)
{
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    for (int a = 0; a < dim; ++a) {
        M.x[a][s] = positions[s * dim + a];
        M.v[a][s] = velocities ? velocities[s * dim + a] : 0.0;
    }
    M.rho[s] = densities ? densities[s] : 0.0;
    M.m[s] = masses[s];
    M.h[s] = lengths ? lengths[s] : hDefault;
    M.fluid[s] = fluid[s] ? 1 : 0;
    M.orig[s] = s;
}

// ------------------------------------------------------------------------------------------
// Float64 neighbour rows (src/pysurf/sphCompiled.py:133-234): the same test, r^2 < radius^2
// with r^2 = dx*dx + dy*dy + dz*dz rounded term by term and the periodic component taken to
// its nearest image, so the sets match the reference's bit for bit.  Rows come in the walk's
// order; count == null fills, otherwise counts.
// ------------------------------------------------------------------------------------------

template <int D>
__global__ void neighbourRowsKernel(Params P, Frame F, const int64_t *offsets, int *rowsOut, long long *counts,
                                    double radius2)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.n) return;
    double xi[3] = {F.x[0][i], F.x[1][i], D == 3 ? F.x[2][i] : 0.0};
    int images = 1;
    double radius = sqrt(radius2), imageY = xi[1];
    if (P.period > 0.0) {
        double y = xi[1] - P.period * floor(xi[1] / P.period);
        if (y < radius || y > P.period - radius) {
            images = 2;
            imageY = xi[1] + (y < 0.5 * P.period ? P.period : -P.period);
        }
    }
    long long found = 0;
    long long write = counts ? 0 : offsets[F.orig[i]];
    // each grid level (coarse, then fine), the particle's own cells and then its image's
    for (int level = 0; level < P.levels; ++level) {
        // the coarse grid's ncs cells cover 2 h; the fine grid's as many cells as the radius spans
        const int n = level == 0 ? P.ncs : (int)ceil(radius / P.fineWidth);
        const CellBox own = cellBox(P, level, F.cell[i], xi, false, D, n);
        for (int image = 0; image < images; ++image) {
            const double pos[3] = {xi[0], image ? imageY : xi[1], xi[2]};
            const CellBox box = image ? cellBox(P, level, F.cell[i], pos, true, D, n) : own;
            for (int zz = box.z0; zz <= box.z1; ++zz)
            for (int yy = box.y0; yy <= box.y1; ++yy) {
                if (image == 1 && yy >= own.y0 && yy <= own.y1) continue;
                const int row = box.first + (zz * box.ny + yy) * box.nx;
                const int begin = F.cellStart[row + box.x0], end = F.cellStart[row + box.x1 + 1];
                for (int j = begin; j < end; ++j) {
                    if (j == i) continue;
                    double dx = __dsub_rn(xi[0], F.x[0][j]);
                    double dy = __dsub_rn(xi[1], F.x[1][j]);
                    double dz = D == 3 ? __dsub_rn(xi[2], F.x[2][j]) : 0.0;
                    if (P.period > 0.0) dy = __dsub_rn(dy, __dmul_rn(P.period, rint(dy / P.period)));
                    double s = __dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy));
                    s = __dadd_rn(s, __dmul_rn(dz, dz));
                    if (s < radius2) {
                        if (!counts) rowsOut[write + found] = F.orig[j];
                        ++found;
                    }
                }
            }
        }
    }
    if (counts) counts[F.orig[i]] = found;
}

// ------------------------------------------------------------------------------------------
// The reference's cell key (src/pysurf/sphSolver.py:1379-1408), float64, caller order.
// ------------------------------------------------------------------------------------------

__global__ void cellOrderKeyKernel(int n, int dim, const double *positions, double width, long long nx, long long ny,
                                   long long nz, long long *keys)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    long long c[3] = {0, 0, 0};
    long long shape[3] = {nx, ny, nz};
    for (int a = 0; a < dim; ++a) {
        long long f = (long long)floor(positions[i * dim + a] / width);
        long long r = f % shape[a];
        c[a] = r < 0 ? r + shape[a] : r;
    }
    keys[i] = (c[2] * ny + c[1]) * nx + c[0];
}

// ------------------------------------------------------------------------------------------
// Split (src/pysurf/sphRefinement.py:136-190): each chosen fluid particle becomes 2^dim
// daughters a quarter of its spacing from it along every axis, mass / 2^dim and h times the
// ratio; the first daughter keeps the mother's slot, the others append in the caller's order of
// the mothers.  rank[o] is the exclusive count of chosen mothers before caller index o.
// ------------------------------------------------------------------------------------------

__global__ void splitKernel(int n, int dim, MasterView M, const uint8_t *chosenByCaller, const int *rankByCaller,
                            double rho0, double lengthRatio, int total)
{
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    int o = M.orig[s];
    if (!chosenByCaller[o] || !M.fluid[s]) return;
    const int count = 1 << dim;
    // numpy takes (m / rho0) ** 0.5 as a square root, and ** (1/3) as a power
    double spacing = dim == 2 ? sqrt(M.m[s] / rho0) : pow(M.m[s] / rho0, 1.0 / 3.0);
    double mass = M.m[s] / (double)count;
    double length = M.h[s] * lengthRatio;
    double base[3] = {M.x[0][s], M.x[1][s], dim == 3 ? M.x[2][s] : 0.0};
    int r = rankByCaller[o];
    for (int k = 0; k < count; ++k) {
        int slot = k == 0 ? s : n + r * (count - 1) + (k - 1);
        int callerIndex = k == 0 ? o : total + r * (count - 1) + (k - 1);
        for (int a = 0; a < dim; ++a) {
            // corner k: bit (dim - 1 - a) of k picks -1/4 or +1/4 along axis a (itertools.product order)
            int bit = (k >> (dim - 1 - a)) & 1;
            M.x[a][slot] = base[a] + spacing * (bit ? 0.25 : -0.25);
            if (k > 0) M.v[a][slot] = M.v[a][s];
        }
        if (k > 0) {
            M.rho[slot] = M.rho[s];
            M.fluid[slot] = 1;
        }
        M.m[slot] = mass;
        M.h[slot] = length;
        M.orig[slot] = callerIndex;
    }
}

// ------------------------------------------------------------------------------------------
// Host-side launchers
// ------------------------------------------------------------------------------------------

static inline int blocksFor(long long n, int block) { return (int)((n + block - 1) / block); }

int scanTiles(int total) { return blocksFor(total, kScanTile); }

void launchCellSort(const Params &P, int n, const MasterView &M, const CellSortBuffers &B, int *cellStart,
                    int *sortedCell, const Control *ctl, cudaStream_t st)
{
    if (n == 0) return;
    const int total = P.cells + 1, tiles = scanTiles(total);
    cellCountKernel<<<blocksFor(n, 256), 256, 0, st>>>(P, n, M.x[0], M.x[1], M.x[2], M.h, B.slotCell, B.slotWithin,
                                                       B.cellCount, ctl);
    cellScanReduceKernel<<<tiles, kScanThreads, 0, st>>>(B.cellCount, total, B.partials, ctl);
    cellScanApplyKernel<<<tiles, kScanThreads, 0, st>>>(B.cellCount, total, B.partials, cellStart, ctl);
    cellPlaceKernel<<<blocksFor(n, 256), 256, 0, st>>>(n, B.slotCell, B.slotWithin, M.orig, cellStart, B.bucket, ctl);
    cellRankKernel<<<blocksFor(n, 256), 256, 0, st>>>(n, B.bucket, B.slotCell, cellStart, B.perm, sortedCell, ctl);
}

void launchGather(const Params &P, int n, const int *perm, const MasterView &from, const MasterView &to,
                  const Frame &F, const Control *ctl, cudaStream_t st)
{
    if (n == 0) return;
    gatherKernel<<<blocksFor(n, 256), 256, 0, st>>>(P, n, perm, from, to, F, ctl);
}

void launchLoadFields(const Params &P, int n, const int *orig, const double *v, const double *rho, const double *p,
                      double deviationReference, const Frame &F, cudaStream_t st)
{
    if (n == 0) return;
    loadFieldsKernel<<<blocksFor(n, 256), 256, 0, st>>>(P, n, orig, v, rho, p, deviationReference, F);
}

void launchLoadMaster(int n, int dim, const double *x, const double *v, const double *rho, const double *m,
                      const uint8_t *fluid, const double *h, double hDefault, const MasterView &M, cudaStream_t st)
{
    if (n == 0) return;
    loadMasterKernel<<<blocksFor(n, 256), 256, 0, st>>>(n, dim, x, v, rho, m, fluid, h, hDefault, M);
}

void launchStepEnd(Control *ctl, cudaStream_t st) { stepEndKernel<<<1, 1, 0, st>>>(ctl); }

cudaError_t kernelAttributes(cudaFuncAttributes *attributes)
{
    return cudaFuncGetAttributes(attributes, gatherKernel);
}

void launchEnforce(const Params &P, const Frame &F, const Enforcement &E, cudaStream_t st)
{
    if (P.n == 0 || E.kind == 0) return;
    enforceKernel<<<blocksFor(P.n, 256), 256, 0, st>>>(P, F, E);
}

void launchColumnSums(const double *columns, long long stride, int n, int count, double *out, cudaStream_t st)
{
    if (count <= 0) return;
    columnSumKernel<<<count, kColumnSumThreads, 0, st>>>(columns, stride, n, out);
}

void launchFluidEnergy(const Params &P, const Frame &F, double *columns, long long stride, cudaStream_t st)
{
    if (P.n == 0) return;
    fluidEnergyKernel<<<blocksFor(P.n, 256), 256, 0, st>>>(P, F, columns, stride);
}

void launchRefreshDensity(int n, const double *rho, float *out, cudaStream_t st)
{
    if (n == 0) return;
    refreshDensityKernel<<<blocksFor(n, 256), 256, 0, st>>>(n, rho, out);
}

void launchPull(int n, int dim, const MasterView &M, const Frame &F, const float4 *acc, const PullRows &R,
                cudaStream_t st)
{
    if (n == 0) return;
    if (dim == 2) pullKernel<2><<<blocksFor(n, 256), 256, 0, st>>>(n, M, F, acc, R);
    else pullKernel<3><<<blocksFor(n, 256), 256, 0, st>>>(n, M, F, acc, R);
}

void launchScatterFloat4(int n, int dim, const int *orig, const float4 *values, double *out, cudaStream_t st)
{
    if (n == 0) return;
    scatterFloat4Kernel<<<blocksFor(n, 256), 256, 0, st>>>(n, dim, orig, values, out);
}

void launchFrame(int n, int dim, const MasterView &M, float *positions, float *speeds, uint8_t *fluid, cudaStream_t st)
{
    if (n == 0) return;
    frameKernel<<<blocksFor(n, 256), 256, 0, st>>>(n, dim, M, positions, speeds, fluid);
}

void launchScatterFloat(int n, const int *orig, const float *values, double *out, cudaStream_t st)
{
    if (n == 0) return;
    scatterFloatKernel<<<blocksFor(n, 256), 256, 0, st>>>(n, orig, values, out);
}

void launchScatterMatrix(int n, int dim, const int *orig, const Frame &F, int which, double *out, cudaStream_t st)
{
    if (n == 0) return;
    if (which == 0) scatterMatrixKernel<<<blocksFor(n, 256), 256, 0, st>>>(n, dim, orig, F.G0, F.G1, F.G2, out);
    else scatterMatrixKernel<<<blocksFor(n, 256), 256, 0, st>>>(n, dim, orig, F.L0, F.L1, F.L2, out);
}

void launchScatterPressure(int n, int dim, const int *orig, const Frame &F, double *out, cudaStream_t st)
{
    if (n == 0) return;
    if (dim == 2) scatterPressureKernel<2><<<blocksFor(n, 256), 256, 0, st>>>(n, orig, F, out);
    else scatterPressureKernel<3><<<blocksFor(n, 256), 256, 0, st>>>(n, orig, F, out);
}

void launchNeighbourRows(const Params &P, const Frame &F, const int64_t *offsets, int *rows, long long *counts,
                         double radius2, cudaStream_t st)
{
    if (P.n == 0) return;
    if (P.dim == 2) neighbourRowsKernel<2><<<blocksFor(P.n, kBlock), kBlock, 0, st>>>(P, F, offsets, rows, counts, radius2);
    else neighbourRowsKernel<3><<<blocksFor(P.n, kBlock), kBlock, 0, st>>>(P, F, offsets, rows, counts, radius2);
}

void launchCellOrderKey(int n, int dim, const double *positions, double width, const long long shape[3],
                        long long *keys, cudaStream_t st)
{
    if (n == 0) return;
    cellOrderKeyKernel<<<blocksFor(n, 256), 256, 0, st>>>(n, dim, positions, width, shape[0], shape[1], shape[2], keys);
}

void launchSplit(int n, int dim, const MasterView &M, const uint8_t *chosen, const int *rank, double rho0,
                 double lengthRatio, int total, cudaStream_t st)
{
    if (n == 0) return;
    splitKernel<<<blocksFor(n, 256), 256, 0, st>>>(n, dim, M, chosen, rank, rho0, lengthRatio, total);
}

}  // namespace sph
