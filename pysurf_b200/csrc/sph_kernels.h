// sph_kernels.h -- host-side view of the kernels in sph_kernels.cu.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "sph_internal.cuh"

namespace sph {

// The float64 master state's arrays, in one buffer set's order.
struct MasterView {
    double *x[3], *v[3], *rho, *m, *h;
    uint8_t *fluid;
    int *orig;
};

// The boundary the device steps enforce (kind 0 none, 1 container, 2 bed, 3 height field).
struct Enforcement {
    int kind;
    double lower[3], upper[3];
    int openTop;
    const double *bedX, *bedZ;
    int bedCount;
    double clearance;
    int sideWalls;
    double width;
    int offshoreWall;
    double wallX, pistonSpeed, endLimit;
    const double *table;
    int tableNx, tableNy;
    double originX, originY, stepX, stepY, lowY, highY, lowX, highX;
};

enum class Stage { ShepardSum, ShepardApply, Wall, Gradients, Momentum, Kick, Continuity, Xsph, List, Closure, ShiftFields, Shift, ShiftDrift, FrameDensity };

struct LaunchArgs {
    Params P;
    Frame F;
    cudaStream_t stream;
    Control *ctl;
    int maxima;             // Momentum: fold the fluid maxima into ctl and take the time step
    Enforcement E;
    int flag;               // Wall: write the density too; Continuity / Xsph: the epilogue's mode
    int wantG, wantL, wantRho;
    float floorDet;
    const float *densities; // Xsph: the densities it divides by; null for the frame's
    int threads;            // threads per particle in the sweeps: 1, 2, 4 or 8
    int *maxCount;          // List: the largest neighbour count goes here (atomic max), when given
};

void launchStage(const LaunchArgs &A, Stage stage);

// A merge of split particles (sph_merge.cu): the current master and the buffer it moves into, with
// that buffer's frame, the step's parameters, the frame's accelerations and pressures, the energy
// budget's rows (null when off), the caller-order mask on the device, and where the caller-order
// source of each particle after goes.
struct MergeArgs {
    int n, dim;
    MasterView master, next;
    Frame nextFrame;
    Params params;
    float4 *acc;
    const float *pres;
    double *energy;
    int energyStride, energyTerms;
    const uint8_t *mask;
    double referenceDensity, referenceMass, lengthRatio;
    long long *source;
    cudaStream_t stream;
};
struct MergeResultDevice {
    int groups, newCount;
    double removedEnergy;
    const char *error;
};
// 0, or -1 with out.error set.  With no group found, or a failure before the merge itself (no
// memory for the scratch, too few fluid particles after the boundary to fill its places), the state
// is untouched.
int runMerge(const MergeArgs &in, MergeResultDevice &out);
// The counting sort's scratch: slotCell, slotWithin, perm (n entries), bucket (n pairs), cellCount
// (numCells + 1 entries, all zero between sorts), partials (scanTiles(numCells + 1) entries).
struct CellSortBuffers {
    int *slotCell, *slotWithin, *perm, *cellCount, *partials;
    int2 *bucket;
};
int scanTiles(int total);
// Sorts the slots of M by (cell, caller index): cellStart (numCells + 1 lower bounds), perm and the
// sorted slots' cells.
void launchCellSort(const Params &P, int n, const MasterView &M, const CellSortBuffers &B, int *cellStart,
                    int *sortedCell, const Control *ctl, cudaStream_t st);
void launchGather(const Params &P, int n, const int *perm, const MasterView &from, const MasterView &to,
                  const Frame &F, const Control *ctl, cudaStream_t st);
void launchLoadFields(const Params &P, int n, const int *orig, const double *v, const double *rho, const double *p,
                      double deviationReference, const Frame &F, cudaStream_t st);
void launchLoadMaster(int n, int dim, const double *x, const double *v, const double *rho, const double *m,
                      const uint8_t *fluid, const double *h, double hDefault, const MasterView &M, cudaStream_t st);
// The attributes of one of the library's kernels as loaded on the current device (binaryVersion:
// the architecture the kernels were compiled for, 100 for sm_100a).
cudaError_t kernelAttributes(cudaFuncAttributes *attributes);
void launchStepEnd(Control *ctl, cudaStream_t st);
void launchEnforce(const Params &P, const Frame &F, const Enforcement &E, cudaStream_t st);
// Sums `count` columns of n rows, `stride` doubles apart, each in a fixed order, into out[0 .. count).
void launchColumnSums(const double *columns, long long stride, int n, int count, double *out, cudaStream_t st);
// Each slot's kinetic, potential and elastic energy (zero on the boundary) into three columns.
void launchFluidEnergy(const Params &P, const Frame &F, double *columns, long long stride, cudaStream_t st);
void launchRefreshDensity(int n, const double *rho, float *out, cudaStream_t st);
// The fields a pull asks for, each into its own caller-order rows (null: not asked for).
struct PullRows {
    double *x, *v, *rho, *m, *h, *p, *a;
    uint8_t *fluid;
    // framed: the frame holds this state's pressures and a step's accelerations.  When it does not
    // (a push, a split or a merge since the last step), p is the Tait pressure of the master density,
    // the pressure the next frame will hold, and a is zero: no step has taken it for this state.
    int framed, tension;
    double rho0, stiffness;
};
// Every asked field in one pass: slot s to caller place M.orig[s]; p from the frame, a from acc.
void launchPull(int n, int dim, const MasterView &M, const Frame &F, const float4 *acc, const PullRows &R,
                cudaStream_t st);
void launchScatterFloat4(int n, int dim, const int *orig, const float4 *values, double *out, cudaStream_t st);
void launchScatterFloat(int n, const int *orig, const float *values, double *out, cudaStream_t st);
// Caller-order float32 positions (n x dim), float32 speeds and fluid flags of every particle.
void launchFrame(int n, int dim, const MasterView &M, float *positions, float *speeds, uint8_t *fluid, cudaStream_t st);
void launchScatterMatrix(int n, int dim, const int *orig, const Frame &F, int which, double *out, cudaStream_t st);
void launchScatterPressure(int n, int dim, const int *orig, const Frame &F, double *out, cudaStream_t st);
void launchNeighbourRows(const Params &P, const Frame &F, const int64_t *offsets, int *rows, long long *counts,
                         double radius2, cudaStream_t st);
void launchCellOrderKey(int n, int dim, const double *positions, double width, const long long shape[3],
                        long long *keys, cudaStream_t st);
// A band across the tank (3D sections): the fluid with |y - center| < half; y null for all of it.
struct Band {
    const double *y;
    double center, half;
};
void launchSurfaceTops(int n, const MasterView &M, int vertical, const Band &band, double x0, double width,
                       long long count, unsigned long long *scratch, double *out, cudaStream_t st);
void launchFaceCells(int n, const MasterView &M, int vertical, const Band &band, double lowX, double highX,
                     double lowZ, double half, double start, double base, double spacing, long long columns,
                     long long bands, uint8_t *marks, cudaStream_t st);
void launchBedSheet(int n, const MasterView &M, int vertical, const Band &band, const double *bx, const double *bz,
                    int m, double wetHeight, double *out, int *count, cudaStream_t st);
void launchCrestZone(int n, const MasterView &M, int dim, double x0, double y0, double width, long long nx,
                     long long ny, unsigned long long *tops, double threshold, double minMass, uint8_t *chosen,
                     cudaStream_t st);
void launchSplit(int n, int dim, const MasterView &M, const uint8_t *chosen, const int *rank, double rho0,
                 double lengthRatio, int total, cudaStream_t st);

}  // namespace sph
