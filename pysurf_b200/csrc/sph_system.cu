// sph_system.cu -- the particle-system handle behind the C-ABI (include/pysurf_b200.h).
//
// One handle holds one particle system on one device: the float64 master state (double
// buffered), the float32 sweep frame, the cell list and the sort scratch, all sized to a
// capacity that grows by a quarter at a time as the reference's device arrays do
// (src/pysurf/sphGpu.py:1572-1594).  Host arrays move through pinned staging, or straight from
// the caller's memory when it is pinned already.
//
// A device-resident step is captured once into a CUDA graph, twice over: a step moves the master
// to the other buffer, so one graph starts from each.  Runs of steps replay them alternately;
// each step's time step is taken on the device from its own maxima, and the host reads the clock
// back only when it must decide whether to launch more.  Events between the stages of each graph
// time every stage of the last step (sph_stage_times).
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <string>
#include <thread>
#include <vector>

#include "../../include/pysurf_b200.h"
#include "sph_kernels.h"

using namespace sph;

namespace {

constexpr int kStageCount = 7;      // cells, filter, wall, gradients, momentum, kick, continuity

thread_local std::string lastError;

int fail(int code, const std::string &message)
{
    lastError = message;
    return code;
}

#define CUDA_TRY(expr)                                                                                   \
    do {                                                                                                 \
        cudaError_t err_ = (expr);                                                                       \
        if (err_ != cudaSuccess)                                                                         \
            return fail(err_ == cudaErrorMemoryAllocation ? SPH_ERR_NOMEM : SPH_ERR_CUDA,               \
                        std::string(#expr) + ": " + cudaGetErrorString(err_));                           \
    } while (0)

#define TRY(expr)                                                                                        \
    do {                                                                                                 \
        int status_ = (expr);                                                                            \
        if (status_ != SPH_OK) return status_;                                                           \
    } while (0)

double sigmaUnit(int kind, int dim)
{
    const double pi = 3.14159265358979323846;
    if (kind == 1) return dim == 2 ? 7.0 / (4.0 * pi) : 21.0 / (16.0 * pi);
    return dim == 2 ? 10.0 / (7.0 * pi) : 1.0 / pi;
}

// W(r) at h in float64 (src/pysurf/sphKernels.py:108-648), for the shift's W(dx).
double kernelValueHost(int kind, int dim, double r, double h)
{
    const double q = r / h, sigma = sigmaUnit(kind, dim) / (dim == 2 ? h * h : h * h * h);
    if (q >= 2.0) return 0.0;
    if (kind == 1) {
        const double rest = 1.0 - 0.5 * q;
        return sigma * rest * rest * rest * rest * (2.0 * q + 1.0);
    }
    if (q < 1.0) return sigma * (1.0 - 1.5 * q * q + 0.75 * q * q * q);
    return sigma * 0.25 * (2.0 - q) * (2.0 - q) * (2.0 - q);
}

template <class T>
int deviceAlloc(T **ptr, size_t count)
{
    *ptr = nullptr;
    if (count == 0) count = 1;
    cudaError_t err = cudaMalloc((void **)ptr, count * sizeof(T));
    if (err != cudaSuccess) return fail(SPH_ERR_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(err));
    return SPH_OK;
}

}  // namespace

namespace sph {
// Sets what sph_last_error() reports on this thread, for entry points defined in other files.
void recordError(const std::string &message) { lastError = message; }
}  // namespace sph

// The shortest neighbour table row worth keeping when memory caps the row below the largest count.
constexpr int kMinTableRow = 64;

struct SphSystem {
    // configuration
    int device = 0;
    int dim = 2, kind = 0;
    double h = 0.0;
    double domainMin[3] = {0, 0, 0}, domainMax[3] = {0, 0, 0};
    double period = 0.0;
    int precise = 1;
    int ncs = 3;                // cells per support: 2h / 3 wide cells trim the candidates
    int64_t gridShape[3] = {1, 1, 1};
    // physics (setPhysics) and the sums' switches
    double rho0 = 1000.0, c0 = 1.0, alpha = 0.0, boundaryFactor = 0.0, gravity[3] = {0, 0, 0};
    double xsphEpsilon = 0.0, densityFloor = 0.0;
    int diffusionMode = 0;
    double diffusionDelta = 0.1, diffusionC0 = 1.0, diffusionRho0 = 1000.0, diffusionG = 0.0;
    int wallExtrapolated = 0, tension = 0, corrected = 0, limited = 0;
    int shifting = 0, shiftLocal = 0;   // particle shifting, its W(dx) and its size's c0 Ma 4 h
    double spacingKernel = 1.0, shiftScale = 0.0;
    float4 *shiftGrad = nullptr, *shiftPlain = nullptr, *shiftRhoGrad = nullptr, *shiftOut = nullptr,
           *shiftDv = nullptr;
    int closure = 0;            // delta-LES-SPH closure, with its sound speed, rho0 and the water's viscosity
    double closureC0 = 1.0, closureRho0 = 1000.0, closureNu = 0.0;
    float2 *eddy = nullptr;
    // the energy budget (src/pysurf/sphEnergy.py): each particle's running total of each term, by
    // caller index, and the momentum sweep's parts of a; energyCap rows, made while it is on
    int budget = 0;
    int compensated = 0;        // compensated momentum and continuity sums
    double *energy = nullptr;
    float4 *parts = nullptr;
    int energyCap = 0;
    double *dSums = nullptr;    // the column sums' results (kEnergyTerms doubles)
    bool physicsSet = false;
    Enforcement enforcement{};
    double *bedX = nullptr, *bedZ = nullptr, *table = nullptr;
    // state
    int n = 0, capacity = 0;
    bool mixedH = false;
    double hMin = 0.0;
    int cur = 0;
    bool resident = false;      // master holds velocities and densities (push)
    bool framed = false;        // the frame is in the master's order (its pressures are current)
    bool cellsFresh = false;    // the cell list matches the master's positions
    // grid
    double origin[3] = {0, 0, 0}, cellWidth = 0.0;
    int nc[3] = {1, 1, 1};
    int numCells = 1;           // the coarse grid's cells
    // the fine level (particles shorter than h): its longest h, its grid, and its cells
    double fineMax = 0.0;
    int levels = 1;
    double fineOrigin[3] = {0, 0, 0}, fineWidth = 0.0;
    int fineNc[3] = {1, 1, 1};
    int fineCells = 0;
    // device memory
    MasterView master[2]{};
    float4 *pa = nullptr, *pb = nullptr, *kin = nullptr, *G[3] = {}, *L[3] = {}, *gradRho = nullptr, *acc = nullptr,
           *vec = nullptr;
    float4 *aux = nullptr, *low = nullptr;
    float *pres = nullptr, *rate = nullptr, *scalar = nullptr;
    int *cell = nullptr, *cellStart = nullptr;
    CellSortBuffers sortBuffers = {};
    Control *ctl = nullptr;
    // Caller-order float64 staging on the device, kStageSlots rows of capacity doubles:
    //   inputs   0-2 vectors, 3 densities, 4 pressures (loadState: 0-2 x, 3-5 v, 6 rho, 7 m, 8 h)
    //   outputs  5-13 (up to dim x dim per particle); a pull's fields 0-12
    static constexpr int kStageSlots = 14;
    static constexpr int kOutSlot = 5;
    double *dStage = nullptr;
    uint8_t *dStageU8 = nullptr;
    int *dRank = nullptr;
    Control *hCtl = nullptr;    // pinned
    // the neighbour table: listCap entries a slot (0: the sweeps walk the cells), stride capacity
    int *nbr = nullptr, *ncount = nullptr, *dMaxCount = nullptr;
    void *surface = nullptr;        // the breaking tracker's read scratch
    size_t surfaceBytes = 0;
    size_t nbrEntries = 0;
    int listCap = 0;
    int tableMode = 1;          // 0 never build the table, 1 build it when it fits the budget
    bool listDirty = true;      // the table's size must be taken again before the next step
    int listSizedFor = -1;      // the particle count the table's size was taken for
    int threads = 4;            // threads per particle in the sweeps
    int cellStartCapacity = 0;
    // execution
    cudaStream_t stream = nullptr;
    bool ownStream = false;
    cudaGraphExec_t graphs[2] = {nullptr, nullptr};  // one step from master buffer 0, one from buffer 1
    cudaEvent_t stageEvents[2][kStageCount + 1] = {};
    bool graphDirty = true;
    bool graphFilter = false;
    int graphNodes = 0;
    int lastGraph = 0;
    int beginCur = 0;
    long long beginStep = 0;
    long long enqueued = 0;
    cudaEvent_t evStart = nullptr, evStop = nullptr;
    cudaEvent_t uploaded = nullptr;     // after a load's copies in, before the kernels that read them
    double lastAdvanceMs = 0.0;

    // ---- memory ------------------------------------------------------------------------------

    int freeArrays()
    {
        for (int b = 0; b < 2; ++b) {
            MasterView &M = master[b];
            for (int a = 0; a < 3; ++a) { cudaFree(M.x[a]); cudaFree(M.v[a]); }
            cudaFree(M.rho); cudaFree(M.m); cudaFree(M.h); cudaFree(M.fluid); cudaFree(M.orig);
            M = MasterView{};
        }
        void *ptrs[] = {pa, pb, kin, G[0], G[1], G[2], L[0], L[1], L[2], gradRho, acc, vec, aux, low, pres, rate,
                        scalar, cell, sortBuffers.slotCell, sortBuffers.slotWithin, sortBuffers.perm,
                        sortBuffers.bucket, dStage, dStageU8, dRank, nbr, ncount, eddy, shiftGrad, shiftPlain,
                        shiftRhoGrad, shiftOut, shiftDv};
        for (void *p : ptrs) cudaFree(p);
        eddy = nullptr;
        shiftGrad = shiftPlain = shiftRhoGrad = shiftOut = shiftDv = nullptr;
        nbr = ncount = nullptr;
        nbrEntries = 0;
        listCap = 0;
        listDirty = true;
        pa = pb = kin = gradRho = acc = vec = nullptr;
        for (int a = 0; a < 3; ++a) G[a] = L[a] = nullptr;
        aux = low = nullptr; pres = rate = scalar = nullptr; cell = nullptr;
        sortBuffers.slotCell = sortBuffers.slotWithin = sortBuffers.perm = nullptr;
        sortBuffers.bucket = nullptr;
        dStage = nullptr; dStageU8 = nullptr; dRank = nullptr;
        capacity = 0;
        return SPH_OK;
    }

    // Arrays for at least `count` particles; with `preserve`, the current master survives.
    int reserve(int count, bool preserve)
    {
        if (count <= capacity) return SPH_OK;
        int cap = std::max(count, (int)(1.25 * capacity));
        MasterView old = master[cur];
        // keep the current master by moving it into freshly allocated arrays
        MasterView fresh{};
        for (int a = 0; a < 3; ++a) {
            TRY(deviceAlloc(&fresh.x[a], cap));
            TRY(deviceAlloc(&fresh.v[a], cap));
        }
        TRY(deviceAlloc(&fresh.rho, cap));
        TRY(deviceAlloc(&fresh.m, cap));
        TRY(deviceAlloc(&fresh.h, cap));
        TRY(deviceAlloc(&fresh.fluid, cap));
        TRY(deviceAlloc(&fresh.orig, cap));
        if (preserve && n > 0) {
            for (int a = 0; a < dim; ++a) {
                CUDA_TRY(cudaMemcpyAsync(fresh.x[a], old.x[a], n * sizeof(double), cudaMemcpyDeviceToDevice, stream));
                CUDA_TRY(cudaMemcpyAsync(fresh.v[a], old.v[a], n * sizeof(double), cudaMemcpyDeviceToDevice, stream));
            }
            CUDA_TRY(cudaMemcpyAsync(fresh.rho, old.rho, n * sizeof(double), cudaMemcpyDeviceToDevice, stream));
            CUDA_TRY(cudaMemcpyAsync(fresh.m, old.m, n * sizeof(double), cudaMemcpyDeviceToDevice, stream));
            CUDA_TRY(cudaMemcpyAsync(fresh.h, old.h, n * sizeof(double), cudaMemcpyDeviceToDevice, stream));
            CUDA_TRY(cudaMemcpyAsync(fresh.fluid, old.fluid, n, cudaMemcpyDeviceToDevice, stream));
            CUDA_TRY(cudaMemcpyAsync(fresh.orig, old.orig, n * sizeof(int), cudaMemcpyDeviceToDevice, stream));
            CUDA_TRY(cudaStreamSynchronize(stream));
        }
        // the old master goes with the rest; the fresh one becomes buffer 0
        if (old.x[0] == master[0].x[0]) master[0] = MasterView{};
        else master[1] = MasterView{};
        for (int a = 0; a < 3; ++a) { cudaFree(old.x[a]); cudaFree(old.v[a]); }
        cudaFree(old.rho); cudaFree(old.m); cudaFree(old.h); cudaFree(old.fluid); cudaFree(old.orig);
        freeArrays();
        capacity = cap;
        master[0] = fresh;
        cur = 0;
        MasterView &M = master[1];
        for (int a = 0; a < 3; ++a) {
            TRY(deviceAlloc(&M.x[a], cap));
            TRY(deviceAlloc(&M.v[a], cap));
        }
        TRY(deviceAlloc(&M.rho, cap));
        TRY(deviceAlloc(&M.m, cap));
        TRY(deviceAlloc(&M.h, cap));
        TRY(deviceAlloc(&M.fluid, cap));
        TRY(deviceAlloc(&M.orig, cap));
        TRY(deviceAlloc(&pa, cap));
        TRY(deviceAlloc(&pb, cap));
        TRY(deviceAlloc(&kin, cap));
        TRY(deviceAlloc(&aux, cap));
        TRY(deviceAlloc(&low, cap));
        TRY(deviceAlloc(&pres, cap));
        for (int a = 0; a < 3; ++a) { TRY(deviceAlloc(&G[a], cap)); TRY(deviceAlloc(&L[a], cap)); }
        TRY(deviceAlloc(&gradRho, cap));
        TRY(deviceAlloc(&acc, cap));
        TRY(deviceAlloc(&vec, cap));
        TRY(deviceAlloc(&eddy, cap));
        for (float4 **p : {&shiftGrad, &shiftPlain, &shiftRhoGrad, &shiftOut, &shiftDv}) {
            TRY(deviceAlloc(p, cap));
            CUDA_TRY(cudaMemsetAsync(*p, 0, sizeof(float4) * cap, stream));
        }
        TRY(deviceAlloc(&rate, cap));
        TRY(deviceAlloc(&scalar, cap));
        TRY(deviceAlloc(&cell, cap));
        TRY(deviceAlloc(&sortBuffers.slotCell, cap));
        TRY(deviceAlloc(&sortBuffers.slotWithin, cap));
        TRY(deviceAlloc(&sortBuffers.perm, cap));
        TRY(deviceAlloc(&sortBuffers.bucket, cap));
        TRY(deviceAlloc(&dStage, (size_t)kStageSlots * cap));
        TRY(deviceAlloc(&dStageU8, cap));
        TRY(deviceAlloc(&dRank, cap));
        TRY(deviceAlloc(&ncount, cap));
        CUDA_TRY(cudaMemsetAsync(acc, 0, sizeof(float4) * cap, stream));
        CUDA_TRY(cudaMemsetAsync(kin, 0, sizeof(float4) * cap, stream));
        CUDA_TRY(cudaMemsetAsync(aux, 0, sizeof(float4) * cap, stream));
        CUDA_TRY(cudaMemsetAsync(low, 0, sizeof(float4) * cap, stream));
        CUDA_TRY(cudaMemsetAsync(pres, 0, sizeof(float) * cap, stream));
        CUDA_TRY(cudaMemsetAsync(eddy, 0, sizeof(float2) * cap, stream));
        graphDirty = true;
        framed = false;
        return reserveBudget(preserve);
    }

    // The energy budget's arrays for the capacity, while the budget is on; with `preserve` the
    // running totals of the first n caller indices survive, every other row starts at zero.
    int reserveBudget(bool preserve)
    {
        if (!budget || (energy && energyCap >= capacity)) return SPH_OK;
        const int cap = std::max(capacity, 1);
        double *fresh = nullptr;
        float4 *freshParts = nullptr;
        TRY(deviceAlloc(&fresh, (size_t)kEnergyTerms * cap));
        TRY(deviceAlloc(&freshParts, (size_t)4 * cap));
        CUDA_TRY(cudaMemsetAsync(fresh, 0, sizeof(double) * kEnergyTerms * cap, stream));
        CUDA_TRY(cudaMemsetAsync(freshParts, 0, sizeof(float4) * 4 * cap, stream));
        if (preserve && energy && n > 0)
            CUDA_TRY(cudaMemcpy2DAsync(fresh, sizeof(double) * cap, energy, sizeof(double) * energyCap,
                                       sizeof(double) * std::min(n, energyCap), kEnergyTerms,
                                       cudaMemcpyDeviceToDevice, stream));
        CUDA_TRY(cudaStreamSynchronize(stream));
        cudaFree(energy);
        cudaFree(parts);
        energy = fresh;
        parts = freshParts;
        energyCap = cap;
        graphDirty = true;
        return SPH_OK;
    }

    // ---- grid ----------------------------------------------------------------------------------

    int setupGrid()
    {
        cellWidth = 2.0 * h / ncs;
        long long total = 1;
        for (int a = 0; a < 3; ++a) {
            if (a < dim) {
                origin[a] = domainMin[a] - cellWidth;
                nc[a] = (int)ceil((domainMax[a] - domainMin[a]) / cellWidth) + 3;
            } else {
                origin[a] = 0.0;
                nc[a] = 1;
            }
            total *= nc[a];
        }
        // cap the cells as the reference caps its grid; wider cells keep the stencil valid
        while (total > (1ll << 25)) {
            cellWidth *= 1.25;
            total = 1;
            for (int a = 0; a < dim; ++a) {
                nc[a] = (int)ceil((domainMax[a] - domainMin[a]) / cellWidth) + 3;
                total *= nc[a];
            }
        }
        numCells = (int)total;
        TRY(setupLevels());
        // the reference's hash grid shape (src/pysurf/sphGpu.py:1466-1478)
        double extent[3] = {0, 0, 0};
        for (int a = 0; a < dim; ++a) extent[a] = domainMax[a] - domainMin[a];
        long long cells[3];
        for (int a = 0; a < 3; ++a) {
            long long c = (long long)ceil(extent[a] / (2.0 * h)) + 3;
            cells[a] = c > 1 ? c : 1;
        }
        if (dim == 2) cells[2] = 1;
        while (cells[0] * cells[1] * cells[2] > (1ll << 25))
            for (int a = 0; a < 3; ++a) cells[a] = std::max((long long)(cells[a] * 0.8), 1ll);
        for (int a = 0; a < 3; ++a) gridShape[a] = cells[a];
        graphDirty = true;
        cellsFresh = false;
        listDirty = true;
        return SPH_OK;
    }

    // The fine level's grid, when some particles are shorter than h (a split's daughters): cells
    // 2 fineMax / ncs wide over the same domain, capped as the coarse grid is; then the cell
    // list's arrays for both grids.
    int setupLevels()
    {
        levels = fineMax > 0.0 ? 2 : 1;
        long long fine = 0;
        fineWidth = 0.0;
        for (int a = 0; a < 3; ++a) { fineOrigin[a] = 0.0; fineNc[a] = 1; }
        if (levels == 2) {
            fineWidth = 2.0 * fineMax / ncs;
            while (true) {
                fine = 1;
                for (int a = 0; a < dim; ++a) {
                    fineOrigin[a] = domainMin[a] - fineWidth;
                    fineNc[a] = (int)ceil((domainMax[a] - domainMin[a]) / fineWidth) + 3;
                    fine *= fineNc[a];
                }
                if (fine <= (1ll << 25)) break;
                fineWidth *= 1.25;
            }
        }
        fineCells = (int)fine;
        const int total = numCells + fineCells;
        if (total + 1 > cellStartCapacity) {
            cudaFree(cellStart);
            cudaFree(sortBuffers.cellCount);
            cudaFree(sortBuffers.partials);
            cellStart = sortBuffers.cellCount = sortBuffers.partials = nullptr;
            cellStartCapacity = 0;
            TRY(deviceAlloc(&cellStart, total + 1));
            TRY(deviceAlloc(&sortBuffers.cellCount, total + 1));
            TRY(deviceAlloc(&sortBuffers.partials, scanTiles(total + 1)));
            // the counts are zero between sorts: each sort's scan clears what its count added
            CUDA_TRY(cudaMemsetAsync(sortBuffers.cellCount, 0, sizeof(int) * (total + 1), stream));
            cellStartCapacity = total + 1;
        }
        graphDirty = true;
        cellsFresh = false;
        listDirty = true;
        return SPH_OK;
    }

    // The fine level from the particles' lengths: the longest below h (0 for none).
    int takeLevels(const double *lengths, int count)
    {
        double longest = 0.0;
        if (lengths)
            for (int i = 0; i < count; ++i)
                if (lengths[i] < h && lengths[i] > longest) longest = lengths[i];
        return takeFineLength(longest);
    }

    // The fine level from its longest length, found by the caller (0 for none).
    int takeFineLength(double longest)
    {
        if (longest == fineMax) return SPH_OK;
        fineMax = longest;
        return setupLevels();
    }

    // ---- parameters ----------------------------------------------------------------------------

    Params params() const
    {
        Params P{};
        P.n = n;
        P.dim = dim;
        P.kind = kind;
        P.mixedH = mixedH ? 1 : 0;
        P.hMax = (float)h;
        P.sigmaUnit = (float)sigmaUnit(kind, dim);
        for (int a = 0; a < 3; ++a) { P.origin[a] = origin[a]; P.nc[a] = nc[a]; }
        P.cellWidth = cellWidth;
        P.ncs = ncs;
        P.precise = precise;
        P.levels = levels;
        for (int a = 0; a < 3; ++a) { P.fineOrigin[a] = fineOrigin[a]; P.fineNc[a] = fineNc[a]; }
        P.fineWidth = fineWidth;
        P.fineFirst = numCells;
        P.cells = numCells + fineCells;
        P.fineMax = (float)fineMax;
        P.fineBelow = h;
        P.period = period;
        P.periodF = (float)period;
        P.c0 = (float)c0;
        P.alpha = (float)alpha;
        P.boundaryFactor = (float)boundaryFactor;
        for (int a = 0; a < 3; ++a) { P.g[a] = (float)gravity[a]; P.gravity64[a] = gravity[a]; }
        P.rho0 = rho0;
        P.stiffness = rho0 * c0 * c0 / 7.0;
        P.densityFloor = densityFloor;
        P.devReference = diffusionRho0;
        P.halfInvRho0 = (float)(0.5 / diffusionRho0);
        P.tension = tension;
        P.diffusion = diffusionMode;
        P.diffusionFactor = (float)(2.0 * diffusionDelta * diffusionC0);
        P.hydrostaticSlope = (float)(diffusionRho0 * diffusionG / (diffusionC0 * diffusionC0));
        P.corrected = corrected;
        P.limited = limited;
        P.closure = closure;
        P.waterTerm = (float)(2.0 * (dim + 2) * closureNu / closureC0);
        P.closureRho0 = (float)closureRho0;
        P.closureC0 = (float)closureC0;
        P.shifting = shifting;
        P.shiftLocal = shiftLocal;
        P.spacingKernel = (float)spacingKernel;
        P.shiftThreshold = dim == 2 ? 1.5f : 2.4f;          // src/pysurf/sphSolver.py:265
        P.lopsidedness = kind == 1 ? 0.4f : 0.3f;           // src/pysurf/sphSolver.py:266
        P.shiftScale = shiftScale;
        P.shiftDt = 0.0;
        P.wallExtrapolated = wallExtrapolated;
        P.xsphEpsilon = (float)xsphEpsilon;
        P.listCap = listCap;
        P.listStride = capacity;
        P.budget = budget && energy ? 1 : 0;
        P.energyStride = energyCap;
        P.compensated = compensated;
        return P;
    }

    Frame frame() const
    {
        Frame F{};
        F.pa = pa; F.pb = pb; F.kin = kin; F.aux = aux; F.low = low; F.pres = pres;
        F.cell = cell; F.cellStart = cellStart;
        F.G0 = G[0]; F.G1 = G[1]; F.G2 = G[2];
        F.L0 = L[0]; F.L1 = L[1]; F.L2 = L[2];
        F.gradRho = gradRho; F.acc = acc; F.rate = rate; F.scalar = scalar; F.vec = vec; F.eddy = eddy;
        F.shiftGrad = shiftGrad; F.shiftPlain = shiftPlain; F.shiftRhoGrad = shiftRhoGrad; F.shift = shiftOut;
        F.shiftDv = shiftDv;
        F.nbr = nbr; F.ncount = ncount;
        F.energy = energy; F.parts = parts;
        const MasterView &M = master[cur];
        for (int a = 0; a < 3; ++a) { F.x[a] = M.x[a]; F.v[a] = M.v[a]; }
        F.rho = M.rho; F.m = M.m; F.h = M.h; F.fluid = M.fluid; F.orig = M.orig;
        return F;
    }

    LaunchArgs args(Control *control) const
    {
        LaunchArgs A{};
        A.P = params();
        A.F = frame();
        A.stream = stream;
        A.ctl = control;
        A.maxima = control ? 1 : 0;
        A.E = enforcement;
        A.floorDet = (float)pow(0.25, dim);
        A.threads = threads;
        return A;
    }

    // ---- cell list -----------------------------------------------------------------------------

    // Sort the master by (cell, caller index), permute it into the other buffer, and build the
    // frame and the cell list.
    // control: the device clock that gates the step (null: always runs).
    void rebuild(const Control *control = nullptr)
    {
        if (n == 0) return;
        Params P = params();
        launchCellSort(P, n, master[cur], sortBuffers, cellStart, cell, control, stream);
        int next = 1 - cur;
        Frame F = frame();
        const MasterView &to = master[next];
        for (int a = 0; a < 3; ++a) { F.x[a] = to.x[a]; F.v[a] = to.v[a]; }
        F.rho = to.rho; F.m = to.m; F.h = to.h; F.fluid = to.fluid; F.orig = to.orig;
        launchGather(P, n, sortBuffers.perm, master[cur], to, F, control, stream);
        cur = next;
        framed = true;
        cellsFresh = true;
        if (listCap > 0) {
            LaunchArgs A = args(const_cast<Control *>(control));
            launchStage(A, Stage::List);
        }
    }

    // Take the neighbour table's size from the current cell list: the largest count now, with room
    // to grow by a quarter, or as many entries a particle as three quarters of the free device
    // memory holds when that is less (the particles with more walk their cells).  Syncs.
    int sizeList()
    {
        listDirty = false;
        listSizedFor = n;
        if (n == 0 || tableMode == 0) {
            if (listCap) graphDirty = true;
            listCap = 0;
            return SPH_OK;
        }
        if (!cellsFresh) rebuild();
        if (!dMaxCount) TRY(deviceAlloc(&dMaxCount, 1));
        CUDA_TRY(cudaMemsetAsync(dMaxCount, 0, sizeof(int), stream));
        const int keep = listCap;
        listCap = 0;    // count only
        LaunchArgs A = args(nullptr);
        A.maxCount = dMaxCount;
        launchStage(A, Stage::List);
        int most = 0;
        CUDA_TRY(cudaMemcpyAsync(&most, dMaxCount, sizeof(int), cudaMemcpyDeviceToHost, stream));
        CUDA_TRY(cudaStreamSynchronize(stream));
        int cap = ((most + most / 4 + 8) + 7) & ~7;
        size_t entries = (size_t)cap * (size_t)capacity;
        if (entries > nbrEntries) {
            cudaFree(nbr);
            nbr = nullptr;
            nbrEntries = 0;
            size_t freeBytes = 0, totalBytes = 0;
            cudaMemGetInfo(&freeBytes, &totalBytes);
            const size_t room = freeBytes / 4 * 3 / sizeof(int) / (size_t)std::max(capacity, 1);
            if ((size_t)cap > room) cap = (int)(room & ~(size_t)7);
            entries = (size_t)cap * (size_t)capacity;
            if (cap < kMinTableRow || deviceAlloc(&nbr, entries) != SPH_OK) {
                nbr = nullptr;
                cap = 0;
                cudaGetLastError();
            } else {
                nbrEntries = entries;
            }
        }
        listCap = cap;
        if (listCap != keep) graphDirty = true;
        if (listCap > 0) {
            A = args(nullptr);
            launchStage(A, Stage::List);
        }
        CUDA_TRY(cudaGetLastError());
        return SPH_OK;
    }

    // ---- staging -------------------------------------------------------------------------------

    // Copy a caller array of `count` elements of `size` bytes to device memory at `dst`.
    int upload(void *dst, const void *src, size_t bytes, cudaMemcpyKind kind = cudaMemcpyHostToDevice)
    {
        if (bytes == 0) return SPH_OK;
        // pinned caller memory copies by DMA behind the return; pageable memory is staged by the
        // driver before the call returns; device memory (kind DeviceToDevice) copies in stream order
        CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, kind, stream));
        return SPH_OK;
    }

    int download(void *dst, const void *src, size_t bytes, cudaMemcpyKind kind = cudaMemcpyDeviceToHost)
    {
        if (bytes == 0) return SPH_OK;
        CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, kind, stream));
        return SPH_OK;
    }

    double *stage(int slot) const { return dStage + (size_t)slot * capacity; }

    int readError()
    {
        CUDA_TRY(cudaMemcpyAsync(hCtl, ctl, sizeof(Control), cudaMemcpyDeviceToHost, stream));
        CUDA_TRY(cudaStreamSynchronize(stream));
        if (hCtl->error & kErrNonFinite) return fail(SPH_ERR_NONFINITE, "the state stopped being finite");
        if (hCtl->error & kErrTimeStep) return fail(SPH_ERR_TIMESTEP, "the time step collapsed");
        return SPH_OK;
    }

    int writeControl()
    {
        CUDA_TRY(cudaMemcpyAsync(ctl, hCtl, sizeof(Control), cudaMemcpyHostToDevice, stream));
        return SPH_OK;
    }
};

// ================================================================================================
// C-ABI
// ================================================================================================

#define CHECK_SYS(sys)                                                                                   \
    do {                                                                                                 \
        if (!(sys)) return fail(SPH_ERR_INVALID, "null handle");                                        \
        cudaSetDevice((sys)->device);                                                                    \
    } while (0)

extern "C" {

const char *sph_last_error(void) { return lastError.c_str(); }

int sph_version(void) { return 1; }

int sph_kernel_architecture(int *version)
{
    if (!version) return fail(SPH_ERR_INVALID, "null output");
    cudaFuncAttributes attributes{};
    CUDA_TRY(kernelAttributes(&attributes));
    *version = attributes.binaryVersion;
    return SPH_OK;
}

int sph_create(int dimensions, double smoothing_length, const double *domain_min, const double *domain_max,
               double period, int precise, int kernel_type, int device, SphSystem **out)
{
    if (!out) return fail(SPH_ERR_INVALID, "null output handle");
    *out = nullptr;
    if (dimensions != 2 && dimensions != 3) return fail(SPH_ERR_INVALID, "dimensions must be 2 or 3");
    if (!(smoothing_length > 0.0)) return fail(SPH_ERR_INVALID, "the smoothing length must be positive");
    if (kernel_type != 0 && kernel_type != 1) return fail(SPH_ERR_INVALID, "kernel type must be 0 or 1");
    if (period > 0.0 && dimensions != 3) return fail(SPH_ERR_INVALID, "a periodic axis needs three dimensions");
    if (!domain_min || !domain_max) return fail(SPH_ERR_INVALID, "null domain");
    CUDA_TRY(cudaSetDevice(device));
    SphSystem *s = new SphSystem();
    s->device = device;
    s->dim = dimensions;
    s->kind = kernel_type;
    s->h = smoothing_length;
    s->period = period > 0.0 ? period : 0.0;
    s->precise = precise ? 1 : 0;
    for (int a = 0; a < dimensions; ++a) {
        s->domainMin[a] = domain_min[a];
        s->domainMax[a] = std::max(domain_max[a], domain_min[a]);
    }
    s->hMin = smoothing_length;
    int status = SPH_OK;
    if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess) status = SPH_ERR_CUDA;
    s->ownStream = true;
    if (status == SPH_OK && cudaMalloc((void **)&s->ctl, sizeof(Control)) != cudaSuccess) status = SPH_ERR_NOMEM;
    if (status == SPH_OK && cudaMallocHost((void **)&s->hCtl, sizeof(Control)) != cudaSuccess) status = SPH_ERR_NOMEM;
    if (status == SPH_OK && (cudaEventCreate(&s->evStart) != cudaSuccess || cudaEventCreate(&s->evStop) != cudaSuccess ||
                             cudaEventCreateWithFlags(&s->uploaded, cudaEventDisableTiming) != cudaSuccess))
        status = SPH_ERR_CUDA;
    for (int b = 0; b < 2 && status == SPH_OK; ++b)
        for (int k = 0; k <= kStageCount && status == SPH_OK; ++k)
            if (cudaEventCreate(&s->stageEvents[b][k]) != cudaSuccess) status = SPH_ERR_CUDA;
    if (status == SPH_OK) status = s->setupGrid();
    if (status != SPH_OK) {
        sph_destroy(s);
        return fail(status, "sph_create: " + lastError);
    }
    memset(s->hCtl, 0, sizeof(Control));
    s->hCtl->active = 1;
    cudaMemcpy(s->ctl, s->hCtl, sizeof(Control), cudaMemcpyHostToDevice);
    *out = s;
    return SPH_OK;
}

int sph_destroy(SphSystem *sys)
{
    if (!sys) return SPH_OK;
    cudaSetDevice(sys->device);
    if (sys->stream) cudaStreamSynchronize(sys->stream);
    for (int b = 0; b < 2; ++b) {
        if (sys->graphs[b]) cudaGraphExecDestroy(sys->graphs[b]);
        for (int k = 0; k <= kStageCount; ++k)
            if (sys->stageEvents[b][k]) cudaEventDestroy(sys->stageEvents[b][k]);
    }
    sys->freeArrays();
    cudaFree(sys->energy);
    cudaFree(sys->parts);
    cudaFree(sys->dSums);
    cudaFree(sys->cellStart);
    cudaFree(sys->sortBuffers.cellCount);
    cudaFree(sys->sortBuffers.partials);
    cudaFree(sys->dMaxCount);
    cudaFree(sys->surface);
    cudaFree(sys->ctl);
    cudaFree(sys->bedX);
    cudaFree(sys->bedZ);
    cudaFree(sys->table);
    if (sys->hCtl) cudaFreeHost(sys->hCtl);
    if (sys->evStart) cudaEventDestroy(sys->evStart);
    if (sys->evStop) cudaEventDestroy(sys->evStop);
    if (sys->uploaded) cudaEventDestroy(sys->uploaded);
    if (sys->ownStream && sys->stream) cudaStreamDestroy(sys->stream);
    delete sys;
    return SPH_OK;
}

int sph_grid_shape(const SphSystem *sys, int64_t shape[3])
{
    if (!sys || !shape) return fail(SPH_ERR_INVALID, "null argument");
    for (int a = 0; a < 3; ++a) shape[a] = sys->gridShape[a];
    return SPH_OK;
}

int sph_set_cells_per_support(SphSystem *sys, int cells)
{
    CHECK_SYS(sys);
    if (cells < 1 || cells > 4) return fail(SPH_ERR_INVALID, "cells per support must be 1 to 4");
    sys->ncs = cells;
    return sys->setupGrid();
}

int sph_set_sweep_options(SphSystem *sys, int neighbor_table, int threads_per_particle)
{
    CHECK_SYS(sys);
    if (neighbor_table != 0 && neighbor_table != 1) return fail(SPH_ERR_INVALID, "neighbor_table must be 0 or 1");
    if (threads_per_particle != 1 && threads_per_particle != 2 && threads_per_particle != 4 &&
        threads_per_particle != 8)
        return fail(SPH_ERR_INVALID, "threads per particle must be 1, 2, 4 or 8");
    sys->tableMode = neighbor_table;
    sys->threads = threads_per_particle;
    sys->listDirty = true;
    sys->graphDirty = true;
    if (neighbor_table == 0 && sys->listCap) sys->listCap = 0;
    return SPH_OK;
}

int sph_neighbor_table(const SphSystem *sys, int64_t *row_capacity)
{
    if (!sys || !row_capacity) return fail(SPH_ERR_INVALID, "null argument");
    *row_capacity = sys->listCap;
    return SPH_OK;
}

int sph_set_stream(SphSystem *sys, void *stream)
{
    CHECK_SYS(sys);
    cudaStreamSynchronize(sys->stream);
    if (sys->ownStream && sys->stream) cudaStreamDestroy(sys->stream);
    if (stream) {
        sys->stream = (cudaStream_t)stream;
        sys->ownStream = false;
    } else {
        CUDA_TRY(cudaStreamCreateWithFlags(&sys->stream, cudaStreamNonBlocking));
        sys->ownStream = true;
    }
    sys->graphDirty = true;
    return SPH_OK;
}

int sph_set_diffusion(SphSystem *sys, int mode, double delta, double sound_speed, double reference_density,
                      double gravity)
{
    CHECK_SYS(sys);
    if (mode < 0 || mode > 3) return fail(SPH_ERR_INVALID, "diffusion mode must be 0 to 3");
    if (!(sound_speed > 0.0)) return fail(SPH_ERR_INVALID, "the sound speed must be positive");
    sys->diffusionMode = mode;
    sys->diffusionDelta = delta;
    sys->diffusionC0 = sound_speed;
    sys->diffusionRho0 = reference_density;
    sys->diffusionG = gravity;
    sys->graphDirty = true;
    return SPH_OK;
}

int sph_set_wall_pressure(SphSystem *sys, int extrapolated)
{
    CHECK_SYS(sys);
    sys->wallExtrapolated = extrapolated ? 1 : 0;
    sys->graphDirty = true;
    return SPH_OK;
}

int sph_set_negative_pressure(SphSystem *sys, int enabled)
{
    CHECK_SYS(sys);
    sys->tension = enabled ? 1 : 0;
    sys->graphDirty = true;
    return SPH_OK;
}

int sph_set_continuity_correction(SphSystem *sys, int enabled)
{
    CHECK_SYS(sys);
    sys->corrected = enabled ? 1 : 0;
    sys->graphDirty = true;
    return SPH_OK;
}

int sph_set_closure(SphSystem *sys, int enabled, double sound_speed, double reference_density,
                    double kinematic_viscosity)
{
    CHECK_SYS(sys);
    if (enabled && (!(sound_speed > 0.0) || !(reference_density > 0.0) || !(kinematic_viscosity >= 0.0)))
        return fail(SPH_ERR_INVALID, "the closure needs a positive sound speed and density, a viscosity >= 0");
    sys->closure = enabled ? 1 : 0;
    if (enabled) {
        sys->closureC0 = sound_speed;
        sys->closureRho0 = reference_density;
        sys->closureNu = kinematic_viscosity;
    }
    sys->graphDirty = true;
    return SPH_OK;
}

int sph_set_shifting(SphSystem *sys, int enabled, double mach, double spacing, double sound_speed, int local)
{
    CHECK_SYS(sys);
    if (enabled && (!(spacing > 0.0) || !(sound_speed > 0.0) || !(mach >= 0.0)))
        return fail(SPH_ERR_INVALID, "shifting needs a positive spacing and sound speed, a Mach number >= 0");
    if (enabled && sys->mixedH)
        return fail(SPH_ERR_INVALID, "particle shifting needs one smoothing length for every particle");
    sys->shifting = enabled ? 1 : 0;
    if (enabled) {
        sys->shiftLocal = local ? 1 : 0;
        sys->spacingKernel = kernelValueHost(sys->kind, sys->dim, spacing, sys->h);
        sys->shiftScale = sound_speed * mach * 4.0 * sys->h;
    }
    sys->graphDirty = true;
    return SPH_OK;
}

int sph_set_energy_budget(SphSystem *sys, int enabled)
{
    CHECK_SYS(sys);
    if (enabled && sys->compensated)
        return fail(SPH_ERR_UNSUPPORTED, "the energy budget's sweeps keep plain sums; turn compensated sums off first");
    sys->budget = enabled ? 1 : 0;
    if (enabled) TRY(sys->reserveBudget(true));
    sys->graphDirty = true;
    return SPH_OK;
}

int sph_set_compensated_sums(SphSystem *sys, int enabled)
{
    CHECK_SYS(sys);
    if (enabled && sys->budget)
        return fail(SPH_ERR_UNSUPPORTED, "the energy budget's sweeps keep plain sums; turn the budget off first");
    sys->compensated = enabled ? 1 : 0;
    sys->graphDirty = true;
    return SPH_OK;
}

int sph_energy_sums(SphSystem *sys, double *sums)
{
    CHECK_SYS(sys);
    if (!sums) return fail(SPH_ERR_INVALID, "null argument");
    if (!sys->budget) return fail(SPH_ERR_STATE, "the energy budget is off; see sph_set_energy_budget");
    for (int t = 0; t < kEnergyTerms; ++t) sums[t] = 0.0;
    if (sys->n == 0 || !sys->energy) return SPH_OK;
    if (!sys->dSums) TRY(deviceAlloc(&sys->dSums, kEnergyTerms));
    double *out = sys->dSums;
    launchColumnSums(sys->energy, sys->energyCap, sys->n, kEnergyTerms, out, sys->stream);
    CUDA_TRY(cudaGetLastError());
    TRY(sys->download(sums, out, sizeof(double) * kEnergyTerms));
    CUDA_TRY(cudaStreamSynchronize(sys->stream));
    return SPH_OK;
}

int sph_fluid_energy(SphSystem *sys, double *energies)
{
    CHECK_SYS(sys);
    if (!energies) return fail(SPH_ERR_INVALID, "null argument");
    if (!sys->resident) return fail(SPH_ERR_STATE, "no device state: call sph_push first");
    if (!sys->physicsSet) return fail(SPH_ERR_STATE, "call sph_set_physics first");
    energies[0] = energies[1] = energies[2] = 0.0;
    if (sys->n == 0) return SPH_OK;
    if (!sys->dSums) TRY(deviceAlloc(&sys->dSums, kEnergyTerms));
    double *columns = sys->stage(SphSystem::kOutSlot), *out = sys->dSums;
    launchFluidEnergy(sys->params(), sys->frame(), columns, sys->capacity, sys->stream);
    launchColumnSums(columns, sys->capacity, sys->n, 3, out, sys->stream);
    CUDA_TRY(cudaGetLastError());
    TRY(sys->download(energies, out, sizeof(double) * 3));
    CUDA_TRY(cudaStreamSynchronize(sys->stream));
    return SPH_OK;
}

int sph_set_viscosity_limiter(SphSystem *sys, int enabled)
{
    CHECK_SYS(sys);
    sys->limited = enabled ? 1 : 0;
    sys->graphDirty = true;
    return SPH_OK;
}

int sph_set_physics(SphSystem *sys, double reference_density, double sound_speed, double alpha,
                    double boundary_viscosity_factor, const double *gravity, double xsph_epsilon, double density_floor)
{
    CHECK_SYS(sys);
    if (!gravity) return fail(SPH_ERR_INVALID, "null gravity");
    if (!(reference_density > 0.0) || !(sound_speed > 0.0))
        return fail(SPH_ERR_INVALID, "the reference density and sound speed must be positive");
    sys->rho0 = reference_density;
    sys->c0 = sound_speed;
    sys->alpha = alpha;
    sys->boundaryFactor = boundary_viscosity_factor;
    for (int a = 0; a < 3; ++a) sys->gravity[a] = a < sys->dim ? gravity[a] : 0.0;
    sys->xsphEpsilon = xsph_epsilon;
    sys->densityFloor = density_floor;
    sys->physicsSet = true;
    sys->graphDirty = true;
    return SPH_OK;
}

// ---- host steps -------------------------------------------------------------------------------

// kind: cudaMemcpyHostToDevice for the caller's host arrays, cudaMemcpyDeviceToDevice for its
// device arrays (the lengths, which the host checks, are then read back first).
// A push's smoothing lengths at a glance: their range, how many are not the grid's h, and the longest
// below h (the fine level's, 0 for none).  Order-free, so the host threads that share a long array
// give the bits one thread would.
struct LengthRange {
    double top, bottom, below;
    long long others;
};

static LengthRange scanLengthSpan(const double *lengths, long long begin, long long end, double h)
{
    LengthRange r{lengths[begin], lengths[begin], 0.0, 0};
    for (long long i = begin; i < end; ++i) {
        const double l = lengths[i];
        r.top = std::max(r.top, l);
        r.bottom = std::min(r.bottom, l);
        r.others += l != h;
        r.below = std::max(r.below, l < h ? l : 0.0);
    }
    return r;
}

static LengthRange scanLengths(const double *lengths, int n, double h)
{
    const unsigned cores = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    const int parts = n >= (1 << 20) ? (int)cores : 1;
    if (parts == 1) return scanLengthSpan(lengths, 0, n, h);
    std::vector<LengthRange> found(parts);
    std::vector<std::thread> threads;
    for (int t = 1; t < parts; ++t) {
        const long long begin = (long long)n * t / parts, end = (long long)n * (t + 1) / parts;
        try {
            threads.emplace_back([&found, lengths, begin, end, h, t] { found[t] = scanLengthSpan(lengths, begin, end, h); });
        } catch (...) {
            found[t] = scanLengthSpan(lengths, begin, end, h);     // no thread to be had: scan the part here
        }
    }
    found[0] = scanLengthSpan(lengths, 0, (long long)n / parts, h);
    for (auto &thread : threads) thread.join();
    LengthRange r = found[0];
    for (int t = 1; t < parts; ++t) {
        r.top = std::max(r.top, found[t].top);
        r.bottom = std::min(r.bottom, found[t].bottom);
        r.below = std::max(r.below, found[t].below);
        r.others += found[t].others;
    }
    return r;
}

static int loadState(SphSystem *sys, int64_t count, const double *positions, const double *velocities,
                     const double *densities, const double *masses, const uint8_t *is_fluid, const double *lengths,
                     cudaMemcpyKind kind = cudaMemcpyHostToDevice)
{
    if (count < 0 || count > (int64_t)0x3FFFFFFF) return fail(SPH_ERR_INVALID, "particle count out of range");
    if (count > 0 && (!positions || !masses || !is_fluid)) return fail(SPH_ERR_INVALID, "null state array");
    int n = (int)count;
    const double *deviceLengths = nullptr;
    std::vector<double> hostLengths;
    if (kind == cudaMemcpyDeviceToDevice && lengths && n > 0) {
        deviceLengths = lengths;
        hostLengths.resize(n);
        CUDA_TRY(cudaMemcpyAsync(hostLengths.data(), deviceLengths, sizeof(double) * n, cudaMemcpyDeviceToHost,
                                 sys->stream));
        CUDA_TRY(cudaStreamSynchronize(sys->stream));
        lengths = hostLengths.data();
    }
    double hMax = 0.0, hMin = sys->h, fineLongest = 0.0;
    bool mixed = false;
    if (lengths && n > 0) {
        const LengthRange range = scanLengths(lengths, n, sys->h);
        hMax = range.top;
        hMin = range.bottom;
        mixed = range.others > 0;
        fineLongest = range.below;
        if (hMax > sys->h * (1.0 + 1e-9))
            return fail(SPH_ERR_INVALID, "a smoothing length of " + std::to_string(hMax) + " m exceeds the " +
                                             std::to_string(sys->h) + " m the cell list is built for");
        if (!(hMin > 0.0)) return fail(SPH_ERR_INVALID, "smoothing lengths must be positive");
    }
    if (mixed && sys->shifting)
        return fail(SPH_ERR_INVALID, "particle shifting needs one smoothing length for every particle");
    TRY(sys->reserve(n, false));
    TRY(sys->takeFineLength(lengths ? fineLongest : 0.0));
    if (sys->n != n) sys->graphDirty = true;
    sys->n = n;
    sys->mixedH = mixed;
    sys->hMin = lengths && n > 0 ? hMin : sys->h;
    if (n == 0) return SPH_OK;
    int dim = sys->dim;
    double *sx = sys->stage(0), *sv = sys->stage(3), *srho = sys->stage(6), *sm = sys->stage(7), *sh = sys->stage(8);
    TRY(sys->upload(sx, positions, sizeof(double) * n * dim, kind));
    if (velocities) TRY(sys->upload(sv, velocities, sizeof(double) * n * dim, kind));
    if (densities) TRY(sys->upload(srho, densities, sizeof(double) * n, kind));
    TRY(sys->upload(sm, masses, sizeof(double) * n, kind));
    if (deviceLengths) TRY(sys->upload(sh, deviceLengths, sizeof(double) * n, kind));
    else if (lengths) TRY(sys->upload(sh, lengths, sizeof(double) * n));
    TRY(sys->upload(sys->dStageU8, is_fluid, n, kind));
    CUDA_TRY(cudaEventRecord(sys->uploaded, sys->stream));
    sys->cur = 0;
    launchLoadMaster(n, dim, sx, velocities ? sv : nullptr, densities ? srho : nullptr, sm, sys->dStageU8,
                     lengths ? sh : nullptr, sys->h, sys->master[0], sys->stream);
    CUDA_TRY(cudaGetLastError());
    sys->framed = false;
    sys->cellsFresh = false;    // new positions: the cell list is sorted again before its next use
    return SPH_OK;
}

int sph_update(SphSystem *sys, int64_t n, const double *positions, const double *masses, const uint8_t *is_fluid,
               const double *lengths)
{
    CHECK_SYS(sys);
    TRY(loadState(sys, n, positions, nullptr, nullptr, masses, is_fluid, lengths));
    sys->resident = false;
    sys->rebuild();
    if (sys->listDirty) TRY(sys->sizeList());
    CUDA_TRY(cudaGetLastError());
    // the caller's arrays are free once the copies in are done (pinned memory copies behind the return)
    if (sys->n > 0) CUDA_TRY(cudaEventSynchronize(sys->uploaded));
    return SPH_OK;
}

static int needFrame(SphSystem *sys)
{
    if (sys->n > 0 && (!sys->framed || !sys->cellsFresh)) sys->rebuild();
    return SPH_OK;
}

// Upload caller-order fields into the frame.
static int loadFields(SphSystem *sys, const double *v, const double *rho, const double *p)
{
    int n = sys->n, dim = sys->dim;
    if (n == 0) return SPH_OK;
    double *sv = sys->stage(0), *srho = sys->stage(3), *sp = sys->stage(4);
    if (v) TRY(sys->upload(sv, v, sizeof(double) * n * dim));
    if (rho) TRY(sys->upload(srho, rho, sizeof(double) * n));
    if (p) TRY(sys->upload(sp, p, sizeof(double) * n));
    Params P = sys->params();
    launchLoadFields(P, n, sys->master[sys->cur].orig, v ? sv : nullptr, rho ? srho : nullptr, p ? sp : nullptr,
                     sys->diffusionRho0, sys->frame(), sys->stream);
    CUDA_TRY(cudaGetLastError());
    return SPH_OK;
}

static int finish(SphSystem *sys, double *out, size_t count)
{
    if (sys->n == 0) return SPH_OK;
    double *dOut = sys->stage(SphSystem::kOutSlot);
    TRY(sys->download(out, dOut, sizeof(double) * count));
    CUDA_TRY(cudaStreamSynchronize(sys->stream));
    CUDA_TRY(cudaGetLastError());
    return SPH_OK;
}

int sph_pair_accelerations(SphSystem *sys, const double *velocities, const double *densities, const double *pressures,
                           double sound_speed, double alpha, double boundary_factor, const double *gravity,
                           double *out)
{
    CHECK_SYS(sys);
    TRY(needFrame(sys));
    if (sys->n > 0 && (!velocities || !densities || !pressures || !gravity || !out))
        return fail(SPH_ERR_INVALID, "null argument");
    if (sys->n == 0) return SPH_OK;
    TRY(loadFields(sys, velocities, densities, pressures));
    LaunchArgs A = sys->args(nullptr);
    A.P.c0 = (float)sound_speed;
    A.P.alpha = (float)alpha;
    A.P.boundaryFactor = (float)boundary_factor;
    for (int a = 0; a < 3; ++a) A.P.g[a] = a < sys->dim ? (float)gravity[a] : 0.0f;
    if (sys->limited || sys->closure) {
        A.wantG = 1;
        launchStage(A, Stage::Gradients);
    }
    if (sys->closure) launchStage(A, Stage::Closure);     // kept for the next continuityRate, as the reference does
    launchStage(A, Stage::Momentum);
    launchScatterFloat4(sys->n, sys->dim, A.F.orig, sys->acc, sys->stage(SphSystem::kOutSlot), sys->stream);
    return finish(sys, out, (size_t)sys->n * sys->dim);
}

int sph_continuity_rate(SphSystem *sys, const double *velocities, const double *densities, double *out)
{
    CHECK_SYS(sys);
    TRY(needFrame(sys));
    if (sys->n == 0) return SPH_OK;
    if (!velocities || !out) return fail(SPH_ERR_INVALID, "null argument");
    bool needsDensity = sys->diffusionMode != 0 || sys->corrected;
    if (needsDensity && !densities)
        return fail(SPH_ERR_INVALID, "the diffusive term and the correction need the densities");
    TRY(loadFields(sys, velocities, needsDensity ? densities : nullptr, nullptr));
    LaunchArgs A = sys->args(nullptr);
    if (sys->corrected || sys->diffusionMode == 3) {
        A.wantL = 1;
        A.wantRho = sys->diffusionMode == 3;
        launchStage(A, Stage::Gradients);
        A.wantL = A.wantRho = 0;
    }
    A.flag = 0;
    launchStage(A, Stage::Continuity);
    launchScatterFloat(sys->n, A.F.orig, sys->rate, sys->stage(SphSystem::kOutSlot), sys->stream);
    return finish(sys, out, sys->n);
}

int sph_xsph_velocity(SphSystem *sys, const double *velocities, const double *densities, double epsilon, double *out)
{
    CHECK_SYS(sys);
    TRY(needFrame(sys));
    if (sys->n == 0) return SPH_OK;
    if (!velocities || !densities || !out) return fail(SPH_ERR_INVALID, "null argument");
    TRY(loadFields(sys, velocities, densities, nullptr));
    LaunchArgs A = sys->args(nullptr);
    A.P.xsphEpsilon = (float)epsilon;
    A.flag = 0;
    A.densities = nullptr;
    launchStage(A, Stage::Xsph);
    launchScatterFloat4(sys->n, sys->dim, A.F.orig, sys->vec, sys->stage(SphSystem::kOutSlot), sys->stream);
    return finish(sys, out, (size_t)sys->n * sys->dim);
}

int sph_wall_pressure(SphSystem *sys, const double *densities, const double *pressures, const double *gravity,
                      double reference_density, double sound_speed, double *out)
{
    CHECK_SYS(sys);
    TRY(needFrame(sys));
    if (sys->n == 0) return SPH_OK;
    if (!densities || !pressures || !gravity || !out) return fail(SPH_ERR_INVALID, "null argument");
    TRY(loadFields(sys, nullptr, densities, pressures));
    LaunchArgs A = sys->args(nullptr);
    for (int a = 0; a < 3; ++a) A.P.g[a] = a < sys->dim ? (float)gravity[a] : 0.0f;
    A.P.rho0 = reference_density;
    A.P.stiffness = reference_density * sound_speed * sound_speed / 7.0;
    A.flag = 0;
    launchStage(A, Stage::Wall);
    launchScatterPressure(sys->n, sys->dim, A.F.orig, A.F, sys->stage(SphSystem::kOutSlot), sys->stream);
    return finish(sys, out, sys->n);
}

int sph_shepard_density(SphSystem *sys, const double *densities, double *out)
{
    CHECK_SYS(sys);
    TRY(needFrame(sys));
    if (sys->n == 0) return SPH_OK;
    if (!densities || !out) return fail(SPH_ERR_INVALID, "null argument");
    TRY(loadFields(sys, nullptr, densities, nullptr));
    LaunchArgs A = sys->args(nullptr);
    launchStage(A, Stage::ShepardSum);
    launchScatterFloat(sys->n, A.F.orig, sys->scalar, sys->stage(SphSystem::kOutSlot), sys->stream);
    return finish(sys, out, sys->n);
}

int sph_velocity_gradients(SphSystem *sys, const double *velocities, const double *densities, double *out)
{
    CHECK_SYS(sys);
    TRY(needFrame(sys));
    if (sys->n == 0) return SPH_OK;
    if (!velocities || !densities || !out) return fail(SPH_ERR_INVALID, "null argument");
    TRY(loadFields(sys, velocities, densities, nullptr));
    LaunchArgs A = sys->args(nullptr);
    A.wantG = 1;
    launchStage(A, Stage::Gradients);
    launchScatterMatrix(sys->n, sys->dim, A.F.orig, A.F, 0, sys->stage(SphSystem::kOutSlot), sys->stream);
    return finish(sys, out, (size_t)sys->n * sys->dim * sys->dim);
}

int sph_closure_coefficients(SphSystem *sys, const double *velocities, const double *densities, double *alphas,
                             double *deltas)
{
    CHECK_SYS(sys);
    TRY(needFrame(sys));
    if (!sys->closure) return fail(SPH_ERR_STATE, "the closure is off: call sph_set_closure first");
    if (sys->n == 0) return SPH_OK;
    if (!velocities || !densities || !alphas || !deltas) return fail(SPH_ERR_INVALID, "null argument");
    TRY(loadFields(sys, velocities, densities, nullptr));
    LaunchArgs A = sys->args(nullptr);
    A.wantG = 1;
    launchStage(A, Stage::Gradients);
    launchStage(A, Stage::Closure);
    // the two halves of (alpha, delta), scattered to the caller's order
    std::vector<float2> packed(sys->n);
    std::vector<int> orig(sys->n);
    CUDA_TRY(cudaMemcpyAsync(packed.data(), sys->eddy, sizeof(float2) * sys->n, cudaMemcpyDeviceToHost, sys->stream));
    CUDA_TRY(cudaMemcpyAsync(orig.data(), A.F.orig, sizeof(int) * sys->n, cudaMemcpyDeviceToHost, sys->stream));
    CUDA_TRY(cudaStreamSynchronize(sys->stream));
    for (int s = 0; s < sys->n; ++s) {
        alphas[orig[s]] = packed[s].x;
        deltas[orig[s]] = packed[s].y;
    }
    return SPH_OK;
}

int sph_shifting_displacement(SphSystem *sys, const double *densities, double time_step, const double *velocities,
                              double *shifts, double *density_changes, double *velocity_changes)
{
    CHECK_SYS(sys);
    TRY(needFrame(sys));
    if (!sys->shifting) return fail(SPH_ERR_STATE, "shifting is off: call sph_set_shifting first");
    if (sys->mixedH) return fail(SPH_ERR_INVALID, "particle shifting needs one smoothing length for every particle");
    if (sys->n == 0) return SPH_OK;
    if (!densities || !velocities || !shifts || !density_changes || !velocity_changes)
        return fail(SPH_ERR_INVALID, "null argument");
    TRY(loadFields(sys, velocities, densities, nullptr));
    LaunchArgs A = sys->args(nullptr);
    A.P.shiftDt = time_step;
    launchStage(A, Stage::ShiftFields);
    launchStage(A, Stage::Shift);
    const int n = sys->n, dim = sys->dim;
    double *out = sys->stage(SphSystem::kOutSlot);
    launchScatterFloat4(n, dim, A.F.orig, sys->shiftOut, out, sys->stream);
    TRY(sys->download(shifts, out, sizeof(double) * n * dim));
    CUDA_TRY(cudaStreamSynchronize(sys->stream));
    launchScatterFloat4(n, dim, A.F.orig, sys->shiftDv, out, sys->stream);
    TRY(sys->download(velocity_changes, out, sizeof(double) * n * dim));
    CUDA_TRY(cudaStreamSynchronize(sys->stream));
    // the density changes ride in the shifts' fourth lane
    std::vector<float4> packed(n);
    std::vector<int> orig(n);
    CUDA_TRY(cudaMemcpyAsync(packed.data(), sys->shiftOut, sizeof(float4) * n, cudaMemcpyDeviceToHost, sys->stream));
    CUDA_TRY(cudaMemcpyAsync(orig.data(), A.F.orig, sizeof(int) * n, cudaMemcpyDeviceToHost, sys->stream));
    CUDA_TRY(cudaStreamSynchronize(sys->stream));
    for (int s = 0; s < n; ++s) density_changes[orig[s]] = packed[s].w;
    return SPH_OK;
}

int sph_correction_matrices(SphSystem *sys, const double *densities, double *out)
{
    CHECK_SYS(sys);
    TRY(needFrame(sys));
    if (sys->n == 0) return SPH_OK;
    if (!densities || !out) return fail(SPH_ERR_INVALID, "null argument");
    TRY(loadFields(sys, nullptr, densities, nullptr));
    LaunchArgs A = sys->args(nullptr);
    A.wantL = 1;
    launchStage(A, Stage::Gradients);
    launchScatterMatrix(sys->n, sys->dim, A.F.orig, A.F, 1, sys->stage(SphSystem::kOutSlot), sys->stream);
    return finish(sys, out, (size_t)sys->n * sys->dim * sys->dim);
}

int sph_density_gradients(SphSystem *sys, const double *densities, double *out)
{
    CHECK_SYS(sys);
    TRY(needFrame(sys));
    if (sys->n == 0) return SPH_OK;
    if (!densities || !out) return fail(SPH_ERR_INVALID, "null argument");
    TRY(loadFields(sys, nullptr, densities, nullptr));
    LaunchArgs A = sys->args(nullptr);
    A.wantRho = 1;
    launchStage(A, Stage::Gradients);
    launchScatterFloat4(sys->n, sys->dim, A.F.orig, sys->gradRho, sys->stage(SphSystem::kOutSlot), sys->stream);
    return finish(sys, out, (size_t)sys->n * sys->dim);
}

// ---- device-resident steps ------------------------------------------------------------------------

static int pushState(SphSystem *sys, int64_t n, const double *positions, const double *velocities,
                     const double *densities, const double *masses, const uint8_t *is_fluid, const double *lengths,
                     cudaMemcpyKind kind)
{
    CHECK_SYS(sys);
    if (n > 0 && (!velocities || !densities)) return fail(SPH_ERR_INVALID, "null state array");
    TRY(loadState(sys, n, positions, velocities, densities, masses, is_fluid, lengths, kind));
    sys->resident = true;
    // the cell list, the frame and the table follow at the first step or host-step call; the table
    // keeps its row length unless the count changed (a particle whose row is too short walks)
    if (sys->listCap == 0 || sys->listSizedFor != sys->n) sys->listDirty = true;
    // the energy budget counts from the push (src/pysurf/sphGpu.py:2207-2221)
    if (sys->budget && sys->energy)
        CUDA_TRY(cudaMemsetAsync(sys->energy, 0, sizeof(double) * kEnergyTerms * sys->energyCap, sys->stream));
    CUDA_TRY(cudaGetLastError());
    // the caller's arrays are free once the copies in are done; the kernels after them run on
    // behind the return, in stream order before any later call's work
    CUDA_TRY(sys->n > 0 ? cudaEventSynchronize(sys->uploaded) : cudaStreamSynchronize(sys->stream));
    return SPH_OK;
}

int sph_push(SphSystem *sys, int64_t n, const double *positions, const double *velocities, const double *densities,
             const double *masses, const uint8_t *is_fluid, const double *lengths)
{
    return pushState(sys, n, positions, velocities, densities, masses, is_fluid, lengths, cudaMemcpyHostToDevice);
}

int sph_push_device(SphSystem *sys, int64_t n, const double *positions, const double *velocities,
                    const double *densities, const double *masses, const uint8_t *is_fluid, const double *lengths)
{
    return pushState(sys, n, positions, velocities, densities, masses, is_fluid, lengths, cudaMemcpyDeviceToDevice);
}

int sph_frame(SphSystem *sys, float *positions, float *speeds, uint8_t *is_fluid)
{
    CHECK_SYS(sys);
    if (!positions || !speeds || !is_fluid) return fail(SPH_ERR_INVALID, "null argument");
    if (!sys->resident) return fail(SPH_ERR_STATE, "no device state: call sph_push first");
    const int n = sys->n, dim = sys->dim;
    if (n == 0) return SPH_OK;
    // float32 rows in the output staging: positions, then speeds
    float *pos = reinterpret_cast<float *>(sys->stage(SphSystem::kOutSlot));
    float *speed = reinterpret_cast<float *>(sys->stage(SphSystem::kOutSlot + 2));
    launchFrame(n, dim, sys->master[sys->cur], pos, speed, sys->dStageU8, sys->stream);
    CUDA_TRY(cudaGetLastError());
    TRY(sys->download(positions, pos, sizeof(float) * (size_t)n * dim));
    TRY(sys->download(speeds, speed, sizeof(float) * (size_t)n));
    TRY(sys->download(is_fluid, sys->dStageU8, (size_t)n));
    CUDA_TRY(cudaStreamSynchronize(sys->stream));
    return SPH_OK;
}

int sph_count(const SphSystem *sys, int64_t *n)
{
    if (!sys || !n) return fail(SPH_ERR_INVALID, "null argument");
    *n = sys->n;
    return SPH_OK;
}

static int pullState(SphSystem *sys, double *positions, double *velocities, double *densities, double *pressures,
                     double *accelerations, double *masses, double *lengths, uint8_t *is_fluid, cudaMemcpyKind kind)
{
    CHECK_SYS(sys);
    int n = sys->n, dim = sys->dim;
    if (n == 0) return SPH_OK;
    // one launch puts every asked field into caller order in its own staging rows (0 .. 12), then
    // the copies out follow in stream order, and one sync at the end
    int slot = 0;
    auto rows = [&](const void *host, int width) -> double * {
        if (!host) return nullptr;
        double *p = sys->stage(slot);
        slot += width;
        return p;
    };
    PullRows R{};
    R.x = rows(positions, dim);
    R.v = rows(velocities, dim);
    R.rho = rows(densities, 1);
    R.m = rows(masses, 1);
    R.h = rows(lengths, 1);
    R.p = rows(pressures, 1);
    R.a = rows(accelerations, dim);
    R.fluid = is_fluid ? sys->dStageU8 : nullptr;
    R.framed = sys->framed ? 1 : 0;
    R.tension = sys->tension;
    R.rho0 = sys->rho0;
    R.stiffness = sys->rho0 * sys->c0 * sys->c0 / 7.0;
    launchPull(n, dim, sys->master[sys->cur], sys->frame(), sys->acc, R, sys->stream);
    CUDA_TRY(cudaGetLastError());
    const size_t column = sizeof(double) * (size_t)n;
    if (R.x) TRY(sys->download(positions, R.x, column * dim, kind));
    if (R.v) TRY(sys->download(velocities, R.v, column * dim, kind));
    if (R.rho) TRY(sys->download(densities, R.rho, column, kind));
    if (R.m) TRY(sys->download(masses, R.m, column, kind));
    if (R.h) TRY(sys->download(lengths, R.h, column, kind));
    if (R.p) TRY(sys->download(pressures, R.p, column, kind));
    if (R.a) TRY(sys->download(accelerations, R.a, column * dim, kind));
    if (R.fluid) TRY(sys->download(is_fluid, R.fluid, (size_t)n, kind));
    CUDA_TRY(cudaStreamSynchronize(sys->stream));
    CUDA_TRY(cudaGetLastError());
    return SPH_OK;
}

int sph_pull(SphSystem *sys, double *positions, double *velocities, double *densities, double *pressures,
             double *accelerations, double *masses, double *lengths, uint8_t *is_fluid)
{
    return pullState(sys, positions, velocities, densities, pressures, accelerations, masses, lengths, is_fluid,
                     cudaMemcpyDeviceToHost);
}

int sph_pull_device(SphSystem *sys, double *positions, double *velocities, double *densities, double *pressures,
                    double *accelerations, double *masses, double *lengths, uint8_t *is_fluid)
{
    return pullState(sys, positions, velocities, densities, pressures, accelerations, masses, lengths, is_fluid,
                     cudaMemcpyDeviceToDevice);
}

int sph_clear_boundary(SphSystem *sys)
{
    CHECK_SYS(sys);
    sys->enforcement = Enforcement{};
    sys->graphDirty = true;
    return SPH_OK;
}

int sph_set_boundary_container(SphSystem *sys, const double *lower, const double *upper, int open_top)
{
    CHECK_SYS(sys);
    if (!lower || !upper) return fail(SPH_ERR_INVALID, "null bounds");
    Enforcement E{};
    E.kind = 1;
    for (int a = 0; a < sys->dim; ++a) { E.lower[a] = lower[a]; E.upper[a] = upper[a]; }
    E.openTop = open_top ? 1 : 0;
    sys->enforcement = E;
    sys->graphDirty = true;
    return SPH_OK;
}

int sph_set_boundary_bed(SphSystem *sys, const double *bed_x, const double *bed_z, int64_t count, double clearance,
                         int side_walls, double width, int offshore_wall, double wall_x, double piston_speed,
                         double end_limit)
{
    CHECK_SYS(sys);
    if (!bed_x || !bed_z || count < 2) return fail(SPH_ERR_INVALID, "a bed needs at least two vertices");
    for (int64_t k = 1; k < count; ++k)
        if (!(bed_x[k] > bed_x[k - 1])) return fail(SPH_ERR_INVALID, "bed x must increase strictly");
    cudaFree(sys->bedX);
    cudaFree(sys->bedZ);
    TRY(deviceAlloc(&sys->bedX, count));
    TRY(deviceAlloc(&sys->bedZ, count));
    CUDA_TRY(cudaMemcpy(sys->bedX, bed_x, sizeof(double) * count, cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(sys->bedZ, bed_z, sizeof(double) * count, cudaMemcpyHostToDevice));
    Enforcement E{};
    E.kind = 2;
    E.bedX = sys->bedX;
    E.bedZ = sys->bedZ;
    E.bedCount = (int)count;
    E.clearance = clearance;
    E.sideWalls = side_walls ? 1 : 0;
    E.width = width;
    E.offshoreWall = offshore_wall ? 1 : 0;
    E.wallX = wall_x;
    E.pistonSpeed = piston_speed;
    E.endLimit = end_limit;
    sys->enforcement = E;
    sys->graphDirty = true;
    return SPH_OK;
}

int sph_set_boundary_height_field(SphSystem *sys, const double *table, int64_t nx, int64_t ny, double origin_x,
                                  double origin_y, double step_x, double step_y, double clearance, double low_y,
                                  double high_y, int offshore_wall, double low_x, double high_x)
{
    CHECK_SYS(sys);
    if (sys->dim != 3) return fail(SPH_ERR_INVALID, "a height field needs three dimensions");
    if (!table || nx < 1 || ny < 1) return fail(SPH_ERR_INVALID, "an empty height table");
    cudaFree(sys->table);
    TRY(deviceAlloc(&sys->table, (size_t)(nx * ny)));
    CUDA_TRY(cudaMemcpy(sys->table, table, sizeof(double) * nx * ny, cudaMemcpyHostToDevice));
    Enforcement E{};
    E.kind = 3;
    E.table = sys->table;
    E.tableNx = (int)nx;
    E.tableNy = (int)ny;
    E.originX = origin_x;
    E.originY = origin_y;
    E.stepX = step_x;
    E.stepY = step_y;
    E.clearance = clearance;
    E.lowY = low_y;
    E.highY = high_y;
    E.offshoreWall = offshore_wall ? 1 : 0;
    E.lowX = low_x;
    E.highX = high_x;
    sys->enforcement = E;
    sys->graphDirty = true;
    return SPH_OK;
}

int sph_enforce_boundary(SphSystem *sys)
{
    CHECK_SYS(sys);
    if (sys->n == 0) return SPH_OK;
    launchEnforce(sys->params(), sys->frame(), sys->enforcement, sys->stream);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaStreamSynchronize(sys->stream));
    sys->cellsFresh = false;    // the positions moved; the next step re-sorts anyway
    return SPH_OK;
}

// The stages a step's events bracket, in order (sph_stage_times reports them in this order).
static const char *const kStageNames[kStageCount] = {"cells", "filter", "wall", "gradients", "momentum", "kick",
                                                      "continuity"};

// Records the event of stage k when a set of events is given (inside a captured step graph).
static void mark(SphSystem *sys, cudaEvent_t *events, int k)
{
    if (events) cudaEventRecordWithFlags(events[k], sys->stream, cudaEventRecordExternal);
}

// The first half of a step: cell list, optional filter, wall pressure, gradients, momentum.
// filter: the Shepard stage is enqueued (the device decides each step whether it is due).
static void enqueueRates(SphSystem *sys, bool filter, cudaEvent_t *events = nullptr)
{
    mark(sys, events, 0);
    sys->rebuild(sys->ctl);
    mark(sys, events, 1);
    LaunchArgs A = sys->args(sys->ctl);
    if (filter) {
        launchStage(A, Stage::ShepardSum);
        launchStage(A, Stage::ShepardApply);
    }
    mark(sys, events, 2);
    if (sys->wallExtrapolated) {
        A.flag = 1;
        launchStage(A, Stage::Wall);
    }
    mark(sys, events, 3);
    bool wantL = sys->corrected || sys->diffusionMode == 3;
    if (sys->limited || sys->closure || wantL) {
        A.wantG = sys->limited || sys->closure;
        A.wantL = wantL;
        A.wantRho = sys->diffusionMode == 3;
        launchStage(A, Stage::Gradients);
        A.wantG = A.wantL = A.wantRho = 0;
    }
    // the closure's coefficients, from this step's starting velocities (the diffusion reuses them)
    if (sys->closure) launchStage(A, Stage::Closure);
    mark(sys, events, 4);
    launchStage(A, Stage::Momentum);
    mark(sys, events, 5);
}

// The second half: kick, continuity with the density update, XSPH, drift and enforcement.
static void enqueueIntegrate(SphSystem *sys, cudaEvent_t *events = nullptr)
{
    LaunchArgs A = sys->args(sys->ctl);
    launchStage(A, Stage::Kick);
    mark(sys, events, 6);
    if (sys->shifting) {
        // the density update, then the shift from the step's starting geometry, the updated
        // densities and the kicked velocities, then one drift (src/pysurf/sphSolver.py:1760-1785)
        A.flag = 1;
        launchStage(A, Stage::Continuity);
        int useTransport = 0;
        if (sys->xsphEpsilon > 0.0) {
            launchRefreshDensity(sys->n, A.F.rho, sys->scalar, sys->stream);
            A.densities = sys->scalar;
            A.flag = 0;
            launchStage(A, Stage::Xsph);
            useTransport = 1;
        }
        launchStage(A, Stage::FrameDensity);
        launchStage(A, Stage::ShiftFields);
        launchStage(A, Stage::Shift);
        A.flag = useTransport;
        launchStage(A, Stage::ShiftDrift);
    } else if (sys->xsphEpsilon > 0.0) {
        A.flag = 1;
        launchStage(A, Stage::Continuity);
        launchRefreshDensity(sys->n, A.F.rho, sys->scalar, sys->stream);
        A.flag = 2;
        A.densities = sys->scalar;
        launchStage(A, Stage::Xsph);
    } else {
        A.flag = 2;
        launchStage(A, Stage::Continuity);
    }
    mark(sys, events, 7);
}

int sph_resident_rates(SphSystem *sys, int filter_density, double *max_speed, double *max_acceleration)
{
    CHECK_SYS(sys);
    if (!sys->resident) return fail(SPH_ERR_STATE, "no device state: call sph_push first");
    if (!sys->physicsSet) return fail(SPH_ERR_STATE, "call sph_set_physics first");
    Control &c = *sys->hCtl;
    c.active = 1;
    c.hostDt = 1;
    c.filterNow = filter_density ? 1 : 0;
    c.filterInterval = 0;
    c.ticket = 0;
    c.error = 0;
    c.vmax = c.amax = 0.0;
    c.vmaxBits = c.amaxBits = 0;
    if (sys->n == 0) {
        if (max_speed) *max_speed = 0.0;
        if (max_acceleration) *max_acceleration = 0.0;
        return SPH_OK;
    }
    if (sys->listDirty) TRY(sys->sizeList());
    TRY(sys->writeControl());
    enqueueRates(sys, filter_density != 0);
    CUDA_TRY(cudaGetLastError());
    TRY(sys->readError());
    if (max_speed) *max_speed = sys->hCtl->vmax;
    if (max_acceleration) *max_acceleration = sys->hCtl->amax;
    return SPH_OK;
}

int sph_resident_integrate(SphSystem *sys, double time_step)
{
    CHECK_SYS(sys);
    if (!sys->resident) return fail(SPH_ERR_STATE, "no device state: call sph_push first");
    if (!(time_step > 0.0) || !isfinite(time_step)) return fail(SPH_ERR_INVALID, "the time step must be positive");
    if (sys->n == 0) return SPH_OK;
    Control &c = *sys->hCtl;
    c.active = 1;
    c.hostDt = 1;
    c.dt = time_step;
    c.error = 0;
    TRY(sys->writeControl());
    enqueueIntegrate(sys);
    CUDA_TRY(cudaGetLastError());
    TRY(sys->readError());
    sys->cellsFresh = false;
    return SPH_OK;
}

// Two single-step graphs, one from each master buffer (a step moves the master to the other
// buffer), each with events between its stages.
static int captureSteps(SphSystem *sys, bool filter)
{
    for (int b = 0; b < 2; ++b) {
        if (sys->graphs[b]) { cudaGraphExecDestroy(sys->graphs[b]); sys->graphs[b] = nullptr; }
    }
    const int keep = sys->cur;
    for (int b = 0; b < 2; ++b) {
        sys->cur = b;
        cudaGraph_t g;
        CUDA_TRY(cudaStreamBeginCapture(sys->stream, cudaStreamCaptureModeThreadLocal));
        enqueueRates(sys, filter, sys->stageEvents[b]);
        enqueueIntegrate(sys, sys->stageEvents[b]);
        launchStepEnd(sys->ctl, sys->stream);
        cudaError_t err = cudaStreamEndCapture(sys->stream, &g);
        if (err != cudaSuccess) return fail(SPH_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(err));
        err = cudaGraphInstantiate(&sys->graphs[b], g, 0);
        if (err == cudaSuccess) {
            size_t nodes = 0;
            cudaGraphGetNodes(g, nullptr, &nodes);
            sys->graphNodes = (int)nodes;
        }
        cudaGraphDestroy(g);
        if (err != cudaSuccess) return fail(SPH_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(err));
    }
    sys->cur = keep;
    sys->graphFilter = filter;
    sys->graphDirty = false;
    return SPH_OK;
}

int sph_begin_steps(SphSystem *sys, double time, int64_t step, double last_dt, double until_time, int64_t max_step,
                    double shortest_length, double cfl, double max_time_step, int64_t filter_interval)
{
    CHECK_SYS(sys);
    if (!sys->resident) return fail(SPH_ERR_STATE, "no device state: call sph_push first");
    if (!sys->physicsSet) return fail(SPH_ERR_STATE, "call sph_set_physics first");
    if (!(shortest_length > 0.0) || !(cfl > 0.0) || !(max_time_step > 0.0))
        return fail(SPH_ERR_INVALID, "the shortest length, CFL number and largest step must be positive");
    if (filter_interval < 0) return fail(SPH_ERR_INVALID, "the filter interval must not be negative");
    Control &c = *sys->hCtl;
    c.time = time;
    c.untilTime = until_time;
    c.step = step;
    c.lastStep = max_step;
    c.hMin = shortest_length;
    c.cfl = cfl;
    c.maxTimeStep = max_time_step;
    c.soundSpeed = sys->c0;
    c.filterInterval = filter_interval;
    c.filterNow = 0;
    c.hostDt = 0;
    c.ticket = 0;
    c.vmaxBits = c.amaxBits = 0;
    c.error = 0;
    c.active = (time < until_time && step < max_step) ? 1 : 0;
    c.dt = last_dt;
    // sizing the table may re-sort (moving the master), so it comes before the buffer is noted
    if (sys->listDirty) TRY(sys->sizeList());
    sys->beginStep = step;
    sys->beginCur = sys->cur;
    sys->enqueued = 0;
    if (sys->n == 0) return SPH_OK;
    TRY(sys->writeControl());
    bool filter = filter_interval > 0;
    if (sys->graphDirty || !sys->graphs[0] || filter != sys->graphFilter) TRY(captureSteps(sys, filter));
    return SPH_OK;
}

int sph_enqueue_steps(SphSystem *sys, int64_t count)
{
    CHECK_SYS(sys);
    if (count < 0) return fail(SPH_ERR_INVALID, "a negative step count");
    if (sys->n == 0) return SPH_OK;
    if (!sys->graphs[0]) return fail(SPH_ERR_STATE, "call sph_begin_steps first");
    for (int64_t k = 0; k < count; ++k) {
        CUDA_TRY(cudaGraphLaunch(sys->graphs[sys->cur], sys->stream));
        sys->lastGraph = sys->cur;
        sys->cur ^= 1;
        ++sys->enqueued;
    }
    return SPH_OK;
}

int sph_finish_steps(SphSystem *sys, double *time, int64_t *step, double *last_dt)
{
    CHECK_SYS(sys);
    if (sys->n > 0) {
        CUDA_TRY(cudaMemcpyAsync(sys->hCtl, sys->ctl, sizeof(Control), cudaMemcpyDeviceToHost, sys->stream));
        CUDA_TRY(cudaStreamSynchronize(sys->stream));
        CUDA_TRY(cudaGetLastError());
        // each step that ran moved the master to the other buffer; steps that did not, did nothing
        const Control &c = *sys->hCtl;
        sys->cur = sys->beginCur ^ (int)((c.step - sys->beginStep) & 1);
        sys->cellsFresh = false;
    }
    const Control &c = *sys->hCtl;
    if (time) *time = c.time;
    if (step) *step = c.step;
    if (last_dt) *last_dt = c.dt;
    if (c.error & kErrNonFinite) return fail(SPH_ERR_NONFINITE, "the state stopped being finite");
    if (c.error & kErrTimeStep) return fail(SPH_ERR_TIMESTEP, "the time step collapsed");
    return SPH_OK;
}

int sph_advance(SphSystem *sys, double *time, int64_t *step, double *last_dt, double until_time, int64_t max_step,
                double shortest_length, double cfl, double max_time_step, int64_t filter_interval)
{
    CHECK_SYS(sys);
    if (!time || !step) return fail(SPH_ERR_INVALID, "null clock");
    TRY(sph_begin_steps(sys, *time, *step, last_dt ? *last_dt : 0.0, until_time, max_step, shortest_length, cfl,
                        max_time_step, filter_interval));
    sys->lastAdvanceMs = 0.0;
    if (sys->n == 0 || !sys->hCtl->active) return SPH_OK;
    CUDA_TRY(cudaEventRecord(sys->evStart, sys->stream));
    const long long maxLaunch = 1 << 20;
    double t = *time, dt = last_dt ? *last_dt : 0.0;
    // a first batch as long as the last step size suggests, within the step limit
    double guess = dt > 0.0 ? (until_time - t) / dt + 1.0 : 2.0;
    long long launches = (long long)std::max(1.0, std::min({guess, (double)(max_step - *step), (double)maxLaunch}));
    int64_t s = *step;
    int status = SPH_OK;
    for (int round = 0; round < 1000000; ++round) {
        TRY(sph_enqueue_steps(sys, launches));
        CUDA_TRY(cudaEventRecord(sys->evStop, sys->stream));
        status = sph_finish_steps(sys, &t, &s, &dt);
        const Control &c = *sys->hCtl;
        if (status != SPH_OK || !c.active) break;
        // launch about as many steps as the clock still needs at the last step's size
        double remaining = c.dt > 0.0 ? (c.untilTime - c.time) / c.dt : 1.0;
        double left = (double)(c.lastStep - c.step);
        launches = (long long)std::max(1.0, std::min({remaining + 1.0, left, (double)maxLaunch}));
    }
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, sys->evStart, sys->evStop);
    sys->lastAdvanceMs = ms;
    *time = t;
    *step = s;
    if (last_dt) *last_dt = dt;
    return status;
}

int sph_last_advance_ms(const SphSystem *sys, double *ms)
{
    if (!sys || !ms) return fail(SPH_ERR_INVALID, "null argument");
    *ms = sys->lastAdvanceMs;
    return SPH_OK;
}

int sph_stage_times(SphSystem *sys, double *ms, int64_t capacity, int64_t *count)
{
    CHECK_SYS(sys);
    if (!count) return fail(SPH_ERR_INVALID, "null argument");
    *count = kStageCount;
    if (!ms || capacity < kStageCount) return ms ? fail(SPH_ERR_CAPACITY, "need one entry per stage") : SPH_OK;
    if (!sys->graphs[0] || sys->enqueued == 0) return fail(SPH_ERR_STATE, "no step has run since sph_begin_steps");
    CUDA_TRY(cudaStreamSynchronize(sys->stream));
    cudaEvent_t *events = sys->stageEvents[sys->lastGraph];
    for (int k = 0; k < kStageCount; ++k) {
        float t = 0.0f;
        CUDA_TRY(cudaEventElapsedTime(&t, events[k], events[k + 1]));
        ms[k] = t;
    }
    return SPH_OK;
}

const char *sph_stage_name(int64_t stage)
{
    return stage >= 0 && stage < kStageCount ? kStageNames[stage] : "";
}

int sph_step_launches(SphSystem *sys, int64_t *kernels)
{
    CHECK_SYS(sys);
    if (!kernels) return fail(SPH_ERR_INVALID, "null argument");
    *kernels = 0;
    if (!sys->graphs[0]) return fail(SPH_ERR_STATE, "call sph_begin_steps first");
    // the graph's nodes less its event records (kStageCount + 1 of them)
    *kernels = sys->graphNodes - (kStageCount + 1);
    return SPH_OK;
}

// ---- utilities ---------------------------------------------------------------------------------

int sph_cell_order_key(const double *positions, int64_t n, int dimensions, double cell_width, const int64_t *shape,
                       int64_t *keys, int device)
{
    if (n < 0 || (n > 0 && (!positions || !keys)) || !shape) return fail(SPH_ERR_INVALID, "null argument");
    if (dimensions != 2 && dimensions != 3) return fail(SPH_ERR_INVALID, "dimensions must be 2 or 3");
    if (!(cell_width > 0.0)) return fail(SPH_ERR_INVALID, "the cell width must be positive");
    for (int a = 0; a < 3; ++a)
        if (shape[a] < 1) return fail(SPH_ERR_INVALID, "grid shape entries must be positive");
    if (n == 0) return SPH_OK;
    CUDA_TRY(cudaSetDevice(device));
    double *dx = nullptr;
    long long *dk = nullptr;
    CUDA_TRY(cudaMalloc((void **)&dx, sizeof(double) * n * dimensions));
    cudaError_t err = cudaMalloc((void **)&dk, sizeof(long long) * n);
    if (err != cudaSuccess) { cudaFree(dx); return fail(SPH_ERR_NOMEM, "cudaMalloc"); }
    cudaMemcpy(dx, positions, sizeof(double) * n * dimensions, cudaMemcpyHostToDevice);
    long long shp[3] = {shape[0], shape[1], shape[2]};
    launchCellOrderKey((int)n, dimensions, dx, cell_width, shp, dk, 0);
    err = cudaMemcpy(keys, dk, sizeof(long long) * n, cudaMemcpyDeviceToHost);
    cudaFree(dx);
    cudaFree(dk);
    if (err != cudaSuccess) return fail(SPH_ERR_CUDA, cudaGetErrorString(err));
    return SPH_OK;
}

int sph_neighbor_list(SphSystem *sys, double radius, int64_t *offsets, int32_t *neighbors, int64_t capacity,
                      int64_t *total)
{
    CHECK_SYS(sys);
    if (!offsets || !total) return fail(SPH_ERR_INVALID, "null argument");
    if (!(radius > 0.0) || radius > 2.0 * sys->h * (1.0 + 1e-12))
        return fail(SPH_ERR_INVALID, "the radius must be positive and within the cell list's support");
    int n = sys->n;
    offsets[0] = 0;
    *total = 0;
    if (n == 0) return SPH_OK;
    if (!sys->cellsFresh) sys->rebuild();
    Params P = sys->params();
    Frame F = sys->frame();
    long long *dCounts = (long long *)sys->stage(SphSystem::kOutSlot);
    launchNeighbourRows(P, F, nullptr, nullptr, dCounts, radius * radius, sys->stream);
    std::vector<long long> counts(n);
    CUDA_TRY(cudaMemcpyAsync(counts.data(), dCounts, sizeof(long long) * n, cudaMemcpyDeviceToHost, sys->stream));
    CUDA_TRY(cudaStreamSynchronize(sys->stream));
    for (int i = 0; i < n; ++i) offsets[i + 1] = offsets[i] + counts[i];
    *total = offsets[n];
    if (!neighbors || capacity < *total) return neighbors ? fail(SPH_ERR_CAPACITY, "neighbour array too small") : SPH_OK;
    int64_t *dOffsets = nullptr;
    int *dRows = nullptr;
    CUDA_TRY(cudaMalloc((void **)&dOffsets, sizeof(int64_t) * (n + 1)));
    cudaError_t err = cudaMalloc((void **)&dRows, sizeof(int) * std::max<int64_t>(*total, 1));
    if (err != cudaSuccess) { cudaFree(dOffsets); return fail(SPH_ERR_NOMEM, "cudaMalloc"); }
    cudaMemcpyAsync(dOffsets, offsets, sizeof(int64_t) * (n + 1), cudaMemcpyHostToDevice, sys->stream);
    launchNeighbourRows(P, F, dOffsets, dRows, nullptr, radius * radius, sys->stream);
    cudaMemcpyAsync(neighbors, dRows, sizeof(int) * *total, cudaMemcpyDeviceToHost, sys->stream);
    err = cudaStreamSynchronize(sys->stream);
    cudaFree(dOffsets);
    cudaFree(dRows);
    if (err != cudaSuccess) return fail(SPH_ERR_CUDA, cudaGetErrorString(err));
    return SPH_OK;
}

// ---- the breaking tracker's reads ---------------------------------------------------------------

// Scratch of at least `bytes` for the tracker's reads (grown as needed, kept with the handle).
static int surfaceScratch(SphSystem *sys, size_t bytes, void **out)
{
    if (bytes > sys->surfaceBytes) {
        cudaFree(sys->surface);
        sys->surface = nullptr;
        sys->surfaceBytes = 0;
        CUDA_TRY(cudaMalloc(&sys->surface, bytes));
        sys->surfaceBytes = bytes;
    }
    *out = sys->surface;
    return SPH_OK;
}

int sph_split_crest_zone(SphSystem *sys, double x0, double y0, double width, int64_t nx, int64_t ny,
                         double threshold, double min_mass, double reference_density, double length_ratio,
                         int64_t *split)
{
    CHECK_SYS(sys);
    if (!split || nx <= 0 || ny <= 0 || nx * ny > (1ll << 28) || !(width > 0.0))
        return fail(SPH_ERR_INVALID, "bad columns");
    if (!sys->resident) return fail(SPH_ERR_STATE, "no device state: call sph_push first");
    *split = 0;
    const int n = sys->n;
    if (n == 0) return SPH_OK;
    void *scratch = nullptr;
    TRY(surfaceScratch(sys, sizeof(unsigned long long) * (size_t)nx * (size_t)ny, &scratch));
    launchCrestZone(n, sys->master[sys->cur], sys->dim, x0, y0, width, nx, ny, (unsigned long long *)scratch,
                    threshold, min_mass, sys->dStageU8, sys->stream);
    CUDA_TRY(cudaGetLastError());
    // the zone in the caller's order, then the split as sph_split takes it
    std::vector<uint8_t> mask(n);
    CUDA_TRY(cudaMemcpyAsync(mask.data(), sys->dStageU8, n, cudaMemcpyDeviceToHost, sys->stream));
    CUDA_TRY(cudaStreamSynchronize(sys->stream));
    return sph_split(sys, mask.data(), reference_density, length_ratio, split);
}

// The reads of the fluid a tracker update takes (sph_surface.cu), over the whole fluid in 2D or a
// section's band across the tank in 3D; x along the tank, the vertical the last axis.
static int readBand(SphSystem *sys, bool section, double center, double half, Band *band, int *vertical)
{
    if (!sys->resident) return fail(SPH_ERR_STATE, "no device state: call sph_push first");
    if (!section && sys->dim != 2) return fail(SPH_ERR_UNSUPPORTED, "the whole-fluid surface reads are 2D");
    if (section && sys->dim != 3) return fail(SPH_ERR_UNSUPPORTED, "the section reads are 3D");
    if (section && !(half > 0.0)) return fail(SPH_ERR_INVALID, "a section's half width must be positive");
    *band = Band{section ? sys->master[sys->cur].x[1] : nullptr, center, half};
    *vertical = sys->dim - 1;
    return SPH_OK;
}

static int readTops(SphSystem *sys, bool section, double center, double half, double x0, double width, int64_t count,
             double *tops)
{
    CHECK_SYS(sys);
    if (!tops || count <= 0 || count > (1ll << 28) || !(width > 0.0)) return fail(SPH_ERR_INVALID, "bad columns");
    Band band;
    int vertical;
    TRY(readBand(sys, section, center, half, &band, &vertical));
    void *scratch = nullptr;
    TRY(surfaceScratch(sys, sizeof(double) * 2 * (size_t)count, &scratch));
    unsigned long long *bits = (unsigned long long *)scratch;
    double *values = (double *)scratch + count;
    launchSurfaceTops(sys->n, sys->master[sys->cur], vertical, band, x0, width, count, bits, values, sys->stream);
    CUDA_TRY(cudaGetLastError());
    TRY(sys->download(tops, values, sizeof(double) * count));
    CUDA_TRY(cudaStreamSynchronize(sys->stream));
    return SPH_OK;
}

static int readFaceCells(SphSystem *sys, bool section, double center, double halfBand, double low_x, double high_x,
                  double low_z, double half, double start, double base, double spacing, int64_t columns, int64_t bands,
                  uint8_t *marks)
{
    CHECK_SYS(sys);
    if (!marks || columns <= 0 || bands <= 0 || columns * bands > (1ll << 30) || !(spacing > 0.0))
        return fail(SPH_ERR_INVALID, "bad window");
    Band band;
    int vertical;
    TRY(readBand(sys, section, center, halfBand, &band, &vertical));
    const size_t bytes = (size_t)columns * (size_t)bands;
    void *scratch = nullptr;
    TRY(surfaceScratch(sys, bytes, &scratch));
    launchFaceCells(sys->n, sys->master[sys->cur], vertical, band, low_x, high_x, low_z, half, start, base, spacing,
                    columns, bands, (uint8_t *)scratch, sys->stream);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaMemcpyAsync(marks, scratch, bytes, cudaMemcpyDeviceToHost, sys->stream));
    CUDA_TRY(cudaStreamSynchronize(sys->stream));
    return SPH_OK;
}

static int readBedSheet(SphSystem *sys, bool section, double center, double half, const double *bed_x, const double *bed_z,
                 int64_t bed_count, double wet_height, double *xs, int64_t capacity, int64_t *count)
{
    CHECK_SYS(sys);
    if (!bed_x || !bed_z || !count || bed_count < 2 || bed_count > (1 << 24) || capacity < 0 || (capacity && !xs))
        return fail(SPH_ERR_INVALID, "bad bed or output");
    Band band;
    int vertical;
    TRY(readBand(sys, section, center, half, &band, &vertical));
    const int m = (int)bed_count, n = sys->n;
    void *scratch = nullptr;
    TRY(surfaceScratch(sys, sizeof(double) * (2 * (size_t)m + 1 + (size_t)n), &scratch));
    double *bx = (double *)scratch, *bz = bx + m;
    int *dCount = (int *)(bz + m);
    double *out = bz + m + 1;
    CUDA_TRY(cudaMemcpyAsync(bx, bed_x, sizeof(double) * m, cudaMemcpyHostToDevice, sys->stream));
    CUDA_TRY(cudaMemcpyAsync(bz, bed_z, sizeof(double) * m, cudaMemcpyHostToDevice, sys->stream));
    launchBedSheet(n, sys->master[sys->cur], vertical, band, bx, bz, m, wet_height, out, dCount, sys->stream);
    CUDA_TRY(cudaGetLastError());
    int found = 0;
    CUDA_TRY(cudaMemcpyAsync(&found, dCount, sizeof(int), cudaMemcpyDeviceToHost, sys->stream));
    CUDA_TRY(cudaStreamSynchronize(sys->stream));
    *count = found;
    const int64_t copy = std::min<int64_t>(found, capacity);
    if (copy > 0) {
        TRY(sys->download(xs, out, sizeof(double) * copy));
        CUDA_TRY(cudaStreamSynchronize(sys->stream));
    }
    return SPH_OK;
}

int sph_surface_tops(SphSystem *sys, double x0, double width, int64_t count, double *tops)
{
    return readTops(sys, false, 0.0, 0.0, x0, width, count, tops);
}

int sph_face_cells(SphSystem *sys, double low_x, double high_x, double low_z, double half, double start,
                   double base, double spacing, int64_t columns, int64_t bands, uint8_t *marks)
{
    return readFaceCells(sys, false, 0.0, 0.0, low_x, high_x, low_z, half, start, base, spacing, columns, bands, marks);
}

int sph_bed_sheet(SphSystem *sys, const double *bed_x, const double *bed_z, int64_t bed_count, double wet_height,
                  double *xs, int64_t capacity, int64_t *count)
{
    return readBedSheet(sys, false, 0.0, 0.0, bed_x, bed_z, bed_count, wet_height, xs, capacity, count);
}

int sph_section_tops(SphSystem *sys, double y, double half_width, double x0, double width, int64_t count, double *tops)
{
    return readTops(sys, true, y, half_width, x0, width, count, tops);
}

int sph_section_face_cells(SphSystem *sys, double y, double half_width, double low_x, double high_x, double low_z,
                           double half, double start, double base, double spacing, int64_t columns, int64_t bands,
                           uint8_t *marks)
{
    return readFaceCells(sys, true, y, half_width, low_x, high_x, low_z, half, start, base, spacing, columns, bands,
                         marks);
}

int sph_section_bed_sheet(SphSystem *sys, double y, double half_width, const double *bed_x, const double *bed_z,
                          int64_t bed_count, double wet_height, double *xs, int64_t capacity, int64_t *count)
{
    return readBedSheet(sys, true, y, half_width, bed_x, bed_z, bed_count, wet_height, xs, capacity, count);
}

int sph_split(SphSystem *sys, const uint8_t *mask, double reference_density, double length_ratio, int64_t *split)
{
    CHECK_SYS(sys);
    if (!mask || !split) return fail(SPH_ERR_INVALID, "null argument");
    if (!sys->resident) return fail(SPH_ERR_STATE, "no device state: call sph_push first");
    if (!(length_ratio > 0.0) || length_ratio > 1.0) return fail(SPH_ERR_INVALID, "the length ratio must be in (0, 1]");
    if (sys->shifting && length_ratio != 1.0)
        return fail(SPH_ERR_INVALID, "particle shifting needs one smoothing length for every particle");
    int n = sys->n, dim = sys->dim;
    *split = 0;
    if (n == 0) return SPH_OK;
    // which mothers split, and their ranks in the caller's order, from the caller's mask and the
    // device's fluid flags (read back in caller order)
    std::vector<uint8_t> flags(n);
    std::vector<int> orig(n);
    const MasterView &M0 = sys->master[sys->cur];
    CUDA_TRY(cudaMemcpyAsync(flags.data(), M0.fluid, n, cudaMemcpyDeviceToHost, sys->stream));
    CUDA_TRY(cudaMemcpyAsync(orig.data(), M0.orig, sizeof(int) * n, cudaMemcpyDeviceToHost, sys->stream));
    CUDA_TRY(cudaStreamSynchronize(sys->stream));
    std::vector<uint8_t> chosen(n, 0);
    for (int s = 0; s < n; ++s) chosen[orig[s]] = mask[orig[s]] && flags[s] ? 1 : 0;
    std::vector<int> rank(n);
    int count = 0;
    for (int o = 0; o < n; ++o) { rank[o] = count; count += chosen[o]; }
    if (count == 0) return SPH_OK;
    int perMother = (1 << dim) - 1;
    long long grown = (long long)n + (long long)count * perMother;
    if (grown > 0x3FFFFFFF) return fail(SPH_ERR_INVALID, "too many particles after the split");
    TRY(sys->reserve((int)grown, true));
    if (sys->budget && sys->energy)     // the daughters' totals start at zero; the mothers keep theirs
        CUDA_TRY(cudaMemset2DAsync(sys->energy + n, sizeof(double) * sys->energyCap, 0,
                                   sizeof(double) * (size_t)(grown - n), kEnergyTerms, sys->stream));
    const MasterView &M = sys->master[sys->cur];
    CUDA_TRY(cudaMemcpyAsync(sys->dStageU8, chosen.data(), n, cudaMemcpyHostToDevice, sys->stream));
    CUDA_TRY(cudaMemcpyAsync(sys->dRank, rank.data(), sizeof(int) * n, cudaMemcpyHostToDevice, sys->stream));
    launchSplit(n, dim, M, sys->dStageU8, sys->dRank, reference_density, length_ratio, n, sys->stream);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaStreamSynchronize(sys->stream));
    sys->n = (int)grown;
    sys->mixedH = true;
    sys->hMin = std::min(sys->hMin, sys->h * length_ratio);
    // hMin: the shortest length present, taken on the host from the master
    std::vector<double> lengths(sys->n);
    CUDA_TRY(cudaMemcpy(lengths.data(), M.h, sizeof(double) * sys->n, cudaMemcpyDeviceToHost));
    double hMin = lengths[0];
    bool mixed = false;
    for (double v : lengths) { hMin = std::min(hMin, v); if (v != sys->h) mixed = true; }
    sys->hMin = hMin;
    sys->mixedH = mixed;
    TRY(sys->takeLevels(lengths.data(), sys->n));
    sys->framed = false;
    sys->cellsFresh = false;    // the daughters have no cell yet: the next use sorts again
    sys->graphDirty = true;
    sys->listDirty = true;
    *split = count;
    return SPH_OK;
}

int sph_merge(SphSystem *sys, const uint8_t *mask, double reference_density, double reference_mass,
              double length_ratio, int64_t *groups, double *removed_energy, int64_t *source)
{
    CHECK_SYS(sys);
    if (!mask || !groups || !removed_energy) return fail(SPH_ERR_INVALID, "null argument");
    if (!sys->resident) return fail(SPH_ERR_STATE, "no device state: call sph_push first");
    if (!(reference_density > 0.0) || !(reference_mass > 0.0) || !(length_ratio > 0.0) || length_ratio > 1.0)
        return fail(SPH_ERR_INVALID, "the reference density and mass must be positive, the length ratio in (0, 1]");
    if (sys->shifting) return fail(SPH_ERR_INVALID, "particle shifting takes one smoothing length throughout");
    *groups = 0;
    *removed_energy = 0.0;
    const int n = sys->n;
    if (n == 0) return SPH_OK;
    if (!sys->framed) sys->rebuild();       // the frame's pressures in the master's order
    TRY(sys->upload(sys->dStageU8, mask, n));
    long long *dSource = nullptr;
    TRY(deviceAlloc(&dSource, n));
    MergeArgs in{};
    in.n = n;
    in.dim = sys->dim;
    in.master = sys->master[sys->cur];
    in.next = sys->master[1 - sys->cur];
    in.nextFrame = sys->frame();
    for (int a = 0; a < 3; ++a) { in.nextFrame.x[a] = in.next.x[a]; in.nextFrame.v[a] = in.next.v[a]; }
    in.nextFrame.rho = in.next.rho; in.nextFrame.m = in.next.m; in.nextFrame.h = in.next.h;
    in.nextFrame.fluid = in.next.fluid; in.nextFrame.orig = in.next.orig;
    in.params = sys->params();
    in.acc = sys->acc;
    in.pres = sys->pres;
    in.energy = sys->budget && sys->energy ? sys->energy : nullptr;
    in.energyStride = sys->energyCap;
    in.energyTerms = kEnergyTerms;
    in.mask = sys->dStageU8;
    in.referenceDensity = reference_density;
    in.referenceMass = reference_mass;
    in.lengthRatio = length_ratio;
    in.source = dSource;
    in.stream = sys->stream;
    MergeResultDevice out{};
    const int status = runMerge(in, out);
    if (status != 0) {
        cudaFree(dSource);
        return fail(SPH_ERR_CUDA, std::string("merge: ") + (out.error ? out.error : "failed"));
    }
    if (out.groups > 0) {
        sys->cur = 1 - sys->cur;
        sys->n = out.newCount;
        sys->framed = true;
        sys->cellsFresh = false;
        sys->listDirty = true;
        sys->graphDirty = true;
        std::vector<double> lengths(sys->n);
        CUDA_TRY(cudaMemcpy(lengths.data(), sys->master[sys->cur].h, sizeof(double) * sys->n, cudaMemcpyDeviceToHost));
        double hMin = lengths.empty() ? sys->h : lengths[0];
        bool mixed = false;
        for (double v : lengths) { hMin = std::min(hMin, v); if (v != sys->h) mixed = true; }
        sys->hMin = hMin;
        sys->mixedH = mixed;
        TRY(sys->takeLevels(lengths.data(), sys->n));
        if (source) {
            std::vector<long long> from(sys->n);
            CUDA_TRY(cudaMemcpy(from.data(), dSource, sizeof(long long) * sys->n, cudaMemcpyDeviceToHost));
            for (int k = 0; k < sys->n; ++k) source[k] = from[k];
        }
    } else if (source) {
        for (int k = 0; k < n; ++k) source[k] = k;
    }
    cudaFree(dSource);
    *groups = out.groups;
    *removed_energy = out.removedEnergy;
    return SPH_OK;
}

}  // extern "C"
