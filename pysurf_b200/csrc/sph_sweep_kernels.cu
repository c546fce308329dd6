// sph_sweep_kernels.cu -- the neighbour sweeps of the delta-SPH step.
//
//   list  the step's neighbour table, from one walk over the cells
//   S     Shepard filter (src/pysurf/sphGpu.py:768-802, 1040-1056)
//   A     wall pressure: boundary rows over fluid neighbours (src/pysurf/sphSolver.py:1045-1106;
//         src/pysurf/sphGpu.py:804-854)
//   B     gradients: fluid rows, velocity gradient G (src/pysurf/sphSolver.py:1151-1190), correction L
//         (656-689) and renormalized density gradient (691-716), from one pass over the neighbours
//   C     momentum: fluid rows (src/pysurf/sphSolver.py:1122-1149, 1192-1230, 1328-1356;
//         src/pysurf/sphGpu.py:303-414), with the fluid maxima (1072-1082) and the time step
//         (src/pysurf/sphSolver.py:1410-1424) in the epilogue
//   D     continuity (src/pysurf/sphSolver.py:623-654, 718-822; src/pysurf/sphGpu.py:430-545), with
//         the density update (1111-1140), and, when XSPH is off, the drift and the enforcement
//   X     XSPH (src/pysurf/sphSolver.py:1358-1377; src/pysurf/sphGpu.py:725-766), then drift and
//         enforcement
//
// Each sweep is templated on the dimension D, the kernel K (0 cubic spline, 1 Wendland C2) and
// the threads per particle T.  Sums are float32 in a fixed order, no atomics on them.
#include <climits>
#include <math.h>

#include "sph_enforce.cuh"
#include "sph_kernels.h"
#include "sph_sweeps.cuh"

namespace sph {

// Blocks an SM the energy budget's momentum and continuity sweeps are built for: their extra
// accumulators need about 100 registers a thread in 2D (5 blocks of 128 threads leave 102).
template <int D>
constexpr int budgetMinBlocks() { return D == 2 ? 5 : 4; }
// The gradients and continuity sweeps carry float64 sums beside their float32 ones (M; the wall pairs'
// terms), so they take more registers a thread and fewer resident blocks.  Continuity also keeps the
// next neighbour's five rows in flight: at 4 blocks in 3D (128 registers, none spilled) it runs 16-25%
// faster than at 5 (96, spilling) on the ridges, and at 5 in 2D (102) 3.5% faster than at 6 on the
// beach (measured).
#ifndef SPH_PRECISE_MIN_BLOCKS
#define SPH_PRECISE_MIN_BLOCKS 5
#endif
#ifndef SPH_PRECISE_MIN_BLOCKS_3D
#define SPH_PRECISE_MIN_BLOCKS_3D 4
#endif
template <int D>
constexpr int preciseMinBlocks() { return D == 2 ? SPH_PRECISE_MIN_BLOCKS : SPH_PRECISE_MIN_BLOCKS_3D; }
// The 3D gradients sweep keeps three 3 x 3 float32 sums and the float64 M: at 4 blocks (128
// registers) it ran 7-17% faster than at 5 on the ridges; in 2D 6 blocks (80 registers) ran 3%
// faster than 5 on the beach (measured).
#ifndef SPH_GRADIENT_MIN_BLOCKS
#define SPH_GRADIENT_MIN_BLOCKS 6
#endif
#ifndef SPH_GRADIENT_MIN_BLOCKS_3D
#define SPH_GRADIENT_MIN_BLOCKS_3D 4
#endif
template <int D>
constexpr int gradientMinBlocks() { return D == 2 ? SPH_GRADIENT_MIN_BLOCKS : SPH_GRADIENT_MIN_BLOCKS_3D; }

// ------------------------------------------------------------------------------------------
// The neighbour table
// ------------------------------------------------------------------------------------------

#ifndef SPH_LIST_TRIM
#define SPH_LIST_TRIM 1
#endif

// Each slot's neighbours in the walk's order (forEachNeighbour's, with its tests), from a group of
// L lanes: lane t tests candidates t, t + L, ... of each run of the stencil, and the group's ballot
// places the accepted ones in order.  The count is the whole count even when the row is full (the
// sweeps then walk the cells for that slot).  maxCount: the largest count, when given.
//
// A stencil row is trimmed to the cells within the search's reach of the particle, taken in cell
// units from the particle's place in its cell (a particle outside the grid, whose cell is clamped,
// searches its whole stencil).  The reach carries slack over the coarse test's bound, so every
// candidate the coarse test passes stays: the accepted neighbours and their order are those of the
// whole stencil.  PRECISE: separations from point and remainder; MIXED: smoothing lengths differ.
template <int D, int L, bool PRECISE, bool MIXED>
__global__ void __launch_bounds__(kBlock) listKernel(Params P, Frame F, const Control *ctl, int *maxCount)
{
    if (ctl && !ctl->active) return;
    const Group<L> G = groupOf<L>();
    const int i = G.i;
    if (i >= P.n) return;           // a group's lanes share i, so groups leave whole
    const int t = G.t;
    const int shift = (threadIdx.x & 31) & ~(L - 1);
    const unsigned lower = (1u << t) - 1u;
    const float4 Ai = __ldg(&F.pa[i]), Bi = __ldg(&F.pb[i]);
    const float hI = fabsf(signedLengthIn<D>(Ai, Bi));
    // a boundary row holds its fluid neighbours only (forEachNeighbour says why)
    const bool fluidOnly = signedLengthIn<D>(Ai, Bi) <= 0.0f;
    float pi[3], li[3];
    pointIn<D>(Ai, pi);
    remainderIn<D>(Ai, Bi, li);
    const float reach = MIXED ? hI + P.hMax : 2.0f * P.hMax;
    const float limit = kCandidateMargin * reach * reach;
    const float support = MIXED ? 0.0f : support2(P.hMax);
    const float sure = PRECISE ? sureBound(P, support, hI, pi) : 0.0f;
    double shift64 = 0.0;
    bool seam = false;
    if (D == 3 && P.period > 0.0 && (pi[1] < reach || pi[1] > P.periodF - reach)) {
        seam = true;
        shift64 = pi[1] < 0.5f * P.periodF ? P.period : -P.period;
    }
    const int ownCell = F.cell[i];
    const float fineReach = hI + P.fineMax, fineLimit = kCandidateMargin * fineReach * fineReach;
    int *column = F.nbr + 4 * (size_t)i;
    int count = 0;
    // search s: grid level s >> 1 (coarse, fine), origin s & 1 (the particle, its periodic image)
    for (int search = 0; search < (MIXED ? 4 : 2); ++search) {
        const int level = MIXED ? search >> 1 : 0, image = search & 1;
        if (level >= P.levels || (image && !seam)) continue;
        const double pos[3] = {(double)pi[0] + (double)li[0], (double)pi[1] + (double)li[1] + (image ? shift64 : 0.0),
                               D == 3 ? (double)pi[2] + (double)li[2] : 0.0};
        const CellBox box = cellBox(P, level, ownCell, pos, image != 0, D, searchCells(P, level, hI), !MIXED);
        const float searchLimit = level ? fineLimit : limit;
        const double width = level ? P.fineWidth : P.cellWidth;
        const double *origin = level ? P.fineOrigin : P.origin;
        // the particle's place in the centre cell, in cell widths, and the reach in cell widths with slack
        const float invW = (float)(1.0 / width);
        const float fx = (float)(((double)pi[0] - origin[0]) / width) - (float)box.cx;
        const float fz = D == 3 ? (float)(((double)pi[2] - origin[2]) / width) - (float)box.cz : 0.5f;
        const float R = (1.001f * sqrtf(searchLimit) + 5.0e-7f * (fabsf(pi[0]) + fabsf(pi[1]) + fabsf(pi[2]))) * invW +
                        1.0e-3f;
        const float offset = image ? (float)shift64 : 0.0f;
        const float fy = (float)(((double)pi[1] + (image ? shift64 : 0.0) - origin[1]) / width) - (float)box.cy;
        const bool trim = SPH_LIST_TRIM && fx >= 0.0f && fx < 1.0f && fy >= 0.0f && fy < 1.0f && fz >= 0.0f &&
                          fz < 1.0f;
        for (int zz = box.z0; zz <= box.z1; ++zz) {
            const int oz = zz - box.cz;
            const float dz = oz > 0 ? (float)oz - fz : (oz < 0 ? fz - (float)(oz + 1) : 0.0f);
            for (int yy = box.y0; yy <= box.y1; ++yy) {
                int xa = box.x0, xb = box.x1;
                if (trim) {
                    const int oy = yy - box.cy;
                    const float dy = oy > 0 ? (float)oy - fy : (oy < 0 ? fy - (float)(oy + 1) : 0.0f);
                    const float rem = R * R - dy * dy - dz * dz;
                    if (rem < 0.0f) continue;
                    const float ext = sqrtf(rem);
                    xa = max(box.x0, box.cx + (int)floorf(fx - ext));
                    xb = min(box.x1, box.cx + (int)floorf(fx + ext));
                }
                const int row = box.first + (zz * box.ny + yy) * box.nx;
                const int first = __ldg(&F.cellStart[row + xa]), end = __ldg(&F.cellStart[row + xb + 1]);
                for (int base = first; base < end; base += L) {
                    const int j = base + t;
                    bool accepted = false;
                    if (j < end && j != i) {
                        const float4 A = __ldg(&F.pa[j]);
                        float pj[3];
                        pointIn<D>(A, pj);
                        const bool inRow = !fluidOnly || (D == 3 ? A.w > 0.0f : __ldg(&F.fluid[j]) != 0);
                        const float coarse = inRow ? coarseDistance2<D>(pi, pj, offset) : searchLimit;
                        if (PRECISE && !image && level == 0 && coarse < sure) {
                            accepted = true;
                        } else if (coarse < searchLimit) {
                            const float4 B = (D == 3 && PRECISE) || MIXED ? __ldg(&F.pb[j]) : A;
                            float r2 = coarse;      // the float32 points' separation is the coarse one
                            if (PRECISE) {
                                float lj[3], d[3];
                                remainderIn<D>(A, B, lj);
                                r2 = separation2<D, 1>(P, pi, li, pj, lj, offset, image, shift64, d);
                            }
                            const float bound = MIXED ? support2(0.5f * (hI + fabsf(signedLengthIn<D>(A, B)))) : support;
                            accepted = r2 < bound;
                        }
                    }
                    const unsigned bits = (__ballot_sync(G.mask, accepted) >> shift) & ((L >= 32 ? 0u : 1u << L) - 1u);
                    if (accepted) {
                        const int k = count + __popc(bits & lower);
                        if (k < P.listCap)
                            column[((size_t)(k >> 2) * P.listStride) * 4 + (k & 3)] = image ? (j | (int)0x80000000) : j;
                    }
                    count += __popc(bits);
                }
            }
        }
    }
    if (t != 0) return;
    F.ncount[i] = count;
    if (maxCount) atomicMax(maxCount, count);
}

// The same table from a warp that takes a batch of up to kBatch particles of one cell together
// (the 3D table; launchList says why):
// every particle of a cell has the same stencil, so each candidate is loaded once and tested against
// the whole batch, one ballot a particle placing the accepted ones in that particle's order.  Each
// particle accepts only the candidates of its own trimmed run of each row, exactly as listKernel
// (and the sweeps' walk) would offer them, so its row holds the same entries in the same order;
// the union of the batch's runs only decides which candidates the warp loads.
//
// A warp owns the batches that start in its kBatch slots: a batch starts at a cell's first slot and
// every kBatch slots after it, so each slot belongs to one batch.
#ifndef SPH_LIST_BATCH
#define SPH_LIST_BATCH 8
#endif
constexpr int kBatch = SPH_LIST_BATCH;

// A batch member as the warp's lanes read it, in 16-byte rows so that each read is one shared load:
// the run and flags decide whether the member takes a chunk at all, the point its coarse test, the
// remainder only the few candidates near the edge of its support.  The set-up lane writes the
// search's bounds into point.w and rest.w as each search starts.
constexpr int kMemberSeam = 1;          // the member searches its periodic image too
constexpr int kMemberFluidOnly = 2;     // a boundary member: its row holds fluid neighbours only
struct alignas(16) BatchMember {
    float4 point;       // the float32 point; w: this search's sure bound (0 where none applies)
    float4 rest;        // the remainder; w: this search's coarse limit
    int4 run;           // this row's run of candidates [x, y), the member's slot, its flags
    float4 bounds;      // the limit on the coarse grid, on the fine grid, the sure bound, hI
    double shift64;     // the periodic image's shift (0 when it is not searched)
    float offset;       // the shift as float32
    float unused;
};

// No blocks-a-multiprocessor bound: at the compiler's default the kernel keeps about 24 warps an
// SM with a few spills, faster than 85-116 registers and no spills at 3 to 6 blocks, or 64
// registers at 8 (measured).
template <int D, bool PRECISE, bool MIXED>
__global__ void __launch_bounds__(kBlock) cellListKernel(Params P, Frame F, const Control *ctl, int *maxCount)
{
    if (ctl && !ctl->active) return;
    __shared__ BatchMember members[kBlock / 32][kBatch];
    const int lane = threadIdx.x & 31;
    const int warp = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    BatchMember *mine = members[threadIdx.x >> 5];
    const int first = warp * kBatch;
    if (first >= P.n) return;               // whole warps leave together
    const int last = min(first + kBatch, P.n);
    const unsigned lower = (1u << lane) - 1u;
    const float support = MIXED ? 0.0f : support2(P.hMax);
    // the batches that start in this warp's slots
    bool starts = false;
    if (lane < kBatch && first + lane < last) {
        const int s = first + lane;
        starts = (s - __ldg(&F.cellStart[F.cell[s]])) % kBatch == 0;
    }
    unsigned pending = __ballot_sync(0xFFFFFFFFu, starts);
    while (pending) {
        const int b0 = first + __ffs(pending) - 1;
        pending &= pending - 1;
        const int ownCell = F.cell[b0];
        const int count = min(kBatch, __ldg(&F.cellStart[ownCell + 1]) - b0);
        // lane p < count sets up member p
        float hIp = 0.0f, pip[3] = {0, 0, 0}, lip[3] = {0, 0, 0};
        double shiftp = 0.0;
        bool seamp = false;
        if (lane < count) {
            const int i = b0 + lane;
            const float4 Ai = __ldg(&F.pa[i]), Bi = __ldg(&F.pb[i]);
            hIp = fabsf(signedLengthIn<D>(Ai, Bi));
            pointIn<D>(Ai, pip);
            remainderIn<D>(Ai, Bi, lip);
            const float reach = MIXED ? hIp + P.hMax : 2.0f * P.hMax;
            if (D == 3 && P.period > 0.0 && (pip[1] < reach || pip[1] > P.periodF - reach)) {
                seamp = true;
                shiftp = pip[1] < 0.5f * P.periodF ? P.period : -P.period;
            }
            const float fineReach = hIp + P.fineMax;
            BatchMember &m = mine[lane];
            m.point = make_float4(pip[0], pip[1], pip[2], 0.0f);
            m.rest = make_float4(lip[0], lip[1], lip[2], 0.0f);
            m.run = make_int4(0, 0, i, (seamp ? kMemberSeam : 0) |
                                           (signedLengthIn<D>(Ai, Bi) <= 0.0f ? kMemberFluidOnly : 0));
            m.bounds = make_float4(kCandidateMargin * reach * reach, kCandidateMargin * fineReach * fineReach,
                                   PRECISE ? sureBound(P, support, hIp, pip) : 0.0f, hIp);
            m.shift64 = shiftp;
            m.offset = (float)shiftp;
        }
        const bool anySeam = __any_sync(0xFFFFFFFFu, seamp);
        int counted[kBatch];
#pragma unroll
        for (int p = 0; p < kBatch; ++p) counted[p] = 0;
        // search s: grid level s >> 1 (coarse, fine), origin s & 1 (the particle, its periodic image)
        for (int search = 0; search < (MIXED ? 4 : 2); ++search) {
            const int level = MIXED ? search >> 1 : 0, image = search & 1;
            if (level >= P.levels || (image && !anySeam)) continue;
            // lane p: this search's bounds for the others, its own box, its place in the centre cell,
            // and its reach in cell widths
            const bool takes = lane < count && (!image || seamp);
            CellBox box{};
            float fx = 0.0f, fy = 0.0f, fz = 0.0f, R = 0.0f;
            bool trim = false;
            if (lane < count) {
                const float4 bounds = mine[lane].bounds;
                const float lim = level ? bounds.y : bounds.x;
                mine[lane].point.w = PRECISE && !image && level == 0 ? bounds.z : 0.0f;
                mine[lane].rest.w = lim;
                if (takes) {
                    const double pos[3] = {(double)pip[0] + (double)lip[0],
                                           (double)pip[1] + (double)lip[1] + (image ? shiftp : 0.0),
                                           D == 3 ? (double)pip[2] + (double)lip[2] : 0.0};
                    box = cellBox(P, level, ownCell, pos, image != 0, D, searchCells(P, level, hIp), !MIXED);
                    const double width = level ? P.fineWidth : P.cellWidth;
                    const double *origin = level ? P.fineOrigin : P.origin;
                    const float invW = (float)(1.0 / width);
                    fx = (float)(((double)pip[0] - origin[0]) / width) - (float)box.cx;
                    fz = D == 3 ? (float)(((double)pip[2] - origin[2]) / width) - (float)box.cz : 0.5f;
                    fy = (float)(((double)pip[1] + (image ? shiftp : 0.0) - origin[1]) / width) - (float)box.cy;
                    R = (1.001f * sqrtf(lim) + 5.0e-7f * (fabsf(pip[0]) + fabsf(pip[1]) + fabsf(pip[2]))) * invW +
                        1.0e-3f;
                    trim = SPH_LIST_TRIM && fx >= 0.0f && fx < 1.0f && fy >= 0.0f && fy < 1.0f && fz >= 0.0f &&
                           fz < 1.0f;
                }
            }
            // the grid's shape (the same for every member) and the union of the members' rows
            const int gridFirst = level ? P.fineFirst : 0;
            const int nx = level ? P.fineNc[0] : P.nc[0], ny = level ? P.fineNc[1] : P.nc[1];
            const int zLo = __reduce_min_sync(0xFFFFFFFFu, takes ? box.z0 : INT_MAX);
            const int zHi = __reduce_max_sync(0xFFFFFFFFu, takes ? box.z1 : INT_MIN);
            const int yLo = __reduce_min_sync(0xFFFFFFFFu, takes ? box.y0 : INT_MAX);
            const int yHi = __reduce_max_sync(0xFFFFFFFFu, takes ? box.y1 : INT_MIN);
            for (int zz = zLo; zz <= zHi; ++zz) {
                for (int yy = yLo; yy <= yHi; ++yy) {
                    const int row = gridFirst + (zz * ny + yy) * nx;
                    // lane p: its run of this row, trimmed to its reach
                    int a = 0, b = 0;
                    if (takes && zz >= box.z0 && zz <= box.z1 && yy >= box.y0 && yy <= box.y1) {
                        int xa = box.x0, xb = box.x1;
                        bool empty = false;
                        if (trim) {
                            const int oz = zz - box.cz, oy = yy - box.cy;
                            const float dz = oz > 0 ? (float)oz - fz : (oz < 0 ? fz - (float)(oz + 1) : 0.0f);
                            const float dy = oy > 0 ? (float)oy - fy : (oy < 0 ? fy - (float)(oy + 1) : 0.0f);
                            const float rem = R * R - dy * dy - dz * dz;
                            if (rem < 0.0f) {
                                empty = true;
                            } else {
                                const float ext = sqrtf(rem);
                                xa = max(box.x0, box.cx + (int)floorf(fx - ext));
                                xb = min(box.x1, box.cx + (int)floorf(fx + ext));
                            }
                        }
                        if (!empty) {
                            a = __ldg(&F.cellStart[row + xa]);
                            b = __ldg(&F.cellStart[row + xb + 1]);
                        }
                    }
                    if (lane < count) { mine[lane].run.x = a; mine[lane].run.y = b; }
                    const int uA = __reduce_min_sync(0xFFFFFFFFu, a < b ? a : INT_MAX);
                    const int uB = __reduce_max_sync(0xFFFFFFFFu, a < b ? b : INT_MIN);
                    __syncwarp();
                    for (int base = uA; base < uB; base += 32) {
                        const int j = base + lane;
                        const bool valid = j < uB;
                        float4 A = make_float4(0, 0, 0, 0), B = A;
                        float pj[3] = {0, 0, 0}, lj[3] = {0, 0, 0}, hJ = 0.0f;
                        bool fluidJ = false;
                        if (valid) {
                            A = __ldg(&F.pa[j]);
                            pointIn<D>(A, pj);
                            // the remainders with the point, although a candidate under `sure` needs
                            // none: loading them only for the precise test slowed the 3D table by 11%
                            if ((D == 3 && PRECISE) || MIXED) B = __ldg(&F.pb[j]);
                            if (PRECISE) remainderIn<D>(A, D == 3 ? B : A, lj);
                            if (MIXED) hJ = fabsf(signedLengthIn<D>(A, B));
                            fluidJ = D == 3 ? A.w > 0.0f : __ldg(&F.fluid[j]) != 0;
                        }
#pragma unroll
                        for (int p = 0; p < kBatch; ++p) {
                            if (p >= count) continue;      // count is the warp's: the loop keeps its trip count
                            const int4 run = mine[p].run;
                            if (run.x >= run.y || run.y <= base || run.x >= base + 32) continue;   // the whole warp
                            if (image && !(run.w & kMemberSeam)) continue;
                            bool accepted = false;
                            if (valid && j >= run.x && j < run.y && j != run.z &&
                                (fluidJ || !(run.w & kMemberFluidOnly))) {
                                const float4 point = mine[p].point;
                                const float mp[3] = {point.x, point.y, point.z};
                                const float offset = image ? mine[p].offset : 0.0f;
                                const float coarse = coarseDistance2<D>(mp, pj, offset);
                                if (PRECISE && coarse < point.w) {
                                    accepted = true;
                                } else {
                                    const float4 rest = mine[p].rest;
                                    if (coarse < rest.w) {
                                        float r2 = coarse;
                                        if (PRECISE) {
                                            const float ml[3] = {rest.x, rest.y, rest.z};
                                            float d[3];
                                            r2 = separation2<D, 1>(P, mp, ml, pj, lj, offset, image,
                                                                   image ? mine[p].shift64 : 0.0, d);
                                        }
                                        const float bound =
                                            MIXED ? support2(0.5f * (mine[p].bounds.w + hJ)) : support;
                                        accepted = r2 < bound;
                                    }
                                }
                            }
                            const unsigned bits = __ballot_sync(0xFFFFFFFFu, accepted);
                            if (accepted) {
                                const int k = counted[p] + __popc(bits & lower);
                                if (k < P.listCap) {
                                    int *column = F.nbr + 4 * (size_t)run.z;
                                    column[((size_t)(k >> 2) * P.listStride) * 4 + (k & 3)] =
                                        image ? (j | (int)0x80000000) : j;
                                }
                            }
                            counted[p] += __popc(bits);
                        }
                    }
                    __syncwarp();
                }
            }
        }
        int own = 0;
#pragma unroll
        for (int p = 0; p < kBatch; ++p)
            if (lane == p) own = counted[p];
        if (lane < count) {
            F.ncount[b0 + lane] = own;
            if (maxCount) atomicMax(maxCount, own);
        }
        __syncwarp();
    }
}

// ------------------------------------------------------------------------------------------
// Sweep S: the Shepard filter
// ------------------------------------------------------------------------------------------

__device__ __forceinline__ bool filterDue(const Control *ctl)
{
    if (!ctl) return true;
    if (!ctl->active) return false;
    if (ctl->filterInterval > 0) return ctl->step > 0 && ctl->step % ctl->filterInterval == 0;
    return ctl->filterNow != 0;
}

template <int D, int K>
struct ShepardVisit {
    static constexpr bool kSkipCoincident = false;
    static constexpr bool kKinetic = false;
    static constexpr bool kBoundaryRows = true;
    static constexpr bool kWholeBoundaryRows = true;    // the host-step call returns boundary rows too
    const Frame &F;
    Smoothing<K, D> S;
    float num, den;
    __device__ bool accept(bool) const { return true; }
    __device__ void operator()(int j, const float *, float r, float h, bool, int, const float4 &B, const float4 &)
    {
        const KernelAt k = S.at(h);
        const float4 X = auxRow<D>(F, j);
        float w = kernelValue<K>(r * k.invH, k);
        num += massIn<D>(B) * w;
        den += volumeIn<D>(B, X) * w;
    }
};

template <int D, int K, int T, bool FINE>
__global__ void __launch_bounds__(kBlock, sweepMinBlocks<D>()) shepardKernel(Params P, Frame F, const Control *ctl)
{
    if (!filterDue(ctl)) return;
    const Group<T> G = groupOf<T>();
    const int i = G.i;
    if (i >= P.n) return;
    const float hs = signedLength<D>(F, i);
    // a device step filters the fluid alone; the host-step call (no control block) returns every row
    if (ctl && hs <= 0.0f) return;
    float hI = fabsf(hs);
    // the particle itself first, as the reference's sums start (src/pysurf/sphGpu.py:781-783)
    float own = sigmaAt(P.sigmaUnit, hI, D);
    float mi = massOf<D>(F, i);
    ShepardVisit<D, K> visit{F, Smoothing<K, D>(P), G.t == 0 ? mi * own : 0.0f,
                             G.t == 0 ? volumeOf<D>(F, i) * own : 0.0f};
    forEachNeighbour<D, T, FINE>(P, F, i, G.t, hI, visit);
    float num = groupSum<T>(visit.num, G.mask), den = groupSum<T>(visit.den, G.mask);
    if (G.t != 0) return;
    F.scalar[i] = num / den;
}

// The fluid takes its filtered density (float64 from the float32 filter, as the reference
// stores it), its deviation and its pressure; the boundary keeps its own.
template <int D>
__global__ void applyShepardKernel(Params P, Frame F, const Control *ctl)
{
    if (!filterDue(ctl)) return;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.n || !F.fluid[i]) return;
    float filtered = F.scalar[i];
    double rho = (double)filtered;
    // the filter's change of elastic energy (src/pysurf/sphGpu.py:1043-1056)
    if (P.budget) addEnergy(P, F, i, kFilter, F.m[i] * (elasticEnergy(P, rho) - elasticEnergy(P, F.rho[i])));
    F.rho[i] = rho;
    storeDensity<D>(F, i, massOf<D>(F, i), rho, P.devReference, (float)taitPressure(P, rho, true));
}

// ------------------------------------------------------------------------------------------
// Sweep A: extrapolated wall pressure
// ------------------------------------------------------------------------------------------

template <int D, int K, bool HOLD = false>
struct WallVisit {
    static constexpr bool kSkipCoincident = false;
    static constexpr bool kKinetic = true;
    static constexpr bool kBoundaryRows = true;         // it runs boundary rows only
    const Params &P; const Frame &F;
    Smoothing<K, D, HOLD> S;
    float weight, total;
    __device__ bool accept(bool fluidJ) const { return fluidJ; }
    __device__ void operator()(int j, const float *d, float r, float h, bool, int, const float4 &, const float4 &Kj)
    {
        const KernelAt k = S.at(h);
        float w = kernelValue<K>(r * k.invH, k);
        float gd = P.g[0] * d[0] + P.g[1] * d[1] + (D == 3 ? P.g[2] * d[2] : 0.0f);
        weight += w;
        total += w * (pressureOf<D>(F, j) + densityIn<D>(Kj) * gd);
    }
};

// Boundary rows only write their own entries and only fluid entries are read, so the frame is
// updated in place.  writeDensity: the master float64 density takes Tait^-1(p_w) too.
template <int D, int K, int T, bool FINE>
__global__ void __launch_bounds__(kBlock, sweepMinBlocks<D>())
wallPressureKernel(Params P, Frame F, const Control *ctl, int writeDensity)
{
    if (ctl && !ctl->active) return;
    const Group<T> G = groupOf<T>();
    const int i = G.i;
    if (i >= P.n) return;
    float hs = signedLength<D>(F, i);
    if (hs > 0.0f) return;
    WallVisit<D, K, FINE> visit{P, F, Smoothing<K, D, FINE>(P, -hs), 0.0f, 0.0f};
    forEachNeighbour<D, T, FINE>(P, F, i, G.t, -hs, visit);
    float weight = groupSum<T>(visit.weight, G.mask), total = groupSum<T>(visit.total, G.mask);
    if (G.t != 0) return;
    float p = 0.0f;
    if (weight > 0.0f) p = fmaxf(total / weight, 0.0f);
    F.scalar[i] = p;
    if (writeDensity) {
        double rho = P.rho0 * pow(1.0 + (double)p / P.stiffness, 1.0 / 7.0);
        storeDensity<D>(F, i, massOf<D>(F, i), rho, P.devReference, p);
        F.rho[i] = rho;
        return;
    }
    // the density stays; the pressure and p / rho^2 take p_w
    const float rho = densityOf<D>(F, i), ratio = p / (rho * rho);
    F.pres[i] = p;
    if (D == 2) F.kin[i].w = ratio;
    else F.aux[i].x = ratio;
}

// ------------------------------------------------------------------------------------------
// Sweep B: G, L and grad rho from one pass
// ------------------------------------------------------------------------------------------

// M (for L) is summed in float64 from float64 kernel gradients: L multiplies continuity's cancelling
// terms (a wall's velocity jump), where an L off by float32's summation error would move the rate by
// more than 1e-5 of its largest value against the float64 sums.  Its upper triangle, packed.
template <int D>
__device__ __forceinline__ constexpr int packed(int a, int b) { return a * D - a * (a - 1) / 2 + (b - a); }

template <int D, int K, bool HOLD = false>
struct GradientVisit {
    static constexpr bool kSkipCoincident = true;
    static constexpr bool kPipelined = true;
    static constexpr bool kAuxRow = D == 3;
    static constexpr bool kKinetic = true;
    const Frame &F;
    Smoothing<K, D, HOLD> kernel;
    bool wantG, wantL, wantRho;
    float vi[3], devI;
    float S[3][3], Mf[D * (D + 1) / 2], gsum[3];     // Mf: its upper triangle, packed
    float4 rowX;
    double M[D * (D + 1) / 2];
    __device__ bool accept(bool) const { return true; }
    __device__ void operator()(int j, const float *d, float r, float h, bool fluidJ, int, const float4 &B,
                               const float4 &Kj)
    {
        const KernelAt k = kernel.at(h);
        const float4 X = D == 3 ? rowX : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        if (wantL) {
            double dd[3] = {(double)d[0], (double)d[1], (double)d[2]}, r2 = 0.0;
            for (int a = 0; a < D; ++a) r2 = fma(dd[a], dd[a], r2);
            const double rf = (double)r, rr = fma(fma(-rf, rf, r2), 0.5 / rf, rf);
            const double w64 = (double)volumeIn<D>(B, X) * kernelGradient64<K>(rr, k);
            for (int a = 0; a < D; ++a) {
                const double wa = -w64 * dd[a];
                for (int b = a; b < D; ++b) M[packed<D>(a, b)] = fma(wa, dd[b], M[packed<D>(a, b)]);
            }
        }
        float w = volumeIn<D>(B, X) * kernelGradient<K>(r * k.invH, k);
        if (wantG && fluidJ) {
            float vj[3];
            velocityIn<D>(Kj, vj);
            for (int a = 0; a < D; ++a) {
                for (int b = 0; b < D; ++b) S[a][b] += w * (vj[a] - vi[a]) * d[b];
                const float wa = -w * d[a];
                for (int b = a; b < D; ++b) Mf[packed<D>(a, b)] += wa * d[b];
            }
        }
        if (wantRho) {
            float t = w * (deviationIn<D>(B, X) - devI);
            for (int a = 0; a < D; ++a) gsum[a] += t * d[a];
        }
    }
};

template <int D, int T>
__device__ __forceinline__ void groupSumMatrix(float M[3][3], unsigned mask)
{
    for (int a = 0; a < D; ++a)
        for (int b = 0; b < D; ++b) M[a][b] = groupSum<T>(M[a][b], mask);
}

template <int D, int K, int T, bool FINE>
__global__ void __launch_bounds__(kBlock, gradientMinBlocks<D>())
gradientKernel(Params P, Frame F, const Control *ctl, int wantG, int wantL, int wantRho, float floorDet)
{
    if (ctl && !ctl->active) return;
    const Group<T> G = groupOf<T>();
    const int i = G.i;
    if (i >= P.n) return;
    float hs = signedLength<D>(F, i);
    if (hs <= 0.0f) {
        if (G.t != 0) return;
        float zero[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
        float ident[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
        if (wantG) storeMatrix<D>(F.G0, F.G1, F.G2, i, zero);
        if (wantL) storeMatrix<D>(F.L0, F.L1, F.L2, i, ident);
        if (wantRho) F.gradRho[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        return;
    }
    GradientVisit<D, K, FINE> visit{F, Smoothing<K, D, FINE>(P, hs), wantG != 0, wantL != 0 || wantRho != 0, wantRho != 0};
    velocityOf<D>(F, i, visit.vi);
    visit.devI = deviationOf<D>(F, i);
    for (int a = 0; a < 3; ++a) {
        visit.gsum[a] = 0.0f;
        for (int b = 0; b < 3; ++b) visit.S[a][b] = 0.0f;
    }
    for (int q = 0; q < D * (D + 1) / 2; ++q) { visit.M[q] = 0.0; visit.Mf[q] = 0.0f; }
    forEachNeighbour<D, T, FINE>(P, F, i, G.t, hs, visit);
    float Mf[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
    if (wantG) {
        groupSumMatrix<D, T>(visit.S, G.mask);
        for (int a = 0; a < D; ++a)
            for (int b = a; b < D; ++b) Mf[a][b] = Mf[b][a] = groupSum<T>(visit.Mf[packed<D>(a, b)], G.mask);
    }
    double M[3][3] = {{1.0, 0.0, 0.0}, {0.0, 1.0, 0.0}, {0.0, 0.0, 1.0}};
    if (wantL || wantRho)
        for (int a = 0; a < D; ++a)
            for (int b = a; b < D; ++b) M[a][b] = M[b][a] = groupSum<T>(visit.M[packed<D>(a, b)], G.mask);
    if (wantRho)
        for (int a = 0; a < D; ++a) visit.gsum[a] = groupSum<T>(visit.gsum[a], G.mask);
    if (G.t != 0) return;
    if (wantG) {
        float Gm[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
        if (determinant<D>(Mf) >= floorDet) {
            float inv[3][3];
            inverse<D>(Mf, inv);
            for (int a = 0; a < D; ++a)
                for (int b = 0; b < D; ++b) {
                    float t = 0.0f;
                    for (int c = 0; c < D; ++c) t += visit.S[a][c] * inv[c][b];
                    Gm[a][b] = t;
                }
        }
        storeMatrix<D>(F.G0, F.G1, F.G2, i, Gm);
    }
    if (wantL || wantRho) {
        // L = M^-1 in float64, rounded once
        float L[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
        if (determinant<D>(M) >= (double)floorDet) {
            double inv[3][3];
            inverse<D>(M, inv);
            for (int a = 0; a < D; ++a)
                for (int b = 0; b < D; ++b) L[a][b] = (float)inv[a][b];
        }
        if (wantL) storeMatrix<D>(F.L0, F.L1, F.L2, i, L);
        if (wantRho) {
            float g[3] = {0.0f, 0.0f, 0.0f};
            for (int a = 0; a < D; ++a)
                for (int b = 0; b < D; ++b) g[a] += L[a][b] * visit.gsum[b];
            F.gradRho[i] = make_float4(g[0], g[1], g[2], 0.0f);
        }
    }
}

// ------------------------------------------------------------------------------------------
// Sweep C: accelerations, fluid maxima, time step
// ------------------------------------------------------------------------------------------

// BUDGET: the sum split for the energy budget too, into the pressure and the viscosity of fluid
// and of boundary neighbours (src/pysurf/sphGpu.py:400-414).  COMP: the sum compensated (Dot2),
// its running error in comp.
template <int D, int K, bool BUDGET, bool COMP = false>
struct MomentumVisit {
    static constexpr bool kSkipCoincident = true;
    static constexpr bool kPipelined = true;
    static constexpr bool kAuxRow = D == 3;
    static constexpr bool kKinetic = true;
    const Params &P; const Frame &F;
    Smoothing<K, D> S;
    float vi[3], rhoI, own, viscosityScale;   // viscosityScale: -alpha c0
    float alphaI;                               // closure: this particle's eddy alpha
    float slopeI[D * (D + 1) / 2];              // r . G_i r's coefficients: G_aa, and G_ab + G_ba (a < b)
    float total[3];
    float comp[COMP ? 3 : 1];
    float parts[BUDGET ? 4 : 1][3];
    float4 rowX;
    __device__ bool accept(bool) const { return true; }
    __device__ void operator()(int j, const float *d, float r, float h, bool fluidJ, int, const float4 &B,
                               const float4 &Kj)
    {
        const KernelAt k = S.at(h);
        const float q = r * k.invH;
        float vj[3];
        velocityIn<D>(Kj, vj);
        float rel[3] = {vi[0] - vj[0], vi[1] - vj[1], vi[2] - vj[2]};
        float approach = rel[0] * d[0] + rel[1] * d[1] + (D == 3 ? rel[2] * d[2] : 0.0f);
        const float plain = approach;           // before the limiter reconstructs it
        float viscosity = 0.0f;
        if (approach < 0.0f && P.limited && fluidJ) {
            // the slopes r . G r along the pair, each a quadratic form in r: only G's symmetric part
            // enters, so r's products d_a d_b (a <= b) serve both particles
            float Gj[3][3];
            loadMatrix<D>(F.G0, F.G1, F.G2, j, Gj);
            float slopeIJ = 0.0f, slopeJ = 0.0f;
            for (int a = 0; a < D; ++a)
                for (int b = a; b < D; ++b) {
                    const float dd = d[a] * d[b], gj = a == b ? Gj[a][a] : Gj[a][b] + Gj[b][a];
                    slopeIJ += slopeI[packed<D>(a, b)] * dd;
                    slopeJ += gj * dd;
                }
            float limiter = 0.0f;
            if (slopeIJ * slopeJ > 0.0f) {
                // 4 R / (1 + R)^2 at R = slopeI / slopeJ, as 4 slopeI slopeJ / (slopeI + slopeJ)^2
                const float sum = slopeIJ + slopeJ;
                // the fast division (2 ulp) takes 8% off the momentum sweep; its range limit (a
                // denominator past 2^126) lies far beyond any pair's slopes
                limiter = fminf(1.0f, __fdividef(4.0f * slopeIJ * slopeJ, sum * sum));
                if (q < kCloseDistance) {
                    float fade = (q - kCloseDistance) * (1.0f / kFoldWidth);
                    limiter *= expf(-fade * fade);
                }
            }
            // (v_ij - (phi / 2) (G_i + G_j) r) . r = v_ij . r - (phi / 2) (r . G_i r + r . G_j r)
            approach = plain - 0.5f * limiter * (slopeIJ + slopeJ);
        }
        if (approach < 0.0f) {
            // -alpha c0 h (v_ij . r_ij) / ((r^2 + 0.01 h^2) (rho_i + rho_j) / 2); the denominator is
            // a positive normal float for any physical pair, which __fdividef takes to 2 ulp
            viscosity = __fdividef(viscosityScale * h * approach,
                                   (r * r + k.soft) * (0.5f * (rhoI + densityIn<D>(Kj))));
            if (!fluidJ) viscosity *= P.boundaryFactor;
        }
        if (P.closure && fluidJ) {
            // delta-LES-SPH: -(K nu / (c0 h) + harmonic mean of the alphas) c0 h rho0 (v_ij . r_ij) /
            // (r^2 rho_i rho_j) on every fluid pair, approaching or not (src/pysurf/sphGpu.py:388-396)
            const float alphaJ = __ldg(&F.eddy[j].x), both = alphaI + alphaJ;
            const float mean = both > 0.0f ? 2.0f * alphaI * alphaJ / both : 0.0f;
            viscosity += -(P.waterTerm / h + mean) * P.c0 * h * P.closureRho0 * plain
                       / (r * r * rhoI * densityIn<D>(Kj));
        }
        const float ratioJ = D == 2 ? Kj.w : rowX.x;
        // explicit roundings on the sum's path, so the budget's extra uses of its terms cannot
        // change how the compiler fuses them: the tracked step is the plain step, bit for bit
        const float pressureTerm = __fadd_rn(own, ratioJ);
        float coefficient = -__fadd_rn(pressureTerm, viscosity) * massIn<D>(B);
        float f = coefficient * kernelGradient<K>(q, k);
        if constexpr (COMP) {
            for (int a = 0; a < D; ++a) addProduct(f, d[a], total[a], comp[a]);
        } else {
            for (int a = 0; a < D; ++a) total[a] = __fmaf_rn(f, d[a], total[a]);
        }
        if constexpr (BUDGET) {
            const float grad = massIn<D>(B) * kernelGradient<K>(q, k);
            const float fp = -pressureTerm * grad, fv = -viscosity * grad;
            if (fluidJ) {
                for (int a = 0; a < D; ++a) { parts[0][a] += fp * d[a]; parts[1][a] += fv * d[a]; }
            } else {
                for (int a = 0; a < D; ++a) { parts[2][a] += fp * d[a]; parts[3][a] += fv * d[a]; }
            }
        }
    }
};

__device__ __forceinline__ double cflTimeStep(double h, double c0, double vmax, double amax, double cfl, double maxdt)
{
    double dt = cfl * h / (c0 + vmax);
    if (amax > 1e-12) dt = fmin(dt, cfl * sqrt(h / amax));
    return fmin(dt, maxdt);
}

__device__ __forceinline__ double warpMax(double value)
{
    for (int offset = 16; offset > 0; offset >>= 1) value = fmax(value, __shfl_xor_sync(0xFFFFFFFFu, value, offset));
    return value;
}

// The step's fluid maxima without a block barrier: each warp folds its lanes' values and lane 0
// raises the running maxima (atomicMax on the bits of non-negative doubles, which is order-free);
// the last warp to finish takes the time step in float64 and clears the running values.
__device__ __forceinline__ void foldMaxima(Control *ctl, double speed, double accel, int warps)
{
    // non-negative, and a NaN counts as 0 as fmax would take it
    speed = warpMax(speed > 0.0 ? speed : 0.0);
    accel = warpMax(accel > 0.0 ? accel : 0.0);
    if ((threadIdx.x & 31) != 0) return;
    atomicMax(&ctl->vmaxBits, (unsigned long long)__double_as_longlong(speed));
    atomicMax(&ctl->amaxBits, (unsigned long long)__double_as_longlong(accel));
    __threadfence();
    if (atomicAdd(&ctl->ticket, 1u) != (unsigned)(warps - 1)) return;
    __threadfence();
    const double vmax = __longlong_as_double((long long)atomicMax(&ctl->vmaxBits, 0ull));
    const double amax = __longlong_as_double((long long)atomicMax(&ctl->amaxBits, 0ull));
    ctl->vmax = vmax;
    ctl->amax = amax;
    ctl->vmaxBits = 0;
    ctl->amaxBits = 0;
    ctl->ticket = 0;
    if (!ctl->hostDt) {
        const double dt = cflTimeStep(ctl->hMin, ctl->soundSpeed, vmax, amax, ctl->cfl, ctl->maxTimeStep);
        if (!(dt > 0.0) || !isfinite(dt)) ctl->error |= kErrTimeStep;
        ctl->dt = dt;
    }
}

// maxima: fold the fluid maxima into ctl and take the time step (the device steps); 0 for the
// host-step sums.
template <int D, int K, int T, bool BUDGET, bool FINE, bool COMP = false>
__global__ void __launch_bounds__(kBlock, BUDGET ? budgetMinBlocks<D>() : sweepMinBlocks<D>())
momentumKernel(Params P, Frame F, Control *ctl, int maxima)
{
    if (ctl && !ctl->active) return;
    const Group<T> G = groupOf<T>();
    const int i = G.i;
    double speed = 0.0, accel = 0.0;
    if (i < P.n) {
        float hs = signedLength<D>(F, i);
        if (hs <= 0.0f) {
            if (G.t == 0) F.acc[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        } else {
            MomentumVisit<D, K, BUDGET, COMP> visit{P, F, Smoothing<K, D>(P)};
            velocityOf<D>(F, i, visit.vi);
            visit.rhoI = densityOf<D>(F, i);
            visit.own = pressureRatioOf<D>(F, i);
            visit.viscosityScale = -P.alpha * P.c0;
            visit.alphaI = P.closure ? F.eddy[i].x : 0.0f;
            if (P.limited) {
                float Gi[3][3];
                loadMatrix<D>(F.G0, F.G1, F.G2, i, Gi);
                for (int a = 0; a < D; ++a)
                    for (int b = a; b < D; ++b) visit.slopeI[packed<D>(a, b)] = a == b ? Gi[a][a] : Gi[a][b] + Gi[b][a];
            }
            visit.total[0] = visit.total[1] = visit.total[2] = 0.0f;
            if constexpr (COMP) for (int a = 0; a < 3; ++a) visit.comp[a] = 0.0f;
            if constexpr (BUDGET)
                for (int q = 0; q < 4; ++q) visit.parts[q][0] = visit.parts[q][1] = visit.parts[q][2] = 0.0f;
            forEachNeighbour<D, T, FINE>(P, F, i, G.t, hs, visit);
            if constexpr (COMP) {
                for (int a = 0; a < D; ++a) visit.total[a] = groupSumCompensated<T>(visit.total[a], visit.comp[a], G.mask);
            } else {
                for (int a = 0; a < D; ++a) visit.total[a] = groupSum<T>(visit.total[a], G.mask);
            }
            if constexpr (BUDGET) {
                for (int q = 0; q < 4; ++q) {
                    for (int a = 0; a < D; ++a) visit.parts[q][a] = groupSum<T>(visit.parts[q][a], G.mask);
                    if (G.t == 0)
                        F.parts[(size_t)q * P.energyStride + i] =
                            make_float4(visit.parts[q][0], visit.parts[q][1], D == 3 ? visit.parts[q][2] : 0.0f, 0.0f);
                }
            }
            if (G.t == 0) {
                float a[3] = {visit.total[0] + P.g[0], visit.total[1] + P.g[1],
                              D == 3 ? visit.total[2] + P.g[2] : 0.0f};
                F.acc[i] = make_float4(a[0], a[1], a[2], 0.0f);
                double v2 = 0.0;
                for (int c = 0; c < D; ++c) v2 += F.v[c][i] * F.v[c][i];
                speed = sqrt(v2);
                accel = (double)sqrtf(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
            }
        }
    }
    if (maxima) foldMaxima(ctl, speed, accel, (int)(gridDim.x * (blockDim.x >> 5)));
}

// The delta-LES-SPH closure's coefficients (src/pysurf/sphGpu.py:699-723): ||D|| = sqrt(2 D:D) of the
// strain D = (G + G^T) / 2, alpha_i = 2 (dim + 2) (C_S l / h)^2 h ||D|| / c0 and
// delta_i = (C_delta l / h)^2 h ||D|| / c0, l = 2 h, C_S 0.12, C_delta 1.5, each at most 0.2;
// zero on the boundary.  G is the gradients sweep's, from this step's starting velocities.
template <int D>
__global__ void closureKernel(Params P, Frame F, const Control *ctl)
{
    if (ctl && !ctl->active) return;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.n) return;
    const float hs = signedLength<D>(F, i);
    if (hs <= 0.0f) {
        F.eddy[i] = make_float2(0.0f, 0.0f);
        return;
    }
    float G[3][3];
    loadMatrix<D>(F.G0, F.G1, F.G2, i, G);
    float sum = 0.0f;
    for (int a = 0; a < D; ++a)
        for (int b = 0; b < D; ++b) {
            const float e = 0.5f * (G[a][b] + G[b][a]);
            sum += e * e;
        }
    const float scale = hs * sqrtf(2.0f * sum) / P.closureC0;
    constexpr float smagorinsky = (0.12f * 2.0f) * (0.12f * 2.0f), diffusion = (1.5f * 2.0f) * (1.5f * 2.0f);
    F.eddy[i] = make_float2(fminf(2.0f * (D + 2) * smagorinsky * scale, 0.2f), fminf(diffusion * scale, 0.2f));
}

// v += a dt on the fluid (src/pysurf/sphGpu.py:1084-1109); the frame takes the kicked velocity.
template <int D>
__global__ void kickKernel(Params P, Frame F, Control *ctl)
{
    if (!ctl->active) return;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.n || !F.fluid[i]) return;
    double dt = ctl->dt;
    float4 a = F.acc[i];
    double v[3] = {0.0, 0.0, 0.0}, mean[3] = {0.0, 0.0, 0.0};
    float av[3] = {a.x, a.y, a.z};
    for (int c = 0; c < D; ++c) {
        const double start = F.v[c][i];
        v[c] = start + (double)av[c] * dt;
        F.v[c][i] = v[c];
        mean[c] = 0.5 * (start + v[c]);
    }
    if (P.budget) {
        // each part of a, and gravity, does the work m a . (v + v') / 2 dt (src/pysurf/sphGpu.py:1084-1109)
        const double m = F.m[i];
        for (int q = 0; q < 4; ++q) {
            const float4 part = F.parts[(size_t)q * P.energyStride + i];
            const float pv[3] = {part.x, part.y, part.z};
            double work = 0.0;
            for (int c = 0; c < D; ++c) work += (double)pv[c] * mean[c];
            addEnergy(P, F, i, kPressureFluid + q, m * work * dt);
        }
        double work = 0.0;
        for (int c = 0; c < D; ++c) work += (double)P.g[c] * mean[c];
        addEnergy(P, F, i, kGravityWork, m * work * dt);
    }
    float4 k = F.kin[i], low = F.low[i];
    k.x = (float)v[0]; k.y = (float)v[1];
    low.x = (float)(v[0] - (double)k.x); low.y = (float)(v[1] - (double)k.y);
    if (D == 3) { k.z = (float)v[2]; low.z = (float)(v[2] - (double)k.z); }
    F.kin[i] = k;
    F.low[i] = low;
}

// Drift (src/pysurf/sphGpu.py:1142-1186), the periodic wrap and the enforcement of one fluid slot.
template <int D>
__device__ __forceinline__ void driftAndEnforce(const Params &P, const Frame &F, const Enforcement &E, int i, double dt,
                                                const double *transport, Control *ctl)
{
    double x[3] = {0.0, 0.0, 0.0}, v[3] = {0.0, 0.0, 0.0}, lift = 0.0;
    for (int a = 0; a < D; ++a) {
        v[a] = F.v[a][i];
        const double start = F.x[a][i];
        x[a] = start + (transport ? transport[a] : v[a]) * dt;
        lift += P.gravity64[a] * (x[a] - start);
    }
    // the drift's change of potential energy, from the displacement as stored (src/pysurf/sphGpu.py:1168-1170)
    if (P.budget) addEnergy(P, F, i, kDrift, -F.m[i] * lift);
    if (P.period > 0.0) x[1] = x[1] - P.period * floor(x[1] / P.period);
    enforceTracked(P, F, E, D, i, x, v);
    bool finite = true;
    for (int a = 0; a < D; ++a) {
        F.x[a][i] = x[a];
        F.v[a][i] = v[a];
        finite = finite && isfinite(x[a]) && isfinite(v[a]);
    }
    if (!finite) atomicOr(&ctl->error, kErrNonFinite);
}

// ------------------------------------------------------------------------------------------
// Sweep D: continuity with the density update, drift and enforcement
// ------------------------------------------------------------------------------------------

// BUDGET: the rate split for the energy budget too: the plain sum over fluid and over boundary
// neighbours, the corrected sum (the correction's part is its difference) and the diffusion
// (src/pysurf/sphGpu.py:476-545).  COMP: the float32 sum compensated (Dot2), its running error in comp.
//
// The rate's terms cancel: next to a wall a particle's velocity jumps to the boundary's zero, and
// sum_j m_j (v_i - v_j) . grad W_ij over a near-symmetric support is a small remainder of large
// terms.  So each term keeps float64's digits where that matters: velocity and deviation differences
// come from the float32 values and their remainders (the frame's low row), and the pairs of a fluid
// and a boundary particle -- every pair of a boundary row, the wall's pairs of a fluid row -- take
// their separation, distance, kernel gradient and term in float64, summed apart in float64 (cross).
// Fluid pairs, whose velocity differences are small, keep float32 arithmetic.
template <int D, int K, bool BUDGET, bool COMP = false>
struct ContinuityVisit {
    static constexpr bool kSkipCoincident = true;
    static constexpr bool kPipelined = true;
    static constexpr bool kAuxRow = D == 3;
    static constexpr bool kLowRow = true;
    static constexpr bool kKinetic = true;
    static constexpr bool kBoundaryRows = true;         // every row
    const Params &P; const Frame &F;
    Smoothing<K, D> S;
    int self;               // this particle's slot
    bool boundaryI, diffuses, corrected;
    float vi[3], vlI[3], devI, devLoI, Li[3][3], gi[3];
    float deltaI;           // closure: this particle's eddy delta
    float total, comp;
    double cross;           // the fluid-boundary pairs' terms in float64
    float plainFluid, plainWall, continuity, diffusive;     // BUDGET
    float4 rowX, rowLow;
    __device__ bool accept(bool fluidJ) const { return !(boundaryI && !fluidJ); }
    __device__ void operator()(int j, const float *d, float r, float h, bool fluidJ, int image, const float4 &B,
                               const float4 &Kj)
    {
        const KernelAt k = S.at(h);
        float vj[3];
        velocityIn<D>(Kj, vj);
        const float4 lowJ = rowLow;
        const float vlJ[3] = {lowJ.x, lowJ.y, lowJ.z};
        if (boundaryI == fluidJ) {
            // a fluid-boundary pair, in float64: x_i - x_j from the points and remainders, the distance
            // by one Newton step from the float32 root, (dW/dr) / r, (v_i - v_j) . L_i (x_i - x_j)
            const float4 A = __ldg(&F.pa[j]);
            float pi[3], li[3], pj[3], lj[3];
            pointOf<D>(F, self, pi);
            remainderOf<D>(F, self, li);
            pointIn<D>(A, pj);
            remainderIn<D>(A, B, lj);
            double dd[3] = {0.0, 0.0, 0.0}, r2 = 0.0;
            for (int a = 0; a < D; ++a) {
                dd[a] = ((double)pi[a] - (double)pj[a]) + ((double)li[a] - (double)lj[a]);
                if (a == 1 && image) dd[a] += pi[1] < 0.5f * P.periodF ? P.period : -P.period;
                r2 = fma(dd[a], dd[a], r2);
            }
            const double rf = (double)r, rr = fma(fma(-rf, rf, r2), 0.5 / rf, rf);
            const double grad = kernelGradient64<K>(rr, k);
            double dot = 0.0;
            for (int a = 0; a < D; ++a) {
                double ld = dd[a];
                if (corrected) {
                    ld = 0.0;
                    for (int b = 0; b < D; ++b) ld = fma((double)Li[a][b], dd[b], ld);
                }
                dot = fma(((double)vi[a] + (double)vlI[a]) - ((double)vj[a] + (double)vlJ[a]), ld, dot);
            }
            const double term = (double)massIn<D>(B) * dot * grad;
            cross += term;
            if constexpr (BUDGET) {
                double plainDot = dot;
                if (corrected) {
                    plainDot = 0.0;
                    for (int a = 0; a < D; ++a)
                        plainDot = fma(((double)vi[a] + (double)vlI[a]) - ((double)vj[a] + (double)vlJ[a]), dd[a], plainDot);
                }
                const float plain = (float)((double)massIn<D>(B) * plainDot * grad);
                continuity = __fadd_rn(continuity, (float)term);
                if (fluidJ) plainFluid += plain; else plainWall += plain;
            }
            return;     // a pair with a boundary member does not diffuse
        }
        const float grad = kernelGradient<K>(r * k.invH, k);    // (dW/dr) / r
        float dv[3];
        for (int a = 0; a < D; ++a)
            dv[a] = __fadd_rn(__fsub_rn(vi[a], vj[a]), __fsub_rn(vlI[a], vlJ[a]));
        float dot = 0.0f;
        if (corrected) {
            for (int a = 0; a < D; ++a) {
                float ld = 0.0f;
                for (int b = 0; b < D; ++b) ld += Li[a][b] * d[b];
                dot += dv[a] * ld;
            }
        } else {
            for (int a = 0; a < D; ++a) dot += dv[a] * d[a];
        }
        // explicit roundings on the sum's path (see the momentum sweep)
        const float massDot = massIn<D>(B) * dot;
        if constexpr (COMP) addProduct(massDot, grad, total, comp);
        else total = __fmaf_rn(massDot, grad, total);
        if constexpr (BUDGET) {
            float plainDot = dot;
            if (corrected) {
                plainDot = 0.0f;
                for (int a = 0; a < D; ++a) plainDot += dv[a] * d[a];
            }
            const float plain = massIn<D>(B) * plainDot * grad;
            continuity = __fmaf_rn(massDot, grad, continuity);
            if (fluidJ) plainFluid += plain; else plainWall += plain;
        }
        if (diffuses && fluidJ) {
            const float4 X = D == 3 ? rowX : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            const float devJ = deviationIn<D>(B, X);
            // rho_j - rho_i from the float32 deviations and their remainders, so it keeps float64's
            // digits (the leading difference is exact for neighbours' nearly equal deviations)
            const float remainder = __fsub_rn(lowJ.w, devLoI);
            float difference;
            if (P.diffusion == 2) {
                // less the hydrostatic difference k dz (1 + e)^-5 (src/pysurf/sphSolver.py:718-735), with
                // k = rho0 g / c0^2 and e the pair's mean deviation over rho0.  Near rest it cancels most
                // of rho_j - rho_i, so it is taken in two parts: k dz off the leading difference in one
                // fused rounding, then the small k dz e S / (1 + e)^5 back on, where
                // S = 1 + (1 + e) + ... + (1 + e)^4 makes (1 + e)^5 - 1 = e S without cancelling.
                const float e = __fmul_rn(__fadd_rn(devI, devJ), P.halfInvRho0);
                const float ratio = __fadd_rn(1.0f, e), sq = __fmul_rn(ratio, ratio), fifth = __fmul_rn(__fmul_rn(sq, sq), ratio);
                const float S = __fadd_rn(__fadd_rn(__fadd_rn(1.0f, ratio), __fadd_rn(sq, __fmul_rn(sq, ratio))),
                                          __fmul_rn(sq, sq));
                const float slope = __fmul_rn(P.hydrostaticSlope, d[D - 1]);
                const float leading = __fmaf_rn(-P.hydrostaticSlope, d[D - 1], __fsub_rn(devJ, devI));
                difference = __fadd_rn(__fadd_rn(leading, remainder), __fdividef(__fmul_rn(__fmul_rn(slope, e), S), fifth));
            } else {
                difference = __fadd_rn(__fsub_rn(devJ, devI), remainder);
            }
            if (P.diffusion == 3) {
                float4 gj = __ldg(&F.gradRho[j]);
                float gjv[3] = {gj.x, gj.y, gj.z};
                float t = 0.0f;
                for (int a = 0; a < D; ++a) t += (gi[a] + gjv[a]) * d[a];
                difference += 0.5f * t;
            }
            // 2 delta c0 h V_j (difference) (-(dW/dr) r) / (r^2 + 0.01 h^2), with (dW/dr) r = grad r^2;
            // with the closure, 2 delta c0 is 2 c0 times the harmonic mean of the two deltas
            float factor = P.diffusionFactor;
            if (P.closure) {
                const float deltaJ = __ldg(&F.eddy[j].y), both = deltaI + deltaJ;
                factor = both > 0.0f ? 2.0f * P.closureC0 * (2.0f * deltaI * deltaJ / both) : 0.0f;
            }
            const float r2 = r * r;
            const float head = factor * h * volumeIn<D>(B, X) * difference * (-grad), ratio = __fdividef(r2, r2 + k.soft);
            if constexpr (COMP) addProduct(head, ratio, total, comp);
            else total = __fmaf_rn(head, ratio, total);
            if constexpr (BUDGET) diffusive = __fmaf_rn(head, ratio, diffusive);
        }
    }
};

// mode 0: the rate only; 1: advance the density; 2: advance, drift and enforce.
template <int D, int K, int T, bool BUDGET, bool FINE, bool COMP = false>
__global__ void __launch_bounds__(kBlock, BUDGET ? budgetMinBlocks<D>() : preciseMinBlocks<D>())
continuityKernel(Params P, Frame F, Control *ctl, Enforcement E, int mode)
{
    if (ctl && !ctl->active) return;
    const Group<T> G = groupOf<T>();
    const int i = G.i;
    if (i >= P.n) return;
    float hs = signedLength<D>(F, i);
    ContinuityVisit<D, K, BUDGET, COMP> visit{P, F, Smoothing<K, D>(P)};
    visit.boundaryI = hs <= 0.0f;
    visit.diffuses = P.diffusion != 0 && !visit.boundaryI;
    visit.corrected = P.corrected && !visit.boundaryI;
    velocityOf<D>(F, i, visit.vi);
    const float4 lowI = F.low[i];
    visit.vlI[0] = lowI.x; visit.vlI[1] = lowI.y; visit.vlI[2] = lowI.z;
    visit.devLoI = lowI.w;
    visit.self = i;
    visit.cross = 0.0;
    visit.devI = deviationOf<D>(F, i);
    visit.deltaI = P.closure && visit.diffuses ? F.eddy[i].y : 0.0f;
    if (visit.corrected) loadMatrix<D>(F.L0, F.L1, F.L2, i, visit.Li);
    visit.gi[0] = visit.gi[1] = visit.gi[2] = 0.0f;
    if (visit.diffuses && P.diffusion == 3) {
        float4 g = F.gradRho[i];
        visit.gi[0] = g.x; visit.gi[1] = g.y; visit.gi[2] = g.z;
    }
    visit.total = visit.comp = 0.0f;
    visit.plainFluid = visit.plainWall = visit.continuity = visit.diffusive = 0.0f;
    forEachNeighbour<D, T, FINE>(P, F, i, G.t, fabsf(hs), visit);
    float rate;
    if constexpr (COMP) rate = groupSumCompensated<T>(visit.total, visit.comp, G.mask);
    else rate = groupSum<T>(visit.total, G.mask);
    // the fluid-boundary pairs' float64 sum joins before the one rounding to float32
    rate = (float)((double)rate + groupSum<T>(visit.cross, G.mask));
    float parts[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    if constexpr (BUDGET) {
        const float plainFluid = groupSum<T>(visit.plainFluid, G.mask);
        const float plainWall = groupSum<T>(visit.plainWall, G.mask);
        const float continuity = groupSum<T>(visit.continuity, G.mask);
        parts[0] = plainFluid;
        parts[1] = plainWall;
        parts[2] = visit.corrected ? continuity - plainFluid - plainWall : 0.0f;
        parts[3] = groupSum<T>(visit.diffusive, G.mask);
    }
    if (G.t != 0) return;
    F.rate[i] = rate;
    if (mode == 0) return;
    double dt = ctl->dt;
    const double start = F.rho[i];
    double rho = start + (double)rate * dt;
    const double unfloored = rho;
    bool fluid = hs > 0.0f;
    if (P.densityFloor > 0.0 && fluid) rho = fmax(rho, P.densityFloor);
    F.rho[i] = rho;
    if (BUDGET && fluid) {
        // each part of the rate over the secant slope of e, and the floor's change (src/pysurf/sphGpu.py:1111-1140)
        const double m = F.m[i], slope = elasticSlope(P, start, unfloored);
        for (int q = 0; q < 4; ++q) addEnergy(P, F, i, kContinuityFluid + q, m * slope * (double)parts[q] * dt);
        addEnergy(P, F, i, kFloor, m * (elasticEnergy(P, rho) - elasticEnergy(P, unfloored)));
    }
    if (!isfinite(rho)) atomicOr(&ctl->error, kErrNonFinite);
    if (mode == 2 && fluid) driftAndEnforce<D>(P, F, E, i, dt, nullptr, ctl);
}

// ------------------------------------------------------------------------------------------
// Sweep X: XSPH over fluid pairs, with the densities the step has just advanced
// ------------------------------------------------------------------------------------------

template <int D, int K>
struct XsphVisit {
    static constexpr bool kSkipCoincident = false;
    static constexpr bool kKinetic = true;
    const Frame &F; const float *densities;
    Smoothing<K, D> S;
    float vi[3], rhoI, corr[3];
    __device__ bool accept(bool fluidJ) const { return fluidJ; }
    __device__ void operator()(int j, const float *, float r, float h, bool, int, const float4 &B, const float4 &Kj)
    {
        const KernelAt k = S.at(h);
        float w = kernelValue<K>(r * k.invH, k);
        float rhoJ = densities ? densities[j] : densityIn<D>(Kj);
        float weight = massIn<D>(B) * w / (0.5f * (rhoI + rhoJ));
        float vj[3];
        velocityIn<D>(Kj, vj);
        for (int a = 0; a < D; ++a) corr[a] += weight * (vj[a] - vi[a]);
    }
};

// densities: the float32 densities the sum divides by (null: the frame's).  mode 0: the transport
// velocity into F.vec only; 2: drift with it and enforce.
template <int D, int K, int T, bool FINE>
__global__ void __launch_bounds__(kBlock, sweepMinBlocks<D>())
xsphKernel(Params P, Frame F, Control *ctl, Enforcement E, const float *densities, int mode)
{
    if (ctl && !ctl->active) return;
    const Group<T> G = groupOf<T>();
    const int i = G.i;
    if (i >= P.n) return;
    float hs = signedLength<D>(F, i);
    float v[3];
    velocityOf<D>(F, i, v);
    if (hs <= 0.0f) {
        if (G.t == 0) F.vec[i] = make_float4(v[0], v[1], v[2], 0.0f);
        return;
    }
    XsphVisit<D, K> visit{F, densities, Smoothing<K, D>(P)};
    visit.vi[0] = v[0]; visit.vi[1] = v[1]; visit.vi[2] = v[2];
    visit.rhoI = densities ? densities[i] : densityOf<D>(F, i);
    visit.corr[0] = visit.corr[1] = visit.corr[2] = 0.0f;
    forEachNeighbour<D, T, FINE>(P, F, i, G.t, hs, visit);
    for (int a = 0; a < D; ++a) visit.corr[a] = groupSum<T>(visit.corr[a], G.mask);
    if (G.t != 0) return;
    float t[3];
    for (int a = 0; a < 3; ++a) t[a] = v[a] + P.xsphEpsilon * visit.corr[a];
    F.vec[i] = make_float4(t[0], t[1], t[2], 0.0f);
    if (mode != 2) return;
    double transport[3] = {(double)t[0], (double)t[1], (double)t[2]};
    driftAndEnforce<D>(P, F, E, i, ctl->dt, transport, ctl);
}

// ------------------------------------------------------------------------------------------
// Particle shifting (src/pysurf/sphGpu.py:856-1008; src/pysurf/sphSolver.py:824-1010), after the
// density update, from the step's starting geometry (the frame's points), the updated densities and
// the kicked velocities
// ------------------------------------------------------------------------------------------

// The frame takes the updated float64 densities: rho, rho - rho0, V = m / rho (p and p / rho^2
// are not read again this step).
template <int D>
__global__ void frameDensityKernel(Params P, Frame F, const Control *ctl)
{
    if (ctl && !ctl->active) return;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.n) return;
    storeDensity<D>(F, i, massOf<D>(F, i), F.rho[i], P.devReference, F.pres[i]);
}

// Over every neighbour of a fluid slot: grad C with the anti-clumping weight 1 + 0.2 (W / W(dx))^4,
// grad C0, div r = -sum V_j r_ij . grad W_ij, grad rho from the deviations.
template <int D, int K>
struct ShiftFieldsVisit {
    static constexpr bool kSkipCoincident = true;
    static constexpr bool kKinetic = false;
    const Params &P; const Frame &F;
    Smoothing<K, D> S;
    float devI, gradient[3], plain[3], densityGradient[3], total;
    __device__ bool accept(bool) const { return true; }
    __device__ void operator()(int j, const float *d, float r, float h, bool, int, const float4 &B, const float4 &)
    {
        const KernelAt k = S.at(h);
        const float q = r * k.invH;
        const float4 X = auxRow<D>(F, j);
        const float volume = volumeIn<D>(B, X);
        const float grad = kernelGradient<K>(q, k);         // (dW/dr) / r
        const float ratio = kernelValue<K>(q, k) / P.spacingKernel, square = ratio * ratio;
        const float weight = 1.0f + 0.2f * square * square;
        const float difference = deviationIn<D>(B, X) - devI;
        for (int a = 0; a < D; ++a) {
            const float weighted = volume * grad * d[a];
            plain[a] += weighted;
            gradient[a] += weight * weighted;
            densityGradient[a] += difference * weighted;
        }
        total -= volume * grad * r * r;
    }
};

template <int D, int K, int T, bool FINE>
__global__ void __launch_bounds__(kBlock, sweepMinBlocks<D>()) shiftFieldsKernel(Params P, Frame F, const Control *ctl)
{
    if (ctl && !ctl->active) return;
    const Group<T> G = groupOf<T>();
    const int i = G.i;
    if (i >= P.n) return;
    const float hs = signedLength<D>(F, i);
    if (hs <= 0.0f) {
        if (G.t != 0) return;
        const float4 zero = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        F.shiftGrad[i] = zero;
        F.shiftPlain[i] = make_float4(0.0f, 0.0f, 0.0f, 1.0e6f);
        F.shiftRhoGrad[i] = zero;
        return;
    }
    ShiftFieldsVisit<D, K> visit{P, F, Smoothing<K, D>(P)};
    visit.devI = deviationOf<D>(F, i);
    for (int a = 0; a < 3; ++a) visit.gradient[a] = visit.plain[a] = visit.densityGradient[a] = 0.0f;
    visit.total = 0.0f;
    forEachNeighbour<D, T, FINE>(P, F, i, G.t, hs, visit);
    float c[3] = {0.0f, 0.0f, 0.0f}, g[3] = {0.0f, 0.0f, 0.0f}, rg[3] = {0.0f, 0.0f, 0.0f};
    for (int a = 0; a < D; ++a) {
        c[a] = groupSum<T>(visit.plain[a], G.mask);
        g[a] = groupSum<T>(visit.gradient[a], G.mask);
        rg[a] = groupSum<T>(visit.densityGradient[a], G.mask);
    }
    float total = groupSum<T>(visit.total, G.mask);
    if (G.t != 0) return;
    // a lopsided support marks the free surface (src/pysurf/sphSolver.py:889-902)
    if (hs * sqrtf(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]) > P.lopsidedness) total = -1.0f;
    F.shiftGrad[i] = make_float4(g[0], g[1], g[2], 0.0f);
    F.shiftPlain[i] = make_float4(c[0], c[1], c[2], total);
    F.shiftRhoGrad[i] = make_float4(rg[0], rg[1], rg[2], 0.0f);
}

// The surface neighbours of a slot: whether there is one within the support, and the
// kernel-weighted sum of their outward normals -grad C0 / |grad C0|.
template <int D, int K>
struct SurfaceVisit {
    static constexpr bool kSkipCoincident = false;
    static constexpr bool kKinetic = false;
    const Params &P; const Frame &F;
    Smoothing<K, D> S;
    float normal[3];
    int vicinity;
    __device__ bool accept(bool fluidJ) const { return fluidJ; }
    __device__ void operator()(int j, const float *, float r, float h, bool, int, const float4 &, const float4 &)
    {
        const float4 plainJ = __ldg(&F.shiftPlain[j]);
        if (!(plainJ.w < P.shiftThreshold)) return;
        vicinity = 1;
        const float length = sqrtf(plainJ.x * plainJ.x + plainJ.y * plainJ.y + plainJ.z * plainJ.z);
        if (length > 0.0f) {
            const KernelAt k = S.at(h);
            const float w = kernelValue<K>(r * k.invH, k) / length;
            normal[0] -= w * plainJ.x;
            normal[1] -= w * plainJ.y;
            normal[2] -= w * plainJ.z;
        }
    }
};

// The velocity at the shifted position: sum_j V_j (v_j - v_i) (grad W_ij . shift) over fluid pairs.
template <int D, int K>
struct ShiftedVelocityVisit {
    static constexpr bool kSkipCoincident = true;
    static constexpr bool kKinetic = true;
    const Params &P; const Frame &F;
    Smoothing<K, D> S;
    float vi[3], shift[3], change[3];
    __device__ bool accept(bool fluidJ) const { return fluidJ; }
    __device__ void operator()(int j, const float *d, float r, float h, bool, int, const float4 &B, const float4 &Kj)
    {
        const KernelAt k = S.at(h);
        const float4 X = auxRow<D>(F, j);
        float dot = 0.0f;
        for (int a = 0; a < D; ++a) dot += d[a] * shift[a];
        const float f = volumeIn<D>(B, X) * kernelGradient<K>(r * k.invH, k) * dot;
        float vj[3];
        velocityIn<D>(Kj, vj);
        for (int a = 0; a < D; ++a) change[a] += f * (vj[a] - vi[a]);
    }
};

// The shift of a fluid slot off the free surface: -size grad C, along the surface next to a
// surface particle (none where h |grad C| > 0.03 there), with the density change shift . grad rho
// and the velocity change at the new position.  size: CFL Ma (2h)^2 with CFL = c0 dt / h, or
// 2 h |v_i| dt (local).
template <int D, int K, int T, bool FINE>
__global__ void __launch_bounds__(kBlock, sweepMinBlocks<D>()) shiftKernel(Params P, Frame F, const Control *ctl)
{
    if (ctl && !ctl->active) return;
    const Group<T> G = groupOf<T>();
    const int i = G.i;
    if (i >= P.n) return;
    const float4 zero = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    const float hs = signedLength<D>(F, i);
    if (hs <= 0.0f || !(F.shiftPlain[i].w >= P.shiftThreshold)) {
        if (G.t == 0) { F.shift[i] = zero; F.shiftDv[i] = zero; }
        return;
    }
    SurfaceVisit<D, K> surface{P, F, Smoothing<K, D>(P)};
    surface.normal[0] = surface.normal[1] = surface.normal[2] = 0.0f;
    surface.vicinity = 0;
    forEachNeighbour<D, T, FINE>(P, F, i, G.t, hs, surface);
    float normal[3];
    for (int a = 0; a < 3; ++a) normal[a] = groupSum<T>(surface.normal[a], G.mask);
    const bool vicinity = groupSum<T>((float)surface.vicinity, G.mask) > 0.0f;
    float vi[3];
    velocityOf<D>(F, i, vi);
    const double dt = ctl ? ctl->dt : P.shiftDt;
    const float size =
        P.shiftLocal ? (float)(2.0 * (double)hs * (double)sqrtf(vi[0] * vi[0] + vi[1] * vi[1] + vi[2] * vi[2]) * dt)
                     : (float)(P.shiftScale * dt);
    const float4 g = F.shiftGrad[i];
    float shift[3] = {-size * g.x, -size * g.y, -size * g.z};
    if (vicinity) {
        if (hs * sqrtf(g.x * g.x + g.y * g.y + g.z * g.z) > 0.03f) {
            shift[0] = shift[1] = shift[2] = 0.0f;
        } else {
            const float weight = sqrtf(normal[0] * normal[0] + normal[1] * normal[1] + normal[2] * normal[2]);
            if (weight > 0.0f) {
                float dot = 0.0f;
                for (int a = 0; a < 3; ++a) { normal[a] /= weight; dot += shift[a] * normal[a]; }
                for (int a = 0; a < 3; ++a) shift[a] -= dot * normal[a];
            }
        }
    }
    if (D == 2) shift[2] = 0.0f;
    const float4 rg = F.shiftRhoGrad[i];
    const float densityChange = shift[0] * rg.x + shift[1] * rg.y + shift[2] * rg.z;
    float change[3] = {0.0f, 0.0f, 0.0f};
    if (shift[0] != 0.0f || shift[1] != 0.0f || shift[2] != 0.0f) {
        ShiftedVelocityVisit<D, K> velocity{P, F, Smoothing<K, D>(P)};
        for (int a = 0; a < 3; ++a) { velocity.vi[a] = vi[a]; velocity.shift[a] = shift[a]; velocity.change[a] = 0.0f; }
        forEachNeighbour<D, T, FINE>(P, F, i, G.t, hs, velocity);
        for (int a = 0; a < D; ++a) change[a] = groupSum<T>(velocity.change[a], G.mask);
    }
    if (G.t != 0) return;
    F.shift[i] = make_float4(shift[0], shift[1], shift[2], densityChange);
    F.shiftDv[i] = make_float4(change[0], change[1], change[2], 0.0f);
}

// The drift of a shifting step (src/pysurf/sphGpu.py:1142-1186): x += u dt + shift, rho and v take
// their changes, then the periodic wrap and the enforcement.  transport: XSPH's F.vec, else v.
template <int D>
__global__ void shiftDriftKernel(Params P, Frame F, Control *ctl, Enforcement E, int useTransport)
{
    if (!ctl->active) return;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.n || !F.fluid[i]) return;
    const double dt = ctl->dt;
    const float4 s = F.shift[i], dv = F.shiftDv[i];
    const float4 u = F.vec[i];
    const float sh[3] = {s.x, s.y, s.z}, dvel[3] = {dv.x, dv.y, dv.z}, ut[3] = {u.x, u.y, u.z};
    double x[3] = {0.0, 0.0, 0.0}, v[3] = {0.0, 0.0, 0.0}, lift = 0.0, kinetic = 0.0, shiftLift = 0.0;
    for (int a = 0; a < D; ++a) {
        const double velocity = useTransport ? (double)ut[a] : F.v[a][i], start = F.x[a][i];
        x[a] = start + velocity * dt;
        lift += P.gravity64[a] * (x[a] - start);
        x[a] = x[a] + (double)sh[a];
        shiftLift += P.gravity64[a] * (double)sh[a];
        v[a] = F.v[a][i] + (double)dvel[a];
        kinetic += v[a] * v[a] - F.v[a][i] * F.v[a][i];
    }
    const double rhoStart = F.rho[i];
    F.rho[i] = rhoStart + (double)s.w;
    if (P.budget) {
        // the drift's change of potential energy, and the shift's of kinetic, elastic and potential
        // energy (src/pysurf/sphGpu.py:1166-1183)
        const double m = F.m[i];
        addEnergy(P, F, i, kDrift, -m * lift);
        addEnergy(P, F, i, kShifting,
                  m * (0.5 * kinetic + elasticEnergy(P, F.rho[i]) - elasticEnergy(P, rhoStart) - shiftLift));
    }
    if (P.period > 0.0) x[1] = x[1] - P.period * floor(x[1] / P.period);
    enforceTracked(P, F, E, D, i, x, v);
    bool finite = isfinite(F.rho[i]);
    for (int a = 0; a < D; ++a) {
        F.x[a][i] = x[a];
        F.v[a][i] = v[a];
        finite = finite && isfinite(x[a]) && isfinite(v[a]);
    }
    if (!finite) atomicOr(&ctl->error, kErrNonFinite);
}

// ------------------------------------------------------------------------------------------
// Launchers
// ------------------------------------------------------------------------------------------

static inline int blocksFor(long long n, int block) { return (int)((n + block - 1) / block); }

#ifndef SPH_LIST_LANES_2D
#define SPH_LIST_LANES_2D 8
#endif
constexpr int kListLanes2 = SPH_LIST_LANES_2D;
constexpr int kListLanes3 = 4;

// The table kernel: lanes a slot (the 2D stencil's runs are longer), and its precision and
// smoothing-length forms.
// The table kernel a dimension takes: in 3D a cell holds about 8 particles, and the cell batches
// build the table a quarter faster than lanes a particle (19.8 against 14.4 ms a step on the 16-ppd
// ridge, 17.1 against 13.1 on the refined 12-ppd one); a 2D cell holds about 4, too few to pay for
// a batch's setup (0.149 against 0.112 ms on the 64-ppd beach), so 2D keeps the lanes.
template <int D>
static void launchList(const LaunchArgs &A)
{
    if (D == 3) {
        const int grid = blocksFor((long long)blocksFor(A.P.n, kBatch) * 32, kBlock);
        cudaStream_t st = A.stream;
        if (A.P.precise && !A.P.mixedH) cellListKernel<D, true, false><<<grid, kBlock, 0, st>>>(A.P, A.F, A.ctl, A.maxCount);
        else if (A.P.precise) cellListKernel<D, true, true><<<grid, kBlock, 0, st>>>(A.P, A.F, A.ctl, A.maxCount);
        else if (!A.P.mixedH) cellListKernel<D, false, false><<<grid, kBlock, 0, st>>>(A.P, A.F, A.ctl, A.maxCount);
        else cellListKernel<D, false, true><<<grid, kBlock, 0, st>>>(A.P, A.F, A.ctl, A.maxCount);
        return;
    }
    constexpr int L = D == 2 ? kListLanes2 : kListLanes3;
    const int grid = blocksFor((long long)A.P.n * L, kBlock);
    cudaStream_t st = A.stream;
    if (A.P.precise && !A.P.mixedH) listKernel<D, L, true, false><<<grid, kBlock, 0, st>>>(A.P, A.F, A.ctl, A.maxCount);
    else if (A.P.precise) listKernel<D, L, true, true><<<grid, kBlock, 0, st>>>(A.P, A.F, A.ctl, A.maxCount);
    else if (!A.P.mixedH) listKernel<D, L, false, false><<<grid, kBlock, 0, st>>>(A.P, A.F, A.ctl, A.maxCount);
    else listKernel<D, L, false, true><<<grid, kBlock, 0, st>>>(A.P, A.F, A.ctl, A.maxCount);
}

template <int D, int K, int T, bool FINE>
static void launchT(const LaunchArgs &A, Stage stage)
{
    const Params &P = A.P;
    const Frame &F = A.F;
    const int grid = blocksFor((long long)P.n * T, kBlock), pointwise = blocksFor(P.n, kBlock);
    if (P.n == 0) return;
    cudaStream_t st = A.stream;
    switch (stage) {
    case Stage::ShepardSum: shepardKernel<D, K, T, FINE><<<grid, kBlock, 0, st>>>(P, F, A.ctl); break;
    case Stage::ShepardApply: applyShepardKernel<D><<<pointwise, kBlock, 0, st>>>(P, F, A.ctl); break;
    case Stage::Wall: wallPressureKernel<D, K, T, FINE><<<grid, kBlock, 0, st>>>(P, F, A.ctl, A.flag); break;
    case Stage::Gradients:
        gradientKernel<D, K, T, FINE><<<grid, kBlock, 0, st>>>(P, F, A.ctl, A.wantG, A.wantL, A.wantRho, A.floorDet);
        break;
    case Stage::Momentum:
        if (P.budget && A.maxima) momentumKernel<D, K, T, true, FINE><<<grid, kBlock, 0, st>>>(P, F, A.ctl, A.maxima);
        else if (P.compensated)
            momentumKernel<D, K, T, false, FINE, true><<<grid, kBlock, 0, st>>>(P, F, A.ctl, A.maxima);
        else momentumKernel<D, K, T, false, FINE><<<grid, kBlock, 0, st>>>(P, F, A.ctl, A.maxima);
        break;
    case Stage::Kick: kickKernel<D><<<pointwise, kBlock, 0, st>>>(P, F, A.ctl); break;
    case Stage::Continuity:
        // the budget's parts matter only where the step advances the density
        if (P.budget && A.flag != 0) continuityKernel<D, K, T, true, FINE><<<grid, kBlock, 0, st>>>(P, F, A.ctl, A.E, A.flag);
        else if (P.compensated)
            continuityKernel<D, K, T, false, FINE, true><<<grid, kBlock, 0, st>>>(P, F, A.ctl, A.E, A.flag);
        else continuityKernel<D, K, T, false, FINE><<<grid, kBlock, 0, st>>>(P, F, A.ctl, A.E, A.flag);
        break;
    case Stage::Xsph: xsphKernel<D, K, T, FINE><<<grid, kBlock, 0, st>>>(P, F, A.ctl, A.E, A.densities, A.flag); break;
    case Stage::List: launchList<D>(A); break;
    case Stage::Closure: closureKernel<D><<<pointwise, kBlock, 0, st>>>(P, F, A.ctl); break;
    case Stage::ShiftFields: shiftFieldsKernel<D, K, T, false><<<grid, kBlock, 0, st>>>(P, F, A.ctl); break;
    case Stage::Shift: shiftKernel<D, K, T, false><<<grid, kBlock, 0, st>>>(P, F, A.ctl); break;
    case Stage::ShiftDrift: shiftDriftKernel<D><<<pointwise, kBlock, 0, st>>>(P, F, A.ctl, A.E, A.flag); break;
    case Stage::FrameDensity: frameDensityKernel<D><<<pointwise, kBlock, 0, st>>>(P, F, A.ctl); break;
    }
}

template <int D, int K>
static void launchDK(const LaunchArgs &A, Stage stage)
{
    if (A.P.levels > 1) {
        // the shifting sweeps never see two levels (shifting needs one smoothing length)
        if (A.threads >= 8) launchT<D, K, 8, true>(A, stage);
        else if (A.threads == 4) launchT<D, K, 4, true>(A, stage);
        else if (A.threads == 2) launchT<D, K, 2, true>(A, stage);
        else launchT<D, K, 1, true>(A, stage);
    } else {
        if (A.threads >= 8) launchT<D, K, 8, false>(A, stage);
        else if (A.threads == 4) launchT<D, K, 4, false>(A, stage);
        else if (A.threads == 2) launchT<D, K, 2, false>(A, stage);
        else launchT<D, K, 1, false>(A, stage);
    }
}

void launchStage(const LaunchArgs &A, Stage stage)
{
    const int D = A.P.dim, K = A.P.kind;
    if (D == 2 && K == 0) launchDK<2, 0>(A, stage);
    else if (D == 2 && K == 1) launchDK<2, 1>(A, stage);
    else if (D == 3 && K == 0) launchDK<3, 0>(A, stage);
    else launchDK<3, 1>(A, stage);
}

}  // namespace sph
