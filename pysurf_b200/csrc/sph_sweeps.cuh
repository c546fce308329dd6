// sph_sweeps.cuh -- the neighbour walk every sweep shares, and its neighbour table.
//
// A particle's neighbours lie in the cells within +-ncs of its own along each axis; cells are
// numbered x fastest, so each (y, z) row of the stencil is one contiguous run of the sorted
// order, [cellStart[first], cellStart[last + 1]).  Candidates are tested on their float32 points
// first (the reference's coarse test, src/pysurf/sphGpu.py:330-336), and only survivors take the
// precise separation (hi_i - hi_j) + (lo_i - lo_j).
//
// Each step the table kernel walks the cells once and records, per particle, the neighbours the
// walk accepts, in the walk's order, in a table of 16-byte chunks: entries 4c .. 4c + 3 of particle
// i form chunk c, stored at c * stride + i, so a lane takes four neighbours with one load and a
// warp's loads of chunk c are contiguous.  The sweeps then read the table
// instead of walking the cells: no candidate that fails the distance test is visited again, so
// a warp's lanes stay busy.  A particle with more neighbours than its row holds walks the cells
// instead.  Table and walk feed one loop body, the visitor called from one place, so a sweep
// gives the same bits either way.
//
// T threads serve one particle: lane t of the group takes the particle's neighbours in chunks t,
// t + T, t + 2T, ... (neighbour k, counted in the walk's order, is in chunk k / 4), and the group
// sums its partial sums with a
// butterfly of shuffles, which gives every lane the same bits (each level adds two values whose
// order does not matter).  T = 1 is the plain one-thread-per-particle sweep.
//
// A periodic y axis (3D) is searched a second time from the particle's image across the seam
// when it lies within its reach of the seam (src/pysurf/sphGpu.py:206-225).  Each search tests
// its candidates against its own origin (the particle, or its image); a period longer than twice
// the reach (the solver requires twice the support, src/pysurf/sphSolver.py:1465-1467) keeps any
// neighbour from passing both tests.  Pairs across the seam take their separation in float64:
// their points are a period apart and their float32 difference would lose the digits the split
// keeps.  The table marks such pairs in the entry's top bit.
#pragma once

#include <type_traits>

#include "sph_internal.cuh"

namespace sph {

// The lanes of a group of T threads that serve one particle.
template <int T>
struct Group {
    int i;              // the particle (sorted slot)
    int t;              // this thread's lane in the group
    unsigned mask;      // the group's lanes in the warp
};

template <int T>
__device__ __forceinline__ Group<T> groupOf()
{
    const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    Group<T> G;
    G.i = (int)(g / T);
    G.t = (int)(g % T);
    const int lane = threadIdx.x & 31;
    G.mask = T >= 32 ? 0xFFFFFFFFu : (((1u << T) - 1u) << (lane & ~(T - 1)));
    return G;
}

// The group's sum, the same bits on every lane.
template <int T>
__device__ __forceinline__ float groupSum(float value, unsigned mask)
{
    for (int offset = T / 2; offset > 0; offset >>= 1) value += __shfl_xor_sync(mask, value, offset, T);
    return value;
}

template <int T>
__device__ __forceinline__ double groupSum(double value, unsigned mask)
{
    for (int offset = T / 2; offset > 0; offset >>= 1) value += __shfl_xor_sync(mask, value, offset, T);
    return value;
}

// Compensated accumulation (Ogita, Rump and Oishi, "Accurate sum and dot product", SIAM J. Sci.
// Comput. 26 (2005), Dot2): a running sum s with a running error c.  Each term a b enters as its
// rounded product p and the product's exact error fma(a, b, -p); Knuth's TwoSum gives the exact
// error of s + p.  Both errors gather in c, so s + c is the sum as if taken in twice the precision.
// Every rounding is an explicit intrinsic, so no contraction changes a bit.
__device__ __forceinline__ void twoSum(float a, float b, float &sum, float &error)
{
    sum = __fadd_rn(a, b);
    const float bv = __fsub_rn(sum, a);
    error = __fadd_rn(__fsub_rn(a, __fsub_rn(sum, bv)), __fsub_rn(b, bv));
}

__device__ __forceinline__ void addProduct(float a, float b, float &s, float &c)
{
    const float p = __fmul_rn(a, b);
    const float productError = __fmaf_rn(a, b, -p);
    float sum, sumError;
    twoSum(s, p, sum, sumError);
    s = sum;
    c = __fadd_rn(c, __fadd_rn(productError, sumError));
}

// The group's compensated sum, the same bits on every lane: TwoSum is exact whichever operand comes
// first, so each lane's pair of partner values combines to the same (s, c).
template <int T>
__device__ __forceinline__ float groupSumCompensated(float s, float c, unsigned mask)
{
    for (int offset = T / 2; offset > 0; offset >>= 1) {
        const float s2 = __shfl_xor_sync(mask, s, offset, T), c2 = __shfl_xor_sync(mask, c, offset, T);
        float sum, error;
        twoSum(s, s2, sum, error);
        s = sum;
        c = __fadd_rn(__fadd_rn(c, c2), error);
    }
    return __fadd_rn(s, c);
}

// The coarse test's squared distance between float32 points, and a pair's separation and squared
// distance.  Each takes its roundings from explicit intrinsics, so that the table kernel and the
// walk, compiled apart, reach the same decision on a pair at the edge of the support.  The support
// test is r^2 < (2 h)^2, so a rejected candidate takes no square root; it parts from the
// reference's r < 2 h only where the two roundings straddle 2 h, where W and grad W vanish.
template <int D>
__device__ __forceinline__ float coarseDistance2(const float pi[3], const float pj[3], float offset)
{
    const float cx = __fsub_rn(pi[0], pj[0]), cy = __fsub_rn(__fadd_rn(pi[1], offset), pj[1]);
    float r2 = __fadd_rn(__fmul_rn(cx, cx), __fmul_rn(cy, cy));
    if (D == 3) {
        const float cz = __fsub_rn(pi[2], pj[2]);
        r2 = __fadd_rn(r2, __fmul_rn(cz, cz));
    }
    return r2;
}

// d = x_i - x_j from the points and remainders (image: across the periodic seam, in float64); r^2.
// PRECISE 1 or 0 fixes the form at compile time, -1 takes it from P.precise.
template <int D, int PRECISE = -1>
__device__ __forceinline__ float separation2(const Params &P, const float pi[3], const float li[3], const float pj[3],
                                            const float lj[3], float offset, int image, double shift64, float d[3])
{
    if (PRECISE == 0 || (PRECISE < 0 && !P.precise)) {
        // separationPrecision 'float32': the points alone (src/pysurf/sphGpu.py:227-242)
        d[0] = __fsub_rn(pi[0], pj[0]);
        d[1] = __fsub_rn(__fadd_rn(pi[1], offset), pj[1]);
        d[2] = D == 3 ? __fsub_rn(pi[2], pj[2]) : 0.0f;
    } else if (!image) {
        for (int a = 0; a < D; ++a) d[a] = __fadd_rn(__fsub_rn(pi[a], pj[a]), __fsub_rn(li[a], lj[a]));
        if (D == 2) d[2] = 0.0f;
    } else {
        for (int a = 0; a < D; ++a)
            d[a] = (float)(((double)pi[a] + (double)li[a]) - ((double)pj[a] + (double)lj[a]));
        d[1] = (float)((((double)pi[1] + (double)li[1]) + shift64) - ((double)pj[1] + (double)lj[1]));
        if (D == 2) d[2] = 0.0f;
    }
    float r2 = __fadd_rn(__fmul_rn(d[0], d[0]), __fmul_rn(d[1], d[1]));
    if (D == 3) r2 = __fadd_rn(r2, __fmul_rn(d[2], d[2]));
    return r2;
}

// A pair's distance from its squared distance: the hardware reciprocal square root (about 2 ulp)
// times r^2, 0 for a coincident pair.  The support is decided on r^2, so r only enters the kernel's
// value and gradient, where its rounding is of the float32 terms' own size; continuity's and the
// correction matrix's float64 parts take one Newton step from it to float64's digits.
__device__ __forceinline__ float pairDistance(float r2)
{
    return r2 > 0.0f ? r2 * rsqrtf(r2) : 0.0f;
}

// (2 h)^2, the support test's bound.
__device__ __forceinline__ float support2(float h)
{
    const float w = __fmul_rn(2.0f, h);
    return __fmul_rn(w, w);
}

// A squared distance under which the coarse test's float32 points alone decide a pair at one
// smoothing length: a coarse r^2 below it leaves the precise r^2 (separation2, points plus
// remainders, not across the seam) below `support`.  The frame's remainders are the float32 rest
// of each float64 coordinate, |l| <= 2^-24 |x| (gatherKernel), so each axis of the separation
// moves by at most 6e-8 (|p_i| + |p_j|) over the points' difference, and a candidate under the
// bound has |p_j| <= |p_i| + 2h per axis; 1e-5 of 2h covers the roundings of both distances and of
// the bound itself (a few float32 roundings).  So a table built with it holds the same entries.
__device__ __forceinline__ float sureSupport2(float support, const float pi[3])
{
    const float s = sqrtf(support);
    const float spread = 6.0e-8f * (2.0f * (fabsf(pi[0]) + fabsf(pi[1]) + fabsf(pi[2])) + 3.0f * s) + 1.0e-37f;
    const float edge = fmaxf(s * (1.0f - 1.0e-5f) - spread, 0.0f);
    return edge * edge;
}

// The table kernels' bound for a particle of length hI at point pi: sureSupport2 of the support its
// coarse-grid candidates share.  One smoothing length: (2 h)^2.  Two grid levels: every particle on
// the coarse grid has h >= P.fineBelow, so its float32 length is at least P.hMax and each pair's
// support is at least that of (hI + P.hMax) / 2 (the roundings are monotone); the fine grid's
// candidates take the precise test.  Mixed lengths on one grid: none (0).
__device__ __forceinline__ float sureBound(const Params &P, float support, float hI, const float pi[3])
{
    if (P.mixedH) return P.levels > 1 ? sureSupport2(support2(0.5f * (hI + P.hMax)), pi) : 0.0f;
    return sureSupport2(support, pi);
}

// What a walk needs to set up each of a particle's searches: its sorted cell, point, remainder,
// length, and the periodic image's shift when it lies near the seam.
struct Origin {
    int cell;
    float hI;
    bool seam;
    double shift64;
};

// The candidates of slot i, one at a time: its table row when the row holds them all, else the
// cells of its searches.  Search s is of grid level s >> 1 (coarse, then fine when the particles
// carry two levels of smoothing length) from origin s & 1 (the particle, then its periodic image
// when it lies near the seam).
// FINE: the particles carry two levels of smoothing length (else only the coarse grid is searched).
template <int D, bool FINE>
struct Candidates {
    // table
    const int4 *column;
    int stride, count, k, step;
    int4 chunk;         // the entries still to visit of the current chunk, first in x
    int4 ahead;         // this lane's next chunk, loaded while the current one's neighbours are summed
    // walk
    bool walking;
    int search, first, nx, ny, x0, x1, y0, y1, z1, zz, yy, j, end;
    const int *cellStart;

    __device__ __forceinline__ void startRow()
    {
        const int row = first + (zz * ny + yy) * nx;
        j = __ldg(&cellStart[row + x0]) - 1;
        end = __ldg(&cellStart[row + x1 + 1]);
    }

    // Starts search s when it applies (its level is present, its image is wanted); false if not.
    __device__ __forceinline__ bool startSearch(const Params &P, const Origin &O, const float pi[3], const float li[3],
                                                int s)
    {
        const int level = FINE ? s >> 1 : 0, image = s & 1;
        if ((!FINE && s >= 2) || level >= P.levels || (image && !O.seam)) return false;
        const double pos[3] = {(double)pi[0] + (double)li[0],
                               (double)pi[1] + (double)li[1] + (image ? O.shift64 : 0.0),
                               D == 3 ? (double)pi[2] + (double)li[2] : 0.0};
        const CellBox B = cellBox(P, level, O.cell, pos, image != 0, D, searchCells(P, level, O.hI), !FINE);
        first = B.first;
        nx = B.nx;
        ny = B.ny;
        x0 = B.x0;
        x1 = B.x1;
        y0 = B.y0;
        y1 = B.y1;
        z1 = B.z1;
        zz = B.z0;
        yy = B.y0;
        search = s;
        startRow();
        return true;
    }

    // The next candidate into (jOut, imageOut, levelOut); false when there are none left.
    __device__ __forceinline__ bool next(const Params &P, const Origin &O, const float pi[3], const float li[3],
                                         int &jOut, int &imageOut, int &levelOut)
    {
        if (!walking) {
            if (k >= count) return false;
            if ((k & 3) == 0) {
                // the table streams from DRAM: the lane's next chunk is requested a chunk ahead
                chunk = ahead;
                const int next = (k >> 2) + step;
                if (4 * next < count) ahead = __ldg(column + (size_t)next * stride);
            }
            const int entry = chunk.x;
            chunk.x = chunk.y; chunk.y = chunk.z; chunk.z = chunk.w;
            // the chunk's last entry passes to this lane's next chunk
            k = (k & 3) == 3 ? k + 1 + 4 * (step - 1) : k + 1;
            jOut = entry & 0x7FFFFFFF;
            imageOut = entry < 0 ? 1 : 0;
            levelOut = 0;
            return true;
        }
        while (true) {
            if (++j < end) {
                jOut = j;
                imageOut = search & 1;
                levelOut = FINE ? search >> 1 : 0;
                return true;
            }
            if (yy < y1) {
                ++yy;
            } else if (zz < z1) {
                ++zz;
                yy = y0;
            } else {
                constexpr int searches = FINE ? 4 : 2;
                int s = search + 1;
                while (s < searches && !startSearch(P, O, pi, li, s)) ++s;
                if (s >= searches) return false;
                continue;
            }
            startRow();
        }
    }
};

// Visit the neighbours of slot i.  Every neighbour j != i with r^2 < (2 h_ij)^2 (the table's
// criterion) is counted in the walk's order; lane t of T takes those whose count k has k / 4 = t
// mod T (the table's chunks t, t + T, ...).  Of those, the visitor gets (j, d, r, h_ij, fluidJ,
// image, pb row of j, kin row of j when Visitor::kKinetic) when Visitor::accept(fluidJ), and
// r >= 1e-12 where Visitor::kSkipCoincident.
// useTable: false forces the walk (the table kernel itself).
// A boundary particle's row holds its fluid neighbours only: every sweep that reads boundary rows
// takes fluid neighbours alone (the wall pressure, continuity), except a visitor that says
// kWholeBoundaryRows (the Shepard sum, whose boundary rows the host-step call returns), which walks
// a boundary row's cells for all of them.
template <class V, class = void>
struct WholeBoundaryRows {
    static constexpr bool value = false;
};
template <class V>
struct WholeBoundaryRows<V, std::void_t<decltype(V::kWholeBoundaryRows)>> {
    static constexpr bool value = V::kWholeBoundaryRows;
};
// Whether a sweep walks boundary rows at all (kBoundaryRows); the others run fluid rows only and
// skip the row's kind at compile time.
template <class V, class = void>
struct BoundaryRows {
    static constexpr bool value = false;
};
template <class V>
struct BoundaryRows<V, std::void_t<decltype(V::kBoundaryRows)>> {
    static constexpr bool value = V::kBoundaryRows;
};

// Whether a sweep reading its particle's table row keeps the next neighbour's rows in flight while it
// sums the current one (kPipelined): one more neighbour's loads in registers, the same visits in the
// same order, so the same bits.
template <class V, class = void>
struct Pipelined {
    static constexpr bool value = false;
};
template <class V>
struct Pipelined<V, std::void_t<decltype(V::kPipelined)>> {
    static constexpr bool value = V::kPipelined;
};

// Whether a visitor reads a neighbour's aux row (3D: P2, deviation, V) or remainder row (kAuxRow,
// kLowRow): the walk loads them with the others, so the pipeline keeps them in flight too, and hands
// them to the visitor in its rowX / rowLow.
template <class V, class = void>
struct AuxRow {
    static constexpr bool value = false;
};
template <class V>
struct AuxRow<V, std::void_t<decltype(V::kAuxRow)>> {
    static constexpr bool value = V::kAuxRow;
};
template <class V, class = void>
struct LowRow {
    static constexpr bool value = false;
};
template <class V>
struct LowRow<V, std::void_t<decltype(V::kLowRow)>> {
    static constexpr bool value = V::kLowRow;
};

template <int D, class Visitor>
__device__ __forceinline__ void loadExtra(const Frame &F, int j, float4 &X, float4 &L)
{
    if constexpr (AuxRow<Visitor>::value) X = auxRow<D>(F, j);
    if constexpr (LowRow<Visitor>::value) L = __ldg(&F.low[j]);
}

// One table entry's visit: the separation from the rows already loaded, the support's r, the visitor.
template <int D, class Visitor>
__device__ __forceinline__ void visitEntry(const Params &P, const float pi[3], const float li[3], double shift64,
                                           float hI, int j, int image, const float4 &A, const float4 &B,
                                           const float4 &Kj, const float4 &X, const float4 &L, Visitor &visit)
{
    const float offset = image ? (float)shift64 : 0.0f;
    float pj[3], lj[3], d[3];
    pointIn<D>(A, pj);
    const float hs = signedLengthIn<D>(A, B);
    const bool fluidJ = hs > 0.0f;
    if (!visit.accept(fluidJ)) return;
    remainderIn<D>(A, B, lj);
    const float r2 = separation2<D>(P, pi, li, pj, lj, offset, image, shift64, d);
    const float h = P.mixedH ? 0.5f * (hI + fabsf(hs)) : P.hMax;
    const float r = pairDistance(r2);
    if (Visitor::kSkipCoincident && r < 1.0e-12f) return;
    if constexpr (AuxRow<Visitor>::value) visit.rowX = X;
    if constexpr (LowRow<Visitor>::value) visit.rowLow = L;
    visit(j, d, r, h, fluidJ, image, B, Kj);
}

template <int D, class Visitor>
__device__ __forceinline__ void loadRows(const Frame &F, int j, float4 &A, float4 &B, float4 &Kj)
{
    A = __ldg(&F.pa[j]);
    B = __ldg(&F.pb[j]);
    Kj = Visitor::kKinetic ? __ldg(&F.kin[j]) : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
}

template <int D, int T, bool FINE, class Visitor>
__device__ __forceinline__ void forEachNeighbour(const Params &P, const Frame &F, int i, int t, float hI,
                                                 Visitor &visit, bool useTable = true)
{
    const bool boundaryRow = BoundaryRows<Visitor>::value && signedLength<D>(F, i) <= 0.0f;
    const bool wholeRow = WholeBoundaryRows<Visitor>::value && boundaryRow;
    const bool fluidOnly = boundaryRow && !wholeRow;     // the row the table holds, in the walk too
    float pi[3], li[3];
    pointOf<D>(F, i, pi);
    remainderOf<D>(F, i, li);
    const float reach = P.mixedH ? hI + P.hMax : 2.0f * P.hMax;
    const float limit = kCandidateMargin * reach * reach;
    // the coarse test's bound for fine candidates: no fine neighbour lies past hI + fineMax
    const float fineReach = hI + P.fineMax;
    const float fineLimit = kCandidateMargin * fineReach * fineReach;
    Origin O;
    O.cell = 0;
    O.hI = hI;
    O.shift64 = 0.0;
    O.seam = false;
    if (D == 3 && P.period > 0.0 && (pi[1] < reach || pi[1] > P.periodF - reach)) {
        O.seam = true;
        O.shift64 = pi[1] < 0.5f * P.periodF ? P.period : -P.period;
    }
    const double shift64 = O.shift64;

    Candidates<D, FINE> C;
    const int count = useTable && P.listCap > 0 && !wholeRow ? __ldg(&F.ncount[i]) : 0;
    C.walking = wholeRow || !(useTable && P.listCap > 0 && count <= P.listCap);
    if (!C.walking) {
        C.column = reinterpret_cast<const int4 *>(F.nbr) + i;
        C.stride = P.listStride;
        C.count = count;
        C.k = 4 * t;
        if (C.k < count) C.ahead = __ldg(C.column + (size_t)t * C.stride);
        C.step = T;
    } else {
        O.cell = F.cell[i];
        C.cellStart = F.cellStart;
        C.startSearch(P, O, pi, li, 0);
    }

    int counted = 0, j = 0, image = 0, level = 0;
    if constexpr (Pipelined<Visitor>::value) {
        if (!C.walking) {
            // a software pipeline over the row: the next entry's rows load while this one is summed
            float4 A, B, Kj, X, L;
            bool more = C.next(P, O, pi, li, j, image, level);
            if (more) { loadRows<D, Visitor>(F, j, A, B, Kj); loadExtra<D, Visitor>(F, j, X, L); }
            while (more) {
                int jn = 0, imagen = 0;
                float4 An, Bn, Kn, Xn, Ln;
                more = C.next(P, O, pi, li, jn, imagen, level);
                if (more) { loadRows<D, Visitor>(F, jn, An, Bn, Kn); loadExtra<D, Visitor>(F, jn, Xn, Ln); }
                visitEntry<D>(P, pi, li, shift64, hI, j, image, A, B, Kj, X, L, visit);
                j = jn; image = imagen; A = An; B = Bn; Kj = Kn; X = Xn; L = Ln;
            }
            return;
        }
    }
    while (C.next(P, O, pi, li, j, image, level)) {
        const float offset = image ? (float)shift64 : 0.0f;     // the search's origin: particle or image
        const float4 A = __ldg(&F.pa[j]);
        float pj[3];
        pointIn<D>(A, pj);
        if (C.walking && (coarseDistance2<D>(pi, pj, offset) >= (FINE && level ? fineLimit : limit) || j == i)) continue;
        const float4 B = __ldg(&F.pb[j]);
        // the kinematic row too, with the others, when the visitor reads it
        const float4 Kj = Visitor::kKinetic ? __ldg(&F.kin[j]) : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        const float hs = signedLengthIn<D>(A, B);
        const bool fluidJ = hs > 0.0f;
        if (C.walking && fluidOnly && !fluidJ) continue;     // not in the row: not counted either
        // a lone lane may skip a rejected neighbour before its separation; a group counts every one
        if ((T == 1 || !C.walking) && !visit.accept(fluidJ)) continue;
        float lj[3];
        remainderIn<D>(A, B, lj);
        float d[3];
        const float r2 = separation2<D>(P, pi, li, pj, lj, offset, image, shift64, d);
        const float h = P.mixedH ? 0.5f * (hI + fabsf(hs)) : P.hMax;
        if (C.walking) {
            if (r2 >= support2(h)) continue;
            if (T > 1) {
                if ((counted++ >> 2) % T != t) continue;
                if (!visit.accept(fluidJ)) continue;
            }
        }
        const float r = pairDistance(r2);
        if (Visitor::kSkipCoincident && r < 1.0e-12f) continue;
        if constexpr (AuxRow<Visitor>::value) visit.rowX = auxRow<D>(F, j);
        if constexpr (LowRow<Visitor>::value) visit.rowLow = __ldg(&F.low[j]);
        visit(j, d, r, h, fluidJ, image, B, Kj);
    }
}

}  // namespace sph
