// sph_sweeps.cuh -- the neighbour walk every sweep shares.
//
// One thread per sorted particle.  A particle's neighbours lie in the cells within +-ncs of its
// own along each axis; cells are numbered x fastest, so each (y, z) row of the stencil is one
// contiguous run of the sorted order, [cellStart[first], cellStart[last + 1]).  Threads of a
// warp hold neighbouring particles of the same few cells, walk the same runs in step, and read
// the same neighbour records, which the L1 cache serves to all of them at once.
//
// Candidates are tested on their float32 points first (the reference's coarse test,
// src/pysurf/sphGpu.py:330-336), and only survivors take the precise separation
// (hi_i - hi_j) + (lo_i - lo_j).
//
// A periodic y axis (3D) is searched a second time from the particle's image across the seam
// when it lies within its reach of the seam (src/pysurf/sphGpu.py:206-225).  Each walk tests its
// candidates against its own origin (the particle, or its image), and a period longer than twice
// the reach (the solver requires twice the support, src/pysurf/sphSolver.py:1465-1467) keeps any
// neighbour from passing both tests.  Pairs across the seam take their separation in float64:
// their points are a period apart and their float32 difference would lose the digits the split
// keeps.
#pragma once

#include "sph_internal.cuh"

namespace sph {

// Walk the neighbours of slot i.  The visitor gets (j, d[3], r, h_ij, fluidJ) for every j != i
// with r < 2 h_ij, and r >= 1e-12 when Visitor::kSkipCoincident.  Visitor::accept(fluidJ) is
// asked first and may skip a neighbour before its separation is taken.
template <int D, class Visitor>
__device__ __forceinline__ void walkNeighbours(const Params &P, const Frame &F, int i, float hI, Visitor &visit)
{
    float pi[3], li[3];
    pointOf<D>(F, i, pi);
    remainderOf<D>(F, i, li);
    const float reach = P.mixedH ? hI + P.hMax : 2.0f * P.hMax;
    const float limit = kCandidateMargin * reach * reach;
    const int nx = P.nc[0], ny = P.nc[1], nz = P.nc[2];
    const int c = F.cell[i];
    const int cx = c % nx, cy = (c / nx) % ny, cz = c / (nx * ny);
    const int ncs = P.ncs;
    const int x0 = max(cx - ncs, 0), x1 = min(cx + ncs, nx - 1);
    const int z0 = D == 3 ? max(cz - ncs, 0) : 0, z1 = D == 3 ? min(cz + ncs, nz - 1) : 0;

    // image search: the particle's image across the periodic seam, if within reach of it
    int images = 1;
    float shift = 0.0f;
    double shift64 = 0.0;
    int cyImage = cy;
    if (D == 3 && P.period > 0.0) {
        if (pi[1] < reach || pi[1] > P.periodF - reach) {
            images = 2;
            shift64 = pi[1] < 0.5f * P.periodF ? P.period : -P.period;
            shift = (float)shift64;
            double y = (double)pi[1] + (double)li[1] + shift64;
            cyImage = cellCoordinate(y, P.origin[1], P.cellWidth, ny);
        }
    }

    for (int image = 0; image < images; ++image) {
        const int yc = image == 0 ? cy : cyImage;
        const float offset = image == 0 ? 0.0f : shift;     // the walk's origin: the particle, or its image
        const int y0 = max(yc - ncs, 0), y1 = min(yc + ncs, ny - 1);
        for (int zz = z0; zz <= z1; ++zz) {
            for (int yy = y0; yy <= y1; ++yy) {
                const int row = (zz * ny + yy) * nx;
                const int begin = __ldg(&F.cellStart[row + x0]);
                const int end = __ldg(&F.cellStart[row + x1 + 1]);
                for (int j = begin; j < end; ++j) {
                    float pj[3];
                    pointOf<D>(F, j, pj);
                    float cxv = pi[0] - pj[0];
                    float cyv = (pi[1] + offset) - pj[1];
                    float czv = D == 3 ? pi[2] - pj[2] : 0.0f;
                    float coarse = cxv * cxv + cyv * cyv + czv * czv;
                    if (coarse >= limit || j == i) continue;
                    const float hs = signedLength<D>(F, j);
                    const bool fluidJ = hs > 0.0f;
                    if (!visit.accept(fluidJ)) continue;
                    float lj[3];
                    remainderOf<D>(F, j, lj);
                    float d[3];
                    if (!P.precise) {
                        // separationPrecision 'float32': the points alone (src/pysurf/sphGpu.py:227-242)
                        d[0] = cxv; d[1] = cyv; d[2] = czv;
                    } else if (image == 0) {
                        d[0] = (pi[0] - pj[0]) + (li[0] - lj[0]);
                        d[1] = (pi[1] - pj[1]) + (li[1] - lj[1]);
                        d[2] = D == 3 ? (pi[2] - pj[2]) + (li[2] - lj[2]) : 0.0f;
                    } else {
                        for (int a = 0; a < D; ++a)
                            d[a] = (float)(((double)pi[a] + (double)li[a]) - ((double)pj[a] + (double)lj[a]));
                        d[1] = (float)((((double)pi[1] + (double)li[1]) + shift64) - ((double)pj[1] + (double)lj[1]));
                    }
                    const float r2 = d[0] * d[0] + d[1] * d[1] + (D == 3 ? d[2] * d[2] : 0.0f);
                    const float r = sqrtf(r2);
                    const float h = P.mixedH ? 0.5f * (hI + fabsf(hs)) : P.hMax;
                    if (r >= 2.0f * h) continue;
                    if (Visitor::kSkipCoincident && r < 1.0e-12f) continue;
                    visit(j, d, r, h, fluidJ);
                }
            }
        }
    }
}

}  // namespace sph
