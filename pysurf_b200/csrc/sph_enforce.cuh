// sph_enforce.cuh -- the boundary enforcement of one fluid particle, float64.
#pragma once

#include "sph_kernels.h"

namespace sph {

// ------------------------------------------------------------------------------------------
// Enforcement (src/pysurf/sphBoundaries.py:126-147, 295-344, 597-640; sphGpu.py:1197-1419),
// float64, applied to one fluid particle.
// ------------------------------------------------------------------------------------------

__device__ __forceinline__ void enforceOne(const Enforcement &E, int dim, double *x, double *v)
{
    const double zero = 0.0, one = 1.0;
    if (E.kind == 1) {
        for (int a = 0; a < dim; ++a) {
            if (x[a] < E.lower[a]) { x[a] = E.lower[a]; v[a] = fmax(v[a], zero); }
            if (a < dim - 1 || !E.openTop)
                if (x[a] > E.upper[a]) { x[a] = E.upper[a]; v[a] = fmin(v[a], zero); }
        }
    } else if (E.kind == 2) {
        const int vert = dim - 1;
        int lo = 0, hi = E.bedCount - 1;
        while (hi - lo > 1) {
            int mid = (lo + hi) / 2;
            if (E.bedX[mid] <= x[0]) lo = mid; else hi = mid;
        }
        double run = E.bedX[lo + 1] - E.bedX[lo], rise = E.bedZ[lo + 1] - E.bedZ[lo];
        double share = fmin(fmax((x[0] - E.bedX[lo]) / run, zero), one);
        double bed = E.bedZ[lo] + share * rise;
        if (x[vert] < bed + E.clearance) {
            x[vert] = bed + E.clearance;
            double slope = rise / run, length = sqrt(one + slope * slope);
            double nx = -slope / length, nz = one / length;
            double inward = v[0] * nx + v[vert] * nz;
            if (inward < zero) { v[0] = v[0] - inward * nx; v[vert] = v[vert] - inward * nz; }
        }
        if (E.sideWalls) {
            if (x[1] < E.clearance) { x[1] = E.clearance; v[1] = fmax(v[1], zero); }
            if (x[1] > E.width - E.clearance) { x[1] = E.width - E.clearance; v[1] = fmin(v[1], zero); }
        }
        if (E.offshoreWall && x[0] < E.wallX + E.clearance) {
            x[0] = E.wallX + E.clearance;
            v[0] = fmax(v[0], E.pistonSpeed);
        }
        if (x[0] > E.endLimit) { x[0] = E.endLimit; v[0] = fmin(v[0], zero); }
    } else if (E.kind == 3) {
        const int nxT = E.tableNx, nyT = E.tableNy;
        double rawX = (x[0] - E.originX) / E.stepX, rawY = (x[1] - E.originY) / E.stepY;
        double fx = fmin(fmax(rawX, zero), (double)(nxT - 1)), fy = fmin(fmax(rawY, zero), (double)(nyT - 1));
        int ix = (int)floor(fx), iy = (int)floor(fy);
        double u = fx - (double)ix, w = fy - (double)iy;
        double wx[4], wy[4], sx[4], sy[4];
        double u2 = u * u, u3 = u2 * u, w2 = w * w, w3 = w2 * w;
        wx[0] = -0.5 * u3 + u2 - 0.5 * u; wx[1] = 1.5 * u3 - 2.5 * u2 + 1.0;
        wx[2] = -1.5 * u3 + 2.0 * u2 + 0.5 * u; wx[3] = 0.5 * u3 - 0.5 * u2;
        wy[0] = -0.5 * w3 + w2 - 0.5 * w; wy[1] = 1.5 * w3 - 2.5 * w2 + 1.0;
        wy[2] = -1.5 * w3 + 2.0 * w2 + 0.5 * w; wy[3] = 0.5 * w3 - 0.5 * w2;
        sx[0] = -1.5 * u2 + 2.0 * u - 0.5; sx[1] = 4.5 * u2 - 5.0 * u; sx[2] = -4.5 * u2 + 4.0 * u + 0.5;
        sx[3] = 1.5 * u2 - u;
        sy[0] = -1.5 * w2 + 2.0 * w - 0.5; sy[1] = 4.5 * w2 - 5.0 * w; sy[2] = -4.5 * w2 + 4.0 * w + 0.5;
        sy[3] = 1.5 * w2 - w;
        double bed = 0.0, slopeX = 0.0, slopeY = 0.0;
        for (int a = 0; a < 4; ++a) {
            int row = clampi(iy - 1 + a, 0, nyT - 1);
            double along = 0.0, alongSlope = 0.0;
            for (int b = 0; b < 4; ++b) {
                double value = E.table[row * nxT + clampi(ix - 1 + b, 0, nxT - 1)];
                along += wx[b] * value;
                alongSlope += sx[b] * value;
            }
            bed += wy[a] * along;
            slopeX += wy[a] * alongSlope;
            slopeY += sy[a] * along;
        }
        slopeX = slopeX / E.stepX;
        slopeY = slopeY / E.stepY;
        if (rawX < zero || rawX > (double)(nxT - 1)) slopeX = zero;
        if (rawY < zero || rawY > (double)(nyT - 1)) slopeY = zero;
        if (x[2] < bed + E.clearance) {
            x[2] = bed + E.clearance;
            double length = sqrt(slopeX * slopeX + slopeY * slopeY + one);
            double n0 = -slopeX / length, n1 = -slopeY / length, n2 = one / length;
            double inward = v[0] * n0 + v[1] * n1 + v[2] * n2;
            if (inward < zero) { v[0] -= inward * n0; v[1] -= inward * n1; v[2] -= inward * n2; }
        }
        if (x[1] < E.lowY) { x[1] = E.lowY; v[1] = fmax(v[1], zero); }
        if (x[1] > E.highY) { x[1] = E.highY; v[1] = fmin(v[1], zero); }
        if (E.offshoreWall && x[0] < E.lowX) { x[0] = E.lowX; v[0] = fmax(v[0], zero); }
        if (x[0] > E.highX) { x[0] = E.highX; v[0] = fmin(v[0], zero); }
    }
}

// enforceOne on fluid slot i; with the energy budget on, the enforcement's change of kinetic and
// potential energy, m ((|v'|^2 - |v|^2) / 2 - g . (x' - x)), goes to the clamp's column
// (src/pysurf/sphGpu.py:1189-1230).
__device__ __forceinline__ void enforceTracked(const Params &P, const Frame &F, const Enforcement &E, int dim, int i,
                                               double *x, double *v)
{
    if (!P.budget) {
        enforceOne(E, dim, x, v);
        return;
    }
    const double x0[3] = {x[0], x[1], x[2]}, v0[3] = {v[0], v[1], v[2]};
    enforceOne(E, dim, x, v);
    double kinetic = 0.0, lift = 0.0;
    for (int a = 0; a < dim; ++a) {
        kinetic += v[a] * v[a] - v0[a] * v0[a];
        lift += P.gravity64[a] * (x[a] - x0[a]);
    }
    addEnergy(P, F, i, kClamp, F.m[i] * (0.5 * kinetic - lift));
}

}  // namespace sph
