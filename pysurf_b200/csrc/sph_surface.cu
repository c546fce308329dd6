// sph_surface.cu -- the breaking tracker's reads of the fluid, and the crest zone, on the device.
//
// A tracker update needs three small things from the fluid's positions (in 3D, a section's: the
// fluid in a band across the tank, read in its (x, z) plane), not the positions themselves: each column's highest particle (the free surface, src/pysurf/waveBreaking.py:129-162),
// the cells a particle marks in the window ahead of the crest (the face lean, 559-634), and the x
// of the particles on the bed's water sheet (the waterline, 636-656).  Each kernel does the
// reference's float64 arithmetic term by term, with explicitly rounded operations where a fused
// multiply-add could otherwise change a bit, so the host reads the same values it would from
// pulled positions.
#include <math.h>

#include "sph_kernels.h"

namespace sph {

// A double's bits reordered so that unsigned order is the doubles' order (0: below every double).
__device__ __forceinline__ unsigned long long orderedBits(double v)
{
    const unsigned long long u = (unsigned long long)__double_as_longlong(v);
    return (u >> 63) ? ~u : (u | 0x8000000000000000ull);
}

__device__ __forceinline__ double fromOrderedBits(unsigned long long o)
{
    const unsigned long long u = (o >> 63) ? (o & 0x7FFFFFFFFFFFFFFFull) : ~o;
    return __longlong_as_double((long long)u);
}

// A section's band across the tank (3D): the fluid with |y - center| < half, the comparison the
// reference's section mask takes in float64 (src/pysurf/BreakingWave3D.py:461-468); y null takes all.
__device__ __forceinline__ bool inBand(const Band &B, int s)
{
    return !B.y || fabs(__dsub_rn(B.y[s], B.center)) < B.half;
}

// tops[c] = the largest height of a fluid particle whose column floor((x - x0) / width) is c.
__global__ void surfaceTopKernel(int n, const double *x, const double *z, const uint8_t *fluid, Band band, double x0,
                                 double width, long long count, unsigned long long *tops)
{
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n || !fluid[s] || !inBand(band, s)) return;
    const double c = floor((x[s] - x0) / width);
    if (!(c >= 0.0 && c < (double)count)) return;
    atomicMax(&tops[(long long)c], orderedBits(z[s]));
}

__global__ void surfaceTopDecodeKernel(long long count, const unsigned long long *tops, double *out)
{
    long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= count) return;
    out[c] = tops[c] ? fromOrderedBits(tops[c]) : -INFINITY;
}

// The face window's cells: a fluid particle with lowX <= x < highX and z > lowZ marks the cells
// (band0 + db, column0 + dc), db, dc in {0, 1}, column0 = floor((x - half - start) / spacing),
// band0 = floor((z - half - base) / spacing), those inside columns x bands.
__global__ void faceCellsKernel(int n, const double *x, const double *z, const uint8_t *fluid, Band band, double lowX,
                                double highX, double lowZ, double half, double start, double base, double spacing,
                                long long columns, long long bands, uint8_t *marks)
{
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n || !fluid[s] || !inBand(band, s)) return;
    const double xv = x[s], zv = z[s];
    if (!(xv >= lowX && xv < highX && zv > lowZ)) return;
    const double c0 = floor(__dsub_rn(__dsub_rn(xv, half), start) / spacing);
    const double b0 = floor(__dsub_rn(__dsub_rn(zv, half), base) / spacing);
    for (int db = 0; db < 2; ++db)
        for (int dc = 0; dc < 2; ++dc) {
            const double c = c0 + dc, b = b0 + db;
            if (c >= 0.0 && c < (double)columns && b >= 0.0 && b < (double)bands)
                marks[(long long)b * columns + (long long)c] = 1;
        }
}

// numpy.interp(x, bedX, bedZ): the end values outside, the vertex value on a vertex, else
// slope (x - x_j) + z_j with the slope (z_j+1 - z_j) / (x_j+1 - x_j).
__device__ __forceinline__ double bedElevation(double v, const double *bx, const double *bz, int m)
{
    if (isnan(v)) return v;
    if (v <= bx[0]) return bz[0];
    if (v >= bx[m - 1]) return bz[m - 1];
    int lo = 0, hi = m - 1;                 // bx[lo] <= v < bx[hi]
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (bx[mid] <= v) lo = mid; else hi = mid;
    }
    if (v == bx[lo]) return bz[lo];
    const double slope = __dsub_rn(bz[lo + 1], bz[lo]) / __dsub_rn(bx[lo + 1], bx[lo]);
    return __dadd_rn(__dmul_rn(slope, __dsub_rn(v, bx[lo])), bz[lo]);
}

// The x of every fluid particle less than wetHeight above the bed, in no set order.
__global__ void bedSheetKernel(int n, const double *x, const double *z, const uint8_t *fluid, Band band,
                               const double *bx, const double *bz, int m, double wetHeight, double *out, int *count)
{
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n || !fluid[s] || !inBand(band, s)) return;
    const double xv = x[s];
    if (__dsub_rn(z[s], bedElevation(xv, bx, bz, m)) < wetHeight) out[atomicAdd(count, 1)] = xv;
}

// The crest zone: tops[cy * nx + cx] = the highest fluid particle (vertical axis dim - 1) of the
// column (cx, cy) of width `width` from (x0, y0) (cy = 0 in 2D).
__global__ void columnTopsKernel(int n, MasterView M, int dim, double x0, double y0, double width, long long nx,
                                 long long ny, unsigned long long *tops)
{
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n || !M.fluid[s]) return;
    const double cx = floor((M.x[0][s] - x0) / width);
    const double cy = dim == 3 ? floor((M.x[1][s] - y0) / width) : 0.0;
    if (!(cx >= 0.0 && cx < (double)nx && cy >= 0.0 && cy < (double)ny)) return;
    atomicMax(&tops[(long long)cy * nx + (long long)cx], orderedBits(M.x[dim - 1][s]));
}

// chosen[caller index] = 1 for a fluid particle of at least minMass (not yet split) whose column's
// top stands above `threshold`.
__global__ void crestZoneKernel(int n, MasterView M, int dim, double x0, double y0, double width, long long nx,
                                long long ny, const unsigned long long *tops, double threshold, double minMass,
                                uint8_t *chosen)
{
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    bool zone = false;
    if (M.fluid[s] && M.m[s] >= minMass) {
        const double cx = floor((M.x[0][s] - x0) / width);
        const double cy = dim == 3 ? floor((M.x[1][s] - y0) / width) : 0.0;
        if (cx >= 0.0 && cx < (double)nx && cy >= 0.0 && cy < (double)ny) {
            const unsigned long long top = tops[(long long)cy * nx + (long long)cx];
            zone = top != 0 && fromOrderedBits(top) > threshold;
        }
    }
    chosen[M.orig[s]] = zone ? 1 : 0;
}

static inline int blocksFor(long long n, int block) { return (int)((n + block - 1) / block); }

void launchCrestZone(int n, const MasterView &M, int dim, double x0, double y0, double width, long long nx,
                     long long ny, unsigned long long *tops, double threshold, double minMass, uint8_t *chosen,
                     cudaStream_t st)
{
    cudaMemsetAsync(tops, 0, sizeof(unsigned long long) * nx * ny, st);
    if (n == 0) return;
    columnTopsKernel<<<blocksFor(n, 256), 256, 0, st>>>(n, M, dim, x0, y0, width, nx, ny, tops);
    crestZoneKernel<<<blocksFor(n, 256), 256, 0, st>>>(n, M, dim, x0, y0, width, nx, ny, tops, threshold, minMass,
                                                       chosen);
}

void launchSurfaceTops(int n, const MasterView &M, int vertical, const Band &band, double x0, double width,
                       long long count, unsigned long long *scratch, double *out, cudaStream_t st)
{
    cudaMemsetAsync(scratch, 0, sizeof(unsigned long long) * count, st);
    if (n > 0)
        surfaceTopKernel<<<blocksFor(n, 256), 256, 0, st>>>(n, M.x[0], M.x[vertical], M.fluid, band, x0, width, count,
                                                            scratch);
    surfaceTopDecodeKernel<<<blocksFor(count, 256), 256, 0, st>>>(count, scratch, out);
}

void launchFaceCells(int n, const MasterView &M, int vertical, const Band &band, double lowX, double highX,
                     double lowZ, double half, double start, double base, double spacing, long long columns,
                     long long bands, uint8_t *marks, cudaStream_t st)
{
    cudaMemsetAsync(marks, 0, (size_t)columns * (size_t)bands, st);
    if (n > 0)
        faceCellsKernel<<<blocksFor(n, 256), 256, 0, st>>>(n, M.x[0], M.x[vertical], M.fluid, band, lowX, highX, lowZ,
                                                           half, start, base, spacing, columns, bands, marks);
}

void launchBedSheet(int n, const MasterView &M, int vertical, const Band &band, const double *bx, const double *bz,
                    int m, double wetHeight, double *out, int *count, cudaStream_t st)
{
    cudaMemsetAsync(count, 0, sizeof(int), st);
    if (n > 0)
        bedSheetKernel<<<blocksFor(n, 256), 256, 0, st>>>(n, M.x[0], M.x[vertical], M.fluid, band, bx, bz, m,
                                                          wetHeight, out, count);
}

}  // namespace sph
