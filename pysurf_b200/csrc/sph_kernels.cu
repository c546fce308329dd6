// sph_kernels.cu -- the B200 kernels of the delta-SPH step.
//
//   cell list      keys (cell, caller index) -> LSD radix sort -> cell lower bounds -> one gather
//                  that permutes the float64 master and builds the float32 frame (with the Tait
//                  pressure and the density deviation fused in)
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

#include "sph_kernels.h"
#include "sph_sweeps.cuh"

namespace sph {

// ------------------------------------------------------------------------------------------
// Cell list
// ------------------------------------------------------------------------------------------

// Each slot's key: its cell in the high bits, the caller's index in the low bits.
__global__ void cellKeysKernel(Params P, int n, const double *x0, const double *x1, const double *x2,
                               const int *orig, int origBits, unsigned long long *keys, int *vals, const Control *ctl)
{
    if (ctl && !ctl->active) return;
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    int cx = cellCoordinate(x0[s], P.origin[0], P.cellWidth, P.nc[0]);
    int cy = cellCoordinate(x1[s], P.origin[1], P.cellWidth, P.nc[1]);
    int cz = P.dim == 3 ? cellCoordinate(x2[s], P.origin[2], P.cellWidth, P.nc[2]) : 0;
    unsigned long long c = (unsigned long long)((cz * P.nc[1] + cy) * P.nc[0] + cx);
    keys[s] = (c << origBits) | (unsigned long long)(unsigned)orig[s];
    vals[s] = s;
}

// Radix sort, 8-bit digits, least significant first.  A tile is kRadixItems keys per thread of a
// 256-thread block, taken in rounds of 256 consecutive keys so that ranks stay stable.
constexpr int kRadixThreads = 256;
constexpr int kRadixItems = 8;
constexpr int kRadixTile = kRadixThreads * kRadixItems;

__global__ void radixHistogramKernel(const unsigned long long *keys, int n, int shift, unsigned *counts, int blocks,
                                     const Control *ctl)
{
    if (ctl && !ctl->active) return;
    __shared__ unsigned hist[256];
    hist[threadIdx.x] = 0;
    __syncthreads();
    int base = blockIdx.x * kRadixTile;
    for (int k = 0; k < kRadixItems; ++k) {
        int idx = base + k * kRadixThreads + threadIdx.x;
        if (idx < n) atomicAdd(&hist[(keys[idx] >> shift) & 0xFF], 1u);
    }
    __syncthreads();
    counts[threadIdx.x * blocks + blockIdx.x] = hist[threadIdx.x];
}

// Exclusive scan of the digit-major counts in one block.
__global__ void radixScanKernel(unsigned *counts, int total, const Control *ctl)
{
    if (ctl && !ctl->active) return;
    __shared__ unsigned partial[1024];
    int t = threadIdx.x;
    int per = (total + blockDim.x - 1) / blockDim.x;
    int lo = t * per, hi = min(lo + per, total);
    unsigned sum = 0;
    for (int k = lo; k < hi; ++k) sum += counts[k];
    partial[t] = sum;
    __syncthreads();
    for (int offset = 1; offset < blockDim.x; offset <<= 1) {
        unsigned add = t >= offset ? partial[t - offset] : 0;
        __syncthreads();
        partial[t] += add;
        __syncthreads();
    }
    unsigned running = t > 0 ? partial[t - 1] : 0;
    for (int k = lo; k < hi; ++k) {
        unsigned c = counts[k];
        counts[k] = running;
        running += c;
    }
}

__global__ void radixScatterKernel(const unsigned long long *keysIn, const int *valsIn, int n, int shift,
                                   const unsigned *offsets, int blocks, unsigned long long *keysOut, int *valsOut,
                                   const Control *ctl)
{
    if (ctl && !ctl->active) return;
    __shared__ unsigned running[256];
    __shared__ unsigned warpCount[kRadixThreads / 32][256];
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    running[t] = offsets[t * blocks + blockIdx.x];
    const int base = blockIdx.x * kRadixTile;
    for (int k = 0; k < kRadixItems; ++k) {
        for (int w = 0; w < kRadixThreads / 32; ++w) warpCount[w][t] = 0;
        __syncthreads();
        int idx = base + k * kRadixThreads + t;
        bool valid = idx < n;
        unsigned long long key = valid ? keysIn[idx] : 0ull;
        int digit = valid ? (int)((key >> shift) & 0xFF) : 256 + lane;   // invalid lanes match nobody
        unsigned peers = __match_any_sync(0xFFFFFFFFu, digit);
        unsigned below = peers & ((1u << lane) - 1u);
        int rankInWarp = __popc(below);
        if (valid && below == 0) warpCount[warp][digit] = __popc(peers);
        __syncthreads();
        // thread t owns digit t: exclusive prefix over the warps, in place
        unsigned sum = 0;
        for (int w = 0; w < kRadixThreads / 32; ++w) {
            unsigned c = warpCount[w][t];
            warpCount[w][t] = sum;
            sum += c;
        }
        __syncthreads();
        if (valid) {
            unsigned pos = running[digit] + warpCount[warp][digit] + rankInWarp;
            keysOut[pos] = key;
            valsOut[pos] = valsIn[idx];
        }
        __syncthreads();
        running[t] += sum;
        __syncthreads();
    }
}

// cellStart[c] = the first sorted slot whose cell is >= c, for c = 0 .. numCells.
__global__ void cellStartKernel(const unsigned long long *sortedKeys, int n, int origBits, int numCells,
                                int *cellStart, const Control *ctl)
{
    if (ctl && !ctl->active) return;
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c > numCells) return;
    int lo = 0, hi = n;
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if ((int)(sortedKeys[mid] >> origBits) < c) lo = mid + 1; else hi = mid;
    }
    cellStart[c] = lo;
}

__device__ __forceinline__ double taitPressure(const Params &P, double rho, bool fluid)
{
    double ratio = rho / P.rho0, sq = ratio * ratio;
    double p = P.stiffness * (sq * sq * sq * ratio - 1.0);
    if (!P.tension || !fluid) p = p > 0.0 ? p : 0.0;
    return p;
}

// Permute the master into the new order (from the old buffers) and build the float32 frame:
// points and remainders (src/pysurf/sphGpu.py:1010-1019), float32 velocity and density
// (1021-1029), deviation (1031-1038) and the Tait pressure (1058-1070).
__global__ void gatherKernel(Params P, int n, const int *perm, const unsigned long long *sortedKeys, int origBits,
                             MasterView from, MasterView to, Frame F, const Control *ctl)
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
    F.cell[s] = (int)(sortedKeys[s] >> origBits);
    float hi[3], lo[3];
    for (int a = 0; a < 3; ++a) {
        hi[a] = (float)x[a];
        lo[a] = (float)(x[a] - (double)hi[a]);
    }
    float hs = fl ? h : -h;
    float p = (float)taitPressure(P, rho, fl != 0);
    float dev = (float)(rho - P.devReference);
    if (P.dim == 2) {
        F.pa[s] = make_float4(hi[0], hi[1], lo[0], lo[1]);
        F.pb[s] = make_float4(m, hs, dev, 0.0f);
        F.kin[s] = make_float4((float)v[0], (float)v[1], (float)rho, p);
    } else {
        F.pa[s] = make_float4(hi[0], hi[1], hi[2], hs);
        F.pb[s] = make_float4(lo[0], lo[1], lo[2], m);
        F.kin[s] = make_float4((float)v[0], (float)v[1], (float)v[2], (float)rho);
        F.aux[s] = make_float2(p, dev);
    }
}

// The frame's velocity, density, deviation and pressure from caller-order float64 arrays (the
// host-step sums take these from the caller each call).  Any of them may be null.
__global__ void loadFieldsKernel(Params P, int n, const int *orig, const double *velocities, const double *densities,
                                 const double *pressures, double deviationReference, Frame F)
{
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    int o = orig[s];
    float4 k = F.kin[s];
    if (velocities) {
        k.x = (float)velocities[o * P.dim];
        k.y = (float)velocities[o * P.dim + 1];
        if (P.dim == 3) k.z = (float)velocities[o * P.dim + 2];
    }
    if (P.dim == 2) {
        if (densities) {
            k.z = (float)densities[o];
            F.pb[s].z = (float)(densities[o] - deviationReference);
        }
        if (pressures) k.w = (float)pressures[o];
    } else {
        if (densities) {
            k.w = (float)densities[o];
            F.aux[s].y = (float)(densities[o] - deviationReference);
        }
        if (pressures) F.aux[s].x = (float)pressures[o];
    }
    F.kin[s] = k;
}

// ------------------------------------------------------------------------------------------
// Sweep S: Shepard filter (src/pysurf/sphGpu.py:768-802, 1040-1056)
// ------------------------------------------------------------------------------------------

template <int D, int K>
struct ShepardVisit {
    static constexpr bool kSkipCoincident = false;
    const Params &P; const Frame &F;
    float num, den;
    __device__ bool accept(bool) const { return true; }
    __device__ void operator()(int j, const float *, float r, float h, bool)
    {
        float w = kernelValue<K>(r / h, sigmaAt(P.sigmaUnit, h, D));
        float mj = massOf<D>(F, j);
        num += mj * w;
        den += mj / densityOf<D>(F, j) * w;
    }
};

// Whether this step filters: the host's flag, or every filterInterval steps after the first.
__device__ __forceinline__ bool filterDue(const Control *ctl)
{
    if (!ctl) return true;
    if (!ctl->active) return false;
    if (ctl->filterInterval > 0) return ctl->step > 0 && ctl->step % ctl->filterInterval == 0;
    return ctl->filterNow != 0;
}

template <int D, int K>
__global__ void shepardKernel(Params P, Frame F, const Control *ctl)
{
    if (!filterDue(ctl)) return;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.n) return;
    float hI = fabsf(signedLength<D>(F, i));
    float own = sigmaAt(P.sigmaUnit, hI, D);
    float mi = massOf<D>(F, i);
    ShepardVisit<D, K> visit{P, F, mi * own, mi / densityOf<D>(F, i) * own};
    walkNeighbours<D>(P, F, i, hI, visit);
    F.scalar[i] = visit.num / visit.den;
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
    F.rho[i] = rho;
    float p = (float)taitPressure(P, rho, true);
    float dev = (float)(rho - P.devReference);
    if (D == 2) {
        F.kin[i].z = filtered; F.kin[i].w = p; F.pb[i].z = dev;
    } else {
        F.kin[i].w = filtered; F.aux[i] = make_float2(p, dev);
    }
}

// ------------------------------------------------------------------------------------------
// Sweep A: extrapolated wall pressure (src/pysurf/sphSolver.py:1045-1106; sphGpu.py:804-854)
// ------------------------------------------------------------------------------------------

template <int D, int K>
struct WallVisit {
    static constexpr bool kSkipCoincident = false;
    const Params &P; const Frame &F;
    float weight, total;
    __device__ bool accept(bool fluidJ) const { return fluidJ; }
    __device__ void operator()(int j, const float *d, float r, float h, bool)
    {
        float w = kernelValue<K>(r / h, sigmaAt(P.sigmaUnit, h, D));
        float gd = P.g[0] * d[0] + P.g[1] * d[1] + (D == 3 ? P.g[2] * d[2] : 0.0f);
        weight += w;
        total += w * (pressureOf<D>(F, j) + densityOf<D>(F, j) * gd);
    }
};

// Boundary rows only write their own entries and only fluid entries are read, so the frame is
// updated in place.  writeDensity: the master float64 density takes Tait^-1(p_w) too.
template <int D, int K>
__global__ void wallPressureKernel(Params P, Frame F, const Control *ctl, int writeDensity)
{
    if (ctl && !ctl->active) return;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.n) return;
    float hs = signedLength<D>(F, i);
    if (hs > 0.0f) return;
    WallVisit<D, K> visit{P, F, 0.0f, 0.0f};
    walkNeighbours<D>(P, F, i, -hs, visit);
    float p = 0.0f;
    if (visit.weight > 0.0f) p = fmaxf(visit.total / visit.weight, 0.0f);
    double rho = P.rho0 * pow(1.0 + (double)p / P.stiffness, 1.0 / 7.0);
    float dev = (float)(rho - P.devReference);
    F.scalar[i] = p;
    if (D == 2) {
        F.kin[i].w = p;
        if (writeDensity) { F.kin[i].z = (float)rho; F.pb[i].z = dev; }
    } else {
        F.aux[i].x = p;
        if (writeDensity) { F.kin[i].w = (float)rho; F.aux[i].y = dev; }
    }
    if (writeDensity) F.rho[i] = rho;
}

// ------------------------------------------------------------------------------------------
// Sweep B: velocity gradient (src/pysurf/sphSolver.py:1151-1190; sphGpu.py:643-697),
// correction matrix (656-689; 593-641) and renormalized density gradient (691-716; 547-591),
// all from one walk over the same neighbours.
// ------------------------------------------------------------------------------------------

template <int D, int K>
struct GradientVisit {
    static constexpr bool kSkipCoincident = true;
    const Params &P; const Frame &F;
    bool wantG, wantL, wantRho;
    float vi[3], devI;
    float S[3][3], Mf[3][3], M[3][3], gsum[3];
    __device__ bool accept(bool) const { return true; }
    __device__ void operator()(int j, const float *d, float r, float h, bool fluidJ)
    {
        float slope = kernelSlope<K>(r / h, h, sigmaAt(P.sigmaUnit, h, D));
        float w = massOf<D>(F, j) / densityOf<D>(F, j) * slope / r;
        if (wantG && fluidJ) {
            float vj[3];
            velocityOf<D>(F, j, vj);
            for (int a = 0; a < D; ++a)
                for (int b = 0; b < D; ++b) {
                    S[a][b] += w * (vj[a] - vi[a]) * d[b];
                    Mf[a][b] += -w * d[a] * d[b];
                }
        }
        if (wantL)
            for (int a = 0; a < D; ++a)
                for (int b = 0; b < D; ++b) M[a][b] += -w * d[a] * d[b];
        if (wantRho) {
            float t = w * (deviationOf<D>(F, j) - devI);
            for (int a = 0; a < D; ++a) gsum[a] += t * d[a];
        }
    }
};

template <int D, int K>
__global__ void gradientKernel(Params P, Frame F, const Control *ctl, int wantG, int wantL, int wantRho, float floorDet)
{
    if (ctl && !ctl->active) return;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.n) return;
    float hs = signedLength<D>(F, i);
    float zero[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    float ident[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
    if (hs <= 0.0f) {
        if (wantG) storeMatrix<D>(F.G0, F.G1, F.G2, i, zero);
        if (wantL) storeMatrix<D>(F.L0, F.L1, F.L2, i, ident);
        if (wantRho) F.gradRho[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        return;
    }
    GradientVisit<D, K> visit{P, F, wantG != 0, wantL != 0 || wantRho != 0, wantRho != 0};
    velocityOf<D>(F, i, visit.vi);
    visit.devI = deviationOf<D>(F, i);
    for (int a = 0; a < 3; ++a) {
        visit.gsum[a] = 0.0f;
        for (int b = 0; b < 3; ++b) { visit.S[a][b] = 0.0f; visit.Mf[a][b] = 0.0f; visit.M[a][b] = 0.0f; }
    }
    walkNeighbours<D>(P, F, i, hs, visit);
    if (wantG) {
        float G[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
        if (determinant<D>(visit.Mf) >= floorDet) {
            float inv[3][3];
            inverse<D>(visit.Mf, inv);
            for (int a = 0; a < D; ++a)
                for (int b = 0; b < D; ++b) {
                    float t = 0.0f;
                    for (int c = 0; c < D; ++c) t += visit.S[a][c] * inv[c][b];
                    G[a][b] = t;
                }
        }
        storeMatrix<D>(F.G0, F.G1, F.G2, i, G);
    }
    if (wantL || wantRho) {
        float L[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
        if (determinant<D>(visit.M) >= floorDet) inverse<D>(visit.M, L);
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
// Sweep C: accelerations (src/pysurf/sphSolver.py:1122-1149, 1192-1230, 1328-1356;
// src/pysurf/sphGpu.py:303-414) with the fluid maxima (1072-1082) and the time step
// (src/pysurf/sphSolver.py:1410-1424) in the epilogue.
// ------------------------------------------------------------------------------------------

template <int D, int K>
struct MomentumVisit {
    static constexpr bool kSkipCoincident = true;
    const Params &P; const Frame &F;
    float vi[3], rhoI, own;
    float Gi[3][3];
    float total[3];
    __device__ bool accept(bool) const { return true; }
    __device__ void operator()(int j, const float *d, float r, float h, bool fluidJ)
    {
        float vj[3];
        velocityOf<D>(F, j, vj);
        float rel[3] = {vi[0] - vj[0], vi[1] - vj[1], vi[2] - vj[2]};
        float approach = rel[0] * d[0] + rel[1] * d[1] + (D == 3 ? rel[2] * d[2] : 0.0f);
        float rhoJ = densityOf<D>(F, j);
        float viscosity = 0.0f;
        if (approach < 0.0f && P.limited && fluidJ) {
            float Gj[3][3];
            loadMatrix<D>(F.G0, F.G1, F.G2, j, Gj);
            float rampI[3] = {0, 0, 0}, rampJ[3] = {0, 0, 0};
            float slopeI = 0.0f, slopeJ = 0.0f;
            for (int a = 0; a < D; ++a) {
                for (int b = 0; b < D; ++b) { rampI[a] += Gi[a][b] * d[b]; rampJ[a] += Gj[a][b] * d[b]; }
                slopeI += d[a] * rampI[a];
                slopeJ += d[a] * rampJ[a];
            }
            float limiter = 0.0f;
            if (slopeI * slopeJ > 0.0f) {
                float ratio = slopeI / slopeJ;
                limiter = fminf(1.0f, 4.0f * ratio / ((1.0f + ratio) * (1.0f + ratio)));
                float eta = r / h;
                if (eta < kCloseDistance) {
                    float fade = (eta - kCloseDistance) / kFoldWidth;
                    limiter *= expf(-fade * fade);
                }
            }
            approach = 0.0f;
            for (int a = 0; a < D; ++a) approach += (rel[a] - 0.5f * limiter * (rampI[a] + rampJ[a])) * d[a];
        }
        if (approach < 0.0f) {
            float mu = h * approach / (r * r + kViscositySoftening * h * h);
            viscosity = -P.alpha * P.c0 * mu / (0.5f * (rhoI + rhoJ));
            if (!fluidJ) viscosity *= P.boundaryFactor;
        }
        float coefficient = -(own + pressureOf<D>(F, j) / (rhoJ * rhoJ) + viscosity) * massOf<D>(F, j);
        float slope = kernelSlope<K>(r / h, h, sigmaAt(P.sigmaUnit, h, D));
        float f = coefficient * slope / r;
        for (int a = 0; a < D; ++a) total[a] += f * d[a];
    }
};

__device__ __forceinline__ double blockMax(double value, double *shared)
{
    for (int offset = 16; offset > 0; offset >>= 1) value = fmax(value, __shfl_down_sync(0xFFFFFFFFu, value, offset));
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) shared[warp] = value;
    __syncthreads();
    if (warp == 0) {
        value = lane < (int)(blockDim.x >> 5) ? shared[lane] : 0.0;
        for (int offset = 16; offset > 0; offset >>= 1) value = fmax(value, __shfl_down_sync(0xFFFFFFFFu, value, offset));
    }
    return value;
}

__device__ __forceinline__ double cflTimeStep(double h, double c0, double vmax, double amax, double cfl, double maxdt)
{
    double dt = cfl * h / (c0 + vmax);
    if (amax > 1e-12) dt = fmin(dt, cfl * sqrt(h / amax));
    return fmin(dt, maxdt);
}

template <int D, int K>
__global__ void __launch_bounds__(kBlock) momentumKernel(Params P, Frame F, Control *ctl, double *blockMaxima)
{
    __shared__ double shared[kBlock / 32];
    __shared__ bool last;
    if (ctl && !ctl->active) return;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double speed = 0.0, accel = 0.0;
    if (i < P.n) {
        float hs = signedLength<D>(F, i);
        if (hs <= 0.0f) {
            F.acc[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        } else {
            MomentumVisit<D, K> visit{P, F};
            velocityOf<D>(F, i, visit.vi);
            visit.rhoI = densityOf<D>(F, i);
            visit.own = pressureOf<D>(F, i) / (visit.rhoI * visit.rhoI);
            if (P.limited) loadMatrix<D>(F.G0, F.G1, F.G2, i, visit.Gi);
            visit.total[0] = visit.total[1] = visit.total[2] = 0.0f;
            walkNeighbours<D>(P, F, i, hs, visit);
            float a[3] = {visit.total[0] + P.g[0], visit.total[1] + P.g[1], D == 3 ? visit.total[2] + P.g[2] : 0.0f};
            F.acc[i] = make_float4(a[0], a[1], a[2], 0.0f);
            double v2 = 0.0;
            for (int c = 0; c < D; ++c) v2 += F.v[c][i] * F.v[c][i];
            speed = sqrt(v2);
            accel = (double)sqrtf(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
        }
    }
    if (!blockMaxima) return;
    double bs = blockMax(speed, shared);
    double ba = blockMax(accel, shared);
    if (threadIdx.x == 0) {
        blockMaxima[2 * blockIdx.x] = bs;
        blockMaxima[2 * blockIdx.x + 1] = ba;
        __threadfence();
        unsigned ticket = atomicAdd(&ctl->ticket, 1u);
        last = ticket == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    // The last block reduces every block's maxima (max is order-free, so this is deterministic)
    __threadfence();
    double vmax = 0.0, amax = 0.0;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) {
        vmax = fmax(vmax, ((volatile double *)blockMaxima)[2 * b]);
        amax = fmax(amax, ((volatile double *)blockMaxima)[2 * b + 1]);
    }
    vmax = blockMax(vmax, shared);
    amax = blockMax(amax, shared);
    if (threadIdx.x == 0) {
        ctl->vmax = vmax;
        ctl->amax = amax;
        ctl->ticket = 0;
        if (!ctl->hostDt) {
            double dt = cflTimeStep(ctl->hMin, ctl->soundSpeed, vmax, amax, ctl->cfl, ctl->maxTimeStep);
            if (!(dt > 0.0) || !isfinite(dt)) ctl->error |= kErrTimeStep;
            ctl->dt = dt;
        }
    }
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
    double v[3] = {0.0, 0.0, 0.0};
    float av[3] = {a.x, a.y, a.z};
    for (int c = 0; c < D; ++c) {
        v[c] = F.v[c][i] + (double)av[c] * dt;
        F.v[c][i] = v[c];
    }
    float4 k = F.kin[i];
    k.x = (float)v[0]; k.y = (float)v[1];
    if (D == 3) k.z = (float)v[2];
    F.kin[i] = k;
}

// ------------------------------------------------------------------------------------------
// Enforcement (src/pysurf/sphBoundaries.py:126-147, 295-344, 597-640; sphGpu.py:1197-1419),
// float64, applied to one fluid particle.
// ------------------------------------------------------------------------------------------

__device__ void enforceOne(const Enforcement &E, int dim, double *x, double *v)
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

// Drift (src/pysurf/sphGpu.py:1142-1186), the periodic wrap and the enforcement of one fluid slot.
__device__ __forceinline__ void driftAndEnforce(const Params &P, const Frame &F, const Enforcement &E, int i, double dt,
                                                const double *transport, Control *ctl)
{
    double x[3] = {0.0, 0.0, 0.0}, v[3] = {0.0, 0.0, 0.0};
    for (int a = 0; a < P.dim; ++a) {
        v[a] = F.v[a][i];
        x[a] = F.x[a][i] + (transport ? transport[a] : v[a]) * dt;
    }
    if (P.period > 0.0) x[1] = x[1] - P.period * floor(x[1] / P.period);
    enforceOne(E, P.dim, x, v);
    bool finite = true;
    for (int a = 0; a < P.dim; ++a) {
        F.x[a][i] = x[a];
        F.v[a][i] = v[a];
        finite = finite && isfinite(x[a]) && isfinite(v[a]);
    }
    if (!finite) atomicOr(&ctl->error, kErrNonFinite);
}

// ------------------------------------------------------------------------------------------
// Sweep D: continuity (src/pysurf/sphSolver.py:623-654, 718-822; src/pysurf/sphGpu.py:430-545)
// with the density update (1111-1140), and, when XSPH is off, the drift and the enforcement.
// ------------------------------------------------------------------------------------------

template <int D, int K>
struct ContinuityVisit {
    static constexpr bool kSkipCoincident = true;
    const Params &P; const Frame &F;
    bool boundaryI, diffuses, corrected;
    float vi[3], devI, Li[3][3], gi[3];
    float total;
    __device__ bool accept(bool fluidJ) const { return !(boundaryI && !fluidJ); }
    __device__ void operator()(int j, const float *d, float r, float h, bool fluidJ)
    {
        float slope = kernelSlope<K>(r / h, h, sigmaAt(P.sigmaUnit, h, D));
        float vj[3];
        velocityOf<D>(F, j, vj);
        float mj = massOf<D>(F, j);
        float dot = 0.0f;
        if (corrected) {
            for (int a = 0; a < D; ++a) {
                float ld = 0.0f;
                for (int b = 0; b < D; ++b) ld += Li[a][b] * d[b];
                dot += (vi[a] - vj[a]) * ld;
            }
        } else {
            for (int a = 0; a < D; ++a) dot += (vi[a] - vj[a]) * d[a];
        }
        total += mj * dot * slope / r;
        if (diffuses && fluidJ) {
            float devJ = deviationOf<D>(F, j);
            float difference = devJ - devI;
            if (P.diffusion == 2) {
                float ratio = 1.0f + 0.5f * (devI + devJ) / P.rho0F;
                float sq = ratio * ratio;
                difference -= P.rho0F * P.gravityOverSound * d[D - 1] / (sq * sq * ratio);
            } else if (P.diffusion == 3) {
                float4 gj = __ldg(&F.gradRho[j]);
                float gjv[3] = {gj.x, gj.y, gj.z};
                float t = 0.0f;
                for (int a = 0; a < D; ++a) t += (gi[a] + gjv[a]) * d[a];
                difference += 0.5f * t;
            }
            total += P.diffusionFactor * h * mj / densityOf<D>(F, j) * difference * (-slope * r)
                   / (r * r + kViscositySoftening * h * h);
        }
    }
};

// mode 0: the rate only; 1: advance the density; 2: advance, drift and enforce.
template <int D, int K>
__global__ void continuityKernel(Params P, Frame F, Control *ctl, Enforcement E, int mode)
{
    if (ctl && !ctl->active) return;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.n) return;
    float hs = signedLength<D>(F, i);
    ContinuityVisit<D, K> visit{P, F};
    visit.boundaryI = hs <= 0.0f;
    visit.diffuses = P.diffusion != 0 && !visit.boundaryI;
    visit.corrected = P.corrected && !visit.boundaryI;
    velocityOf<D>(F, i, visit.vi);
    visit.devI = deviationOf<D>(F, i);
    if (visit.corrected) loadMatrix<D>(F.L0, F.L1, F.L2, i, visit.Li);
    visit.gi[0] = visit.gi[1] = visit.gi[2] = 0.0f;
    if (visit.diffuses && P.diffusion == 3) {
        float4 g = F.gradRho[i];
        visit.gi[0] = g.x; visit.gi[1] = g.y; visit.gi[2] = g.z;
    }
    visit.total = 0.0f;
    walkNeighbours<D>(P, F, i, fabsf(hs), visit);
    float rate = visit.total;
    F.rate[i] = rate;
    if (mode == 0) return;
    double dt = ctl->dt;
    double rho = F.rho[i] + (double)rate * dt;
    bool fluid = hs > 0.0f;
    if (P.densityFloor > 0.0 && fluid) rho = fmax(rho, P.densityFloor);
    F.rho[i] = rho;
    if (!isfinite(rho)) atomicOr(&ctl->error, kErrNonFinite);
    if (mode == 2 && fluid) driftAndEnforce(P, F, E, i, dt, nullptr, ctl);
}

// ------------------------------------------------------------------------------------------
// Sweep X: XSPH (src/pysurf/sphSolver.py:1358-1377; src/pysurf/sphGpu.py:725-766) over fluid
// pairs, with the densities the step has just advanced.
// ------------------------------------------------------------------------------------------

template <int D, int K>
struct XsphVisit {
    static constexpr bool kSkipCoincident = false;
    const Params &P; const Frame &F; const float *densities;
    float vi[3], rhoI, corr[3];
    __device__ bool accept(bool fluidJ) const { return fluidJ; }
    __device__ void operator()(int j, const float *, float r, float h, bool)
    {
        float w = kernelValue<K>(r / h, sigmaAt(P.sigmaUnit, h, D));
        float rhoJ = densities ? densities[j] : densityOf<D>(F, j);
        float weight = massOf<D>(F, j) * w / (0.5f * (rhoI + rhoJ));
        float vj[3];
        velocityOf<D>(F, j, vj);
        for (int a = 0; a < D; ++a) corr[a] += weight * (vj[a] - vi[a]);
    }
};

// densities: the float32 densities the sum divides by (the scalar scratch, refreshed from the
// master after the density update).  mode 0: the transport velocity into F.vec only; 2: drift
// with it and enforce.
template <int D, int K>
__global__ void xsphKernel(Params P, Frame F, Control *ctl, Enforcement E, const float *densities, int mode)
{
    if (ctl && !ctl->active) return;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.n) return;
    float hs = signedLength<D>(F, i);
    float v[3];
    velocityOf<D>(F, i, v);
    if (hs <= 0.0f) {
        F.vec[i] = make_float4(v[0], v[1], v[2], 0.0f);
        return;
    }
    XsphVisit<D, K> visit{P, F, densities};
    visit.vi[0] = v[0]; visit.vi[1] = v[1]; visit.vi[2] = v[2];
    visit.rhoI = densities ? densities[i] : densityOf<D>(F, i);
    visit.corr[0] = visit.corr[1] = visit.corr[2] = 0.0f;
    walkNeighbours<D>(P, F, i, hs, visit);
    float t[3];
    for (int a = 0; a < 3; ++a) t[a] = v[a] + P.xsphEpsilon * visit.corr[a];
    F.vec[i] = make_float4(t[0], t[1], t[2], 0.0f);
    if (mode != 2) return;
    double transport[3] = {(double)t[0], (double)t[1], (double)t[2]};
    driftAndEnforce(P, F, E, i, ctl->dt, transport, ctl);
}

__global__ void refreshDensityKernel(int n, const double *rho, float *out)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = (float)rho[i];
}

// ------------------------------------------------------------------------------------------
// Pointwise
// ------------------------------------------------------------------------------------------

__global__ void enforceKernel(int n, int dim, MasterView M, Enforcement E)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || !M.fluid[i]) return;
    double x[3] = {0, 0, 0}, v[3] = {0, 0, 0};
    for (int a = 0; a < dim; ++a) { x[a] = M.x[a][i]; v[a] = M.v[a][i]; }
    enforceOne(E, dim, x, v);
    for (int a = 0; a < dim; ++a) { M.x[a][i] = x[a]; M.v[a][i] = v[a]; }
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
__global__ void scatterDoubleKernel(int n, int dim, const int *orig, const double *const *columns, double *out)
{
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    int o = orig[s];
    for (int a = 0; a < dim; ++a) out[o * dim + a] = columns[a][s];
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
    const int nx = P.nc[0], ny = P.nc[1], nz = P.nc[2];
    const int c = F.cell[i];
    const int cx = c % nx, cy = (c / nx) % ny, cz = c / (nx * ny);
    const int ncs = P.ncs;
    const int x0 = max(cx - ncs, 0), x1 = min(cx + ncs, nx - 1);
    const int z0 = D == 3 ? max(cz - ncs, 0) : 0, z1 = D == 3 ? min(cz + ncs, nz - 1) : 0;
    int images = 1, cyImage = cy;
    double radius = sqrt(radius2);
    if (P.period > 0.0) {
        double y = xi[1] - P.period * floor(xi[1] / P.period);
        if (y < radius || y > P.period - radius) {
            images = 2;
            cyImage = cellCoordinate(xi[1] + (y < 0.5 * P.period ? P.period : -P.period), P.origin[1], P.cellWidth, ny);
        }
    }
    long long found = 0;
    long long write = counts ? 0 : offsets[F.orig[i]];
    for (int image = 0; image < images; ++image) {
        const int yc = image == 0 ? cy : cyImage;
        const int y0 = max(yc - ncs, 0), y1 = min(yc + ncs, ny - 1);
        for (int zz = z0; zz <= z1; ++zz)
            for (int yy = y0; yy <= y1; ++yy) {
                if (image == 1 && yy >= cy - ncs && yy <= cy + ncs) continue;
                const int row = (zz * ny + yy) * nx;
                const int begin = F.cellStart[row + x0], end = F.cellStart[row + x1 + 1];
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

template <int D, int K>
static void launchSweepsT(const LaunchArgs &A, Stage stage)
{
    const Params &P = A.P;
    const Frame &F = A.F;
    int grid = blocksFor(P.n, kBlock);
    if (grid == 0) return;
    cudaStream_t st = A.stream;
    switch (stage) {
    case Stage::ShepardSum:
        shepardKernel<D, K><<<grid, kBlock, 0, st>>>(P, F, A.ctl);
        break;
    case Stage::ShepardApply:
        applyShepardKernel<D><<<grid, kBlock, 0, st>>>(P, F, A.ctl);
        break;
    case Stage::Wall:
        wallPressureKernel<D, K><<<grid, kBlock, 0, st>>>(P, F, A.ctl, A.flag);
        break;
    case Stage::Gradients:
        gradientKernel<D, K><<<grid, kBlock, 0, st>>>(P, F, A.ctl, A.wantG, A.wantL, A.wantRho, A.floorDet);
        break;
    case Stage::Momentum:
        momentumKernel<D, K><<<grid, kBlock, 0, st>>>(P, F, A.ctl, A.blockMaxima);
        break;
    case Stage::Kick:
        kickKernel<D><<<grid, kBlock, 0, st>>>(P, F, A.ctl);
        break;
    case Stage::Continuity:
        continuityKernel<D, K><<<grid, kBlock, 0, st>>>(P, F, A.ctl, A.E, A.flag);
        break;
    case Stage::Xsph:
        xsphKernel<D, K><<<grid, kBlock, 0, st>>>(P, F, A.ctl, A.E, A.densities, A.flag);
        break;
    }
}

void launchStage(const LaunchArgs &A, Stage stage)
{
    int D = A.P.dim, K = A.P.kind;
    if (D == 2 && K == 0) launchSweepsT<2, 0>(A, stage);
    else if (D == 2 && K == 1) launchSweepsT<2, 1>(A, stage);
    else if (D == 3 && K == 0) launchSweepsT<3, 0>(A, stage);
    else launchSweepsT<3, 1>(A, stage);
}

void launchCellKeys(const Params &P, int n, const MasterView &M, int origBits, unsigned long long *keys, int *vals,
                    const Control *ctl, cudaStream_t st)
{
    if (n == 0) return;
    cellKeysKernel<<<blocksFor(n, 256), 256, 0, st>>>(P, n, M.x[0], M.x[1], M.x[2], M.orig, origBits, keys, vals, ctl);
}

int radixBlocks(int n) { return blocksFor(n, kRadixTile); }

void launchRadixSort(int n, int bits, unsigned long long *keys, int *vals, unsigned long long *keysAlt, int *valsAlt,
                     unsigned *counts, const Control *ctl, cudaStream_t st, unsigned long long **keysOut,
                     int **valsOut)
{
    int blocks = radixBlocks(n);
    unsigned long long *kin = keys, *kout = keysAlt;
    int *vin = vals, *vout = valsAlt;
    for (int shift = 0; shift < bits && n > 0; shift += 8) {
        radixHistogramKernel<<<blocks, kRadixThreads, 0, st>>>(kin, n, shift, counts, blocks, ctl);
        radixScanKernel<<<1, 1024, 0, st>>>(counts, 256 * blocks, ctl);
        radixScatterKernel<<<blocks, kRadixThreads, 0, st>>>(kin, vin, n, shift, counts, blocks, kout, vout, ctl);
        unsigned long long *tk = kin; kin = kout; kout = tk;
        int *tv = vin; vin = vout; vout = tv;
    }
    *keysOut = kin;
    *valsOut = vin;
}

void launchCellStart(const unsigned long long *sortedKeys, int n, int origBits, int numCells, int *cellStart,
                     const Control *ctl, cudaStream_t st)
{
    cellStartKernel<<<blocksFor(numCells + 1, 256), 256, 0, st>>>(sortedKeys, n, origBits, numCells, cellStart, ctl);
}

void launchGather(const Params &P, int n, const int *perm, const unsigned long long *sortedKeys, int origBits,
                  const MasterView &from, const MasterView &to, const Frame &F, const Control *ctl, cudaStream_t st)
{
    if (n == 0) return;
    gatherKernel<<<blocksFor(n, 256), 256, 0, st>>>(P, n, perm, sortedKeys, origBits, from, to, F, ctl);
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

void launchEnforce(int n, int dim, const MasterView &M, const Enforcement &E, cudaStream_t st)
{
    if (n == 0 || E.kind == 0) return;
    enforceKernel<<<blocksFor(n, 256), 256, 0, st>>>(n, dim, M, E);
}

void launchRefreshDensity(int n, const double *rho, float *out, cudaStream_t st)
{
    if (n == 0) return;
    refreshDensityKernel<<<blocksFor(n, 256), 256, 0, st>>>(n, rho, out);
}

void launchScatterDouble(int n, int dim, const int *orig, const double *const *columns, double *out, cudaStream_t st)
{
    if (n == 0) return;
    scatterDoubleKernel<<<blocksFor(n, 256), 256, 0, st>>>(n, dim, orig, columns, out);
}

void launchScatterFloat4(int n, int dim, const int *orig, const float4 *values, double *out, cudaStream_t st)
{
    if (n == 0) return;
    scatterFloat4Kernel<<<blocksFor(n, 256), 256, 0, st>>>(n, dim, orig, values, out);
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
