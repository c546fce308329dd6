// sph_noalloc.cu -- the fluid maxima and the CFL time step, for callers that cannot allocate.
//
// Some callers of this library cannot call cudaMalloc: an application whose device memory is
// all owned by its own pool allocator (a framework's caching allocator, say) and which forbids
// any allocation outside it, or a control loop that must not enter the CUDA allocator while it
// runs, because an allocation can wait on the device and take unbounded time.  Those callers
// own their buffers and pass them in.  sph_fluid_maxima_noalloc serves them: it is the reduction
// the momentum sweep ends with (the largest fluid speed and acceleration, then the time step of
// src/pysurf/sphSolver.py:1410-1424), over caller-owned device arrays, and it allocates nothing.
//
// Its scratch (one partial maximum per tile of particles, and the counter that finds the last
// tile) is the file-scope array below, a fixed 64 KiB plus 256 bytes that every GPU which loads
// this library holds until the process exits.  It caps a call at kMaxTiles tiles of kTile
// particles, 16,777,216 particles; larger calls are refused before anything is launched.
//
// Every call shares the array and leaves its contents behind; the counter is cleared at the
// start of each call.  Calls that overlap on the GPU (on two streams, or from two threads) race
// on the array and must not be made.
//
// The first call on each device looks the array's device address up (cudaGetSymbolAddress, with
// that device current) and keeps it; make that first call before any stream capture begins.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <mutex>
#include <string>

#include "../../include/pysurf_b200.h"

namespace sph {
void recordError(const std::string &message);
}

namespace {

constexpr int kThreads = 256;
constexpr int kItems = 16;
constexpr int kTile = kThreads * kItems;            // particles a block reduces
constexpr int kMaxTiles = 4096;                     // partials the scratch holds
constexpr long long kMaxParticles = (long long)kTile * kMaxTiles;
constexpr int kCounterDoubles = 32;                 // the first 256 bytes hold the tile counter

// [0, 256 B): the counter of finished tiles (unsigned int); then (speed, acceleration) per tile.
static __device__ __align__(256) double gMaximaScratch[kCounterDoubles + 2 * kMaxTiles];

int refuse(int code, const std::string &message)
{
    sph::recordError(message);      // what sph_last_error() reports
    return code;
}

__device__ __forceinline__ double warpMax(double value)
{
    for (int offset = 16; offset > 0; offset >>= 1) value = fmax(value, __shfl_down_sync(0xFFFFFFFFu, value, offset));
    return value;
}

__device__ __forceinline__ double blockMaxOf(double value, double *shared)
{
    value = warpMax(value);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) shared[warp] = value;
    __syncthreads();
    value = lane < kThreads / 32 ? shared[lane] : 0.0;
    if (warp == 0) value = warpMax(value);
    return value;
}

// Each block reduces one tile; the block that finishes last reduces the partials and writes
// (max |v|, max |a|, dt) to `out`.  |v| is taken in float64 and |a| as a float32 length, as the
// reference's device maxima are (src/pysurf/sphGpu.py:1072-1082).
__global__ void __launch_bounds__(kThreads)
maximaNoAllocKernel(const double *velocities, const double *accelerations, const uint8_t *fluid, int n, int dim,
                    double h, double c0, double cfl, double maxdt, double *scratch, double *out)
{
    __shared__ double shared[kThreads / 32];
    __shared__ bool last;
    unsigned int *counter = reinterpret_cast<unsigned int *>(scratch);
    double *partial = scratch + kCounterDoubles;
    double speed = 0.0, accel = 0.0;
    const int base = blockIdx.x * kTile;
    for (int k = 0; k < kItems; ++k) {
        const int i = base + k * kThreads + threadIdx.x;
        if (i >= n || !fluid[i]) continue;
        double v2 = 0.0;
        float a[3] = {0.0f, 0.0f, 0.0f};
        for (int c = 0; c < dim; ++c) {
            const double vc = velocities[(size_t)i * dim + c];
            v2 += vc * vc;
            a[c] = (float)accelerations[(size_t)i * dim + c];
        }
        speed = fmax(speed, sqrt(v2));
        accel = fmax(accel, (double)sqrtf(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]));
    }
    speed = blockMaxOf(speed, shared);
    accel = blockMaxOf(accel, shared);
    if (threadIdx.x == 0) {
        partial[2 * blockIdx.x] = speed;
        partial[2 * blockIdx.x + 1] = accel;
        __threadfence();
        last = atomicAdd(counter, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    double vmax = 0.0, amax = 0.0;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += kThreads) {
        vmax = fmax(vmax, ((volatile double *)partial)[2 * b]);
        amax = fmax(amax, ((volatile double *)partial)[2 * b + 1]);
    }
    vmax = blockMaxOf(vmax, shared);
    amax = blockMaxOf(amax, shared);
    if (threadIdx.x == 0) {
        double dt = cfl * h / (c0 + vmax);
        if (amax > 1e-12) dt = fmin(dt, cfl * sqrt(h / amax));
        out[0] = vmax;
        out[1] = amax;
        out[2] = fmin(dt, maxdt);
    }
}

// The scratch's device address on each device, looked up once per device with it current.
std::mutex setupLock;
double *scratchAddress[64] = {};

int scratchFor(int device, double **address)
{
    if (device < 0 || device >= 64) return refuse(SPH_ERR_INVALID, "device index out of range");
    std::lock_guard<std::mutex> guard(setupLock);
    if (!scratchAddress[device]) {
        void *p = nullptr;
        cudaError_t err = cudaGetSymbolAddress(&p, gMaximaScratch);
        if (err != cudaSuccess)
            return refuse(SPH_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(err));
        scratchAddress[device] = static_cast<double *>(p);
    }
    *address = scratchAddress[device];
    return SPH_OK;
}

}  // namespace

extern "C" {

int sph_fluid_maxima_noalloc(const double *velocities, const double *accelerations, const uint8_t *is_fluid,
                             int64_t n, int dimensions, double smoothing_length, double sound_speed, double cfl,
                             double max_time_step, double *out, void *stream)
{
    if (!velocities || !accelerations || !is_fluid || !out) return refuse(SPH_ERR_INVALID, "null device pointer");
    if (dimensions != 2 && dimensions != 3) return refuse(SPH_ERR_INVALID, "dimensions must be 2 or 3");
    if (n < 1) return refuse(SPH_ERR_INVALID, "at least one particle is needed");
    if (n > kMaxParticles)
        return refuse(SPH_ERR_INVALID, std::to_string(n) + " particles exceed the " + std::to_string(kMaxParticles) +
                                           " this entry point's fixed scratch holds");
    if (!(smoothing_length > 0.0) || !(sound_speed > 0.0) || !(cfl > 0.0) || !(max_time_step > 0.0))
        return refuse(SPH_ERR_INVALID, "h, c0, the CFL number and the largest step must be positive");
    int device = 0;
    cudaError_t err = cudaGetDevice(&device);
    if (err != cudaSuccess) return refuse(SPH_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(err));
    double *scratch = nullptr;
    int status = scratchFor(device, &scratch);
    if (status != SPH_OK) return status;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // the tile counter must start at zero; the partials are all written before they are read
    err = cudaMemsetAsync(scratch, 0, kCounterDoubles * sizeof(double), s);
    if (err != cudaSuccess) return refuse(SPH_ERR_CUDA, std::string("cudaMemsetAsync: ") + cudaGetErrorString(err));
    const int tiles = (int)((n + kTile - 1) / kTile);
    maximaNoAllocKernel<<<tiles, kThreads, 0, s>>>(velocities, accelerations, is_fluid, (int)n, dimensions,
                                                   smoothing_length, sound_speed, cfl, max_time_step, scratch, out);
    err = cudaGetLastError();
    if (err != cudaSuccess) return refuse(SPH_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(err));
    return SPH_OK;
}

}  // extern "C"
