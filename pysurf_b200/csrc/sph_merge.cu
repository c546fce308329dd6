// sph_merge.cu -- merging split particles back (src/pysurf/sphRefinement.py:192-311), on the device.
//
// The chosen split fluid particles of each level are binned into cubes the size of a particle one
// level coarser; in every cube holding 2^dim or more, the 2^dim nearest its centre (ties to the lower
// caller index) merge into one, and a second pass on a grid moved half a cube takes up most of the
// rest.  The merged particle takes the group's mass, centre of mass, momentum and volume, the
// mass-weighted pressure and acceleration, and its members' mean smoothing length over the split's
// ratio; it takes the place of the member with the lowest caller index, and fluid from the end of
// the caller's order fills the places the others leave among the boundary's, so every boundary
// particle keeps its index.
//
// Here the grouping is two stable radix sorts (by distance to the cube's centre, then by cube), so
// each cube's members come in the reference's order; the compaction is a handful of scans in caller
// order; and one gather moves the master into its new, shorter order.  Nothing goes to the host
// but the counts that size the next launch.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>
#include <cub/device/device_select.cuh>
#include <climits>
#include <math.h>

#include <vector>

#include "sph_kernels.h"

namespace sph {

namespace {

constexpr int kMaxMergeLevel = 16;
constexpr int kMaxGroup = 8;        // 2^dim members a group, 3D

inline int blocks(long long n, int block) { return (int)((n + block - 1) / block); }

// Each caller index's slot; the level (times split) of each chosen split fluid particle, 0 for
// any other; how many of each level; the boundary's last caller index.
__global__ void levelsKernel(int n, int dim, MasterView M, const uint8_t *mask, double referenceMass, int *slotOf,
                             int *level, int *levelCount, int *lastBoundary)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const int o = M.orig[s];
    slotOf[o] = s;
    int chosen = 0;
    if (M.fluid[s]) {
        // src/pysurf/sphRefinement.py:123-134: rint(log2(m_ref / m) / dim)
        const double k = rint(log2(referenceMass / M.m[s]) / dim);
        if (mask[o] && k >= 1.0 && k <= (double)kMaxMergeLevel) chosen = (int)k;
    } else {
        atomicMax(lastBoundary, o);
    }
    level[o] = chosen;
    if (chosen) atomicAdd(&levelCount[chosen], 1);
}

__global__ void freeKernel(int n, const int *level, const uint8_t *taken, int which, uint8_t *flag)
{
    const int o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o < n) flag[o] = level[o] == which && !taken[o];
}

// For free particle k (caller index F[k]): its cube's integer coordinates, floor(x / cell + offset),
// its squared distance from the cube's centre (numpy's order: (u - floor u - 1/2)^2 summed over the
// axes in turn), and the coordinates' bounds.
__global__ void keysKernel(int nf, int dim, const int *F, const int *slotOf, MasterView M, double cell, double offset,
                           long long *keys, unsigned long long *distance, int *iota, long long *bounds)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nf) return;
    const int s = slotOf[F[k]];
    double d2 = 0.0;
    for (int a = 0; a < dim; ++a) {
        const double u = __dadd_rn(__ddiv_rn(M.x[a][s], cell), offset);
        const double f = floor(u);
        const double t = __dsub_rn(__dsub_rn(u, f), 0.5);
        d2 = __dadd_rn(d2, __dmul_rn(t, t));
        const long long key = (long long)f;
        keys[(size_t)k * 3 + a] = key;
        atomicMin(&bounds[a], key);
        atomicMax(&bounds[3 + a], key);
    }
    distance[k] = (unsigned long long)__double_as_longlong(d2);    // non-negative: bits order as values
    iota[k] = k;
}

// The cube's index as numpy ravels it (C order over the bounds' box), for the k in distance order.
__global__ void flatKernel(int nf, int dim, const long long *keys, const long long *bounds, const int *order,
                           unsigned long long *flat)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= nf) return;
    const int k = order[p];
    unsigned long long f = 0;
    for (int a = 0; a < dim; ++a)
        f = f * (unsigned long long)(bounds[3 + a] - bounds[a] + 1) + (unsigned long long)(keys[(size_t)k * 3 + a] - bounds[a]);
    flat[p] = f;
}

// In the sorted order (cube, distance, index): each particle's rank in its cube, -1 unless it is
// one of its cube's first `size` and the cube holds `size` or more; head marks a group's first.
__global__ void runsKernel(int nf, const unsigned long long *flat, int size, int *rank, int *head)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= nf) return;
    const unsigned long long f = flat[p];
    int start = p;
    while (start > 0 && flat[start - 1] == f) --start;
    int end = p + 1;
    while (end < nf && flat[end] == f) ++end;
    const int r = p - start;
    const bool take = r < size && end - start >= size;
    rank[p] = take ? r : -1;
    head[p] = take && r == 0 ? 1 : 0;
}

__global__ void recordKernel(int nf, const int *order, const int *F, const int *rank, const int *groupIndex, int base,
                             int size, int *members, uint8_t *taken)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= nf) return;
    const int r = rank[p];
    if (r < 0) return;
    const int g = base + groupIndex[p - r];
    const int o = F[order[p]];
    members[(size_t)g * size + r] = o;
    taken[o] = 1;
}

// One group's members in caller order (np.sort, axis 1), in place; all but the first go.
__global__ void orderGroupsKernel(int groups, int size, int *members, uint8_t *gone)
{
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= groups) return;
    int o[kMaxGroup];
    for (int k = 0; k < size; ++k) o[k] = members[(size_t)g * size + k];
    for (int k = 1; k < size; ++k)
        for (int q = k; q > 0 && o[q - 1] > o[q]; --q) { const int t = o[q]; o[q] = o[q - 1]; o[q - 1] = t; }
    for (int k = 0; k < size; ++k) members[(size_t)g * size + k] = o[k];
    for (int k = 1; k < size; ++k) gone[o[k]] = 1;
}

// One group (its members in caller order): the merged particle into the first's slot.
__global__ void groupsKernel(int groups, int size, int dim, const int *members, const int *slotOf, MasterView M,
                             float4 *acc, double lengthRatio, double *removed, float *mergedPressure,
                             const float *pres, double *energy, int energyStride, int energyTerms)
{
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= groups) return;
    int o[kMaxGroup], s[kMaxGroup];
    for (int k = 0; k < size; ++k) o[k] = members[(size_t)g * size + k];
    for (int k = 0; k < size; ++k) s[k] = slotOf[o[k]];
    double total = 0.0, volume = 0.0, length = 0.0;
    for (int k = 0; k < size; ++k) {
        const double m = M.m[s[k]];
        total += m;
        volume += m / M.rho[s[k]];
        length += M.h[s[k]];
    }
    double x[3] = {0, 0, 0}, v[3] = {0, 0, 0}, a[3] = {0, 0, 0}, p = 0.0;
    for (int k = 0; k < size; ++k) {
        const double w = M.m[s[k]] / total;
        const float4 ak = acc[s[k]];
        const float ac[3] = {ak.x, ak.y, ak.z};
        for (int d = 0; d < dim; ++d) {
            x[d] += w * M.x[d][s[k]];
            v[d] += w * M.v[d][s[k]];
            a[d] += w * (double)ac[d];
        }
        p += w * (double)pres[s[k]];
    }
    // the kinetic energy of the members' motion about the group's centre of mass
    double spread = 0.0;
    for (int k = 0; k < size; ++k) {
        double r2 = 0.0;
        for (int d = 0; d < dim; ++d) {
            const double r = M.v[d][s[k]] - v[d];
            r2 += r * r;
        }
        spread += M.m[s[k]] * r2;
    }
    removed[g] = 0.5 * spread;
    const int first = s[0];
    for (int d = 0; d < dim; ++d) {
        M.x[d][first] = x[d];
        M.v[d][first] = v[d];
    }
    M.rho[first] = total / volume;
    M.m[first] = total;
    M.h[first] = length / size / lengthRatio;
    acc[first] = make_float4((float)a[0], (float)a[1], (float)a[2], 0.0f);
    mergedPressure[o[0]] = (float)p;
    if (energy) {
        // the members' running energy totals go with the merged particle
        for (int t = 0; t < energyTerms; ++t) {
            double sum = energy[(size_t)t * energyStride + o[0]];
            for (int k = 1; k < size; ++k) {
                sum += energy[(size_t)t * energyStride + o[k]];
                energy[(size_t)t * energyStride + o[k]] = 0.0;
            }
            energy[(size_t)t * energyStride + o[0]] = sum;
        }
    }
}

// The places a merge leaves among the boundary's (holes), and the surviving fluid after the
// boundary's last place (the tail).
__global__ void holesKernel(int n, const uint8_t *gone, const int *lastBoundary, int *hole, int *tail)
{
    const int o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= n) return;
    const int last = *lastBoundary;
    hole[o] = gone[o] && o <= last ? 1 : 0;
    tail[o] = !gone[o] && o > last ? 1 : 0;
}

// The last H of the tail move, the k-th of them into the k-th hole; what survives where.
__global__ void moversKernel(int n, const uint8_t *gone, const int *hole, const int *holeRank, const int *tail,
                             const int *tailRank, int holes, int tails, int *holeOf, int *moverOf, int *alive)
{
    const int o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= n) return;
    if (hole[o]) holeOf[holeRank[o]] = o;
    const bool mover = tail[o] && tailRank[o] >= tails - holes;
    if (mover) moverOf[tailRank[o] - (tails - holes)] = o;
    alive[o] = (!gone[o] && !mover) || hole[o] ? 1 : 0;
}

// Each caller index's index after the merge (-1: merged away), and the source of each index after.
__global__ void renumberKernel(int n, const int *hole, const int *holeRank, const int *moverOf, const int *alive,
                               const int *newIndex, int *newCaller, long long *source)
{
    const int o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= n || !alive[o]) return;
    const int from = hole[o] ? moverOf[holeRank[o]] : o;
    newCaller[from] = newIndex[o];
    source[newIndex[o]] = from;
}

__global__ void survivorsKernel(int n, const int *orig, const int *newCaller, uint8_t *flag)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < n) flag[s] = newCaller[orig[s]] >= 0;
}

// After the gather into the new order: the new caller indices, the merged pressures and the
// accelerations in the new order.
__global__ void afterGatherKernel(int n, int *orig, const int *newCaller, const float *mergedPressure, float *pres,
                                  const int *perm, const float4 *accOld, float4 *accNew)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int o = orig[k];
    const float p = mergedPressure[o];
    if (!isnan(p)) pres[k] = p;
    orig[k] = newCaller[o];
    accNew[k] = accOld[perm[k]];
}

__global__ void energyRowsKernel(int n, const int *newCaller, const double *old, double *energy, int stride, int terms)
{
    const int o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= n) return;
    const int to = newCaller[o];
    if (to < 0) return;
    for (int t = 0; t < terms; ++t) energy[(size_t)t * stride + to] = old[(size_t)t * stride + o];
}

__global__ void iotaKernel(int n, int *out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = i;
}

__global__ void fillFloatKernel(int n, float *out, float value)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = value;
}

// Device scratch that frees itself.
struct Scratch {
    std::vector<void *> held;
    ~Scratch() { for (void *p : held) cudaFree(p); }
    template <typename T>
    T *get(size_t count)
    {
        void *p = nullptr;
        if (cudaMalloc(&p, sizeof(T) * (count ? count : 1)) != cudaSuccess) return nullptr;
        held.push_back(p);
        return static_cast<T *>(p);
    }
};

#define MERGE_TRY(expr)                                                                                              \
    do {                                                                                                             \
        cudaError_t e_ = (expr);                                                                                     \
        if (e_ != cudaSuccess) { out.error = cudaGetErrorString(e_); return -1; }                                    \
    } while (0)
#define MERGE_NEED(ptr)                                                                                              \
    do {                                                                                                             \
        if (!(ptr)) { out.error = "out of device memory for the merge"; return -1; }                                 \
    } while (0)

template <typename T>
int download(T *host, const T *device, size_t count, cudaStream_t st)
{
    if (cudaMemcpyAsync(host, device, sizeof(T) * count, cudaMemcpyDeviceToHost, st) != cudaSuccess) return -1;
    return cudaStreamSynchronize(st) == cudaSuccess ? 0 : -1;
}

}  // namespace

int runMerge(const MergeArgs &in, MergeResultDevice &out)
{
    const int n = in.n, dim = in.dim, size = 1 << dim;
    cudaStream_t st = in.stream;
    out.groups = 0;
    out.removedEnergy = 0.0;
    out.newCount = n;
    Scratch scratch;
    int *slotOf = scratch.get<int>(n), *level = scratch.get<int>(n);
    int *levelCount = scratch.get<int>(kMaxMergeLevel + 1), *lastBoundary = scratch.get<int>(1);
    uint8_t *taken = scratch.get<uint8_t>(n), *flag = scratch.get<uint8_t>(n), *gone = scratch.get<uint8_t>(n);
    int *callers = scratch.get<int>(n);        // 0 .. n - 1, the indices the selections pick from
    MERGE_NEED(slotOf && level && levelCount && lastBoundary && taken && flag && gone && callers);
    iotaKernel<<<blocks(n, 256), 256, 0, st>>>(n, callers);
    MERGE_TRY(cudaMemsetAsync(levelCount, 0, sizeof(int) * (kMaxMergeLevel + 1), st));
    const int minusOne = -1;
    MERGE_TRY(cudaMemcpyAsync(lastBoundary, &minusOne, sizeof(int), cudaMemcpyHostToDevice, st));
    MERGE_TRY(cudaMemsetAsync(taken, 0, n, st));
    MERGE_TRY(cudaMemsetAsync(gone, 0, n, st));
    levelsKernel<<<blocks(n, 256), 256, 0, st>>>(n, dim, in.master, in.mask, in.referenceMass, slotOf, level,
                                                  levelCount, lastBoundary);
    MERGE_TRY(cudaGetLastError());
    int counts[kMaxMergeLevel + 1];
    if (download(counts, levelCount, kMaxMergeLevel + 1, st)) { out.error = "merge: level counts"; return -1; }
    long long eligible = 0;
    for (int l = 1; l <= kMaxMergeLevel; ++l) eligible += counts[l];
    if (eligible < size) return 0;

    // the groups, level by level, each in two passes
    int *F = scratch.get<int>(eligible), *selected = scratch.get<int>(1);
    long long *keys = scratch.get<long long>(eligible * 3), *bounds = scratch.get<long long>(6);
    unsigned long long *distance = scratch.get<unsigned long long>(eligible),
                       *distanceSorted = scratch.get<unsigned long long>(eligible),
                       *flat = scratch.get<unsigned long long>(eligible),
                       *flatSorted = scratch.get<unsigned long long>(eligible);
    int *iota = scratch.get<int>(eligible), *byDistance = scratch.get<int>(eligible), *order = scratch.get<int>(eligible);
    int *rank = scratch.get<int>(eligible), *head = scratch.get<int>(eligible), *groupIndex = scratch.get<int>(eligible);
    int *members = scratch.get<int>(eligible + size);
    MERGE_NEED(F && selected && keys && bounds && distance && distanceSorted && flat && flatSorted && iota &&
               byDistance && order && rank && head && groupIndex && members);
    // CUB's scratch, sized for the largest of its calls
    size_t tempBytes = 0, need = 0;
    cub::DeviceSelect::Flagged(nullptr, need, callers, flag, F, selected, n, st);
    tempBytes = need > tempBytes ? need : tempBytes;
    cub::DeviceRadixSort::SortPairs(nullptr, need, distance, distanceSorted, iota, byDistance, (int)eligible, 0, 64, st);
    tempBytes = need > tempBytes ? need : tempBytes;
    cub::DeviceScan::ExclusiveSum(nullptr, need, head, groupIndex, n, st);
    tempBytes = need > tempBytes ? need : tempBytes;
    void *temp = scratch.get<unsigned char>(tempBytes);
    MERGE_NEED(temp);
    const double offsets[2] = {0.0, 0.5};
    int groups = 0;
    for (int l = 1; l <= kMaxMergeLevel; ++l) {
        if (counts[l] == 0) continue;
        // cubes the size of a particle one level coarser
        const double cell = pow(in.referenceMass / pow((double)size, (double)(l - 1)) / in.referenceDensity, 1.0 / dim);
        for (int pass = 0; pass < 2; ++pass) {
            freeKernel<<<blocks(n, 256), 256, 0, st>>>(n, level, taken, l, flag);
            size_t bytes = tempBytes;
            MERGE_TRY(cub::DeviceSelect::Flagged(temp, bytes, callers, flag, F, selected, n,
                                                 st));
            int nf = 0;
            if (download(&nf, selected, 1, st)) { out.error = "merge: free count"; return -1; }
            if (nf < size) break;
            const long long far[6] = {LLONG_MAX, LLONG_MAX, LLONG_MAX, LLONG_MIN, LLONG_MIN, LLONG_MIN};
            MERGE_TRY(cudaMemcpyAsync(bounds, far, sizeof(far), cudaMemcpyHostToDevice, st));
            keysKernel<<<blocks(nf, 256), 256, 0, st>>>(nf, dim, F, slotOf, in.master, cell, offsets[pass], keys,
                                                         distance, iota, bounds);
            // (cube, distance, index): by distance first, then a stable sort by cube
            bytes = tempBytes;
            MERGE_TRY(cub::DeviceRadixSort::SortPairs(temp, bytes, distance, distanceSorted, iota, byDistance, nf, 0, 64,
                                                      st));
            flatKernel<<<blocks(nf, 256), 256, 0, st>>>(nf, dim, keys, bounds, byDistance, flat);
            bytes = tempBytes;
            MERGE_TRY(cub::DeviceRadixSort::SortPairs(temp, bytes, flat, flatSorted, byDistance, order, nf, 0, 64, st));
            runsKernel<<<blocks(nf, 256), 256, 0, st>>>(nf, flatSorted, size, rank, head);
            bytes = tempBytes;
            MERGE_TRY(cub::DeviceScan::ExclusiveSum(temp, bytes, head, groupIndex, nf, st));
            int lastIndex = 0, lastHead = 0;
            if (download(&lastIndex, groupIndex + nf - 1, 1, st) || download(&lastHead, head + nf - 1, 1, st)) {
                out.error = "merge: group count";
                return -1;
            }
            recordKernel<<<blocks(nf, 256), 256, 0, st>>>(nf, order, F, rank, groupIndex, groups, size, members, taken);
            MERGE_TRY(cudaGetLastError());
            groups += lastIndex + lastHead;
        }
    }
    if (groups == 0) return 0;

    // everything the rest needs, before anything of the state changes: a failure from here to the
    // merge itself (no memory, too few fluid particles to fill the boundary's places) leaves it whole
    double *removed = scratch.get<double>(groups);
    double *energyOld = in.energy ? scratch.get<double>((size_t)in.energyTerms * in.energyStride) : nullptr;
    float *mergedPressure = scratch.get<float>(n);
    int *hole = scratch.get<int>(n), *holeRank = scratch.get<int>(n), *tail = scratch.get<int>(n),
        *tailRank = scratch.get<int>(n), *alive = scratch.get<int>(n), *newIndex = scratch.get<int>(n),
        *newCaller = scratch.get<int>(n), *holeOf = scratch.get<int>(n), *moverOf = scratch.get<int>(n);
    int *perm = scratch.get<int>(n), *kept = scratch.get<int>(1);
    float4 *accNew = scratch.get<float4>(n);
    MERGE_NEED(removed && (energyOld || !in.energy) && mergedPressure && hole && holeRank && tail && tailRank &&
               alive && newIndex && newCaller && holeOf && moverOf && perm && kept && accNew);
    orderGroupsKernel<<<blocks(groups, 128), 128, 0, st>>>(groups, size, members, gone);

    // the compaction in caller order
    holesKernel<<<blocks(n, 256), 256, 0, st>>>(n, gone, lastBoundary, hole, tail);
    size_t bytes = tempBytes;
    MERGE_TRY(cub::DeviceScan::ExclusiveSum(temp, bytes, hole, holeRank, n, st));
    bytes = tempBytes;
    MERGE_TRY(cub::DeviceScan::ExclusiveSum(temp, bytes, tail, tailRank, n, st));
    int ends[4];
    if (download(&ends[0], holeRank + n - 1, 1, st) || download(&ends[1], hole + n - 1, 1, st) ||
        download(&ends[2], tailRank + n - 1, 1, st) || download(&ends[3], tail + n - 1, 1, st)) {
        out.error = "merge: hole counts";
        return -1;
    }
    const int holes = ends[0] + ends[1], tails = ends[2] + ends[3];
    if (tails < holes) {
        out.error = "too few fluid particles follow the boundary to fill the places a merge leaves among it";
        return -1;
    }
    moversKernel<<<blocks(n, 256), 256, 0, st>>>(n, gone, hole, holeRank, tail, tailRank, holes, tails, holeOf, moverOf,
                                                  alive);
    bytes = tempBytes;
    MERGE_TRY(cub::DeviceScan::ExclusiveSum(temp, bytes, alive, newIndex, n, st));
    int lastNew = 0, lastAlive = 0;
    if (download(&lastNew, newIndex + n - 1, 1, st) || download(&lastAlive, alive + n - 1, 1, st)) {
        out.error = "merge: survivor count";
        return -1;
    }
    const int newCount = lastNew + lastAlive;
    MERGE_TRY(cudaMemsetAsync(newCaller, 0xFF, sizeof(int) * n, st));
    renumberKernel<<<blocks(n, 256), 256, 0, st>>>(n, hole, holeRank, moverOf, alive, newIndex, newCaller, in.source);

    // the merged particles, into their groups' first slots
    fillFloatKernel<<<blocks(n, 256), 256, 0, st>>>(n, mergedPressure, nanf(""));
    groupsKernel<<<blocks(groups, 128), 128, 0, st>>>(groups, size, dim, members, slotOf, in.master, in.acc,
                                                       in.lengthRatio, removed, mergedPressure, in.pres,
                                                       in.energy, in.energyStride, in.energyTerms);
    MERGE_TRY(cudaGetLastError());
    std::vector<double> perGroup(groups);
    if (download(perGroup.data(), removed, groups, st)) { out.error = "merge: removed energy"; return -1; }
    for (double e : perGroup) out.removedEnergy += e;

    // the master into its new order: the surviving slots, in slot order, gathered
    survivorsKernel<<<blocks(n, 256), 256, 0, st>>>(n, in.master.orig, newCaller, flag);
    bytes = tempBytes;
    MERGE_TRY(cub::DeviceSelect::Flagged(temp, bytes, callers, flag, perm, kept, n, st));
    Params P = in.params;
    P.n = newCount;
    launchGather(P, newCount, perm, in.master, in.next, in.nextFrame, nullptr, st);
    afterGatherKernel<<<blocks(newCount, 256), 256, 0, st>>>(newCount, in.next.orig, newCaller, mergedPressure,
                                                              in.nextFrame.pres, perm, in.acc, accNew);
    MERGE_TRY(cudaMemcpyAsync(in.acc, accNew, sizeof(float4) * newCount, cudaMemcpyDeviceToDevice, st));
    if (in.energy) {
        MERGE_TRY(cudaMemcpyAsync(energyOld, in.energy, sizeof(double) * in.energyTerms * in.energyStride,
                                  cudaMemcpyDeviceToDevice, st));
        MERGE_TRY(cudaMemsetAsync(in.energy, 0, sizeof(double) * in.energyTerms * in.energyStride, st));
        energyRowsKernel<<<blocks(n, 256), 256, 0, st>>>(n, newCaller, energyOld, in.energy, in.energyStride,
                                                          in.energyTerms);
    }
    MERGE_TRY(cudaGetLastError());
    MERGE_TRY(cudaStreamSynchronize(st));
    out.groups = groups;
    out.newCount = newCount;
    return 0;
}

}  // namespace sph
