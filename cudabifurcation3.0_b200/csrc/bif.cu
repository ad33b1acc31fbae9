// Bifurcation diagrams and peak-based maps: integrate -> peaks -> KDE / DBSCAN.
//
// Reference pipeline (per chunk of points, three kernels and two HBM round trips
// of the full trajectory): calculateDiscreteModelCUDA writes record doubles per
// point (cudaLibrary.cu:78-117), peakFinderCUDA scans them (:220-284), then
// kdeCUDA (:356-441) or dbscanCUDA (:457-624) reduce each point.
//
// Here one fused kernel does all of it.  Each lane of a warp owns one point and
// keeps the ODE state in registers; the recorded variable is never stored: a
// streaming state machine reproduces peakFinder exactly (see PeakStream) and
// only the peaks (and intervals) go to a per-warp scratch slice in HBM.  Then
// the warp reduces its 32 points one after the other, cooperatively:
//   KDE    -- lanes take 32 consecutive sample positions; each sums its kernel
//             terms over the peaks in the reference's peak order (double sum of
//             FP32 expf), so the sums are bit-identical; the plateau state
//             machine then runs over the 32 sums via shuffles.
//   DBSCAN -- labels and the reference's neighbour "stack" become two bitsets
//             in shared memory; the inner neighbour loop over k is a ballot
//             (its iterations are independent in the reference), popcount
//             updates the neighbour counter.
// Results leave as one coalesced 32-wide store per warp.
#include <type_traits>

#include "bif_device.cuh"

namespace cbf {

namespace {

constexpr int kBifWarps = 4;
constexpr int kBifThreads = kBifWarps * 32;
// Peak slots per lane in the first pass of a KDE/DBSCAN/Ostrovsky map.  The
// reference's bound min(maxAmountOfPeaks, record/2) can be 10 000 and more;
// sizing every lane's scratch for it leaves room for 2-3 blocks per SM.  Points
// with more peaks than this (but not more than maxAmountOfPeaks, which only
// need the count) are listed and recomputed in a second pass at full capacity.
constexpr int kFirstPassPeaks = 1024;

// Sort buffer of the DBSCAN neighbour scans (keys per warp, a power of two
// >= 32): only where the peak capacity is at most kFirstPassPeaks, so that a
// block's shared memory stays at most 18 KB and eight blocks fit an SM.
__host__ __device__ inline int bif_sort_cap(int task, int peakCap)
{
    return task_with_intervals(task) && peakCap <= kFirstPassPeaks ? dbscan_sort_cap(peakCap) : 0;
}

// Points whose first-pass peak list was truncated: grid index and output slot.
struct Overflow {
    long long* g;
    long long* p;
    unsigned long long* count;
};

// ---------------------------------------------------------------------------
template <class S, int TASK>
__global__ void __launch_bounds__(kBifThreads) bif_kernel(const DevJob J, void* __restrict__ d_out,
                                                          int* __restrict__ d_aux,
                                                          double* scrPeaks,
                                                          double* scrInt,
                                                          int bitWords, int sortCap,
                                                          int* __restrict__ err, const Overflow ov)
{
    extern __shared__ unsigned smem[];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const long long warpId = (long long)blockIdx.x * kBifWarps + wib;
    const long long nWarps = (long long)gridDim.x * kBifWarps;
    const long long nTiles = (J.nPoints + 31) / 32;
    const int cap = J.peakCap;
    unsigned* L = smem + (size_t)wib * dbscan_warp_words(bitWords, sortCap);
    unsigned* Sb = L + bitWords;
    const DbscanSort so = dbscan_sort_area(L, bitWords, sortCap);

    for (long long tile = warpId; tile < nTiles; tile += nWarps) {
        const long long p = tile * 32 + lane;
        const bool valid = p < J.nPoints;
        const long long g = grid_index(J, p);

        if (TASK == CBF_TASK_PEAKS) {
            if (valid) {
                double* pk = (double*)d_out + p * (long long)cap;
                d_aux[p] = integrate_point<S, TASK>(J, g, pk, nullptr, cap, nullptr, nullptr);
            }
            continue;
        }
        if (TASK == CBF_TASK_TRAJECTORY) {
            if (valid) {
                double* tr = (double*)d_out + p * (long long)cap;
                integrate_point<S, TASK>(J, g, nullptr, nullptr, 0, tr, d_aux + p);
            }
            continue;
        }

        const long long slot0 = warpId * 32;
        double* myPk = scrPeaks + (slot0 + lane) * (long long)cap;
        double* myIv = task_with_intervals(TASK) ? scrInt + (slot0 + lane) * (long long)cap : nullptr;
        int n = 0, div = 0;
        OstrovskyFlags of;
        of.init(J.ostThr);
        if (valid) n = integrate_point<S, TASK>(J, g, myPk, myIv, cap, nullptr, &div, &of);
        // A truncated peak list whose result needs every peak goes to the second pass.
        const bool over = valid && ov.count && n > cap && n <= J.maxPeaks;
        if (over) {
            const unsigned long long k = atomicAdd(ov.count, 1ull);
            ov.g[k] = g;
            ov.p[k] = p;
        }
        __syncwarp();

        int res = 0;
        const int live = (int)min(32ll, J.nPoints - tile * 32);
        for (int j = 0; j < live; ++j) {
            const int nj = __shfl_sync(kFull, over ? 0 : n, j);
            const double* pk = scrPeaks + (slot0 + j) * (long long)cap;
            int r;
            if (TASK == CBF_TASK_KDE) {
                r = kde_warp(J, pk, nj, lane);
            } else {
                const double* iv = scrInt + (slot0 + j) * (long long)cap;
                r = dbscan_warp(J, pk, iv, nj, lane, L, Sb, err, so);
            }
            if (lane == j) res = r;
        }
        if (valid && !over) {
            if (TASK == CBF_TASK_OSTROVSKY)
                ((double*)d_out)[p] = ostrovsky_value(n, div != 0, of, res);
            else
                ((int*)d_out)[p] = res;
        }
        __syncwarp();
    }
}

template <class T>
__global__ void scatter_kernel(const T* __restrict__ src, const long long* __restrict__ slot, long long n,
                               T* __restrict__ dst)
{
    const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) dst[slot[k]] = src[k];
}

// One launch of the fused kernel over the job's points (synchronises `s`).
template <class S, int TASK>
cudaError_t bif_pass(const DevJob& J, void* d_out, int* d_aux, const Overflow& ov, cudaStream_t s)
{
    const long long nTiles = (J.nPoints + 31) / 32;
    if (nTiles == 0) return cudaSuccess;
    const bool needScratch = (TASK == CBF_TASK_KDE || task_with_intervals(TASK));
    const int bitWords = task_with_intervals(TASK) ? (J.peakCap + 31) / 32 : 0;
    const int sortCap = bif_sort_cap(TASK, J.peakCap);
    const size_t smemBytes = (size_t)kBifWarps * dbscan_warp_words(bitWords, sortCap) * sizeof(unsigned);

    auto kern = bif_kernel<S, TASK>;
    cudaError_t e;
    if (smemBytes > 48 * 1024) {
        e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smemBytes);
        if (e != cudaSuccess) return e;
    }
    int dev = 0, sms = 0, perSm = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, kern, kBifThreads, smemBytes)) != cudaSuccess)
        return e;
    if (perSm < 1) return cudaErrorInvalidConfiguration;

    long long blocks = (nTiles + kBifWarps - 1) / kBifWarps;
    const long long resident = (long long)sms * perSm;
    if (blocks > resident) blocks = resident;

    double* scrPeaks = nullptr;
    double* scrInt = nullptr;
    int* err = nullptr;
    if (needScratch) {
        // Per-warp scratch: 32 points x cap peaks (x2 with intervals).  Bound it.
        const size_t perBlock = (size_t)kBifThreads * J.peakCap * sizeof(double) *
                                (task_with_intervals(TASK) ? 2 : 1);
        size_t freeB = 0, totalB = 0;
        if ((e = cudaMemGetInfo(&freeB, &totalB)) != cudaSuccess) return e;
        size_t budget = freeB / 4;
        const size_t cap8 = (size_t)8 << 30;
        if (budget > cap8) budget = cap8;
        long long fit = (long long)(budget / perBlock);
        if (fit < 1) fit = 1;
        if (blocks > fit) blocks = fit;
        const size_t bytes = (size_t)blocks * perBlock;
        if ((e = cudaMallocAsync((void**)&scrPeaks, bytes + 256, s)) != cudaSuccess) return e;
        if (task_with_intervals(TASK)) scrInt = scrPeaks + (size_t)blocks * kBifThreads * J.peakCap;
        err = (int*)((char*)scrPeaks + bytes);
        if ((e = cudaMemsetAsync(err, 0, sizeof(int), s)) != cudaSuccess) return e;
    }
    kern<<<(unsigned)blocks, kBifThreads, smemBytes, s>>>(J, d_out, d_aux, scrPeaks, scrInt, bitWords, sortCap,
                                                          err, ov);
    note_launch();
    e = cudaGetLastError();
    if (needScratch) {
        int hostErr = 0;
        cudaError_t e2 = cudaMemcpyAsync(&hostErr, err, sizeof(int), cudaMemcpyDeviceToHost, s);
        cudaError_t e3 = cudaFreeAsync(scrPeaks, s);
        if (e == cudaSuccess) e = e2;
        if (e == cudaSuccess) e = e3;
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e == cudaSuccess && hostErr) return cudaErrorAssert;
    }
    return e;
}

// KDE / DBSCAN / Ostrovsky maps whose peak capacity exceeds kFirstPassPeaks run
// a first pass with that capacity -- more blocks per SM -- listing the points
// whose peaks did not fit, then a second pass over that list at full capacity,
// whose results are scattered into place.  Every point runs the same per-point
// code as in a single pass, so the output is identical.
template <class S, int TASK>
cudaError_t launch_bif_t(const DevJob& J, void* d_out, int* d_aux, cudaStream_t s)
{
    constexpr bool split = TASK == CBF_TASK_KDE || TASK == CBF_TASK_DBSCAN || TASK == CBF_TASK_OSTROVSKY;
    if (!split || J.peakCap <= kFirstPassPeaks || J.nPoints == 0)
        return bif_pass<S, TASK>(J, d_out, d_aux, Overflow{nullptr, nullptr, nullptr}, s);
    using Out = typename std::conditional<TASK == CBF_TASK_OSTROVSKY, double, int>::type;
    const long long n = J.nPoints;
    char* mem = nullptr;
    // list of grid indices and slots, count, and the second pass's outputs
    const size_t bytes = (size_t)n * (2 * sizeof(long long) + sizeof(Out)) + 256;
    cudaError_t e = cudaMallocAsync((void**)&mem, bytes, s);
    if (e != cudaSuccess) return e;
    Overflow ov{(long long*)mem, (long long*)mem + n, (unsigned long long*)((long long*)mem + 2 * n)};
    Out* tmp = (Out*)((char*)mem + (size_t)n * 2 * sizeof(long long) + 256);
    unsigned long long count = 0;
    e = cudaMemsetAsync(ov.count, 0, sizeof(unsigned long long), s);
    if (e == cudaSuccess) {
        DevJob J1 = J;
        J1.peakCap = kFirstPassPeaks;
        e = bif_pass<S, TASK>(J1, d_out, d_aux, ov, s);
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(&count, ov.count, sizeof(count), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e == cudaSuccess && count > 0) {
        DevJob J2 = J;
        J2.pointIndex = ov.g;
        J2.firstPoint = 0;
        J2.nPoints = (long long)count;
        e = bif_pass<S, TASK>(J2, tmp, nullptr, Overflow{nullptr, nullptr, nullptr}, s);
        if (e == cudaSuccess) {
            scatter_kernel<Out><<<(unsigned)(((long long)count + 255) / 256), 256, 0, s>>>(tmp, ov.p, (long long)count,
                                                                                         (Out*)d_out);
            note_launch();
            e = cudaGetLastError();
        }
    }
    cudaError_t e2 = cudaFreeAsync(mem, s);
    if (e == cudaSuccess) e = e2;
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    return e;
}

template <class S>
cudaError_t launch_bif_s(const DevJob& J, void* d_out, int* d_aux, cudaStream_t s)
{
    switch (J.task) {
    case CBF_TASK_PEAKS: return launch_bif_t<S, CBF_TASK_PEAKS>(J, d_out, d_aux, s);
    case CBF_TASK_KDE: return launch_bif_t<S, CBF_TASK_KDE>(J, d_out, d_aux, s);
    case CBF_TASK_DBSCAN: return launch_bif_t<S, CBF_TASK_DBSCAN>(J, d_out, d_aux, s);
    case CBF_TASK_TRAJECTORY: return launch_bif_t<S, CBF_TASK_TRAJECTORY>(J, d_out, d_aux, s);
    case CBF_TASK_OSTROVSKY: return launch_bif_t<S, CBF_TASK_OSTROVSKY>(J, d_out, d_aux, s);
    default: return cudaErrorInvalidValue;
    }
}

// One pass of the fused kernel with caller-provided scratch (no allocation);
// synchronises `s` to read the error flag.
template <class S, int TASK>
cudaError_t prealloc_pass(const DevJob& J, void* d_out, double* scratch, size_t scratchBytes, int* err,
                          const Overflow& ov, cudaStream_t s)
{
    const long long nTiles = (J.nPoints + 31) / 32;
    if (nTiles == 0) return cudaSuccess;
    const int bitWords = (TASK == CBF_TASK_DBSCAN) ? (J.peakCap + 31) / 32 : 0;
    const int sortCap = bif_sort_cap(TASK, J.peakCap);
    const size_t smemBytes = (size_t)kBifWarps * dbscan_warp_words(bitWords, sortCap) * sizeof(unsigned);
    auto kern = bif_kernel<S, TASK>;
    cudaError_t e;
    if (smemBytes > 48 * 1024) {
        e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smemBytes);
        if (e != cudaSuccess) return e;
    }
    int dev = 0, sms = 0, perSm = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, kern, kBifThreads, smemBytes)) != cudaSuccess)
        return e;
    if (perSm < 1) return cudaErrorInvalidConfiguration;
    const size_t perBlock = (size_t)kBifThreads * J.peakCap * sizeof(double) *
                            (task_with_intervals(TASK) ? 2 : 1);
    long long blocks = (nTiles + kBifWarps - 1) / kBifWarps;
    const long long resident = (long long)sms * perSm;
    if (blocks > resident) blocks = resident;
    const long long fit = (long long)(scratchBytes / perBlock);
    if (fit < 1) return cudaErrorInvalidValue;
    if (blocks > fit) blocks = fit;
    double* scrInt = (TASK == CBF_TASK_DBSCAN) ? scratch + (size_t)blocks * kBifThreads * J.peakCap : nullptr;
    kern<<<(unsigned)blocks, kBifThreads, smemBytes, s>>>(J, d_out, nullptr, scratch, scrInt, bitWords, sortCap,
                                                          err, ov);
    note_launch();
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    int hostErr = 0;
    if ((e = cudaMemcpyAsync(&hostErr, err, sizeof(int), cudaMemcpyDeviceToHost, s)) != cudaSuccess) return e;
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return e;
    return hostErr ? cudaErrorAssert : cudaSuccess;
}

// KDE / DBSCAN map with caller-provided scratch, in the regular entry point's two
// passes: when the peak capacity exceeds kFirstPassPeaks, a first pass at that
// capacity (many more blocks fit the scratch) lists the points whose peaks did
// not fit, a second pass recomputes them at full capacity and their results are
// scattered into place -- the same per-point code, the same map.  The scratch
// holds the overflow list (grid index and slot, 16 B per point) and the second
// pass's results (4 B per point) of a chunk of points in front of the peak
// buffers; the chunk is sized so that the list takes at most a quarter of the
// scratch and one block still fits at full capacity.  Without room for that,
// every point runs once at full capacity.
template <class S, int TASK>
cudaError_t launch_bif_prealloc_t(const DevJob& J, void* d_out, double* scratch, size_t scratchBytes,
                                  int* err, cudaStream_t s)
{
    const Overflow none{nullptr, nullptr, nullptr};
    if (J.nPoints == 0) return cudaSuccess;
    const size_t perBlockFull = (size_t)kBifThreads * J.peakCap * sizeof(double) * (task_with_intervals(TASK) ? 2 : 1);
    const size_t perPoint = 2 * sizeof(long long) + sizeof(int);
    size_t listBytes = scratchBytes / 4;
    if (scratchBytes < perBlockFull + 1024) listBytes = 0;
    else if (listBytes > scratchBytes - perBlockFull - 1024) listBytes = scratchBytes - perBlockFull - 1024;
    long long chunk = (long long)(listBytes / perPoint);
    if (J.peakCap <= kFirstPassPeaks || chunk < 32)
        return prealloc_pass<S, TASK>(J, d_out, scratch, scratchBytes, err, none, s);
    if (chunk > J.nPoints) chunk = J.nPoints;
    char* base = (char*)scratch;
    long long* listG = (long long*)base;
    long long* listP = listG + chunk;
    int* tmp = (int*)(listP + chunk);
    const size_t countOff = ((size_t)((char*)(tmp + chunk) - base) + 255) / 256 * 256;
    unsigned long long* count = (unsigned long long*)(base + countOff);
    const size_t peakOff = countOff + 256;
    double* peaks = (double*)(base + peakOff);
    const size_t peakBytes = scratchBytes - peakOff;
    cudaError_t e = cudaSuccess;
    for (long long first = 0; first < J.nPoints && e == cudaSuccess; first += chunk) {
        const long long m = (J.nPoints - first < chunk) ? J.nPoints - first : chunk;
        DevJob J1 = J;
        if (J.pointIndex) J1.pointIndex = J.pointIndex + first;
        else J1.firstPoint = J.firstPoint + first;
        J1.nPoints = m;
        J1.peakCap = kFirstPassPeaks;
        int* out = (int*)d_out + first;
        unsigned long long n2 = 0;
        e = cudaMemsetAsync(count, 0, sizeof(unsigned long long), s);
        if (e == cudaSuccess) e = prealloc_pass<S, TASK>(J1, out, peaks, peakBytes, err, Overflow{listG, listP, count}, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(&n2, count, sizeof(n2), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e == cudaSuccess && n2 > 0) {
            DevJob J2 = J;
            J2.pointIndex = listG;
            J2.firstPoint = 0;
            J2.nPoints = (long long)n2;
            e = prealloc_pass<S, TASK>(J2, tmp, peaks, peakBytes, err, none, s);
            if (e == cudaSuccess) {
                scatter_kernel<int><<<(unsigned)(((long long)n2 + 255) / 256), 256, 0, s>>>(tmp, listP, (long long)n2,
                                                                                         out);
                note_launch();
                e = cudaGetLastError();
            }
        }
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    return e;
}

template <class S>
cudaError_t launch_bif_prealloc_s(const DevJob& J, void* d_out, double* scratch, size_t scratchBytes,
                                  int* err, cudaStream_t s)
{
    switch (J.task) {
    case CBF_TASK_KDE: return launch_bif_prealloc_t<S, CBF_TASK_KDE>(J, d_out, scratch, scratchBytes, err, s);
    case CBF_TASK_DBSCAN: return launch_bif_prealloc_t<S, CBF_TASK_DBSCAN>(J, d_out, scratch, scratchBytes, err, s);
    default: return cudaErrorInvalidValue;
    }
}

static_assert(kBifThreads == kBifBlockThreads, "block size shared with other translation units");

}  // namespace

cudaError_t launch_bif_prealloc(const DevJob& J, void* d_out, double* scratch, size_t scratchBytes,
                                int* err, cudaStream_t s)
{
    switch (J.system) {
    case CBF_SYS_MEMRISTIVE5: return launch_bif_prealloc_s<Memristive5>(J, d_out, scratch, scratchBytes, err, s);
    case CBF_SYS_ROSSLER: return launch_bif_prealloc_s<Rossler>(J, d_out, scratch, scratchBytes, err, s);
    case CBF_SYS_LORENZ: return J.scaledStep ? launch_bif_prealloc_s<LorenzScaled>(J, d_out, scratch, scratchBytes, err, s) : launch_bif_prealloc_s<Lorenz>(J, d_out, scratch, scratchBytes, err, s);
    case CBF_SYS_CHEN: return J.scaledStep ? launch_bif_prealloc_s<ChenScaled>(J, d_out, scratch, scratchBytes, err, s) : launch_bif_prealloc_s<Chen>(J, d_out, scratch, scratchBytes, err, s);
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_bif(const DevJob& J, void* d_out, int* d_aux, cudaStream_t s)
{
    switch (J.system) {
    case CBF_SYS_MEMRISTIVE5: return launch_bif_s<Memristive5>(J, d_out, d_aux, s);
    case CBF_SYS_ROSSLER: return launch_bif_s<Rossler>(J, d_out, d_aux, s);
    case CBF_SYS_LORENZ: return J.scaledStep ? (J.unitStep ? launch_bif_s<LorenzScaledU>(J, d_out, d_aux, s) : launch_bif_s<LorenzScaled>(J, d_out, d_aux, s)) : launch_bif_s<Lorenz>(J, d_out, d_aux, s);
    case CBF_SYS_CHEN: return J.scaledStep ? (J.unitStep ? launch_bif_s<ChenScaledU>(J, d_out, d_aux, s) : launch_bif_s<ChenScaled>(J, d_out, d_aux, s)) : launch_bif_s<Chen>(J, d_out, d_aux, s);
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace cbf
