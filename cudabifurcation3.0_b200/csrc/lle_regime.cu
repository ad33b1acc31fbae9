// LLE map with a peak-count regime class per point, in one pass.
//
// The LLE is computed exactly as by the LLE kernels (LLEKernelCUDA semantics,
// cudaLibrary.cu:666-908).  During the first `regimeSteps` steps after the
// transient, the base trajectory's x[writableVar] is sampled before every step
// (the record semantics of loopCalculateDiscreteModel, cudaLibrary.cu:59-62) and
// fed to the streaming peak finder; the class is the reference's DBSCAN cluster
// count of those (peak, interval) pairs (dbscan, cudaLibrary.cu:457-529), with
//   0  when the trajectory diverged inside the window or has no peaks,
//   15 when its LLE exceeds regimeChaosLle (if > 0; no clustering needed), when
//      it has more than maxAmountOfPeaks peaks, or 15 or more clusters.
// A window whose samples span less than regimeMinAmp is class 0 as well: an
// equilibrium reached to FP64 precision can still wobble by an ulp and show
// spurious peaks.  The window costs one peak-state update per step on top of the LLE; the
// transient is shared.  This is the plain FP64 method that labels the surrogate's
// training data and recomputes the points it cannot be trusted with.
#include "bif_device.cuh"
#include "lle_device.cuh"

namespace cbf {
namespace {

constexpr int kRegWarps = 4;
constexpr int kRegThreads = kRegWarps * 32;
constexpr int kNumClasses = 16;

// One point: returns the LLE; *n = emitted peaks in the window, -1 if the
// divergence test fired inside it; *amp = max - min of the window's samples.
template <class S, bool IC>
__device__ double lle_regime_point(const DevJob& J, long long g, double* pk, double* iv, int cap,
                                   int* nOut, double* amp)
{
    constexpr int D = S::DIM;
    double x[1][D], y[1][D];
    typename S::Coef c[1];
    {
        double v[CBF_MAX_VALUES];
        setup_point<D>(J, g, x[0], v);
        c[0] = S::prep(v, J.h);
        to_stored<S>(x[0], c[0]);
    }
    run_checked<S, 1>(x, c, J.nSkip, J);
    {
        double z[D];
        lle_seed<D, IC>(g, J.seedChunk, z);
#pragma unroll
        for (int i = 0; i < D; ++i) y[0][i] = stored_comp<S>(z[i] * J.lleEps, i, c[0]) + x[0][i];
    }
    double result = 0;
    // Renormalisation (cudaLibrary.cu:757-776) after each interval.
    auto renorm = [&]() {
        double tt = 0;
#pragma unroll
        for (int l = 0; l < D; ++l) {
            const double d = phys_comp<S>(x[0][l] - y[0][l], l, c[0]);
            tt += d * d;
        }
        tt = sqrt(tt) / J.lleEps;
        result += log(tt);
        if (tt != 0) tt = (1 / tt);
#pragma unroll
        for (int i = 0; i < D; ++i) y[0][i] = x[0][i] - ((x[0][i] - y[0][i]) * tt);
    };
    int b = 0;
    {
        // The intervals that overlap the window, with the peak stream; its state
        // is dead after this block, so the loop below is the LLE kernel's loop.
        PeakStream ps;
        ps.init();
        double lo = INFINITY, hi = -INFINITY;
        bool regimeDiv = false;
        int t = 0;  // step index since the transient
        for (; b < J.nRecord && t < J.regimeSteps; ++b) {
            // Intervals overlapping the window: the peak stream fed before every
            // x step and the divergence test after every step; a trajectory's
            // interval ends at its first failed test (loopCalculateDiscreteModel,
            // cudaLibrary.cu:55-74).  The window is ~2 % of the steps, so it uses
            // the exact per-step test directly instead of the run-then-replay
            // scheme of the loop below, whose state snapshots would set the
            // register count of the whole kernel.
            bool ax = true, ay = true;
            for (int i = 0; i < J.nNT; ++i, ++t) {
                if (ax) {
                    if (t < J.regimeSteps) {
                        const double v = phys_comp<S>(pick<D>(x[0], J.writableVar), J.writableVar, c[0]);
                        lo = fmin(lo, v);
                        hi = fmax(hi, v);
                        ps.push<true>(v, t, pk, iv, cap);
                    }
                    S::step(x[0], c[0]);
                    if (J.checkDiv && diverged(x[0][0], J.divThresh)) {
                        ax = false;
                        if (t < J.regimeSteps) regimeDiv = true;
                    }
                }
                if (ay) {
                    S::step(y[0], c[0]);
                    if (J.checkDiv && diverged(y[0][0], J.divThresh)) ay = false;
                }
            }
            renorm();
        }
        *nOut = regimeDiv ? -1 : ps.emitted();
        *amp = hi - lo;
    }
    for (; b < J.nRecord; ++b) {
        run_pair<S, 1>(x, y, c, J.nNT, J);
        renorm();
    }
    return result / J.tMax;
}

// LLE and regime class of the lane's grid point g (`valid` false: the lane idles
// through the integration), the warp cooperating on the DBSCAN epilogues of
// lanes 0..live-1; *lleOut = the lane's LLE.
template <class S, bool IC>
__device__ __forceinline__ int regime_tile(const DevJob& J, long long g, bool valid, int live, int lane,
                                           double* scrPk, double* scrIv, long long slot0, unsigned* L,
                                           unsigned* Sb, const DbscanSort& so, int* err, double* lleOut)
{
    const int cap = J.peakCap;
    double* myPk = scrPk + (slot0 + lane) * (long long)cap;
    double* myIv = scrIv + (slot0 + lane) * (long long)cap;
    int n = 0;
    double lv = 0, amp = 0;
    if (valid) lv = lle_regime_point<S, IC>(J, g, myPk, myIv, cap, &n, &amp);
    if (amp < J.regimeMinAmp) n = 0;  // no oscillation
    __syncwarp();
    int res = 0;
    for (int j = 0; j < live; ++j) {
        const int nj = __shfl_sync(kFull, n, j);
        const double lj = __shfl_sync(kFull, lv, j);
        int r;
        if (nj <= 0) r = 0;
        else if (J.regimeChaosLle > 0 && lj > J.regimeChaosLle) r = kNumClasses - 1;
        else if (nj > J.maxPeaks) r = kNumClasses - 1;
        else {
            const double* pk = scrPk + (slot0 + j) * (long long)cap;
            const double* iv = scrIv + (slot0 + j) * (long long)cap;
            r = min(dbscan_warp(J, pk, iv, nj, lane, L, Sb, err, so), kNumClasses - 1);
        }
        if (lane == j) res = r;
    }
    *lleOut = lv;
    return res;
}

// Six blocks per SM, like the autotuned LLE map kernel: 80 registers, no spill.
// nDev (optional): the job's point count read on the device, in place of
// J.nPoints (a point list whose length a previous kernel wrote).
template <class S, bool IC>
__global__ void __launch_bounds__(kRegThreads, 6) lle_regime_kernel(DevJob J, double* __restrict__ lle,
                                                                 int* __restrict__ cls, double* scrPk,
                                                                 double* scrIv, int bitWords, int sortCap,
                                                                 int* err, const long long* nDev)
{
    extern __shared__ unsigned smem[];
    if (nDev) J.nPoints = *nDev;
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const long long warpId = (long long)blockIdx.x * kRegWarps + wib;
    const long long nWarps = (long long)gridDim.x * kRegWarps;
    const long long nTiles = (J.nPoints + 31) / 32;
    unsigned* L = smem + (size_t)wib * dbscan_warp_words(bitWords, sortCap);
    unsigned* Sb = L + bitWords;
    const DbscanSort so = dbscan_sort_area(L, bitWords, sortCap);
    const long long slot0 = warpId * 32;

    for (long long tile = warpId; tile < nTiles; tile += nWarps) {
        const long long p = tile * 32 + lane;
        const bool valid = p < J.nPoints;
        const int live = (int)min(32ll, J.nPoints - tile * 32);
        double lv = 0;
        const int res = regime_tile<S, IC>(J, valid ? grid_index(J, p) : 0, valid, live, lane, scrPk, scrIv,
                                           slot0, L, Sb, so, err, &lv);
        if (valid) {
            lle[p] = lv;
            cls[p] = res;
        }
        __syncwarp();
    }
}

template <class S, bool IC>
cudaError_t launch_t(const DevJob& J, double* d_lle, int* d_cls, cudaStream_t s)
{
    const long long nTiles = (J.nPoints + 31) / 32;
    if (nTiles == 0) return cudaSuccess;
    const int bitWords = (J.peakCap + 31) / 32;
    const int sortCap = dbscan_sort_cap(J.peakCap);
    const size_t smemBytes = (size_t)kRegWarps * dbscan_warp_words(bitWords, sortCap) * sizeof(unsigned);
    auto kern = lle_regime_kernel<S, IC>;
    cudaError_t e;
    if (smemBytes > 48 * 1024) {
        e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smemBytes);
        if (e != cudaSuccess) return e;
    }
    int dev = 0, sms = 0, perSm = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, kern, kRegThreads, smemBytes)) != cudaSuccess)
        return e;
    if (perSm < 1) return cudaErrorInvalidConfiguration;
    long long blocks = (nTiles + kRegWarps - 1) / kRegWarps;
    if (blocks > (long long)sms * perSm) blocks = (long long)sms * perSm;
    const size_t perBlock = (size_t)kRegThreads * J.peakCap * sizeof(double) * 2;
    size_t freeB = 0, totalB = 0;
    if ((e = cudaMemGetInfo(&freeB, &totalB)) != cudaSuccess) return e;
    size_t budget = freeB / 4;
    if (budget > ((size_t)8 << 30)) budget = (size_t)8 << 30;
    long long fit = (long long)(budget / perBlock);
    if (fit < 1) fit = 1;
    if (blocks > fit) blocks = fit;
    const size_t bytes = (size_t)blocks * perBlock;
    double* scr = nullptr;
    if ((e = cudaMallocAsync((void**)&scr, bytes + 256, s)) != cudaSuccess) return e;
    double* scrIv = scr + (size_t)blocks * kRegThreads * J.peakCap;
    int* err = (int*)((char*)scr + bytes);
    if ((e = cudaMemsetAsync(err, 0, sizeof(int), s)) == cudaSuccess) {
        kern<<<(unsigned)blocks, kRegThreads, smemBytes, s>>>(J, d_lle, d_cls, scr, scrIv, bitWords, sortCap, err,
                                                              nullptr);
        note_launch();
        e = cudaGetLastError();
    }
    int hostErr = 0;
    cudaError_t e2 = cudaMemcpyAsync(&hostErr, err, sizeof(int), cudaMemcpyDeviceToHost, s);
    cudaError_t e3 = cudaFreeAsync(scr, s);
    if (e == cudaSuccess) e = e2;
    if (e == cudaSuccess) e = e3;
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e == cudaSuccess && hostErr) return cudaErrorAssert;
    return e;
}

template <class S>
cudaError_t launch_s(const DevJob& J, double* d_lle, int* d_cls, cudaStream_t s)
{
    return J.sweepIC ? launch_t<S, true>(J, d_lle, d_cls, s) : launch_t<S, false>(J, d_lle, d_cls, s);
}

// The kernel on a device point list of *nDev <= maxPoints entries: one block per
// resident slot (at most the list's tiles), caller-provided scratch, no
// allocation and no host synchronisation (the caller reads `err`).
template <class S>
cudaError_t launch_list_s(const DevJob& J, const long long* nDev, long long maxPoints, double* d_lle, int* d_cls,
                          double* scratch, size_t scratchBytes, int* err, cudaStream_t s)
{
    const int bitWords = (J.peakCap + 31) / 32;
    const int sortCap = dbscan_sort_cap(J.peakCap);
    const size_t smemBytes = (size_t)kRegWarps * dbscan_warp_words(bitWords, sortCap) * sizeof(unsigned);
    auto kern = lle_regime_kernel<S, false>;
    cudaError_t e;
    if (smemBytes > 48 * 1024) {
        e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smemBytes);
        if (e != cudaSuccess) return e;
    }
    int dev = 0, sms = 0, perSm = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, kern, kRegThreads, smemBytes)) != cudaSuccess)
        return e;
    if (perSm < 1) return cudaErrorInvalidConfiguration;
    long long blocks = (maxPoints + kRegThreads - 1) / kRegThreads;
    if (blocks > (long long)sms * perSm) blocks = (long long)sms * perSm;
    const size_t perBlock = (size_t)kRegThreads * J.peakCap * sizeof(double) * 2;
    if ((size_t)blocks * perBlock > scratchBytes) blocks = (long long)(scratchBytes / perBlock);
    if (blocks < 1) return cudaErrorInvalidValue;
    double* scrIv = scratch + (size_t)blocks * kRegThreads * J.peakCap;
    kern<<<(unsigned)blocks, kRegThreads, smemBytes, s>>>(J, d_lle, d_cls, scratch, scrIv, bitWords, sortCap, err,
                                                          nDev);
    note_launch();
    return cudaGetLastError();
}

template <class S>
long long resident_s(const DevJob& J)
{
    const int bitWords = (J.peakCap + 31) / 32;
    const int sortCap = dbscan_sort_cap(J.peakCap);
    const size_t smemBytes = (size_t)kRegWarps * dbscan_warp_words(bitWords, sortCap) * sizeof(unsigned);
    auto kern = J.sweepIC ? lle_regime_kernel<S, true> : lle_regime_kernel<S, false>;
    if (smemBytes > 48 * 1024)
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smemBytes);
    int dev = 0, sms = 0, perSm = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, kern, kRegThreads, smemBytes) != cudaSuccess)
        return 0;
    return (long long)sms * perSm * kRegThreads;
}

}  // namespace

long long lle_regime_resident_points(const DevJob& J)
{
    switch (J.system) {
    case CBF_SYS_MEMRISTIVE5: return resident_s<Memristive5>(J);
    case CBF_SYS_ROSSLER: return resident_s<Rossler>(J);
    case CBF_SYS_LORENZ: return J.scaledStep ? (J.unitStep ? resident_s<LorenzScaledU>(J) : resident_s<LorenzScaled>(J)) : resident_s<Lorenz>(J);
    case CBF_SYS_CHEN: return J.scaledStep ? (J.unitStep ? resident_s<ChenScaledU>(J) : resident_s<ChenScaled>(J)) : resident_s<Chen>(J);
    default: return 0;
    }
}

cudaError_t launch_lle_regime(const DevJob& J, double* d_lle, int* d_cls, cudaStream_t s)
{
    switch (J.system) {
    case CBF_SYS_MEMRISTIVE5: return launch_s<Memristive5>(J, d_lle, d_cls, s);
    case CBF_SYS_ROSSLER: return launch_s<Rossler>(J, d_lle, d_cls, s);
    case CBF_SYS_LORENZ: return J.scaledStep ? (J.unitStep ? launch_s<LorenzScaledU>(J, d_lle, d_cls, s) : launch_s<LorenzScaled>(J, d_lle, d_cls, s)) : launch_s<Lorenz>(J, d_lle, d_cls, s);
    case CBF_SYS_CHEN: return J.scaledStep ? (J.unitStep ? launch_s<ChenScaledU>(J, d_lle, d_cls, s) : launch_s<ChenScaled>(J, d_lle, d_cls, s)) : launch_s<Chen>(J, d_lle, d_cls, s);
    default: return cudaErrorInvalidValue;
    }
}

size_t lle_regime_scratch_bytes(const DevJob& J)
{
    const long long resident = lle_regime_resident_points(J);
    return (size_t)(resident > 0 ? resident : 0) * J.peakCap * sizeof(double) * 2;
}

cudaError_t launch_lle_regime_list(const DevJob& J, const long long* nDev, long long maxPoints, double* d_lle,
                                   int* d_cls, double* scratch, size_t scratchBytes, int* err, cudaStream_t s)
{
    if (J.sweepIC || !J.pointIndex || maxPoints <= 0) return cudaErrorInvalidValue;
    switch (J.system) {
    case CBF_SYS_ROSSLER: return launch_list_s<Rossler>(J, nDev, maxPoints, d_lle, d_cls, scratch, scratchBytes, err, s);
    case CBF_SYS_LORENZ:
        return J.scaledStep ? (J.unitStep ? launch_list_s<LorenzScaledU>(J, nDev, maxPoints, d_lle, d_cls, scratch, scratchBytes, err, s) : launch_list_s<LorenzScaled>(J, nDev, maxPoints, d_lle, d_cls, scratch, scratchBytes, err, s))
                            : launch_list_s<Lorenz>(J, nDev, maxPoints, d_lle, d_cls, scratch, scratchBytes, err, s);
    case CBF_SYS_CHEN:
        return J.scaledStep ? (J.unitStep ? launch_list_s<ChenScaledU>(J, nDev, maxPoints, d_lle, d_cls, scratch, scratchBytes, err, s) : launch_list_s<ChenScaled>(J, nDev, maxPoints, d_lle, d_cls, scratch, scratchBytes, err, s))
                            : launch_list_s<Chen>(J, nDev, maxPoints, d_lle, d_cls, scratch, scratchBytes, err, s);
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace cbf
