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
#include "engine.cuh"

namespace cbf {

namespace {

constexpr int kBifWarps = 4;
constexpr int kBifThreads = kBifWarps * 32;
constexpr unsigned kFull = 0xffffffffu;

// ---------------------------------------------------------------------------
// Streaming restatement of peakFinder (cudaLibrary.cu:220-266) over the samples
// d[0..N) in arrival order.  Candidate i is judged when d[i+1] arrives:
//   NORMAL : d[i] > d[i-1] && d[i] >= d[i+1] -> peak at i if d[i] > d[i+1],
//            otherwise a plateau begins (inner loop of :229-246);
//   PLATEAU: compare the plateau value with the next sample: larger -> peak at
//            the plateau end j; smaller -> no peak; equal -> continue;
//   SKIP   : after a peak or a rising plateau the reference sets i = j+1 and its
//            ++i moves on to j+2, so the next arrival is not a candidate.
// The first detected peak is dropped and intervals are (t[k+1]-t[k]) * 0.01
// (:250-262).  NaN is absorbing for these systems, so the inner loop's
// run-to-the-end case never yields a peak, as here.
struct PeakStream {
    double prev1, prev2, pval;
    int mode;       // 0 NORMAL, 1 PLATEAU, 2 SKIP
    int detected;
    int lastT;

    __device__ __forceinline__ void init()
    {
        prev1 = prev2 = pval = 0.0;
        mode = 0;
        detected = 0;
        lastT = 0;
    }

    template <bool WITH_INTERVALS>
    __device__ __forceinline__ void emit(double val, int t, double* pk, double* iv, int cap)
    {
        if (detected >= 1) {
            const int k = detected - 1;
            if (k < cap) {
                pk[k] = val;
                if (WITH_INTERVALS) iv[k] = (double)(t - lastT) * kPeakIntervalUnit;
            }
        }
        lastT = t;
        ++detected;
    }

    template <bool WITH_INTERVALS>
    __device__ __forceinline__ void push(double v, int t, double* pk, double* iv, int cap)
    {
        if (t >= 2) {
            if (mode == 2) {
                mode = 0;
            } else if (mode == 1) {
                if (pval < v) {
                    mode = 2;
                } else if (pval > v) {
                    emit<WITH_INTERVALS>(pval, t - 1, pk, iv, cap);
                    mode = 2;
                }
            } else if (prev1 > prev2 && prev1 >= v) {
                if (prev1 > v) {
                    emit<WITH_INTERVALS>(prev1, t - 1, pk, iv, cap);
                    mode = 2;
                } else {
                    mode = 1;
                    pval = prev1;
                }
            }
        }
        prev2 = prev1;
        prev1 = v;
    }

    __device__ __forceinline__ int emitted() const { return detected > 1 ? detected - 1 : 0; }
};

template <int D>
__device__ __forceinline__ double pick(const double (&x)[D], int wv)
{
    double r = x[0];
#pragma unroll
    for (int i = 1; i < D; ++i)
        if (i == wv) r = x[i];
    return r;
}

// One point: transient (unchecked, cudaLibrary.cu:107-108), then the recorded
// loop (:110-114) feeding the peak stream.  Returns the emitted peak count, 0 on
// divergence (peakFinderCUDA turns the -1 flag into 0, :277-281).
template <class S, int TASK>
__device__ int integrate_point(const DevJob& J, long long g, double* pk, double* iv, int cap,
                               double* traj, int* divFlag)
{
    constexpr int D = S::DIM;
    double x[D], v[CBF_MAX_VALUES];
    setup_point<D>(J, g, x, v);
    const typename S::Coef c = S::prep(v, J.h);

#pragma unroll 4
    for (int i = 0; i < J.nSkip; ++i) S::step(x, c);

    const int wv = J.writableVar;
    PeakStream ps;
    ps.init();
    bool div = false;
    int t = 0;
    for (; t < J.nRecord; ++t) {
        const double val = pick<D>(x, wv);
        if (TASK == CBF_TASK_TRAJECTORY)
            traj[t] = val;
        else
            ps.push<TASK == CBF_TASK_DBSCAN>(val, t, pk, iv, cap);
        for (int j = 0; j < J.preScaller - 1; ++j) S::step(x, c);
        S::step(x, c);
        if (J.checkDiv && diverged(pick<D>(x, wv), J.divThresh)) {
            div = true;
            ++t;
            break;
        }
    }
    if (TASK == CBF_TASK_TRAJECTORY) {
        // Samples after a divergence are never written by the reference; make them NaN.
        for (; t < J.nRecord; ++t) traj[t] = __longlong_as_double(0x7ff8000000000000ll);
        *divFlag = div ? 1 : 0;
        return 0;
    }
    return div ? 0 : ps.emitted();
}

// ---------------------------------------------------------------------------
// KDE mode count of one point (kde, cudaLibrary.cu:356-422), whole warp.
__device__ int kde_warp(const DevJob& J, const double* pk, int n, int lane)
{
    if (n == 0) return 0;
    if (n == 1 || n == 2) return 1;
    if (n > J.maxPeaks) return J.maxPeaks;

    const double k1 = J.kdeFixed ? (double)J.kdeSampling : (double)(J.kdeSampling * n);
    const double k2 = (J.kdeI2 - J.kdeI1) / (k1 - 1);
    // `for (int w = 0; w < k1 - 1; ++w)`: k1 is integral, so W = k1 - 1 iterations.
    const int W = (k1 - 1 > 0) ? (int)ceil(k1 - 1) : 0;
    const double skip = J.kdeSkip;
    const double H = J.kdeH;

    double pp = 0, pr = 0, cur = 0;
    bool strange = false;
    int res = 0;
    for (int base = 0; base < W; base += 32) {
        const int w = base + lane;
        double d2 = 0;
        if (w < W) {
            const double delt = w * k2 + J.kdeI1;
            for (int m = 0; m < n; ++m) {
                const double dd = pk[m] - delt;
                // |dd| > 16|H| makes the FP32 exponent argument <= -128, where expf
                // is exactly +0 (checked exhaustively on the device by
                // cbf_probe_expf_zero), and adding +0 leaves the sum unchanged.
                if (!(fabs(dd) > skip)) {
                    const double tmp = dd / H;
                    d2 += (double)expf((float)(-((tmp * tmp) / 2)));
                }
            }
        }
        const int cnt = min(32, W - base);
        for (int j = 0; j < cnt; ++j) {
            const double val = __shfl_sync(kFull, d2, j);
            pp = pr;
            pr = cur;
            cur = val;
            if (base + j < 2) continue;
            if (strange) {
                if (pr == cur) continue;
                else if (pr < cur) { strange = false; continue; }
                else if (pr > cur) { strange = false; ++res; continue; }
            } else if (pr > pp && pr > cur) {
                ++res;
                continue;
            } else if (pr > pp && pr == cur) {
                strange = true;
                continue;
            }
        }
    }
    if (pr < cur) ++res;
    return res;
}

// ---------------------------------------------------------------------------
// DBSCAN cluster count of one point (dbscan, cudaLibrary.cu:457-529), whole warp.
// helpfulArray[k] (label, nonzero once set) -> bitset L; helpfulArray[n+k] (the
// "stack", holds k or 0) -> bitset S: popping slot m yields m if set, else 0.
__device__ int dbscan_warp(const DevJob& J, const double* pk,
                           const double* iv, int n, int lane, unsigned* L,
                           unsigned* Sb, int* err)
{
    if (n <= 0) return 0;
    if (n == 1) return 1;
    if (n > J.maxPeaks) return 0;

    const int words = (n + 31) >> 5;
    for (int w = lane; w < words; w += 32) {
        L[w] = 0u;
        Sb[w] = 0u;
    }
    __syncwarp();

    const double eps = J.dbEps;
    const double skip = J.dbSkip;
    int cluster = 0;
    int num = 0;
    long long guard = (long long)n * n + 4ll * n + 16;
    for (int i = 0; i < n; i++) {
        if (--guard < 0) {
            if (lane == 0) atomicExch(err, 1);
            return 0;
        }
        int center = -1;
        if (num >= 1) {
            const int m = num - 1;
            const bool set = (Sb[m >> 5] >> (m & 31)) & 1u;
            __syncwarp();
            if (lane == 0) Sb[m >> 5] &= ~(1u << (m & 31));
            __syncwarp();
            i = set ? m : 0;
            num = num - 1;
            center = i;
        } else if (!((L[i >> 5] >> (i & 31)) & 1u)) {
            num = 0;
            ++cluster;
            __syncwarp();
            if (lane == 0) L[i >> 5] |= 1u << (i & 31);
            __syncwarp();
            center = i;
        }
        if (center < 0) continue;

        const double x1 = pk[center];
        const double y1 = iv[center];
        for (int base = 0; base < n - 1; base += 32) {
            const int k = base + lane;
            bool cand = false;
            if (k < n - 1 && k != center && !((L[base >> 5] >> lane) & 1u)) {
                const double x2 = pk[k];
                const double y2 = iv[k];
                if (x1 == x2 && y1 == y2) {
                    cand = 0.0 < eps;  // distance() returns 0 on exact equality (:447-448)
                } else {
                    const double dx = x2 - x1;
                    const double dy = y2 - y1;
                    // hypotf(dx, dy) >= max(|dx|, |dy|) up to a few ulps, so pairs with
                    // a coordinate gap >= 4*eps can never be closer than eps.
                    if (!(fabs(dx) >= skip || fabs(dy) >= skip))
                        cand = (double)hypotf((float)dx, (float)dy) < eps;
                }
            }
            const unsigned b = __ballot_sync(kFull, cand);
            if (b) {
                if (lane == 0) {
                    L[base >> 5] |= b;
                    Sb[base >> 5] |= b;
                }
                num += __popc(b);
            }
        }
        __syncwarp();
    }
    return cluster - 1;
}

// ---------------------------------------------------------------------------
template <class S, int TASK>
__global__ void __launch_bounds__(kBifThreads) bif_kernel(const DevJob J, void* __restrict__ d_out,
                                                          int* __restrict__ d_aux,
                                                          double* scrPeaks,
                                                          double* scrInt,
                                                          int bitWords, int* __restrict__ err)
{
    extern __shared__ unsigned smem[];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const long long warpId = (long long)blockIdx.x * kBifWarps + wib;
    const long long nWarps = (long long)gridDim.x * kBifWarps;
    const long long nTiles = (J.nPoints + 31) / 32;
    const int cap = J.peakCap;
    unsigned* L = smem + (size_t)wib * 2 * bitWords;
    unsigned* Sb = L + bitWords;

    for (long long tile = warpId; tile < nTiles; tile += nWarps) {
        const long long p = tile * 32 + lane;
        const bool valid = p < J.nPoints;
        const long long g = J.firstPoint + p;

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
        double* myIv = (TASK == CBF_TASK_DBSCAN) ? scrInt + (slot0 + lane) * (long long)cap : nullptr;
        int n = 0;
        if (valid) n = integrate_point<S, TASK>(J, g, myPk, myIv, cap, nullptr, nullptr);
        __syncwarp();

        int res = 0;
        const int live = (int)min(32ll, J.nPoints - tile * 32);
        for (int j = 0; j < live; ++j) {
            const int nj = __shfl_sync(kFull, n, j);
            const double* pk = scrPeaks + (slot0 + j) * (long long)cap;
            int r;
            if (TASK == CBF_TASK_KDE) {
                r = kde_warp(J, pk, nj, lane);
            } else {
                const double* iv = scrInt + (slot0 + j) * (long long)cap;
                r = dbscan_warp(J, pk, iv, nj, lane, L, Sb, err);
            }
            if (lane == j) res = r;
        }
        if (valid) ((int*)d_out)[p] = res;
        __syncwarp();
    }
}

template <class S, int TASK>
cudaError_t launch_bif_t(const DevJob& J, void* d_out, int* d_aux, cudaStream_t s)
{
    const long long nTiles = (J.nPoints + 31) / 32;
    if (nTiles == 0) return cudaSuccess;
    const bool needScratch = (TASK == CBF_TASK_KDE || TASK == CBF_TASK_DBSCAN);
    const int bitWords = (TASK == CBF_TASK_DBSCAN) ? (J.peakCap + 31) / 32 : 0;
    const size_t smemBytes = (size_t)kBifWarps * 2 * bitWords * sizeof(unsigned);

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
                                (TASK == CBF_TASK_DBSCAN ? 2 : 1);
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
        if (TASK == CBF_TASK_DBSCAN) scrInt = scrPeaks + (size_t)blocks * kBifThreads * J.peakCap;
        err = (int*)((char*)scrPeaks + bytes);
        if ((e = cudaMemsetAsync(err, 0, sizeof(int), s)) != cudaSuccess) return e;
    }
    kern<<<(unsigned)blocks, kBifThreads, smemBytes, s>>>(J, d_out, d_aux, scrPeaks, scrInt, bitWords, err);
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

template <class S>
cudaError_t launch_bif_s(const DevJob& J, void* d_out, int* d_aux, cudaStream_t s)
{
    switch (J.task) {
    case CBF_TASK_PEAKS: return launch_bif_t<S, CBF_TASK_PEAKS>(J, d_out, d_aux, s);
    case CBF_TASK_KDE: return launch_bif_t<S, CBF_TASK_KDE>(J, d_out, d_aux, s);
    case CBF_TASK_DBSCAN: return launch_bif_t<S, CBF_TASK_DBSCAN>(J, d_out, d_aux, s);
    case CBF_TASK_TRAJECTORY: return launch_bif_t<S, CBF_TASK_TRAJECTORY>(J, d_out, d_aux, s);
    default: return cudaErrorInvalidValue;
    }
}

template <class S, int TASK>
cudaError_t launch_bif_prealloc_t(const DevJob& J, void* d_out, double* scratch, size_t scratchBytes,
                                  int* err, cudaStream_t s)
{
    const long long nTiles = (J.nPoints + 31) / 32;
    if (nTiles == 0) return cudaSuccess;
    const int bitWords = (TASK == CBF_TASK_DBSCAN) ? (J.peakCap + 31) / 32 : 0;
    const size_t smemBytes = (size_t)kBifWarps * 2 * bitWords * sizeof(unsigned);
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
                            (TASK == CBF_TASK_DBSCAN ? 2 : 1);
    long long blocks = (nTiles + kBifWarps - 1) / kBifWarps;
    const long long resident = (long long)sms * perSm;
    if (blocks > resident) blocks = resident;
    const long long fit = (long long)(scratchBytes / perBlock);
    if (fit < 1) return cudaErrorInvalidValue;
    if (blocks > fit) blocks = fit;
    double* scrInt = (TASK == CBF_TASK_DBSCAN) ? scratch + (size_t)blocks * kBifThreads * J.peakCap : nullptr;
    kern<<<(unsigned)blocks, kBifThreads, smemBytes, s>>>(J, d_out, nullptr, scratch, scrInt, bitWords, err);
    note_launch();
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    int hostErr = 0;
    if ((e = cudaMemcpyAsync(&hostErr, err, sizeof(int), cudaMemcpyDeviceToHost, s)) != cudaSuccess) return e;
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return e;
    return hostErr ? cudaErrorAssert : cudaSuccess;
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
    case CBF_SYS_LORENZ: return launch_bif_prealloc_s<Lorenz>(J, d_out, scratch, scratchBytes, err, s);
    case CBF_SYS_CHEN: return launch_bif_prealloc_s<Chen>(J, d_out, scratch, scratchBytes, err, s);
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_bif(const DevJob& J, void* d_out, int* d_aux, cudaStream_t s)
{
    switch (J.system) {
    case CBF_SYS_MEMRISTIVE5: return launch_bif_s<Memristive5>(J, d_out, d_aux, s);
    case CBF_SYS_ROSSLER: return launch_bif_s<Rossler>(J, d_out, d_aux, s);
    case CBF_SYS_LORENZ: return launch_bif_s<Lorenz>(J, d_out, d_aux, s);
    case CBF_SYS_CHEN: return launch_bif_s<Chen>(J, d_out, d_aux, s);
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace cbf
