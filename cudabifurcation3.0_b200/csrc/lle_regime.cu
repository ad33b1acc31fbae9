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
template <class S, bool IC>
__global__ void __launch_bounds__(kRegThreads, 6) lle_regime_kernel(const DevJob J, double* __restrict__ lle,
                                                                 int* __restrict__ cls, double* scrPk,
                                                                 double* scrIv, int bitWords, int sortCap,
                                                                 int* err)
{
    extern __shared__ unsigned smem[];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const long long warpId = (long long)blockIdx.x * kRegWarps + wib;
    const long long nWarps = (long long)gridDim.x * kRegWarps;
    const long long nTiles = (J.nPoints + 31) / 32;
    const int cap = J.peakCap;
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

// ---------------------------------------------------------------------------
// Plain recompute of a surrogate-refined map in one persistent launch (RefineCtx,
// engine.cuh).

template <class S>
long long resident_s(const DevJob& J);

constexpr int kExpandOnly = 1 << 30;  // queue item: re-expand a computed point (its depth dropped)
constexpr int kQueueEmpty = -1;
// A queue shorter than a tile is taken as a partial tile once it has waited this
// long (a point's integration takes ~0.1 s on a busy device).
constexpr unsigned long long kStarveNs = 20000000ull;

__device__ __forceinline__ unsigned long long vload(const unsigned long long* p)
{
    return *(const volatile unsigned long long*)p;
}

// Make item v visible to the consumers; the pending count rises first, so that
// no warp sees the work finished while v is on its way.
__device__ __forceinline__ void refine_push(const RefineCtx& R, int v)
{
    atomicAdd(&R.counters[3], 1ull);
    const unsigned long long pos = atomicAdd(&R.counters[1], 1ull);
    if (pos < R.qCap) {
        *(volatile int*)&R.queue[pos] = v;
    } else {  // cannot happen for a queue of the planned size; reported, never waited for
        atomicExch(R.err, 3);
        atomicAdd(&R.counters[3], ~0ull);
    }
}

// The neighbours of g (Chebyshev radius) get depth <= d + 1; a neighbour reached
// for the first time is queued for computation, one computed earlier whose depth
// dropped is queued for another expansion if its class surprised.  The fences
// pair with the computing lane's: either that lane reads the lowered depth, or
// this one sees its done/surprised bits.
__device__ void refine_expand(const RefineCtx& R, long long g, int d)
{
    const int row = (int)(g / R.nPts), col = (int)(g % R.nPts);
    const int nd = d + 1;
    atomicMax(&R.stats->deepest, nd);
    for (int dr = -R.radius; dr <= R.radius; ++dr) {
        const int r = row + dr;
        if (r < 0 || r >= R.nPts) continue;
        for (int dc = -R.radius; dc <= R.radius; ++dc) {
            const int q = col + dc;
            if (q < 0 || q >= R.nPts) continue;
            const long long nb = (long long)r * R.nPts + q;
            const int old = atomicMin(&R.depth[nb], nd);
            if (old == kRefUnreached) {
                refine_push(R, (int)nb);
            } else if (nd < old && nd < R.maxDepth) {
                __threadfence();
                const unsigned char f = *(const volatile unsigned char*)&R.flag[nb];
                if ((f & kRefDone) && (f & kRefSurprised)) refine_push(R, (int)nb | kExpandOnly);
            }
        }
    }
}

// Surprised training labels (depth 0) seed the expansion.
__global__ void refine_seed_kernel(const RefineCtx R)
{
    const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= R.nLabel || !R.labelSurprise[k] || R.maxDepth < 1) return;
    refine_expand(R, R.labelIdx[k], 0);
}

// Depth 0 for labels, unreached elsewhere (rule points get theirs below);
// pending = rule count.
__global__ void refine_init_kernel(const RefineCtx R, long long n)
{
    const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (g == 0) R.counters[3] = (unsigned long long)*R.nRule;
    if (g >= n) return;
    R.depth[g] = (R.flag[g] & kRefLabel) ? 0 : kRefUnreached;
}

// Rule point i (ascending grid index) starts at depth i * maxDepth / nRule: the
// rule points enter the expansion spread over its depth levels, so that the
// deepest chain -- and the whole recompute -- ends after about maxDepth tile
// durations however many rule points there are; the rule points late in the
// list get the fewer expansion steps.  Depths stay a pure function of the map
// (the least start depth plus path length over all roots), whatever order the
// warps run in.
__global__ void refine_rule_depth_kernel(const RefineCtx R, long long cap)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long nRule = *R.nRule;
    if (i >= nRule || i >= cap) return;
    R.depth[R.rule[i]] = (int)(((long long)R.maxDepth * i) / nRule);
}

template <class S>
__global__ void __launch_bounds__(kRegThreads, 6) regime_refine_kernel(const DevJob J, const RefineCtx R,
                                                                       double* scrIv, int bitWords, int sortCap)
{
    extern __shared__ unsigned smem[];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const long long warpId = (long long)blockIdx.x * kRegWarps + wib;
    unsigned* L = smem + (size_t)wib * dbscan_warp_words(bitWords, sortCap);
    unsigned* Sb = L + bitWords;
    const DbscanSort so = dbscan_sort_area(L, bitWords, sortCap);
    const long long slot0 = warpId * 32;
    const unsigned long long nRule = (unsigned long long)*R.nRule;

    for (;;) {
        // Lane 0 takes a tile: 32 rule points while any are left, then 32 queued
        // expansion points, and a partial tile of the queue only when no tile in
        // flight can still add to it or fewer than a quarter of the warps are
        // busy.  A warp's FP64
        // instructions cost the pipe the same with 1 active lane as with 32, so
        // partial tiles on a busy device would slow every other tile down.
        unsigned long long base = 0;
        int cnt = 0, fromQueue = 0;
        if (lane == 0) {
            unsigned long long idleSince = 0;
            const unsigned long long quarter = (unsigned long long)gridDim.x * kRegWarps / 4;
            for (;;) {
                const unsigned long long t = vload(&R.counters[1]);
                const unsigned long long tt = t < R.qCap ? t : R.qCap;
                const unsigned long long h = vload(&R.counters[0]);
                const unsigned long long avail = h < tt ? tt - h : 0;
                const bool ruleLeft = vload(&R.counters[2]) < nRule;
                unsigned long long now;
                asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(now));
                bool takeQueue = avail >= 32;
                if (!takeQueue && avail > 0) {
                    if (!ruleLeft && (vload(&R.counters[3]) <= avail || vload(&R.counters[4]) < quarter)) {
                        takeQueue = true;
                    } else {
                        // a short queue may not wait for ever: an expansion chain
                        // stalled here would finish alone at the end, one level
                        // after the other
                        const unsigned long long since = vload(&R.counters[5]);
                        if (since == 0) atomicCAS(&R.counters[5], 0ull, now);
                        else if (now - since > kStarveNs) takeQueue = true;
                    }
                }
                if (takeQueue) {
                    const unsigned long long k = avail < 32 ? avail : 32;
                    if (atomicCAS(&R.counters[0], h, h + k) == h) {
                        atomicExch(&R.counters[5], 0ull);
                        base = h;
                        cnt = (int)k;
                        fromQueue = 1;
                        break;
                    }
                    continue;
                }
                if (ruleLeft) {
                    const unsigned long long r = atomicAdd(&R.counters[2], 32ull);
                    if (r < nRule) {
                        base = r;
                        cnt = (int)(nRule - r < 32 ? nRule - r : 32);
                        break;
                    }
                    continue;
                }
                if (vload(&R.counters[3]) == 0) break;  // nothing queued and nothing in flight
                if (!idleSince) idleSince = now;
                if (now - idleSince > R.maxIdleNs) {
                    atomicExch(R.err, 2);
                    break;
                }
                __nanosleep(2000);
            }
            if (cnt > 0) atomicAdd(&R.counters[4], 1ull);  // busy warps
        }
        cnt = __shfl_sync(kFull, cnt, 0);
        if (cnt == 0) break;
        base = __shfl_sync(kFull, base, 0);
        fromQueue = __shfl_sync(kFull, fromQueue, 0);

        int item = -1;
        if (lane < cnt) {
            if (fromQueue) {
                // the slot was reserved before this warp took it; its value follows shortly
                for (int spin = 0; spin < (1 << 22); ++spin) {
                    item = *(const volatile int*)&R.queue[base + lane];
                    if (item != kQueueEmpty) break;
                    __nanosleep(200);
                }
                if (item == kQueueEmpty) atomicExch(R.err, 4);
            } else {
                item = (int)R.rule[base + lane];
            }
        }
        const bool expandOnly = item >= 0 && (item & kExpandOnly);
        const bool compute = item >= 0 && !expandOnly;
        const long long g = item >= 0 ? (long long)(item & ~kExpandOnly) : 0;

        double lv = 0;
        const int res = regime_tile<S, false>(J, g, compute, cnt, lane, R.scrPk, scrIv, slot0, L, Sb, so, R.err, &lv);

        // merge into the map; statistics of the predictions replaced
        unsigned long long b = 0, lc = 0, au = 0, ao = 0, aa = 0, ch = 0, ex = 0, cp = 0;
        double es = 0, em = 0;
        int d = kRefUnreached;
        bool expand = false;
        if (compute) {
            const unsigned char f = R.flag[g];
            const int pc = R.mapCls[g];
            const double pl = R.mapLle[g];
            const bool sur = pc != res;
            cp = 1;
            b = (f & kRefBoundary) != 0;
            lc = (f & kRefLowConf) != 0;
            au = (f & kRefAudit) != 0;
            ex = (f & kRefReasons) == 0;
            ch = sur;
            if ((f & kRefReasons) == kRefAudit) {
                ao = 1;
                aa = !sur;
                const double e = fabs(pl - lv);
                if (isfinite(e)) es = em = e;
            }
            R.mapLle[g] = lv;
            R.mapCls[g] = res;
            R.src[g] = 2;
            *(volatile unsigned char*)&R.flag[g] = f | kRefDone | (sur ? kRefSurprised : 0);
            __threadfence();
            d = *(const volatile int*)&R.depth[g];
            expand = sur;
        } else if (expandOnly) {
            d = *(const volatile int*)&R.depth[g];
            expand = true;
        }
        if (expand && d < R.maxDepth) refine_expand(R, g, d);
#pragma unroll
        for (int o = 16; o; o >>= 1) {
            b += __shfl_down_sync(kFull, b, o);
            lc += __shfl_down_sync(kFull, lc, o);
            au += __shfl_down_sync(kFull, au, o);
            ao += __shfl_down_sync(kFull, ao, o);
            aa += __shfl_down_sync(kFull, aa, o);
            ch += __shfl_down_sync(kFull, ch, o);
            ex += __shfl_down_sync(kFull, ex, o);
            cp += __shfl_down_sync(kFull, cp, o);
            es += __shfl_down_sync(kFull, es, o);
            em = fmax(em, __shfl_down_sync(kFull, em, o));
        }
        __syncwarp();
        __threadfence();
        if (lane == 0) {
            RefineStats* st = R.stats;
            if (b) atomicAdd(&st->boundary, b);
            if (lc) atomicAdd(&st->lowConf, lc);
            if (au) atomicAdd(&st->audit, au);
            if (ao) atomicAdd(&st->auditOnly, ao);
            if (aa) atomicAdd(&st->auditOnlyAgree, aa);
            if (ch) atomicAdd(&st->changed, ch);
            if (ex) atomicAdd(&st->expanded, ex);
            if (cp) atomicAdd(&st->computed, cp);
            atomicAdd(&st->tiles, 1ull);
            if (es != 0) atomicAdd(&st->errSum, es);
            if (em > 0) atomicMax(&st->errMaxBits, (unsigned long long)__double_as_longlong(em));
            atomicAdd(&R.counters[3], (unsigned long long)(-(long long)cnt));  // this tile is finished
            atomicAdd(&R.counters[4], ~0ull);
        }
    }
}

template <class S>
size_t refine_scratch_bytes_s(const DevJob& J)
{
    const long long resident = resident_s<S>(J);
    return (size_t)resident * J.peakCap * sizeof(double) * 2;
}

template <class S>
cudaError_t launch_refine_s(const DevJob& J, const RefineCtx& R, cudaStream_t s)
{
    const long long n = (long long)R.nPts * R.nPts;
    const int bitWords = (J.peakCap + 31) / 32;
    const int sortCap = dbscan_sort_cap(J.peakCap);
    const size_t smemBytes = (size_t)kRegWarps * dbscan_warp_words(bitWords, sortCap) * sizeof(unsigned);
    auto kern = regime_refine_kernel<S>;
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
    // one block per resident slot (idle warps wait, bounded, for the expansion items of busy ones)
    long long blocks = (long long)sms * perSm;
    const size_t perBlock = (size_t)kRegThreads * J.peakCap * sizeof(double) * 2;
    if ((size_t)blocks * perBlock > R.scrBytes) blocks = (long long)(R.scrBytes / perBlock);
    if (blocks < 1) return cudaErrorInvalidValue;
    refine_init_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(R, n);
    refine_rule_depth_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(R, n);
    note_launch(2);
    if (R.nLabel > 0 && R.maxDepth > 0) {
        refine_seed_kernel<<<(unsigned)((R.nLabel + 255) / 256), 256, 0, s>>>(R);
        note_launch();
    }
    double* scrIv = R.scrPk + (size_t)blocks * kRegThreads * J.peakCap;
    kern<<<(unsigned)blocks, kRegThreads, smemBytes, s>>>(J, R, scrIv, bitWords, sortCap);
    note_launch();
    return cudaGetLastError();
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
        kern<<<(unsigned)blocks, kRegThreads, smemBytes, s>>>(J, d_lle, d_cls, scr, scrIv, bitWords, sortCap, err);
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
    case CBF_SYS_LORENZ: return J.scaledStep ? resident_s<LorenzScaled>(J) : resident_s<Lorenz>(J);
    case CBF_SYS_CHEN: return J.scaledStep ? resident_s<ChenScaled>(J) : resident_s<Chen>(J);
    default: return 0;
    }
}

size_t refine_scratch_bytes(const DevJob& J)
{
    switch (J.system) {
    case CBF_SYS_ROSSLER: return refine_scratch_bytes_s<Rossler>(J);
    case CBF_SYS_LORENZ:
        return J.scaledStep ? refine_scratch_bytes_s<LorenzScaled>(J) : refine_scratch_bytes_s<Lorenz>(J);
    case CBF_SYS_CHEN: return J.scaledStep ? refine_scratch_bytes_s<ChenScaled>(J) : refine_scratch_bytes_s<Chen>(J);
    default: return 0;
    }
}

cudaError_t launch_regime_refine(const DevJob& J, const RefineCtx& R, cudaStream_t s)
{
    switch (J.system) {
    case CBF_SYS_ROSSLER: return launch_refine_s<Rossler>(J, R, s);
    case CBF_SYS_LORENZ: return J.scaledStep ? launch_refine_s<LorenzScaled>(J, R, s) : launch_refine_s<Lorenz>(J, R, s);
    case CBF_SYS_CHEN: return J.scaledStep ? launch_refine_s<ChenScaled>(J, R, s) : launch_refine_s<Chen>(J, R, s);
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_lle_regime(const DevJob& J, double* d_lle, int* d_cls, cudaStream_t s)
{
    switch (J.system) {
    case CBF_SYS_MEMRISTIVE5: return launch_s<Memristive5>(J, d_lle, d_cls, s);
    case CBF_SYS_ROSSLER: return launch_s<Rossler>(J, d_lle, d_cls, s);
    case CBF_SYS_LORENZ: return J.scaledStep ? launch_s<LorenzScaled>(J, d_lle, d_cls, s) : launch_s<Lorenz>(J, d_lle, d_cls, s);
    case CBF_SYS_CHEN: return J.scaledStep ? launch_s<ChenScaled>(J, d_lle, d_cls, s) : launch_s<Chen>(J, d_lle, d_cls, s);
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace cbf
