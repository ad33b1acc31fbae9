// Per-point device code of the fused bifurcation kernel: the streaming peak
// finder, the per-point integration and the warp-cooperative KDE / DBSCAN
// epilogues.  Shared by the map kernel (bif.cu) and the batch kernel (batch.cu).
#pragma once

#include "engine.cuh"

namespace cbf {
namespace {

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
struct NoPeakHook {
    __device__ __forceinline__ void operator()(double, int) const {}
};

// Flags of peakFinderCUDAForCalculationOfPeriodicityByOstrovsky
// (cudaLibrary.cu:288-352) kept while the peaks stream by, over every peak:
// non-increasing consecutive peaks (flag 0), peaks from the second on above /
// not above the threshold (flags 1, 2), and the last recorded sample (flag 4).
struct OstrovskyFlags {
    double prev, last, thr;
    bool nonInc, one, zero;
    __device__ __forceinline__ void init(double threshold)
    {
        thr = threshold;
        prev = last = 0.0;
        nonInc = true;
        one = zero = false;
    }
    __device__ __forceinline__ void operator()(double val, int k)
    {
        if (k >= 1) {
            if (val - prev > 0) nonInc = false;
            if (val > thr) one = true;
            else zero = true;
        }
        prev = val;
    }
};

// dbscanCUDAForCalculationOfPeriodicityByOstrovsky (cudaLibrary.cu:628-662):
// the cluster count (dbscanDouble = dbscan as a double) rewritten by the flags.
// A diverged point has flag 3 only: the reference never writes its other flags,
// which are false on zero-filled memory.
__device__ __forceinline__ double ostrovsky_value(int n, bool div, const OstrovskyFlags& f, int clusters)
{
    bool f0, f1, f2, f3, f4;
    if (div) {
        f0 = f1 = f2 = f4 = false;
        f3 = true;
    } else {
        f0 = f.nonInc;
        f1 = f.one && f.zero;
        f2 = !(f.one && !f.zero);
        f3 = (n == 0 || n == 1);
        f4 = f.last > f.thr;
    }
    double out = (double)clusters;
    if (f2) out = -1 * out;
    if (f3) out = f4 ? 1 : -1;
    if (f1) out = 0;
    if (f0) out = out > 0 ? 0.5 : (out == 0 ? 0 : -0.5);
    return out;
}

// Tasks whose peaks carry intervals (DBSCAN on (peak, interval) pairs).
__host__ __device__ constexpr bool task_with_intervals(int task)
{
    return task == CBF_TASK_DBSCAN || task == CBF_TASK_OSTROVSKY;
}

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

    // hook(value, k) sees every emitted peak k = 0, 1, ... (also past cap).
    template <bool WITH_INTERVALS, class Hook>
    __device__ __forceinline__ void emit(double val, int t, double* pk, double* iv, int cap, Hook& hook)
    {
        if (detected >= 1) {
            const int k = detected - 1;
            hook(val, k);
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
        NoPeakHook h;
        push<WITH_INTERVALS>(v, t, pk, iv, cap, h);
    }

    template <bool WITH_INTERVALS, class Hook>
    __device__ __forceinline__ void push(double v, int t, double* pk, double* iv, int cap, Hook& hook)
    {
        if (t >= 2) {
            if (mode == 2) {
                mode = 0;
            } else if (mode == 1) {
                if (pval < v) {
                    mode = 2;
                } else if (pval > v) {
                    emit<WITH_INTERVALS>(pval, t - 1, pk, iv, cap, hook);
                    mode = 2;
                }
            } else if (prev1 > prev2 && prev1 >= v) {
                if (prev1 > v) {
                    emit<WITH_INTERVALS>(prev1, t - 1, pk, iv, cap, hook);
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
                               double* traj, int* divFlag, OstrovskyFlags* of = nullptr)
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
        if (TASK == CBF_TASK_TRAJECTORY) {
            traj[t] = val;
        } else if (TASK == CBF_TASK_OSTROVSKY) {
            of->last = val;
            ps.push<true>(val, t, pk, iv, cap, *of);
        } else {
            ps.push<task_with_intervals(TASK)>(val, t, pk, iv, cap);
        }
        for (int j = 0; j < J.preScaller - 1; ++j) S::step(x, c);
        S::step(x, c);
        if (J.checkDiv && diverged(pick<D>(x, wv), J.divThresh)) {
            div = true;
            ++t;
            break;
        }
    }
    if (TASK == CBF_TASK_OSTROVSKY) *divFlag = div ? 1 : 0;
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

}  // namespace
}  // namespace cbf
