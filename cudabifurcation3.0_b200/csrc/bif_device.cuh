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
    to_stored<S>(x, c);

#pragma unroll 4
    for (int i = 0; i < J.nSkip; ++i) S::step(x, c);

    const int wv = J.writableVar;
    PeakStream ps;
    ps.init();
    bool div = false;
    int t = 0;
    for (; t < J.nRecord; ++t) {
        const double val = phys_comp<S>(pick<D>(x, wv), wv, c);
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
        if (J.checkDiv && diverged(phys_comp<S>(pick<D>(x, wv), wv, c), J.divThresh)) {
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
    const double invH = J.kdeInvH;

    double pp = 0, pr = 0, cur = 0;
    bool strange = false;
    int res = 0;
    for (int base = 0; base < W; base += 32) {
        const int w = base + lane;
        const int cnt = min(32, W - base);
        const double delt = w * k2 + J.kdeI1;
        // delt is monotone in w (rounded products and sums are), so the chunk's
        // samples lie in [dlo, dhi], and rounded subtraction is monotone too: a
        // peak with fl(p - dhi) > skip or fl(p - dlo) < -skip has |fl(p - delt)|
        // > skip for every lane, i.e. it adds exactly +0 everywhere.  One ballot
        // per 32 peaks drops those; the rest are summed in ascending m as before.
        // A NaN bound fails both comparisons and keeps every peak.
        const double dFirst = __shfl_sync(kFull, delt, 0);
        const double dLast = __shfl_sync(kFull, delt, cnt - 1);
        const double dlo = k2 >= 0 ? dFirst : dLast;
        const double dhi = k2 >= 0 ? dLast : dFirst;
        double d2 = 0;
        for (int g = 0; g < n; g += 32) {
            const int m = g + lane;
            const double pv = m < n ? pk[m] : 0.0;
            const bool near = m < n && !(pv - dhi > skip) && !(pv - dlo < -skip);
            unsigned mask = __ballot_sync(kFull, near);
            while (mask) {
                const int j = __ffs(mask) - 1;
                mask &= mask - 1;
                const double dd = __shfl_sync(kFull, pv, j) - delt;
                // |dd| > 16|H| makes the FP32 exponent argument <= -128, where expf
                // is exactly +0 (checked exhaustively on the device by
                // cbf_probe_expf_zero), and adding +0 leaves the sum unchanged.
                if (w < W && !(fabs(dd) > skip)) {
                    const double tmp = invH != 0.0 ? dd * invH : dd / H;
                    d2 += (double)expf((float)(-((tmp * tmp) / 2)));
                }
            }
        }
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
// DBSCAN (dbscan, cudaLibrary.cu:457-529), whole warp per point.
//
// helpfulArray[k] (label, nonzero once set) -> bitset L; helpfulArray[n+k] (the
// "stack", holds k or 0) -> bitset S: popping slot m yields m if set, else 0.
// One scan of a centre c adds to L and S exactly the set
//     {k < n-1 : k != c, k unlabelled, near(c, k)}
// and counts it into the stack depth.  The reference visits k in ascending
// order, but each k once, and nothing it sets is read again within the scan,
// so the order is immaterial.  Three facts make most scans avoidable without
// changing any label, stack bit or count:
//   * a scan of a centre with no near k at all adds nothing ("scan-empty");
//   * a second scan of a centre adds nothing (its near k are all labelled
//     after the first, and labels are never cleared);
//   * once every k < n-1 is labelled, no scan adds anything.
// A neighbour has |fl(p_k - p_c)| < skip (skip = 4 eps bounds the FP32 hypot
// from below), hence p_k in [A, B] = p_c -/+ (2 skip + 4 ulp(p_c)) (rounded).
// The peaks are sorted by a 32-bit key: the top 22 bits of an order-preserving
// encoding of float(p_k) over the 10-bit index k.  Rounding to float and
// truncating are monotone, so every candidate's key lies between the keys of A
// and B: one window of sorted positions.  The scan-empty marks come from a few
// probes per peak, and a real scan tests the window only, each candidate with
// the exact test.  Chaotic points -- hundreds of peaks, almost all of them
// singleton clusters -- then cost a sort and a word-wise walk instead of n
// scans over n peaks.
constexpr int kDbscanIdxBits = 10;
constexpr int kDbscanSortCap = 1 << kDbscanIdxBits;  // scanned peaks (n - 1) a warp sorts
constexpr unsigned kDbscanIdxMask = (1u << kDbscanIdxBits) - 1u;
constexpr int kDbscanProbes = 32;  // per peak, in the scan-empty test; more: not marked

struct DbscanSort {
    unsigned* key = nullptr;  // sorted (coarse value << 10 | index)
    unsigned* E = nullptr;    // scan-empty marks (bitset)
    unsigned* D = nullptr;    // centres scanned once (bitset)
    int cap = 0;              // entries of key; 0: no sorted path
};

// 32-bit words of shared memory per warp: the bitsets L and S of `bitWords`
// words each, and with `sortCap` > 0 (a power of two, 32..1024) also E, D and
// the sort keys.
__host__ __device__ inline int dbscan_warp_words(int bitWords, int sortCap)
{
    return sortCap > 0 ? 4 * bitWords + sortCap : 2 * bitWords;
}

// Sort keys per warp for peak lists of up to `peakCap` peaks: a power of two
// >= 32, or 0 (no sorted path) when peakCap exceeds kDbscanSortCap.
__host__ __device__ inline int dbscan_sort_cap(int peakCap)
{
    if (peakCap > kDbscanSortCap) return 0;
    int c = 32;
    while (c < peakCap) c <<= 1;
    return c;
}

__device__ inline DbscanSort dbscan_sort_area(unsigned* warpWords, int bitWords, int sortCap)
{
    DbscanSort so;
    if (sortCap > 0) {
        so.E = warpWords + 2 * bitWords;
        so.D = so.E + bitWords;
        so.key = so.D + bitWords;
        so.cap = sortCap;
    }
    return so;
}

// Top 22 bits of an order-preserving encoding of float(v): non-decreasing in v
// (-0 is folded onto +0).
__device__ __forceinline__ unsigned dbscan_coarse(double v)
{
    float f = (float)v;
    if (f == 0.0f) f = 0.0f;
    const unsigned u = __float_as_uint(f);
    return ((u & 0x80000000u) ? ~u : (u | 0x80000000u)) >> kDbscanIdxBits;
}

// distance(...) < eps of the reference (cudaLibrary.cu:445-453) with c = (x1, y1)
// the centre: 0 on exact equality, else the FP32 hypot of the double
// differences.  hypotf(dx, dy) >= max(|dx|, |dy|) up to a few ulps, so a
// coordinate gap >= skip = 4 eps can never be closer than eps.
__device__ __forceinline__ bool dbscan_near(double x1, double y1, double x2, double y2, double eps,
                                            double skip)
{
    if (x1 == x2 && y1 == y2) return 0.0 < eps;
    const double dx = x2 - x1;
    const double dy = y2 - y1;
    if (fabs(dx) >= skip || fabs(dy) >= skip) return false;
    return (double)hypotf((float)dx, (float)dy) < eps;
}

// Bitonic sort of the first P = 2^k >= M keys; the entries past M are
// 0xffffffff and sort last (no finite value reaches that key).  Returns false
// if a value is not finite (the caller then keeps the chunked scans).
__device__ bool dbscan_sort(const DbscanSort& so, const double* pk, int M, int P, int lane)
{
    bool bad = false;
    for (int k = lane; k < P; k += 32) {
        unsigned key = 0xffffffffu;
        if (k < M) {
            const double v = pk[k];
            if (!isfinite(v)) bad = true;
            key = (dbscan_coarse(v) << kDbscanIdxBits) | (unsigned)k;
        }
        so.key[k] = key;
    }
    if (__any_sync(kFull, bad)) return false;
    __syncwarp();
    for (int size = 2; size <= P; size <<= 1) {
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            for (int t = lane; t < (P >> 1); t += 32) {
                const int i = 2 * t - (t & (stride - 1));
                const int j = i + stride;
                const unsigned ki = so.key[i], kj = so.key[j];
                if ((ki > kj) == ((i & size) == 0)) {
                    so.key[i] = kj;
                    so.key[j] = ki;
                }
            }
            __syncwarp();
        }
    }
    return true;
}

// Coarse keys bounding the candidates of a centre at x1 (finite): every k with
// |fl(p_k - x1)| < skip has p_k within x1 -/+ (2 skip + 4 ulp(x1)).
__device__ __forceinline__ void dbscan_bounds(double x1, double skip, unsigned& cA, unsigned& cB)
{
    const double half = 2.0 * skip + fabs(x1) * 0x1p-50;
    cA = dbscan_coarse(x1 - half);
    cB = dbscan_coarse(x1 + half);
}

// Scan-empty marks: E[c] set iff no k < M (k != c) is near c, found by probing
// the sorted neighbours of c outwards while their keys stay within c's bounds.
// A peak with more than kDbscanProbes probes, and the unsorted last peak, stay
// unmarked (their scans run).  E and D are cleared here.
__device__ void dbscan_mark_empty(const DbscanSort& so, const double* pk, const double* iv, int n, int M,
                                  double eps, double skip, int lane)
{
    const int words = (n + 31) >> 5;
    for (int w = lane; w < words; w += 32) {
        so.E[w] = 0u;
        so.D[w] = 0u;
    }
    __syncwarp();
    for (int pos = lane; pos < M; pos += 32) {
        const int c = (int)(so.key[pos] & kDbscanIdxMask);
        const double x1 = pk[c];
        const double y1 = iv[c];
        unsigned cA, cB;
        dbscan_bounds(x1, skip, cA, cB);
        bool near = false;
        int probes = 0;
        for (int q = pos + 1; q < M && !near; ++q) {
            const unsigned kq = so.key[q];
            if ((kq >> kDbscanIdxBits) > cB) break;
            if (++probes > kDbscanProbes) { near = true; break; }
            const int k = (int)(kq & kDbscanIdxMask);
            near = dbscan_near(x1, y1, pk[k], iv[k], eps, skip);
        }
        for (int q = pos - 1; q >= 0 && !near; --q) {
            const unsigned kq = so.key[q];
            if ((kq >> kDbscanIdxBits) < cA) break;
            if (++probes > kDbscanProbes) { near = true; break; }
            const int k = (int)(kq & kDbscanIdxMask);
            near = dbscan_near(x1, y1, pk[k], iv[k], eps, skip);
        }
        if (!near) atomicOr(&so.E[c >> 5], 1u << (c & 31));
    }
    __syncwarp();
}

// Number of sorted positions < M whose coarse value c satisfies pred(c), for a
// predicate true on a prefix: the last entry of each of 32 segments first (the
// non-empty segments whose last entry passes are a prefix of the lanes), then
// the entries of the first segment whose last entry fails.
template <class Pred>
__device__ int dbscan_prefix(const unsigned* key, int M, int lane, Pred pred)
{
    const int seg = (M + 31) >> 5;
    const int first = lane * seg;
    const bool in1 = first < M && pred(key[min(first + seg, M) - 1] >> kDbscanIdxBits);
    const int c = __popc(__ballot_sync(kFull, in1));
    const int pos = c * seg + lane;
    const bool in2 = lane < seg && pos < M && pred(key[pos] >> kDbscanIdxBits);
    return min(M, c * seg + __popc(__ballot_sync(kFull, in2)));
}

// The scan of `center` over k = 0..M-1 in chunks of 32 (label word per chunk).
// Returns the number of indices added to L and S.
__device__ int dbscan_scan_chunked(const double* pk, const double* iv, int M, int center, double x1,
                                   double y1, double eps, double skip, unsigned* L, unsigned* Sb,
                                   int lane)
{
    int added = 0;
    for (int base = 0; base < M; base += 32) {
        const int k = base + lane;
        bool cand = false;
        if (k < M && k != center && !((L[base >> 5] >> lane) & 1u))
            cand = dbscan_near(x1, y1, pk[k], iv[k], eps, skip);
        const unsigned b = __ballot_sync(kFull, cand);
        if (b) {
            if (lane == 0) {
                L[base >> 5] |= b;
                Sb[base >> 5] |= b;
            }
            added += __popc(b);
        }
    }
    return added;
}

// The scan of `center` over the sorted positions [lo, hi) that hold every
// candidate.  Returns the number of indices added to L and S.
__device__ int dbscan_scan_window(const DbscanSort& so, const double* pk, const double* iv, int lo, int hi,
                                  int center, double x1, double y1, double eps, double skip, unsigned* L,
                                  unsigned* Sb, int lane)
{
    int added = 0;
    for (int base = lo; base < hi; base += 32) {
        const int pos = base + lane;
        bool cand = false;
        int k = 0;
        if (pos < hi) {
            k = (int)(so.key[pos] & kDbscanIdxMask);
            if (k != center && !((L[k >> 5] >> (k & 31)) & 1u))
                cand = dbscan_near(x1, y1, pk[k], iv[k], eps, skip);
        }
        const unsigned b = __ballot_sync(kFull, cand);
        if (b) {
            if (cand) {
                atomicOr(&L[k >> 5], 1u << (k & 31));
                atomicOr(&Sb[k >> 5], 1u << (k & 31));
            }
            added += __popc(b);
        }
    }
    return added;
}

// First index j >= i that is unlabelled and not scan-empty, or n.
__device__ int dbscan_next_open(const unsigned* L, const unsigned* E, int n, int i, int lane)
{
    const int words = (n + 31) >> 5;
    for (int w0 = i >> 5; w0 < words; w0 += 32) {
        const int w = w0 + lane;
        unsigned open = 0u;
        if (w < words) {
            open = ~L[w] & ~E[w];
            if (w == (i >> 5)) open &= ~0u << (i & 31);
            if (w == words - 1 && (n & 31)) open &= (1u << (n & 31)) - 1u;
        }
        const unsigned b = __ballot_sync(kFull, open != 0u);
        if (b) {
            const int f = __ffs(b) - 1;
            const unsigned ow = __shfl_sync(kFull, open, f);
            return ((w0 + f) << 5) + __ffs(ow) - 1;
        }
    }
    return n;
}

// The reference's walk over i in [i, j) with an empty stack, where every
// unlabelled index is scan-empty: labelled ones are no-ops, each unlabelled one
// opens a cluster, is labelled, and its scan adds nothing.  Labels them all;
// returns (clusters opened, of which among the scanned indices < M).
__device__ int2 dbscan_open_run(unsigned* L, int i, int j, int M, int lane)
{
    int opened = 0, openedScanned = 0;
    const int wEnd = (j - 1) >> 5;
    for (int w0 = i >> 5; w0 <= wEnd; w0 += 32) {
        const int w = w0 + lane;
        unsigned m = 0u;
        if (w <= wEnd) {
            m = ~L[w];
            if (w == (i >> 5)) m &= ~0u << (i & 31);
            const int top = j - (w << 5);  // >= 1: bits below it lie in [i, j)
            if (top < 32) m &= (1u << top) - 1u;
            if (m) L[w] |= m;
        }
        const int c = __popc(m);
        const int cLast = (w <= wEnd && (M >> 5) == w) ? (int)((m >> (M & 31)) & 1u) : 0;
        opened += __reduce_add_sync(kFull, c);
        openedScanned += __reduce_add_sync(kFull, c - cLast);
    }
    __syncwarp();
    return make_int2(opened, openedScanned);
}

// DBSCAN cluster count of one point; `so` (shared memory of this warp) enables
// the sorted path for points with n - 1 <= so.cap peaks.
__device__ int dbscan_warp(const DevJob& J, const double* pk,
                           const double* iv, int n, int lane, unsigned* L,
                           unsigned* Sb, int* err, DbscanSort so = DbscanSort())
{
    if (n <= 0) return 0;
    if (n == 1) return 1;
    if (n > J.maxPeaks) return 0;

    const int words = (n + 31) >> 5;
    for (int w = lane; w < words; w += 32) {
        L[w] = 0u;
        Sb[w] = 0u;
    }

    const double eps = J.dbEps;
    const double skip = J.dbSkip;
    const int M = n - 1;  // indices 0..n-2 are scanned; the last peak never is
    int P = 32;
    while (P < M) P <<= 1;
    const bool sorted = so.cap > 0 && M <= so.cap && skip > 0 && isfinite(skip) &&
                        dbscan_sort(so, pk, M, P, lane);
    if (sorted) dbscan_mark_empty(so, pk, iv, n, M, eps, skip, lane);
    __syncwarp();

    int cluster = 0;
    int num = 0;
    int nlab = 0;  // labels set among the scanned indices 0..n-2
    long long guard = (long long)n * n + 4ll * n + 16;
    for (int i = 0; i < n; i++) {
        if (--guard < 0) {
            if (lane == 0) atomicExch(err, 1);
            return 0;
        }
        if (sorted && num == 0) {
            const int j = dbscan_next_open(L, so.E, n, i, lane);
            if (j > i) {
                const int2 r = dbscan_open_run(L, i, j, M, lane);
                cluster += r.x;
                nlab += r.y;
                guard -= j - i;
                i = j;
                if (i >= n) break;
            }
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
            if (i < M) ++nlab;
        }
        if (center < 0 || nlab >= M) continue;

        const double x1 = pk[center];
        const double y1 = iv[center];
        int added;
        if (sorted) {
            const unsigned bit = 1u << (center & 31);
            if ((so.E[center >> 5] | so.D[center >> 5]) & bit) continue;
            if (lane == 0) so.D[center >> 5] |= bit;
        }
        if (sorted && isfinite(x1)) {
            unsigned cA, cB;
            dbscan_bounds(x1, skip, cA, cB);
            const int lo = dbscan_prefix(so.key, M, lane, [cA](unsigned c) { return c < cA; });
            const int hi = dbscan_prefix(so.key, M, lane, [cB](unsigned c) { return c <= cB; });
            if (2 * (hi - lo) <= M)
                added = dbscan_scan_window(so, pk, iv, lo, hi, center, x1, y1, eps, skip, L, Sb, lane);
            else
                added = dbscan_scan_chunked(pk, iv, M, center, x1, y1, eps, skip, L, Sb, lane);
        } else {
            added = dbscan_scan_chunked(pk, iv, M, center, x1, y1, eps, skip, L, Sb, lane);
        }
        num += added;
        nlab += added;
        __syncwarp();
    }
    return cluster - 1;
}

}  // namespace
}  // namespace cbf
