// Per-point device code of the LLE kernels: checked integration with the exact
// divergence semantics and the paired x/y renormalisation intervals.  Shared by
// the map kernel (lle.cu) and the batch kernel (batch.cu).
#pragma once

#include "engine.cuh"

namespace cbf {
namespace {

constexpr int kTransientChunk = 512;

template <int D>
__device__ __forceinline__ void copy_state(double (&d)[D], const double (&s)[D])
{
#pragma unroll
    for (int i = 0; i < D; ++i) d[i] = s[i];
}

// loopCalculateDiscreteModel(x, values, h, n, 1, 0, maxValue, nullptr) for PPT
// independent points: n steps each, a point stops after its first step with
// |x[0]| past the bound and stays stopped for the rest of the call.  UNR: the
// unrolling of the step loop (a kernel-shape parameter).
template <class S, int PPT, int UNR = 2>
__device__ __forceinline__ void run_checked(double (&x)[PPT][S::DIM],
                                            const typename S::Coef (&c)[PPT], int n,
                                            const DevJob& J)
{
    if (!J.checkDiv) {
#pragma unroll UNR
        for (int i = 0; i < n; ++i) {
#pragma unroll
            for (int j = 0; j < PPT; ++j) S::step(x[j], c[j]);
        }
        return;
    }
    bool alive[PPT];
#pragma unroll
    for (int j = 0; j < PPT; ++j) alive[j] = true;
    for (int done = 0; done < n; done += kTransientChunk) {
        const int m = min(kTransientChunk, n - done);
        double x0[PPT][S::DIM];
        HiTrack tr[PPT];
#pragma unroll
        for (int j = 0; j < PPT; ++j) {
            copy_state<S::DIM>(x0[j], x[j]);
            tr[j].init();
        }
        // two steps per update of the tracker
#pragma unroll UNR
        for (int i = 0; i + 1 < m; i += 2) {
#pragma unroll
            for (int j = 0; j < PPT; ++j) {
                S::step(x[j], c[j]);
                const double a = x[j][0];
                S::step(x[j], c[j]);
                tr[j].add2(a, x[j][0]);
            }
        }
        if (m & 1) {
#pragma unroll
            for (int j = 0; j < PPT; ++j) {
                S::step(x[j], c[j]);
                tr[j].add1(x[j][0]);
            }
        }
#pragma unroll
        for (int j = 0; j < PPT; ++j) {
            if (!alive[j]) {
                copy_state<S::DIM>(x[j], x0[j]);  // stopped earlier: state frozen
            } else if (tr[j].maybe(J.divHi)) {
                copy_state<S::DIM>(x[j], x0[j]);
                for (int i = 0; i < m; ++i) {
                    S::step(x[j], c[j]);
                    if (diverged(x[j][0], J.divThresh)) {
                        alive[j] = false;
                        break;
                    }
                }
            }
        }
    }
}

// The two NT-interval integrations of one renormalisation block
// (cudaLibrary.cu:748-754) for PPT points, interleaved; each trajectory stops at
// its own first violation within the interval.
template <class S, int PPT, int UNR = 2>
__device__ __forceinline__ void run_pair(double (&x)[PPT][S::DIM], double (&y)[PPT][S::DIM],
                                         const typename S::Coef (&c)[PPT], int n, const DevJob& J)
{
    if (!J.checkDiv) {
#pragma unroll UNR
        for (int i = 0; i < n; ++i) {
#pragma unroll
            for (int j = 0; j < PPT; ++j) {
                S::step(x[j], c[j]);
                S::step(y[j], c[j]);
            }
        }
        return;
    }
    double x0[PPT][S::DIM], y0[PPT][S::DIM];
    HiTrack tr[PPT];  // x and y of a point share one tracker
#pragma unroll
    for (int j = 0; j < PPT; ++j) {
        copy_state<S::DIM>(x0[j], x[j]);
        copy_state<S::DIM>(y0[j], y[j]);
        tr[j].init();
    }
#pragma unroll UNR
    for (int i = 0; i < n; ++i) {
#pragma unroll
        for (int j = 0; j < PPT; ++j) {
            S::step(x[j], c[j]);
            S::step(y[j], c[j]);
            tr[j].add2(x[j][0], y[j][0]);
        }
    }
#pragma unroll
    for (int j = 0; j < PPT; ++j) {
        if (tr[j].maybe(J.divHi)) {  // either trajectory may have stopped: replay both exactly
            copy_state<S::DIM>(x[j], x0[j]);
            for (int i = 0; i < n; ++i) {
                S::step(x[j], c[j]);
                if (diverged(x[j][0], J.divThresh)) break;
            }
            copy_state<S::DIM>(y[j], y0[j]);
            for (int i = 0; i < n; ++i) {
                S::step(y[j], c[j]);
                if (diverged(y[j][0], J.divThresh)) break;
            }
        }
    }
}

// One point of LLEKernelCUDA / LLEKernelICCUDA (cudaLibrary.cu:666-908).
template <class S, bool IC>
__device__ __forceinline__ double lle_point(const DevJob& J, long long g)
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
    double z[D];
    lle_seed<D, IC>(g, J.seedChunk, z);
#pragma unroll
    for (int i = 0; i < D; ++i) y[0][i] = stored_comp<S>(z[i] * J.lleEps, i, c[0]) + x[0][i];
    double result = 0;
    for (int b = 0; b < J.nRecord; ++b) {
        run_pair<S, 1>(x, y, c, J.nNT, J);
        double t = 0;
#pragma unroll
        for (int l = 0; l < D; ++l) {
            const double d = phys_comp<S>(x[0][l] - y[0][l], l, c[0]);
            t += d * d;
        }
        t = sqrt(t) / J.lleEps;
        result += log(t);
        if (t != 0) t = (1 / t);
#pragma unroll
        for (int i = 0; i < D; ++i) y[0][i] = x[0][i] - ((x[0][i] - y[0][i]) * t);
    }
    return result / J.tMax;
}

}  // namespace
}  // namespace cbf
