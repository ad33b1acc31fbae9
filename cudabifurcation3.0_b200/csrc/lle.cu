// Largest Lyapunov exponent maps (Benettin two-trajectory method).
//
// Semantics: LLEKernelCUDA / LLEKernelICCUDA, Library/cudaLibrary.cu:666-908.
// Design (B200): one thread owns one grid point for its whole life; the base
// trajectory x and the perturbed trajectory y live in registers and are advanced
// in the same loop body, giving the scheduler two independent FP64 dependency
// chains per thread (the reference integrates x for NT/h steps, then y, each from
// shared memory).  Parameter-only quantities are hoisted once per point.
//
// Divergence: the reference checks |x[0]| against maxValue after EVERY step and
// stops that integration at the first violation (loopCalculateDiscreteModel,
// cudaLibrary.cu:69-71).  Here each renormalisation interval first runs
// unchecked while folding the high word of |x[0]| and |y[0]| into a running
// integer max (ALU pipe, off the FP64 pipe); only if that max reaches the high
// word of the exact threshold is the interval replayed from a register snapshot
// with the exact per-step check.  Results are identical; the common case pays
// two integer ops per step.
#include "engine.cuh"

namespace cbf {

namespace {

constexpr int kLleThreads = 128;
constexpr int kTransientChunk = 512;

template <class S>
__device__ __forceinline__ void copy_state(double (&d)[S::DIM], const double (&s)[S::DIM])
{
#pragma unroll
    for (int i = 0; i < S::DIM; ++i) d[i] = s[i];
}

// loopCalculateDiscreteModel(x, values, h, n, 1, 0, maxValue, nullptr) for one
// trajectory: n steps, stop after the first step with |x[0]| past the bound.
template <class S>
__device__ __forceinline__ void run_checked(double (&x)[S::DIM], const typename S::Coef& c,
                                            int n, const DevJob& J)
{
    if (!J.checkDiv) {
#pragma unroll 4
        for (int i = 0; i < n; ++i) S::step(x, c);
        return;
    }
    for (int done = 0; done < n; done += kTransientChunk) {
        const int m = min(kTransientChunk, n - done);
        double x0[S::DIM];
        copy_state<S>(x0, x);
        unsigned mx = 0;
#pragma unroll 4
        for (int i = 0; i < m; ++i) {
            S::step(x, c);
            mx = max(mx, abs_hi(x[0]));
        }
        if (mx >= J.divHi) {
            copy_state<S>(x, x0);
            for (int i = 0; i < m; ++i) {
                S::step(x, c);
                if (diverged(x[0], J.divThresh)) return;
            }
        }
    }
}

// The two NT-interval integrations of one renormalisation block
// (cudaLibrary.cu:748-754), interleaved; each stops at its own first violation.
template <class S>
__device__ __forceinline__ void run_pair(double (&x)[S::DIM], double (&y)[S::DIM],
                                         const typename S::Coef& c, int n, const DevJob& J)
{
    if (!J.checkDiv) {
#pragma unroll 2
        for (int i = 0; i < n; ++i) {
            S::step(x, c);
            S::step(y, c);
        }
        return;
    }
    double x0[S::DIM], y0[S::DIM];
    copy_state<S>(x0, x);
    copy_state<S>(y0, y);
    unsigned mx = 0, my = 0;
#pragma unroll 2
    for (int i = 0; i < n; ++i) {
        S::step(x, c);
        S::step(y, c);
        mx = max(mx, abs_hi(x[0]));
        my = max(my, abs_hi(y[0]));
    }
    if (mx >= J.divHi) {
        copy_state<S>(x, x0);
        for (int i = 0; i < n; ++i) {
            S::step(x, c);
            if (diverged(x[0], J.divThresh)) break;
        }
    }
    if (my >= J.divHi) {
        copy_state<S>(y, y0);
        for (int i = 0; i < n; ++i) {
            S::step(y, c);
            if (diverged(y[0], J.divThresh)) break;
        }
    }
}

template <class S, bool IC>
__global__ void __launch_bounds__(kLleThreads) lle_kernel(const DevJob J, double* __restrict__ out)
{
    constexpr int D = S::DIM;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < J.nPoints; p += stride) {
        const long long g = J.firstPoint + p;
        double x[D], v[CBF_MAX_VALUES];
        setup_point<D>(J, g, x, v);
        const typename S::Coef c = S::prep(v, J.h);

        double z[D];
        lle_seed<D, IC>(g, J.seedChunk, z);

        run_checked<S>(x, c, J.nSkip, J);

        double y[D];
#pragma unroll
        for (int i = 0; i < D; ++i) y[i] = z[i] * J.lleEps + x[i];

        double result = 0;
        for (int b = 0; b < J.nRecord; ++b) {
            run_pair<S>(x, y, c, J.nNT, J);
            double t = 0;
#pragma unroll
            for (int l = 0; l < D; ++l) t += (x[l] - y[l]) * (x[l] - y[l]);
            t = sqrt(t) / J.lleEps;
            result += log(t);
            if (t != 0) t = (1 / t);
#pragma unroll
            for (int j = 0; j < D; ++j) y[j] = x[j] - ((x[j] - y[j]) * t);
        }
        out[p] = result / J.tMax;
    }
}

template <int D, bool IC>
__global__ void lle_seed_kernel(const DevJob J, double* __restrict__ out)
{
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= J.nPoints) return;
    double z[D];
    lle_seed<D, IC>(J.firstPoint + p, J.seedChunk, z);
#pragma unroll
    for (int i = 0; i < D; ++i) out[p * D + i] = z[i];
}

template <int D>
cudaError_t launch_seeds_d(const DevJob& J, double* d_out, cudaStream_t s)
{
    const long long blocks = (J.nPoints + 127) / 128;
    if (blocks == 0) return cudaSuccess;
    if (J.sweepIC)
        lle_seed_kernel<D, true><<<(unsigned)blocks, 128, 0, s>>>(J, d_out);
    else
        lle_seed_kernel<D, false><<<(unsigned)blocks, 128, 0, s>>>(J, d_out);
    note_launch();
    return cudaGetLastError();
}

template <class S, bool IC>
cudaError_t launch_lle_t(const DevJob& J, double* d_out, cudaStream_t s)
{
    const long long blocks = (J.nPoints + kLleThreads - 1) / kLleThreads;
    const unsigned grid = (unsigned)(blocks < (1ll << 30) ? blocks : (1ll << 30));
    if (grid == 0) return cudaSuccess;
    lle_kernel<S, IC><<<grid, kLleThreads, 0, s>>>(J, d_out);
    note_launch();
    return cudaGetLastError();
}

template <class S>
cudaError_t launch_lle_s(const DevJob& J, double* d_out, cudaStream_t s)
{
    return J.sweepIC ? launch_lle_t<S, true>(J, d_out, s) : launch_lle_t<S, false>(J, d_out, s);
}

}  // namespace

cudaError_t launch_lle(const DevJob& J, double* d_out, cudaStream_t s)
{
    switch (J.system) {
    case CBF_SYS_MEMRISTIVE5: return launch_lle_s<Memristive5>(J, d_out, s);
    case CBF_SYS_ROSSLER: return launch_lle_s<Rossler>(J, d_out, s);
    case CBF_SYS_LORENZ: return launch_lle_s<Lorenz>(J, d_out, s);
    case CBF_SYS_CHEN: return launch_lle_s<Chen>(J, d_out, s);
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_lle_seeds(const DevJob& J, double* d_out, cudaStream_t s)
{
    switch (J.system) {
    case CBF_SYS_MEMRISTIVE5: return launch_seeds_d<Memristive5::DIM>(J, d_out, s);
    case CBF_SYS_ROSSLER: return launch_seeds_d<Rossler::DIM>(J, d_out, s);
    case CBF_SYS_LORENZ: return launch_seeds_d<Lorenz::DIM>(J, d_out, s);
    case CBF_SYS_CHEN: return launch_seeds_d<Chen::DIM>(J, d_out, s);
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace cbf
