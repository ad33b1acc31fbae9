// Largest Lyapunov exponent maps (Benettin two-trajectory method).
//
// Semantics: LLEKernelCUDA / LLEKernelICCUDA, Library/cudaLibrary.cu:666-908.
// Design (B200): a thread owns PPT grid points (1 or 2) for their whole life;
// for each point the base trajectory x and the perturbed trajectory y live in
// registers and are advanced in the same loop body, giving the scheduler 2*PPT
// independent FP64 dependency chains per thread (the reference integrates x for
// NT/h steps, then y, each from shared memory).  Parameter-only quantities are
// hoisted once per point.  The kernel is instantiated in a few shapes (points per
// thread, block size, register cap); the autotuner in capi.cu times them on the
// device and picks one per system.
//
// Divergence: the reference checks |x[0]| against maxValue after EVERY step and
// stops that integration at the first violation (loopCalculateDiscreteModel,
// cudaLibrary.cu:69-71).  Here each renormalisation interval first runs
// unchecked while folding the high word of |x[0]| and |y[0]| into a running
// integer max (ALU pipe, off the FP64 pipe); only if that max reaches the high
// word of the exact threshold is the interval replayed from a register snapshot
// with the exact per-step check.  Results are identical; the common case pays
// two integer ops per step.
#include "lle_device.cuh"

namespace cbf {

namespace {

template <class S, bool IC, int PPT, int THREADS, int MINB, int UNR>
__global__ void __launch_bounds__(THREADS, MINB) lle_kernel(const DevJob J, double* __restrict__ out)
{
    constexpr int D = S::DIM;
    const long long nq = (J.nPoints + PPT - 1) / PPT;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < nq; q += stride) {
        double x[PPT][D], y[PPT][D];
        typename S::Coef c[PPT];
#pragma unroll
        for (int j = 0; j < PPT; ++j) {
            long long p = q * PPT + j;
            if (p >= J.nPoints) p = J.nPoints - 1;  // tail lane repeats a point, never stores it
            double v[CBF_MAX_VALUES];
            setup_point<D>(J, grid_index(J, p), x[j], v);
            c[j] = S::prep(v, J.h);
            to_stored<S>(x[j], c[j]);
        }

        run_checked<S, PPT, UNR>(x, c, J.nSkip, J);

#pragma unroll
        for (int j = 0; j < PPT; ++j) {
            long long p = q * PPT + j;
            if (p >= J.nPoints) p = J.nPoints - 1;
            double z[D];
            lle_seed<D, IC>(grid_index(J, p), J.seedChunk, z);
#pragma unroll
            for (int i = 0; i < D; ++i) y[j][i] = stored_comp<S>(z[i] * J.lleEps, i, c[j]) + x[j][i];
        }

        double result[PPT];
#pragma unroll
        for (int j = 0; j < PPT; ++j) result[j] = 0;
        for (int b = 0; b < J.nRecord; ++b) {
            run_pair<S, PPT, UNR>(x, y, c, J.nNT, J);
#pragma unroll
            for (int j = 0; j < PPT; ++j) {
                double t = 0;
#pragma unroll
                for (int l = 0; l < D; ++l) {
                    const double d = phys_comp<S>(x[j][l] - y[j][l], l, c[j]);
                    t += d * d;
                }
                t = sqrt(t) / J.lleEps;
                result[j] += log(t);
                if (t != 0) t = (1 / t);
#pragma unroll
                for (int i = 0; i < D; ++i) y[j][i] = x[j][i] - ((x[j][i] - y[j][i]) * t);
            }
        }
#pragma unroll
        for (int j = 0; j < PPT; ++j) {
            const long long p = q * PPT + j;
            if (p < J.nPoints) out[p] = result[j] / J.tMax;
        }
    }
}

template <int D, bool IC>
__global__ void lle_seed_kernel(const DevJob J, double* __restrict__ out)
{
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= J.nPoints) return;
    double z[D];
    lle_seed<D, IC>(grid_index(J, p), J.seedChunk, z);
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

template <class S, bool IC, int PPT, int THREADS, int MINB, int UNR = 2>
cudaError_t launch_variant(const DevJob& J, double* d_out, cudaStream_t s)
{
    const long long nq = (J.nPoints + PPT - 1) / PPT;
    const long long blocks = (nq + THREADS - 1) / THREADS;
    const unsigned grid = (unsigned)(blocks < (1ll << 30) ? blocks : (1ll << 30));
    if (grid == 0) return cudaSuccess;
    lle_kernel<S, IC, PPT, THREADS, MINB, UNR><<<grid, THREADS, 0, s>>>(J, d_out);
    note_launch();
    return cudaGetLastError();
}

// The kernel shapes the autotuner chooses from: {points per thread, threads per
// block, minimum resident blocks per SM (a register cap for the compiler),
// unrolling of the step loop}.
//   0: 1 pt, 128 thr, >= 8 blocks/SM  (<= 64 registers, 32 warps/SM), unroll 2  default
//   1: 1 pt, 128 thr, no cap, unroll 2
//   2: 1 pt, 256 thr, >= 4 blocks/SM  (<= 64 registers), unroll 2
//   3: 2 pt, 128 thr, >= 4 blocks/SM  (<= 128 registers, 4 chains per thread), unroll 2
//   4: 2 pt, 128 thr, >= 3 blocks/SM  (<= 170 registers), unroll 2
//   5: 1 pt, 128 thr, no cap, unroll 4
//   6: 1 pt, 128 thr, >= 8 blocks/SM, unroll 4
//   7: 1 pt, 128 thr, no cap, unroll 8
template <class S, bool IC>
cudaError_t launch_lle_v(const DevJob& J, double* d_out, cudaStream_t s, int variant)
{
    switch (variant) {
    case 1: return launch_variant<S, IC, 1, 128, 1>(J, d_out, s);
    case 2: return launch_variant<S, IC, 1, 256, 4>(J, d_out, s);
    case 3: return launch_variant<S, IC, 2, 128, 4>(J, d_out, s);
    case 4: return launch_variant<S, IC, 2, 128, 3>(J, d_out, s);
    case 5: return launch_variant<S, IC, 1, 128, 1, 4>(J, d_out, s);
    case 6: return launch_variant<S, IC, 1, 128, 8, 4>(J, d_out, s);
    case 7: return launch_variant<S, IC, 1, 128, 1, 8>(J, d_out, s);
    default: return launch_variant<S, IC, 1, 128, 8>(J, d_out, s);
    }
}

template <class S>
cudaError_t launch_lle_s(const DevJob& J, double* d_out, cudaStream_t s, int variant)
{
    return J.sweepIC ? launch_lle_v<S, true>(J, d_out, s, variant)
                     : launch_lle_v<S, false>(J, d_out, s, variant);
}

}  // namespace

cudaError_t launch_lle_variant(const DevJob& J, double* d_out, cudaStream_t s, int variant)
{
    switch (J.system) {
    case CBF_SYS_MEMRISTIVE5: return launch_lle_s<Memristive5>(J, d_out, s, variant);
    case CBF_SYS_ROSSLER: return launch_lle_s<Rossler>(J, d_out, s, variant);
    case CBF_SYS_LORENZ: return J.scaledStep ? (J.unitStep ? launch_lle_s<LorenzScaledU>(J, d_out, s, variant) : launch_lle_s<LorenzScaled>(J, d_out, s, variant)) : launch_lle_s<Lorenz>(J, d_out, s, variant);
    case CBF_SYS_CHEN: return J.scaledStep ? (J.unitStep ? launch_lle_s<ChenScaledU>(J, d_out, s, variant) : launch_lle_s<ChenScaled>(J, d_out, s, variant)) : launch_lle_s<Chen>(J, d_out, s, variant);
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_lle(const DevJob& J, double* d_out, cudaStream_t s)
{
    return launch_lle_variant(J, d_out, s, lle_variant_for(J.system));
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
