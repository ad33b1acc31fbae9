// Lyapunov spectrum maps (LSKernelCUDA, cudaLibrary.cu:960-1100; host drivers
// LS1D / LS2D, hostLibrary.cu:1802-2082).
//
// One thread = one grid point for its whole life: the base trajectory and the D
// perturbation vectors (D = the system's dimension) stay in registers, and the
// D+1 trajectories of a renormalisation interval are advanced in one loop body
// -- D+1 independent FP64 dependency chains per thread, where the reference runs
// them one after the other from shared memory.  Each trajectory stops at its own
// first divergence-test violation in the interval, as the reference's separate
// loopCalculateDiscreteModel calls do (unchecked run with the high-word max on
// the ALU pipe, exact replay only when the threshold's high word is reached).
// After every interval the deviations are orthonormalised by the reference's
// classical Gram-Schmidt (projections against the not yet normalised earlier
// rows, then normalisation; cudaLibrary.cu:913-956) in its operation order, and
// log(norm / eps) accumulates into each exponent.  The reference's zeroing of
// the result on divergence is overwritten by its final store, so only the early
// stop has an effect, and only that is reproduced.
#include "lle_device.cuh"

namespace cbf {
namespace {

constexpr int kLsThreads = 128;

// loopCalculateDiscreteModel(t[j], values, h, n, 1, 0, maxValue) for M
// trajectories sharing one parameter set.
template <class S, int M>
__device__ __forceinline__ void run_multi(double (&t)[M][S::DIM], const typename S::Coef& c, int n,
                                          const DevJob& J)
{
    if (!J.checkDiv) {
#pragma unroll 2
        for (int i = 0; i < n; ++i) {
#pragma unroll
            for (int j = 0; j < M; ++j) S::step(t[j], c);
        }
        return;
    }
    double t0[M][S::DIM];
    unsigned mx[M];
#pragma unroll
    for (int j = 0; j < M; ++j) {
        copy_state<S::DIM>(t0[j], t[j]);
        mx[j] = 0;
    }
#pragma unroll 2
    for (int i = 0; i < n; ++i) {
#pragma unroll
        for (int j = 0; j < M; ++j) {
            S::step(t[j], c);
            mx[j] = max(mx[j], abs_hi(t[j][0]));
        }
    }
#pragma unroll
    for (int j = 0; j < M; ++j) {
        if (mx[j] >= J.divHi) {
            copy_state<S::DIM>(t[j], t0[j]);
            for (int i = 0; i < n; ++i) {
                S::step(t[j], c);
                if (diverged(t[j][0], J.divThresh)) break;
            }
        }
    }
}

// gramSchmidtProcess(a, b, D, den): rows of a -> orthonormal rows of b.
template <int D, bool DEN>
__device__ __forceinline__ void gram_schmidt(const double (&a)[D][D], double (&b)[D][D], double (&den)[D])
{
#pragma unroll
    for (int i = 0; i < D; ++i) {
#pragma unroll
        for (int k = 0; k < D; ++k) b[i][k] = a[i][k];
#pragma unroll
        for (int j = 0; j < i; ++j) {
            double num = 0, dd = 0;
#pragma unroll
            for (int k = 0; k < D; ++k) {
                num += a[i][k] * b[j][k];
                dd += b[j][k] * b[j][k];
            }
            const double frac = dd == 0 ? 0 : num / dd;
#pragma unroll
            for (int k = 0; k < D; ++k) b[i][k] -= frac * b[j][k];
        }
    }
#pragma unroll
    for (int i = 0; i < D; ++i) {
        double d = 0;
#pragma unroll
        for (int k = 0; k < D; ++k) d += b[i][k] * b[i][k];
        d = sqrt(d);
#pragma unroll
        for (int k = 0; k < D; ++k) b[i][k] = d == 0 ? 0 : b[i][k] / d;
        if (DEN) den[i] = d;
    }
}

// One point: the D exponents into out[0..D).  t[0] is the base trajectory,
// t[1+j] the j-th perturbed one.
template <class S>
__device__ void ls_point(const DevJob& J, long long g, double* __restrict__ out)
{
    constexpr int D = S::DIM;
    double t[D + 1][D];
    typename S::Coef c;
    {
        double v[CBF_MAX_VALUES];
        setup_point<D>(J, g, t[0], v);
        c = S::prep(v, J.h);
        to_stored<S>(t[0], c);
    }
    {
        double x1[1][D];
        typename S::Coef c1[1] = {c};
        copy_state<D>(x1[0], t[0]);
        run_checked<S, 1>(x1, c1, J.nSkip, J);  // transient, checked (cudaLibrary.cu:1016)
        copy_state<D>(t[0], x1[0]);
    }
    double z[D][D], w[D][D], den[D], res[D];
    ls_seed<D>(g, J.seedChunk, z);
    gram_schmidt<D, false>(z, w, den);
#pragma unroll
    for (int j = 0; j < D; ++j) {
        res[j] = 0;
#pragma unroll
        for (int i = 0; i < D; ++i) t[1 + j][i] = stored_comp<S>(w[j][i] * J.lleEps, i, c) + t[0][i];
    }
    for (int b = 0; b < J.nRecord; ++b) {
        run_multi<S, D + 1>(t, c, J.nNT, J);
#pragma unroll
        for (int k = 0; k < D; ++k)
#pragma unroll
            for (int l = 0; l < D; ++l) w[k][l] = phys_comp<S>(t[1 + k][l] - t[0][l], l, c);
        gram_schmidt<D, true>(w, z, den);
#pragma unroll
        for (int k = 0; k < D; ++k) {
            res[k] += log(den[k] / J.lleEps);
#pragma unroll
            for (int j = 0; j < D; ++j) t[1 + k][j] = t[0][j] + stored_comp<S>(z[k][j] * J.lleEps, j, c);
        }
    }
#pragma unroll
    for (int i = 0; i < D; ++i) out[i] = res[i] / J.tMax;
}

template <class S>
__global__ void __launch_bounds__(kLsThreads) ls_kernel(const DevJob J, double* __restrict__ out)
{
    const long long p = (long long)blockIdx.x * kLsThreads + threadIdx.x;
    if (p >= J.nPoints) return;
    ls_point<S>(J, grid_index(J, p), out + p * S::DIM);
}

template <int D>
__global__ void ls_seed_kernel(const DevJob J, double* __restrict__ out)
{
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= J.nPoints) return;
    double z[D][D];
    ls_seed<D>(grid_index(J, p), J.seedChunk, z);
#pragma unroll
    for (int j = 0; j < D; ++j)
#pragma unroll
        for (int i = 0; i < D; ++i) out[(p * D + j) * D + i] = z[j][i];
}

template <class S>
cudaError_t launch_s(const DevJob& J, double* d_out, cudaStream_t s)
{
    const long long blocks = (J.nPoints + kLsThreads - 1) / kLsThreads;
    if (blocks == 0) return cudaSuccess;
    ls_kernel<S><<<(unsigned)blocks, kLsThreads, 0, s>>>(J, d_out);
    note_launch();
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_ls(const DevJob& J, double* d_out, cudaStream_t s)
{
    switch (J.system) {
    case CBF_SYS_MEMRISTIVE5: return launch_s<Memristive5>(J, d_out, s);
    case CBF_SYS_ROSSLER: return launch_s<Rossler>(J, d_out, s);
    case CBF_SYS_LORENZ: return J.scaledStep ? launch_s<LorenzScaled>(J, d_out, s) : launch_s<Lorenz>(J, d_out, s);
    case CBF_SYS_CHEN: return J.scaledStep ? launch_s<ChenScaled>(J, d_out, s) : launch_s<Chen>(J, d_out, s);
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_ls_seeds(const DevJob& J, double* d_out, cudaStream_t s)
{
    const long long blocks = (J.nPoints + 127) / 128;
    if (blocks == 0) return cudaSuccess;
    if (J.nIC == 5)
        ls_seed_kernel<5><<<(unsigned)blocks, 128, 0, s>>>(J, d_out);
    else
        ls_seed_kernel<3><<<(unsigned)blocks, 128, 0, s>>>(J, d_out);
    note_launch();
    return cudaGetLastError();
}

}  // namespace cbf
