// One system sampled with a step offset (modelingOneSystemDenis,
// hostLibrary.cu:162-239; calculateDiscreteModelDenisCUDA, cudaLibrary.cu:121-161).
//
// Thread idx < T = (int)(hSpecial/h) runs idx steps of h from the initial
// conditions (no divergence test), then records x[writableVar] before each of
// I = (int)(tMax/hSpecial) steps of hSpecial into out[idx + i*T]: the T threads
// interleave into one series sampled every h.  The output has (int)(tMax/h)
// entries; writes past it are dropped (the reference's device writes are not
// bounded) and entries no thread writes are NaN (the reference prints
// uninitialised host memory there).
#include "bif_device.cuh"

namespace cbf {
namespace {

struct OffsetJob {
    DevJob J;
    double hSpecial;
    int T, I;
    long long n;
};

__global__ void fill_nan_kernel(double* __restrict__ out, long long n)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = __longlong_as_double(0x7ff8000000000000ll);
}

template <class S>
__global__ void offset_trajectory_kernel(const OffsetJob O, double* __restrict__ out)
{
    constexpr int D = S::DIM;
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= O.T) return;
    double x[D];
#pragma unroll
    for (int i = 0; i < D; ++i) x[i] = O.J.ic[i];
    {
        const typename S::Coef c = S::prep(O.J.values, O.J.h);
        for (int s = 0; s < idx; ++s) S::step(x, c);
    }
    const typename S::Coef c = S::prep(O.J.values, O.hSpecial);
    for (int i = 0; i < O.I; ++i) {
        const long long j = (long long)idx + (long long)i * O.T;
        if (j < O.n) out[j] = pick<D>(x, O.J.writableVar);
        S::step(x, c);
    }
}

template <class S>
cudaError_t launch_s(const OffsetJob& O, double* d_out, cudaStream_t s)
{
    if (O.T <= 0) return cudaSuccess;
    offset_trajectory_kernel<S><<<(O.T + 127) / 128, 128, 0, s>>>(O, d_out);
    note_launch();
    return cudaGetLastError();
}

}  // namespace
}  // namespace cbf

using namespace cbf;

extern "C" cbf_status cbf_modeling_one_system(int32_t system, double tMax, double h, double hSpecial,
                                              int32_t nIC, const double* ic, int32_t writableVar,
                                              const double* values, int32_t nV, double* out, int64_t outLen)
{
    if (!ic || !values || (!out && outLen > 0)) return report_error(CBF_ERR_INVALID_ARG, "null argument");
    if (!(h > 0) || !(hSpecial > 0) || !isfinite(tMax) || !isfinite(h) || !isfinite(hSpecial))
        return report_error(CBF_ERR_INVALID_ARG, "h and hSpecial must be positive, tMax finite");
    const double nd = tMax / h, td = hSpecial / h, id = tMax / hSpecial;
    if (!(nd < 2147483648.0) || !(td < 2147483648.0) || !(id < 2147483648.0))
        return report_error(CBF_ERR_INVALID_ARG, "tMax/h, hSpecial/h and tMax/hSpecial must fit an int");
    OffsetJob O;
    memset(&O, 0, sizeof(O));
    cbf_job j;
    cbf_job_init(&j);
    j.task = CBF_TASK_TRAJECTORY;  // lowered only to validate the system, its state and parameters
    j.system = system;
    j.dims = 1;
    j.nPts = 2;
    j.idxMut[0] = 0;
    j.nIC = nIC;
    j.nV = nV;
    j.h = h;
    j.tMax = 0;
    j.writableVar = writableVar;
    for (int i = 0; i < nIC && i < CBF_MAX_DIM; ++i) j.ic[i] = ic[i];
    for (int i = 0; i < nV && i < CBF_MAX_VALUES; ++i) j.values[i] = values[i];
    cbf_status st = lower_job_for(&j, &O.J);
    if (st != CBF_OK) return st;
    O.hSpecial = hSpecial;
    O.T = nd >= 0 ? (int)td : 0;
    O.I = id >= 0 ? (int)id : 0;
    O.n = nd >= 0 ? (long long)(int)nd : 0;
    if (outLen < O.n) return report_error(CBF_ERR_INVALID_ARG, "output holds fewer than (int)(tMax/h) values");
    if (O.n == 0) return CBF_OK;
    cudaStream_t s;
    if ((st = library_default_stream(&s)) != CBF_OK) return st;
    double* d = nullptr;
    cudaError_t e = cudaMallocAsync((void**)&d, (size_t)O.n * sizeof(double), s);
    if (e != cudaSuccess) return report_cuda_error(e, "allocation");
    fill_nan_kernel<<<(unsigned)((O.n + 255) / 256), 256, 0, s>>>(d, O.n);
    note_launch();
    e = cudaGetLastError();
    if (e == cudaSuccess) {
        switch (system) {
        case CBF_SYS_MEMRISTIVE5: e = launch_s<Memristive5>(O, d, s); break;
        case CBF_SYS_ROSSLER: e = launch_s<Rossler>(O, d, s); break;
        case CBF_SYS_LORENZ: e = launch_s<Lorenz>(O, d, s); break;
        case CBF_SYS_CHEN: e = launch_s<Chen>(O, d, s); break;
        default: e = cudaErrorInvalidValue; break;
        }
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, d, (size_t)O.n * sizeof(double), cudaMemcpyDeviceToHost, s);
    cudaFreeAsync(d, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return report_cuda_error(e, "step-offset trajectory");
    return CBF_OK;
}
