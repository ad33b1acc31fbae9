// Measurement and self-check kernels.
//   fp64_fma_kernel   -- FP64 FMA throughput of this GPU: the denominator of the
//                        integrator's roofline (one FMA = 2 flops).
//   expf_zero_kernel  -- exhaustive check that the device expf is exactly +0 for
//                        every float at or below a threshold; this is what makes
//                        the KDE epilogue's skip of far terms exact.
//   grid_coords_kernel-- the parameter values the kernels assign to grid points.
#include <string.h>

#include "engine.cuh"

namespace cbf {

namespace {

constexpr int kChains = 16;

__global__ void __launch_bounds__(256) fp64_fma_kernel(double* out, int iters, double a, double b)
{
    double r[kChains];
#pragma unroll
    for (int c = 0; c < kChains; ++c) r[c] = (threadIdx.x + c) * 1e-6;
#pragma unroll 4
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int c = 0; c < kChains; ++c) r[c] = fma(r[c], a, b);
    }
    double s = 0;
#pragma unroll
    for (int c = 0; c < kChains; ++c) s += r[c];
    if (s == -1.0) out[blockIdx.x] = s;  // never true; keeps the chains alive
}

__global__ void expf_zero_kernel(unsigned first, unsigned last, unsigned long long* count)
{
    unsigned long long local = 0;
    const unsigned long long n = (unsigned long long)last - first + 1;
    for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (unsigned long long)gridDim.x * blockDim.x) {
        const float x = __uint_as_float(first + (unsigned)i);
        if (expf(x) != 0.0f) ++local;
    }
    if (local) atomicAdd(count, local);
}

__global__ void grid_coords_kernel(const DevJob J, double* out)
{
    const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= J.nPoints) return;
    const long long g = grid_index(J, k);
    const bool exact = J.exactGrid != 0;
    out[k * 2 + 0] = grid_value(g, J.nPts, J.ranges[0], J.ranges[1], 0, exact);
    out[k * 2 + 1] = J.dims > 1 ? grid_value(g, J.nPts, J.ranges[2], J.ranges[3], 1, exact) : 0.0;
}

}  // namespace

cudaError_t launch_grid_coords(const DevJob& J, double* d_out, cudaStream_t s)
{
    const long long blocks = (J.nPoints + 255) / 256;
    if (blocks == 0) return cudaSuccess;
    grid_coords_kernel<<<(unsigned)blocks, 256, 0, s>>>(J, d_out);
    note_launch();
    return cudaGetLastError();
}

cudaError_t probe_fp64_peak(double ms, double* tflops)
{
    cudaError_t e;
    int dev = 0, sms = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    const int blocks = sms * 8;
    const int threads = 256;
    double* out = nullptr;
    if ((e = cudaMalloc(&out, sizeof(double) * blocks)) != cudaSuccess) return e;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    // Calibrate the iteration count on a short run, then time one long launch.
    int iters = 1 << 12;
    float t = 0.f;
    for (int round = 0; round < 6; ++round) {
        cudaEventRecord(e0);
        fp64_fma_kernel<<<blocks, threads>>>(out, iters, 0.9999999, 1e-7);
        note_launch();
        cudaEventRecord(e1);
        if ((e = cudaEventSynchronize(e1)) != cudaSuccess) break;
        cudaEventElapsedTime(&t, e0, e1);
        if (t >= ms * 0.8) break;
        double scale = (t > 0.05f) ? (ms / t) : 16.0;
        if (scale > 16.0) scale = 16.0;
        if (scale < 1.5) scale = 1.5;
        const double next = iters * scale;
        iters = next > (double)(1 << 30) ? (1 << 30) : (int)next;
    }
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e == cudaSuccess && t > 0.f) {
        const double flops = 2.0 * kChains * (double)iters * (double)blocks * threads;
        *tflops = flops / (t * 1e-3) / 1e12;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    return e;
}

cudaError_t probe_expf_zero(float threshold, unsigned long long* count)
{
    cudaError_t e;
    if (!(threshold < 0.0f)) return cudaErrorInvalidValue;
    unsigned long long* d = nullptr;
    if ((e = cudaMalloc(&d, sizeof(unsigned long long))) != cudaSuccess) return e;
    cudaMemset(d, 0, sizeof(unsigned long long));
    // Negative floats: larger magnitude <-> larger bit pattern, up to -inf (0xff800000).
    unsigned first = 0;
    memcpy(&first, &threshold, sizeof(first));
    const unsigned last = 0xff800000u;
    expf_zero_kernel<<<1184, 256>>>(first, last, d);
    note_launch();
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpy(count, d, sizeof(unsigned long long), cudaMemcpyDeviceToHost);
    cudaFree(d);
    return e;
}

}  // namespace cbf
