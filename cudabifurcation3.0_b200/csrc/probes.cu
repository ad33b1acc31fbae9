// Measurement and self-check kernels.
//   fp64_fma_kernel   -- FP64 FMA throughput of this GPU: the denominator of the
//                        integrator's roofline (one FMA = 2 flops).
//   step_chain_kernel -- the FP64 issue rate the map kernels' step and
//                        divergence tracking reach as a bare instruction stream:
//                        what the LLE kernel's pipe fraction is compared with.
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

// The FP64 issue rate the map kernels' instruction stream can reach, apart from
// any map: each thread advances CH independent copies of the rescaled Chen step
// at s = 1/2 (the 8-instruction form, per-thread coefficients from a ∈ [35, 36))
// for `iters` steps and, when TRACK, folds them into the map kernels' divergence
// trackers (two three-input maxima per pair of values).
template <int CH, bool TRACK>
__global__ void __launch_bounds__(128) step_chain_kernel(double* out, int iters)
{
    using S = ChenScaledU;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const double v[4] = {0.5, 35.0 + 1e-7 * (t & 1023), 3.0, 28.0};
    const typename S::Coef q = S::prep(v, 0.002);
    double X[CH][3];
#pragma unroll
    for (int c = 0; c < CH; ++c) {
        X[c][0] = 0.1 + 1e-3 * c;
        X[c][1] = 0.1;
        X[c][2] = 0.1;
        to_stored<S>(X[c], q);
    }
    HiTrack tr;
    tr.init();
#pragma unroll 2
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int c = 0; c < CH; ++c) S::step(X[c], q);
        if (TRACK) {
            if (CH == 1) tr.add1(X[0][0]);
#pragma unroll
            for (int c = 0; c + 1 < CH; c += 2) tr.add2(X[c][0], X[c + 1][0]);
        }
    }
    double s = (double)tr.s + (double)tr.u;
#pragma unroll
    for (int c = 0; c < CH; ++c) s += X[c][0] + X[c][1] + X[c][2];
    if (s == -1.0) out[blockIdx.x] = s;  // never true; keeps the chains alive
}

template <int CH, bool TRACK>
float time_step_chains(int blocks, double* out, int iters)
{
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0);
    step_chain_kernel<CH, TRACK><<<blocks, 128>>>(out, iters);
    note_launch();
    cudaEventRecord(e1);
    float t = -1.f;
    if (cudaEventSynchronize(e1) == cudaSuccess) cudaEventElapsedTime(&t, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return t;
}

float time_step_chains_for(int chains, bool track, int blocks, double* out, int iters)
{
    switch (chains * 2 + (track ? 1 : 0)) {
    case 2: return time_step_chains<1, false>(blocks, out, iters);
    case 3: return time_step_chains<1, true>(blocks, out, iters);
    case 4: return time_step_chains<2, false>(blocks, out, iters);
    case 5: return time_step_chains<2, true>(blocks, out, iters);
    case 8: return time_step_chains<4, false>(blocks, out, iters);
    default: return time_step_chains<4, true>(blocks, out, iters);
    }
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

// FP64 lane instructions per second of step_chain_kernel with `chains` (1, 2, 4)
// chains per thread at `blocksPerSm` blocks of 128 threads per SM, the launch
// sized to run about `ms` milliseconds.
cudaError_t probe_fp64_step(int chains, bool track, int blocksPerSm, double ms, double* instrPerSec)
{
    if ((chains != 1 && chains != 2 && chains != 4) || blocksPerSm < 1 || blocksPerSm > 16 || !(ms > 0))
        return cudaErrorInvalidValue;
    cudaError_t e;
    int dev = 0, sms = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    const int blocks = sms * blocksPerSm;
    double* out = nullptr;
    if ((e = cudaMalloc(&out, sizeof(double) * blocks)) != cudaSuccess) return e;
    // Calibrate the step count on short runs, then time one long launch.
    int iters = 1 << 10;
    float t = 0.f;
    for (int round = 0; round < 8; ++round) {
        t = time_step_chains_for(chains, track, blocks, out, iters);
        if ((e = cudaGetLastError()) != cudaSuccess || t < 0.f) break;
        if (t >= ms * 0.8) break;
        double scale = (t > 0.05f) ? (ms / t) : 16.0;
        if (scale > 16.0) scale = 16.0;
        if (scale < 1.5) scale = 1.5;
        const double next = iters * scale;
        iters = next > (double)(1 << 28) ? (1 << 28) : (int)next;
    }
    if (e == cudaSuccess && t < 0.f) e = cudaErrorUnknown;
    if (e == cudaSuccess && t > 0.f) {
        const double instr = 8.0 * chains * (double)iters * (double)blocks * 128.0;
        *instrPerSec = instr / (t * 1e-3);
    }
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
