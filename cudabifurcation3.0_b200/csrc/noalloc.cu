// DBSCAN cluster-count map that allocates no device memory.
//
// Some callers cannot call cudaMalloc: applications whose device memory is owned
// by another allocator (a framework's caching pool, a fixed budget handed out at
// start-up), and latency-critical loops where an allocation's implicit device
// synchronisation, or an out-of-memory failure half-way through a run, is not
// acceptable.  cbf_bifurcation2d_dbscan_noalloc serves them: the caller passes
// the output buffer, and the per-warp peak/interval scratch the fused kernel
// needs comes from one file-scope device array of fixed size.  The array sits in
// this translation unit's own module; under lazy module loading (the CUDA
// default) a device reserves it at the first call made on that device -- the
// address lookup loads the module -- so that first call can fail with out of
// memory and belongs at start-up.  A device keeps the array until the process
// exits.  Each call waits for its stream to finish, to read the error flag.
//
// Maps with long peak lists run the regular entry point's two passes inside the
// array (a first pass with 1024 peak slots per point, the overflow points again
// at full capacity), so that many more blocks fit than at full capacity.
//
// The array is shared by every call: calls that overlap on the GPU (from several
// host threads, or on several streams) race on it and must be serialised by the
// caller.  Its first 256 bytes hold the kernel's error flag, which every call
// clears before launching; the rest is peak scratch that every call overwrites
// before reading.
#include <stdio.h>

#include <mutex>

#include "engine.cuh"

namespace cbf {
namespace {

constexpr size_t kNoAllocScratchBytes = (size_t)64 << 20;  // 64 MiB per device
constexpr size_t kNoAllocHeaderBytes = 256;                 // error flag, keeps 256 B alignment

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_mu;
void* g_scratch_addr[64];  // device address of g_noalloc_scratch, per device

// Host code must not use g_noalloc_scratch directly: there it names a host-side
// stand-in, not device memory.  The device address is looked up once per device,
// with that device current, on the first call made on it, and cached; a
// cudaDeviceReset invalidates the cached address.
cbf_status scratch_address(void** out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return report_cuda_error(e, "cudaGetDevice");
    if (dev < 0 || dev >= 64) return report_error(CBF_ERR_INVALID_ARG, "device index out of range");
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return report_cuda_error(e, "cudaGetSymbolAddress(no-allocation scratch)");
        g_scratch_addr[dev] = p;
    }
    *out = g_scratch_addr[dev];
    return CBF_OK;
}

}  // namespace
}  // namespace cbf

using namespace cbf;

extern "C" cbf_status cbf_bifurcation2d_dbscan_noalloc(
    int32_t system, double tMax, int32_t nPts, double h, int32_t nIC, const double* ic,
    const double* ranges, const int32_t* idxMut, int32_t writableVar, double maxValue,
    int32_t maxAmountOfPeaks, double transientTime, const double* values, int32_t nV,
    int32_t preScaller, double eps, int32_t* d_out, void* stream)
{
    if (!ic || !ranges || !idxMut || !values)
        return report_error(CBF_ERR_INVALID_ARG, "null input array");
    if (nIC < 1 || nIC > CBF_MAX_DIM || nV < 1 || nV > CBF_MAX_VALUES)
        return report_error(CBF_ERR_INVALID_ARG, "amountOfInitialConditions/amountOfValues out of range");
    cbf_job j;
    cbf_job_init(&j);
    j.task = CBF_TASK_DBSCAN;
    j.system = system;
    j.dims = 2;
    j.nPts = nPts;
    j.h = h;
    j.tMax = tMax;
    j.transientTime = transientTime;
    j.maxValue = maxValue;
    j.writableVar = writableVar;
    j.preScaller = preScaller;
    j.maxAmountOfPeaks = maxAmountOfPeaks;
    j.dbscanEps = eps;
    j.nIC = nIC;
    j.nV = nV;
    for (int i = 0; i < nIC; ++i) j.ic[i] = ic[i];
    for (int i = 0; i < nV; ++i) j.values[i] = values[i];
    for (int i = 0; i < 4; ++i) j.ranges[i] = ranges[i];
    j.idxMut[0] = idxMut[0];
    j.idxMut[1] = idxMut[1];

    DevJob d;
    cbf_status st = lower_job_for(&j, &d);
    if (st != CBF_OK) return st;
    if (d.nPoints == 0) return CBF_OK;
    if (!d_out) return report_error(CBF_ERR_INVALID_ARG, "null device output");

    // One block of the fused kernel needs its 128 lanes' peak and interval slices.
    const size_t perBlock = (size_t)kBifBlockThreads * d.peakCap * 2 * sizeof(double);
    const size_t usable = kNoAllocScratchBytes - kNoAllocHeaderBytes;
    if (perBlock > usable) {
        char msg[256];
        snprintf(msg, sizeof(msg),
                 "no-allocation DBSCAN: min(maxAmountOfPeaks, record/2) = %d peaks per point needs "
                 "%zu bytes per block, the fixed 64 MiB scratch holds at most %zu peaks per point",
                 d.peakCap, perBlock, usable / ((size_t)kBifBlockThreads * 2 * sizeof(double)));
        return report_error(CBF_ERR_INVALID_ARG, msg);
    }

    void* base = nullptr;
    if ((st = scratch_address(&base)) != CBF_OK) return st;
    cudaStream_t s = (cudaStream_t)stream;
    int* err = (int*)base;
    double* scratch = (double*)((unsigned char*)base + kNoAllocHeaderBytes);
    cudaError_t e = cudaMemsetAsync(err, 0, sizeof(int), s);
    if (e != cudaSuccess) return report_cuda_error(e, "clear no-allocation error flag");
    e = launch_bif_prealloc(d, d_out, scratch, usable, err, s);
    if (e == cudaErrorAssert) return report_error(CBF_ERR_INTERNAL, "device-side iteration guard fired");
    if (e != cudaSuccess) return report_cuda_error(e, "no-allocation DBSCAN launch");
    return CBF_OK;
}
