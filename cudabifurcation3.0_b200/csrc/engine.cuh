// Internal definitions shared by the kernels and the C-ABI layer.
#pragma once
#include <limits.h>

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/cbf.h"
#include "systems.cuh"

namespace cbf {

constexpr double kPeakIntervalUnit = 0.01;  // peakFinder's default h (cudaLibrary.cuh:204)

// A validated job in the form the kernels consume (passed by value).
struct DevJob {
    double ranges[4];
    double ic[CBF_MAX_DIM];
    double values[CBF_MAX_VALUES];
    double h;
    double maxValue;
    double divThresh;   // |x| >= divThresh  <=>  fabsf((float)x) > maxValue
    double lleEps;
    double tMax;
    double kdeI1, kdeI2, kdeH;
    double kdeSkip;     // terms with |peak - delta| > kdeSkip are exactly 0 (see kde epilogue)
    double kdeInvH;     // 1/kdeH when kdeH = +-2^k and 1/kdeH is a normal double, else 0
    double dbEps;
    double dbSkip;      // pairs with |dx| or |dy| >= dbSkip are never neighbours
    long long firstPoint;
    long long nPoints;
    long long seedChunk;
    const long long* pointIndex;  // optional device list of grid indices (see cbf_job)
    int regimeSteps;    // LLE_REGIME: recorded steps after the transient
    double regimeMinAmp;  // LLE_REGIME: window range below this -> class 0
    double regimeChaosLle;  // LLE_REGIME: > 0 and LLE above it -> class 15
    double ostThr;      // OSTROVSKY: periodicity threshold
    int nPts, dims, nIC, nV;
    int idxMut0, idxMut1;
    int writableVar, preScaller;
    int nSkip;          // transient steps: (int)(transientTime / h)
    int nRecord;        // recorded samples (int)(tMax/h/preScaller); LLE: (int)(tMax/NT)
    int nNT;            // LLE steps per renormalisation (int)(size_t)(NT/h)
    int checkDiv;       // maxValue != 0 and can ever fire
    unsigned divHi;     // high word of divThresh (conservative fast check)
    int exactGrid;
    int maxPeaks;
    int kdeSampling;
    int kdeFixed;
    int peakCap;        // peaks stored per point
    int task;
    int system;
    int sweepIC;
    int scaledStep;     // Chen/Lorenz: the rescaled step (systems.cuh, QuadScaled) for this job
    int unitStep;       // ... with k = h1 (s = 1/2): its 8-instruction form
};

// Grid index of the job's k-th point: an explicit list, or a contiguous range.
__device__ __forceinline__ long long grid_index(const DevJob& J, long long k)
{
    return J.pointIndex ? J.pointIndex[k] : J.firstPoint + k;
}

// getValueByIdx (cudaLibrary.cu:210-216): `(int)idx / powf(nPts, v)` is a float
// division, so above 2^24 the index is rounded; exactGrid uses integer math.
__device__ __forceinline__ double grid_value(long long g, int nPts, double start, double finish,
                                             int axis, bool exact)
{
    int cell;
    if (!exact) {
        float p = powf((float)nPts, (float)axis);
        float q = (float)(int)g / p;
        cell = ((int)q) % nPts;
    } else {
        long long d = (axis == 0) ? 1 : (long long)nPts;
        cell = (int)((g / d) % nPts);
    }
    return start + (double)cell * ((double)(finish - start) / (double)(nPts - 1));
}

// Set up one point: ICs and values copied, swept entries overwritten
// (cudaLibrary.cu:96-105; IC variant :183-192).  Fully unrolled so that the
// arrays stay in registers even though the swept indices are runtime values.
template <int DIM>
__device__ __forceinline__ void setup_point(const DevJob& J, long long g, double (&x)[DIM],
                                            double (&v)[CBF_MAX_VALUES])
{
    const bool exact = J.exactGrid != 0;
    const double p0 = grid_value(g, J.nPts, J.ranges[0], J.ranges[1], 0, exact);
    const double p1 = (J.dims > 1) ? grid_value(g, J.nPts, J.ranges[2], J.ranges[3], 1, exact) : 0.0;
    const int m0 = J.idxMut0;
    const int m1 = (J.dims > 1) ? J.idxMut1 : -1;
#pragma unroll
    for (int i = 0; i < DIM; ++i) {
        double t = J.ic[i];
        if (J.sweepIC) {
            if (i == m0) t = p0;
            if (i == m1) t = p1;
        }
        x[i] = t;
    }
#pragma unroll
    for (int i = 0; i < CBF_MAX_VALUES; ++i) {
        double t = J.values[i];
        if (!J.sweepIC) {
            if (i == m0) t = p0;
            if (i == m1) t = p1;
        }
        v[i] = t;
    }
}

__device__ __forceinline__ unsigned abs_hi(double v)
{
    return (unsigned)(__double_as_longlong(v) >> 32) & 0x7fffffffu;
}

// Conservative magnitude tracker of a stream of doubles against a threshold T:
// |v| >= T needs hi(|v|) >= hi(T) (the high word is monotone in the magnitude),
// and the signed high word of v is hi(|v|) for v >= 0, while its unsigned high
// word is 2^31 + hi(|v|) for v < 0.  So the signed maximum of the high words
// reaches hi(T) only if some positive value may have reached T, and the
// unsigned maximum reaches 2^31 + hi(T) only if some negative one may have
// (NaNs count as reaching it).  Two three-input maxima (the sm_90+ DPX integer
// instructions) take two values per update with no masking: half the integer
// work of tracking max |hi| of each value, which competes with the FP64 step
// for issue slots.
struct HiTrack {
    int s;
    unsigned u;
    __device__ __forceinline__ void init()
    {
        s = INT_MIN;
        u = 0;
    }
    __device__ __forceinline__ void add2(double a, double b)
    {
        const int ha = __double2hiint(a), hb = __double2hiint(b);
        s = __vimax3_s32(s, ha, hb);
        u = __vimax3_u32(u, (unsigned)ha, (unsigned)hb);
    }
    __device__ __forceinline__ void add1(double a)
    {
        const int ha = __double2hiint(a);
        s = max(s, ha);
        u = max(u, (unsigned)ha);
    }
    // hiT = the threshold's high word without sign (DevJob::divHi)
    __device__ __forceinline__ bool maybe(unsigned hiT) const { return s >= (int)hiT || u >= 0x80000000u + hiT; }
};

// Exact divergence test of loopCalculateDiscreteModel (cudaLibrary.cu:69-71).
__device__ __forceinline__ bool diverged(double v, double thresh)
{
    return fabs(v) >= thresh;
}

// Deterministic LLE perturbation direction from the chunk-local thread index
// (cudaLibrary.cu:720-732; IC variant :843-855), normalised in double.
template <int D, bool IC>
__device__ __forceinline__ void lle_seed(long long g, long long seedChunk, double (&z)[D])
{
    const int idx = (int)(seedChunk > 0 ? (g % seedChunk) : g);
    double zPower = 0;
#pragma unroll
    for (int i = 0; i < D; ++i) {
        if (!IC) {
            const unsigned u = (unsigned)idx * ((unsigned)i * (unsigned)idx + 1u) + 1u;
            z[i] = 0.5 * (double)sinf((float)(int)u);
        } else {
            const double arg = 0.2171828 * (i + 1) + idx + (0.2171828 + i * idx);
            z[i] = (double)sinf((float)arg) * 0.5;
        }
        zPower += z[i] * z[i];
    }
    zPower = sqrt(zPower);
#pragma unroll
    for (int i = 0; i < D; ++i) z[i] /= zPower;
}

// Initial perturbation rows of the Lyapunov-spectrum kernel (LSKernelCUDA,
// cudaLibrary.cu:1001-1013): row j, entry i = 0.5 sinf(0.2171828 (i+1)(j+1) + idx
// + (0.2171828 + i j idx)) in the reference's operation order (double sum, FP32
// sinf), idx the chunk-local index; each row normalised to length 1.
template <int D>
__device__ __forceinline__ void ls_seed(long long g, long long seedChunk, double (&z)[D][D])
{
    const int idx = (int)(seedChunk > 0 ? (g % seedChunk) : g);
#pragma unroll
    for (int j = 0; j < D; ++j) {
        double zPower = 0;
#pragma unroll
        for (int i = 0; i < D; ++i) {
            const double arg = 0.2171828 * (i + 1) * (j + 1) + idx + (0.2171828 + i * j * idx);
            z[j][i] = (double)sinf((float)arg) * 0.5;
            zPower += z[j][i] * z[j][i];
        }
        zPower = sqrt(zPower);
#pragma unroll
        for (int i = 0; i < D; ++i) z[j][i] /= zPower;
    }
}

// Kernel launch bookkeeping (defined in capi.cu).
void note_launch(unsigned n = 1);

// Threads per block of the fused bifurcation kernel (bif.cu).
constexpr int kBifBlockThreads = 128;

// Launchers (defined in lle.cu / bif.cu / probes.cu).  All return a CUDA error.
cudaError_t launch_lle(const DevJob& J, double* d_out, cudaStream_t s);
// LLE kernel shapes (lle.cu): the autotuner's search space.
constexpr int kNumLleVariants = CBF_NUM_LLE_VARIANTS;
cudaError_t launch_lle_variant(const DevJob& J, double* d_out, cudaStream_t s, int variant);
// The shape cbf_run uses for `system` on the current device (capi.cu).
int lle_variant_for(int system);
cudaError_t launch_bif(const DevJob& J, void* d_out, int* d_aux, cudaStream_t s);
cudaError_t launch_grid_coords(const DevJob& J, double* d_out, cudaStream_t s);
cudaError_t launch_lle_seeds(const DevJob& J, double* d_out, cudaStream_t s);
// Lyapunov spectrum: nIC exponents per point (d_out[p*nIC + i]); seed rows
// (nIC x nIC per point) for parity checks.
cudaError_t launch_ls(const DevJob& J, double* d_out, cudaStream_t s);
cudaError_t launch_ls_seeds(const DevJob& J, double* d_out, cudaStream_t s);
cudaError_t launch_lle_regime(const DevJob& J, double* d_lle, int* d_class, cudaStream_t s);
// Points the LLE_REGIME kernel keeps in flight at once on the current device.
long long lle_regime_resident_points(const DevJob& J);
// The LLE_REGIME kernel over a device point list (J.pointIndex) whose length
// *nDev (at most maxPoints) a previous kernel wrote, with caller-provided
// scratch of lle_regime_scratch_bytes(J); no allocation, no host
// synchronisation: a device-side check sets *err (zero on entry).
size_t lle_regime_scratch_bytes(const DevJob& J);
cudaError_t launch_lle_regime_list(const DevJob& J, const long long* nDev, long long maxPoints, double* d_lle,
                                   int* d_cls, double* scratch, size_t scratchBytes, int* err, cudaStream_t s);

// KDE/DBSCAN with caller-provided scratch (no allocation): `scratch` holds
// `scratchBytes` of peak buffers, `err` one int that must be zero on entry.
// Synchronises `s` to read `err`.
cudaError_t launch_bif_prealloc(const DevJob& J, void* d_out, double* scratch, size_t scratchBytes,
                                int* err, cudaStream_t s);

// Job lowering and error reporting shared with other translation units (capi.cu).
cbf_status lower_job_for(const cbf_job* job, DevJob* d);
// The library's stream for calls given no stream (created once per device).
cbf_status library_default_stream(cudaStream_t* s);
cbf_status report_error(cbf_status st, const char* message);
cbf_status report_cuda_error(cudaError_t e, const char* where);

}  // namespace cbf
