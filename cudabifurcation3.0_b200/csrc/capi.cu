// C-ABI launch layer: validation, job lowering, launches, host-buffer wrappers.
// Errors are returned as cbf_status codes (never exit()); the detail string of
// the last failure is kept per host thread.
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include <atomic>
#include <mutex>
#include <string>

#include "engine.cuh"

namespace cbf {

cudaError_t probe_fp64_peak(double ms, double* tflops);
cudaError_t probe_expf_zero(float threshold, unsigned long long* count);
cudaError_t probe_fp64_step(int chains, bool track, int blocksPerSm, double ms, double* instrPerSec);

namespace {

std::atomic<unsigned long long> g_launches{0};
thread_local std::string g_last_error;

cbf_status fail(cbf_status st, const char* fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return st;
}

cbf_status cuda_fail(cudaError_t e, const char* where)
{
    const cbf_status st = (e == cudaErrorMemoryAllocation) ? CBF_ERR_OUT_OF_MEMORY
                          : (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver)
                              ? CBF_ERR_NO_DEVICE
                          : (e == cudaErrorAssert) ? CBF_ERR_INTERNAL
                                                   : CBF_ERR_CUDA;
    return fail(st, "%s: %s (%s)", where, cudaGetErrorString(e), cudaGetErrorName(e));
}

#define CBF_CUDA(call)                                   \
    do {                                                 \
        cudaError_t e_ = (call);                         \
        if (e_ != cudaSuccess) return cuda_fail(e_, #call); \
    } while (0)

int system_dim(int sys)
{
    switch (sys) {
    case CBF_SYS_MEMRISTIVE5: return Memristive5::DIM;
    case CBF_SYS_ROSSLER: return Rossler::DIM;
    case CBF_SYS_LORENZ: return Lorenz::DIM;
    case CBF_SYS_CHEN: return Chen::DIM;
    default: return -1;
    }
}

int system_nv(int sys)
{
    switch (sys) {
    case CBF_SYS_MEMRISTIVE5: return Memristive5::NV;
    case CBF_SYS_ROSSLER: return Rossler::NV;
    case CBF_SYS_LORENZ: return Lorenz::NV;
    case CBF_SYS_CHEN: return Chen::NV;
    default: return -1;
    }
}

// (int) of a double the way the reference truncates, refusing values an int
// cannot hold (the reference would have undefined behaviour there).
bool to_int(double v, int* out)
{
    if (!(v > -2147483648.0 && v < 2147483648.0)) return false;
    *out = (int)v;
    return true;
}

std::mutex g_stream_mu;
cudaStream_t g_streams[64];
bool g_stream_made[64];

// The library's scratch buffers come from the device's default stream-ordered
// pool (cudaMallocAsync).  With the pool's default release threshold (0) every
// synchronisation hands the memory back to the driver and the next call maps it
// again -- tens of milliseconds for the ~0.6 GB peak scratch of a map launch.
// Keep up to 16 GB cached between calls instead (set once per device).
std::atomic<bool> g_pool_set[64];

void keep_pool_memory()
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64 || g_pool_set[dev].load()) return;
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
        uint64_t threshold = 16ull << 30;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold);
    }
    g_pool_set[dev].store(true);
}

cbf_status library_stream(cudaStream_t* s)
{
    keep_pool_memory();
    int dev = 0;
    CBF_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return fail(CBF_ERR_INVALID_ARG, "device %d out of range", dev);
    std::lock_guard<std::mutex> lk(g_stream_mu);
    if (!g_stream_made[dev]) {
        CBF_CUDA(cudaStreamCreateWithFlags(&g_streams[dev], cudaStreamNonBlocking));
        g_stream_made[dev] = true;
    }
    *s = g_streams[dev];
    return CBF_OK;
}

// Chosen LLE kernel shape per device and system (-1: default shape 0).
std::atomic<int> g_lle_variant[64][CBF_NUM_SYSTEMS];
std::once_flag g_variant_init;

void init_variants()
{
    for (int d = 0; d < 64; ++d)
        for (int k = 0; k < CBF_NUM_SYSTEMS; ++k) g_lle_variant[d][k].store(-1);
}

}  // namespace

int lle_variant_for(int system)
{
    std::call_once(g_variant_init, init_variants);
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 0;
    if (system < 0 || system >= CBF_NUM_SYSTEMS) return 0;
    const int v = g_lle_variant[dev][system].load();
    return v < 0 ? 0 : v;
}

void note_launch(unsigned n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

// Smallest T >= 0 with  fabs(x) >= T  <=>  (double)fabsf((float)x) > M  for all x.
// Rounding to float is monotone, so the condition is an up-set in |x|; its edge
// is the rounding midpoint below the smallest float F > M (ties go to even).
void divergence_threshold(double M, int* active, double* T)
{
    *active = 0;
    *T = INFINITY;
    if (M == 0 || isnan(M)) return;  // disabled, or the comparison never holds
    if (M < 0) { *active = 1; *T = 0.0; return; }
    if (isinf(M)) return;            // nothing is greater than +inf
    float fm = (float)M;
    float F = ((double)fm > M) ? fm : nextafterf(fm, INFINITY);
    double mid;
    bool even;
    if (isinf(F)) {
        mid = ldexp(1.0, 128) - ldexp(1.0, 103);  // FLT_MAX + half an ulp
        even = true;
    } else {
        const float P = nextafterf(F, 0.0f);
        mid = ((double)P + (double)F) * 0.5;
        unsigned bits;
        memcpy(&bits, &F, sizeof(bits));
        even = (bits & 1u) == 0;
    }
    *active = 1;
    *T = even ? mid : nextafter(mid, INFINITY);
}

namespace {

// Whether every point of a Chen or Lorenz job can run the rescaled step
// (systems.cuh, QuadScaled): s = values[0] not swept, k = h s at least 2^-64 in
// magnitude, and every value each other parameter takes (the fixed value, or all
// nPts values of its swept axis, whatever points the job selects) finite and
// within 2^64 in magnitude, with A = values[1] (a or sigma) and the step's
// denominators 1 + h1 A, 1 - k B, 1 + h1 B and the y-equation factors (Chen
// 1 + k c, 1 - h1 c; Lorenz 1 - k, 1 + h1) at least 2^-64 in magnitude.  Every
// derived coefficient then lies far inside the double range and sy, sz are
// nonzero.  The oracle applies the same rule.
bool scaled_step_ok(const cbf_job* j)
{
    const bool chen = j->system == CBF_SYS_CHEN, lorenz = j->system == CBF_SYS_LORENZ;
    if (!chen && !lorenz) return false;
    const double big = 0x1p64, small = 0x1p-64;
    auto fin = [&](double v) { return isfinite(v) && fabs(v) <= big; };
    auto away = [&](double v) { return isfinite(v) && fabs(v) >= small; };
    int sweptAxis[CBF_MAX_VALUES];
    for (int i = 0; i < CBF_MAX_VALUES; ++i) sweptAxis[i] = -1;
    if (!j->sweepIC)
        for (int a = 0; a < j->dims && a < 2; ++a)
            if (j->idxMut[a] >= 0 && j->idxMut[a] < CBF_MAX_VALUES) sweptAxis[j->idxMut[a]] = a;
    if (sweptAxis[0] >= 0) return false;
    const double h = j->h, s = j->values[0];
    if (!(fin(h) && away(h) && fin(s))) return false;
    const double k = h * s, h1 = h * (1.0 - s);
    if (!away(k)) return false;
    if (lorenz && !(away(1.0 - k) && away(1.0 + h1))) return false;
    for (int slot = 1; slot <= 3; ++slot) {
        const int ax = sweptAxis[slot];
        const int count = ax < 0 ? 1 : j->nPts;
        for (int cell = 0; cell < count; ++cell) {
            // the values grid_value produces for this axis (engine.cuh)
            const double v = ax < 0 ? j->values[slot]
                                    : j->ranges[2 * ax] + (double)cell * ((double)(j->ranges[2 * ax + 1] -
                                                                                    j->ranges[2 * ax]) /
                                                                          (double)(j->nPts - 1));
            if (!fin(v)) return false;
            bool ok = true;
            if (slot == 1) ok = away(v) && away(1.0 + h1 * v);                      // a / sigma
            else if (chen && slot == 2) ok = away(1.0 - k * v) && away(1.0 + h1 * v);  // b
            else if (chen && slot == 3) ok = away(1.0 + k * v) && away(1.0 - h1 * v);  // c
            else if (lorenz && slot == 3) ok = away(1.0 - k * v) && away(1.0 + h1 * v);  // beta
            if (!ok) return false;
        }
    }
    return true;
}

cbf_status lower_job(const cbf_job* j, DevJob* d)
{
    if (!j || !d) return fail(CBF_ERR_INVALID_ARG, "null job");
    memset(d, 0, sizeof(*d));
    const int dim = system_dim(j->system);
    if (dim < 0) return fail(CBF_ERR_UNKNOWN_SYSTEM, "unknown system id %d", j->system);
    if (j->task < CBF_TASK_PEAKS || j->task > CBF_TASK_OSTROVSKY)
        return fail(CBF_ERR_INVALID_ARG, "unknown task %d", j->task);
    if (j->dims != 1 && j->dims != 2) return fail(CBF_ERR_INVALID_ARG, "dims must be 1 or 2 (got %d)", j->dims);
    if (j->nPts < 1) return fail(CBF_ERR_INVALID_ARG, "nPts must be >= 1 (got %d)", j->nPts);
    if (j->nIC != dim)
        return fail(CBF_ERR_INVALID_ARG, "system %d has %d state variables, got %d initial conditions",
                    j->system, dim, j->nIC);
    if (j->nV < system_nv(j->system) || j->nV > CBF_MAX_VALUES)
        return fail(CBF_ERR_INVALID_ARG, "system %d needs %d..%d values, got %d", j->system,
                    system_nv(j->system), CBF_MAX_VALUES, j->nV);
    const int limit = j->sweepIC ? j->nIC : j->nV;
    for (int i = 0; i < j->dims; ++i)
        if (j->idxMut[i] < 0 || j->idxMut[i] >= limit)
            return fail(CBF_ERR_INVALID_ARG, "indicesOfMutVars[%d]=%d out of range [0,%d)", i,
                        j->idxMut[i], limit);
    // The LLE and LS kernels always check x[0] and ignore writableVar
    // (cudaLibrary.cu:735-753, 1049-1060).
    const bool lleTask = (j->task == CBF_TASK_LLE || j->task == CBF_TASK_LLE_REGIME || j->task == CBF_TASK_LS);
    if (j->task != CBF_TASK_LLE && j->task != CBF_TASK_LS && (j->writableVar < 0 || j->writableVar >= dim))
        return fail(CBF_ERR_INVALID_ARG, "writableVar %d out of range [0,%d)", j->writableVar, dim);
    if (!(isfinite(j->h) && j->h != 0)) return fail(CBF_ERR_INVALID_ARG, "h must be finite and nonzero");

    long long total = 1;
    for (int i = 0; i < j->dims; ++i) total *= j->nPts;
    const long long nPoints = j->nPoints > 0 ? j->nPoints : total;
    if (j->firstPoint < 0 || j->nPoints < 0)
        return fail(CBF_ERR_INVALID_ARG, "negative point range");
    if (j->pointIndex && j->nPoints <= 0)
        return fail(CBF_ERR_INVALID_ARG, "a point list needs nPoints > 0");
    if (j->firstPoint + nPoints > 2147483647ll)
        return fail(CBF_ERR_INVALID_ARG, "grid index exceeds the int range of getValueByIdx");

    d->task = j->task;
    d->system = j->system;
    d->sweepIC = j->sweepIC ? 1 : 0;
    d->scaledStep = scaled_step_ok(j) ? 1 : 0;
    d->unitStep = d->scaledStep && j->h * j->values[0] == j->h * (1.0 - j->values[0]);
    d->dims = j->dims;
    d->nPts = j->nPts;
    d->nIC = j->nIC;
    d->nV = j->nV;
    d->idxMut0 = j->idxMut[0];
    d->idxMut1 = j->dims > 1 ? j->idxMut[1] : -1;
    d->writableVar = j->writableVar;
    d->exactGrid = (j->flags & CBF_FLAG_EXACT_GRID) ? 1 : 0;
    d->firstPoint = j->firstPoint;
    d->nPoints = nPoints;
    d->pointIndex = (const long long*)j->pointIndex;
    for (int i = 0; i < 4; ++i) d->ranges[i] = j->ranges[i];
    for (int i = 0; i < CBF_MAX_DIM; ++i) d->ic[i] = i < j->nIC ? j->ic[i] : 0.0;
    for (int i = 0; i < CBF_MAX_VALUES; ++i) d->values[i] = i < j->nV ? j->values[i] : 0.0;
    d->h = j->h;
    d->maxValue = j->maxValue;
    divergence_threshold(j->maxValue, &d->checkDiv, &d->divThresh);
    {
        long long bits;
        memcpy(&bits, &d->divThresh, sizeof(bits));
        d->divHi = (unsigned)((unsigned long long)bits >> 32) & 0x7fffffffu;
    }
    if (!to_int(j->transientTime / j->h, &d->nSkip))
        return fail(CBF_ERR_INVALID_ARG, "transientTime/h does not fit an int");
    if (d->nSkip < 0) d->nSkip = 0;

    if (lleTask) {
        if (!(j->NT != 0 && isfinite(j->NT))) return fail(CBF_ERR_INVALID_ARG, "NT must be finite and nonzero");
        if (!to_int(j->tMax / j->NT, &d->nRecord))
            return fail(CBF_ERR_INVALID_ARG, "tMax/NT does not fit an int");
        const double nt = j->NT / j->h;
        if (!(nt >= 0 && nt < 2147483648.0))
            return fail(CBF_ERR_INVALID_ARG, "NT/h must be in [0, 2^31)");
        d->nNT = (int)(size_t)nt;
        if (d->nRecord < 0) d->nRecord = 0;
        d->lleEps = j->lleEps;
        d->tMax = j->tMax;
        if (j->seedChunk < 0) return fail(CBF_ERR_INVALID_ARG, "seedChunk must be >= 0");
        d->seedChunk = j->seedChunk;
        if (j->task == CBF_TASK_LLE_REGIME) {
            if (!to_int(j->regimeTime / j->h, &d->regimeSteps) || d->regimeSteps < 0)
                return fail(CBF_ERR_INVALID_ARG, "regimeTime/h must be in [0, 2^31)");
            d->maxPeaks = j->maxAmountOfPeaks;
            if (!(j->regimeMinAmp >= 0)) return fail(CBF_ERR_INVALID_ARG, "regimeMinAmp must be >= 0");
            d->regimeMinAmp = j->regimeMinAmp;
            d->regimeChaosLle = j->regimeChaosLle;
            const int half = d->regimeSteps / 2 > 0 ? d->regimeSteps / 2 : 1;
            const int cap = j->maxAmountOfPeaks < half ? j->maxAmountOfPeaks : half;
            d->peakCap = cap > 0 ? cap : 1;
            const double e = j->dbscanEps;
            d->dbEps = e;
            if (!(e > 0)) d->dbSkip = 0.0;
            else if (!(4.0 * e >= 1.1754943508222875e-38) || isinf(e)) d->dbSkip = INFINITY;
            else d->dbSkip = 4.0 * e;
        }
    } else {
        if (j->preScaller < 1) return fail(CBF_ERR_INVALID_ARG, "preScaller must be >= 1");
        d->preScaller = j->preScaller;
        if (!to_int(j->tMax / j->h / (double)j->preScaller, &d->nRecord))
            return fail(CBF_ERR_INVALID_ARG, "tMax/h/preScaller does not fit an int");
        if (d->nRecord < 0) d->nRecord = 0;
        const int half = d->nRecord / 2 > 0 ? d->nRecord / 2 : 1;
        switch (j->task) {
        case CBF_TASK_PEAKS:
            d->peakCap = j->peakCapacity > 0 ? j->peakCapacity : half;
            break;
        case CBF_TASK_TRAJECTORY:
            d->peakCap = j->peakCapacity > 0 ? j->peakCapacity : (d->nRecord > 0 ? d->nRecord : 1);
            if (d->peakCap < d->nRecord)
                return fail(CBF_ERR_INVALID_ARG, "trajectory row stride %d < record %d", d->peakCap, d->nRecord);
            break;
        default: {
            d->maxPeaks = j->maxAmountOfPeaks;
            int cap = j->maxAmountOfPeaks < half ? j->maxAmountOfPeaks : half;
            d->peakCap = cap > 0 ? cap : 1;
            break;
        }
        }
        if (j->task == CBF_TASK_KDE) {
            d->kdeSampling = j->kdeSampling;
            d->kdeFixed = (j->flags & CBF_FLAG_KDE_FIXED) ? 1 : 0;
            d->kdeI1 = j->kdeI1;
            d->kdeI2 = j->kdeI2;
            d->kdeH = j->kdeH;
            d->kdeSkip = 16.0 * fabs(j->kdeH);
            // For H = +-2^k, x / H and x * (1/H) are the same exact real rounded
            // once, so the epilogue may multiply (bit-identical, no FP64 divide).
            int ex = 0;
            const double mant = frexp(fabs(j->kdeH), &ex);
            const double inv = 1.0 / j->kdeH;
            d->kdeInvH = (mant == 0.5 && std::isnormal(inv)) ? inv : 0.0;
        }
        if (j->task == CBF_TASK_OSTROVSKY) d->ostThr = j->ostrovskyThreshold;
        if (j->task == CBF_TASK_DBSCAN || j->task == CBF_TASK_OSTROVSKY) {
            const double e = j->dbscanEps;
            d->dbEps = e;
            if (!(e > 0)) d->dbSkip = 0.0;                        // nothing is ever a neighbour
            else if (!(4.0 * e >= 1.1754943508222875e-38) || isinf(e)) d->dbSkip = INFINITY;
            else d->dbSkip = 4.0 * e;
        }
    }
    return CBF_OK;
}

size_t out_bytes(const DevJob& d)
{
    switch (d.task) {
    case CBF_TASK_LLE:
    case CBF_TASK_LLE_REGIME: return (size_t)d.nPoints * sizeof(double);
    case CBF_TASK_LS: return (size_t)d.nPoints * (size_t)d.nIC * sizeof(double);
    case CBF_TASK_OSTROVSKY: return (size_t)d.nPoints * sizeof(double);
    case CBF_TASK_KDE:
    case CBF_TASK_DBSCAN: return (size_t)d.nPoints * sizeof(int);
    default: return (size_t)d.nPoints * (size_t)d.peakCap * sizeof(double);
    }
}

size_t aux_bytes(const DevJob& d)
{
    return (d.task == CBF_TASK_PEAKS || d.task == CBF_TASK_TRAJECTORY || d.task == CBF_TASK_LLE_REGIME)
               ? (size_t)d.nPoints * sizeof(int)
               : 0;
}

cbf_status run_lowered(const DevJob& d, void* d_out, void* d_aux, cudaStream_t s)
{
    cudaError_t e;
    if (d.nPoints == 0) return CBF_OK;
    keep_pool_memory();
    if (d.task == CBF_TASK_LLE)
        e = launch_lle(d, (double*)d_out, s);
    else if (d.task == CBF_TASK_LLE_REGIME)
        e = launch_lle_regime(d, (double*)d_out, (int*)d_aux, s);
    else if (d.task == CBF_TASK_LS)
        e = launch_ls(d, (double*)d_out, s);
    else
        e = launch_bif(d, d_out, (int*)d_aux, s);
    if (e == cudaErrorAssert) return fail(CBF_ERR_INTERNAL, "device-side iteration guard fired");
    if (e != cudaSuccess) return cuda_fail(e, "kernel launch");
    return CBF_OK;
}

cbf_status run_host_impl(const cbf_job* job, void* out, void* aux)
{
    DevJob d;
    cbf_status st = lower_job(job, &d);
    if (st != CBF_OK) return st;
    if (d.nPoints == 0) return CBF_OK;
    if (!out) return fail(CBF_ERR_INVALID_ARG, "null output buffer");
    if (aux_bytes(d) && !aux) return fail(CBF_ERR_INVALID_ARG, "null aux buffer");
    cudaStream_t s;
    if ((st = library_stream(&s)) != CBF_OK) return st;
    void* d_out = nullptr;
    void* d_aux = nullptr;
    const size_t ob = out_bytes(d), ab = aux_bytes(d);
    CBF_CUDA(cudaMallocAsync(&d_out, ob, s));
    if (ab) {
        cudaError_t e = cudaMallocAsync(&d_aux, ab, s);
        if (e != cudaSuccess) {
            cudaFreeAsync(d_out, s);
            return cuda_fail(e, "cudaMallocAsync(aux)");
        }
    }
    st = run_lowered(d, d_out, d_aux, s);
    if (st == CBF_OK) {
        cudaError_t e = cudaMemcpyAsync(out, d_out, ob, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess && ab) e = cudaMemcpyAsync(aux, d_aux, ab, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) st = cuda_fail(e, "copy results to host");
    }
    cudaFreeAsync(d_out, s);
    if (d_aux) cudaFreeAsync(d_aux, s);
    return st;
}

void fill_common(cbf_job* j, int32_t system, int dims, int32_t nPts, double h, int32_t nIC,
                 const double* ic, const double* ranges, const int32_t* idxMut, int32_t wv,
                 double maxValue, double transientTime, const double* values, int32_t nV)
{
    cbf_job_init(j);
    j->system = system;
    j->dims = dims;
    j->nPts = nPts;
    j->h = h;
    j->nIC = nIC;
    for (int i = 0; i < nIC && i < CBF_MAX_DIM; ++i) j->ic[i] = ic[i];
    for (int i = 0; i < 2 * dims; ++i) j->ranges[i] = ranges[i];
    for (int i = 0; i < dims; ++i) j->idxMut[i] = idxMut[i];
    j->writableVar = wv;
    j->maxValue = maxValue;
    j->transientTime = transientTime;
    j->nV = nV;
    for (int i = 0; i < nV && i < CBF_MAX_VALUES; ++i) j->values[i] = values[i];
}

cbf_status check_ptrs(int32_t nIC, const double* ic, const double* ranges, const int32_t* idx,
                      const double* values, int32_t nV)
{
    if (!ic || !ranges || !idx || !values) return fail(CBF_ERR_INVALID_ARG, "null input array");
    if (nIC < 1 || nIC > CBF_MAX_DIM) return fail(CBF_ERR_INVALID_ARG, "amountOfInitialConditions %d out of range", nIC);
    if (nV < 1 || nV > CBF_MAX_VALUES) return fail(CBF_ERR_INVALID_ARG, "amountOfValues %d out of range", nV);
    return CBF_OK;
}

cbf_status bif1d(bool ic_sweep, int32_t system, double tMax, int32_t nPts, double h, int32_t nIC,
                 const double* ic, const double* ranges, const int32_t* idxMut, int32_t wv,
                 double maxValue, double transientTime, const double* values, int32_t nV,
                 int32_t preScaller, double* outPeaks, int32_t cap, int32_t* outCounts)
{
    cbf_status st = check_ptrs(nIC, ic, ranges, idxMut, values, nV);
    if (st != CBF_OK) return st;
    cbf_job j;
    fill_common(&j, system, 1, nPts, h, nIC, ic, ranges, idxMut, wv, maxValue, transientTime, values, nV);
    j.task = CBF_TASK_PEAKS;
    j.sweepIC = ic_sweep ? 1 : 0;
    j.tMax = tMax;
    j.preScaller = preScaller;
    const int need = cbf_peak_capacity(&j);
    if (cap < need) return fail(CBF_ERR_INVALID_ARG, "peakCapacity %d < record/2 = %d", cap, need);
    j.peakCapacity = cap;
    return run_host_impl(&j, outPeaks, outCounts);
}

cbf_status map2d(bool ic_sweep, int task, int32_t system, double tMax, int32_t nPts, double h,
                 int32_t nIC, const double* ic, const double* ranges, const int32_t* idxMut,
                 int32_t wv, double maxValue, int32_t maxPeaks, double transientTime,
                 const double* values, int32_t nV, int32_t preScaller, int32_t kdeSampling,
                 double i1, double i2, double smooth, double eps, int32_t* out)
{
    cbf_status st = check_ptrs(nIC, ic, ranges, idxMut, values, nV);
    if (st != CBF_OK) return st;
    cbf_job j;
    fill_common(&j, system, 2, nPts, h, nIC, ic, ranges, idxMut, wv, maxValue, transientTime, values, nV);
    j.task = task;
    j.sweepIC = ic_sweep ? 1 : 0;
    j.tMax = tMax;
    j.preScaller = preScaller;
    j.maxAmountOfPeaks = maxPeaks;
    j.kdeSampling = kdeSampling;
    j.kdeI1 = i1;
    j.kdeI2 = i2;
    j.kdeH = smooth;
    j.dbscanEps = eps;
    return run_host_impl(&j, out, nullptr);
}

cbf_status ostrovsky(int32_t system, double tMax, int32_t nPts, double h, int32_t nIC, const double* ic,
                     const double* ranges, const int32_t* idxMut, int32_t wv, double maxValue,
                     int32_t maxPeaks, double transientTime, const double* values, int32_t nV,
                     int32_t preScaller, double eps, double threshold, double* out)
{
    cbf_status st = check_ptrs(nIC, ic, ranges, idxMut, values, nV);
    if (st != CBF_OK) return st;
    cbf_job j;
    fill_common(&j, system, 2, nPts, h, nIC, ic, ranges, idxMut, wv, maxValue, transientTime, values, nV);
    j.task = CBF_TASK_OSTROVSKY;
    j.sweepIC = 1;  // the reference integrates with calculateDiscreteModelICCUDA (hostLibrary.cu:843)
    j.tMax = tMax;
    j.preScaller = preScaller;
    j.maxAmountOfPeaks = maxPeaks;
    j.dbscanEps = eps;
    j.ostrovskyThreshold = threshold;
    return run_host_impl(&j, out, nullptr);
}

cbf_status lle(bool ic_sweep, int dims, int32_t system, double tMax, double NT, int32_t nPts,
               double h, double eps, const double* ic, int32_t nIC, const double* ranges,
               const int32_t* idxMut, int32_t wv, double maxValue, double transientTime,
               const double* values, int32_t nV, int64_t seedChunk, double* out)
{
    cbf_status st = check_ptrs(nIC, ic, ranges, idxMut, values, nV);
    if (st != CBF_OK) return st;
    cbf_job j;
    fill_common(&j, system, dims, nPts, h, nIC, ic, ranges, idxMut, wv, maxValue, transientTime, values, nV);
    j.task = CBF_TASK_LLE;
    j.sweepIC = ic_sweep ? 1 : 0;
    j.tMax = tMax;
    j.NT = NT;
    j.lleEps = eps;
    j.seedChunk = seedChunk;
    return run_host_impl(&j, out, nullptr);
}

cbf_status ls(int dims, int32_t system, double tMax, double NT, int32_t nPts, double h, double eps,
              const double* ic, int32_t nIC, const double* ranges, const int32_t* idxMut, int32_t wv,
              double maxValue, double transientTime, const double* values, int32_t nV,
              int64_t seedChunk, double* out)
{
    cbf_status st = check_ptrs(nIC, ic, ranges, idxMut, values, nV);
    if (st != CBF_OK) return st;
    cbf_job j;
    fill_common(&j, system, dims, nPts, h, nIC, ic, ranges, idxMut, wv, maxValue, transientTime, values, nV);
    j.task = CBF_TASK_LS;
    j.tMax = tMax;
    j.NT = NT;
    j.lleEps = eps;
    j.seedChunk = seedChunk;
    return run_host_impl(&j, out, nullptr);
}

}  // namespace

cbf_status lower_job_for(const cbf_job* job, DevJob* d) { return lower_job(job, d); }
cbf_status run_job_lowered(const DevJob& d, void* d_out, void* d_aux, cudaStream_t s)
{
    return run_lowered(d, d_out, d_aux, s);
}
cbf_status library_default_stream(cudaStream_t* s) { return library_stream(s); }
cbf_status report_error(cbf_status st, const char* message) { return fail(st, "%s", message); }
cbf_status report_cuda_error(cudaError_t e, const char* where) { return cuda_fail(e, where); }

}  // namespace cbf

using namespace cbf;

extern "C" {

int32_t cbf_abi_version(void) { return CBF_ABI_VERSION; }

const char* cbf_status_string(cbf_status s)
{
    switch (s) {
    case CBF_OK: return "ok";
    case CBF_ERR_INVALID_ARG: return "invalid argument";
    case CBF_ERR_UNKNOWN_SYSTEM: return "unknown system";
    case CBF_ERR_CUDA: return "CUDA error";
    case CBF_ERR_OUT_OF_MEMORY: return "out of device memory";
    case CBF_ERR_NO_DEVICE: return "no CUDA device";
    case CBF_ERR_IO: return "I/O error";
    case CBF_ERR_TIMEOUT: return "device wait timed out";
    case CBF_ERR_INTERNAL: return "internal consistency check failed";
    default: return "unknown status";
    }
}

const char* cbf_last_error(void) { return g_last_error.c_str(); }

uint64_t cbf_kernel_launches(void) { return g_launches.load(std::memory_order_relaxed); }

cbf_status cbf_device_count(int32_t* count)
{
    if (!count) return fail(CBF_ERR_INVALID_ARG, "null count");
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess) {
        *count = 0;
        return cuda_fail(e, "cudaGetDeviceCount");
    }
    *count = n;
    return CBF_OK;
}

cbf_status cbf_set_device(int32_t device)
{
    CBF_CUDA(cudaSetDevice(device));
    return CBF_OK;
}

void cbf_job_init(cbf_job* j)
{
    if (!j) return;
    memset(j, 0, sizeof(*j));
    j->task = CBF_TASK_LLE;
    j->system = CBF_SYS_MEMRISTIVE5;
    j->dims = 2;
    j->preScaller = 1;
}

int32_t cbf_record_length(const cbf_job* j)
{
    if (!j) return -1;
    int v = 0;
    if (j->task == CBF_TASK_LLE || j->task == CBF_TASK_LLE_REGIME || j->task == CBF_TASK_LS) {
        if (j->NT == 0 || !to_int(j->tMax / j->NT, &v)) return -1;
    } else {
        if (j->h == 0 || j->preScaller < 1 || !to_int(j->tMax / j->h / (double)j->preScaller, &v)) return -1;
    }
    return v;
}

int32_t cbf_peak_capacity(const cbf_job* j)
{
    const int32_t r = cbf_record_length(j);
    if (r < 0) return -1;
    return r / 2 > 0 ? r / 2 : 1;
}

int64_t cbf_job_points(const cbf_job* j)
{
    if (!j) return -1;
    if (j->nPoints > 0) return j->nPoints;
    long long t = 1;
    for (int i = 0; i < j->dims; ++i) t *= j->nPts;
    return t;
}

cbf_status cbf_validate(const cbf_job* job)
{
    DevJob d;
    return lower_job(job, &d);
}

int32_t cbf_job_scaled_step(const cbf_job* job)
{
    DevJob d;
    if (lower_job(job, &d) != CBF_OK) return -1;
    return d.scaledStep ? (d.unitStep ? 2 : 1) : 0;
}

cbf_status cbf_run(const cbf_job* job, void* d_out, void* d_aux, void* stream)
{
    DevJob d;
    cbf_status st = lower_job(job, &d);
    if (st != CBF_OK) return st;
    if (d.nPoints == 0) return CBF_OK;
    if (!d_out) return fail(CBF_ERR_INVALID_ARG, "null device output");
    if (aux_bytes(d) && !d_aux) return fail(CBF_ERR_INVALID_ARG, "null device aux buffer");
    return run_lowered(d, d_out, d_aux, (cudaStream_t)stream);
}

cbf_status cbf_run_host(const cbf_job* job, void* out, void* aux) { return run_host_impl(job, out, aux); }

cbf_status cbf_bifurcation1d(int32_t system, double tMax, int32_t nPts, double h, int32_t nIC,
                             const double* ic, const double* ranges, const int32_t* idxMut,
                             int32_t wv, double maxValue, double transientTime,
                             const double* values, int32_t nV, int32_t preScaller,
                             double* outPeaks, int32_t peakCapacity, int32_t* outCounts)
{
    return bif1d(false, system, tMax, nPts, h, nIC, ic, ranges, idxMut, wv, maxValue, transientTime,
                 values, nV, preScaller, outPeaks, peakCapacity, outCounts);
}

cbf_status cbf_bifurcation1d_ic(int32_t system, double tMax, int32_t nPts, double h, int32_t nIC,
                                const double* ic, const double* ranges, const int32_t* idxMut,
                                int32_t wv, double maxValue, double transientTime,
                                const double* values, int32_t nV, int32_t preScaller,
                                double* outPeaks, int32_t peakCapacity, int32_t* outCounts)
{
    return bif1d(true, system, tMax, nPts, h, nIC, ic, ranges, idxMut, wv, maxValue, transientTime,
                 values, nV, preScaller, outPeaks, peakCapacity, outCounts);
}

cbf_status cbf_bifurcation2d_kde(int32_t system, double tMax, int32_t nPts, double h, int32_t nIC,
                                 const double* ic, const double* ranges, const int32_t* idxMut,
                                 int32_t wv, double maxValue, int32_t maxPeaks, double transientTime,
                                 const double* values, int32_t nV, int32_t preScaller,
                                 int32_t kdeSampling, double i1, double i2, double smooth,
                                 int32_t* out)
{
    return map2d(false, CBF_TASK_KDE, system, tMax, nPts, h, nIC, ic, ranges, idxMut, wv, maxValue,
                 maxPeaks, transientTime, values, nV, preScaller, kdeSampling, i1, i2, smooth, 0.0, out);
}

cbf_status cbf_bifurcation2d_kde_ic(int32_t system, double tMax, int32_t nPts, double h, int32_t nIC,
                                    const double* ic, const double* ranges, const int32_t* idxMut,
                                    int32_t wv, double maxValue, int32_t maxPeaks,
                                    double transientTime, const double* values, int32_t nV,
                                    int32_t preScaller, int32_t kdeSampling, double i1, double i2,
                                    double smooth, int32_t* out)
{
    return map2d(true, CBF_TASK_KDE, system, tMax, nPts, h, nIC, ic, ranges, idxMut, wv, maxValue,
                 maxPeaks, transientTime, values, nV, preScaller, kdeSampling, i1, i2, smooth, 0.0, out);
}

cbf_status cbf_bifurcation2d_dbscan(int32_t system, double tMax, int32_t nPts, double h, int32_t nIC,
                                    const double* ic, const double* ranges, const int32_t* idxMut,
                                    int32_t wv, double maxValue, int32_t maxPeaks,
                                    double transientTime, const double* values, int32_t nV,
                                    int32_t preScaller, double eps, int32_t* out)
{
    return map2d(false, CBF_TASK_DBSCAN, system, tMax, nPts, h, nIC, ic, ranges, idxMut, wv,
                 maxValue, maxPeaks, transientTime, values, nV, preScaller, 0, 0.0, 0.0, 0.0, eps, out);
}

cbf_status cbf_bifurcation2d_dbscan_ic(int32_t system, double tMax, int32_t nPts, double h,
                                       int32_t nIC, const double* ic, const double* ranges,
                                       const int32_t* idxMut, int32_t wv, double maxValue,
                                       int32_t maxPeaks, double transientTime, const double* values,
                                       int32_t nV, int32_t preScaller, double eps, int32_t* out)
{
    return map2d(true, CBF_TASK_DBSCAN, system, tMax, nPts, h, nIC, ic, ranges, idxMut, wv,
                 maxValue, maxPeaks, transientTime, values, nV, preScaller, 0, 0.0, 0.0, 0.0, eps, out);
}

cbf_status cbf_lle1d(int32_t system, double tMax, double NT, int32_t nPts, double h, double eps,
                     const double* ic, int32_t nIC, const double* ranges, const int32_t* idxMut,
                     int32_t wv, double maxValue, double transientTime, const double* values,
                     int32_t nV, int64_t seedChunk, double* out)
{
    return lle(false, 1, system, tMax, NT, nPts, h, eps, ic, nIC, ranges, idxMut, wv, maxValue,
               transientTime, values, nV, seedChunk, out);
}

cbf_status cbf_lle1d_ic(int32_t system, double tMax, double NT, int32_t nPts, double h, double eps,
                        const double* ic, int32_t nIC, const double* ranges, const int32_t* idxMut,
                        int32_t wv, double maxValue, double transientTime, const double* values,
                        int32_t nV, int64_t seedChunk, double* out)
{
    return lle(true, 1, system, tMax, NT, nPts, h, eps, ic, nIC, ranges, idxMut, wv, maxValue,
               transientTime, values, nV, seedChunk, out);
}

cbf_status cbf_lle2d(int32_t system, double tMax, double NT, int32_t nPts, double h, double eps,
                     const double* ic, int32_t nIC, const double* ranges, const int32_t* idxMut,
                     int32_t wv, double maxValue, double transientTime, const double* values,
                     int32_t nV, int64_t seedChunk, double* out)
{
    return lle(false, 2, system, tMax, NT, nPts, h, eps, ic, nIC, ranges, idxMut, wv, maxValue,
               transientTime, values, nV, seedChunk, out);
}

cbf_status cbf_lle2d_ic(int32_t system, double tMax, double NT, int32_t nPts, double h, double eps,
                        const double* ic, int32_t nIC, const double* ranges, const int32_t* idxMut,
                        int32_t wv, double maxValue, double transientTime, const double* values,
                        int32_t nV, int64_t seedChunk, double* out)
{
    return lle(true, 2, system, tMax, NT, nPts, h, eps, ic, nIC, ranges, idxMut, wv, maxValue,
               transientTime, values, nV, seedChunk, out);
}

cbf_status cbf_ostrovsky2d(int32_t system, double tMax, int32_t nPts, double h, int32_t nIC,
                           const double* ic, const double* ranges, const int32_t* idxMut, int32_t wv,
                           double maxValue, int32_t maxPeaks, double transientTime,
                           const double* values, int32_t nV, int32_t preScaller, double eps,
                           double ostrovskyThreshold, double* out)
{
    return ostrovsky(system, tMax, nPts, h, nIC, ic, ranges, idxMut, wv, maxValue, maxPeaks, transientTime,
                     values, nV, preScaller, eps, ostrovskyThreshold, out);
}

cbf_status cbf_ls1d(int32_t system, double tMax, double NT, int32_t nPts, double h, double eps,
                    const double* ic, int32_t nIC, const double* ranges, const int32_t* idxMut,
                    int32_t wv, double maxValue, double transientTime, const double* values,
                    int32_t nV, int64_t seedChunk, double* out)
{
    return ls(1, system, tMax, NT, nPts, h, eps, ic, nIC, ranges, idxMut, wv, maxValue, transientTime,
              values, nV, seedChunk, out);
}

cbf_status cbf_ls2d(int32_t system, double tMax, double NT, int32_t nPts, double h, double eps,
                    const double* ic, int32_t nIC, const double* ranges, const int32_t* idxMut,
                    int32_t wv, double maxValue, double transientTime, const double* values,
                    int32_t nV, int64_t seedChunk, double* out)
{
    return ls(2, system, tMax, NT, nPts, h, eps, ic, nIC, ranges, idxMut, wv, maxValue, transientTime,
              values, nV, seedChunk, out);
}

cbf_status cbf_grid_coordinates(const cbf_job* job, double* out_host)
{
    DevJob d;
    cbf_status st = lower_job(job, &d);
    if (st != CBF_OK) return st;
    if (!out_host) return fail(CBF_ERR_INVALID_ARG, "null output");
    if (d.nPoints == 0) return CBF_OK;
    cudaStream_t s;
    if ((st = library_stream(&s)) != CBF_OK) return st;
    double* dd = nullptr;
    const size_t bytes = (size_t)d.nPoints * 2 * sizeof(double);
    CBF_CUDA(cudaMallocAsync((void**)&dd, bytes, s));
    cudaError_t e = launch_grid_coords(d, dd, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(out_host, dd, bytes, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaFreeAsync(dd, s);
    if (e != cudaSuccess) return cuda_fail(e, "grid coordinates");
    return CBF_OK;
}

cbf_status cbf_set_lle_variant(int32_t system, int32_t variant)
{
    std::call_once(g_variant_init, init_variants);
    if (system < 0 || system >= CBF_NUM_SYSTEMS) return fail(CBF_ERR_UNKNOWN_SYSTEM, "unknown system %d", system);
    if (variant < -1 || variant >= kNumLleVariants) return fail(CBF_ERR_INVALID_ARG, "variant %d out of range", variant);
    int dev = 0;
    CBF_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return fail(CBF_ERR_INVALID_ARG, "device %d out of range", dev);
    g_lle_variant[dev][system].store(variant);
    return CBF_OK;
}

int32_t cbf_get_lle_variant(int32_t system) { return lle_variant_for(system); }

// Times every LLE kernel shape on a shortened copy of the job: the job's first
// points (two full waves of the most occupying shape), its transient cut to 1024
// steps, 8 renormalisation intervals of at most 1000 steps.  Per-step cost does
// not depend on where in the trajectory a step falls, so the ranking carries over.
cbf_status cbf_autotune(const cbf_job* job, int32_t* chosen, double* msPerVariant)
{
    std::call_once(g_variant_init, init_variants);
    DevJob d;
    cbf_status st = lower_job(job, &d);
    if (st != CBF_OK) return st;
    if (d.task != CBF_TASK_LLE) return fail(CBF_ERR_INVALID_ARG, "cbf_autotune tunes LLE jobs");
    int dev = 0, sms = 0;
    CBF_CUDA(cudaGetDevice(&dev));
    CBF_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    DevJob t = d;
    const long long trial = (long long)sms * 2048 * 2 * 2;
    if (t.nPoints > trial) t.nPoints = trial;
    if (t.nSkip > 1024) t.nSkip = 1024;
    if (t.nRecord > 8) t.nRecord = 8;
    if (t.nRecord < 1) t.nRecord = 1;
    if (t.nNT > 1000) t.nNT = 1000;
    if (t.nNT < 1) t.nNT = 1;
    cudaStream_t s;
    if ((st = library_stream(&s)) != CBF_OK) return st;
    double* out = nullptr;
    CBF_CUDA(cudaMallocAsync((void**)&out, (size_t)t.nPoints * sizeof(double), s));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float best = 0.f;
    int bestV = 0;
    cudaError_t e = cudaSuccess;
    for (int v = 0; v < kNumLleVariants && e == cudaSuccess; ++v) {
        e = launch_lle_variant(t, out, s, v);  // warm-up (module load, caches)
        if (e != cudaSuccess) break;
        cudaEventRecord(e0, s);
        e = launch_lle_variant(t, out, s, v);
        cudaEventRecord(e1, s);
        if (e == cudaSuccess) e = cudaEventSynchronize(e1);
        float ms = 0.f;
        if (e == cudaSuccess) cudaEventElapsedTime(&ms, e0, e1);
        if (msPerVariant) msPerVariant[v] = ms;
        if (v == 0 || ms < best) {
            best = ms;
            bestV = v;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFreeAsync(out, s);
    if (e != cudaSuccess) return cuda_fail(e, "autotune");
    if (dev >= 0 && dev < 64) g_lle_variant[dev][d.system].store(bestV);
    if (chosen) *chosen = bestV;
    return CBF_OK;
}

cbf_status cbf_lle_seeds(const cbf_job* job, double* out_host)
{
    DevJob d;
    cbf_status st = lower_job(job, &d);
    if (st != CBF_OK) return st;
    if (d.task != CBF_TASK_LLE && d.task != CBF_TASK_LLE_REGIME && d.task != CBF_TASK_LS)
        return fail(CBF_ERR_INVALID_ARG, "cbf_lle_seeds needs an LLE or LS job");
    if (!out_host) return fail(CBF_ERR_INVALID_ARG, "null output");
    if (d.nPoints == 0) return CBF_OK;
    cudaStream_t s;
    if ((st = library_stream(&s)) != CBF_OK) return st;
    double* dd = nullptr;
    const size_t per = d.task == CBF_TASK_LS ? (size_t)d.nIC * d.nIC : (size_t)d.nIC;
    const size_t bytes = (size_t)d.nPoints * per * sizeof(double);
    CBF_CUDA(cudaMallocAsync((void**)&dd, bytes, s));
    cudaError_t e = d.task == CBF_TASK_LS ? launch_ls_seeds(d, dd, s) : launch_lle_seeds(d, dd, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(out_host, dd, bytes, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaFreeAsync(dd, s);
    if (e != cudaSuccess) return cuda_fail(e, "lle seeds");
    return CBF_OK;
}

cbf_status cbf_probe_fp64_peak(double ms, double* tflops)
{
    if (!tflops || !(ms > 0)) return fail(CBF_ERR_INVALID_ARG, "bad probe arguments");
    cudaError_t e = probe_fp64_peak(ms, tflops);
    if (e != cudaSuccess) return cuda_fail(e, "fp64 probe");
    return CBF_OK;
}

cbf_status cbf_probe_fp64_step(int32_t chains, int32_t tracking, int32_t blocksPerSm, double ms,
                               double* fp64InstrPerSec)
{
    if (!fp64InstrPerSec) return fail(CBF_ERR_INVALID_ARG, "null output");
    if ((chains != 1 && chains != 2 && chains != 4) || blocksPerSm < 1 || blocksPerSm > 16 || !(ms > 0))
        return fail(CBF_ERR_INVALID_ARG, "chains must be 1, 2 or 4, blocksPerSm in [1, 16], ms > 0");
    cudaError_t e = probe_fp64_step(chains, tracking != 0, blocksPerSm, ms, fp64InstrPerSec);
    if (e != cudaSuccess) return cuda_fail(e, "FP64 step probe");
    return CBF_OK;
}

cbf_status cbf_probe_expf_zero(float threshold, uint64_t* count)
{
    if (!count) return fail(CBF_ERR_INVALID_ARG, "null count");
    unsigned long long c = 0;
    cudaError_t e = probe_expf_zero(threshold, &c);
    if (e != cudaSuccess) return cuda_fail(e, "expf probe");
    *count = c;
    return CBF_OK;
}

cbf_status cbf_divergence_threshold(double maxValue, int32_t* active, double* threshold)
{
    if (!active || !threshold) return fail(CBF_ERR_INVALID_ARG, "null output");
    int a = 0;
    double t = 0;
    divergence_threshold(maxValue, &a, &t);
    *active = a;
    *threshold = t;
    return CBF_OK;
}

}  // extern "C"
