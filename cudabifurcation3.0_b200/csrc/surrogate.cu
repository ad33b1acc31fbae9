// Surrogate-refined LLE + regime map of a 2-D parameter sweep.
//
// The plain FP64 method (the LLE_REGIME kernels: LLEKernelCUDA semantics plus the
// peak-count regime class) labels a coarse sub-grid of the map -- every
// (nPts/coarseSide)-th row and column -- and a seeded random sample of points.
// The network of mlp.cu is trained on those labels on the GPU, predicts LLE,
// class and confidence for every grid point, and the plain method then
// recomputes every point
//   * on a predicted regime boundary (a neighbour within boundaryRadius has
//     another predicted class),
//   * whose softmax confidence is below confThreshold,
//   * in a seeded random audit sample (auditFraction of the grid).
// Wherever the plain class of a label or a recomputed point differs from the
// network's, its neighbours (expandRadius) are recomputed in a later round, for
// maxWaves rounds: thin structures the network cannot resolve (periodic windows
// inside chaos) are traced from any point that hits them.  Labelled and
// recomputed points carry plain values; the rest carry the network's
// prediction.  The audit points that no other rule selected measure the error of
// the kept predictions.  Everything runs on one stream.  The rounds are planned
// on the device (plan_kernel): the host reads the labels back once (to normalise
// the LLE targets), the number of rule-selected points once (to bound the
// rounds) and waits once at the end.
#include <math.h>
#include <string.h>

#include <mutex>
#include <vector>

#include "mlp.cuh"

namespace cbf {
namespace {

constexpr int kChunk = 4096;          // points per compaction block
constexpr int kChunkThreads = 256;
// flag bits: reasons to recompute, then the point's state
constexpr unsigned char kBoundary = 1, kLowConf = 2, kAudit = 4, kExpand = 8;
constexpr unsigned char kReasons = kBoundary | kLowConf | kAudit | kExpand;
constexpr unsigned char kDone = 0x40, kLabel = 0x80;

__device__ __forceinline__ unsigned long long mix64(unsigned long long z)
{
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// Training points: the coarse sub-grid (cs x cs, stride `stride`) then nRand
// seeded random grid points.  Grid index g = row * nPts + column (axis 0 fastest).
__global__ void label_index_kernel(long long* __restrict__ idx, int cs, int stride, int nPts, long long nRand,
                                   long long nPoints, unsigned long long seed)
{
    const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long nCoarse = (long long)cs * cs;
    if (k >= nCoarse + nRand) return;
    if (k < nCoarse) {
        const long long r = k / cs, c = k % cs;
        idx[k] = r * stride * (long long)nPts + c * stride;
    } else {
        idx[k] = (long long)(mix64(seed ^ mix64((unsigned long long)k)) % (unsigned long long)nPoints);
    }
}

// Labels into the map.  surprise[k]: the network's class at the label's point
// differed from the plain class (of duplicated points at least the first
// reader sees the prediction, so the set of surprised points is deterministic).
__global__ void label_scatter_kernel(const long long* __restrict__ idx, long long n, const double* __restrict__ lle,
                                     const int* __restrict__ cls, double* __restrict__ mapLle,
                                     int* __restrict__ mapCls, unsigned char* __restrict__ flag,
                                     unsigned char* __restrict__ src, unsigned char* __restrict__ surprise)
{
    const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const long long g = idx[k];
    surprise[k] = mapCls[g] != cls[k];
    mapLle[g] = lle[k];
    mapCls[g] = cls[k];
    flag[g] = kLabel;
    src[g] = 1;
}

// The prediction without a network: each grid point takes the LLE and class of
// the nearest point of the coarse label grid (labels 0..cs*cs-1, the point
// (r*stride, c*stride) at index r*cs + c), confidence 1.
__global__ void nearest_label_kernel(const double* __restrict__ labLle, const int* __restrict__ labCls, int cs,
                                     int stride, int nPts, long long nPoints, double* __restrict__ lle,
                                     int* __restrict__ cls, float* __restrict__ conf)
{
    const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= nPoints) return;
    const int row = (int)(g / nPts), col = (int)(g % nPts);
    const int cr = min(cs - 1, (row + stride / 2) / stride);
    const int cc = min(cs - 1, (col + stride / 2) / stride);
    const long long k = (long long)cr * cs + cc;
    lle[g] = labLle[k];
    cls[g] = labCls[k];
    conf[g] = 1.0f;
}

// Refinement reasons of every grid point from the predicted classes/confidences.
__global__ void mask_kernel(const int* __restrict__ cls, const float* __restrict__ conf, int nPts, long long nPoints,
                            int radius, float confThr, unsigned long long auditCut, unsigned long long seed,
                            unsigned char* __restrict__ flag, unsigned char* __restrict__ src)
{
    const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= nPoints) return;
    const int row = (int)(g / nPts), col = (int)(g % nPts);
    const int c = cls[g];
    unsigned char f = 0;
    for (int dr = -radius; dr <= radius && !(f & kBoundary); ++dr) {
        const int r = row + dr;
        if (r < 0 || r >= nPts) continue;
        for (int dc = -radius; dc <= radius; ++dc) {
            const int q = col + dc;
            if (q < 0 || q >= nPts) continue;
            if (cls[(long long)r * nPts + q] != c) {
                f |= kBoundary;
                break;
            }
        }
    }
    if (!(conf[g] >= confThr)) f |= kLowConf;
    if (mix64(seed ^ mix64((unsigned long long)g + 0x5851F42D4C957F2Dull)) < auditCut) f |= kAudit;
    flag[g] = f;
    src[g] = 0;
}

// Points with one of the `want` reasons and none of the `exclude` bits that are
// neither labels nor computed.
__device__ __forceinline__ bool selected(unsigned char f, unsigned char want, unsigned char exclude)
{
    return (f & want) && !(f & (kLabel | kDone | exclude));
}

// `stop` (optional): nonzero once the recompute rounds have ended; every round
// kernel then returns at once.
__global__ void __launch_bounds__(kChunkThreads) count_kernel(const unsigned char* __restrict__ flag, long long n,
                                                              unsigned char want, unsigned char exclude,
                                                              int* __restrict__ blockCount, const int* stop)
{
    if (stop && *stop) return;
    const long long base = (long long)blockIdx.x * kChunk;
    int total = 0;
    for (int r = 0; r < kChunk; r += kChunkThreads) {
        const long long g = base + r + threadIdx.x;
        total += __syncthreads_count(g < n && selected(flag[g], want, exclude));
    }
    if (threadIdx.x == 0) blockCount[blockIdx.x] = total;
}

// Exclusive prefix over nb block counts (one block of 1024 threads);
// offsets[nb] = total.
__global__ void __launch_bounds__(1024) scan_kernel(const int* __restrict__ blockCount, int nb,
                                                    long long* __restrict__ offsets, const int* stop)
{
    __shared__ long long part[1024];
    if (stop && *stop) return;
    const int per = (nb + 1023) / 1024;
    const int b0 = threadIdx.x * per;
    long long s = 0;
    for (int i = 0; i < per && b0 + i < nb; ++i) s += blockCount[b0 + i];
    part[threadIdx.x] = s;
    __syncthreads();
    for (int d = 1; d < 1024; d <<= 1) {
        const long long v = threadIdx.x >= d ? part[threadIdx.x - d] : 0;
        __syncthreads();
        part[threadIdx.x] += v;
        __syncthreads();
    }
    long long run = part[threadIdx.x] - s;  // exclusive
    for (int i = 0; i < per && b0 + i < nb; ++i) {
        offsets[b0 + i] = run;
        run += blockCount[b0 + i];
    }
    if (threadIdx.x == 1023) offsets[nb] = part[1023];
}

// Selected grid indices in ascending order.
__global__ void __launch_bounds__(kChunkThreads) compact_kernel(const unsigned char* __restrict__ flag, long long n,
                                                                unsigned char want, unsigned char exclude,
                                                                const long long* __restrict__ offsets,
                                                                long long* __restrict__ list, const int* stop)
{
    __shared__ int warpTot[kChunkThreads / 32];
    if (stop && *stop) return;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    long long out = offsets[blockIdx.x];
    const long long base = (long long)blockIdx.x * kChunk;
    for (int r = 0; r < kChunk; r += kChunkThreads) {
        const long long g = base + r + threadIdx.x;
        const bool sel = g < n && selected(flag[g], want, exclude);
        const unsigned ball = __ballot_sync(0xffffffffu, sel);
        if (lane == 0) warpTot[w] = __popc(ball);
        __syncthreads();
        int before = 0, all = 0;
        for (int i = 0; i < kChunkThreads / 32; ++i) {
            if (i < w) before += warpTot[i];
            all += warpTot[i];
        }
        if (sel) list[out + before + __popc(ball & ((1u << lane) - 1u))] = g;
        out += all;
        __syncthreads();
    }
}

// Device state of the recompute: statistics of the replaced predictions, then
// the plan of the current round.
struct Refine {
    unsigned long long boundary, lowConf, audit, auditOnly, auditOnlyAgree, changed, expanded;
    double errSum;
    unsigned long long errMaxBits;
    long long n0;       // rule-selected points fed first (ascending grid index in `rule`)
    long long pos;      // of which taken by the rounds so far
    long long d0;       // audit-only points that fill rounds (ascending, in `fill`)
    long long dpos;     // of which taken so far
    long long nA, nB;   // this round: expansion marks, then rule points rule[from, from + nB)
    long long from;
    long long nC;       // then fill points fill[dfrom, dfrom + nC)
    long long dfrom;
    long long nSel;     // nA + nB + nC: the round's list length
    long long refined;  // points computed by all rounds
    long long tiles;    // 32-point warp tiles of all rounds
    int rounds;         // rounds that computed at least one point
    int stop;           // a round found nothing to compute: the later rounds are empty
    int radius;         // expansion radius after this round
};

// One thread: the round's list is every expansion mark of the previous rounds
// (nMarked, already compacted to the list's head) and the next chunk of rule
// points, at least target/4 of them, so that the chain of expansion rounds
// overlaps the bulk of the recompute; together about `target` points.  Then,
// when audit-only points are kept back (d0 > 0), as many of them as fill the
// round up to a whole number of waves of `wave` resident points (a round with
// nothing else takes `target` of them).
// The expansion after the round uses radius `idleR` when the round fills less
// than half a wave (the chain of expansion rounds alone: the wider ring costs
// no time there), else `busyR`.
__global__ void plan_kernel(const long long* __restrict__ nMarked, Refine* R, long long target, long long wave,
                            int round, int busyR, int idleR)
{
    if (R->stop) return;
    const long long nA = *nMarked;
    long long nB = target - nA > target / 4 ? target - nA : target / 4;
    if (nB > R->n0 - R->pos) nB = R->n0 - R->pos;
    const long long base = nA + nB;
    long long nC = base == 0 ? target : (base + wave - 1) / wave * wave - base;
    if (nC > R->d0 - R->dpos) nC = R->d0 - R->dpos;
    const long long nSel = base + nC;
    R->nA = nA;
    R->nB = nB;
    R->from = R->pos;
    R->pos += nB;
    R->nC = nC;
    R->dfrom = R->dpos;
    R->dpos += nC;
    R->nSel = nSel;
    R->refined += nSel;
    R->tiles += (nSel + 31) / 32;
    R->radius = 2 * nSel < wave ? idleR : busyR;
    if (nSel > 0) R->rounds = round + 1;
    else R->stop = 1;
}

// The round's rule chunk and fill chunk after its expansion marks.
__global__ void copy_rule_kernel(const long long* __restrict__ rule, const long long* __restrict__ fill,
                                 long long* __restrict__ list, const Refine* R)
{
    const long long nA = R->nA, nB = R->nB, from = R->from, nC = R->nC, dfrom = R->dfrom;
    const long long step = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < nB + nC; i += step)
        list[nA + i] = i < nB ? rule[from + i] : fill[dfrom + i - nB];
}

// Plain results into the map; statistics of the predictions they replace;
// surprise[k] = the plain class differs from the predicted one.
__global__ void merge_kernel(const long long* __restrict__ list, const long long* __restrict__ nSel,
                             const double* __restrict__ rl, const int* __restrict__ rc,
                             unsigned char* __restrict__ flag, double* __restrict__ mapLle,
                             int* __restrict__ mapCls, unsigned char* __restrict__ src,
                             unsigned char* __restrict__ surprise, Refine* st)
{
    const long long n = *nSel;
    const long long step = (long long)gridDim.x * blockDim.x;
    unsigned long long b = 0, lc = 0, au = 0, ao = 0, aa = 0, ch = 0, ex = 0;
    double es = 0, em = 0;
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += step) {
        const long long g = list[k];
        const unsigned char f = flag[g];
        const int pc = mapCls[g];
        const double pl = mapLle[g];
        b += (f & kBoundary) != 0;
        lc += (f & kLowConf) != 0;
        au += (f & kAudit) != 0;
        ex += (f & kReasons) == kExpand;
        const bool changed = pc != rc[k];
        ch += changed;
        surprise[k] = (unsigned char)changed;
        if (f == kAudit) {
            ++ao;
            aa += pc == rc[k];
            const double err = fabs(pl - rl[k]);
            if (isfinite(err)) {
                es += err;
                em = fmax(em, err);
            }
        }
        mapLle[g] = rl[k];
        mapCls[g] = rc[k];
        src[g] = 2;
        flag[g] = f | kDone;
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        b += __shfl_down_sync(0xffffffffu, b, o);
        lc += __shfl_down_sync(0xffffffffu, lc, o);
        au += __shfl_down_sync(0xffffffffu, au, o);
        ao += __shfl_down_sync(0xffffffffu, ao, o);
        aa += __shfl_down_sync(0xffffffffu, aa, o);
        ch += __shfl_down_sync(0xffffffffu, ch, o);
        ex += __shfl_down_sync(0xffffffffu, ex, o);
        es += __shfl_down_sync(0xffffffffu, es, o);
        em = fmax(em, __shfl_down_sync(0xffffffffu, em, o));
    }
    if ((threadIdx.x & 31) == 0) {
        if (b) atomicAdd(&st->boundary, b);
        if (lc) atomicAdd(&st->lowConf, lc);
        if (au) atomicAdd(&st->audit, au);
        if (ao) atomicAdd(&st->auditOnly, ao);
        if (aa) atomicAdd(&st->auditOnlyAgree, aa);
        if (ch) atomicAdd(&st->changed, ch);
        if (ex) atomicAdd(&st->expanded, ex);
        if (es != 0) atomicAdd(&st->errSum, es);
        if (em > 0) atomicMax(&st->errMaxBits, (unsigned long long)__double_as_longlong(em));
    }
}

// Neighbours (Chebyshev radius) of every surprised point that no rule selected
// and the plain method has not computed are marked for the next round (rule-
// selected points are computed in their own chunk and expand from there).
// The list length is *nDev when given, else nHost.
__global__ void expand_kernel(const long long* __restrict__ list, const unsigned char* __restrict__ surprise,
                              const long long* __restrict__ nDev, long long nHost, int nPts, int radiusHost,
                              const int* radiusDev, unsigned char* __restrict__ flag)
{
    const long long n = nDev ? *nDev : nHost;
    const int radius = radiusDev ? *radiusDev : radiusHost;
    const long long step = (long long)gridDim.x * blockDim.x;
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += step) {
        if (!surprise[k]) continue;
        const long long g = list[k];
        const int row = (int)(g / nPts), col = (int)(g % nPts);
        for (int dr = -radius; dr <= radius; ++dr) {
            const int r = row + dr;
            if (r < 0 || r >= nPts) continue;
            for (int dc = -radius; dc <= radius; ++dc) {
                const int q = col + dc;
                if (q < 0 || q >= nPts) continue;
                const long long nb = (long long)r * nPts + q;
                if (flag[nb] == 0) flag[nb] = kExpand;
            }
        }
    }
}

template <class F>
cudaError_t launch1d(long long n, cudaStream_t s, F f)
{
    if (n <= 0) return cudaSuccess;
    f((unsigned)((n + 255) / 256), 256);
    note_launch();
    return cudaGetLastError();
}

// The pipeline's buffers, kept per device between calls and grown on demand,
// together with the network (and so its captured training graph): a repeated
// map allocates nothing.  cbf_surrogate_release frees them.
enum Slot {
    kSlotIdx, kSlotLabLle, kSlotLabCls, kSlotX, kSlotYl, kSlotConf, kSlotFlag, kSlotSrc, kSlotBlock,
    kSlotOffsets, kSlotStats, kSlotLsur, kSlotRule, kSlotFill, kSlotList, kSlotRl, kSlotRc, kSlotSur, kSlotErr,
    kSlotScratch, kNumSlots
};

struct Workspace {
    void* ptr[kNumSlots] = {};
    size_t bytes[kNumSlots] = {};
    cbf_mlp* net = nullptr;
    int netBatch = 0;

    template <class T>
    cudaError_t get(int slot, T** p, long long n)
    {
        const size_t need = (size_t)(n > 0 ? n : 1) * sizeof(T);
        if (bytes[slot] < need) {
            if (ptr[slot]) cudaFree(ptr[slot]);
            ptr[slot] = nullptr;
            bytes[slot] = 0;
            cudaError_t e = cudaMalloc(&ptr[slot], need);
            if (e != cudaSuccess) {
                ptr[slot] = nullptr;
                *p = nullptr;
                return e;
            }
            bytes[slot] = need;
        }
        *p = (T*)ptr[slot];
        return cudaSuccess;
    }
    void release()
    {
        for (int i = 0; i < kNumSlots; ++i) {
            if (ptr[i]) cudaFree(ptr[i]);
            ptr[i] = nullptr;
            bytes[i] = 0;
        }
        if (net) cbf_mlp_destroy(net);
        net = nullptr;
        netBatch = 0;
    }
};

constexpr int kMaxDevices = 64;
Workspace g_ws[kMaxDevices];
std::mutex g_ws_mu[kMaxDevices];

// Device copies of the refined map for the host-buffer entry point, kept per
// device between calls like the workspace.
struct HostMapBuffers {
    double* lle = nullptr;
    int* cls = nullptr;
    long long n = 0;
    void release()
    {
        if (lle) cudaFree(lle);
        if (cls) cudaFree(cls);
        lle = nullptr;
        cls = nullptr;
        n = 0;
    }
};
HostMapBuffers g_hostMap[kMaxDevices];
std::mutex g_hostMap_mu[kMaxDevices];

}  // namespace
}  // namespace cbf

using namespace cbf;

extern "C" {

void cbf_surrogate_config_init(cbf_surrogate_config* c)
{
    if (!c) return;
    memset(c, 0, sizeof(*c));
    c->coarseSide = 512;
    c->randomPoints = 65536;
    c->batch = 4096;
    c->trainSteps = 1500;
    c->lr = 2e-3f;
    c->wLle = 1.0f;
    c->confThreshold = 0.4f;
    c->auditFraction = 0.01f;
    c->boundaryRadius = 1;
    c->refine = 1;
    c->seed = 20240101ull;
    c->expandRadius = -1;
    c->maxWaves = 12;
}

cbf_status cbf_lle_map_surrogate(const cbf_job* job, const cbf_surrogate_config* cfg, double* dLle,
                                 int32_t* dCls, uint8_t* dSource, float* dConf, int32_t* dPred,
                                 cbf_surrogate_report* rep, void* stream)
{
    if (!job || !cfg || !dLle || !dCls) return report_error(CBF_ERR_INVALID_ARG, "null argument");
    if (job->task != CBF_TASK_LLE_REGIME || job->dims != 2 || job->sweepIC)
        return report_error(CBF_ERR_INVALID_ARG, "the surrogate map needs a 2-D LLE_REGIME parameter sweep");
    if (job->system != CBF_SYS_ROSSLER && job->system != CBF_SYS_LORENZ && job->system != CBF_SYS_CHEN)
        return report_error(CBF_ERR_INVALID_ARG, "the surrogate supports the Rossler, Lorenz and Chen systems");
    if (job->pointIndex || job->firstPoint != 0 ||
        (job->nPoints != 0 && job->nPoints != (int64_t)job->nPts * job->nPts))
        return report_error(CBF_ERR_INVALID_ARG, "the surrogate map covers the whole grid");
    if (job->nPts < 3 || cfg->coarseSide < 2 || cfg->randomPoints < 0 || cfg->batch < 1 ||
        cfg->trainSteps < 0 || !(cfg->lr > 0) || cfg->boundaryRadius < 0 || cfg->boundaryRadius > 8 ||
        cfg->expandRadius < -1 || cfg->expandRadius > 16 || cfg->maxWaves < 0 || cfg->maxWaves > 1000000 ||
        cfg->predictor < 0 || cfg->predictor > 1 || cfg->auditFill < 0 || cfg->auditFill > 1 || cfg->idleRadius < 0 || cfg->idleRadius > 16 || !(cfg->auditFraction >= 0 && cfg->auditFraction <= 1))
        return report_error(CBF_ERR_INVALID_ARG, "bad surrogate configuration");
    DevJob dj;
    cbf_status st = lower_job_for(job, &dj);
    if (st != CBF_OK) return st;

    cudaStream_t s = (cudaStream_t)stream;
    cudaStream_t own = nullptr;
    if (!s) {
        cudaDeviceSynchronize();
        if (cudaStreamCreateWithFlags(&own, cudaStreamNonBlocking) != cudaSuccess)
            return report_cuda_error(cudaGetLastError(), "stream");
        s = own;
    }
    struct StreamGuard {
        cudaStream_t s;
        ~StreamGuard()
        {
            if (s) cudaStreamDestroy(s);
        }
    } guard{own};

    const int nPts = job->nPts;
    const long long n = (long long)nPts * nPts;
    const int cs = cfg->coarseSide < nPts ? cfg->coarseSide : nPts;
    const int stride = nPts / cs;
    const long long nLab = (long long)cs * cs + cfg->randomPoints;

    cudaEvent_t ev[6];
    for (auto& e : ev) cudaEventCreate(&e);
    struct EventGuard {
        cudaEvent_t* e;
        ~EventGuard()
        {
            for (int i = 0; i < 6; ++i) cudaEventDestroy(e[i]);
        }
    } evGuard{ev};

    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
        return report_error(CBF_ERR_INVALID_ARG, "no usable current device");
    std::lock_guard<std::mutex> wsLock(g_ws_mu[dev]);  // one map at a time per device
    Workspace& buf = g_ws[dev];
    long long* dIdx = nullptr;
    double* labLle = nullptr;
    int* labCls = nullptr;
    float *X = nullptr, *yl = nullptr, *conf = dConf;
    unsigned char *flag = nullptr, *src = dSource;
    int* blockCount = nullptr;
    long long* offsets = nullptr;
    Refine* stats = nullptr;
    const int nb = (int)((n + kChunk - 1) / kChunk);
    cudaError_t e = buf.get(kSlotIdx, &dIdx, nLab);
    if (e == cudaSuccess) e = buf.get(kSlotLabLle, &labLle, nLab);
    if (e == cudaSuccess) e = buf.get(kSlotLabCls, &labCls, nLab);
    if (e == cudaSuccess) e = buf.get(kSlotX, &X, nLab * 4);
    if (e == cudaSuccess) e = buf.get(kSlotYl, &yl, nLab);
    if (e == cudaSuccess && !conf) e = buf.get(kSlotConf, &conf, n);
    if (e == cudaSuccess) e = buf.get(kSlotFlag, &flag, n);
    if (e == cudaSuccess && !src) e = buf.get(kSlotSrc, &src, n);
    if (e == cudaSuccess) e = buf.get(kSlotBlock, &blockCount, nb);
    if (e == cudaSuccess) e = buf.get(kSlotOffsets, &offsets, (long long)nb + 1);
    if (e == cudaSuccess) e = buf.get(kSlotStats, &stats, 1);
    if (e != cudaSuccess) return report_cuda_error(e, "surrogate map buffers");

    // 1. plain labels
    cudaEventRecord(ev[0], s);
    e = launch1d(nLab, s, [&](unsigned b, int t) {
        label_index_kernel<<<b, t, 0, s>>>(dIdx, cs, stride, nPts, cfg->randomPoints, n, cfg->seed);
    });
    if (e != cudaSuccess) return report_cuda_error(e, "label points");
    cbf_job lj = *job;
    lj.pointIndex = (const int64_t*)dIdx;
    lj.nPoints = nLab;
    lj.firstPoint = 0;
    if ((st = cbf_run(&lj, labLle, labCls, s)) != CBF_OK) return st;

    // LLE normalisation on the host (finite labels), targets clipped to +-8 sd.
    std::vector<double> hl(nLab);
    e = cudaMemcpyAsync(hl.data(), labLle, nLab * sizeof(double), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return report_cuda_error(e, "label readback");
    double sum = 0, sum2 = 0;
    long long cnt = 0;
    for (double v : hl)
        if (isfinite(v)) {
            sum += v;
            sum2 += v * v;
            ++cnt;
        }
    const double mean = cnt ? sum / cnt : 0.0;
    double sd = cnt ? sqrt(fmax(sum2 / cnt - mean * mean, 0.0)) : 1.0;
    if (!(sd > 1e-12)) sd = 1.0;
    std::vector<float> hy(nLab);
    for (long long i = 0; i < nLab; ++i) {
        const double v = hl[i];
        const double z = isfinite(v) ? (v - mean) / sd : 0.0;
        hy[i] = (float)fmin(8.0, fmax(-8.0, z));
    }
    e = cudaMemcpyAsync(yl, hy.data(), nLab * sizeof(float), cudaMemcpyHostToDevice, s);
    const FeatureSpec fs = feature_spec(dj);
    if (e == cudaSuccess) e = mlp_features(fs, dIdx, nLab, X, s);
    if (e != cudaSuccess) return report_cuda_error(e, "training set");
    cudaEventRecord(ev[1], s);

    // 2. training
    if (buf.net && buf.netBatch != cfg->batch) {
        cbf_mlp_destroy(buf.net);
        buf.net = nullptr;
    }
    if (!buf.net) {
        if ((st = cbf_mlp_create(cfg->batch, cfg->seed, &buf.net)) != CBF_OK) return st;
        buf.netBatch = cfg->batch;
    } else if ((e = mlp_reset(buf.net, cfg->seed)) != cudaSuccess) {
        return report_cuda_error(e, "network reset");
    }
    cbf_mlp* net = buf.net;
    {
        // Encoding frequencies at a fixed fraction of what the label lattice
        // resolves: scale coarseSide/512 rounded to a power of two (measured best
        // at 512^2 labels with scale 1, at 64^2 with 1/8; higher frequencies than
        // the labels resolve let the network fit between labels at random).
        int ex = (int)lrint(log2((double)cs / 512.0));
        ex = ex < -8 ? -8 : (ex > 4 ? 4 : ex);
        if ((st = cbf_mlp_set_encoding_scale(net, ldexpf(1.0f, ex))) != CBF_OK) return st;
    }
    const bool learned = cfg->predictor == 0;
    const int tail = !learned ? 0 : (cfg->trainSteps < 100 ? cfg->trainSteps : 100);
    std::vector<float> losses(tail > 0 ? tail : 1, 0.f);
    if (learned) {
        st = cbf_mlp_train(net, X, yl, labCls, nLab, cfg->trainSteps - tail, cfg->lr, cfg->trainSteps, cfg->wLle,
                           nullptr, s);
        if (st == CBF_OK && tail > 0)
            st = cbf_mlp_train(net, X, yl, labCls, nLab, tail, cfg->lr, cfg->trainSteps, cfg->wLle, losses.data(),
                               s);
        if (st != CBF_OK) return st;
    }
    cudaEventRecord(ev[2], s);

    // 3. prediction on every grid point (the ablation: the nearest coarse label)
    if (learned)
        e = mlp_predict_grid(net, fs, n, (float)mean, (float)sd, dLle, dCls, conf, s);
    else
        e = launch1d(n, s, [&](unsigned b, int t) {
            nearest_label_kernel<<<b, t, 0, s>>>(labLle, labCls, cs, stride, nPts, n, dLle, dCls, conf);
        });
    if (e == cudaSuccess && dPred) e = cudaMemcpyAsync(dPred, dCls, (size_t)n * sizeof(int32_t), cudaMemcpyDeviceToDevice, s);
    if (e != cudaSuccess) return report_cuda_error(e, "prediction");
    cudaEventRecord(ev[3], s);

    // 4. refinement mask, labels into the map (surprised labels seed the expansion)
    const double frac = cfg->refine ? cfg->auditFraction : 0.0;
    const unsigned long long auditCut =
        frac >= 1.0 ? ~0ull : (unsigned long long)(frac * 18446744073709551616.0);
    const float thr = cfg->refine ? cfg->confThreshold : -1.0f;
    const int radius = cfg->refine ? cfg->boundaryRadius : 0;  // radius 0 marks no boundary
    // expansion radius: automatic = one grid step per 8192 points of side, so
    // that the rounds needed to trace a structure grow slower than nPts
    const int autoR = (nPts + 8191) / 8192;
    const int er = cfg->refine ? (cfg->expandRadius < 0 ? autoR : cfg->expandRadius) : 0;
    unsigned char* lsur = nullptr;
    if ((e = buf.get(kSlotLsur, &lsur, nLab)) != cudaSuccess) return report_cuda_error(e, "label buffers");
    e = launch1d(n, s, [&](unsigned b, int t) {
        mask_kernel<<<b, t, 0, s>>>(dCls, conf, nPts, n, radius, thr, auditCut,
                                    cfg->seed ^ 0xA0761D6478BD642Full, flag, src);
    });
    if (e == cudaSuccess)
        e = launch1d(nLab, s, [&](unsigned b, int t) {
            label_scatter_kernel<<<b, t, 0, s>>>(dIdx, nLab, labLle, labCls, dLle, dCls, flag, src, lsur);
        });
    if (e == cudaSuccess && er > 0)
        e = launch1d(nLab, s, [&](unsigned b, int t) {
            expand_kernel<<<b, t, 0, s>>>(dIdx, lsur, nullptr, nLab, nPts, er, nullptr, flag);
        });
    if (e == cudaSuccess) e = cudaMemsetAsync(stats, 0, sizeof(Refine), s);
    if (e != cudaSuccess) return report_cuda_error(e, "refinement mask");
    cudaEventRecord(ev[4], s);

    // 5. plain recompute in rounds.  The rule-selected points (ascending grid
    // index) are fed in chunks; every round also takes all points the expansion
    // marked in the previous rounds, so the chain of expansion rounds overlaps
    // the bulk of the recompute.  A round is sized to about two waves of
    // resident threads of the LLE_REGIME kernel.  With auditFill, points that
    // only the audit selected are kept back and fill every round up to a whole
    // number of waves.  plan_kernel sizes each round on the device; the host
    // launches a fixed number of rounds, enough for every chunk and every
    // expansion round, and the rounds after the last one with work return at
    // once.
    const bool fillAudit = cfg->auditFill != 0;
    const int idleR = cfg->idleRadius > 0 && er > 0 ? cfg->idleRadius : er;
    const unsigned char want = kBoundary | kLowConf | (fillAudit ? 0 : kAudit);
    long long* rule = nullptr;
    long long* fillList = nullptr;
    long long* list = nullptr;
    double* rl = nullptr;
    int* rc = nullptr;
    unsigned char* sur = nullptr;
    int* rerr = nullptr;
    double* scr = nullptr;
    const size_t scrBytes = lle_regime_scratch_bytes(dj);
    e = buf.get(kSlotRule, &rule, n);
    if (e == cudaSuccess) e = buf.get(kSlotFill, &fillList, fillAudit ? n : 1);
    if (e == cudaSuccess) e = buf.get(kSlotList, &list, n);
    if (e == cudaSuccess) e = buf.get(kSlotRl, &rl, n);
    if (e == cudaSuccess) e = buf.get(kSlotRc, &rc, n);
    if (e == cudaSuccess) e = buf.get(kSlotSur, &sur, n);
    if (e == cudaSuccess) e = buf.get(kSlotErr, &rerr, 1);
    if (e == cudaSuccess) e = buf.get(kSlotScratch, &scr, (long long)(scrBytes / sizeof(double)) + 1);
    if (e != cudaSuccess) return report_cuda_error(e, "recompute buffers");
    if (scrBytes == 0) return report_error(CBF_ERR_INTERNAL, "recompute: no resident LLE_REGIME blocks");
    long long n0 = 0, d0 = 0;
    count_kernel<<<nb, kChunkThreads, 0, s>>>(flag, n, want, 0, blockCount, nullptr);
    scan_kernel<<<1, 1024, 0, s>>>(blockCount, nb, offsets, nullptr);
    compact_kernel<<<nb, kChunkThreads, 0, s>>>(flag, n, want, 0, offsets, rule, nullptr);
    note_launch(3);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(&stats->n0, offsets + nb, sizeof(long long), cudaMemcpyDeviceToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&n0, offsets + nb, sizeof(long long), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && fillAudit) {
        count_kernel<<<nb, kChunkThreads, 0, s>>>(flag, n, kAudit, kBoundary | kLowConf, blockCount, nullptr);
        scan_kernel<<<1, 1024, 0, s>>>(blockCount, nb, offsets, nullptr);
        compact_kernel<<<nb, kChunkThreads, 0, s>>>(flag, n, kAudit, kBoundary | kLowConf, offsets, fillList, nullptr);
        note_launch(3);
        e = cudaGetLastError();
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(&stats->d0, offsets + nb, sizeof(long long), cudaMemcpyDeviceToDevice, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(&d0, offsets + nb, sizeof(long long), cudaMemcpyDeviceToHost, s);
    }
    if (e == cudaSuccess) e = cudaMemsetAsync(rerr, 0, sizeof(int), s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return report_cuda_error(e, "recompute list");
    long long resident = lle_regime_resident_points(dj);
    if (resident < 4096) resident = 4096;
    const long long target = 2 * resident;
    // Rounds with rule points: at most ceil(n0 / (target/4)).  Expansion marks
    // come from the labels and the rounds before round maxWaves, and every round
    // takes all of them: rounds with marks but no rule points, at most
    // maxWaves + 1.  Rounds with fill points alone take `target` of them: at
    // most ceil(d0 / target).  One more round finds nothing and sets `stop`.
    const int maxRounds = (int)((n0 + target / 4 - 1) / (target / 4)) + (er > 0 ? cfg->maxWaves + 1 : 0) +
                          (int)((d0 + target - 1) / target) + 1;
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const long long fillBlocks = (long long)sms * 8;
    auto gridFor = [&](long long m) { return (unsigned)((m + 255) / 256 < fillBlocks ? (m + 255) / 256 : fillBlocks); };
    DevJob rj = dj;
    rj.pointIndex = list;
    rj.firstPoint = 0;
    rj.nPoints = n;
    const long long* nSel = &stats->nSel;
    const int* stop = &stats->stop;
    for (int w = 0; w < maxRounds; ++w) {
        if (w > 0 && w % 64 == 0) {  // long expansion chains: stop launching once a round found nothing
            int hostStop = 0;
            e = cudaMemcpyAsync(&hostStop, stop, sizeof(int), cudaMemcpyDeviceToHost, s);
            if (e == cudaSuccess) e = cudaStreamSynchronize(s);
            if (e != cudaSuccess) return report_cuda_error(e, "recompute rounds");
            if (hostStop) break;
        }
        count_kernel<<<nb, kChunkThreads, 0, s>>>(flag, n, kExpand, 0, blockCount, stop);
        scan_kernel<<<1, 1024, 0, s>>>(blockCount, nb, offsets, stop);
        compact_kernel<<<nb, kChunkThreads, 0, s>>>(flag, n, kExpand, 0, offsets, list, stop);
        plan_kernel<<<1, 1, 0, s>>>(offsets + nb, stats, target, resident, w, er, idleR);
        copy_rule_kernel<<<gridFor(target), 256, 0, s>>>(rule, fillList, list, stats);
        note_launch(5);
        if ((e = cudaGetLastError()) != cudaSuccess) return report_cuda_error(e, "recompute list");
        if ((e = launch_lle_regime_list(rj, nSel, n, rl, rc, scr, scrBytes, rerr, s)) != cudaSuccess)
            return report_cuda_error(e, "recompute");
        merge_kernel<<<gridFor(n), 256, 0, s>>>(list, nSel, rl, rc, flag, dLle, dCls, src, sur, stats);
        note_launch();
        if (er > 0 && w < cfg->maxWaves) {
            expand_kernel<<<gridFor(n), 256, 0, s>>>(list, sur, nSel, 0, nPts, 0, &stats->radius, flag);
            note_launch();
        }
        if ((e = cudaGetLastError()) != cudaSuccess) return report_cuda_error(e, "merge");
    }
    Refine hs;
    memset(&hs, 0, sizeof(hs));
    int hostErr = 0;
    e = cudaMemcpyAsync(&hs, stats, sizeof(Refine), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&hostErr, rerr, sizeof(int), cudaMemcpyDeviceToHost, s);
    cudaEventRecord(ev[5], s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return report_cuda_error(e, "recompute");
    if (hostErr) return report_error(CBF_ERR_INTERNAL, "surrogate recompute: a device-side check failed");
    if (!hs.stop) return report_error(CBF_ERR_INTERNAL, "surrogate recompute: rounds left work undone");

    if (rep) {
        memset(rep, 0, sizeof(*rep));
        rep->points = n;
        rep->labelled = nLab;
        rep->refined = (int64_t)hs.refined;
        rep->expanded = (int64_t)hs.expanded;
        rep->waves = hs.rounds;
        rep->refineTiles = (int64_t)hs.tiles;
        rep->boundary = (int64_t)hs.boundary;
        rep->lowConfidence = (int64_t)hs.lowConf;
        rep->audit = (int64_t)hs.audit;
        rep->auditOnly = (int64_t)hs.auditOnly;
        rep->auditOnlyAgree = (int64_t)hs.auditOnlyAgree;
        rep->refinedChanged = (int64_t)hs.changed;
        rep->auditOnlyLleMeanAbsErr = hs.auditOnly ? hs.errSum / (double)hs.auditOnly : 0.0;
        double mx;
        memcpy(&mx, &hs.errMaxBits, sizeof(mx));
        rep->auditOnlyLleMaxAbsErr = mx;
        rep->lleMean = mean;
        rep->lleStd = sd;
        double ls = 0;
        for (int i = 0; i < tail; ++i) ls += losses[i];
        rep->finalLoss = tail ? (float)(ls / tail) : 0.f;
        float ms[5];
        for (int i = 0; i < 5; ++i) cudaEventElapsedTime(&ms[i], ev[i], ev[i + 1]);
        rep->msLabel = ms[0];
        rep->msTrain = ms[1];
        rep->msPredict = ms[2];
        rep->msMask = ms[3];
        rep->msRefine = ms[4];
        float tot = 0;
        cudaEventElapsedTime(&tot, ev[0], ev[5]);
        rep->msTotal = tot;
    }
    return CBF_OK;
}

void cbf_regime_rules_init(cbf_regime_rules* r)
{
    if (!r) return;
    memset(r, 0, sizeof(*r));
    r->regimeTime = 50.0;
    r->maxAmountOfPeaks = 512;
    r->dbscanEps = 0.02;
    r->regimeMinAmp = 1e-6;
    r->regimeChaosLle = 0.05;
    r->flags = 0;
}

// LLE2D's arguments (hostLibrary.cu:1524-1663) plus the regime rules and the
// surrogate configuration; the refined map is computed into cached device
// buffers on the library's stream and copied into the caller's host arrays.
cbf_status cbf_lle2d_surrogate(int32_t system, double tMax, double NT, int32_t nPts, double h, double eps,
                               const double* initialConditions, int32_t amountOfInitialConditions,
                               const double* ranges, const int32_t* indicesOfMutVars, int32_t writableVar,
                               double maxValue, double transientTime, const double* values,
                               int32_t amountOfValues, int64_t seedChunk, const cbf_regime_rules* rules,
                               const cbf_surrogate_config* cfg, double* outLle, int32_t* outCls,
                               cbf_surrogate_report* report)
{
    if (!initialConditions || !ranges || !indicesOfMutVars || !values || !outLle)
        return report_error(CBF_ERR_INVALID_ARG, "null argument");
    if (amountOfInitialConditions < 1 || amountOfInitialConditions > CBF_MAX_DIM || amountOfValues < 1 ||
        amountOfValues > CBF_MAX_VALUES)
        return report_error(CBF_ERR_INVALID_ARG, "amountOfInitialConditions/amountOfValues out of range");
    cbf_regime_rules r;
    if (rules) r = *rules;
    else cbf_regime_rules_init(&r);
    cbf_surrogate_config c;
    if (cfg) c = *cfg;
    else cbf_surrogate_config_init(&c);
    cbf_job j;
    cbf_job_init(&j);
    j.task = CBF_TASK_LLE_REGIME;
    j.system = system;
    j.dims = 2;
    j.nPts = nPts;
    j.h = h;
    j.tMax = tMax;
    j.NT = NT;
    j.lleEps = eps;
    j.transientTime = transientTime;
    j.maxValue = maxValue;
    j.writableVar = writableVar;
    j.seedChunk = seedChunk;
    j.nIC = amountOfInitialConditions;
    j.nV = amountOfValues;
    for (int i = 0; i < j.nIC; ++i) j.ic[i] = initialConditions[i];
    for (int i = 0; i < j.nV; ++i) j.values[i] = values[i];
    for (int i = 0; i < 4; ++i) j.ranges[i] = ranges[i];
    j.idxMut[0] = indicesOfMutVars[0];
    j.idxMut[1] = indicesOfMutVars[1];
    j.regimeTime = r.regimeTime;
    j.maxAmountOfPeaks = r.maxAmountOfPeaks;
    j.dbscanEps = r.dbscanEps;
    j.regimeMinAmp = r.regimeMinAmp;
    j.regimeChaosLle = r.regimeChaosLle;
    j.flags = r.flags;
    cbf_status st = cbf_validate(&j);
    if (st != CBF_OK) return st;

    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
        return report_error(CBF_ERR_INVALID_ARG, "no usable current device");
    cudaStream_t s = nullptr;
    if ((st = library_default_stream(&s)) != CBF_OK) return st;
    const long long n = (long long)nPts * nPts;
    std::lock_guard<std::mutex> lk(g_hostMap_mu[dev]);
    HostMapBuffers& hm = g_hostMap[dev];
    if (hm.n < n) {
        hm.release();
        cudaError_t e = cudaMalloc((void**)&hm.lle, (size_t)n * sizeof(double));
        if (e == cudaSuccess) e = cudaMalloc((void**)&hm.cls, (size_t)n * sizeof(int));
        if (e != cudaSuccess) {
            hm.release();
            return report_cuda_error(e, "refined map buffers");
        }
        hm.n = n;
    }
    if ((st = cbf_lle_map_surrogate(&j, &c, hm.lle, hm.cls, nullptr, nullptr, nullptr, report, s)) != CBF_OK)
        return st;
    cudaError_t e = cudaMemcpyAsync(outLle, hm.lle, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && outCls)
        e = cudaMemcpyAsync(outCls, hm.cls, (size_t)n * sizeof(int32_t), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return report_cuda_error(e, "refined map readback");
    return CBF_OK;
}

void cbf_surrogate_release(void)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return;
    {
        std::lock_guard<std::mutex> lk(g_hostMap_mu[dev]);
        g_hostMap[dev].release();
    }
    std::lock_guard<std::mutex> lk(g_ws_mu[dev]);
    g_ws[dev].release();
}

}  // extern "C"
