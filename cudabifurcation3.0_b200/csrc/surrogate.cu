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
// network's, its neighbours (expandRadius) are recomputed too, and so on up to
// an expansion depth of maxWaves steps from a rule point or label: thin
// structures the network cannot resolve (periodic windows inside chaos) are
// traced from any point that hits them.  The recompute is one persistent launch
// whose warps pull work from a device queue (lle_regime.cu, RefineCtx); the set
// of computed points, and so the map, does not depend on the order in which the
// warps run.  Labelled and recomputed points carry plain values; the rest carry
// the network's prediction.  The audit points that no other rule selected measure
// the error of the kept predictions.  Everything runs on one stream; the host
// reads the labels back once (to normalise the LLE targets) and waits once at
// the end.
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
constexpr unsigned char kBoundary = kRefBoundary, kLowConf = kRefLowConf, kAudit = kRefAudit;
constexpr unsigned char kDone = kRefDone, kLabel = kRefLabel;

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

// Points with one of the `want` reasons that are neither labels nor computed.
__device__ __forceinline__ bool selected(unsigned char f, unsigned char want)
{
    return (f & want) && !(f & (kLabel | kDone));
}

__global__ void __launch_bounds__(kChunkThreads) count_kernel(const unsigned char* __restrict__ flag, long long n,
                                                              unsigned char want, int* __restrict__ blockCount)
{
    const long long base = (long long)blockIdx.x * kChunk;
    int total = 0;
    for (int r = 0; r < kChunk; r += kChunkThreads) {
        const long long g = base + r + threadIdx.x;
        total += __syncthreads_count(g < n && selected(flag[g], want));
    }
    if (threadIdx.x == 0) blockCount[blockIdx.x] = total;
}

// Exclusive prefix over nb block counts (one block of 1024 threads);
// offsets[nb] = total.
__global__ void __launch_bounds__(1024) scan_kernel(const int* __restrict__ blockCount, int nb,
                                                    long long* __restrict__ offsets)
{
    __shared__ long long part[1024];
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
                                                                unsigned char want,
                                                                const long long* __restrict__ offsets,
                                                                long long* __restrict__ list)
{
    __shared__ int warpTot[kChunkThreads / 32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    long long out = offsets[blockIdx.x];
    const long long base = (long long)blockIdx.x * kChunk;
    for (int r = 0; r < kChunk; r += kChunkThreads) {
        const long long g = base + r + threadIdx.x;
        const bool sel = g < n && selected(flag[g], want);
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
    kSlotOffsets, kSlotStats, kSlotLsur, kSlotRule, kSlotDepth, kSlotQueue, kSlotCounters, kSlotErr,
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
    c->maxWaves = 20;
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
        cfg->predictor < 0 || cfg->predictor > 1 || !(cfg->auditFraction >= 0 && cfg->auditFraction <= 1))
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
    RefineStats* stats = nullptr;
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
    if (e == cudaSuccess) e = cudaMemsetAsync(stats, 0, sizeof(RefineStats), s);
    if (e != cudaSuccess) return report_cuda_error(e, "refinement mask");
    cudaEventRecord(ev[4], s);

    // 5. plain recompute in one persistent launch: the rule-selected points
    // (ascending grid index) and, from every label or computed point whose plain
    // class differs from the prediction, its neighbours within the expansion
    // radius, up to expansion depth maxWaves (RefineCtx, engine.cuh).  The host
    // waits once, at the end.
    const unsigned char want = kBoundary | kLowConf | kAudit;
    long long* rule = nullptr;
    int* depth = nullptr;
    int* queue = nullptr;
    unsigned long long* counters = nullptr;
    int* rerr = nullptr;
    double* scr = nullptr;
    const size_t scrBytes = refine_scratch_bytes(dj);
    // each point enters the queue once for computation, and again only when its
    // depth drops after it was expanded (rare): room for all points and half again
    const unsigned long long qCap = (unsigned long long)n + (unsigned long long)n / 2 + 1024;
    e = buf.get(kSlotRule, &rule, n);
    if (e == cudaSuccess) e = buf.get(kSlotDepth, &depth, n);
    if (e == cudaSuccess) e = buf.get(kSlotQueue, &queue, (long long)qCap);
    if (e == cudaSuccess) e = buf.get(kSlotCounters, &counters, 6);
    if (e == cudaSuccess) e = buf.get(kSlotErr, &rerr, 1);
    if (e == cudaSuccess) e = buf.get(kSlotScratch, &scr, (long long)(scrBytes / sizeof(double)) + 1);
    if (e != cudaSuccess) return report_cuda_error(e, "recompute buffers");
    count_kernel<<<nb, kChunkThreads, 0, s>>>(flag, n, want, blockCount);
    scan_kernel<<<1, 1024, 0, s>>>(blockCount, nb, offsets);
    compact_kernel<<<nb, kChunkThreads, 0, s>>>(flag, n, want, offsets, rule);
    note_launch(3);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemsetAsync(queue, 0xff, qCap * sizeof(int), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(counters, 0, 6 * sizeof(unsigned long long), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(rerr, 0, sizeof(int), s);
    if (e != cudaSuccess) return report_cuda_error(e, "recompute list");
    RefineCtx R;
    memset(&R, 0, sizeof(R));
    R.rule = rule;
    R.nRule = offsets + nb;
    R.queue = queue;
    R.qCap = qCap;
    R.counters = counters;
    R.depth = depth;
    R.flag = flag;
    R.mapLle = dLle;
    R.mapCls = dCls;
    R.src = src;
    R.stats = stats;
    R.err = rerr;
    R.labelIdx = dIdx;
    R.labelSurprise = lsur;
    R.nLabel = nLab;
    R.scrPk = scr;
    R.scrBytes = scrBytes;
    R.nPts = nPts;
    R.radius = er;
    R.maxDepth = er > 0 ? cfg->maxWaves : 0;
    // an idle warp waits while others finish their tiles: allow far more than the
    // integration of one point (~1e-7 s per step at most) before calling it stuck
    const double stepsPerPoint = (double)dj.nSkip + 2.0 * (double)dj.nRecord * (double)dj.nNT;
    R.maxIdleNs = (unsigned long long)(60e9 + stepsPerPoint * 1000.0);
    if ((e = launch_regime_refine(dj, R, s)) != cudaSuccess) return report_cuda_error(e, "recompute");
    RefineStats hs;
    memset(&hs, 0, sizeof(hs));
    int hostErr = 0;
    e = cudaMemcpyAsync(&hs, stats, sizeof(RefineStats), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&hostErr, rerr, sizeof(int), cudaMemcpyDeviceToHost, s);
    cudaEventRecord(ev[5], s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return report_cuda_error(e, "recompute");
    if (hostErr == 2 || hostErr == 4)
        return report_error(CBF_ERR_TIMEOUT, "surrogate recompute: a bounded device-side wait gave up");
    if (hostErr) return report_error(CBF_ERR_INTERNAL, "surrogate recompute: a device-side check failed");

    if (rep) {
        memset(rep, 0, sizeof(*rep));
        rep->points = n;
        rep->labelled = nLab;
        rep->refined = (int64_t)hs.computed;
        rep->expanded = (int64_t)hs.expanded;
        rep->waves = hs.deepest;
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
