// C-ABI of ragged batches (cbf_batch_*): planning, autotuning, graph capture.
#include <string.h>

#include <algorithm>
#include <vector>

#include "engine.cuh"

namespace cbf {

constexpr int kFamilies = 2;  // 0: LLE jobs, 1: peak-based jobs (PEAKS, KDE, DBSCAN)

cudaError_t batch_launch(const void* jobs, int nJobs, const long long* tileEnd,
                         unsigned long long* counter, double* scrPk, double* scrIv, int stride,
                         int bitWords, int* err, int grid, bool withM5, int fam, cudaStream_t s);
int batch_max_blocks_per_sm(int bitWords, bool withM5, int fam);
size_t batch_job_bytes();
int batch_threads();
int batch_tile();
int batch_max_jobs();
void batch_plan(const DevJob* jobs, void* const* outs, void* const* auxs, int n,
                std::vector<unsigned char>& packed, std::vector<long long>& tileEnd,
                std::vector<int>& order);
cbf_status run_job_lowered(const DevJob& d, void* d_out, void* d_aux, cudaStream_t s);

}  // namespace cbf

using namespace cbf;

// The jobs of one kernel family, with their own descriptor table, queue counter
// and grid.
struct BatchFamily {
    std::vector<int> jobIdx;  // indices into cbf_batch::jobs
    void* d_jobs = nullptr;
    long long* d_tileEnd = nullptr;
    bool withM5 = false;      // a job uses the 5-D shipped model
    int maxBlocksPerSm = 0;
    int blocksPerSm = 0;
    long long points = 0;
};

struct cbf_batch {
    int device = 0;
    int nJobs = 0;
    std::vector<DevJob> jobs;
    std::vector<void*> outs, auxs;
    std::vector<int> order;  // all jobs, longest per point first (one-by-one runs)
    BatchFamily fam[kFamilies];
    unsigned long long* d_counter = nullptr;  // [0], [1] queue heads, then the error flag
    int* d_err = nullptr;
    double* d_scrPk = nullptr;
    double* d_scrIv = nullptr;
    int stride = 0;
    int bitWords = 0;
    int sms = 1;
    long long totalPoints = 0;
    cudaStream_t side = nullptr;  // the second family's stream (fork/join)
    cudaEvent_t evFork = nullptr, evJoin = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

namespace {

int family_of(const DevJob& d) { return d.task == CBF_TASK_LLE ? 0 : 1; }

void release_graph(cbf_batch* b)
{
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
}

void release_all(cbf_batch* b)
{
    release_graph(b);
    for (BatchFamily& F : b->fam) {
        cudaFree(F.d_jobs);
        cudaFree(F.d_tileEnd);
        F.d_jobs = nullptr;
        F.d_tileEnd = nullptr;
    }
    cudaFree(b->d_counter);
    cudaFree(b->d_scrPk);
    if (b->evFork) cudaEventDestroy(b->evFork);
    if (b->evJoin) cudaEventDestroy(b->evJoin);
    if (b->side) cudaStreamDestroy(b->side);
    b->d_counter = nullptr;
    b->d_scrPk = nullptr;
    b->d_scrIv = nullptr;
    b->evFork = b->evJoin = nullptr;
    b->side = nullptr;
}

// Descriptor table and tile prefix of family f from `jobs` (the batch's jobs or
// a shortened copy of them).
cbf_status upload(cbf_batch* b, int f, const std::vector<DevJob>& jobs, void** d_jobs, long long** d_end)
{
    const BatchFamily& F = b->fam[f];
    std::vector<DevJob> sub;
    std::vector<void*> outs, auxs;
    for (int i : F.jobIdx) {
        sub.push_back(jobs[i]);
        outs.push_back(b->outs[i]);
        auxs.push_back(b->auxs[i]);
    }
    std::vector<unsigned char> packed;
    std::vector<long long> tileEnd;
    std::vector<int> order;
    batch_plan(sub.data(), outs.data(), auxs.data(), (int)sub.size(), packed, tileEnd, order);
    cudaError_t e = cudaMalloc(d_jobs, packed.size());
    if (e == cudaSuccess) e = cudaMalloc((void**)d_end, tileEnd.size() * sizeof(long long));
    if (e == cudaSuccess) e = cudaMemcpy(*d_jobs, packed.data(), packed.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemcpy(*d_end, tileEnd.data(), tileEnd.size() * sizeof(long long), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return report_cuda_error(e, "batch descriptors");
    return CBF_OK;
}

cbf_status launch_family(cbf_batch* b, int f, void* d_jobs, long long* d_end, int blocksPerSm, cudaStream_t s)
{
    const BatchFamily& F = b->fam[f];
    const int grid = std::max(1, b->sms * blocksPerSm);
    cudaError_t e = batch_launch(d_jobs, (int)F.jobIdx.size(), d_end, b->d_counter + f, b->d_scrPk, b->d_scrIv,
                                 b->stride, f == 1 ? b->bitWords : 0, b->d_err, grid, F.withM5, f, s);
    if (e != cudaSuccess) return report_cuda_error(e, "batch launch");
    return CBF_OK;
}

// One run: the error flag cleared, then every non-empty family's persistent
// kernel; with two families the second runs on the side stream (fork/join by
// events, which stream capture records as parallel branches), so its blocks
// take the SMs the first family's blocks leave as its queue drains.
cbf_status launch_all(cbf_batch* b, cudaStream_t s)
{
    cudaError_t e = cudaMemsetAsync(b->d_err, 0, sizeof(int), s);
    if (e != cudaSuccess) return report_cuda_error(e, "batch error flag");
    const bool two = !b->fam[0].jobIdx.empty() && !b->fam[1].jobIdx.empty();
    if (!two) {
        const int f = b->fam[0].jobIdx.empty() ? 1 : 0;
        return launch_family(b, f, b->fam[f].d_jobs, b->fam[f].d_tileEnd, b->fam[f].blocksPerSm, s);
    }
    if (!b->side) {
        e = cudaStreamCreateWithFlags(&b->side, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->evFork, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->evJoin, cudaEventDisableTiming);
        if (e != cudaSuccess) return report_cuda_error(e, "batch side stream");
    }
    e = cudaEventRecord(b->evFork, s);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(b->side, b->evFork, 0);
    if (e != cudaSuccess) return report_cuda_error(e, "batch fork");
    cbf_status st = launch_family(b, 0, b->fam[0].d_jobs, b->fam[0].d_tileEnd, b->fam[0].blocksPerSm, s);
    cbf_status st2 = launch_family(b, 1, b->fam[1].d_jobs, b->fam[1].d_tileEnd, b->fam[1].blocksPerSm, b->side);
    e = cudaEventRecord(b->evJoin, b->side);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(s, b->evJoin, 0);
    if (st != CBF_OK) return st;
    if (st2 != CBF_OK) return st2;
    if (e != cudaSuccess) return report_cuda_error(e, "batch join");
    return CBF_OK;
}

}  // namespace

extern "C" {

cbf_status cbf_batch_create(const cbf_job* jobs, int32_t nJobs, void* const* d_outs,
                            void* const* d_auxs, cbf_batch** out)
{
    if (!out) return report_error(CBF_ERR_INVALID_ARG, "null batch handle");
    *out = nullptr;
    if (!jobs || !d_outs || nJobs < 1 || nJobs > batch_max_jobs())
        return report_error(CBF_ERR_INVALID_ARG, "a batch holds 1..1024 jobs with output buffers");
    cbf_batch* b = new cbf_batch();
    b->nJobs = nJobs;
    b->jobs.resize(nJobs);
    b->outs.assign(d_outs, d_outs + nJobs);
    b->auxs.assign(nJobs, nullptr);
    bool anyDbscan = false;
    int cap = 0;
    for (int i = 0; i < nJobs; ++i) {
        cbf_status st = lower_job_for(&jobs[i], &b->jobs[i]);
        if (st != CBF_OK) {
            delete b;
            return st;
        }
        const DevJob& d = b->jobs[i];
        if (d.task != CBF_TASK_PEAKS && d.task != CBF_TASK_KDE && d.task != CBF_TASK_DBSCAN &&
            d.task != CBF_TASK_LLE) {
            delete b;
            return report_error(CBF_ERR_INVALID_ARG,
                                "only PEAKS, KDE, DBSCAN and LLE jobs can be batched");
        }
        if (d_auxs) b->auxs[i] = d_auxs[i];
        if (!b->outs[i] || (d.task == CBF_TASK_PEAKS && !b->auxs[i])) {
            delete b;
            return report_error(CBF_ERR_INVALID_ARG, "missing device output buffer for a batch job");
        }
        if (d.task == CBF_TASK_KDE || d.task == CBF_TASK_DBSCAN) cap = std::max(cap, d.peakCap);
        if (d.task == CBF_TASK_DBSCAN) anyDbscan = true;
        BatchFamily& F = b->fam[family_of(d)];
        F.jobIdx.push_back(i);
        if (d.system == CBF_SYS_MEMRISTIVE5) F.withM5 = true;
        F.points += d.nPoints;
        b->totalPoints += d.nPoints;
    }
    cudaError_t e = cudaGetDevice(&b->device);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, b->device);
    if (e != cudaSuccess) {
        delete b;
        return report_cuda_error(e, "device query");
    }
    b->stride = cap;
    b->bitWords = anyDbscan ? (cap + 31) / 32 : 0;
    for (int f = 0; f < kFamilies; ++f) {
        BatchFamily& F = b->fam[f];
        if (F.jobIdx.empty()) continue;
        F.maxBlocksPerSm = batch_max_blocks_per_sm(f == 1 ? b->bitWords : 0, F.withM5, f);
        if (F.maxBlocksPerSm < 1) {
            delete b;
            return report_error(CBF_ERR_INVALID_ARG, "batch kernel does not fit an SM");
        }
    }
    // Peak scratch of the peak family's largest grid within min(8 GB, free/4).
    if (cap > 0 && !b->fam[1].jobIdx.empty()) {
        size_t freeB = 0, totalB = 0;
        cudaMemGetInfo(&freeB, &totalB);
        size_t budget = std::min((size_t)8 << 30, freeB / 4);
        const size_t perBlock = (size_t)batch_threads() * cap * sizeof(double) * (anyDbscan ? 2 : 1);
        int fit = (int)std::min<size_t>(budget / perBlock / (size_t)b->sms, 64);
        if (fit < 1) {
            delete b;
            return report_error(CBF_ERR_OUT_OF_MEMORY, "batch scratch does not fit one block per SM");
        }
        BatchFamily& F = b->fam[1];
        F.maxBlocksPerSm = std::min(F.maxBlocksPerSm, fit);
        const size_t blocks = (size_t)b->sms * F.maxBlocksPerSm;
        e = cudaMalloc((void**)&b->d_scrPk, blocks * perBlock);
        if (e != cudaSuccess) {
            delete b;
            return report_cuda_error(e, "batch scratch");
        }
        if (anyDbscan) b->d_scrIv = b->d_scrPk + blocks * batch_threads() * (size_t)cap;
    }
    for (BatchFamily& F : b->fam) F.blocksPerSm = F.maxBlocksPerSm;
    e = cudaMalloc((void**)&b->d_counter, 256);
    if (e != cudaSuccess) {
        release_all(b);
        delete b;
        return report_cuda_error(e, "batch counter");
    }
    b->d_err = (int*)(b->d_counter + kFamilies);
    {  // one-by-one order over all jobs, longest per point first
        std::vector<unsigned char> packed;
        std::vector<long long> tileEnd;
        batch_plan(b->jobs.data(), b->outs.data(), b->auxs.data(), nJobs, packed, tileEnd, b->order);
    }
    for (int f = 0; f < kFamilies; ++f) {
        if (b->fam[f].jobIdx.empty()) continue;
        cbf_status st = upload(b, f, b->jobs, &b->fam[f].d_jobs, &b->fam[f].d_tileEnd);
        if (st != CBF_OK) {
            release_all(b);
            delete b;
            return st;
        }
    }
    *out = b;
    return CBF_OK;
}

void cbf_batch_destroy(cbf_batch* b)
{
    if (!b) return;
    release_all(b);
    delete b;
}

int64_t cbf_batch_points(const cbf_batch* b) { return b ? b->totalPoints : -1; }

// Blocks per SM of the family with more points.
int32_t cbf_batch_blocks_per_sm(const cbf_batch* b)
{
    if (!b) return -1;
    return b->fam[0].points >= b->fam[1].points ? b->fam[0].blocksPerSm : b->fam[1].blocksPerSm;
}

cbf_status cbf_batch_run(cbf_batch* b, void* stream)
{
    if (!b) return report_error(CBF_ERR_INVALID_ARG, "null batch");
    return launch_all(b, (cudaStream_t)stream);
}

cbf_status cbf_batch_capture(cbf_batch* b, void* stream)
{
    if (!b) return report_error(CBF_ERR_INVALID_ARG, "null batch");
    cudaStream_t s = (cudaStream_t)stream;
    if (!s) {
        cbf_status st = library_default_stream(&s);
        if (st != CBF_OK) return st;
    }
    release_graph(b);
    // Set the shared-memory attributes and create the side stream outside the capture.
    for (int f = 0; f < kFamilies; ++f)
        if (!b->fam[f].jobIdx.empty()) batch_max_blocks_per_sm(f == 1 ? b->bitWords : 0, b->fam[f].withM5, f);
    if (!b->fam[0].jobIdx.empty() && !b->fam[1].jobIdx.empty() && !b->side) {
        cudaError_t ce = cudaStreamCreateWithFlags(&b->side, cudaStreamNonBlocking);
        if (ce == cudaSuccess) ce = cudaEventCreateWithFlags(&b->evFork, cudaEventDisableTiming);
        if (ce == cudaSuccess) ce = cudaEventCreateWithFlags(&b->evJoin, cudaEventDisableTiming);
        if (ce != cudaSuccess) return report_cuda_error(ce, "batch side stream");
    }
    cudaError_t e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return report_cuda_error(e, "cudaStreamBeginCapture");
    cbf_status st = launch_all(b, s);
    cudaGraph_t g = nullptr;
    e = cudaStreamEndCapture(s, &g);
    if (st != CBF_OK) {
        if (g) cudaGraphDestroy(g);
        return st;
    }
    if (e != cudaSuccess) return report_cuda_error(e, "cudaStreamEndCapture");
    b->graph = g;
    e = cudaGraphInstantiate(&b->exec, g, 0);
    if (e != cudaSuccess) {
        release_graph(b);
        return report_cuda_error(e, "cudaGraphInstantiate");
    }
    return CBF_OK;
}

cbf_status cbf_batch_launch(cbf_batch* b, void* stream)
{
    if (!b) return report_error(CBF_ERR_INVALID_ARG, "null batch");
    if (!b->exec) return report_error(CBF_ERR_INVALID_ARG, "cbf_batch_capture has not been called");
    cudaError_t e = cudaGraphLaunch(b->exec, (cudaStream_t)stream);
    if (e != cudaSuccess) return report_cuda_error(e, "cudaGraphLaunch");
    note_launch();
    return CBF_OK;
}

cbf_status cbf_batch_check(cbf_batch* b)
{
    if (!b) return report_error(CBF_ERR_INVALID_ARG, "null batch");
    int err = 0;
    cudaError_t e = cudaMemcpy(&err, b->d_err, sizeof(int), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return report_cuda_error(e, "batch status");
    if (err) return report_error(CBF_ERR_INTERNAL, "device-side iteration guard fired in a batch");
    return CBF_OK;
}

cbf_status cbf_batch_run_sequential(cbf_batch* b, void* stream)
{
    if (!b) return report_error(CBF_ERR_INVALID_ARG, "null batch");
    for (int k = 0; k < b->nJobs; ++k) {
        const int i = b->order[k];
        cbf_status st = run_job_lowered(b->jobs[i], b->outs[i], b->auxs[i], (cudaStream_t)stream);
        if (st != CBF_OK) return st;
    }
    return CBF_OK;
}

// Times the candidate grids (blocks per SM) of each family on a copy of its
// jobs with every transient and record cut by 32x, so each candidate runs the
// same mix of systems, tasks and grid sizes; each family keeps its fastest.
// blocksPerSm receives the choice of the family with more points,
// msPerCandidate[c] the sum over the families that ran candidate c (-1: none).
// The outputs are overwritten by the trial.
cbf_status cbf_batch_autotune(cbf_batch* b, void* stream, int32_t* blocksPerSm, double* msPerCandidate)
{
    if (!b) return report_error(CBF_ERR_INVALID_ARG, "null batch");
    cudaStream_t s = (cudaStream_t)stream;
    std::vector<DevJob> shortJobs = b->jobs;
    for (DevJob& d : shortJobs) {
        d.nSkip = d.nSkip / 32;
        if (d.task == CBF_TASK_LLE) d.nRecord = std::max(1, d.nRecord / 32);
        else d.nRecord = std::max(3, d.nRecord / 32);
    }
    const int cands[8] = {1, 2, 3, 4, 6, 8, 12, 16};
    if (msPerCandidate)
        for (int c = 0; c < 8; ++c) msPerCandidate[c] = -1.0;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cbf_status st = CBF_OK;
    for (int f = 0; f < kFamilies && st == CBF_OK; ++f) {
        BatchFamily& F = b->fam[f];
        if (F.jobIdx.empty()) continue;
        void* dj = nullptr;
        long long* de = nullptr;
        st = upload(b, f, shortJobs, &dj, &de);
        float best = -1.f;
        int bestB = F.maxBlocksPerSm;
        for (int c = 0; c < 8 && st == CBF_OK; ++c) {
            if (cands[c] > F.maxBlocksPerSm) continue;
            cudaMemsetAsync(b->d_err, 0, sizeof(int), s);
            st = launch_family(b, f, dj, de, cands[c], s);  // warm-up
            if (st != CBF_OK) break;
            cudaEventRecord(e0, s);
            st = launch_family(b, f, dj, de, cands[c], s);
            cudaEventRecord(e1, s);
            if (st != CBF_OK) break;
            cudaError_t e = cudaEventSynchronize(e1);
            if (e != cudaSuccess) {
                st = report_cuda_error(e, "batch autotune");
                break;
            }
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            if (msPerCandidate) msPerCandidate[c] = (msPerCandidate[c] < 0 ? 0.0 : msPerCandidate[c]) + ms;
            if (best < 0 || ms < best) {
                best = ms;
                bestB = cands[c];
            }
        }
        cudaFree(dj);
        cudaFree(de);
        if (st == CBF_OK) F.blocksPerSm = bestB;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (st != CBF_OK) return st;
    release_graph(b);  // a captured graph used the old grids
    if (blocksPerSm) *blocksPerSm = cbf_batch_blocks_per_sm(b);
    return CBF_OK;
}

}  // extern "C"
