// C-ABI of ragged batches (cbf_batch_*): planning, autotuning, graph capture.
#include <string.h>

#include <algorithm>
#include <vector>

#include "engine.cuh"

namespace cbf {

cudaError_t batch_launch(const void* jobs, int nJobs, const long long* tileEnd,
                         unsigned long long* counter, double* scrPk, double* scrIv, int stride,
                         int bitWords, int* err, int grid, bool withM5, cudaStream_t s);
int batch_max_blocks_per_sm(int bitWords, bool withM5);
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

struct cbf_batch {
    int device = 0;
    int nJobs = 0;
    std::vector<DevJob> jobs;
    std::vector<void*> outs, auxs;
    std::vector<int> order;
    void* d_jobs = nullptr;
    long long* d_tileEnd = nullptr;
    unsigned long long* d_counter = nullptr;  // [0] queue head, then the error flag
    int* d_err = nullptr;
    double* d_scrPk = nullptr;
    double* d_scrIv = nullptr;
    int stride = 0;
    int bitWords = 0;
    bool withM5 = false;  // a job uses the 5-D shipped model
    int maxBlocksPerSm = 1;
    int blocksPerSm = 1;
    int sms = 1;
    long long totalPoints = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

namespace {

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
    cudaFree(b->d_jobs);
    cudaFree(b->d_tileEnd);
    cudaFree(b->d_counter);
    cudaFree(b->d_scrPk);
    b->d_jobs = nullptr;
    b->d_tileEnd = nullptr;
    b->d_counter = nullptr;
    b->d_scrPk = nullptr;
    b->d_scrIv = nullptr;
}

cbf_status upload(cbf_batch* b, const std::vector<DevJob>& jobs, void** d_jobs, long long** d_end,
                  std::vector<int>* orderOut)
{
    std::vector<unsigned char> packed;
    std::vector<long long> tileEnd;
    std::vector<int> order;
    batch_plan(jobs.data(), b->outs.data(), b->auxs.data(), b->nJobs, packed, tileEnd, order);
    if (orderOut) *orderOut = order;
    cudaError_t e = cudaMalloc(d_jobs, packed.size());
    if (e == cudaSuccess) e = cudaMalloc((void**)d_end, tileEnd.size() * sizeof(long long));
    if (e == cudaSuccess) e = cudaMemcpy(*d_jobs, packed.data(), packed.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemcpy(*d_end, tileEnd.data(), tileEnd.size() * sizeof(long long), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return report_cuda_error(e, "batch descriptors");
    return CBF_OK;
}

cbf_status launch_with(cbf_batch* b, void* d_jobs, long long* d_end, int blocksPerSm, cudaStream_t s)
{
    const int grid = std::max(1, b->sms * blocksPerSm);
    cudaError_t e = batch_launch(d_jobs, b->nJobs, d_end, b->d_counter, b->d_scrPk, b->d_scrIv,
                                 b->stride, b->bitWords, b->d_err, grid, b->withM5, s);
    if (e != cudaSuccess) return report_cuda_error(e, "batch launch");
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
        if (d.system == CBF_SYS_MEMRISTIVE5) b->withM5 = true;
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
    b->maxBlocksPerSm = batch_max_blocks_per_sm(b->bitWords, b->withM5);
    if (b->maxBlocksPerSm < 1) {
        delete b;
        return report_error(CBF_ERR_INVALID_ARG, "batch kernel does not fit an SM");
    }
    // Scratch for the largest grid that fits a budget of min(8 GB, free/4).
    if (cap > 0) {
        size_t freeB = 0, totalB = 0;
        cudaMemGetInfo(&freeB, &totalB);
        size_t budget = std::min((size_t)8 << 30, freeB / 4);
        const size_t perBlock = (size_t)batch_threads() * cap * sizeof(double) * (anyDbscan ? 2 : 1);
        int fit = (int)std::min<size_t>(budget / perBlock / (size_t)b->sms, 64);
        if (fit < 1) {
            delete b;
            return report_error(CBF_ERR_OUT_OF_MEMORY, "batch scratch does not fit one block per SM");
        }
        b->maxBlocksPerSm = std::min(b->maxBlocksPerSm, fit);
        const size_t blocks = (size_t)b->sms * b->maxBlocksPerSm;
        const size_t bytes = blocks * perBlock;
        e = cudaMalloc((void**)&b->d_scrPk, bytes);
        if (e != cudaSuccess) {
            delete b;
            return report_cuda_error(e, "batch scratch");
        }
        if (anyDbscan) b->d_scrIv = b->d_scrPk + blocks * batch_threads() * (size_t)cap;
    }
    b->blocksPerSm = b->maxBlocksPerSm;
    e = cudaMalloc((void**)&b->d_counter, 256);
    if (e != cudaSuccess) {
        release_all(b);
        delete b;
        return report_cuda_error(e, "batch counter");
    }
    b->d_err = (int*)(b->d_counter + 1);
    cbf_status st = upload(b, b->jobs, &b->d_jobs, &b->d_tileEnd, &b->order);
    if (st != CBF_OK) {
        release_all(b);
        delete b;
        return st;
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

int32_t cbf_batch_blocks_per_sm(const cbf_batch* b) { return b ? b->blocksPerSm : -1; }

cbf_status cbf_batch_run(cbf_batch* b, void* stream)
{
    if (!b) return report_error(CBF_ERR_INVALID_ARG, "null batch");
    return launch_with(b, b->d_jobs, b->d_tileEnd, b->blocksPerSm, (cudaStream_t)stream);
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
    // Set the shared-memory attribute outside the capture.
    batch_max_blocks_per_sm(b->bitWords, b->withM5);
    cudaError_t e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return report_cuda_error(e, "cudaStreamBeginCapture");
    cbf_status st = launch_with(b, b->d_jobs, b->d_tileEnd, b->blocksPerSm, s);
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

// Times the candidate grids (blocks per SM) on a copy of the batch with every
// job's transient and record cut by 32x, so each candidate runs the same mix of
// systems, tasks and grid sizes.  The outputs are overwritten by the trial.
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
    void* dj = nullptr;
    long long* de = nullptr;
    cbf_status st = upload(b, shortJobs, &dj, &de, nullptr);
    if (st != CBF_OK) return st;
    const int cands[8] = {1, 2, 3, 4, 6, 8, 12, 16};
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float best = -1.f;
    int bestB = b->maxBlocksPerSm;
    for (int c = 0; c < 8 && st == CBF_OK; ++c) {
        if (msPerCandidate) msPerCandidate[c] = -1.0;
        if (cands[c] > b->maxBlocksPerSm) continue;
        st = launch_with(b, dj, de, cands[c], s);  // warm-up
        if (st != CBF_OK) break;
        cudaEventRecord(e0, s);
        st = launch_with(b, dj, de, cands[c], s);
        cudaEventRecord(e1, s);
        if (st != CBF_OK) break;
        cudaError_t e = cudaEventSynchronize(e1);
        if (e != cudaSuccess) {
            st = report_cuda_error(e, "batch autotune");
            break;
        }
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (msPerCandidate) msPerCandidate[c] = ms;
        if (best < 0 || ms < best) {
            best = ms;
            bestB = cands[c];
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(dj);
    cudaFree(de);
    if (st != CBF_OK) return st;
    b->blocksPerSm = bestB;
    release_graph(b);  // a captured graph used the old grid
    if (blocksPerSm) *blocksPerSm = bestB;
    return CBF_OK;
}

}  // extern "C"
