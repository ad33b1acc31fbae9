// Ragged batches: many map jobs in one persistent launch per kernel family.
//
// The reference runs one map per host call, one chunk and three kernels at a
// time.  A batch here is any mix of jobs -- systems, tasks (LLE, KDE, DBSCAN,
// 1-D peaks), grid sizes, record lengths, step sizes.  Its jobs form two
// families, LLE jobs and peak-based jobs, each executed by ONE persistent
// kernel compiled with that family's code only (so each gets its tasks'
// register count and occupancy); with both present the two kernels run
// concurrently on forked streams:
//   * every job is cut into tiles of 32 points (one warp: a lane per point);
//   * jobs are ordered by estimated cost per point, longest first, and a prefix
//     table of tile counts maps a global tile number to (job, tile);
//   * each warp takes the next tile number from a device counter (atomicAdd by
//     lane 0), so long and short jobs interleave and the tail is made of the
//     cheapest tiles;
//   * a tile runs exactly the per-point code of the map kernels (lle_device.cuh,
//     bif_device.cuh), so batch results equal one-by-one results bit for bit.
// One batch run is "reset error flag; per family: reset counter, launch" and is
// captured once as a CUDA graph for repeated sweeps.  Each family's grid
// (blocks per SM) is chosen by cbf_batch_autotune on a shortened copy of it.
#include <string.h>

#include <algorithm>
#include <vector>

#include "bif_device.cuh"
#include "lle_device.cuh"

namespace cbf {
namespace {

constexpr int kBatchWarps = 4;
constexpr int kBatchThreads = kBatchWarps * 32;
constexpr int kMaxBatchJobs = 1024;
constexpr int kTile = 32;
constexpr int kFamLle = 0, kFamPeaks = 1;

struct BatchJob {
    DevJob job;
    void* out;
    int* aux;
};

template <class S, int TASK>
__device__ __forceinline__ void bif_tile(const DevJob& J, void* out, int* aux, long long p0, int lane,
                                         double* slotPk, double* slotIv, int stride, unsigned* L,
                                         unsigned* Sb, const DbscanSort& so, int* err)
{
    const long long p = p0 + lane;
    const bool valid = p < J.nPoints;
    const long long g = grid_index(J, p);
    if (TASK == CBF_TASK_PEAKS) {
        if (valid) {
            double* pk = (double*)out + p * (long long)J.peakCap;
            aux[p] = integrate_point<S, TASK>(J, g, pk, nullptr, J.peakCap, nullptr, nullptr);
        }
        return;
    }
    double* myPk = slotPk + (long long)lane * stride;
    double* myIv = (TASK == CBF_TASK_DBSCAN) ? slotIv + (long long)lane * stride : nullptr;
    int n = 0;
    if (valid) n = integrate_point<S, TASK>(J, g, myPk, myIv, J.peakCap, nullptr, nullptr);
    __syncwarp();
    int res = 0;
    const int live = (int)min((long long)kTile, J.nPoints - p0);
    for (int j = 0; j < live; ++j) {
        const int nj = __shfl_sync(kFull, n, j);
        const double* pk = slotPk + (long long)j * stride;
        int r;
        if (TASK == CBF_TASK_KDE)
            r = kde_warp(J, pk, nj, lane);
        else
            r = dbscan_warp(J, pk, slotIv + (long long)j * stride, nj, lane, L, Sb, err, so);
        if (lane == j) res = r;
    }
    if (valid) ((int*)out)[p] = res;
    __syncwarp();
}

// FAM: the kernel family -- kFamLle runs LLE jobs only, kFamPeaks the
// peak-based tasks (PEAKS, KDE, DBSCAN).  Each family is compiled with its own
// code only, so its register count and occupancy are those of its tasks.
template <class S, int FAM>
__device__ __forceinline__ void run_tile(const DevJob& J, void* out, int* aux, long long p0, int lane,
                                         double* slotPk, double* slotIv, int stride, unsigned* L,
                                         unsigned* Sb, const DbscanSort& so, int* err)
{
    if constexpr (FAM == kFamLle) {
        const long long p = p0 + lane;
        if (p < J.nPoints) {
            const long long g = grid_index(J, p);
            ((double*)out)[p] = J.sweepIC ? lle_point<S, true>(J, g) : lle_point<S, false>(J, g);
        }
        return;
    } else {
    switch (J.task) {
    case CBF_TASK_KDE:
        bif_tile<S, CBF_TASK_KDE>(J, out, aux, p0, lane, slotPk, slotIv, stride, L, Sb, so, err);
        break;
    case CBF_TASK_DBSCAN:
        bif_tile<S, CBF_TASK_DBSCAN>(J, out, aux, p0, lane, slotPk, slotIv, stride, L, Sb, so, err);
        break;
    case CBF_TASK_PEAKS:
        bif_tile<S, CBF_TASK_PEAKS>(J, out, aux, p0, lane, slotPk, slotIv, stride, L, Sb, so, err);
        break;
    default:
        break;
    }
    }
}

// WITH_M5: also dispatch the 5-D shipped model.  Its wider state raises the
// register count of the whole kernel, so batches of 3-D systems use the
// instantiation without it.
// Both families are bounded to 6 blocks of 128 threads per SM (80 registers):
// the occupancy of the autotuned LLE map kernel, and for the peak family 1.5x
// what its register count would otherwise allow, which is worth the small
// spill of its epilogue paths (batch64: 43.6 s instead of 49.2 s).
template <int FAM, bool WITH_M5>
__global__ void __launch_bounds__(kBatchThreads, 6) batch_kernel(
    const BatchJob* __restrict__ jobs, int nJobs, const long long* __restrict__ tileEnd,
    unsigned long long* counter, double* scrPk, double* scrIv, int stride, int bitWords, int sortCap, int* err)
{
    extern __shared__ unsigned smem[];
    __shared__ long long sEnd[kMaxBatchJobs];
    for (int i = threadIdx.x; i < nJobs; i += blockDim.x) sEnd[i] = tileEnd[i];
    __syncthreads();
    const unsigned long long total = (unsigned long long)sEnd[nJobs - 1];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const long long warpId = (long long)blockIdx.x * kBatchWarps + wib;
    unsigned* L = smem + (size_t)wib * dbscan_warp_words(bitWords, sortCap);
    unsigned* Sb = L + bitWords;
    const DbscanSort so = dbscan_sort_area(L, bitWords, sortCap);
    double* slotPk = scrPk ? scrPk + warpId * kTile * (long long)stride : nullptr;
    double* slotIv = scrIv ? scrIv + warpId * kTile * (long long)stride : nullptr;

    for (;;) {
        unsigned long long t = 0;
        if (lane == 0) t = atomicAdd(counter, 1ull);
        t = __shfl_sync(kFull, t, 0);
        if (t >= total) break;
        int lo = 0, hi = nJobs - 1;  // first job whose tile range ends after t
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if ((unsigned long long)sEnd[mid] > t) hi = mid;
            else lo = mid + 1;
        }
        const long long firstTile = lo ? sEnd[lo - 1] : 0;
        const long long p0 = ((long long)t - firstTile) * kTile;
        void* out = jobs[lo].out;
        int* aux = jobs[lo].aux;
        auto go = [&](const DevJob& J) {
            switch (J.system) {
            case CBF_SYS_MEMRISTIVE5:
                if (WITH_M5) run_tile<Memristive5, FAM>(J, out, aux, p0, lane, slotPk, slotIv, stride, L, Sb, so, err);
                break;
            case CBF_SYS_ROSSLER: run_tile<Rossler, FAM>(J, out, aux, p0, lane, slotPk, slotIv, stride, L, Sb, so, err); break;
            case CBF_SYS_LORENZ:
                if (J.scaledStep && J.unitStep)  // the map kernels' 8-instruction form
                    run_tile<LorenzScaledU, FAM>(J, out, aux, p0, lane, slotPk, slotIv, stride, L, Sb, so, err);
                else if (J.scaledStep)
                    run_tile<LorenzScaled, FAM>(J, out, aux, p0, lane, slotPk, slotIv, stride, L, Sb, so, err);
                else
                    run_tile<Lorenz, FAM>(J, out, aux, p0, lane, slotPk, slotIv, stride, L, Sb, so, err);
                break;
            case CBF_SYS_CHEN:
                if (J.scaledStep && J.unitStep)  // the map kernels' 8-instruction form
                    run_tile<ChenScaledU, FAM>(J, out, aux, p0, lane, slotPk, slotIv, stride, L, Sb, so, err);
                else if (J.scaledStep)
                    run_tile<ChenScaled, FAM>(J, out, aux, p0, lane, slotPk, slotIv, stride, L, Sb, so, err);
                else
                    run_tile<Chen, FAM>(J, out, aux, p0, lane, slotPk, slotIv, stride, L, Sb, so, err);
                break;
            default: break;
            }
        };
        // The LLE family reads its descriptor in place (read-only cache); the
        // peak family keeps a copy (fewer registers in its epilogues).
        if constexpr (FAM == kFamLle) {
            go(jobs[lo].job);
        } else {
            const DevJob J = jobs[lo].job;
            go(J);
        }
    }
}

// Model steps per point, the batch's cost estimate for ordering.
double steps_per_point(const DevJob& d)
{
    if (d.task == CBF_TASK_LLE) return (double)d.nSkip + 2.0 * d.nRecord * (double)d.nNT;
    return (double)d.nSkip + (double)d.nRecord * d.preScaller;
}

}  // namespace

using BatchKernel = void (*)(const BatchJob*, int, const long long*, unsigned long long*, double*, double*,
                            int, int, int, int*);

BatchKernel batch_kernel_for(int fam, bool withM5)
{
    if (fam == kFamLle) return withM5 ? batch_kernel<kFamLle, true> : batch_kernel<kFamLle, false>;
    return withM5 ? batch_kernel<kFamPeaks, true> : batch_kernel<kFamPeaks, false>;
}

cudaError_t batch_launch(const void* jobs, int nJobs, const long long* tileEnd,
                         unsigned long long* counter, double* scrPk, double* scrIv, int stride,
                         int bitWords, int* err, int grid, bool withM5, int fam, cudaStream_t s)
{
    const int sortCap = bitWords > 0 ? dbscan_sort_cap(bitWords * 32) : 0;
    const size_t smem = (size_t)kBatchWarps * dbscan_warp_words(bitWords, sortCap) * sizeof(unsigned);
    auto kern = batch_kernel_for(fam, withM5);
    cudaError_t e;
    if (smem > 48 * 1024) {
        e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    if ((e = cudaMemsetAsync(counter, 0, sizeof(unsigned long long), s)) != cudaSuccess) return e;
    kern<<<grid, kBatchThreads, smem, s>>>((const BatchJob*)jobs, nJobs, tileEnd, counter, scrPk, scrIv,
                                           stride, bitWords, sortCap, err);
    note_launch();
    return cudaGetLastError();
}

int batch_max_blocks_per_sm(int bitWords, bool withM5, int fam)
{
    const int sortCap = bitWords > 0 ? dbscan_sort_cap(bitWords * 32) : 0;
    const size_t smem = (size_t)kBatchWarps * dbscan_warp_words(bitWords, sortCap) * sizeof(unsigned);
    auto kern = batch_kernel_for(fam, withM5);
    if (smem > 48 * 1024)
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int perSm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, kern, kBatchThreads, smem) != cudaSuccess)
        return 0;
    return perSm;
}

size_t batch_job_bytes() { return sizeof(BatchJob); }
int batch_threads() { return kBatchThreads; }
int batch_tile() { return kTile; }
int batch_max_jobs() { return kMaxBatchJobs; }

// Host-side plan: order by cost, prefix tile ends, packed device descriptors.
void batch_plan(const DevJob* jobs, void* const* outs, void* const* auxs, int n,
                std::vector<unsigned char>& packed, std::vector<long long>& tileEnd,
                std::vector<int>& order)
{
    order.resize(n);
    for (int i = 0; i < n; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
        return steps_per_point(jobs[a]) > steps_per_point(jobs[b]);
    });
    packed.assign((size_t)n * sizeof(BatchJob), 0);
    tileEnd.resize(n);
    long long acc = 0;
    for (int k = 0; k < n; ++k) {
        const int i = order[k];
        BatchJob b;
        memset(&b, 0, sizeof(b));
        b.job = jobs[i];
        b.out = outs[i];
        b.aux = auxs ? (int*)auxs[i] : nullptr;
        memcpy(packed.data() + (size_t)k * sizeof(BatchJob), &b, sizeof(b));
        acc += (jobs[i].nPoints + kTile - 1) / kTile;
        tileEnd[k] = acc;
    }
}

}  // namespace cbf
