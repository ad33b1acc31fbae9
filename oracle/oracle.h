/*
 * CPU oracle for the bifurcation hot path -- TEST INFRASTRUCTURE ONLY.
 *
 * This is a plain-C restatement of the reference library's per-point algorithm
 * (CUDABifurcation3.0, Library/cudaLibrary.cu and Library/hostLibrary.cu).  It
 * exists to check the CUDA product path: only tests/, the smoke() hook and the
 * CPU-baseline leg of bench.py may load it.  Nothing in the product links it.
 *
 * Floating-point policy: compiled with -ffp-contract=off, so every expression is
 * evaluated exactly as written in the reference source (no implicit FMA).  The
 * model steps of the Rossler / Lorenz / Chen systems are the library's own
 * definitions (the reference hard-codes one user-supplied system per build); they
 * use explicit fma() in the same places as the CUDA kernels.  FP32 libm calls
 * (sinf, expf, hypotf, powf, fabsf) are glibc's here and CUDA's on the device, so
 * results that depend on them are compared with the tolerance stated by each test.
 *
 * Pinning: the functions that the reference declares __host__ __device__
 * (getValueByIdx, calculateDiscreteModel, loopCalculateDiscreteModel, peakFinder,
 * kde, distance, dbscan) are checked bit-for-bit against the reference's own
 * sources compiled for the host (oracle/Makefile target `ref`) and against the
 * golden vectors under tests/golden/.
 */
#ifndef CBF_ORACLE_H
#define CBF_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    ORC_SYS_MEMRISTIVE5 = 0, /* the model shipped in cudaLibrary.cu:2-44 */
    ORC_SYS_ROSSLER = 1,
    ORC_SYS_LORENZ = 2,
    ORC_SYS_CHEN = 3
};

/* Everything one map computation needs; mirrors the hostLibrary argument lists. */
typedef struct orc_job {
    double ranges[4];
    double ic[8];
    double values[16];
    double h;
    double tMax;
    double transientTime;
    double maxValue;
    double NT;        /* LLE renormalisation interval */
    double lleEps;    /* LLE initial offset */
    double kdeI1, kdeI2, kdeH;
    double dbscanEps;
    int64_t seedChunk; /* LLE seed index = global index mod seedChunk (0: no wrap) */
    int32_t system;
    int32_t sweepIC;   /* 0: sweep values[], 1: sweep initial conditions */
    int32_t dims;      /* 1 or 2 swept axes */
    int32_t nPts;      /* points per axis */
    int32_t nIC;
    int32_t nV;
    int32_t idxMut[2];
    int32_t writableVar;
    int32_t preScaller;
    int32_t maxAmountOfPeaks;
    int32_t kdeSampling;
    double regimeTime;  /* LLE + regime: window after the transient (time units) */
    double regimeMinAmp; /* LLE + regime: window range below this -> class 0 */
    double regimeChaosLle; /* LLE + regime: > 0 and LLE above it -> class 15 */
    double ostrovskyThreshold; /* periodicity classifier threshold */
    int32_t exactGrid; /* 1: grid cell by integer division (the library's CBF_FLAG_EXACT_GRID)
                          instead of getValueByIdx's FP32 index */
} orc_job;

/* cudaLibrary.cu:210-216 */
double orc_get_value_by_idx(int idx, int nPts, double startRange, double finishRange, int valueNumber);
/* cudaLibrary.cu:2-44 and the library's own Rossler/Lorenz/Chen CD steps */
int orc_system_dim(int system);
void orc_model_step(int system, double* x, const double* a, double h);
/* cudaLibrary.cu:55-74; returns 1 (true) or 0 (false) */
int orc_loop(int system, double* x, const double* values, double h, int amountOfIterations,
             int preScaller, int writableVar, double maxValue, double* data,
             int64_t startDataIndex, int writeStep);
/* cudaLibrary.cu:220-266 */
int orc_peak_finder(double* data, int64_t startDataIndex, int amountOfPoints,
                    double* outPeaks, double* timeOfPeaks, double h);
/* cudaLibrary.cu:356-422 */
int orc_kde(const double* data, int64_t startDataIndex, int amountOfPoints, int maxAmountOfPeaks,
            int kdeSampling, double kdeSamplesInterval1, double kdeSamplesInterval2,
            double kdeSmoothH);
/* kde's sampling/mode-count body with a given sample count k1 (cudaLibrary.cu:367-421) */
int orc_kde_k1(const double* data, int64_t startDataIndex, int amountOfPoints, int k1,
               double kdeSamplesInterval1, double kdeSamplesInterval2, double kdeSmoothH);
/* cudaLibrary.cu:445-453 */
double orc_distance(double x1, double y1, double x2, double y2);
/* cudaLibrary.cu:457-529 */
int orc_dbscan(const double* data, const double* intervals, double* helpfulArray,
               int64_t startDataIndex, int amountOfPeaks, int sizeOfHelpfulArray,
               int maxAmountOfPeaks, double eps);

/* Derived sizes, with the reference's own int truncations (hostLibrary.cu:22-23, 1286-1288). */
int orc_record_len(const orc_job* job);   /* (int)(tMax / h / preScaller) */
int orc_skip_len(const orc_job* job);     /* (int)(transientTime / h) */

/* Per point: trajectory of x[writableVar] (cudaLibrary.cu:78-117, IC variant :165-207).
 * Writes record samples into data[0..record); returns 1 if the divergence check fired. */
int orc_trajectory_point(const orc_job* job, int64_t g, double* data);
/* Per point: Benettin LLE (cudaLibrary.cu:666-785, IC variant :789-908). */
double orc_lle_point(const orc_job* job, int64_t g);
/* The same from a given normalised perturbation z (NULL: the seed below).  Lets
 * a check feed the device's FP32 sinf seed so that only the LLE arithmetic is
 * compared. */
double orc_lle_point_seeded(const orc_job* job, int64_t g, const double* z);
/* The seed of cudaLibrary.cu:720-732 (IC variant :843-855) with glibc sinf. */
void orc_lle_seed(const orc_job* job, int64_t g, double* z);

/* Map-level drivers over global points [first, first+count), OpenMP over points.
 * Peaks: outPeaks[k*cap + j], outIntervals likewise (may be NULL), counts[k]
 * (peakFinderCUDA, cudaLibrary.cu:270-284; 1-D host loop hostLibrary.cu:82-143). */
int orc_map_peaks(const orc_job* job, int64_t first, int64_t count, double* outPeaks,
                  double* outIntervals, int32_t* counts, int64_t cap, int nThreads);
/* kdeCUDA path (hostLibrary.cu:498-526) */
int orc_map_kde(const orc_job* job, int64_t first, int64_t count, int32_t* out, int nThreads);
/* dbscanCUDA path (hostLibrary.cu:673-700) */
int orc_map_dbscan(const orc_job* job, int64_t first, int64_t count, int32_t* out, int nThreads);
/* LLEKernelCUDA path (hostLibrary.cu:1598-1623) */
int orc_map_lle(const orc_job* job, int64_t first, int64_t count, double* out, int nThreads);
/* Same with per-point seeds z[k*nIC + i]. */
int orc_map_lle_seeded(const orc_job* job, int64_t first, int64_t count, const double* z,
                       double* out, int nThreads);
/* Same, over an explicit list of global indices (strided samples for the CPU baseline). */
int orc_map_lle_list(const orc_job* job, const int64_t* idx, int64_t count, double* out, int nThreads);
/* The list form with per-point seeds z[k*nIC + i] (NULL: the oracle's own seeds). */
int orc_map_lle_list_seeded(const orc_job* job, const int64_t* idx, int64_t count, const double* z,
                            double* out, int nThreads);

/* LLE plus peak-count regime class (the library's plain labelling method): the
 * LLE of orc_lle_point_seeded; x[writableVar] recorded before every step of the
 * base trajectory for the first (int)(regimeTime/h) steps after the transient;
 * class = 0 if the divergence test fired inside that window, no peak, or the
 * window's samples span less than regimeMinAmp (max - min, fmin/fmax); 15 if
 * regimeChaosLle > 0 and the LLE exceeds it,
 * 15 if more than maxAmountOfPeaks peaks, else min(dbscan, 15). */
double orc_lle_regime_point(const orc_job* job, int64_t g, const double* z, int32_t* cls);
/* modelingOneSystemDenis: one system, step-offset sampling (cudaLibrary.cu:121-161). */
int orc_modeling_one_system(int system, double tMax, double h, double hSpecial, const double* ic, int nIC,
                            int writableVar, const double* values, int nV, double* out, int64_t n);
/* Ostrovsky periodicity classifier (cudaLibrary.cu:288-352, 628-662). */
double orc_ostrovsky_point(const orc_job* job, int64_t g, double* data, double* intervals,
                           double* helpful);
int orc_map_ostrovsky(const orc_job* job, int64_t first, int64_t count, double* out, int nThreads);
/* Lyapunov spectrum (LSKernelCUDA, cudaLibrary.cu:913-1100). */
void orc_projection(const double* a, const double* b, double* minuend, int n);
void orc_gram_schmidt(const double* a, double* b, int n, double* den);
void orc_ls_seed(const orc_job* job, int64_t g, double* z);
void orc_ls_point(const orc_job* job, int64_t g, const double* z, double* out);
int orc_map_ls_list(const orc_job* job, const int64_t* idx, int64_t count, const double* z,
                    double* out, int nThreads);
int orc_map_lle_regime_list(const orc_job* job, const int64_t* idx, int64_t count,
                            const double* z, double* outLle, int32_t* outCls, int nThreads);

/* 1 when a Chen / Lorenz job runs the rescaled 10-operation step (y stored times
 * a per-point constant sy; the library's cbf_job_scaled_step), else 0.  Every
 * per-point routine above follows the form the job runs, and reports, records and
 * checks states in physical units. */
int orc_scaled_step(const orc_job* job);

/* Divergence test of loopCalculateDiscreteModel (cudaLibrary.cu:69-71), exposed for tests. */
int orc_diverged(double v, double maxValue);

#ifdef __cplusplus
}
#endif
#endif
