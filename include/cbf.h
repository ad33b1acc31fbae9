/*
 * cbf.h -- C-ABI launch layer of the B200 bifurcation engine.
 *
 * Plain C types only (pointers, sizes, scalars).  Every function returns a
 * cbf_status and never exits the process; cbf_last_error() gives the detail of
 * the last failure on the calling thread.
 *
 * The reference library (CUDABifurcation3.0) exposes its hot path as C++
 * __host__ functions in Library/hostLibrary.cuh that write a CSV file.  Each
 * host-buffer entry point below replaces one of them: same argument meaning and
 * order (plus a leading `system` id, because the reference hard-codes one ODE
 * per build in Library/cudaLibrary.cu:2-44), results returned in caller buffers
 * instead of a file.  The C++ drop-in facade with the reference's exact
 * signatures and CSV output lives in hostLibrary.h and calls these functions.
 *
 * Semantics follow the reference exactly, including its documented quirks:
 *   - grid value of point g on axis v: getValueByIdx (cudaLibrary.cu:210-216),
 *     FP32 index division included (set CBF_FLAG_EXACT_GRID to opt out);
 *   - peaks: first peak dropped, intervals in units of 0.01 (cudaLibrary.cu:220-284);
 *   - KDE mode count (cudaLibrary.cu:356-441), DBSCAN cluster count
 *     (cudaLibrary.cu:457-624), Benettin LLE (cudaLibrary.cu:666-908).
 */
#ifndef CBF_H
#define CBF_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CBF_ABI_VERSION 1

typedef int32_t cbf_status;
#define CBF_OK 0
#define CBF_ERR_INVALID_ARG 1   /* bad size, index, range, unknown task */
#define CBF_ERR_UNKNOWN_SYSTEM 2
#define CBF_ERR_CUDA 3          /* a CUDA runtime call failed (detail in cbf_last_error) */
#define CBF_ERR_OUT_OF_MEMORY 4
#define CBF_ERR_NO_DEVICE 5
#define CBF_ERR_IO 6            /* façade: output file could not be written */
#define CBF_ERR_TIMEOUT 7       /* a bounded device-side wait gave up */
#define CBF_ERR_INTERNAL 8      /* a device-side consistency check failed */

/* ODE systems (the reference's calculateDiscreteModel is one per build). */
#define CBF_SYS_MEMRISTIVE5 0   /* the 5-D model of cudaLibrary.cu:2-44, values[0..7] */
#define CBF_SYS_ROSSLER 1       /* values = {s, a, b, c} */
#define CBF_SYS_LORENZ 2        /* values = {s, sigma, rho, beta} */
#define CBF_SYS_CHEN 3          /* values = {s, a, b, c} */
#define CBF_NUM_SYSTEMS 4

/* Tasks of the generic job interface. */
#define CBF_TASK_PEAKS 0        /* 1-D diagram: all peaks per point (+counts) */
#define CBF_TASK_KDE 1          /* KDE mode count per point (int32) */
#define CBF_TASK_DBSCAN 2       /* DBSCAN cluster count per point (int32) */
#define CBF_TASK_LLE 3          /* largest Lyapunov exponent per point (double) */
#define CBF_TASK_TRAJECTORY 4   /* recorded x[writableVar] samples per point (+diverged flags) */
#define CBF_TASK_LLE_REGIME 5   /* LLE (double) + peak-count regime class 0..15 (int32, in d_aux):
                                   0 no oscillation in the window (no peak, range below
                                   regimeMinAmp, or diverged), 15 chaotic (LLE above
                                   regimeChaosLle), more than maxAmountOfPeaks peaks or >= 15
                                   clusters, else the DBSCAN cluster count */

#define CBF_TASK_LS 6           /* Lyapunov spectrum: nIC exponents per point (double[n*nIC],
                                   point-major), LSKernelCUDA semantics */
#define CBF_TASK_OSTROVSKY 7    /* Ostrovsky periodicity value per point (double): the DBSCAN
                                   count rewritten by the threshold flags (cudaLibrary.cu:288-352,
                                   628-662); dbscanEps, maxAmountOfPeaks, ostrovskyThreshold */

/* Job flags. */
#define CBF_FLAG_EXACT_GRID 1u  /* integer grid index instead of the FP32 quirk */
#define CBF_FLAG_KDE_FIXED 2u   /* KDE with kdeSampling samples in total, not per peak */

#define CBF_MAX_DIM 8
#define CBF_MAX_VALUES 16

/* One map computation.  Field meaning follows hostLibrary.cuh:29-459. */
typedef struct cbf_job {
    double ranges[4];               /* {start0, end0, start1, end1} */
    double ic[CBF_MAX_DIM];         /* initial conditions */
    double values[CBF_MAX_VALUES];  /* system parameters */
    double h;                       /* integration step */
    double tMax;                    /* record length (time units) */
    double transientTime;
    double maxValue;                /* divergence bound on |x[writableVar]|, 0 disables */
    double NT;                      /* LLE: renormalisation interval */
    double lleEps;                  /* LLE: initial offset */
    double kdeI1, kdeI2, kdeH;      /* KDE sample interval and bandwidth */
    double dbscanEps;
    int64_t seedChunk;              /* LLE seed index = g mod seedChunk (0: g) */
    int64_t firstPoint;             /* first linear grid index of this job */
    int64_t nPoints;                /* points to compute (0: the whole grid) */
    int32_t task;                   /* CBF_TASK_* */
    int32_t system;                 /* CBF_SYS_* */
    int32_t sweepIC;                /* 0: sweep values[], 1: sweep initial conditions */
    int32_t dims;                   /* swept axes: 1 or 2 */
    int32_t nPts;                   /* points per axis */
    int32_t nIC;
    int32_t nV;
    int32_t idxMut[2];              /* swept entries of values[] (or ic[]) */
    int32_t writableVar;            /* recorded / checked state variable */
    int32_t preScaller;             /* steps per recorded sample */
    int32_t maxAmountOfPeaks;
    int32_t kdeSampling;
    uint32_t flags;                 /* CBF_FLAG_* */
    int32_t peakCapacity;           /* PEAKS/TRAJECTORY: row stride of d_out (0: derived) */
    double regimeTime;              /* LLE_REGIME: time units of the base trajectory, right
                                       after the transient, whose peaks define the class */
    const int64_t* pointIndex;      /* optional DEVICE array: point k of the job is grid
                                       index pointIndex[k] (nPoints entries) instead of
                                       firstPoint + k; outputs stay compact */
    double regimeMinAmp;            /* LLE_REGIME: a window whose peak-to-trough range of
                                       x[writableVar] is below this is class 0 (no
                                       oscillation: an equilibrium whose FP64 state still
                                       wobbles by ulps shows spurious peaks); 0 disables */
    double regimeChaosLle;          /* LLE_REGIME: if > 0, points (with an oscillation)
                                       whose LLE exceeds it are class 15 (chaotic) without
                                       clustering their peaks */
    double ostrovskyThreshold;      /* OSTROVSKY: threshold of the periodicity flags */
} cbf_job;

/* ---- library ---------------------------------------------------------- */
int32_t cbf_abi_version(void);
const char* cbf_status_string(cbf_status status);
const char* cbf_last_error(void);
/* Number of kernel launches issued by this library since load. */
uint64_t cbf_kernel_launches(void);
cbf_status cbf_device_count(int32_t* count);
cbf_status cbf_set_device(int32_t device);
/* Fill a job with the reference's defaults (s = 0.5 convention, preScaller 1). */
void cbf_job_init(cbf_job* job);
/* Derived sizes with the reference's int truncations (hostLibrary.cu:22-23,1286-1288). */
int32_t cbf_record_length(const cbf_job* job);   /* (int)(tMax/h/preScaller) or LLE (int)(tMax/NT) */
int32_t cbf_peak_capacity(const cbf_job* job);   /* peaks a PEAKS row can hold = record/2 */
int64_t cbf_job_points(const cbf_job* job);      /* nPoints, or nPts^dims when 0 */
cbf_status cbf_validate(const cbf_job* job);
/* 2 when the job's Chen or Lorenz steps use the rescaled form with s = 1/2 (y and
 * z stored in units of per-point constants; 6 FMA + 2 MUL per step), 1 for the
 * rescaled form with another s (one more MUL), 0 for the 14-instruction form
 * (other systems, s swept or 0, A = 0, or factors near 0 or beyond 2^64), -1 for
 * an invalid job.  All are the same CD step; each form has its own rounding
 * (forms 2 and 1 round identically), and the CPU oracle follows the one the job
 * uses. */
int32_t cbf_job_scaled_step(const cbf_job* job);

/* ---- device-resident interface --------------------------------------- */
/* Run one job on `stream` (a cudaStream_t, NULL = legacy default stream).
 * d_out: LLE double[n]; KDE/DBSCAN int32[n]; PEAKS double[n*cap];
 *        TRAJECTORY double[n*record]; LS double[n*nIC].
 * d_aux: PEAKS int32[n] peak counts; TRAJECTORY int32[n] diverged flags; else unused.
 * Scratch for KDE/DBSCAN is taken from the stream-ordered allocator. */
cbf_status cbf_run(const cbf_job* job, void* d_out, void* d_aux, void* stream);

/* ---- autotuning ------------------------------------------------------ */
/* The LLE kernel exists in CBF_NUM_LLE_VARIANTS shapes (points per thread 1|2,
 * threads per block, register cap, unrolling of the step loop).  cbf_autotune times all of them on a
 * shortened copy of `job` on the current device and makes the fastest the one
 * cbf_run (and every LLE entry point) uses for job->system on this device.
 * msPerVariant (optional) receives each shape's trial time. */
#define CBF_NUM_LLE_VARIANTS 8
cbf_status cbf_autotune(const cbf_job* job, int32_t* chosenVariant, double* msPerVariant);
/* Set (variant >= 0) or reset to the default (-1) the shape for a system. */
cbf_status cbf_set_lle_variant(int32_t system, int32_t variant);
int32_t cbf_get_lle_variant(int32_t system);

/* ---- ragged batches: many jobs, one persistent launch ----------------- */
/* A batch is any mix of LLE / KDE / DBSCAN / 1-D peak jobs (systems, grid sizes,
 * record lengths, steps) executed by one persistent kernel whose warps pull
 * 32-point tiles from a device work queue, longest jobs first.  Results equal
 * those of the same jobs run one by one.  d_outs[i] / d_auxs[i] are the
 * device buffers cbf_run would take for jobs[i] (d_auxs may be NULL when no job
 * needs one).  No counterpart in the reference (it runs one map per call). */
typedef struct cbf_batch cbf_batch;
cbf_status cbf_batch_create(const cbf_job* jobs, int32_t nJobs, void* const* d_outs,
                            void* const* d_auxs, cbf_batch** batch);
void cbf_batch_destroy(cbf_batch* batch);
int64_t cbf_batch_points(const cbf_batch* batch);
int32_t cbf_batch_blocks_per_sm(const cbf_batch* batch);
/* Enqueue one run on `stream` (reset the queue, launch the persistent kernel). */
cbf_status cbf_batch_run(cbf_batch* batch, void* stream);
/* Capture one run as a CUDA graph (on `stream`, or the library's stream when
 * NULL); cbf_batch_launch replays it for repeated sweeps. */
cbf_status cbf_batch_capture(cbf_batch* batch, void* stream);
cbf_status cbf_batch_launch(cbf_batch* batch, void* stream);
/* The same jobs launched one by one through the per-job kernels. */
cbf_status cbf_batch_run_sequential(cbf_batch* batch, void* stream);
/* After the stream has synchronised: CBF_ERR_INTERNAL if a device guard fired. */
cbf_status cbf_batch_check(cbf_batch* batch);
/* Choose the persistent grid (blocks per SM among 1,2,3,4,6,8,12,16) by timing a
 * copy of the batch with transients and records cut 32x; overwrites outputs and
 * drops a captured graph.  msPerCandidate (optional, 8 entries; -1 = skipped). */
cbf_status cbf_batch_autotune(cbf_batch* batch, void* stream, int32_t* blocksPerSm,
                              double* msPerCandidate);

/* ---- the surrogate network ------------------------------------------- */
/* MLP 4 -> (fixed Fourier encoding, 128) -> 256 -> 256 -> 256 -> 17 (SiLU):
 * output 0 = normalised LLE, outputs 1..16 = logits of the 16-way peak-count
 * regime class.  The 4 inputs are (system code, two swept parameters in [-1, 1],
 * third parameter / 10); the encoding keeps them and adds sin(2 pi s p_k),
 * cos(2 pi s p_k) of p_k = b_k0 x1 + b_k1 x2 for 62 fixed frequencies b_k and the
 * network's frequency scale s (cbf_mlp_set_encoding_scale, default 1).  BF16
 * tensor-core products (tcgen05) with FP32 accumulation for forward and
 * backward, FP32 master weights, Adam.  No counterpart in the reference.
 * Parameters are one flat FP32 vector: W1[256x128] b1 W2[256x256] b2
 * W3[256x256] b3 W4[17x256] b4 (W row-major [out][in]). */
typedef struct cbf_mlp cbf_mlp;
int64_t cbf_mlp_num_params(void);
cbf_status cbf_mlp_create(int32_t batch, uint64_t seed, cbf_mlp** mlp);
void cbf_mlp_destroy(cbf_mlp* mlp);
cbf_status cbf_mlp_get_params(cbf_mlp* mlp, float* host, int64_t n);
cbf_status cbf_mlp_set_params(cbf_mlp* mlp, const float* host, int64_t n);
/* Frequency scale of the input encoding, a power of two in [2^-8, 16] (else
 * CBF_ERR_INVALID_ARG).  The frequencies a network can learn from must stay well
 * below what its labels resolve: the surrogate map sets (coarseSide / 512) rounded
 * to a power of two. */
cbf_status cbf_mlp_set_encoding_scale(cbf_mlp* mlp, float scale);
/* The encoding's 62 frequencies (b_k0, b_k1 for k = 0..61, cycles per unit of the
 * [-1, 1] axes) into out[0..124); n must be 124.  Host-only, needs no GPU. */
cbf_status cbf_mlp_encoding_frequencies(float* out, int32_t n);
/* One forward and backward pass on n <= batch host rows (features x[n*4], LLE
 * targets, classes) with loss = wLle*MSE(out0) + CE(out1..16), both batch means;
 * returns loss, the flat gradient and the raw outputs (each optional). */
cbf_status cbf_mlp_forward_backward(cbf_mlp* mlp, const float* x, const float* yLle,
                                    const int32_t* yCls, int32_t n, float wLle, float* loss,
                                    float* grads, float* out);
/* `steps` Adam steps on minibatches drawn from the device training set (captured
 * as a CUDA graph and replayed); the learning rate decays from lr to lr/20 on a
 * cosine over `horizon` optimiser steps (0: constant); losses (optional, host)
 * receives each step's loss.  cbf_mlp_set_params resets the optimiser state. */
cbf_status cbf_mlp_train(cbf_mlp* mlp, const float* dX, const float* dYLle, const int32_t* dYCls,
                         int64_t n, int32_t steps, float lr, int32_t horizon, float wLle,
                         float* losses, void* stream);
/* Predictions for n device feature rows: LLE = out0*lleStd + lleMean, class
 * (argmax), confidence (softmax maximum); each output optional. */
cbf_status cbf_mlp_predict(cbf_mlp* mlp, const float* dX, int64_t n, float lleMean, float lleStd,
                           float* dLle, int32_t* dCls, float* dConf, void* stream);
/* The same outputs for every grid point 0..points-1 of a 2-D sweep of a 3-D
 * system (the surrogate map's prediction step), features generated on the fly,
 * one fused tcgen05 tensor-core kernel (mlp_tc.cuh). */
cbf_status cbf_mlp_predict_grid(cbf_mlp* mlp, const cbf_job* job, float lleMean, float lleStd,
                                double* dLle, int32_t* dCls, float* dConf, void* stream);
/* The network's input features (4 FP32 per point) of grid points dIdx[0..n). */
cbf_status cbf_mlp_grid_features(const cbf_job* job, const int64_t* dIdx, int64_t n, float* dX, void* stream);

/* ---- surrogate-refined LLE + regime map -------------------------------- */
/* No counterpart in the reference.  The plain method (CBF_TASK_LLE_REGIME)
 * labels a coarse sub-grid (every (nPts/coarseSide)-th row and column) and
 * randomPoints seeded random points; the network above is trained on them,
 * predicts every grid point, and the plain method recomputes every point on a
 * predicted regime boundary, below confThreshold softmax confidence, or in the
 * random audit sample; then, in later rounds, the neighbours of every label or
 * recomputed point whose plain class differs from the prediction.  The rule
 * points are computed in chunks of about two waves of resident LLE_REGIME
 * threads, each round together with every point the previous rounds marked.
 * Labelled and recomputed points carry plain values. */
typedef struct cbf_surrogate_config {
    int32_t coarseSide;      /* training sub-grid side (512) */
    int32_t randomPoints;    /* extra random training points (65536) */
    int32_t batch;           /* training minibatch rows (4096) */
    int32_t trainSteps;      /* Adam steps, cosine learning-rate decay over them (1500) */
    float lr;                /* peak learning rate (2e-3) */
    float wLle;              /* weight of the LLE squared error in the loss (1) */
    float confThreshold;     /* recompute points whose softmax maximum is below it (0.4) */
    float auditFraction;     /* random audit sample of the grid, recomputed (0.01) */
    int32_t boundaryRadius;  /* a neighbour within this Chebyshev radius with another
                                predicted class marks a boundary point (1) */
    int32_t refine;          /* 0: keep every prediction (ablation: network alone) */
    uint64_t seed;           /* training points, minibatches, weights and audit sample */
    int32_t expandRadius;    /* neighbours within this radius of a point whose plain class
                                differs from the prediction are recomputed next; -1 (default):
                                ceil(nPts / 8192); 0: no expansion */
    int32_t maxWaves;        /* rounds that expand: the labels and the points computed in
                                the first maxWaves rounds mark their neighbours (12) */
    int32_t predictor;       /* 0: the trained network (default); 1: no network -- every
                                point takes the class and LLE of its nearest coarse-grid
                                label, confidence 1 (the ablation that measures what the
                                learning adds; same mask, audit and expansion rules) */
    int32_t auditFill;       /* 1: points that only the audit sample selected are not fed
                                with the other rule points; they fill every recompute round
                                up to a whole number of waves of resident LLE_REGIME
                                threads (0) */
    int32_t idleRadius;      /* expansion radius after a round that computed fewer points than
                                half a wave of resident LLE_REGIME threads (only the chain
                                of expansion rounds is left; the idle threads pay for the
                                wider ring); 0 (default): expandRadius */
} cbf_surrogate_config;
void cbf_surrogate_config_init(cbf_surrogate_config* cfg);

typedef struct cbf_surrogate_report {
    int64_t points;            /* grid points */
    int64_t labelled;          /* plain training points (kept in the map) */
    int64_t refined;           /* points recomputed by the plain method */
    int64_t boundary;          /* ... of which on a predicted boundary */
    int64_t lowConfidence;     /* ... of which below the confidence threshold */
    int64_t audit;             /* ... of which in the audit sample */
    int64_t auditOnly;         /* audit points no other rule selected */
    int64_t auditOnlyAgree;    /* ... whose predicted class equals the plain class */
    int64_t refinedChanged;    /* recomputed points whose class the plain method changed */
    double auditOnlyLleMeanAbsErr, auditOnlyLleMaxAbsErr;  /* predicted vs plain LLE */
    double lleMean, lleStd;    /* normalisation of the LLE target */
    float finalLoss;           /* mean training loss over the last 100 steps */
    double msLabel, msTrain, msPredict, msMask, msRefine, msTotal;  /* stream time */
    int64_t expanded;          /* recomputed points selected only by the expansion */
    int32_t waves;             /* recompute rounds that computed at least one point */
    int64_t refineTiles;       /* 32-point warp tiles of the recompute rounds (lane use =
                                  refined / (32 * refineTiles)) */
} cbf_surrogate_report;

/* job: a whole-grid 2-D CBF_TASK_LLE_REGIME sweep of the Rossler, Lorenz or
 * Chen system.  dLle double[nPts^2], dCls int32[nPts^2] (device).  Optional
 * device outputs: dSource uint8[nPts^2] (0 predicted, 1 training label, 2
 * recomputed), dConf float[nPts^2] (the network's softmax confidence), dPred
 * int32[nPts^2] (the network's class before any plain value replaced it). */
cbf_status cbf_lle_map_surrogate(const cbf_job* job, const cbf_surrogate_config* cfg, double* dLle,
                                 int32_t* dCls, uint8_t* dSource, float* dConf, int32_t* dPred,
                                 cbf_surrogate_report* report, void* stream);
/* cbf_lle_map_surrogate keeps its work buffers and the network on the device
 * between calls (about 1 GB at 8192^2; calls on one device run one at a time);
 * this frees them for the current device. */
void cbf_surrogate_release(void);

/* The plain method's regime-class rules (CBF_TASK_LLE_REGIME fields): the class
 * of a point comes from the peaks of x[writableVar] during the first
 * regimeTime time units after the transient. */
typedef struct cbf_regime_rules {
    double regimeTime;         /* window after the transient (50) */
    int32_t maxAmountOfPeaks;  /* more peaks than this -> class 15 (512) */
    double dbscanEps;          /* DBSCAN radius on (peak, interval) (0.02) */
    double regimeMinAmp;       /* window range below this -> class 0 (1e-6) */
    double regimeChaosLle;     /* LLE above this -> class 15 (0.05) */
    uint32_t flags;            /* 0: the grid of LLE2D, getValueByIdx's FP32 index
                                  (cudaLibrary.cu:210-216); CBF_FLAG_EXACT_GRID:
                                  integer grid cells (differ from LLE2D's above 2^24
                                  points, i.e. at 8192^2) (0) */
} cbf_regime_rules;
void cbf_regime_rules_init(cbf_regime_rules* rules);

/* Host-buffer form of the surrogate-refined map: LLE2D's arguments
 * (hostLibrary.cu:1524-1663; seedChunk as for cbf_lle2d), the regime rules
 * (NULL: the defaults above) and the surrogate configuration (NULL: the
 * defaults of cbf_surrogate_config_init).  outLle double[nPts^2] and outCls
 * int32[nPts^2] (optional) are host arrays.  Labelled and recomputed points
 * carry plain FP64 values; the others carry the network's prediction, whose
 * error the report's audit fields estimate.  Runs on the library's stream and
 * returns when the map is in the host arrays; device buffers are cached per
 * device between calls (cbf_surrogate_release frees them).  The C++ facade's
 * LLE2D writes this map when cbfSetSurrogate(1) or CBF_SURROGATE=1 is set. */
cbf_status cbf_lle2d_surrogate(int32_t system, double tMax, double NT, int32_t nPts, double h, double eps,
                               const double* initialConditions, int32_t amountOfInitialConditions,
                               const double* ranges, const int32_t* indicesOfMutVars, int32_t writableVar,
                               double maxValue, double transientTime, const double* values,
                               int32_t amountOfValues, int64_t seedChunk, const cbf_regime_rules* rules,
                               const cbf_surrogate_config* cfg, double* outLle, int32_t* outCls,
                               cbf_surrogate_report* report);

/* ---- host-buffer entry points (drop-in for hostLibrary.cuh) ---------- */
/* bifurcation1D, hostLibrary.cuh:29-42 / hostLibrary.cu:7-158.
 * outPeaks[k*peakCapacity + j], outCounts[k]; peakCapacity >= record/2. */
cbf_status cbf_bifurcation1d(int32_t system, double tMax, int32_t nPts, double h,
                             int32_t amountOfInitialConditions, const double* initialConditions,
                             const double* ranges, const int32_t* indicesOfMutVars,
                             int32_t writableVar, double maxValue, double transientTime,
                             const double* values, int32_t amountOfValues, int32_t preScaller,
                             double* outPeaks, int32_t peakCapacity, int32_t* outCounts);
/* bifurcation1DIC, hostLibrary.cuh:89-102 / hostLibrary.cu:243-393 */
cbf_status cbf_bifurcation1d_ic(int32_t system, double tMax, int32_t nPts, double h,
                                int32_t amountOfInitialConditions, const double* initialConditions,
                                const double* ranges, const int32_t* indicesOfMutVars,
                                int32_t writableVar, double maxValue, double transientTime,
                                const double* values, int32_t amountOfValues, int32_t preScaller,
                                double* outPeaks, int32_t peakCapacity, int32_t* outCounts);
/* bifurcation2DKDE, hostLibrary.cuh:129-147 / hostLibrary.cu:397-567; out int32[nPts*nPts] */
cbf_status cbf_bifurcation2d_kde(int32_t system, double tMax, int32_t nPts, double h,
                                 int32_t amountOfInitialConditions, const double* initialConditions,
                                 const double* ranges, const int32_t* indicesOfMutVars,
                                 int32_t writableVar, double maxValue, int32_t maxAmountOfPeaks,
                                 double transientTime, const double* values,
                                 int32_t amountOfValues, int32_t preScaller, int32_t kdeSampling,
                                 double kdeSamplesInterval1, double kdeSamplesInterval2,
                                 double kdeSamplesSmooth, int32_t* out);
/* bifurcation2DKDEIC, hostLibrary.cuh:254-272 / hostLibrary.cu:929-1090 */
cbf_status cbf_bifurcation2d_kde_ic(int32_t system, double tMax, int32_t nPts, double h,
                                    int32_t amountOfInitialConditions,
                                    const double* initialConditions, const double* ranges,
                                    const int32_t* indicesOfMutVars, int32_t writableVar,
                                    double maxValue, int32_t maxAmountOfPeaks,
                                    double transientTime, const double* values,
                                    int32_t amountOfValues, int32_t preScaller,
                                    int32_t kdeSampling, double kdeSamplesInterval1,
                                    double kdeSamplesInterval2, double kdeSamplesSmooth,
                                    int32_t* out);
/* bifurcation2DDBSCAN, hostLibrary.cuh:171-186 / hostLibrary.cu:571-744 */
cbf_status cbf_bifurcation2d_dbscan(int32_t system, double tMax, int32_t nPts, double h,
                                    int32_t amountOfInitialConditions,
                                    const double* initialConditions, const double* ranges,
                                    const int32_t* indicesOfMutVars, int32_t writableVar,
                                    double maxValue, int32_t maxAmountOfPeaks,
                                    double transientTime, const double* values,
                                    int32_t amountOfValues, int32_t preScaller, double eps,
                                    int32_t* out);
/* bifurcation2DDBSCANIC, hostLibrary.cuh:296-311 / hostLibrary.cu:1094-1266 */
cbf_status cbf_bifurcation2d_dbscan_ic(int32_t system, double tMax, int32_t nPts, double h,
                                       int32_t amountOfInitialConditions,
                                       const double* initialConditions, const double* ranges,
                                       const int32_t* indicesOfMutVars, int32_t writableVar,
                                       double maxValue, int32_t maxAmountOfPeaks,
                                       double transientTime, const double* values,
                                       int32_t amountOfValues, int32_t preScaller, double eps,
                                       int32_t* out);
/* LLE1D / LLE1DIC / LLE2D / LLE2DIC, hostLibrary.cuh:334-459 / hostLibrary.cu:1270-1798.
 * seedChunk reproduces the reference's chunk-local seed index (0: global index);
 * the C++ facade computes it the way the reference does. out double[nPts^dims]. */
cbf_status cbf_lle1d(int32_t system, double tMax, double NT, int32_t nPts, double h, double eps,
                     const double* initialConditions, int32_t amountOfInitialConditions,
                     const double* ranges, const int32_t* indicesOfMutVars, int32_t writableVar,
                     double maxValue, double transientTime, const double* values,
                     int32_t amountOfValues, int64_t seedChunk, double* out);
cbf_status cbf_lle1d_ic(int32_t system, double tMax, double NT, int32_t nPts, double h,
                        double eps, const double* initialConditions,
                        int32_t amountOfInitialConditions, const double* ranges,
                        const int32_t* indicesOfMutVars, int32_t writableVar, double maxValue,
                        double transientTime, const double* values, int32_t amountOfValues,
                        int64_t seedChunk, double* out);
cbf_status cbf_lle2d(int32_t system, double tMax, double NT, int32_t nPts, double h, double eps,
                     const double* initialConditions, int32_t amountOfInitialConditions,
                     const double* ranges, const int32_t* indicesOfMutVars, int32_t writableVar,
                     double maxValue, double transientTime, const double* values,
                     int32_t amountOfValues, int64_t seedChunk, double* out);
cbf_status cbf_lle2d_ic(int32_t system, double tMax, double NT, int32_t nPts, double h,
                        double eps, const double* initialConditions,
                        int32_t amountOfInitialConditions, const double* ranges,
                        const int32_t* indicesOfMutVars, int32_t writableVar, double maxValue,
                        double transientTime, const double* values, int32_t amountOfValues,
                        int64_t seedChunk, double* out);

/* One system sampled with a step offset (modelingOneSystemDenis,
 * hostLibrary.cu:162-239): out[(int)(tMax/h)] (outLen at least that) holds the
 * series x[writableVar] at times h*j, integrated with step hSpecial from T =
 * (int)(hSpecial/h) starting offsets; entries no offset reaches are NaN. */
cbf_status cbf_modeling_one_system(int32_t system, double tMax, double h, double hSpecial,
                                   int32_t amountOfInitialConditions, const double* initialConditions,
                                   int32_t writableVar, const double* values, int32_t amountOfValues,
                                   double* out, int64_t outLen);
/* Periodicity map by Ostrovsky's rule (calculationOfPeriodicityByOstrovsky,
 * hostLibrary.cu:748-925): a 2-D sweep of initial conditions, out double[nPts^2]. */
cbf_status cbf_ostrovsky2d(int32_t system, double tMax, int32_t nPts, double h,
                           int32_t amountOfInitialConditions, const double* initialConditions,
                           const double* ranges, const int32_t* indicesOfMutVars, int32_t writableVar,
                           double maxValue, int32_t maxAmountOfPeaks, double transientTime,
                           const double* values, int32_t amountOfValues, int32_t preScaller,
                           double eps, double ostrovskyThreshold, double* out);
/* Lyapunov spectra (hostLibrary.cu:1802-1924 LS1D, :1928-2082 LS2D): out
 * double[points * amountOfInitialConditions], the exponents of point k at
 * out[k*nIC .. k*nIC+nIC).  seedChunk: the chunk the reference's seed index is
 * local to (its nPtsLimiter; 0 = the global index). */
cbf_status cbf_ls1d(int32_t system, double tMax, double NT, int32_t nPts, double h, double eps,
                    const double* initialConditions, int32_t amountOfInitialConditions,
                    const double* ranges, const int32_t* indicesOfMutVars, int32_t writableVar,
                    double maxValue, double transientTime, const double* values,
                    int32_t amountOfValues, int64_t seedChunk, double* out);
cbf_status cbf_ls2d(int32_t system, double tMax, double NT, int32_t nPts, double h, double eps,
                    const double* initialConditions, int32_t amountOfInitialConditions,
                    const double* ranges, const int32_t* indicesOfMutVars, int32_t writableVar,
                    double maxValue, double transientTime, const double* values,
                    int32_t amountOfValues, int64_t seedChunk, double* out);
/* NumPy .npy file (format 1.0, little-endian float64 or int32, C order) of a
 * rows x cols array.  No counterpart in the reference.  cbf_csv_write_map -- so
 * every 2-D map the facade writes -- also writes <path>.npy when the environment
 * variable CBF_NPY_SIDECAR is set to anything but "0". */
cbf_status cbf_npy_write(const char* path, const void* values, int32_t isDouble, int64_t rows,
                         int64_t cols);
/* CSV rows "param, v1, v2, ...\n" (LS1D layout, hostLibrary.cu:1900-1910) for n
 * points with nCols values each (row-major). */
cbf_status cbf_csv_write_rows(const char* path, int32_t nPts, const double* ranges,
                              const double* values, int64_t n, int32_t nCols, int32_t precision);

/* DBSCAN cluster-count map that allocates no device memory.  No counterpart in
 * the reference.  For callers that cannot call cudaMalloc: programs whose device
 * memory belongs to another allocator (a framework's pool, a fixed budget), and
 * latency-critical loops that cannot afford an allocation's implicit
 * synchronisation or an out-of-memory failure mid-run.  Arguments as
 * cbf_bifurcation2d_dbscan (ic/ranges/indices/values are host arrays); d_out is
 * caller-owned device memory of nPts*nPts int32; runs on `stream` (a
 * cudaStream_t; NULL is the legacy default stream, as for cbf_run).  Every call
 * waits on the host until its stream has finished the map, because it reads the
 * kernel's error flag back.  Scratch: a fixed 64 MiB device array inside the
 * library; maps whose min(maxAmountOfPeaks, record/2) exceeds 32 767 peaks per
 * point are rejected with CBF_ERR_INVALID_ARG.  The first call on a device looks
 * up the array's device address; with lazy module loading (the CUDA default)
 * that first call is also when the device reserves the 64 MiB, so it can fail
 * with CBF_ERR_OUT_OF_MEMORY: make it at start-up, before any stream capture.
 * The device keeps the array until the process exits; the looked-up address is
 * cached per device and does not survive a cudaDeviceReset.  All calls share
 * the array: calls that overlap on the GPU race and must be serialised by the
 * caller. */
cbf_status cbf_bifurcation2d_dbscan_noalloc(int32_t system, double tMax, int32_t nPts, double h,
                                            int32_t amountOfInitialConditions,
                                            const double* initialConditions, const double* ranges,
                                            const int32_t* indicesOfMutVars, int32_t writableVar,
                                            double maxValue, int32_t maxAmountOfPeaks,
                                            double transientTime, const double* values,
                                            int32_t amountOfValues, int32_t preScaller, double eps,
                                            int32_t* d_out, void* stream);

/* Generic host-buffer form of cbf_run: copies results into host memory. */
cbf_status cbf_run_host(const cbf_job* job, void* out, void* aux);

/* ---- CSV output with the reference's byte layout ---------------------- */
/* 2-D map (hostLibrary.cu:534-546): values in index order, ", " between values,
 * "\n" before the first value of each new row of nPts, no final newline.
 * headerRanges (4 doubles) adds the "r0 r1\nr2 r3\n" header (:476-480); NULL
 * omits it.  isDouble selects double (%.*g) or int32 (%d) values.  Formatted by
 * CBF_CSV_THREADS threads (default: the CPUs the process may use), same bytes. */
cbf_status cbf_csv_write_map(const char* path, const void* values, int32_t isDouble, int64_t n,
                             int32_t nPts, const double* headerRanges, int32_t precision);
/* 1-D diagram rows "param, peak\n" at precision 12 (hostLibrary.cu:125-138) for
 * points [firstPoint, firstPoint+nPoints); append != 0 appends to the file. */
cbf_status cbf_csv_write_peaks(const char* path, int32_t nPts, const double* ranges,
                               int64_t firstPoint, int64_t nPoints, const double* peaks,
                               int32_t peakCapacity, const int32_t* counts, int32_t append);
/* 1-D LLE rows "param, value\n" (hostLibrary.cu:1368-1378). */
cbf_status cbf_csv_write_pairs(const char* path, int32_t nPts, const double* ranges,
                               const double* values, int64_t n, int32_t precision);

/* ---- probes used for measurement and self-checks --------------------- */
/* Grid coordinates the kernels use for points [first, first+n): out[k*2+axis]. */
cbf_status cbf_grid_coordinates(const cbf_job* job, double* out_host);
/* The normalised LLE perturbation vectors z (nIC per point) the LLE kernels
 * start from for points [first, first+n) (cudaLibrary.cu:720-732, :843-855);
 * out_host[k*nIC + i].  Lets a checker isolate the FP32 sinf of the seed. */
cbf_status cbf_lle_seeds(const cbf_job* job, double* out_host);
/* FP64 FMA throughput of this GPU (TFLOP/s, 2 flops per FMA) over ~`ms` ms. */
cbf_status cbf_probe_fp64_peak(double ms, double* tflops);
/* The rate at which the map kernels' instruction stream issues FP64 instructions
 * with nothing else around it: `chains` (1, 2 or 4) independent copies per thread
 * of the rescaled 8-instruction Chen step, with the divergence tracking when
 * `tracking` != 0, blocksPerSm blocks of 128 threads per SM, about `ms` ms.
 * *fp64InstrPerSec = FP64 lane instructions per second (divide by SMs x 64 x
 * clock for the pipe fraction).  No counterpart in the reference. */
cbf_status cbf_probe_fp64_step(int32_t chains, int32_t tracking, int32_t blocksPerSm, double ms,
                               double* fp64InstrPerSec);
/* Exhaustive device check that expf(x) == 0 for every float x <= threshold;
 * *count receives the number of floats that violate it. */
cbf_status cbf_probe_expf_zero(float threshold, uint64_t* count);
/* The exact form of the reference's divergence test `fabsf(x) > maxValue`
 * (cudaLibrary.cu:69-71) used by the kernels: fires iff fabs(x) >= *threshold,
 * and only when *active is nonzero. */
cbf_status cbf_divergence_threshold(double maxValue, int32_t* active, double* threshold);

#ifdef __cplusplus
}
#endif
#endif /* CBF_H */
