/*
 * CPU oracle -- TEST INFRASTRUCTURE ONLY (see oracle.h for the contract).
 *
 * Every function below restates one function of the reference library
 * (CUDABifurcation3.0) in plain C, keeping the reference's expression order, its
 * int/float/double conversions and its quirks.  The citation above each function
 * names the reference lines it follows.  Compiled with -ffp-contract=off.
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------------------- */
/* Grid index -> parameter value.  cudaLibrary.cu:210-216.
 * `(int)idx / powf((double)nPts, (double)valueNumber)` is a float division: the
 * int index is converted to float (exact only below 2^24) and powf takes floats. */
double orc_get_value_by_idx(int idx, int nPts, double startRange, double finishRange,
                            int valueNumber)
{
    float p = powf((float)nPts, (float)valueNumber);
    float q = (float)idx / p;
    int cell = ((int)q) % nPts;
    return startRange + (double)cell * ((double)(finishRange - startRange) / (double)(nPts - 1));
}

/* The library's exact-grid option: the cell is the integer quotient, the value
 * formula is getValueByIdx's. */
static double exact_value_by_idx(int64_t idx, int nPts, double startRange, double finishRange,
                                 int valueNumber)
{
    const int64_t d = valueNumber == 0 ? 1 : (int64_t)nPts;
    const int cell = (int)((idx / d) % nPts);
    return startRange + (double)cell * ((double)(finishRange - startRange) / (double)(nPts - 1));
}

/* ------------------------------------------------------------------------- */
/* Model steps.  One fixed-step CD (semi-implicit composition) step: an explicit
 * half with k = h*s in reverse variable order, then a linearly implicit half with
 * h1 = h*(1-s) in forward order (the scheme of cudaLibrary.cu:19-43).            */

/* The model shipped in the reference, cudaLibrary.cu:2-44, restated literally.
 * Quirks kept: `float y[5], k` truncates the explicit-half state snapshot and k to
 * FP32 (:19-34); abs(x[4]) is the double overload (fabs) on the host build. */
static void step_memristive5(double* x, const double* a, double h)
{
    float y[5], k;
    k = (float)(h * a[7]);

    x[4] = x[4] + (double)k * (x[0]);
    x[3] = x[3] + (double)k * (-a[2] * x[1] - a[3] * x[3]);
    x[2] = x[2] + (double)k * (a[1] * (x[1] - x[0] - x[2]));
    x[1] = x[1] + (double)k * (-x[2] + x[3]);
    x[0] = x[0] + (double)k * (a[0] * (x[2] - (a[4] + a[5] + a[6] * fabs(x[4])) * x[0]));

    y[0] = (float)x[0];
    y[1] = (float)x[1];
    y[2] = (float)x[2];
    y[3] = (float)x[3];
    y[4] = (float)x[4];

    double h1 = h * (1 - a[7]);

    x[0] = ((double)y[0] + h1 * (a[0] * x[2])) / (1 + h1 * a[0] * (a[4] + a[5] + a[6] * fabs(x[4])));
    x[1] = (double)y[1] + h1 * (-x[2] + x[3]);
    x[2] = ((double)y[2] + h1 * (a[1] * (x[1] - x[0]))) / (1 + h1 * a[1]);
    x[3] = ((double)y[3] + h1 * (-a[2] * x[1])) / (1 + h1 * a[3]);
    x[4] = (double)y[4] + h1 * (x[0]);
}

/* The library's Rossler, Lorenz and Chen CD steps.  Specification (shared with
 * the CUDA kernels, which must match it operation for operation): with k = h*s,
 * h1 = h*(1-s), the explicit half (reverse variable order) and the linearly
 * implicit half (forward order) multiplied out, parameter-only factors hoisted.
 * Coefficients are recomputed here on every step (same values every time). */

/* Rossler x'=-y-z, y'=x+a*y, z'=b+z*(x-c); values = {s, a, b, c}. */
static void step_rossler(double* X, const double* v, double h)
{
    const double s = v[0], a = v[1], b = v[2], c = v[3];
    const double k = h * s;
    const double h1 = h * (1.0 - s);
    const double c1 = 1.0 - k * c;
    const double kb = k * b;
    const double bq = 1.0 + k * a;
    const double hs = k + h1;
    const double r2 = 1.0 / (1.0 - h1 * a);
    const double g = h1 * r2;
    const double h1b = h1 * b;
    const double c2 = 1.0 + h1 * c;
    const double x = X[0], y = X[1], z = X[2];
    const double z1 = fma(z, fma(k, x, c1), kb);       /* z + k*(b + z*(x-c)) */
    const double y1 = fma(bq, y, k * x);               /* y + k*(x + a*y) */
    const double x2 = fma(-hs, y1 + z1, x);            /* x - k*(y1+z1) - h1*(y1+z1) */
    const double y2 = fma(g, x2, r2 * y1);             /* (y1 + h1*x2)/(1 - h1*a) */
    const double z2 = (z1 + h1b) / fma(-h1, x2, c2);   /* (z1 + h1*b)/(1 - h1*(x2-c)) */
    X[0] = x2; X[1] = y2; X[2] = z2;
}

/* Chen x'=a*(y-x), y'=(c-a)*x-x*z+c*y, z'=x*y-b*z; values = {s, a, b, c}. */
static void step_chen(double* X, const double* v, double h)
{
    const double s = v[0], a = v[1], b = v[2], c = v[3];
    const double k = h * s;
    const double h1 = h * (1.0 - s);
    const double ka = k * a;
    const double h1a = h1 * a;
    const double ca = 1.0 - k * b;
    const double cb = 1.0 + k * c;
    const double cma = c - a;
    const double r1 = 1.0 / (1.0 + h1a);
    const double d = (1.0 - ka) * r1;
    const double e = (ka + h1a) * r1;
    const double r2 = 1.0 / (1.0 - h1 * c);
    const double g = h1 * r2;
    const double r3 = 1.0 / (1.0 + h1 * b);
    const double hh = h1 * r3;
    const double x = X[0], y = X[1], z = X[2];
    const double kx = k * x;
    const double z1 = fma(kx, y, ca * z);        /* z + k*(x*y - b*z) */
    const double w = cma - z1;
    const double y1 = fma(kx, w, cb * y);        /* y + k*((c-a)*x - x*z1 + c*y) */
    const double x2 = fma(d, x, e * y1);         /* explicit + implicit x half-steps */
    const double y2 = fma(g * x2, w, r2 * y1);   /* (y1 + h1*x2*((c-a)-z1))/(1 - h1*c) */
    const double z2 = fma(hh * x2, y2, r3 * z1); /* (z1 + h1*x2*y2)/(1 + h1*b) */
    X[0] = x2; X[1] = y2; X[2] = z2;
}

/* Lorenz x'=sigma*(y-x), y'=x*(rho-z)-y, z'=x*y-beta*z; values = {s, sigma, rho, beta}. */
static void step_lorenz(double* X, const double* v, double h)
{
    const double s = v[0], sg = v[1], rho = v[2], beta = v[3];
    const double k = h * s;
    const double h1 = h * (1.0 - s);
    const double ks = k * sg;
    const double h1s = h1 * sg;
    const double ca = 1.0 - k * beta;
    const double cb = 1.0 - k;
    const double r1 = 1.0 / (1.0 + h1s);
    const double d = (1.0 - ks) * r1;
    const double e = (ks + h1s) * r1;
    const double r2 = 1.0 / (1.0 + h1);
    const double g = h1 * r2;
    const double r3 = 1.0 / (1.0 + h1 * beta);
    const double hh = h1 * r3;
    const double x = X[0], y = X[1], z = X[2];
    const double kx = k * x;
    const double z1 = fma(kx, y, ca * z);
    const double w = rho - z1;
    const double y1 = fma(kx, w, cb * y);
    const double x2 = fma(d, x, e * y1);
    const double y2 = fma(g * x2, w, r2 * y1);
    const double z2 = fma(hh * x2, y2, r3 * z1);
    X[0] = x2; X[1] = y2; X[2] = z2;
}

/* The library's rescaled Chen / Lorenz step (systems.cuh, QuadScaled: 8 FP64
 * operations when s = 1/2, where c5 = 1, else 9), for the jobs orc_scaled_step
 * admits.  The state is stored as (x, Y, Z) = (x, sy y, sz z).  With A = a or
 * sigma, B = b or beta, om = 1 - k B, ups = r1 A h, sy = ups cy, sz = om sy / k,
 * the CD step becomes
 *   Z1 = fma(x, Y, Z);  W = fma(al, Z1, be);  Y1 = fma(x, W, Y);  x2 = fma(rho, x, Y1);
 *   q = c5 x2;  Y2 = ly fma(q, W, Y1);  Z2 = lz fma(q, Y2, Z1)
 * (coefficients below, in the kernels' operation order; the kernels skip the
 * product c5 x2 when c5 = 1, which changes nothing). */
typedef struct {
    double al, be, rho, c5, ly, lz, sy, iy, sz, iz;
} scaled_coef;

static void scaled_coef_of(int lorenz, const double* v, double h, scaled_coef* q)
{
    const double s = v[0];
    const double k = h * s;
    const double h1 = h * (1.0 - s);
    const double A = v[1];
    const double B = lorenz ? v[3] : v[2];
    const double W0 = lorenz ? v[2] : v[3] - v[1];
    const double cy = lorenz ? 1.0 - k : 1.0 + k * v[3];
    const double r2 = lorenz ? 1.0 / (1.0 + h1) : 1.0 / (1.0 - h1 * v[3]);
    const double r1 = 1.0 / (1.0 + h1 * A);
    const double r3 = 1.0 / (1.0 + h1 * B);
    const double ups = (r1 * A) * h;
    const double om = 1.0 - k * B;
    q->sy = ups * cy;
    q->sz = (om * q->sy) / k;
    const double uk = ups * k;
    q->al = -(uk * (k / q->sy));
    q->be = uk * W0;
    q->rho = r1 * (1.0 - k * A);
    q->c5 = h1 / k;
    q->ly = cy * r2;
    q->lz = om * r3;
    q->iy = 1.0 / q->sy;
    q->iz = 1.0 / q->sz;
}

static void step_quad_scaled(int lorenz, double* X, const double* v, double h)
{
    scaled_coef q;
    scaled_coef_of(lorenz, v, h, &q);
    const double x = X[0], y = X[1], z = X[2];
    const double z1 = fma(x, y, z);
    const double w = fma(q.al, z1, q.be);
    const double y1 = fma(x, w, y);
    const double x2 = fma(q.rho, x, y1);
    const double qq = q.c5 * x2;
    const double y2 = q.ly * fma(qq, w, y1);
    const double z2 = q.lz * fma(qq, y2, z1);
    X[0] = x2; X[1] = y2; X[2] = z2;
}

/* Internal ids of the rescaled forms (never in a job; setup_point returns them). */
enum { ORC_SCALED = 0x100 };

static int is_scaled(int system) { return (system & ORC_SCALED) != 0; }

int orc_system_dim(int system)
{
    switch (system & ~ORC_SCALED) {
    case ORC_SYS_MEMRISTIVE5: return 5;
    case ORC_SYS_ROSSLER:
    case ORC_SYS_LORENZ:
    case ORC_SYS_CHEN: return 3;
    default: return -1;
    }
}

void orc_model_step(int system, double* x, const double* a, double h)
{
    switch (system) {
    case ORC_SYS_MEMRISTIVE5: step_memristive5(x, a, h); break;
    case ORC_SYS_ROSSLER: step_rossler(x, a, h); break;
    case ORC_SYS_LORENZ: step_lorenz(x, a, h); break;
    case ORC_SYS_CHEN: step_chen(x, a, h); break;
    case ORC_SYS_LORENZ | ORC_SCALED: step_quad_scaled(1, x, a, h); break;
    case ORC_SYS_CHEN | ORC_SCALED: step_quad_scaled(0, x, a, h); break;
    default: break;
    }
}

/* Units of a stored state: component i is stored as (physical * s[i]) and read
 * back as (stored * is[i]); every factor is 1 except y (sy, 1/sy) and z (sz,
 * 1/sz) of a rescaled system.  A multiplication by 1 is exact, so the unscaled
 * systems see their values unchanged. */
typedef struct {
    double s[8], is[8];
} state_units;

static state_units units_of(int system, const double* v, double h)
{
    state_units u;
    for (int i = 0; i < 8; ++i)
        u.s[i] = u.is[i] = 1.0;
    if (is_scaled(system)) {
        scaled_coef q;
        scaled_coef_of((system & ~ORC_SCALED) == ORC_SYS_LORENZ, v, h, &q);
        u.s[1] = q.sy;
        u.is[1] = q.iy;
        u.s[2] = q.sz;
        u.is[2] = q.iz;
    }
    return u;
}

/* Stored component i -> physical. */
static double to_phys(double value, int i, const state_units* u)
{
    return value * u->is[i];
}

/* A physical quantity (initial value or perturbation) of component i -> stored. */
static double to_stored(double value, int i, const state_units* u)
{
    return value * u->s[i];
}

/* Whether a Chen / Lorenz job runs the rescaled step (the library's
 * scaled_step_ok, capi.cu): s not swept; k = h s at least 2^-64 in magnitude;
 * every value of a, b, c (sigma, rho, beta) the job's grid holds finite and
 * within 2^64; A = values[1] and the factors 1 + h1 A, 1 - k B, 1 + h1 B, Chen
 * 1 + k c, 1 - h1 c, Lorenz 1 - k, 1 + h1 at least 2^-64 in magnitude.  Returns
 * 2 when k = h1 (s = 1/2: the library's 8-instruction form), 1 for the other
 * rescaled jobs, 0 otherwise (cbf_job_scaled_step). */
static int fin64(double v) { return isfinite(v) && fabs(v) <= 0x1p64; }
static int away64(double v) { return isfinite(v) && fabs(v) >= 0x1p-64; }

int orc_scaled_step(const orc_job* job)
{
    const int chen = job->system == ORC_SYS_CHEN, lorenz = job->system == ORC_SYS_LORENZ;
    if (!chen && !lorenz)
        return 0;
    int sweptAxis[16];
    for (int i = 0; i < 16; ++i)
        sweptAxis[i] = -1;
    if (!job->sweepIC)
        for (int a = 0; a < job->dims && a < 2; ++a)
            if (job->idxMut[a] >= 0 && job->idxMut[a] < 16)
                sweptAxis[job->idxMut[a]] = a;
    if (sweptAxis[0] >= 0)
        return 0;
    const double h = job->h, s = job->values[0];
    if (!(fin64(h) && away64(h) && fin64(s)))
        return 0;
    const double k = h * s, h1 = h * (1.0 - s);
    if (!away64(k))
        return 0;
    if (lorenz && !(away64(1.0 - k) && away64(1.0 + h1)))
        return 0;
    for (int slot = 1; slot <= 3; ++slot) {
        const int ax = sweptAxis[slot];
        const int count = ax < 0 ? 1 : job->nPts;
        for (int cell = 0; cell < count; ++cell) {
            const double v = ax < 0 ? job->values[slot]
                                    : job->ranges[2 * ax] + (double)cell * ((double)(job->ranges[2 * ax + 1] -
                                                                                      job->ranges[2 * ax]) /
                                                                            (double)(job->nPts - 1));
            if (!fin64(v))
                return 0;
            int ok = 1;
            if (slot == 1)
                ok = away64(v) && away64(1.0 + h1 * v);
            else if (chen && slot == 2)
                ok = away64(1.0 - k * v) && away64(1.0 + h1 * v);
            else if (chen && slot == 3)
                ok = away64(1.0 + k * v) && away64(1.0 - h1 * v);
            else if (lorenz && slot == 3)
                ok = away64(1.0 - k * v) && away64(1.0 + h1 * v);
            if (!ok)
                return 0;
        }
    }
    return k == h1 ? 2 : 1;
}

/* `if (maxValue != 0) if (fabsf(x[writableVar]) > maxValue)`: fabsf rounds the
 * double to FP32, the comparison promotes back to double.  cudaLibrary.cu:69-71 */
int orc_diverged(double v, double maxValue)
{
    return (maxValue != 0) && ((double)fabsf((float)v) > maxValue);
}

/* cudaLibrary.cu:55-74: store x[writableVar] BEFORE stepping, then preScaller
 * steps, then the divergence check; returns false on the first violation. */
int orc_loop(int system, double* x, const double* values, double h, int amountOfIterations,
             int preScaller, int writableVar, double maxValue, double* data,
             int64_t startDataIndex, int writeStep)
{
    /* x[writableVar] in physical units (a rescaled system stores y and z scaled) */
    const state_units u = units_of(system, values, h);
    for (int i = 0; i < amountOfIterations; ++i) {
        if (data != NULL)
            data[startDataIndex + (int64_t)i * writeStep] = to_phys(x[writableVar], writableVar, &u);
        for (int j = 0; j < preScaller - 1; ++j)
            orc_model_step(system, x, values, h);
        orc_model_step(system, x, values, h);
        if (maxValue != 0)
            if ((double)fabsf((float)to_phys(x[writableVar], writableVar, &u)) > maxValue)
                return 0;
    }
    return 1;
}

/* cudaLibrary.cu:220-266.  Quirks kept: a rising plateau sets i=j+1 and the loop's
 * ++i skips sample j+1; after the scan the FIRST peak is dropped and intervals are
 * (t[k+1]-t[k])*h.  Output may alias data (writes never pass the read cursor). */
int orc_peak_finder(double* data, int64_t startDataIndex, int amountOfPoints,
                    double* outPeaks, double* timeOfPeaks, double h)
{
    int amountOfPeaks = 0;
    const int64_t s = startDataIndex;
    for (int64_t i = s + 1; i < s + amountOfPoints - 1; ++i) {
        if (data[i] > data[i - 1] && data[i] >= data[i + 1]) {
            for (int64_t j = i; j < s + amountOfPoints - 1; ++j) {
                if (data[j] < data[j + 1]) {
                    i = j + 1;
                    break;
                }
                if (data[j] > data[j + 1]) {
                    if (outPeaks != NULL)
                        outPeaks[s + amountOfPeaks] = data[j];
                    if (timeOfPeaks != NULL)
                        timeOfPeaks[s + amountOfPeaks] = (double)j;
                    ++amountOfPeaks;
                    i = j + 1;
                    break;
                }
            }
        }
    }
    if (amountOfPeaks > 1) {
        for (int64_t i = 0; i < amountOfPeaks - 1; i++) {
            if (outPeaks != NULL)
                outPeaks[s + i] = outPeaks[s + i + 1];
            if (timeOfPeaks != NULL)
                timeOfPeaks[s + i] = (double)((timeOfPeaks[s + i + 1] - timeOfPeaks[s + i]) * h);
        }
        amountOfPeaks = amountOfPeaks - 1;
    } else {
        amountOfPeaks = 0;
    }
    return amountOfPeaks;
}

/* cudaLibrary.cu:356-422.  Gaussian KDE evaluated at k1-1 sample positions with
 * FP32 expf and a double accumulator in peak order; strict local maxima counted
 * with the `strangePeak` plateau state machine plus a rising tail. */
int orc_kde(const double* data, int64_t startDataIndex, int amountOfPoints, int maxAmountOfPeaks,
            int kdeSampling, double kdeSamplesInterval1, double kdeSamplesInterval2,
            double kdeSmoothH)
{
    if (amountOfPoints == 0)
        return 0;
    if (amountOfPoints == 1 || amountOfPoints == 2)
        return 1;
    if (amountOfPoints > maxAmountOfPeaks)
        return maxAmountOfPeaks;
    return orc_kde_k1(data, startDataIndex, amountOfPoints, kdeSampling * amountOfPoints,
                      kdeSamplesInterval1, kdeSamplesInterval2, kdeSmoothH);
}

/* The sampling and mode-counting body of kde() (cudaLibrary.cu:367-421) with the
 * sample count k1 given directly; kde() uses k1 = kdeSampling * amountOfPoints.
 * A fixed k1 is the library's fixed-sample extension of the same estimator. */
int orc_kde_k1(const double* data, int64_t startDataIndex, int amountOfPoints, int k1i,
               double kdeSamplesInterval1, double kdeSamplesInterval2, double kdeSmoothH)
{
    double k1 = k1i;
    double k2 = (kdeSamplesInterval2 - kdeSamplesInterval1) / (k1 - 1);
    double delt = 0;
    double prevPrevData2 = 0;
    double prevData2 = 0;
    double data2 = 0;
    int strangePeak = 0;
    int resultKde = 0;

    for (int w = 0; w < k1 - 1; ++w) {
        delt = w * k2 + kdeSamplesInterval1;
        prevPrevData2 = prevData2;
        prevData2 = data2;
        data2 = 0;
        for (int m = 0; m < amountOfPoints; ++m) {
            double tempData = (data[startDataIndex + m] - delt) / kdeSmoothH;
            data2 += (double)expf((float)(-((tempData * tempData) / 2)));
        }

        if (w < 2)
            continue;
        if (strangePeak) {
            if (prevData2 == data2)
                continue;
            else if (prevData2 < data2) {
                strangePeak = 0;
                continue;
            } else if (prevData2 > data2) {
                strangePeak = 0;
                ++resultKde;
                continue;
            }
        } else if (prevData2 > prevPrevData2 && prevData2 > data2) {
            ++resultKde;
            continue;
        } else if (prevData2 > prevPrevData2 && prevData2 == data2) {
            strangePeak = 1;
            continue;
        }
    }
    if (prevData2 < data2)
        ++resultKde;
    return resultKde;
}

/* cudaLibrary.cu:445-453: exact-equality shortcut, then FP32 hypotf of the
 * double differences. */
double orc_distance(double x1, double y1, double x2, double y2)
{
    if (x1 == x2 && y1 == y2)
        return 0;
    double dx = x2 - x1;
    double dy = y2 - y1;
    return (double)hypotf((float)dx, (float)dy);
}

/* cudaLibrary.cu:457-529, restated literally: labels at [start, start+n), the
 * "stack" at start+n+k, popped from start+n+NumNeibor-1 into the loop variable;
 * k only ranges over 0..n-2 (the last peak is never a neighbour); returns
 * cluster-1. */
int orc_dbscan(const double* data, const double* intervals, double* helpfulArray,
               int64_t startDataIndex, int amountOfPeaks, int sizeOfHelpfulArray,
               int maxAmountOfPeaks, double eps)
{
    if (amountOfPeaks <= 0)
        return 0;
    if (amountOfPeaks == 1)
        return 1;
    if (amountOfPeaks > maxAmountOfPeaks)
        return 0;

    const int64_t s = startDataIndex;
    int cluster = 0;
    int NumNeibor = 0;

    for (int64_t i = s; i < s + sizeOfHelpfulArray; ++i)
        helpfulArray[i] = 0;

    for (int i = 0; i < amountOfPeaks; i++) {
        if (NumNeibor >= 1) {
            i = (int)helpfulArray[s + amountOfPeaks + NumNeibor - 1];
            helpfulArray[s + amountOfPeaks + NumNeibor - 1] = 0;
            NumNeibor = NumNeibor - 1;
            for (int k = 0; k < amountOfPeaks - 1; k++) {
                if (i != k && helpfulArray[s + k] == 0) {
                    if (orc_distance(data[s + i], intervals[s + i], data[s + k], intervals[s + k]) < eps) {
                        helpfulArray[s + k] = cluster;
                        helpfulArray[s + amountOfPeaks + k] = k;
                        ++NumNeibor;
                    }
                }
            }
        } else if (helpfulArray[s + i] == 0) {
            NumNeibor = 0;
            ++cluster;
            helpfulArray[s + i] = cluster;
            for (int k = 0; k < amountOfPeaks - 1; k++) {
                if (i != k && helpfulArray[s + k] == 0) {
                    if (orc_distance(data[s + i], intervals[s + i], data[s + k], intervals[s + k]) < eps) {
                        helpfulArray[s + k] = cluster;
                        helpfulArray[s + amountOfPeaks + k] = k;
                        ++NumNeibor;
                    }
                }
            }
        }
    }
    return cluster - 1;
}

/* ------------------------------------------------------------------------- */
/* Per-point drivers                                                          */

int orc_record_len(const orc_job* job)
{
    return (int)(job->tMax / job->h / (double)job->preScaller);
}

int orc_skip_len(const orc_job* job)
{
    return (int)(job->transientTime / job->h);
}

/* Per-thread set-up of calculateDiscreteModelCUDA (cudaLibrary.cu:96-105) and of
 * its IC variant (:183-192): copy ICs and values, then overwrite the swept
 * entries with getValueByIdx of the global point index. */
static void setup_point(const orc_job* job, int64_t g, double* x, double* v)
{
    for (int i = 0; i < job->nIC; ++i)
        x[i] = job->ic[i];
    for (int i = 0; i < job->nV; ++i)
        v[i] = job->values[i];
    for (int i = 0; i < job->dims; ++i) {
        double p = job->exactGrid
                       ? exact_value_by_idx(g, job->nPts, job->ranges[i * 2], job->ranges[i * 2 + 1], i)
                       : orc_get_value_by_idx((int)g, job->nPts, job->ranges[i * 2],
                                              job->ranges[i * 2 + 1], i);
        if (job->sweepIC)
            x[job->idxMut[i]] = p;
        else
            v[job->idxMut[i]] = p;
    }
}

/* setup_point, then the state converted to the units the job's step uses; returns
 * the system id the loops integrate (a rescaled form where the job admits it) and
 * sets *u to its units. */
static int setup_state(const orc_job* job, int64_t g, double* x, double* v, state_units* u)
{
    setup_point(job, g, x, v);
    const int sys = orc_scaled_step(job) ? (job->system | ORC_SCALED) : job->system;
    *u = units_of(sys, v, job->h);
    if (is_scaled(sys)) {
        x[1] = x[1] * u->s[1];
        x[2] = x[2] * u->s[2];
    }
    return sys;
}

/* The regime window of the LLE + regime point: x[recVar] (physical) recorded
 * before every step, the LLE's divergence test on x[0] after it (the LLE kernels
 * test x[0] whatever writableVar is, cudaLibrary.cu:735-753); returns 0 at the
 * first violation, like orc_loop. */
static int loop_window(int system, double* x, const double* values, double h, int n, int recVar,
                       double maxValue, double* data)
{
    const state_units u = units_of(system, values, h);
    for (int i = 0; i < n; ++i) {
        data[i] = to_phys(x[recVar], recVar, &u);
        orc_model_step(system, x, values, h);
        if (maxValue != 0 && (double)fabsf((float)x[0]) > maxValue)
            return 0;
    }
    return 1;
}

/* cudaLibrary.cu:107-114 (and :194-201): unchecked transient, then the recorded
 * loop with the divergence check on x[writableVar]. */
int orc_trajectory_point(const orc_job* job, int64_t g, double* data)
{
    double x[8], v[16];
    state_units u;
    const int sys = setup_state(job, g, x, v, &u);
    orc_loop(sys, x, v, job->h, orc_skip_len(job), 1, 0, 0, NULL, 0, 1);
    int ok = orc_loop(sys, x, v, job->h, orc_record_len(job), job->preScaller,
                      job->writableVar, job->maxValue, data, 0, 1);
    return !ok;
}

/* LLEKernelCUDA, cudaLibrary.cu:666-785; IC variant LLEKernelICCUDA :789-908.
 * Quirks kept: the seed uses the chunk-local thread index with int32 wrap (:723)
 * or the IC formula (:846); every loop checks x[0] (writableVar hard-coded to 0)
 * against maxValue and stops THAT integration early, but the LLE sum goes on and
 * the final write overwrites the zero written on divergence (:750-754, :777). */
void orc_lle_seed(const orc_job* job, int64_t g, double* z)
{
    const int nIC = job->nIC;
    const int idx = (int)(job->seedChunk > 0 ? (g % job->seedChunk) : g);
    double zPower = 0;
    for (int i = 0; i < nIC; ++i) {
        if (!job->sweepIC) {
            uint32_t u = (uint32_t)idx * ((uint32_t)i * (uint32_t)idx + 1u) + 1u;
            int32_t arg = (int32_t)u;
            z[i] = 0.5 * (double)sinf((float)arg);
        } else {
            double arg = 0.2171828 * (i + 1) + idx + (0.2171828 + i * idx);
            z[i] = (double)sinf((float)arg) * 0.5;
        }
        zPower += z[i] * z[i];
    }
    zPower = sqrt(zPower);
    for (int i = 0; i < nIC; i++)
        z[i] /= zPower;
}

double orc_lle_point(const orc_job* job, int64_t g)
{
    return orc_lle_point_seeded(job, g, NULL);
}

/* zIn: the normalised perturbation to start from (NULL: orc_lle_seed). */
double orc_lle_point_seeded(const orc_job* job, int64_t g, const double* zIn)
{
    double x[8], y[8], z[8], v[16];
    state_units u;
    const int sys = setup_state(job, g, x, v, &u);

    const int nIC = job->nIC;
    if (zIn) {
        for (int i = 0; i < nIC; ++i)
            z[i] = zIn[i];
    } else {
        orc_lle_seed(job, g, z);
    }

    const double h = job->h;
    const int skip = orc_skip_len(job);
    const int nNT = (int)(size_t)(job->NT / h);
    const int sizeOfBlock = (int)(job->tMax / job->NT);
    const double eps = job->lleEps;

    orc_loop(sys, x, v, h, skip, 1, 0, job->maxValue, NULL, 0, 1);

    /* the perturbation in physical units; distances measured in physical units */
    for (int i = 0; i < nIC; ++i)
        y[i] = to_stored(z[i] * eps, i, &u) + x[i];

    double result = 0;
    for (int i = 0; i < sizeOfBlock; ++i) {
        orc_loop(sys, x, v, h, nNT, 1, 0, job->maxValue, NULL, 0, 1);
        orc_loop(sys, y, v, h, nNT, 1, 0, job->maxValue, NULL, 0, 1);

        double tempData = 0;
        for (int l = 0; l < nIC; ++l) {
            const double d = to_phys(x[l] - y[l], l, &u);
            tempData += d * d;
        }
        tempData = sqrt(tempData) / eps;

        result += log(tempData);

        if (tempData != 0)
            tempData = (1 / tempData);

        for (int j = 0; j < nIC; ++j)
            y[j] = (double)(x[j] - ((x[j] - y[j]) * tempData));
    }
    return result / job->tMax;
}

double orc_lle_regime_point(const orc_job* job, int64_t g, const double* zIn, int32_t* cls)
{
    double x[8], y[8], z[8], v[16];
    state_units u;
    const int sys = setup_state(job, g, x, v, &u);
    const int nIC = job->nIC;
    if (zIn) {
        for (int i = 0; i < nIC; ++i)
            z[i] = zIn[i];
    } else {
        orc_lle_seed(job, g, z);
    }
    const double h = job->h;
    const int nNT = (int)(size_t)(job->NT / h);
    const int sizeOfBlock = (int)(job->tMax / job->NT);
    const double eps = job->lleEps;
    const int win = (int)(job->regimeTime / h);
    int64_t total = (int64_t)nNT * (sizeOfBlock > 0 ? sizeOfBlock : 0);
    const int recorded = (int)(win < total ? win : total);
    double* data = (double*)malloc(sizeof(double) * (size_t)(recorded > 0 ? recorded : 1));
    int regimeDiv = 0;

    orc_loop(sys, x, v, h, orc_skip_len(job), 1, 0, job->maxValue, NULL, 0, 1);
    for (int i = 0; i < nIC; ++i)
        y[i] = to_stored(z[i] * eps, i, &u) + x[i];

    double result = 0;
    int t = 0;
    for (int b = 0; b < sizeOfBlock; ++b) {
        /* the base trajectory's interval, recording while inside the window; the
         * divergence test stops the interval (cudaLibrary.cu:69-71) */
        int inWin = recorded - t;
        if (inWin > nNT) inWin = nNT;
        if (inWin < 0) inWin = 0;
        int ok = 1;
        if (inWin > 0) {
            ok = loop_window(sys, x, v, h, inWin, job->writableVar, job->maxValue, data + t);
            if (!ok) regimeDiv = 1;
        }
        if (ok && nNT - inWin > 0)
            orc_loop(sys, x, v, h, nNT - inWin, 1, 0, job->maxValue, NULL, 0, 1);
        orc_loop(sys, y, v, h, nNT, 1, 0, job->maxValue, NULL, 0, 1);
        t += nNT;

        double tempData = 0;
        for (int l = 0; l < nIC; ++l) {
            const double d = to_phys(x[l] - y[l], l, &u);
            tempData += d * d;
        }
        tempData = sqrt(tempData) / eps;
        result += log(tempData);
        if (tempData != 0)
            tempData = (1 / tempData);
        for (int j = 0; j < nIC; ++j)
            y[j] = (double)(x[j] - ((x[j] - y[j]) * tempData));
    }

    int c = 0;
    double lo = INFINITY, hi = -INFINITY;
    for (int i = 0; i < recorded && !regimeDiv; ++i) {
        lo = fmin(lo, data[i]);
        hi = fmax(hi, data[i]);
    }
    if (!regimeDiv && recorded > 0 && !(hi - lo < job->regimeMinAmp)) {
        double* times = (double*)malloc(sizeof(double) * (size_t)recorded);
        int n = orc_peak_finder(data, 0, recorded, data, times, 0.01);
        if (n > 0 && job->regimeChaosLle > 0 && result / job->tMax > job->regimeChaosLle) {
            c = 15;
        } else if (n > job->maxAmountOfPeaks) {
            c = 15;
        } else if (n > 0) {
            double* helpful = (double*)malloc(sizeof(double) * (size_t)(2 * n + 2));
            c = orc_dbscan(data, times, helpful, 0, n, 2 * n + 2, job->maxAmountOfPeaks,
                           job->dbscanEps);
            free(helpful);
            if (c > 15) c = 15;
        }
        free(times);
    }
    free(data);
    *cls = c;
    return result / job->tMax;
}

/* ------------------------------------------------------------------------- */
/* Map drivers                                                                */

static int threads_or_default(int n)
{
#ifdef _OPENMP
    return n > 0 ? n : omp_get_max_threads();
#else
    (void)n;
    return 1;
#endif
}

int orc_map_peaks(const orc_job* job, int64_t first, int64_t count, double* outPeaks,
                  double* outIntervals, int32_t* counts, int64_t cap, int nThreads)
{
    const int rec = orc_record_len(job);
    if (rec <= 0)
        return -1;
    int err = 0;
#pragma omp parallel num_threads(threads_or_default(nThreads))
    {
        double* data = (double*)malloc(sizeof(double) * (size_t)rec);
        double* peaks = (double*)malloc(sizeof(double) * (size_t)rec);
        double* times = (double*)malloc(sizeof(double) * (size_t)rec);
        if (!data || !peaks || !times) {
#pragma omp atomic write
            err = -2;
        } else {
#pragma omp for schedule(dynamic, 1)
            for (int64_t k = 0; k < count; ++k) {
                int diverged = orc_trajectory_point(job, first + k, data);
                int n = 0;
                if (!diverged)
                    n = orc_peak_finder(data, 0, rec, peaks, times, 0.01);
                counts[k] = n;
                int64_t m = n < cap ? n : cap;
                for (int64_t j = 0; j < m; ++j) {
                    if (outPeaks)
                        outPeaks[k * cap + j] = peaks[j];
                    if (outIntervals)
                        outIntervals[k * cap + j] = times[j];
                }
            }
        }
        free(data);
        free(peaks);
        free(times);
    }
    return err;
}

int orc_map_kde(const orc_job* job, int64_t first, int64_t count, int32_t* out, int nThreads)
{
    const int rec = orc_record_len(job);
    if (rec <= 0)
        return -1;
    int err = 0;
#pragma omp parallel num_threads(threads_or_default(nThreads))
    {
        double* data = (double*)malloc(sizeof(double) * (size_t)rec);
        if (!data) {
#pragma omp atomic write
            err = -2;
        } else {
#pragma omp for schedule(dynamic, 1)
            for (int64_t k = 0; k < count; ++k) {
                int diverged = orc_trajectory_point(job, first + k, data);
                int n = 0;
                if (!diverged)
                    n = orc_peak_finder(data, 0, rec, data, NULL, 0.01); /* in place, :514-515 */
                out[k] = orc_kde(data, 0, n, job->maxAmountOfPeaks, job->kdeSampling,
                                 job->kdeI1, job->kdeI2, job->kdeH);
            }
        }
        free(data);
    }
    return err;
}

int orc_map_dbscan(const orc_job* job, int64_t first, int64_t count, int32_t* out, int nThreads)
{
    const int rec = orc_record_len(job);
    if (rec <= 0)
        return -1;
    int err = 0;
#pragma omp parallel num_threads(threads_or_default(nThreads))
    {
        double* data = (double*)malloc(sizeof(double) * (size_t)rec);
        double* intervals = (double*)malloc(sizeof(double) * (size_t)rec);
        double* helpful = (double*)malloc(sizeof(double) * (size_t)rec);
        if (!data || !intervals || !helpful) {
#pragma omp atomic write
            err = -2;
        } else {
#pragma omp for schedule(dynamic, 1)
            for (int64_t k = 0; k < count; ++k) {
                int diverged = orc_trajectory_point(job, first + k, data);
                int n = 0;
                if (!diverged)
                    n = orc_peak_finder(data, 0, rec, data, intervals, 0.01); /* :689-690 */
                out[k] = orc_dbscan(data, intervals, helpful, 0, n, rec, job->maxAmountOfPeaks,
                                    job->dbscanEps);
            }
        }
        free(data);
        free(intervals);
        free(helpful);
    }
    return err;
}

/* calculationOfPeriodicityByOstrovsky (hostLibrary.cu:748-925) per point:
 * peakFinderCUDAForCalculationOfPeriodicityByOstrovsky (cudaLibrary.cu:288-352)
 * then dbscanCUDAForCalculationOfPeriodicityByOstrovsky (:628-662) with
 * dbscanDouble (:533-605, dbscan's algorithm with a double result).  `data`,
 * `intervals`, `helpful` hold rec doubles.  A point whose recorded loop
 * diverged is -1: the reference sets only flag 3 for it and leaves the other
 * four flags as the allocation left them -- false for zero-filled memory. */
double orc_ostrovsky_point(const orc_job* job, int64_t g, double* data, double* intervals,
                           double* helpful)
{
    const int rec = orc_record_len(job);
    const double thr = job->ostrovskyThreshold;
    int f[5] = {0, 0, 0, 0, 0};
    int n = 0;
    if (orc_trajectory_point(job, g, data)) {
        f[3] = 1;
    } else {
        const double lastPoint = rec > 0 ? data[rec - 1] : 0.0;
        n = orc_peak_finder(data, 0, rec, data, intervals, 0.01);
        f[0] = 1;
        for (int i = 1; i < n; ++i)
            if (data[i] - data[i - 1] > 0) {
                f[0] = 0;
                break;
            }
        int one = 0, zero = 0;
        for (int i = 1; i < n; ++i) {
            if (data[i] > thr)
                one = 1;
            else
                zero = 1;
            if (one && zero)
                break;
        }
        f[1] = one && zero;
        f[2] = !(one && !zero);
        f[3] = (n == 0 || n == 1);
        f[4] = lastPoint > thr;
    }
    double out = (double)orc_dbscan(data, intervals, helpful, 0, n, rec, job->maxAmountOfPeaks,
                                    job->dbscanEps);
    if (f[2])
        out = -1 * out;
    if (f[3])
        out = f[4] ? 1 : -1;
    if (f[1])
        out = 0;
    if (f[0]) {
        if (out > 0)
            out = 0.5;
        else if (out == 0)
            out = 0;
        else
            out = -0.5;
    }
    return out;
}

int orc_map_ostrovsky(const orc_job* job, int64_t first, int64_t count, double* out, int nThreads)
{
    const int rec = orc_record_len(job);
    if (rec <= 0)
        return -1;
    int err = 0;
#pragma omp parallel num_threads(threads_or_default(nThreads))
    {
        double* data = (double*)malloc(sizeof(double) * (size_t)rec);
        double* intervals = (double*)malloc(sizeof(double) * (size_t)rec);
        double* helpful = (double*)malloc(sizeof(double) * (size_t)rec);
        if (!data || !intervals || !helpful) {
#pragma omp atomic write
            err = -2;
        } else {
#pragma omp for schedule(dynamic, 1)
            for (int64_t k = 0; k < count; ++k)
                out[k] = orc_ostrovsky_point(job, first + k, data, intervals, helpful);
        }
        free(data);
        free(intervals);
        free(helpful);
    }
    return err;
}

/* modelingOneSystemDenis (hostLibrary.cu:162-239) with calculateDiscreteModelDenisCUDA
 * (cudaLibrary.cu:121-161): thread idx < T = (int)(hSpecial/h) runs idx steps of h
 * from the initial conditions, then records x[writableVar] before each of
 * (int)(tMax/hSpecial) steps of hSpecial into out[idx + i*T].  out has
 * (int)(tMax/h) entries; writes past it are dropped and entries no thread
 * writes are NaN (the reference leaves them uninitialised).  No divergence test. */
int orc_modeling_one_system(int system, double tMax, double h, double hSpecial, const double* ic, int nIC,
                            int writableVar, const double* values, int nV, double* out, int64_t n)
{
    const int T = (int)(hSpecial / h);
    const int I = (int)(tMax / hSpecial);
    if (nIC <= 0 || nIC > 8 || nV <= 0 || nV > 16)
        return -1;
    for (int64_t j = 0; j < n; ++j)
        out[j] = NAN;
    for (int idx = 0; idx < T; ++idx) {
        double x[8], v[16];
        for (int i = 0; i < nIC; ++i)
            x[i] = ic[i];
        for (int i = 0; i < nV; ++i)
            v[i] = values[i];
        orc_loop(system, x, v, h, idx, 1, 0, 0, NULL, 0, 1);
        for (int i = 0; i < I; ++i) {
            const int64_t j = (int64_t)idx + (int64_t)i * T;
            if (j < n)
                out[j] = x[writableVar];
            orc_loop(system, x, v, hSpecial, 1, 1, 0, 0, NULL, 0, 1);
        }
    }
    return 0;
}

int orc_map_lle(const orc_job* job, int64_t first, int64_t count, double* out, int nThreads)
{
    if ((int)(job->tMax / job->NT) <= 0 || job->nIC <= 0)
        return -1;
#pragma omp parallel for schedule(dynamic, 1) num_threads(threads_or_default(nThreads))
    for (int64_t k = 0; k < count; ++k)
        out[k] = orc_lle_point(job, first + k);
    return 0;
}

int orc_map_lle_seeded(const orc_job* job, int64_t first, int64_t count, const double* z,
                       double* out, int nThreads)
{
    if ((int)(job->tMax / job->NT) <= 0 || job->nIC <= 0)
        return -1;
#pragma omp parallel for schedule(dynamic, 1) num_threads(threads_or_default(nThreads))
    for (int64_t k = 0; k < count; ++k)
        out[k] = orc_lle_point_seeded(job, first + k, z + k * job->nIC);
    return 0;
}

int orc_map_lle_regime_list(const orc_job* job, const int64_t* idx, int64_t count,
                            const double* z, double* outLle, int32_t* outCls, int nThreads)
{
    if ((int)(job->tMax / job->NT) <= 0 || job->nIC <= 0)
        return -1;
#pragma omp parallel for schedule(dynamic, 1) num_threads(threads_or_default(nThreads))
    for (int64_t k = 0; k < count; ++k)
        outLle[k] = orc_lle_regime_point(job, idx[k], z ? z + k * job->nIC : NULL, &outCls[k]);
    return 0;
}

/* ------------------------------------------------------------------------- */
/* Lyapunov spectrum (LSKernelCUDA, cudaLibrary.cu:960-1100).                 */

/* projectionOperator (cudaLibrary.cu:913-927): minuend -= (a.b / b.b) b, with
 * the fraction 0 when b.b == 0; sums accumulated in index order. */
void orc_projection(const double* a, const double* b, double* minuend, int n)
{
    double numerator = 0, denominator = 0;
    for (int i = 0; i < n; ++i) {
        numerator += a[i] * b[i];
        denominator += b[i] * b[i];
    }
    const double fraction = denominator == 0 ? 0 : numerator / denominator;
    for (int i = 0; i < n; ++i)
        minuend[i] -= fraction * b[i];
}

/* gramSchmidtProcess (cudaLibrary.cu:931-956): classical Gram-Schmidt of the n
 * rows of a into b (each row projected against the not yet normalised earlier
 * rows of b), then every row of b normalised; den[i] (optional) = the norm. */
void orc_gram_schmidt(const double* a, double* b, int n, double* den)
{
    for (int i = 0; i < n; ++i) {
        for (int j = 0; j < n; ++j)
            b[j + i * n] = a[j + i * n];
        for (int j = 0; j < i; ++j)
            orc_projection(a + i * n, b + j * n, b + i * n, n);
    }
    for (int i = 0; i < n; ++i) {
        double d = 0;
        for (int j = 0; j < n; ++j)
            d += b[i * n + j] * b[i * n + j];
        d = sqrt(d);
        for (int j = 0; j < n; ++j)
            b[i * n + j] = d == 0 ? 0 : b[i * n + j] / d;
        if (den)
            den[i] = d;
    }
}

/* Initial perturbation rows (cudaLibrary.cu:1001-1013): row j, entry i =
 * 0.5 sinf(0.2171828 (i+1)(j+1) + idx + (0.2171828 + i j idx)) with idx the
 * chunk-local point index, each row normalised to length 1. */
void orc_ls_seed(const orc_job* job, int64_t g, double* z)
{
    const int n = job->nIC;
    const int idx = (int)(job->seedChunk > 0 ? g % job->seedChunk : g);
    for (int j = 0; j < n; ++j) {
        double zPower = 0;
        for (int i = 0; i < n; ++i) {
            const double arg = 0.2171828 * (i + 1) * (j + 1) + idx + (0.2171828 + i * j * idx);
            z[j * n + i] = (double)sinf((float)arg) * 0.5;
            zPower += z[j * n + i] * z[j * n + i];
        }
        zPower = sqrt(zPower);
        for (int i = 0; i < n; ++i)
            z[j * n + i] /= zPower;
    }
}

/* One point of LSKernelCUDA: the nIC exponents into out[0..nIC).  zIn (n*n,
 * optional) replaces the seed rows. */
void orc_ls_point(const orc_job* job, int64_t g, const double* zIn, double* out)
{
    double x[8], y[64], z[64], v[16], den[8], result[8];
    const int n = job->nIC;
    state_units u;
    const int sys = setup_state(job, g, x, v, &u);
    if (zIn) {
        for (int i = 0; i < n * n; ++i)
            z[i] = zIn[i];
    } else {
        orc_ls_seed(job, g, z);
    }
    const double h = job->h;
    const int nNT = (int)(size_t)(job->NT / h);
    const int sizeOfBlock = (int)(job->tMax / job->NT);
    const double eps = job->lleEps;
    for (int i = 0; i < n; ++i)
        result[i] = 0;

    orc_loop(sys, x, v, h, orc_skip_len(job), 1, 0, job->maxValue, NULL, 0, 1);
    orc_gram_schmidt(z, y, n, NULL);
    /* perturbations placed, and deviations orthonormalised, in physical units */
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i)
            y[j * n + i] = to_stored(y[j * n + i] * eps, i, &u) + x[i];

    for (int b = 0; b < sizeOfBlock; ++b) {
        /* every trajectory stops at its own first violation (cudaLibrary.cu:1049-1060) */
        orc_loop(sys, x, v, h, nNT, 1, 0, job->maxValue, NULL, 0, 1);
        for (int j = 0; j < n; ++j)
            orc_loop(sys, y + j * n, v, h, nNT, 1, 0, job->maxValue, NULL, 0, 1);
        for (int k = 0; k < n; ++k)
            for (int l = 0; l < n; ++l)
                y[k * n + l] = to_phys(y[k * n + l] - x[l], l, &u);
        orc_gram_schmidt(y, z, n, den);
        for (int k = 0; k < n; ++k) {
            result[k] += log(den[k] / eps);
            for (int j = 0; j < n; ++j)
                y[k * n + j] = (double)(x[j] + to_stored(z[k * n + j] * eps, j, &u));
        }
    }
    for (int i = 0; i < n; ++i)
        out[i] = result[i] / job->tMax;
}

int orc_map_ls_list(const orc_job* job, const int64_t* idx, int64_t count, const double* z,
                    double* out, int nThreads)
{
    if (job->nIC <= 0 || job->nIC > 8)
        return -1;
    const int n = job->nIC;
#pragma omp parallel for schedule(dynamic, 1) num_threads(threads_or_default(nThreads))
    for (int64_t k = 0; k < count; ++k)
        orc_ls_point(job, idx[k], z ? z + k * n * n : NULL, out + k * n);
    return 0;
}

int orc_map_lle_list(const orc_job* job, const int64_t* idx, int64_t count, double* out, int nThreads)
{
    if ((int)(job->tMax / job->NT) <= 0 || job->nIC <= 0)
        return -1;
#pragma omp parallel for schedule(dynamic, 1) num_threads(threads_or_default(nThreads))
    for (int64_t k = 0; k < count; ++k)
        out[k] = orc_lle_point(job, idx[k]);
    return 0;
}

int orc_map_lle_list_seeded(const orc_job* job, const int64_t* idx, int64_t count, const double* z,
                            double* out, int nThreads)
{
    if ((int)(job->tMax / job->NT) <= 0 || job->nIC <= 0)
        return -1;
#pragma omp parallel for schedule(dynamic, 1) num_threads(threads_or_default(nThreads))
    for (int64_t k = 0; k < count; ++k)
        out[k] = orc_lle_point_seeded(job, idx[k], z ? z + k * job->nIC : NULL);
    return 0;
}
