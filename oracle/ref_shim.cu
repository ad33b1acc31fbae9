// Test-only C-ABI shim over the reference library's own host-callable functions.
//
// Built by `make -C oracle ref` from the reference sources where they lie
// (Library/cudaLibrary.cu, Library/cudaMacros.cu) into oracle/_ref/libcbf_ref.so.
// The reference declares these functions __device__ __host__, so its unmodified
// source compiles them for the host too; this file only re-exports them with
// C linkage so the tests can pin the oracle's restatement bit-for-bit.
// Nothing from the reference is copied: the header is included from its tree.
#include "cudaLibrary.cuh"

// Defined __device__ __host__ in cudaLibrary.cu (:913-956) without a header
// declaration; declared here with the definition's signature.
__device__ __host__ void projectionOperator(double* a, double* b, double* minuend, int amountOfValues);
__device__ __host__ void gramSchmidtProcess(double* a, double* b, int amountOfVectorsAndValuesInVector,
                                            double* denominators);

extern "C" {

// cudaLibrary.cu:210-216
double ref_getValueByIdx(int idx, int nPts, double startRange, double finishRange, int valueNumber)
{
    return getValueByIdx(idx, nPts, startRange, finishRange, valueNumber);
}

// cudaLibrary.cu:2-44 (the 5-D memristive model compiled into the reference)
void ref_calculateDiscreteModel(double* x, const double* a, double h)
{
    calculateDiscreteModel(x, a, h);
}

// cudaLibrary.cu:55-74
int ref_loopCalculateDiscreteModel(double* x, const double* values, double h, int amountOfIterations,
                                   int preScaller, int writableVar, double maxValue, double* data,
                                   int startDataIndex, int writeStep)
{
    return loopCalculateDiscreteModel(x, values, h, amountOfIterations, preScaller, writableVar,
                                      maxValue, data, startDataIndex, writeStep) ? 1 : 0;
}

// cudaLibrary.cu:220-266
int ref_peakFinder(double* data, int startDataIndex, int amountOfPoints, double* outPeaks,
                   double* timeOfPeaks, double h)
{
    return peakFinder(data, startDataIndex, amountOfPoints, outPeaks, timeOfPeaks, h);
}

// cudaLibrary.cu:356-422
int ref_kde(double* data, int startDataIndex, int amountOfPoints, int maxAmountOfPeaks,
            int kdeSampling, double i1, double i2, double smoothH)
{
    return kde(data, startDataIndex, amountOfPoints, maxAmountOfPeaks, kdeSampling, i1, i2, smoothH);
}

// cudaLibrary.cu:445-453
double ref_distance(double x1, double y1, double x2, double y2)
{
    return distance(x1, y1, x2, y2);
}

// cudaLibrary.cu:457-529
int ref_dbscan(double* data, double* intervals, double* helpfulArray, int startDataIndex,
               int amountOfPeaks, int sizeOfHelpfulArray, int maxAmountOfPeaks, double eps)
{
    return dbscan(data, intervals, helpfulArray, startDataIndex, amountOfPeaks, sizeOfHelpfulArray,
                  maxAmountOfPeaks, 0, eps, nullptr);
}

// cudaLibrary.cu:913-927
void ref_projectionOperator(double* a, double* b, double* minuend, int n)
{
    projectionOperator(a, b, minuend, n);
}

// cudaLibrary.cu:931-956
void ref_gramSchmidtProcess(double* a, double* b, int n, double* denominators)
{
    gramSchmidtProcess(a, b, n, denominators);
}

}  // extern "C"
