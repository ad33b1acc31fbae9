// hostLibrary.h -- C++ drop-in facade with the reference's host entry points.
//
// Same names, parameter lists, C++ linkage and behaviour as the reference's
// Library/hostLibrary.cuh (lines cited per function): each call computes the
// map on the GPU (through the C-ABI in cbf.h) and writes the reference's CSV
// layout to the output file.  Error behaviour matches the reference's gpuAssert
// (Library/cudaMacros.cu:3-10): print "GPUassert: <message> <file> <line>" to
// stderr and exit with the error code; an output file that cannot be written
// prints "\nOutput file open error\n" and exits with 1 (hostLibrary.cu:134-138).
//
// Two things the reference fixes at compile time are run-time settings here:
//   - the ODE system (the reference compiles one calculateDiscreteModel):
//     cbfSetSystem(), or the environment variable CBF_SYSTEM
//     (memristive5 | rossler | lorenz | chen); default memristive5, the model the
//     reference ships with;
//   - the output path (OUT_FILE_PATH, hostLibrary.cu:3): cbfSetOutputPath(), or
//     CBF_OUT_FILE_PATH; default "mat.csv" in the working directory.
#ifndef CBF_HOST_LIBRARY_H
#define CBF_HOST_LIBRARY_H

// hostLibrary.cuh:29-42
void bifurcation1D(const double tMax, const int nPts, const double h,
                   const int amountOfInitialConditions, const double* initialConditions,
                   const double* ranges, const int* indicesOfMutVars, const int writableVar,
                   const double maxValue, const double transientTime, const double* values,
                   const int amountOfValues, const int preScaller);

// hostLibrary.cuh:89-102
void bifurcation1DIC(const double tMax, const int nPts, const double h,
                     const int amountOfInitialConditions, const double* initialConditions,
                     const double* ranges, const int* indicesOfMutVars, const int writableVar,
                     const double maxValue, const double transientTime, const double* values,
                     const int amountOfValues, const int preScaller);

// hostLibrary.cuh:129-147
void bifurcation2DKDE(const double tMax, const int nPts, const double h,
                      const int amountOfInitialConditions, const double* initialConditions,
                      const double* ranges, const int* indicesOfMutVars, const int writableVar,
                      const double maxValue, const int maxAmountOfPeaks,
                      const double transientTime, const double* values,
                      const int amountOfValues, const int preScaller, const int in_kdeSampling,
                      const double in_kdeSamplesInterval1, const double in_kdeSamplesInterval2,
                      const double in_kdeSamplesSmooth);

// hostLibrary.cuh:171-186
void bifurcation2DDBSCAN(const double tMax, const int nPts, const double h,
                         const int amountOfInitialConditions, const double* initialConditions,
                         const double* ranges, const int* indicesOfMutVars, const int writableVar,
                         const double maxValue, const int maxAmountOfPeaks,
                         const double transientTime, const double* values,
                         const int amountOfValues, const int preScaller, const double eps);

// hostLibrary.cuh:254-272
void bifurcation2DKDEIC(const double tMax, const int nPts, const double h,
                        const int amountOfInitialConditions, const double* initialConditions,
                        const double* ranges, const int* indicesOfMutVars, const int writableVar,
                        const double maxValue, const int maxAmountOfPeaks,
                        const double transientTime, const double* values,
                        const int amountOfValues, const int preScaller, const int in_kdeSampling,
                        const double in_kdeSamplesInterval1, const double in_kdeSamplesInterval2,
                        const double in_kdeSamplesSmooth);

// hostLibrary.cuh:296-311
void bifurcation2DDBSCANIC(const double tMax, const int nPts, const double h,
                           const int amountOfInitialConditions, const double* initialConditions,
                           const double* ranges, const int* indicesOfMutVars,
                           const int writableVar, const double maxValue,
                           const int maxAmountOfPeaks, const double transientTime,
                           const double* values, const int amountOfValues,
                           const int preScaller, const double eps);

// hostLibrary.cuh:334-348
void LLE1D(const double tMax, const double NT, const int nPts, const double h, const double eps,
           const double* initialConditions, const int amountOfInitialConditions,
           const double* ranges, const int* indicesOfMutVars, const int writableVar,
           const double maxValue, const double transientTime, const double* values,
           const int amountOfValues);

// hostLibrary.cuh:371-385
void LLE1DIC(const double tMax, const double NT, const int nPts, const double h, const double eps,
             const double* initialConditions, const int amountOfInitialConditions,
             const double* ranges, const int* indicesOfMutVars, const int writableVar,
             const double maxValue, const double transientTime, const double* values,
             const int amountOfValues);

// hostLibrary.cuh:408-422
void LLE2D(const double tMax, const double NT, const int nPts, const double h, const double eps,
           const double* initialConditions, const int amountOfInitialConditions,
           const double* ranges, const int* indicesOfMutVars, const int writableVar,
           const double maxValue, const double transientTime, const double* values,
           const int amountOfValues);

// hostLibrary.cuh:445-459
void LLE2DIC(const double tMax, const double NT, const int nPts, const double h, const double eps,
             const double* initialConditions, const int amountOfInitialConditions,
             const double* ranges, const int* indicesOfMutVars, const int writableVar,
             const double maxValue, const double transientTime, const double* values,
             const int amountOfValues);

// One system sampled with a step offset: rows "h*j, x" at precision 12
// (hostLibrary.cu:162-239).
void modelingOneSystemDenis(const double tMax, const double h, const double hSpecial,
                            const int amountOfInitialConditions, const double* initialConditions,
                            const int writableVar, const double* values, const int amountOfValues);

// Periodicity map by Ostrovsky's rule (a 2-D sweep of initial conditions):
// header + map at the default precision (hostLibrary.cu:748-925).
void calculationOfPeriodicityByOstrovsky(const double tMax, const int nPts, const double h,
                                         const int amountOfInitialConditions,
                                         const double* initialConditions, const double* ranges,
                                         const int* indicesOfMutVars, const int writableVar,
                                         const double maxValue, const int maxAmountOfPeaks,
                                         const double transientTime, const double* values,
                                         const int amountOfValues, const int preScaller,
                                         const double eps, const double ostrovskyThreshold);

// Lyapunov spectra.  LS1D writes "param, l1, ..., lN" rows to the output path;
// LS2D writes one map per exponent to <output path><k>.csv, k = 1..N, with the
// 2-D map layout (hostLibrary.cu:1802-2082).
void LS1D(const double tMax, const double NT, const int nPts, const double h, const double eps,
          const double* initialConditions, const int amountOfInitialConditions,
          const double* ranges, const int* indicesOfMutVars, const int writableVar,
          const double maxValue, const double transientTime, const double* values,
          const int amountOfValues);
void LS2D(const double tMax, const double NT, const int nPts, const double h, const double eps,
          const double* initialConditions, const int amountOfInitialConditions,
          const double* ranges, const int* indicesOfMutVars, const int writableVar,
          const double maxValue, const double transientTime, const double* values,
          const int amountOfValues);

// Run-time configuration of what the reference fixes at compile time.
void cbfSetSystem(int system);            // CBF_SYS_* from cbf.h
int cbfGetSystem();
void cbfSetOutputPath(const char* path);  // nullptr restores the default
const char* cbfGetOutputPath();

// Opt-in, no counterpart in the reference: with cbfSetSurrogate(1) (or the
// environment variable CBF_SURROGATE=1; cbfSetSurrogate(-1) returns to the
// environment's choice) LLE2D writes the surrogate-refined LLE map of
// cbf_lle2d_surrogate (cbf.h) -- same grid, seeds, header and layout -- and the
// regime classes beside it in "<path>.regime.csv" (same layout, integers).
void cbfSetSurrogate(int enable);
int cbfGetSurrogate();

// The same settings for bindings without C++ name mangling (ctypes, cgo).
extern "C" {
void cbf_facade_set_system(int system);
void cbf_facade_set_output_path(const char* path);
void cbf_facade_set_surrogate(int enable);
}

#endif  // CBF_HOST_LIBRARY_H
