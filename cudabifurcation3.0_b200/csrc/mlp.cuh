// Internal interface of the surrogate network (mlp.cu) for the surrogate map
// pipeline (surrogate.cu).
#pragma once
#include "engine.cuh"

struct cbf_mlp;

namespace cbf {

// Input features of grid point g of a 2-D parameter sweep of a 3-D system:
//   f0 = system code (Rossler -1, Lorenz 0, Chen +1: the system one-hot folded
//        into one input), f1, f2 = the two swept parameters mapped to [-1, 1]
//        over the sweep ranges, f3 = the remaining parameter / 10.
struct FeatureSpec {
    DevJob J;
    float sys;
    float lo0, inv0, lo1, inv1;  // f = (p - lo) * inv - 1
    float third;
};

FeatureSpec feature_spec(const DevJob& J);

// X[k*4 .. k*4+3] = features of grid point idx[k] (FP32), k < n.
cudaError_t mlp_features(const FeatureSpec& f, const long long* idx, long long n, float* X,
                         cudaStream_t s);

// Predictions for every grid point 0..nPoints-1, features generated on the fly:
// lle (de-normalised, double), cls (argmax), conf (softmax maximum).
cudaError_t mlp_predict_grid(cbf_mlp* m, const FeatureSpec& f, long long nPoints, float lleMean,
                             float lleStd, double* lle, int* cls, float* conf, cudaStream_t s);

// Parameters re-initialised from `seed` exactly as cbf_mlp_create does, Adam
// state and step counter zeroed (the captured training graph is kept unless the
// seed changed).
cudaError_t mlp_reset(cbf_mlp* m, unsigned long long seed);

}  // namespace cbf
