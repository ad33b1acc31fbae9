// ODE systems: one fixed-step CD (semi-implicit composition) step each.
//
// The reference integrates whatever `calculateDiscreteModel` it was compiled with
// (Library/cudaLibrary.cu:2-44): an explicit half-step with k = h*s in reverse
// variable order, then a linearly implicit half-step with h1 = h*(1-s) in forward
// order, s = values[0] (the 5-D shipped model keeps s in values[7]).  The library
// ships that model verbatim plus Rossler, Lorenz and Chen in the same scheme.
//
// The state lives in registers for the whole trajectory.  Each system hoists its
// parameter-only quantities (k, h1, products, reciprocals of the implicit
// denominators) into a Coef struct once per point; the step itself is a fixed
// chain of FP64 FMA/MUL/ADD.  The whole library is compiled with -fmad=false, so
// the only fused operations are the explicit fma() calls below -- the CPU oracle
// (oracle/oracle.c) evaluates the same operations and matches bit for bit.
#pragma once

#include <cuda_runtime.h>
#include <math.h>

namespace cbf {

// ---------------------------------------------------------------------------
// The 5-D memristive model compiled into the reference (cudaLibrary.cu:2-44),
// restated literally: no explicit FMA, and the FP32 quirks of `float y[5], k`
// (:19) kept -- k and the explicit-half snapshot are rounded to float.
struct Memristive5 {
    static constexpr int DIM = 5;
    static constexpr int NV = 8;
    static constexpr int FLOPS = 66;  // adds/subs/muls/divs of one step, abs excluded
    struct Coef {
        double a0, a1, a2, a3, a4, a5, a6;
        double kd;  // (double)(float)(h * a7)
        double h1;  // h * (1 - a7)
    };
    __host__ __device__ static Coef prep(const double* a, double h)
    {
        Coef c;
        c.a0 = a[0]; c.a1 = a[1]; c.a2 = a[2]; c.a3 = a[3];
        c.a4 = a[4]; c.a5 = a[5]; c.a6 = a[6];
        float k = (float)(h * a[7]);
        c.kd = (double)k;
        c.h1 = h * (1 - a[7]);
        return c;
    }
    __device__ __forceinline__ static void step(double* x, const Coef& c)
    {
        const double k = c.kd;
        x[4] = x[4] + k * (x[0]);
        x[3] = x[3] + k * (-c.a2 * x[1] - c.a3 * x[3]);
        x[2] = x[2] + k * (c.a1 * (x[1] - x[0] - x[2]));
        x[1] = x[1] + k * (-x[2] + x[3]);
        x[0] = x[0] + k * (c.a0 * (x[2] - (c.a4 + c.a5 + c.a6 * fabs(x[4])) * x[0]));

        const double y0 = (double)(float)x[0];
        const double y1 = (double)(float)x[1];
        const double y2 = (double)(float)x[2];
        const double y3 = (double)(float)x[3];
        const double y4 = (double)(float)x[4];

        const double h1 = c.h1;
        x[0] = (y0 + h1 * (c.a0 * x[2])) / (1 + h1 * c.a0 * (c.a4 + c.a5 + c.a6 * fabs(x[4])));
        x[1] = y1 + h1 * (-x[2] + x[3]);
        x[2] = (y2 + h1 * (c.a1 * (x[1] - x[0]))) / (1 + h1 * c.a1);
        x[3] = (y3 + h1 * (-c.a2 * x[1])) / (1 + h1 * c.a3);
        x[4] = y4 + h1 * (x[0]);
    }
};

// ---------------------------------------------------------------------------
// Rossler: x' = -y - z, y' = x + a*y, z' = b + z*(x - c); values = {s, a, b, c}.
// The implicit z half-step has a state-dependent denominator (one FP64 divide).
struct Rossler {
    static constexpr int DIM = 3;
    static constexpr int NV = 4;
    static constexpr int FLOPS = 23;
    struct Coef { double a, b, c, k, h1, h1b, r2; };
    __host__ __device__ static Coef prep(const double* v, double h)
    {
        Coef q;
        const double s = v[0];
        q.a = v[1]; q.b = v[2]; q.c = v[3];
        q.k = h * s;
        q.h1 = h * (1.0 - s);
        q.h1b = q.h1 * q.b;
        q.r2 = 1.0 / (1.0 - q.h1 * q.a);
        return q;
    }
    __device__ __forceinline__ static void step(double* X, const Coef& q)
    {
        double x = X[0], y = X[1], z = X[2];
        z = fma(q.k, fma(z, x - q.c, q.b), z);
        y = fma(q.k, fma(q.a, y, x), y);
        x = fma(-q.k, y + z, x);
        x = fma(-q.h1, y + z, x);
        y = fma(q.h1, x, y) * q.r2;
        z = (z + q.h1b) / fma(-q.h1, x - q.c, 1.0);
        X[0] = x; X[1] = y; X[2] = z;
    }
};

// ---------------------------------------------------------------------------
// Lorenz: x' = sigma*(y - x), y' = x*(rho - z) - y, z' = x*y - beta*z;
// values = {s, sigma, rho, beta}.  17 FP64 instructions per step.
struct Lorenz {
    static constexpr int DIM = 3;
    static constexpr int NV = 4;
    static constexpr int FLOPS = 25;
    struct Coef { double rho, beta, k, ks, h1, h1s, r1, r2, r3; };
    __host__ __device__ static Coef prep(const double* v, double h)
    {
        Coef q;
        const double s = v[0], sg = v[1];
        q.rho = v[2]; q.beta = v[3];
        q.k = h * s;
        q.h1 = h * (1.0 - s);
        q.ks = q.k * sg;
        q.h1s = q.h1 * sg;
        q.r1 = 1.0 / (1.0 + q.h1s);
        q.r2 = 1.0 / (1.0 + q.h1);
        q.r3 = 1.0 / (1.0 + q.h1 * q.beta);
        return q;
    }
    __device__ __forceinline__ static void step(double* X, const Coef& q)
    {
        double x = X[0], y = X[1], z = X[2];
        z = fma(q.k, fma(-q.beta, z, x * y), z);
        y = fma(q.k, fma(x, q.rho - z, -y), y);
        x = fma(q.ks, y - x, x);
        x = fma(q.h1s, y, x) * q.r1;
        y = fma(q.h1, x * (q.rho - z), y) * q.r2;
        z = fma(q.h1, x * y, z) * q.r3;
        X[0] = x; X[1] = y; X[2] = z;
    }
};

// ---------------------------------------------------------------------------
// Chen: x' = a*(y - x), y' = (c - a)*x - x*z + c*y, z' = x*y - b*z;
// values = {s, a, b, c}.  18 FP64 instructions (26 flops) per step.
struct Chen {
    static constexpr int DIM = 3;
    static constexpr int NV = 4;
    static constexpr int FLOPS = 26;
    struct Coef { double b, c, k, cma, ka, h1, h1a, r1, r2, r3; };
    __host__ __device__ static Coef prep(const double* v, double h)
    {
        Coef q;
        const double s = v[0], a = v[1];
        q.b = v[2]; q.c = v[3];
        q.k = h * s;
        q.h1 = h * (1.0 - s);
        q.cma = q.c - a;
        q.ka = q.k * a;
        q.h1a = q.h1 * a;
        q.r1 = 1.0 / (1.0 + q.h1a);
        q.r2 = 1.0 / (1.0 - q.h1 * q.c);
        q.r3 = 1.0 / (1.0 + q.h1 * q.b);
        return q;
    }
    __device__ __forceinline__ static void step(double* X, const Coef& q)
    {
        double x = X[0], y = X[1], z = X[2];
        z = fma(q.k, fma(-q.b, z, x * y), z);
        y = fma(q.k, fma(x, q.cma - z, q.c * y), y);
        x = fma(q.ka, y - x, x);
        x = fma(q.h1a, y, x) * q.r1;
        y = fma(q.h1, x * (q.cma - z), y) * q.r2;
        z = fma(q.h1, x * y, z) * q.r3;
        X[0] = x; X[1] = y; X[2] = z;
    }
};

}  // namespace cbf
