// ODE systems: one fixed-step CD (semi-implicit composition) step each.
//
// The reference integrates whatever `calculateDiscreteModel` it was compiled with
// (Library/cudaLibrary.cu:2-44): an explicit half-step with k = h*s in reverse
// variable order, then a linearly implicit half-step with h1 = h*(1-s) in forward
// order, s = values[0] (the 5-D shipped model keeps s in values[7]).  The library
// ships that model verbatim plus Rossler, Lorenz and Chen in the same scheme.
//
// The state lives in registers for the whole trajectory.  Each system hoists its
// parameter-only quantities into a Coef struct once per point; the step itself
// is a fixed chain of FP64 FMA/MUL/ADD.  The whole library is compiled with -fmad=false, so
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
    static constexpr bool SCALED = false;  // state stored in physical units
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
// The three library systems share one evaluation scheme of the CD step.  With
// k = h*s and h1 = h*(1-s), the explicit half (reverse order) and the linearly
// implicit half (forward order) are multiplied out so that every parameter-only
// factor is hoisted and the terms k*x and (c-a)-z1 (rho-z1) are shared:
//   Chen / Lorenz  14 FP64 instructions, critical path 9 (vs 18 / ~17 when each
//                  half-step is evaluated as written);
//   Rossler        10 instructions + one IEEE divide (state-dependent implicit z).
// The mathematics is exactly the CD composition; only the rounding order is
// the library's own, and the CPU oracle follows it operation for operation.

// Rossler: x' = -y - z, y' = x + a*y, z' = b + z*(x - c); values = {s, a, b, c}.
//   z1 = z + k*(b + z*(x - c))          = fma(z, fma(k, x, 1 - k*c), k*b)
//   y1 = y + k*(x + a*y)                = fma(1 + k*a, y, k*x)
//   x2 = x - k*(y1+z1) - h1*(y1+z1)     = fma(-(k + h1), y1 + z1, x)
//   y2 = (y1 + h1*x2) / (1 - h1*a)      = fma(h1*r2, x2, r2*y1)
//   z2 = (z1 + h1*b) / (1 - h1*(x2 - c)) = (z1 + h1*b) / fma(-h1, x2, 1 + h1*c)
struct Rossler {
    static constexpr int DIM = 3;
    static constexpr int NV = 4;
    static constexpr int FLOPS = 17;
    static constexpr bool SCALED = false;
    struct Coef { double k, c1, kb, bq, hs, r2, g, h1, h1b, c2; };
    __host__ __device__ static Coef prep(const double* v, double h)
    {
        Coef q;
        const double s = v[0], a = v[1], b = v[2], c = v[3];
        q.k = h * s;
        q.h1 = h * (1.0 - s);
        q.c1 = 1.0 - q.k * c;
        q.kb = q.k * b;
        q.bq = 1.0 + q.k * a;
        q.hs = q.k + q.h1;
        q.r2 = 1.0 / (1.0 - q.h1 * a);
        q.g = q.h1 * q.r2;
        q.h1b = q.h1 * b;
        q.c2 = 1.0 + q.h1 * c;
        return q;
    }
    __device__ __forceinline__ static void step(double* X, const Coef& q)
    {
        const double x = X[0], y = X[1], z = X[2];
        const double z1 = fma(z, fma(q.k, x, q.c1), q.kb);
        const double y1 = fma(q.bq, y, q.k * x);
        const double x2 = fma(-q.hs, y1 + z1, x);
        const double y2 = fma(q.g, x2, q.r2 * y1);
        const double z2 = (z1 + q.h1b) / fma(-q.h1, x2, q.c2);
        X[0] = x2; X[1] = y2; X[2] = z2;
    }
};

// ---------------------------------------------------------------------------
// Chen: x' = a*(y - x), y' = (c - a)*x - x*z + c*y, z' = x*y - b*z;
// values = {s, a, b, c}.
//   z1 = z + k*(x*y - b*z)                 = fma(k*x, y, (1 - k*b)*z)
//   y1 = y + k*((c-a)*x - x*z1 + c*y)      = fma(k*x, w, (1 + k*c)*y),  w = (c-a) - z1
//   x1 = x + k*a*(y1 - x);  x2 = (x1 + h1*a*y1)/(1 + h1*a)
//                                          = fma((1-k*a)*r1, x, ((k*a + h1*a)*r1)*y1)
//   y2 = (y1 + h1*x2*w) / (1 - h1*c)       = fma((h1*r2)*x2, w, r2*y1)
//   z2 = (z1 + h1*x2*y2) / (1 + h1*b)      = fma((h1*r3)*x2, y2, r3*z1)
struct Chen {
    static constexpr int DIM = 3;
    static constexpr int NV = 4;
    static constexpr int FLOPS = 19;
    static constexpr bool SCALED = false;
    struct Coef { double k, ca, cb, cma, d, e, r2, g, r3, hh; };
    __host__ __device__ static Coef prep(const double* v, double h)
    {
        Coef q;
        const double s = v[0], a = v[1], b = v[2], c = v[3];
        q.k = h * s;
        const double h1 = h * (1.0 - s);
        const double ka = q.k * a;
        const double h1a = h1 * a;
        q.ca = 1.0 - q.k * b;
        q.cb = 1.0 + q.k * c;
        q.cma = c - a;
        const double r1 = 1.0 / (1.0 + h1a);
        q.d = (1.0 - ka) * r1;
        q.e = (ka + h1a) * r1;
        q.r2 = 1.0 / (1.0 - h1 * c);
        q.g = h1 * q.r2;
        q.r3 = 1.0 / (1.0 + h1 * b);
        q.hh = h1 * q.r3;
        return q;
    }
    __device__ __forceinline__ static void step(double* X, const Coef& q)
    {
        const double x = X[0], y = X[1], z = X[2];
        const double kx = q.k * x;
        const double z1 = fma(kx, y, q.ca * z);
        const double w = q.cma - z1;
        const double y1 = fma(kx, w, q.cb * y);
        const double x2 = fma(q.d, x, q.e * y1);
        const double y2 = fma(q.g * x2, w, q.r2 * y1);
        const double z2 = fma(q.hh * x2, y2, q.r3 * z1);
        X[0] = x2; X[1] = y2; X[2] = z2;
    }
};

// ---------------------------------------------------------------------------
// Lorenz: x' = sigma*(y - x), y' = x*(rho - z) - y, z' = x*y - beta*z;
// values = {s, sigma, rho, beta}.  Same scheme as Chen with
// (1 - k*beta), (1 - k), w = rho - z1, sigma in place of a, r2 = 1/(1 + h1).
struct Lorenz {
    static constexpr int DIM = 3;
    static constexpr int NV = 4;
    static constexpr int FLOPS = 19;
    static constexpr bool SCALED = false;
    struct Coef { double k, ca, cb, rho, d, e, r2, g, r3, hh; };
    __host__ __device__ static Coef prep(const double* v, double h)
    {
        Coef q;
        const double s = v[0], sg = v[1], beta = v[3];
        q.rho = v[2];
        q.k = h * s;
        const double h1 = h * (1.0 - s);
        const double ks = q.k * sg;
        const double h1s = h1 * sg;
        q.ca = 1.0 - q.k * beta;
        q.cb = 1.0 - q.k;
        const double r1 = 1.0 / (1.0 + h1s);
        q.d = (1.0 - ks) * r1;
        q.e = (ks + h1s) * r1;
        q.r2 = 1.0 / (1.0 + h1);
        q.g = h1 * q.r2;
        q.r3 = 1.0 / (1.0 + h1 * beta);
        q.hh = h1 * q.r3;
        return q;
    }
    __device__ __forceinline__ static void step(double* X, const Coef& q)
    {
        const double x = X[0], y = X[1], z = X[2];
        const double kx = q.k * x;
        const double z1 = fma(kx, y, q.ca * z);
        const double w = q.rho - z1;
        const double y1 = fma(kx, w, q.cb * y);
        const double x2 = fma(q.d, x, q.e * y1);
        const double y2 = fma(q.g * x2, w, q.r2 * y1);
        const double z2 = fma(q.hh * x2, y2, q.r3 * z1);
        X[0] = x2; X[1] = y2; X[2] = z2;
    }
};

// ---------------------------------------------------------------------------
// Chen and Lorenz in a rescaled state: 8 FP64 instructions per step (6 FMA,
// 2 MUL; 14 flops) when s = 1/2, 9 otherwise, instead of 14.
//
// Written out, both CD steps read (A = a or sigma, B = b or beta)
//   z1 = (1 - kB) z + k x y,  w = W0 - z1,  y1 = cy y + k x w,
//   x2 = r1 (1 - kA) x + r1 A h y1,  y2 = r2 (y1 + h1 x2 w),  z2 = r3 (z1 + h1 x2 y2),
// r1 = 1/(1 + h1 A), r3 = 1/(1 + h1 B); Chen: W0 = c - a, cy = 1 + k c,
// r2 = 1/(1 - h1 c); Lorenz: W0 = rho, cy = 1 - k, r2 = 1/(1 + h1).
// Measuring y and z, and the intermediates, in suitable units turns every
// parameter factor of the quadratic terms into 1: with ups = r1 A h, om = 1 - kB,
// the state is stored as (x, Y, Z) = (x, sy y, sz z), sy = ups cy, sz = om sy / k,
// and one step is
//   Z1 = fma(x, Y, Z) = (sy/k) z1;   W = fma(al, Z1, be) = ups k w;
//   Y1 = fma(x, W, Y) = (sy/cy) y1;  x2 = fma(rho, x, Y1);
//   q = c5 x2;  Y2 = ly fma(q, W, Y1) = sy y2;  Z2 = lz fma(q, Y2, Z1) = sz z2,
// al = -(ups k)(k/sy), be = (ups k) W0, rho = r1 (1 - kA), c5 = h1/k, ly = cy r2,
// lz = om r3.  The two multiplications by ly and lz are the per-step decay of
// the linear parts of y and z, which no constant change of units removes; c5 is
// exactly 1 when k = h1 (s = 1/2), and the UNIT form then skips that product --
// a multiplication by 1.0 is exact, so both forms give identical results and the
// oracle always multiplies.  The mathematics is the CD step; the rounding is this
// form's own, and the oracle evaluates the same operations.  The form needs
// A != 0 and k != 0 (else sy or sz is 0 or undefined) and factors well inside
// the double range; a job whose every point qualifies runs it (capi.cu:
// scaled_step_ok), others the 14-instruction form.  Outputs read y and z as
// Y * (1/sy), Z * (1/sz) (phys_comp); LLE and Lyapunov-spectrum distances are
// taken in physical units.
template <bool LORENZ, bool UNIT>
struct QuadScaled {
    static constexpr int DIM = 3;
    static constexpr int NV = 4;
    static constexpr int FLOPS = UNIT ? 14 : 15;
    static constexpr bool SCALED = true;
    struct Coef { double al, be, rho, c5, ly, lz, sy, iy, sz, iz; };
    __host__ __device__ static Coef prep(const double* v, double h)
    {
        Coef q;
        const double s = v[0];
        const double k = h * s;
        const double h1 = h * (1.0 - s);
        const double A = v[1];
        const double B = LORENZ ? v[3] : v[2];
        const double W0 = LORENZ ? v[2] : v[3] - v[1];
        const double cy = LORENZ ? 1.0 - k : 1.0 + k * v[3];
        const double r2 = LORENZ ? 1.0 / (1.0 + h1) : 1.0 / (1.0 - h1 * v[3]);
        const double r1 = 1.0 / (1.0 + h1 * A);
        const double r3 = 1.0 / (1.0 + h1 * B);
        const double ups = (r1 * A) * h;
        const double om = 1.0 - k * B;
        q.sy = ups * cy;
        q.sz = (om * q.sy) / k;
        const double uk = ups * k;
        q.al = -(uk * (k / q.sy));
        q.be = uk * W0;
        q.rho = r1 * (1.0 - k * A);
        q.c5 = h1 / k;
        q.ly = cy * r2;
        q.lz = om * r3;
        q.iy = 1.0 / q.sy;
        q.iz = 1.0 / q.sz;
        return q;
    }
    __device__ __forceinline__ static void step(double* X, const Coef& q)
    {
        const double x = X[0], y = X[1], z = X[2];
        const double z1 = fma(x, y, z);
        const double w = fma(q.al, z1, q.be);
        const double y1 = fma(x, w, y);
        const double x2 = fma(q.rho, x, y1);
        const double qq = UNIT ? x2 : q.c5 * x2;
        const double y2 = q.ly * fma(qq, w, y1);
        const double z2 = q.lz * fma(qq, y2, z1);
        X[0] = x2; X[1] = y2; X[2] = z2;
    }
};
using ChenScaled = QuadScaled<false, false>;
using LorenzScaled = QuadScaled<true, false>;
using ChenScaledU = QuadScaled<false, true>;    // s = 1/2
using LorenzScaledU = QuadScaled<true, true>;  // s = 1/2

// ---------------------------------------------------------------------------
// Physical view of a stored state.  Systems with SCALED keep component 1 in
// units of Coef::sy and component 2 in units of Coef::sz; component 0, and every
// component of the other systems, is stored in physical units (the conversions
// compile away).

// Component i (a compile-time index after unrolling) of a state difference or
// value, from stored to physical units.
template <class S>
__host__ __device__ __forceinline__ double phys_comp(double v, int i, const typename S::Coef& c)
{
    if constexpr (S::SCALED) return i == 1 ? v * c.iy : (i == 2 ? v * c.iz : v);
    else return v;
}

// A physical quantity (initial value or perturbation) of component i in stored units.
template <class S>
__host__ __device__ __forceinline__ double stored_comp(double v, int i, const typename S::Coef& c)
{
    if constexpr (S::SCALED) return i == 1 ? v * c.sy : (i == 2 ? v * c.sz : v);
    else return v;
}

// A point's physical initial state converted to stored units, in place.
template <class S>
__host__ __device__ __forceinline__ void to_stored(double* x, const typename S::Coef& c)
{
    if constexpr (S::SCALED) {
        x[1] = x[1] * c.sy;
        x[2] = x[2] * c.sz;
    }
}

}  // namespace cbf
