// The surrogate network: 4 inputs -> fixed Fourier encoding (128) -> 256 -> 256
// -> 256 -> 17 (SiLU), BF16 operands, FP32 accumulation, trained and evaluated
// by this file's kernels.
//
// The 4 inputs are the system code, the two swept parameters mapped to [-1, 1]
// and the third parameter / 10.  The encoding, which is not trained, keeps them
// and adds sin(2 pi p_k), cos(2 pi p_k) of p_k = b_k0 x1 + b_k1 x2 for 62 fixed
// frequencies b_k: on raw coordinates a small MLP learns the smooth part of a
// regime map first and cannot resolve its fine structure, so it lost to the
// nearest coarse label; with the encoding it beats it.
//
// Output 0 is the (normalised) LLE, outputs 1..16 the logits of the 16-way
// peak-count regime class.  Parameters live as FP32 masters (Adam state next to
// them) plus BF16 copies that feed the tensor cores.  Every matrix product --
// forward, input gradients, weight gradients, the prediction of explicit
// feature rows -- runs on the 5th-generation tensor cores through one kernel
// (mlp_gemm_tc.cuh: TMA-staged operands, tcgen05.mma into tensor memory, fused
// epilogues); prediction over a whole grid runs as one fused tcgen05 kernel
// (mlp_tc.cuh).  A training step (minibatch gather, 4 forward products, loss,
// 7 backward products with their split-K and bias reductions, Adam) is captured
// once as a CUDA graph and replayed.
#include <cuda.h>
#include <cuda_bf16.h>
#include <math.h>
#include <string.h>

#include <algorithm>
#include <mutex>
#include <vector>

#include "mlp.cuh"

namespace cbf {

// kRaw network inputs, kFreq Fourier frequencies, kIn first-layer inputs
constexpr int kRaw = 4, kFreq = 62, kIn = kRaw + 2 * kFreq, kHid = 256, kOut = 17, kClasses = 16;

namespace {

typedef __nv_bfloat16 bf16;

// Parameter layout of the flat FP32 buffer: W1[256x4] b1 W2[256x256] b2 W3 b3 W4[17x256] b4.
constexpr long long kW1 = 0, kB1 = kW1 + kHid * kIn;
constexpr long long kW2 = kB1 + kHid, kB2 = kW2 + kHid * kHid;
constexpr long long kW3 = kB2 + kHid, kB3 = kW3 + kHid * kHid;
constexpr long long kW4 = kB3 + kHid, kB4 = kW4 + kOut * kHid;
constexpr long long kNumParams = kB4 + kOut;

// Tensor-core operand copies of the weights: seven 256 x 256 BF16 slots (row
// pitch 256), zero outside the weights: W1 (256 x 128), W2, W3,
// W4 (17 x 256, rows padded), W2^T, W3^T, W4^T (256 x 17, K padded to 32).
constexpr long long kSlot = (long long)kHid * kHid;
enum { kSlotW1 = 0, kSlotW2, kSlotW3, kSlotW4, kSlotW2T, kSlotW3T, kSlotW4T, kNumSlots };
constexpr int kXPitch = kIn;   // BF16 first-layer input rows
constexpr int kDOutPitch = 32;  // BF16 output-gradient rows: 17 values padded to K = 32
constexpr int kDOutTRows = 128; // rows of dOut^T (17 used): one full 128-row operand tile

// SiLU z * sigmoid(z) and its derivative.  The sigmoid's quotient uses the
// approximate reciprocal (__fdividef: a few ulp of FP32, far below the BF16
// rounding of every activation) instead of an IEEE division, whose correction
// steps were most of the epilogues' FP32 work; for 1 + e^-z beyond 2^126 it
// returns 0, the limit of z * sigmoid(z) there.
__device__ __forceinline__ uint32_t pack_bf16x2(float lo, float hi)
{
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t*>(&v);
}

// The encoding's frequencies (cycles per unit of the [-1, 1] axes): per value one
// xorshift64 word (state 0x5EED * 0x9E3779B97F4A7C15 + 1), b = (sum of its four
// low bytes - 510) / 16 -- an Irwin-Hall approximation of a normal distribution
// with standard deviation about 9, exact in FP32 (the oracle rebuilds the same
// table).  Measured on the 8192^2 Chen map (512^2 coarse labels + 65 536 random
// points): raw inputs 97.0 % class agreement, nearest coarse label 97.6 %,
// encoded inputs 98.2 %.
struct FreqTable {
    float b[kFreq][2];
};
constexpr FreqTable make_freqs()
{
    FreqTable t{};
    unsigned long long s = 0x5EEDull * 0x9E3779B97F4A7C15ull + 1ull;
    for (int k = 0; k < kFreq; ++k)
        for (int j = 0; j < 2; ++j) {
            s ^= s << 13;
            s ^= s >> 7;
            s ^= s << 17;
            int m = 0;
            for (int i = 0; i < 4; ++i) m += (int)((s >> (8 * i)) & 255ull);
            t.b[k][j] = (float)(m - 510) / 16.0f;
        }
    return t;
}
__constant__ FreqTable c_freq = make_freqs();

// Encoded first-layer inputs 8j .. 8j+7 of raw features x: e[0..3] = x, then
// e[4 + 2k] = sin(2 pi fs p_k), e[5 + 2k] = cos(2 pi fs p_k), p_k = fl(fl(b_k0 x1)
// + fl(b_k1 x2)), fs the network's frequency scale (a power of two, so 2 fs p_k
// is exact; sincospif: exact argument reduction).
__device__ __forceinline__ void encode8(const float (&x)[kRaw], int j, float fs, float (&e)[8])
{
#pragma unroll
    for (int i = 0; i < 8; i += 2) {
        const int f = 8 * j + i;
        if (f < kRaw) {
            e[i] = x[f];
            e[i + 1] = x[f + 1];
        } else {
            const int k = (f - kRaw) >> 1;
            const float p = __fadd_rn(__fmul_rn(c_freq.b[k][0], x[1]), __fmul_rn(c_freq.b[k][1], x[2]));
            sincospif((2.0f * fs) * p, &e[i], &e[i + 1]);
        }
    }
}

__device__ __forceinline__ float silu(float z) { return __fdividef(z, 1.0f + __expf(-z)); }
__device__ __forceinline__ float silu_grad(float z)
{
    const float s = __fdividef(1.0f, 1.0f + __expf(-z));
    return s * (1.0f + z * (1.0f - s));
}

// C[m*c_m + n*c_n] = sum over z of ws[z][m*N + n], slices added in order.
__global__ void splitk_reduce_kernel(const float* __restrict__ ws, int splits, int M, int N,
                                     float* __restrict__ C, long long c_m, long long c_n)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long MN = (long long)M * N;
    if (i >= MN) return;
    float acc = 0.f;
    for (int z = 0; z < splits; ++z) acc += ws[z * MN + i];
    const long long m = i / N, n = i % N;
    C[m * c_m + n * c_n] = acc;
}

// ---- element-wise kernels -------------------------------------------------

__device__ __forceinline__ unsigned long long mix64(unsigned long long z)
{
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// Encoded BF16 row r (x: its raw features) into xb (pitch kIn) and, if xT is
// given, column r of xT (pitch ldT).
__device__ __forceinline__ void put_encoded_row(const float (&x)[kRaw], long long r, float fs,
                                                bf16* __restrict__ xb, bf16* __restrict__ xT, long long ldT)
{
#pragma unroll 1
    for (int j = 0; j < kIn / 8; ++j) {
        float e[8];
        encode8(x, j, fs, e);
        reinterpret_cast<uint4*>(xb + r * kXPitch)[j] =
            make_uint4(pack_bf16x2(e[0], e[1]), pack_bf16x2(e[2], e[3]), pack_bf16x2(e[4], e[5]),
                       pack_bf16x2(e[6], e[7]));
        if (xT) {
#pragma unroll
            for (int i = 0; i < 8; ++i) xT[(8 * j + i) * ldT + r] = __float2bfloat16_rn(e[i]);
        }
    }
}

// Minibatch of B rows drawn uniformly (with replacement) from N, keyed by the
// device step counter so a replayed graph draws a new batch every step.  The
// encoded BF16 rows go to xb and, transposed, to xT (row f = input f, pitch
// ldT) for the first layer's weight gradient.
__global__ void gather_kernel(const float* __restrict__ X, const float* __restrict__ ylle,
                              const int* __restrict__ ycls, long long N, int B,
                              const unsigned long long* step, unsigned long long seed, float fs,
                              bf16* __restrict__ xb, bf16* __restrict__ xT, long long ldT, float* __restrict__ bl,
                              int* __restrict__ bc)
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= B) return;
    const unsigned long long h = mix64(seed ^ mix64(*step * 0x100000001B3ull + (unsigned long long)r));
    const long long i = (long long)(h % (unsigned long long)N);
    float x[kRaw];
#pragma unroll
    for (int f = 0; f < kRaw; ++f) x[f] = X[i * kRaw + f];
    put_encoded_row(x, r, fs, xb, xT, ldT);
    bl[r] = ylle[i];
    bc[r] = ycls[i];
}

// Encoded rows of n raw feature rows X [n x 4] (rows n <= r < rows: zeros).
__global__ void encode_rows_kernel(const float* __restrict__ X, long long n, long long rows, float fs,
                                   bf16* __restrict__ xb, bf16* __restrict__ xT, long long ldT)
{
    const long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= rows) return;
    if (r < n) {
        float x[kRaw];
#pragma unroll
        for (int f = 0; f < kRaw; ++f) x[f] = X[r * kRaw + f];
        put_encoded_row(x, r, fs, xb, xT, ldT);
    } else {
        const bf16 zero = __float2bfloat16_rn(0.0f);
        for (int f = 0; f < kIn; ++f) {
            xb[r * kXPitch + f] = zero;
            if (xT) xT[f * ldT + r] = zero;
        }
    }
}

// Loss: mean squared error on output 0 (normalised LLE) + cross-entropy of
// outputs 1..16; writes dLoss/dOut in FP32 (dOut, pitch 17, for the bias
// gradient), in BF16 (dOutB, pitch 32, columns 17..31 zero) and transposed in
// BF16 (dOutT, pitch ldT) for the products, and accumulates the loss.  Rows
// n <= r < rows (the rest of the last 128-row tile) write zero gradients.
__global__ void loss_kernel(const float* __restrict__ out, const float* __restrict__ yl,
                            const int* __restrict__ yc, int n, int rows, float wLle, float* __restrict__ dOut,
                            bf16* __restrict__ dOutB, bf16* __restrict__ dOutT, long long ldT,
                            float* __restrict__ lossAcc)
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= rows) return;
    const bf16 zero = __float2bfloat16_rn(0.0f);
    if (r >= n) {
        for (int c = 0; c < kDOutPitch; ++c) dOutB[(long long)r * kDOutPitch + c] = zero;
        for (int c = 0; c < kOut; ++c) dOutT[c * ldT + r] = zero;
        return;
    }
    const float* o = out + (long long)r * kOut;
    float d[kOut];
    const float invB = 1.0f / (float)n;
    const float e = o[0] - yl[r];
    d[0] = 2.0f * wLle * e * invB;
    float mx = o[1];
    for (int c = 1; c < kClasses; ++c) mx = fmaxf(mx, o[1 + c]);
    float sum = 0.f;
    for (int c = 0; c < kClasses; ++c) sum += __expf(o[1 + c] - mx);
    const int t = yc[r];
    float lossCe = 0.f;
    for (int c = 0; c < kClasses; ++c) {
        const float p = __expf(o[1 + c] - mx) / sum;
        d[1 + c] = (p - (c == t ? 1.0f : 0.0f)) * invB;
        if (c == t) lossCe = -logf(fmaxf(p, 1e-30f));
    }
    for (int c = 0; c < kOut; ++c) {
        const bf16 v = __float2bfloat16_rn(d[c]);
        dOut[(long long)r * kOut + c] = d[c];
        dOutB[(long long)r * kDOutPitch + c] = v;
        dOutT[c * ldT + r] = v;
    }
    for (int c = kOut; c < kDOutPitch; ++c) dOutB[(long long)r * kDOutPitch + c] = zero;
    atomicAdd(lossAcc, (wLle * e * e + lossCe) * invB);
}

// db[n] = sum over rows of G[m*ld + n]: a 32x32 block per 32 columns, thread
// row ty sums rows ty, ty+32, ..., then the 32 partials are added in order.
__global__ void __launch_bounds__(1024) colsum_kernel(const float* __restrict__ G, int M, int N, long long ld,
                                                     float* __restrict__ db)
{
    __shared__ float part[32][33];
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const int n = blockIdx.x * 32 + tx;
    float s = 0.f;
    if (n < N)
        for (int m = ty; m < M; m += 32) s += G[m * ld + n];
    part[ty][tx] = s;
    __syncthreads();
    if (ty == 0 && n < N) {
        float t = 0.f;
        for (int r = 0; r < 32; ++r) t += part[r][tx];
        db[n] = t;
    }
}

cudaError_t colsum(const float* G, int M, int N, long long ld, float* db, cudaStream_t s)
{
    colsum_kernel<<<(N + 31) / 32, 1024, 0, s>>>(G, M, N, ld, db);
    note_launch();
    return cudaGetLastError();
}

// BF16 weight w = parameter i into its tensor-core operand slots (and, for W2,
// W3 and W4, the transposed slot).
__device__ __forceinline__ void put_weight(bf16* __restrict__ tw, long long i, bf16 w)
{
    if (i < kB1) {
        tw[kSlotW1 * kSlot + (i / kIn) * kHid + i % kIn] = w;
    } else if (i >= kW2 && i < kB2) {
        const long long j = i - kW2;
        tw[kSlotW2 * kSlot + j] = w;
        tw[kSlotW2T * kSlot + (j % kHid) * kHid + j / kHid] = w;
    } else if (i >= kW3 && i < kB3) {
        const long long j = i - kW3;
        tw[kSlotW3 * kSlot + j] = w;
        tw[kSlotW3T * kSlot + (j % kHid) * kHid + j / kHid] = w;
    } else if (i >= kW4 && i < kB4) {
        const long long j = i - kW4;
        tw[kSlotW4 * kSlot + j] = w;
        tw[kSlotW4T * kSlot + (j % kHid) * kHid + j / kHid] = w;
    }
}

// Adam on the flat FP32 parameters; refreshes the BF16 weight copies (flat and
// tensor-core operand slots).
__global__ void adam_kernel(float* __restrict__ p, const float* __restrict__ gr, float* __restrict__ m1,
                            float* __restrict__ m2, bf16* __restrict__ pb, bf16* __restrict__ tw, long long n,
                            float lr0, int horizon, float b1, float b2, float eps, const unsigned long long* step)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const float t = (float)(*step + 1);
    // cosine decay from lr0 to lr0/20 over `horizon` steps (0: constant)
    float lr = lr0;
    if (horizon > 0) {
        const float u = fminf((float)*step / (float)horizon, 1.0f);
        lr = lr0 * (0.05f + 0.95f * 0.5f * (1.0f + cospif(u)));
    }
    if (i < n) {
        const float gi = gr[i];
        const float a = b1 * m1[i] + (1.f - b1) * gi;
        const float v = b2 * m2[i] + (1.f - b2) * gi * gi;
        m1[i] = a;
        m2[i] = v;
        const float ah = a / (1.f - powf(b1, t));
        const float vh = v / (1.f - powf(b2, t));
        const float w = p[i] - lr * ah / (sqrtf(vh) + eps);
        p[i] = w;
        const bf16 wb = __float2bfloat16_rn(w);
        pb[i] = wb;
        put_weight(tw, i, wb);
    }
}

// BF16 copies (flat and operand slots) of the FP32 parameters.
__global__ void expand_params_kernel(const float* __restrict__ p, bf16* __restrict__ pb, bf16* __restrict__ tw,
                                     long long n)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const bf16 wb = __float2bfloat16_rn(p[i]);
    pb[i] = wb;
    put_weight(tw, i, wb);
}

__global__ void bump_kernel(unsigned long long* step) { *step += 1; }

// Prediction head: LLE (de-normalised), argmax class, softmax confidence.
__global__ void head_kernel(const float* __restrict__ out, long long n, float lleMean, float lleStd,
                            float* __restrict__ lle, int* __restrict__ cls, float* __restrict__ conf)
{
    const long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    const float* o = out + r * kOut;
    int best = 0;
    float mx = o[1];
    for (int c = 1; c < kClasses; ++c)
        if (o[1 + c] > mx) {
            mx = o[1 + c];
            best = c;
        }
    float sum = 0.f;
    for (int c = 0; c < kClasses; ++c) sum += __expf(o[1 + c] - mx);
    if (lle) lle[r] = o[0] * lleStd + lleMean;
    if (cls) cls[r] = best;
    if (conf) conf[r] = 1.0f / sum;
}

__device__ __forceinline__ void point_features(const FeatureSpec& f, long long g, float (&x)[kRaw])
{
    const bool exact = f.J.exactGrid != 0;
    const double p0 = grid_value(g, f.J.nPts, f.J.ranges[0], f.J.ranges[1], 0, exact);
    const double p1 = grid_value(g, f.J.nPts, f.J.ranges[2], f.J.ranges[3], 1, exact);
    x[0] = f.sys;
    x[1] = ((float)p0 - f.lo0) * f.inv0 - 1.0f;
    x[2] = ((float)p1 - f.lo1) * f.inv1 - 1.0f;
    x[3] = f.third;
}

__global__ void features_kernel(const FeatureSpec f, const long long* __restrict__ idx, long long n,
                                float* __restrict__ X)
{
    const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    float x[kRaw];
    point_features(f, idx[k], x);
#pragma unroll
    for (int i = 0; i < kRaw; ++i) X[k * kRaw + i] = x[i];
}

#include "mlp_tc.cuh"
#include "mlp_gemm_tc.cuh"

template <class F>
cudaError_t launch1d(long long n, cudaStream_t s, F f)
{
    if (n <= 0) return cudaSuccess;
    const int t = 256;
    const long long b = (n + t - 1) / t;
    f((unsigned)b, t);
    note_launch();
    return cudaGetLastError();
}

}  // namespace

// ---------------------------------------------------------------------------

// Tensor maps of every operand the products read (fixed buffers, built once).
struct TcMaps {
    // A operands (128-row tiles): the training batch ...
    CUtensorMap aX, aH1, aH2, aH3, aDOut, aDZ3, aDZ2, aDOutT, aDZ3T, aDZ2T, aDZ1T;
    // ... and the prediction workspace
    CUtensorMap pX, pH1, pH2, pH3;
    // B operands: weights, transposed weights, transposed activations
    CUtensorMap bW1, bW2, bW3, bW4, bW4T, bW3T, bW2T, bH3T, bH2T, bH1T, bXT;
};

struct Mlp {
    int B = 0;               // training batch
    long long Ba = 0;        // rows of every batch buffer: B rounded up to 128, at least 4096
    unsigned long long seed = 0;
    float encScale = 1.0f;    // frequency scale of the input encoding (a power of two)
    float* params = nullptr;  // FP32 masters (kNumParams)
    float* grads = nullptr;
    float* m1 = nullptr;
    float* m2 = nullptr;
    bf16* pb = nullptr;       // BF16 copies, flat layout (packed for the grid prediction)
    bf16* tw = nullptr;       // BF16 copies in the tensor-core operand slots
    // batch buffers (row-major; "T": transposed, pitch Ba)
    bf16 *xb = nullptr, *xT = nullptr;
    float* xraw = nullptr;     // raw feature rows of cbf_mlp_forward_backward
    float* yl = nullptr;
    int* yc = nullptr;
    float *z1 = nullptr, *z2 = nullptr, *z3 = nullptr;
    bf16 *h1 = nullptr, *h2 = nullptr, *h3 = nullptr;
    bf16 *h1T = nullptr, *h2T = nullptr, *h3T = nullptr;
    float* out = nullptr;
    float* dOut = nullptr;
    bf16 *dOutB = nullptr, *dOutT = nullptr;
    float* dzf = nullptr;     // FP32 dZ3, dZ2, dZ1 (for the bias gradients), Ba x 256 each
    bf16 *dz3 = nullptr, *dz2 = nullptr;
    bf16 *dz3T = nullptr, *dz2T = nullptr, *dz1T = nullptr;
    float* loss = nullptr;
    float* ws = nullptr;      // split-K partials, one region per weight gradient
    int* gemmErr = nullptr;   // set by a product whose bounded wait ran out
    cudaStream_t side = nullptr;  // weight gradients beside the input-gradient chain
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    unsigned long long* step = nullptr;
    TcMaps* maps = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    const float* gX = nullptr;  // training set the graph was captured for
    long long gN = 0;
    float gLr = 0.f;
    int gHorizon = 0;
    float gW = 0.f;
    float gScale = 0.f;
    unsigned long long gSeed = 0;
    // prediction workspace (rows per chunk = kPredRows), no pre-activations
    bf16 *pxb = nullptr, *ph1 = nullptr, *ph2 = nullptr, *ph3 = nullptr;
    float* pout = nullptr;
    // grid prediction on tcgen05: weights in the shared-memory operand layout
    unsigned char* wpack = nullptr;
    int* tcErr = nullptr;
};

constexpr int kPredRows = 262144;

namespace {

template <class T>
cudaError_t alloc_zero(T** p, long long n)
{
    const size_t bytes = (size_t)(n > 0 ? n : 1) * sizeof(T);
    cudaError_t e = cudaMalloc((void**)p, bytes);
    if (e == cudaSuccess) e = cudaMemset(*p, 0, bytes);
    return e;
}

cudaError_t pred_workspace(Mlp* m)
{
    if (m->pxb) return cudaSuccess;
    cudaError_t e = alloc_zero(&m->pxb, (long long)kPredRows * kXPitch);
    if (e == cudaSuccess) e = alloc_zero(&m->ph1, (long long)kPredRows * kHid);
    if (e == cudaSuccess) e = alloc_zero(&m->ph2, (long long)kPredRows * kHid);
    if (e == cudaSuccess) e = alloc_zero(&m->ph3, (long long)kPredRows * kHid);
    if (e == cudaSuccess) e = alloc_zero(&m->pout, (long long)kPredRows * kOut);
    TcMaps& mp = *m->maps;
    if (e == cudaSuccess) e = operand_map(&mp.pX, m->pxb, kPredRows, kXPitch, kXPitch, kGtM, 64);
    if (e == cudaSuccess) e = operand_map(&mp.pH1, m->ph1, kPredRows, kHid, kHid, kGtM, 64);
    if (e == cudaSuccess) e = operand_map(&mp.pH2, m->ph2, kPredRows, kHid, kHid, kGtM, 64);
    if (e == cudaSuccess) e = operand_map(&mp.pH3, m->ph3, kPredRows, kHid, kHid, kGtM, 64);
    return e;
}

// Buffers of one forward pass: A-operand maps of the input and hidden
// activations, and where the pass writes (Z and the transposes may be null).
struct FwdBufs {
    const CUtensorMap *aX, *aH1, *aH2, *aH3;
    float *z1, *z2, *z3;
    bf16 *h1, *h2, *h3;
    bf16 *h1T, *h2T, *h3T;
    long long ldT;
    float* out;
};

FwdBufs train_bufs(Mlp& m)
{
    const TcMaps& mp = *m.maps;
    return FwdBufs{&mp.aX, &mp.aH1, &mp.aH2, &mp.aH3, m.z1, m.z2, m.z3, m.h1, m.h2, m.h3,
                   m.h1T, m.h2T, m.h3T, m.Ba, m.out};
}

FwdBufs pred_bufs(Mlp& m)
{
    const TcMaps& mp = *m.maps;
    return FwdBufs{&mp.pX, &mp.pH1, &mp.pH2, &mp.pH3, nullptr, nullptr, nullptr, m.ph1, m.ph2, m.ph3,
                   nullptr, nullptr, nullptr, 0, m.pout};
}

// Forward on n rows whose BF16 inputs are in the buffer behind f.aX.
cudaError_t forward(Mlp& m, int n, const FwdBufs& f, cudaStream_t s)
{
    const TcMaps& mp = *m.maps;
    cudaError_t e;
    TcGemm g = tc_gemm(kEpiHidden, m.gemmErr);
    g.M = n; g.N = kHid; g.BN = 128; g.Mv = n; g.Nv = kHid;
    g.K = kIn; g.KC = 64; g.kSlice = kIn;
    g.bias = m.params + kB1; g.Z = f.z1; g.ldZ = kHid; g.Hb = f.h1; g.ldh = kHid; g.HT = f.h1T; g.ldht = f.ldT;
    if ((e = gemm_tc(*f.aX, mp.bW1, g, s)) != cudaSuccess) return e;
    g.K = kHid; g.KC = 64; g.kSlice = kHid;
    g.bias = m.params + kB2; g.Z = f.z2; g.Hb = f.h2; g.HT = f.h2T;
    if ((e = gemm_tc(*f.aH1, mp.bW2, g, s)) != cudaSuccess) return e;
    g.bias = m.params + kB3; g.Z = f.z3; g.Hb = f.h3; g.HT = f.h3T;
    if ((e = gemm_tc(*f.aH2, mp.bW3, g, s)) != cudaSuccess) return e;
    g = tc_gemm(kEpiOut, m.gemmErr);
    g.M = n; g.N = 32; g.BN = 32; g.Mv = n; g.Nv = kOut;
    g.K = kHid; g.KC = 64; g.kSlice = kHid;
    g.bias = m.params + kB4; g.C = f.out; g.ldc = kOut;
    return gemm_tc(*f.aH3, mp.bW4, g, s);
}

// K slices of the weight-gradient products (K = the batch rows padded to 64):
// 256 rows each, wider when that would exceed kMaxSplit slices.
constexpr int kMaxSplit = 16;
int wgrad_slice(int K)
{
    int sl = 256;
    while ((K + sl - 1) / sl > kMaxSplit) sl += 64;
    return sl;
}

// Backward from dOut (m.dOut FP32, m.dOutB and m.dOutT BF16) to m.grads.  The
// input gradients dZ3 -> dZ2 -> dZ1 form the chain; each layer's weight and bias
// gradients need only that layer's dZ, so with a side stream they run beside the
// chain (each in its own split-K and FP32 dZ buffers) and join it at the end.
cudaError_t backward(Mlp& m, int n, cudaStream_t s, cudaStream_t side)
{
    const TcMaps& mp = *m.maps;
    float* G = m.grads;
    cudaError_t e;
    const int Kb = (n + 63) / 64 * 64;
    const long long wsLayer = (long long)kMaxSplit * kHid * kHid;
    const long long dzLayer = m.Ba * kHid;
    cudaStream_t sw = side ? side : s;
    // the side stream continues once the chain has produced the next dZ
    auto fork = [&](int i) -> cudaError_t {
        if (!side) return cudaSuccess;
        cudaError_t r = cudaEventRecord(m.ev[i], s);
        return r == cudaSuccess ? cudaStreamWaitEvent(side, m.ev[i], 0) : r;
    };
    TcGemm w = tc_gemm(kEpiWgrad, m.gemmErr);  // dW = dZ^T H_prev over the batch
    w.K = Kb; w.KC = 64; w.kSlice = wgrad_slice(Kb);
    TcGemm d = tc_gemm(kEpiDgrad, m.gemmErr);  // dZ_prev = (dZ W) * silu'(Z_prev)
    d.M = n; d.N = kHid; d.BN = 128; d.Mv = n; d.Nv = kHid;
    d.ldzp = kHid; d.ldc = kHid; d.ldh = kHid; d.ldht = m.Ba;

    // layer 4: dW4 = dOut^T H3, db4 = colsum(dOut) beside dZ3 = (dOut W4) * silu'(Z3)
    if ((e = fork(0)) != cudaSuccess) return e;
    TcGemm g = w;
    g.M = kOut; g.N = kHid; g.BN = 128; g.Mv = kOut; g.Nv = kHid; g.C = G + kW4; g.ldc = kHid; g.ws = m.ws;
    if ((e = gemm_tc(mp.aDOutT, mp.bH3T, g, sw)) != cudaSuccess) return e;
    if ((e = colsum(m.dOut, n, kOut, kOut, G + kB4, sw)) != cudaSuccess) return e;
    g = d;
    g.K = kDOutPitch; g.KC = 32; g.kSlice = kDOutPitch; g.zp = m.z3; g.C = m.dzf; g.Hb = m.dz3; g.HT = m.dz3T;
    if ((e = gemm_tc(mp.aDOut, mp.bW4T, g, s)) != cudaSuccess) return e;
    // layers 3, 2: dW = dZ^T H_prev, db = colsum(dZ) beside dZ_prev
    const CUtensorMap* aDzT[2] = {&mp.aDZ3T, &mp.aDZ2T};
    const CUtensorMap* bHT[2] = {&mp.bH2T, &mp.bH1T};
    const CUtensorMap* aDz[2] = {&mp.aDZ3, &mp.aDZ2};
    const CUtensorMap* bWT[2] = {&mp.bW3T, &mp.bW2T};
    const long long wOff[2] = {kW3, kW2}, bOff[2] = {kB3, kB2};
    const float* zPrev[2] = {m.z2, m.z1};
    bf16* dzPrev[2] = {m.dz2, nullptr};
    bf16* dzPrevT[2] = {m.dz2T, m.dz1T};
    for (int l = 0; l < 2; ++l) {
        if ((e = fork(1 + l)) != cudaSuccess) return e;
        g = w;
        g.M = kHid; g.N = kHid; g.BN = 128; g.Mv = kHid; g.Nv = kHid; g.C = G + wOff[l]; g.ldc = kHid;
        g.ws = m.ws + (1 + l) * wsLayer;
        if ((e = gemm_tc(*aDzT[l], *bHT[l], g, sw)) != cudaSuccess) return e;
        if ((e = colsum(m.dzf + l * dzLayer, n, kHid, kHid, G + bOff[l], sw)) != cudaSuccess) return e;
        g = d;
        g.K = kHid; g.KC = 64; g.kSlice = kHid; g.zp = zPrev[l]; g.C = m.dzf + (l + 1) * dzLayer;
        g.Hb = dzPrev[l]; g.HT = dzPrevT[l];
        if ((e = gemm_tc(*aDz[l], *bWT[l], g, s)) != cudaSuccess) return e;
    }
    // layer 1: dW1 = dZ1^T X, db1 (on the chain), then join the side stream
    g = w;
    g.M = kHid; g.N = kIn; g.BN = 128; g.Mv = kHid; g.Nv = kIn; g.C = G + kW1; g.ldc = kIn;
    g.ws = m.ws + 3 * wsLayer;
    if ((e = gemm_tc(mp.aDZ1T, mp.bXT, g, s)) != cudaSuccess) return e;
    if ((e = colsum(m.dzf + 2 * dzLayer, n, kHid, kHid, G + kB1, s)) != cudaSuccess) return e;
    if (side) {
        if ((e = cudaEventRecord(m.ev[3], side)) != cudaSuccess) return e;
        if ((e = cudaStreamWaitEvent(s, m.ev[3], 0)) != cudaSuccess) return e;
    }
    return cudaSuccess;
}

// Reads and clears the products' error flag (call after a synchronisation).
cudaError_t gemm_status(Mlp& m)
{
    int h = 0;
    cudaError_t e = cudaMemcpy(&h, m.gemmErr, sizeof(int), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && h) {
        cudaMemset(m.gemmErr, 0, sizeof(int));
        e = cudaErrorLaunchTimeout;
    }
    return e;
}

}  // namespace

}  // namespace cbf

using namespace cbf;

struct cbf_mlp : Mlp {};

namespace {

cbf_status mlp_alloc(cbf_mlp* m, int B)
{
    cudaError_t e = cudaSuccess;
    m->B = B;
    const long long Ba = std::max<long long>(4096, ((long long)B + kGtM - 1) / kGtM * kGtM);
    m->Ba = Ba;
#define A_(ptr, n) if (e == cudaSuccess) e = alloc_zero(&m->ptr, (n))
    A_(params, kNumParams); A_(grads, kNumParams); A_(m1, kNumParams); A_(m2, kNumParams);
    A_(pb, kNumParams); A_(tw, kNumSlots * kSlot);
    A_(xb, Ba * kXPitch); A_(xT, kXPitch * Ba); A_(xraw, Ba * kRaw); A_(yl, Ba); A_(yc, Ba);
    A_(z1, Ba * kHid); A_(z2, Ba * kHid); A_(z3, Ba * kHid);
    A_(h1, Ba * kHid); A_(h2, Ba * kHid); A_(h3, Ba * kHid);
    A_(h1T, kHid * Ba); A_(h2T, kHid * Ba); A_(h3T, kHid * Ba);
    A_(out, Ba * kOut); A_(dOut, Ba * kOut); A_(dOutB, Ba * kDOutPitch); A_(dOutT, kDOutTRows * Ba);
    A_(dzf, 3 * Ba * kHid); A_(dz3, Ba * kHid); A_(dz2, Ba * kHid);
    A_(dz3T, kHid * Ba); A_(dz2T, kHid * Ba); A_(dz1T, kHid * Ba);
    A_(loss, 1); A_(step, 1); A_(gemmErr, 1);
    A_(ws, 4ll * kMaxSplit * kHid * kHid);
#undef A_
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&m->side, cudaStreamNonBlocking);
    for (int i = 0; i < 4 && e == cudaSuccess; ++i) e = cudaEventCreateWithFlags(&m->ev[i], cudaEventDisableTiming);
    if (e != cudaSuccess) return report_cuda_error(e, "surrogate network buffers");
    m->maps = new TcMaps();
    TcMaps& mp = *m->maps;
    const auto slot = [&](int k) { return m->tw + k * kSlot; };
#define M_(map, p, R, C, ld, rows, kc) if (e == cudaSuccess) e = operand_map(&mp.map, p, R, C, ld, rows, kc)
    M_(aX, m->xb, Ba, kXPitch, kXPitch, kGtM, 64);
    M_(aH1, m->h1, Ba, kHid, kHid, kGtM, 64);
    M_(aH2, m->h2, Ba, kHid, kHid, kGtM, 64);
    M_(aH3, m->h3, Ba, kHid, kHid, kGtM, 64);
    M_(aDOut, m->dOutB, Ba, kDOutPitch, kDOutPitch, kGtM, 32);
    M_(aDZ3, m->dz3, Ba, kHid, kHid, kGtM, 64);
    M_(aDZ2, m->dz2, Ba, kHid, kHid, kGtM, 64);
    M_(aDOutT, m->dOutT, kDOutTRows, Ba, Ba, kGtM, 64);
    M_(aDZ3T, m->dz3T, kHid, Ba, Ba, kGtM, 64);
    M_(aDZ2T, m->dz2T, kHid, Ba, Ba, kGtM, 64);
    M_(aDZ1T, m->dz1T, kHid, Ba, Ba, kGtM, 64);
    M_(bW1, slot(kSlotW1), kHid, kHid, kHid, 128, 64);
    M_(bW2, slot(kSlotW2), kHid, kHid, kHid, 128, 64);
    M_(bW3, slot(kSlotW3), kHid, kHid, kHid, 128, 64);
    M_(bW4, slot(kSlotW4), kHid, kHid, kHid, 32, 64);
    M_(bW4T, slot(kSlotW4T), kHid, kHid, kHid, 128, 32);
    M_(bW3T, slot(kSlotW3T), kHid, kHid, kHid, 128, 64);
    M_(bW2T, slot(kSlotW2T), kHid, kHid, kHid, 128, 64);
    M_(bH3T, m->h3T, kHid, Ba, Ba, 128, 64);
    M_(bH2T, m->h2T, kHid, Ba, Ba, 128, 64);
    M_(bH1T, m->h1T, kHid, Ba, Ba, 128, 64);
    M_(bXT, m->xT, kXPitch, Ba, Ba, 128, 64);
#undef M_
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(gemm_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGtMaxSmem);
    if (e != cudaSuccess) return report_cuda_error(e, "surrogate network tensor maps");
    return CBF_OK;
}

void mlp_free(cbf_mlp* m)
{
    if (m->exec) cudaGraphExecDestroy(m->exec);
    if (m->graph) cudaGraphDestroy(m->graph);
    void* ptrs[] = {m->params, m->grads, m->m1, m->m2, m->pb, m->tw, m->xb, m->xT, m->xraw, m->yl, m->yc, m->z1,
                    m->z2, m->z3, m->h1, m->h2, m->h3, m->h1T, m->h2T, m->h3T, m->out, m->dOut, m->dOutB,
                    m->dOutT, m->dzf, m->dz3, m->dz2, m->dz3T, m->dz2T, m->dz1T, m->loss, m->ws, m->gemmErr,
                    m->step, m->pxb, m->ph1, m->ph2, m->ph3, m->pout, m->wpack, m->tcErr};
    for (void* p : ptrs) cudaFree(p);
    for (cudaEvent_t ev : m->ev)
        if (ev) cudaEventDestroy(ev);
    if (m->side) cudaStreamDestroy(m->side);
    delete m->maps;
    m->maps = nullptr;
}

// He-style uniform init from a fixed seed (host side, deterministic).
void init_params(std::vector<float>& p, unsigned long long seed)
{
    p.assign(kNumParams, 0.f);
    unsigned long long st = seed * 0x9E3779B97F4A7C15ull + 1;
    auto rnd = [&]() {
        st ^= st << 13;
        st ^= st >> 7;
        st ^= st << 17;
        return (double)(st >> 11) * (1.0 / 9007199254740992.0) * 2.0 - 1.0;
    };
    auto fill = [&](long long off, long long cnt, int fanIn) {
        const double bound = sqrt(6.0 / fanIn);
        for (long long i = 0; i < cnt; ++i) p[off + i] = (float)(rnd() * bound);
    };
    fill(kW1, (long long)kHid * kIn, kIn);
    fill(kW2, (long long)kHid * kHid, kHid);
    fill(kW3, (long long)kHid * kHid, kHid);
    fill(kW4, (long long)kOut * kHid, kHid);
}

cbf_status upload_params(cbf_mlp* m, const float* host)
{
    cudaError_t e = cudaMemcpy(m->params, host, kNumParams * sizeof(float), cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = launch1d(kNumParams, 0, [&](unsigned b, int t) {
            expand_params_kernel<<<b, t>>>(m->params, m->pb, m->tw, kNumParams);
        });
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return report_cuda_error(e, "surrogate parameters");
    return CBF_OK;
}

}  // namespace

extern "C" {

int64_t cbf_mlp_num_params(void) { return kNumParams; }

cbf_status cbf_mlp_create(int32_t batch, uint64_t seed, cbf_mlp** out)
{
    if (!out || batch < 1 || batch > (1 << 20))
        return report_error(CBF_ERR_INVALID_ARG, "batch must be in [1, 2^20]");
    cbf_mlp* m = new cbf_mlp();
    m->seed = seed;
    cbf_status st = mlp_alloc(m, batch);
    if (st != CBF_OK) {
        mlp_free(m);
        delete m;
        return st;
    }
    std::vector<float> p;
    init_params(p, seed);
    st = upload_params(m, p.data());
    if (st != CBF_OK) {
        mlp_free(m);
        delete m;
        return st;
    }
    *out = m;
    return CBF_OK;
}

void cbf_mlp_destroy(cbf_mlp* m)
{
    if (!m) return;
    mlp_free(m);
    delete m;
}

cbf_status cbf_mlp_get_params(cbf_mlp* m, float* host, int64_t n)
{
    if (!m || !host || n != kNumParams) return report_error(CBF_ERR_INVALID_ARG, "bad parameter buffer");
    cudaError_t e = cudaMemcpy(host, m->params, kNumParams * sizeof(float), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return report_cuda_error(e, "read parameters");
    return CBF_OK;
}

cbf_status cbf_mlp_set_params(cbf_mlp* m, const float* host, int64_t n)
{
    if (!m || !host || n != kNumParams) return report_error(CBF_ERR_INVALID_ARG, "bad parameter buffer");
    cudaMemset(m->m1, 0, kNumParams * sizeof(float));
    cudaMemset(m->m2, 0, kNumParams * sizeof(float));
    cudaMemset(m->step, 0, sizeof(unsigned long long));
    return upload_params(m, host);
}

// The encoding's frequency table (kFreq x 2 floats, row-major), as the kernels
// hold it in constant memory; n must be kFreq * 2.
cbf_status cbf_mlp_encoding_frequencies(float* out, int32_t n)
{
    if (!out || n != kFreq * 2) return report_error(CBF_ERR_INVALID_ARG, "the table holds 124 floats");
    constexpr FreqTable tab = make_freqs();
    for (int k = 0; k < kFreq; ++k) {
        out[2 * k] = tab.b[k][0];
        out[2 * k + 1] = tab.b[k][1];
    }
    return CBF_OK;
}

// Frequency scale of the input encoding: a power of two in [2^-8, 16].
cbf_status cbf_mlp_set_encoding_scale(cbf_mlp* m, float scale)
{
    int ex = 0;
    if (!m || !(scale >= 0x1p-8f && scale <= 16.0f) || frexpf(scale, &ex) != 0.5f)
        return report_error(CBF_ERR_INVALID_ARG, "encoding scale must be a power of two in [2^-8, 16]");
    m->encScale = scale;
    return CBF_OK;
}

// One forward + backward on host data (n <= batch rows); for gradient checks.
cbf_status cbf_mlp_forward_backward(cbf_mlp* m, const float* hx, const float* hyl, const int32_t* hyc,
                                    int32_t n, float wLle, float* hloss, float* hgrads, float* hout)
{
    if (!m || !hx || !hyl || !hyc || n < 1 || n > m->B)
        return report_error(CBF_ERR_INVALID_ARG, "bad batch");
    // encoded BF16 input rows and their transpose, zero for the rest of the last tile
    const int rows = (n + kGtM - 1) / kGtM * kGtM;
    cudaError_t e = cudaMemcpy(m->xraw, hx, (size_t)n * kRaw * sizeof(float), cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = launch1d(rows, 0, [&](unsigned b, int t) {
            encode_rows_kernel<<<b, t>>>(m->xraw, n, rows, m->encScale, m->xb, m->xT, m->Ba);
        });
    if (e == cudaSuccess) e = cudaMemcpy(m->yl, hyl, (size_t)n * sizeof(float), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(m->yc, hyc, (size_t)n * sizeof(int), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(m->loss, 0, sizeof(float));
    if (e == cudaSuccess) e = forward(*m, n, train_bufs(*m), 0);
    if (e == cudaSuccess)
        e = launch1d(rows, 0, [&](unsigned b, int t) {
            loss_kernel<<<b, t>>>(m->out, m->yl, m->yc, n, rows, wLle, m->dOut, m->dOutB, m->dOutT, m->Ba,
                                  m->loss);
        });
    if (e == cudaSuccess) e = backward(*m, n, 0, nullptr);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = gemm_status(*m);
    if (e == cudaSuccess && hloss) e = cudaMemcpy(hloss, m->loss, sizeof(float), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && hgrads)
        e = cudaMemcpy(hgrads, m->grads, kNumParams * sizeof(float), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && hout)
        e = cudaMemcpy(hout, m->out, (size_t)n * kOut * sizeof(float), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return report_cuda_error(e, "forward/backward");
    return CBF_OK;
}

// `steps` Adam steps on minibatches drawn from the device training set
// (X [N x 4] FP32 features, normalised LLE targets, classes 0..15).  One step is
// captured as a CUDA graph on first use and replayed.
cbf_status cbf_mlp_train(cbf_mlp* m, const float* dX, const float* dYl, const int32_t* dYc, int64_t N,
                         int32_t steps, float lr, int32_t horizon, float wLle, float* hLosses,
                         void* stream)
{
    if (!m || !dX || !dYl || !dYc || N < 1 || steps < 0)
        return report_error(CBF_ERR_INVALID_ARG, "bad training arguments");
    cudaStream_t s = (cudaStream_t)stream;
    if (!s) return report_error(CBF_ERR_INVALID_ARG, "training needs a non-default stream");
    const int B = m->B;
    cudaError_t e = cudaSuccess;
    if (!m->exec || m->gX != dX || m->gN != N || m->gLr != lr || m->gHorizon != horizon ||
        m->gW != wLle || m->gSeed != m->seed || m->gScale != m->encScale) {
        if (m->exec) cudaGraphExecDestroy(m->exec);
        if (m->graph) cudaGraphDestroy(m->graph);
        m->exec = nullptr;
        m->graph = nullptr;
        e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) return report_cuda_error(e, "begin capture of the training step");
        cudaError_t ce = launch1d(B, s, [&](unsigned b, int t) {
            gather_kernel<<<b, t, 0, s>>>(dX, dYl, (const int*)dYc, N, B, m->step, m->seed, m->encScale,
                                          m->xb, m->xT, m->Ba, m->yl, m->yc);
        });
        const int rows = (B + kGtM - 1) / kGtM * kGtM;
        if (ce == cudaSuccess) ce = forward(*m, B, train_bufs(*m), s);
        if (ce == cudaSuccess)
            ce = launch1d(rows, s, [&](unsigned b, int t) {
                loss_kernel<<<b, t, 0, s>>>(m->out, m->yl, m->yc, B, rows, wLle, m->dOut, m->dOutB, m->dOutT,
                                            m->Ba, m->loss);
            });
        if (ce == cudaSuccess) ce = backward(*m, B, s, m->side);
        if (ce == cudaSuccess)
            ce = launch1d(kNumParams, s, [&](unsigned b, int t) {
                adam_kernel<<<b, t, 0, s>>>(m->params, m->grads, m->m1, m->m2, m->pb, m->tw, kNumParams, lr,
                                            horizon, 0.9f, 0.999f, 1e-8f, m->step);
            });
        if (ce == cudaSuccess) {
            bump_kernel<<<1, 1, 0, s>>>(m->step);
            note_launch();
            ce = cudaGetLastError();
        }
        cudaGraph_t gph = nullptr;
        e = cudaStreamEndCapture(s, &gph);
        if (ce != cudaSuccess) {
            if (gph) cudaGraphDestroy(gph);
            return report_cuda_error(ce, "capture of the training step");
        }
        if (e != cudaSuccess) return report_cuda_error(e, "end capture of the training step");
        m->graph = gph;
        e = cudaGraphInstantiate(&m->exec, gph, 0);
        if (e != cudaSuccess) return report_cuda_error(e, "instantiate the training graph");
        m->gX = dX;
        m->gN = N;
        m->gLr = lr;
        m->gHorizon = horizon;
        m->gW = wLle;
        m->gScale = m->encScale;
        m->gSeed = m->seed;
    }
    for (int i = 0; i < steps && e == cudaSuccess; ++i) {
        if (hLosses) e = cudaMemsetAsync(m->loss, 0, sizeof(float), s);
        if (e == cudaSuccess) e = cudaGraphLaunch(m->exec, s);
        note_launch();
        if (e == cudaSuccess && hLosses)
            e = cudaMemcpyAsync(&hLosses[i], m->loss, sizeof(float), cudaMemcpyDeviceToHost, s);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e == cudaSuccess) e = gemm_status(*m);
    if (e != cudaSuccess) return report_cuda_error(e, "training");
    return CBF_OK;
}

// Predictions for N feature rows (device X [N x 4] FP32): LLE (de-normalised
// with lleMean/lleStd), class, softmax confidence.  Runs in chunks of kPredRows
// rows through its own workspace, then waits for the stream to read the
// products' error flag.
cbf_status cbf_mlp_predict(cbf_mlp* m, const float* dX, int64_t N, float lleMean, float lleStd,
                           float* dLle, int32_t* dCls, float* dConf, void* stream)
{
    if (!m || !dX || N < 0) return report_error(CBF_ERR_INVALID_ARG, "bad prediction arguments");
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e = cudaSuccess;
    if ((e = pred_workspace(m)) != cudaSuccess) return report_cuda_error(e, "prediction workspace");
    for (long long r0 = 0; r0 < N && e == cudaSuccess; r0 += kPredRows) {
        const int n = (int)((N - r0) < kPredRows ? (N - r0) : kPredRows);
        e = launch1d(n, s, [&](unsigned b, int t) {
            encode_rows_kernel<<<b, t, 0, s>>>(dX + r0 * kRaw, n, n, m->encScale, m->pxb, nullptr, 0);
        });
        if (e == cudaSuccess) e = forward(*m, n, pred_bufs(*m), s);
        if (e == cudaSuccess)
            e = launch1d(n, s, [&](unsigned b, int t) {
                head_kernel<<<b, t, 0, s>>>(m->pout, n, lleMean, lleStd, dLle ? dLle + r0 : nullptr,
                                            dCls ? (int*)dCls + r0 : nullptr, dConf ? dConf + r0 : nullptr);
            });
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e == cudaSuccess) e = gemm_status(*m);
    if (e != cudaSuccess) return report_cuda_error(e, "prediction");
    return CBF_OK;
}

cbf_status cbf_mlp_predict_grid(cbf_mlp* m, const cbf_job* job, float lleMean, float lleStd, double* dLle,
                                int32_t* dCls, float* dConf, void* stream)
{
    if (!m || !job || !dLle || !dCls || !dConf) return report_error(CBF_ERR_INVALID_ARG, "bad prediction arguments");
    cbf::DevJob d;
    cbf_status st = cbf::lower_job_for(job, &d);
    if (st != CBF_OK) return st;
    if (d.dims != 2 || d.nIC != 3) return report_error(CBF_ERR_INVALID_ARG, "grid prediction needs a 2-D sweep of a 3-D system");
    const long long n = (long long)d.nPts * d.nPts;
    cudaError_t e = cbf::mlp_predict_grid(m, cbf::feature_spec(d), n, lleMean, lleStd, dLle, (int*)dCls, dConf,
                                          (cudaStream_t)stream);
    if (e != cudaSuccess) return report_cuda_error(e, "grid prediction");
    return CBF_OK;
}

cbf_status cbf_mlp_grid_features(const cbf_job* job, const int64_t* dIdx, int64_t n, float* dX, void* stream)
{
    if (!job || n < 0 || (n > 0 && (!dIdx || !dX))) return report_error(CBF_ERR_INVALID_ARG, "bad feature arguments");
    cbf::DevJob d;
    cbf_status st = cbf::lower_job_for(job, &d);
    if (st != CBF_OK) return st;
    cudaError_t e = cbf::mlp_features(cbf::feature_spec(d), (const long long*)dIdx, n, dX, (cudaStream_t)stream);
    if (e != cudaSuccess) return report_cuda_error(e, "grid features");
    return CBF_OK;
}

}  // extern "C"

namespace cbf {

FeatureSpec feature_spec(const DevJob& J)
{
    FeatureSpec f;
    memset(&f, 0, sizeof(f));
    f.J = J;
    f.sys = J.system == CBF_SYS_ROSSLER ? -1.0f : (J.system == CBF_SYS_LORENZ ? 0.0f : 1.0f);
    f.lo0 = (float)J.ranges[0];
    f.inv0 = J.ranges[1] != J.ranges[0] ? (float)(2.0 / (J.ranges[1] - J.ranges[0])) : 0.0f;
    f.lo1 = (float)J.ranges[2];
    f.inv1 = J.ranges[3] != J.ranges[2] ? (float)(2.0 / (J.ranges[3] - J.ranges[2])) : 0.0f;
    int third = 1;
    while (third == J.idxMut0 || third == J.idxMut1) ++third;
    f.third = third < 4 ? (float)(J.values[third] * 0.1) : 0.0f;
    return f;
}

cudaError_t mlp_features(const FeatureSpec& f, const long long* idx, long long n, float* X, cudaStream_t s)
{
    return launch1d(n, s, [&](unsigned b, int t) { features_kernel<<<b, t, 0, s>>>(f, idx, n, X); });
}

// One fused tcgen05 kernel over the whole grid (mlp_tc.cuh), after packing the
// current BF16 weights into the operand layout.  A wait that ran out inside
// the kernel is reported as cudaErrorLaunchTimeout.
cudaError_t mlp_predict_grid(cbf_mlp* m, const FeatureSpec& f, long long nPoints, float lleMean,
                             float lleStd, double* lle, int* cls, float* conf, cudaStream_t s)
{
    if (nPoints <= 0) return cudaSuccess;
    cudaError_t e = cudaSuccess;
    if (!m->wpack) e = cudaMalloc((void**)&m->wpack, kTcPackBytes);
    if (e == cudaSuccess && !m->tcErr) e = cudaMalloc((void**)&m->tcErr, sizeof(int));
    if (e != cudaSuccess) return e;
    e = launch1d(kTcPackBytes / 2, s,
                 [&](unsigned b, int t) { tc_pack_kernel<<<b, t, 0, s>>>(m->pb, (bf16*)m->wpack); });
    if (e == cudaSuccess) e = cudaMemsetAsync(m->tcErr, 0, sizeof(int), s);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(mlp_predict_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTcSmem);
    int dev = 0, sms = 0;
    if (e == cudaSuccess) e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    const long long tiles = (nPoints + kTcM - 1) / kTcM;
    const unsigned grid = (unsigned)(tiles < sms ? tiles : sms);
    mlp_predict_tc_kernel<<<grid, kTcThreads, kTcSmem, s>>>(f, nPoints, m->encScale, m->wpack, m->params, lleMean,
                                                            lleStd, lle, cls, conf, m->tcErr);
    note_launch();
    e = cudaGetLastError();
    int h = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h, m->tcErr, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e == cudaSuccess && h) e = cudaErrorLaunchTimeout;
    return e;
}

cudaError_t mlp_reset(cbf_mlp* m, unsigned long long seed)
{
    std::vector<float> p;
    init_params(p, seed);
    m->seed = seed;
    cudaError_t e = cudaMemset(m->m1, 0, kNumParams * sizeof(float));
    if (e == cudaSuccess) e = cudaMemset(m->m2, 0, kNumParams * sizeof(float));
    if (e == cudaSuccess) e = cudaMemset(m->step, 0, sizeof(unsigned long long));
    if (e == cudaSuccess && upload_params(m, p.data()) != CBF_OK) e = cudaErrorUnknown;
    return e;
}

}  // namespace cbf
